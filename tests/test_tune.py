"""The launch-shape autotuner's table (no GPU): text round trip, later entries replace earlier ones,
malformed lines and modes are refused."""
import ctypes as C

from warpstore_b200 import ops


def table() -> str:
    need = C.c_size_t()
    ops.lib().ws_tune_table(None, 0, C.byref(need))
    buf = C.create_string_buffer(need.value)
    assert ops.lib().ws_tune_table(buf, need.value, C.byref(need)) == 0
    return buf.value.decode()


def test_table_round_trip():
    lib = ops.lib()
    assert lib.ws_tune_clear() == 0
    assert table() == ""
    text = ("hash:q0123456789abcdef:t10 0 32 -1 0 812.5\ndense_priv:qfedcba9876543210:t16 1 0 3 0 850.0\n"
            "join:b22:p25 0 0 -1 3 1520.0\n")
    assert lib.ws_tune_load(text.encode()) == 0
    assert sorted(table().splitlines()) == sorted(text.splitlines())
    assert lib.ws_tune_load(b"hash:q0123456789abcdef:t10 2 0 700.0\n") == 0   # a line without stages replaces it
    assert "hash:q0123456789abcdef:t10 2 0 -1 0 700.0" in table().splitlines()
    assert lib.ws_tune_load(b"nokeys:q1:t3 0 0 2 650.0\n") == 0               # nor the join slots
    assert "nokeys:q1:t3 0 0 2 0 650.0" in table().splitlines()
    assert len(table().splitlines()) == 4
    assert lib.ws_tune_load(b"join:b1:p1 0 0 -1 1 1.0\n") == 1210             # 1 slot per key
    assert lib.ws_tune_load(b"not a line\n") == 1210
    assert lib.ws_tune_load(b"hash:x:t1 999 0 1.0\n") == 1210                 # CTAs per SM out of range
    assert lib.ws_tune_load(b"nokeys:x:t1 1 0 7 1.0\n") == 1210               # 7 tile stages
    assert lib.ws_tune_load(b"nokeys:x:t1 1 0 0 0 1.0 9\n") == 1210           # a field too many
    assert lib.ws_tune_set_mode(7) == 1210
    assert lib.ws_tune_set_mode(0) == 0
    assert lib.ws_tune_clear() == 0
