"""ws_encode_column_engine: the engine's segment encoding (Table::encodeColumn, src/storage.cu:1093-1192)
on the device — frame of reference (enc 1/2/3), double dictionary (enc 4), decimal doubles (enc 5/6),
raw otherwise — byte for byte against the oracle's restatement, and decoded back through the scans'
encoded gather (ws_gather_enc) to the original values."""
import zlib

import numpy as np
import pytest

from oracle import oracle
from warpstore_b200 import abi, ops

pytestmark = pytest.mark.gpu

N = 1 << 16


def case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "i32_u8":
        x = rng.integers(-100, 150, N).astype(np.int32)
        x[rng.choice(N, 99, replace=False)] = abi.NULL_I32
        return x, abi.PT_I32, 1
    if name == "i32_u16":
        return rng.integers(10**6, 10**6 + 60000, N).astype(np.int32), abi.PT_I32, 2
    if name == "i32_wide":  # no uint32 form for INT columns
        return rng.integers(-2**30, 2**30, N).astype(np.int32), abi.PT_I32, 0
    if name == "i64_u32":
        x = rng.integers(-2**40, -2**40 + 2**32 - 5, N).astype(np.int64)
        x[:7] = abi.NULL_I64
        return x, abi.PT_I64, 3
    if name == "i64_wide":
        return rng.integers(-2**60, 2**60, N).astype(np.int64), abi.PT_I64, 0
    if name == "i64_all_null":
        return np.full(N, abi.NULL_I64, np.int64), abi.PT_I64, 1
    if name == "short":
        return rng.integers(0, 10, 1000).astype(np.int64), abi.PT_I64, 0
    if name == "f64_dict":
        vals = np.concatenate([rng.random(250) * 100, [0.0, -0.0, np.nan, 1e300, -7.5]])
        return rng.choice(vals, N), abi.PT_F64, 4
    if name == "f64_cents":
        x = np.round(rng.integers(0, 50_000, N) * 0.01, 2)
        x[rng.choice(N, 50, replace=False)] = np.nan
        return x, abi.PT_F64, 5
    if name == "f64_prices":
        return np.round(rng.random(N) * 90_000, 2), abi.PT_F64, 6
    if name == "f64_random":
        return rng.random(N), abi.PT_F64, 0
    if name == "f64_scale4_too_wide":  # exact at scale 4, but the offsets need more than 32 bits
        return np.round(rng.random(N) * 10**6, 4), abi.PT_F64, 0
    raise ValueError(name)


@pytest.mark.parametrize("name", ["i32_u8", "i32_u16", "i32_wide", "i64_u32", "i64_wide", "i64_all_null", "short",
                                  "f64_dict", "f64_cents", "f64_prices", "f64_random", "f64_scale4_too_wide"])
def test_engine_encoding_matches_oracle_and_decodes(name):
    x, pt, want_enc = case(name)
    oe, ob = oracle.encode_column_engine(x, pt)
    assert oe == want_enc, f"oracle chose enc {oe}"
    d = ops.DeviceBuffer.from_array(x)
    ptr, nbytes, enc = ops.encode_column_engine(d.ptr, pt, x.size)
    assert enc == oe
    if not enc:
        assert ptr is None and nbytes == 0
        return
    got = ops.device_to_array(ptr, np.uint8, nbytes)
    assert nbytes == ob.size and np.array_equal(got, ob), "encoded bytes differ from the oracle's"
    # decode every row through the encoded gather of the scans
    t = {abi.PT_I32: abi.T_I32N, abi.PT_I64: abi.T_I64N, abi.PT_F64: abi.T_F64}[pt]
    idx = ops.DeviceBuffer.from_array(np.arange(x.size, dtype=np.int32))
    out = ops.DeviceBuffer(x.nbytes)
    ops.gather_enc(abi.ColView(ptr, t, 0, enc, 0), pt, idx.ptr, x.size, out.ptr)
    back = out.to_array(x.dtype)
    ops.tmp_free(ptr)
    if pt == abi.PT_F64:
        assert np.array_equal(back.view(np.int64)[~np.isnan(x)], x.view(np.int64)[~np.isnan(x)])
        assert np.isnan(back[np.isnan(x)]).all()
    else:
        assert np.array_equal(back, x)
