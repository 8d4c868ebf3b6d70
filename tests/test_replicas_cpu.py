"""bench.py's multi-GPU form (replicas only: one independent replica of the workload per rank, no
data-path collective) on CPU: two gloo ranks; the job's step time is the max over ranks and the
whole-job rate counts every rank's rows."""
import os
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        local_ms = [1.5, 2.5][rank]  # the second replica is slower
        m = bench.reduce_max(local_ms, ws, device="cpu")
        bench.barrier(ws)
        out[rank] = (m, bench.whole_job_rate(60_000_000, ws, m))
    finally:
        dist.destroy_process_group()


def test_two_replicas_max_time_and_whole_job_rate():
    ws = 2
    port = 29500 + os.getpid() % 1000
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(ws, port, out), nprocs=ws, start_method="spawn", join=True)
        res = dict(out)
    for rank in range(ws):
        m, rate = res[rank]
        assert m == 2.5
        assert abs(rate - 60_000_000 * 2 / 2.5e-3 / 1e9) < 1e-9
