"""The multi-rank path of bench.py on CPU: two gloo ranks, the whole-job
aggregation (max time over ranks, summed work) and the reference arm, which
only rank 0 runs."""
import os
import socket
import sys

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t, w = bench.aggregate(dist, "cpu", total_s=1.0 + rank, work=10 * (rank + 1))
        # the reference arm: ranks other than 0 exit at once with status 0
        rc = bench.run_reference(bench.parse([]), rank, world) if rank else 0
        out[rank] = (t, w, rc)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_and_reference_arm():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][:2] == (2.0, 30.0) and res[1][:2] == (2.0, 30.0)
    assert res[1][2] == 0


def test_single_rank_aggregate_is_local():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(None, "cpu", 3.5, 7) == (3.5, 7.0)
