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


def test_fp64_roofline_of_the_narrow_phase():
    # flops per stencil from the committed ncu summary x stencils / time,
    # against 148 SMs x 64 FP64 lanes x 2 flops x 1965 MHz
    import bench
    per = bench.per_unit_figures()
    assert per["narrow_fp64_flops_per_vf"] > 0 and per["narrow_fp64_flops_per_ee"] > 0
    assert per["walk_bytes_per_leaf_pair"] > 0
    c = {"vf": 1_000_000, "ee": 2_000_000}
    r = bench.fp64_roofline(c, 1.0, per)
    want = (per["narrow_fp64_flops_per_vf"] * 1e6 + per["narrow_fp64_flops_per_ee"] * 2e6) / 1e-3 / 1e12
    assert abs(r["achieved"] - want) < 1e-9 and r["unit"] == "TFLOP/s"
    assert abs(r["peak"] - 37.22) < 0.01 and abs(r["frac"] - want / r["peak"]) < 1e-12
    assert bench.fp64_roofline(c, 0.0, per) is None and bench.fp64_roofline(c, 1.0, {}) is None
