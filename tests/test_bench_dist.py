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
    # flops per stencil counted on the oracle (profiles/narrow_flops_per_stencil.txt)
    # x stencils / time, against 148 SMs x 64 FP64 lanes x 2 flops x 1965 MHz
    import bench
    per = bench.per_unit_figures()
    assert per["narrow_flops_per_vf"] > 0 and per["narrow_flops_per_ee"] > 0
    assert per["walk_bytes_per_leaf_pair"] > 0
    c = {"vf": 1_000_000, "ee": 2_000_000}
    r = bench.fp64_roofline(c, 1.0, per)
    want = (per["narrow_flops_per_vf"] * 1e6 + per["narrow_flops_per_ee"] * 2e6) / 1e-3 / 1e12
    assert abs(r["achieved"] - want) < 1e-9 and r["unit"] == "TFLOP/s"
    assert abs(r["peak"] - 37.22) < 0.01 and abs(r["frac"] - want / r["peak"]) < 1e-12
    assert bench.fp64_roofline(c, 0.0, per) is None and bench.fp64_roofline(c, 1.0, {}) is None
    # with the FP64 FMA rate measured in the run, that is the denominator
    m = bench.fp64_roofline(c, 1.0, per, measured_tflops=34.0)
    assert m["peak"] == 34.0 and abs(m["frac"] - want / 34.0) < 1e-12 and m["peak_source"].startswith("measured")
    assert abs(m["frac_of_nominal"] - r["frac"]) < 1e-12


def test_committed_flops_match_the_oracle_count():
    # the frozen figures are what oracle/count_flops.py reports for the strip
    # of the benchmark cloth (checked on a smaller strip of the same cloth,
    # whose per-stencil counts agree within a few percent)
    import bench
    from mclccd_b200 import scenes
    from oracle.count_flops import count
    per = bench.per_unit_figures()
    kinds, _ = count(*scenes.wavy_cloth(1025, seed=0, rows=65))
    for k in ("vf", "ee"):
        got = kinds[k]["necessary_flops"] / kinds[k]["stencils"]
        assert abs(got - per[f"narrow_flops_per_{k}"]) < 0.05 * per[f"narrow_flops_per_{k}"], (k, got)


def test_algorithmic_bytes_forms():
    import bench
    c = {"leaf_pairs": 10, "vf": 20, "ee": 30, "discrete": 2, "hits": 25}
    lists = bench.algorithmic_bytes(c, 100)
    fused = bench.algorithmic_bytes(c, 100, fused=True)
    assert fused["expand"] == 0 and fused["walk"] == lists["walk"] and fused["refit"] == lists["refit"]
    # the fused form neither writes nor reads the 16 B stencil records
    assert fused["narrow"] == lists["expand"] + lists["narrow"] - 2 * 16 * (c["vf"] + c["ee"])


def test_reference_arm_line_on_a_small_cloth():
    # the reference arm's JSON line (the reference's own code on the host's
    # cores, same metric, unit and direction as the device arm): a 65 x 65
    # cloth keeps it to seconds
    import json
    import subprocess
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libmclccd_ref.so")):
        import pytest
        pytest.skip("reference oracle not built")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--n", "65",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, check=True,
                         cwd=ROOT).stdout
    line = json.loads([x for x in out.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "stencils/s" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1 and line["value"] > 0
    assert line["config"]["tris"] == 2 * 64 * 64 and line["config"]["stencils_per_step"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == line["value"] and cb["sample"]
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
