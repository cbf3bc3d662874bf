#!/usr/bin/env python
"""CCD step benchmark (update + traverse + ACCD) on the 2.1M-triangle cloth.

Workload: 1025 x 1025 wavy cloth (2,097,152 triangles, float64 V, int32 F,
thickness 1e-4), seeded synthetic data.  One step = BVHTree::update(V0, V1,
F) + traverse(V0, V1, F) through the C ABI; F never changes, so every timed
step takes the refit-only path, and V1 alternates between two seeded draws.
The first (full LBVH build) update is timed separately.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0).  value = candidate stencils / second of the
whole job with inputs resident in HBM; e2e = the same through the C ABI from
pinned host buffers, host<->device copies of inputs and of every hit and
discrete pair inside the timed region.  --impl reference times the
reference's own CPU code (the oracle build of the unmodified reference
sources) on the host cores, on the same full cloth and the same step
(second update with the same F, then traverse), K timed steps after W.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "CCD step ms & stencils/s at 2.1M tris: FP32-certified vs FP64 GPU vs TBB"
UNIT = "stencils/s"


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=1025, help="cloth grid side")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32cert"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the certified/adjoint/batch form measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the 512-scene batch measurement")
    ap.add_argument("--tune", default="", help="launch knobs, e.g. walk_packet=0,accd_grid=2368")
    ap.add_argument("--batch-only", action="store_true", help="only the batching form (prints its JSON object)")
    ap.add_argument("--batch-scenes", default="384,128", help="batching form: 3D cloths,2D annuli")
    ap.add_argument("--batch-tune", default="", help="batching form: fixed knobs instead of the autotuner, "
                                                     "e.g. form=0,wave=4096")
    return ap.parse_args(argv)


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        """Starts the sampler and returns once it is producing samples, so the
        region that follows is covered from its first millisecond."""
        self.n0 = 0
        try:
            # line-buffered, so a sample reaches the file when it is taken
            pre = ["stdbuf", "-oL"] if shutil.which("stdbuf") else []
            self.p = subprocess.Popen(pre + ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                             "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.p.poll() is None:
            with open(self.f.name) as fh:
                n = sum(1 for _ in fh)
            if n >= 1:
                self.n0 = n
                return
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for k, line in enumerate(fh):
                parts = [x.strip() for x in line.split(",")]
                if k >= self.n0 - 1 and len(parts) >= 9:   # from the last sample before the region on
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# Algorithmic work per unit (the frozen per-unit formulas of the roofline).
#   walk   : per query leaf its FP64 box (96 B) + prim id (4) + active (1), the
#            n-1 internal nodes once (64 B), and per leaf pair found the
#            candidate leaf box (96 B) + its prim id (4) + the pair write (8).
#   expand : per leaf pair 8 B read + 2 x (12 B face + 1 B flags) + 16 B per
#            stencil written + 8 B per discrete pair, + the tri-tri gather of
#            6 V1 vertices (144 B) per pair.
#   narrow : per stencil 16 B read + 2 x 4 x 24 B vertex gather (192 B), plus
#            25 B per hit written (int4 stencil, f64 toi, u8 kind).
#   fused  : (expansion, discrete test and ACCD in one kernel, no stencil
#            lists) per leaf pair 8 + 26 + 144 B, 8 B per discrete pair, per
#            stencil the 192 B vertex gather, 25 B per hit.
#   refit  : per leaf 12 B face + 6 x 24 B vertex reads, 96 B FP64 box + 1 B
#            active written, 32 B of node slot written, 64 B per internal node read.
def algorithmic_bytes(c, n, fused=False):
    walk = n * (96 + 4 + 1) + (n - 1) * 64 + c["leaf_pairs"] * (96 + 4 + 8)
    refit = n * (12 + 144 + 96 + 1 + 32) + (n - 1) * 64
    if fused:
        narrow = c["leaf_pairs"] * (8 + 26 + 144) + 8 * c["discrete"] + (c["vf"] + c["ee"]) * 192 + 25 * c["hits"]
        return {"walk": walk, "expand": 0, "narrow": narrow, "refit": refit}
    expand = c["leaf_pairs"] * (8 + 26 + 144) + 16 * (c["vf"] + c["ee"]) + 8 * c["discrete"]
    narrow = (c["vf"] + c["ee"]) * (16 + 192) + 25 * c["hits"]
    return {"walk": walk, "expand": expand, "narrow": narrow, "refit": refit}


def per_unit_figures():
    """The committed per-unit figures: DRAM bytes per unit of each stage from
    the ncu summary (profiles/dram_traffic_per_unit.txt) and FP64 flops per
    VF / EE stencil of the narrow phase counted on the oracle
    (profiles/narrow_flops_per_stencil.txt, oracle/count_flops.py)."""
    per = {}
    for name in ("dram_traffic_per_unit.txt", "narrow_flops_per_stencil.txt"):
        try:
            with open(os.path.join(ROOT, "profiles", name)) as f:
                for line in f:
                    parts = line.split()
                    if len(parts) == 2 and not line.startswith("#"):
                        per[parts[0]] = float(parts[1])
        except OSError:
            pass
    return per


# FP64 peak of a B200: 148 SMs x 64 FP64 FMA lanes x 2 flops at the 1965 MHz
# maximum SM clock (no measured FP64 figure is available to divide by).
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def fp64_roofline(c, narrow_ms, per=None, measured_tflops=None):
    """FP64 roofline of the narrow phase: the flops per VF and EE stencil
    counted on the oracle (the necessary work: add, multiply, divide and
    square root one flop each) times this run's stencils, over the narrow
    stage's time.  The peak is the FP64 FMA rate measured in this run
    (mclccd_fp64_fma_rate) when given, else the nominal figure."""
    per = per_unit_figures() if per is None else per
    if "narrow_flops_per_vf" not in per or not narrow_ms or narrow_ms <= 0:
        return None
    flops = per["narrow_flops_per_vf"] * c["vf"] + per.get("narrow_flops_per_ee", 0.0) * c["ee"]
    achieved = flops / (narrow_ms / 1e3) / 1e12
    if measured_tflops:
        peak, src = measured_tflops, ("measured in this run: FP64 FMA throughput of this GPU "
                                      "(mclccd_fp64_fma_rate, 8 independent FMA chains per thread)")
    else:
        peak, src = FP64_PEAK_TFLOPS, "nominal: 148 SMs x 64 FP64 FMA lanes x 2 flops x 1965 MHz"
    return {"achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "flops": flops,
            "peak_source": src, "peak_nominal": FP64_PEAK_TFLOPS, "frac_of_nominal": achieved / FP64_PEAK_TFLOPS,
            "flops_source": "oracle/count_flops.py: necessary FP64 operations per stencil, per kind "
                            "(profiles/narrow_flops_per_stencil.txt)"}


def measured_traffic(c, fused=False):
    """DRAM bytes per stage of one step from the per-unit figures of the
    committed ncu summary, scaled by this run's unit counts."""
    per = per_unit_figures()
    if not per:
        return {}
    out = {}
    sten = c["vf"] + c["ee"]
    if "walk_bytes_per_leaf_pair" in per:
        out["walk"] = per["walk_bytes_per_leaf_pair"] * c["leaf_pairs"]
    if fused:
        if "fused_bytes_per_stencil" in per:
            out["narrow"] = per["fused_bytes_per_stencil"] * sten
        return out
    if "expand_bytes_per_stencil" in per:
        out["expand"] = per["expand_bytes_per_stencil"] * sten
    if "narrow_bytes_per_stencil" in per:
        out["narrow"] = per["narrow_bytes_per_stencil"] * sten
    return out


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def aggregate(dist, device, total_s, work):
    """Whole-job figures over the ranks: the slowest rank's time and the
    summed work (every rank takes the same two collective steps)."""
    if dist is None:
        return total_s, float(work)
    import torch
    t = torch.tensor([total_s, float(work)], dtype=torch.float64, device=device)
    tmax = t.clone()
    dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
    tsum = t.clone()
    dist.all_reduce(tsum, op=dist.ReduceOp.SUM)
    return float(tmax[0]), float(tsum[1])


def run_reference(args, rank, world):
    """The reference arm: the reference's own CPU implementation (the oracle
    build of the unmodified reference sources, all host threads) on the same
    workload and step as the device arm -- the 1025 x 1025 wavy cloth, one
    first update (full build) untimed, then per step update(V0, V1, F) with
    V1 alternating between the two seeded draws (the reference rebuilds its
    Kd-tree on every update) and traverse with the default ACCD; hooks are
    no-op counters.  K steps are timed after W; rank 0 only."""
    if rank != 0:
        return 0
    from mclccd_b200 import scenes
    from oracle.ref import REF_SO, Port, Reference
    V0, V1a, F, eta = scenes.wavy_cloth(args.n, seed=0)
    V1b = scenes.wavy_redraw(V0, 1)
    if os.path.exists(REF_SO):
        R, kind = Reference(), "reference"
        cores = R.L.ref_threads()
        r = R.time_steps(V0, V1a, V1b, F, eta, args.warmup + args.steps)
        ms_all, sten_all = r["ms"], r["stencils"]
    else:   # the oracle restatement, single-threaded, one step at a time
        R, kind, cores = None, "port", 1
        ms_all, sten_all = [], []
        for it in range(args.warmup + args.steps):
            V1 = V1b if it % 2 == 0 else V1a
            t0 = time.perf_counter()
            p = Port().run(V0, V1, F, eta)
            ms_all.append((time.perf_counter() - t0) * 1e3)
            sten_all.append(len(p["cand_sten"]))
    times = ms_all[args.warmup:]
    sten = sten_all[args.warmup:]
    ms = float(np.mean(times))
    val = float(np.sum(sten)) / (np.sum(times) / 1e3)
    sample = (f"the full workload, {args.steps} timed steps after {args.warmup}: second update (same F, V1 "
              f"alternating two draws) + traverse with the default ACCD, {len(F)} tris, "
              f"{int(np.mean(sten))} stencils per step")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"wavy cloth {args.n}x{args.n} ({len(F)} tris), thickness 1e-4, refit-only "
                                   "update + traverse + ACCD per step (F unchanged, V1 alternates two seeded draws)",
                       "tris": int(len(F)), "stencils_per_step": int(np.mean(sten)),
                       "step_ms_all": [float(x) for x in times]},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(V0, V1a, V1b, F, eta, n_sten):
    from oracle.ref import REF_SO, Reference
    if not os.path.exists(REF_SO):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": "reference build missing"}
    R = Reference()
    r = R.time(V0, V1a, F, eta, V1b=V1b)
    ms = r["ms_update_again"] + r["ms_traverse"]
    return {"value": n_sten / (ms / 1e3), "unit": UNIT, "cores": r["threads"], "kind": "reference",
            "sample": (f"one full step of the same workload ({len(F)} tris): second update (same F) "
                       f"{r['ms_update_again']:.0f} ms + traverse {r['ms_traverse']:.0f} ms; first update "
                       f"{r['ms_update_first']:.0f} ms"),
            "ms_per_step": ms}


def run_b200(args, rank, world, local):
    import torch
    from mclccd_b200 import MEM_HOST, PREC_FP32_CERTIFIED, PREC_FP64, BVHTree, scenes
    torch.cuda.set_device(local)
    if args.batch_only:
        if rank == 0:
            print(json.dumps(measure_batch(args)), flush=True)
        return 0
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    V0, V1a, F, eta = scenes.wavy_cloth(args.n, seed=0)
    V1b = scenes.wavy_redraw(V0, 1)
    n = len(F)
    dev = torch.device("cuda", local)
    dV0, dV1a, dV1b, dF = (torch.from_numpy(a).to(dev) for a in (V0, V1a, V1b, F))
    stream = torch.cuda.current_stream()
    prec = PREC_FP32_CERTIFIED if args.precision == "fp32cert" else PREC_FP64
    tree = BVHTree(3, precision=prec)
    tree.options.box_eta = tree.options.vf_ccd_eta = tree.options.ee_ccd_eta = eta
    tree.options.profile = True
    if args.tune:
        tree.set_tuning(**{k: int(v) for k, v in (kv.split("=") for kv in args.tune.split(","))})
    tree.set_stream(stream.cuda_stream)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    # first update: full build (representative flags, Morton, sort, hierarchy,
    # refit).  A tiny build first loads the kernels' code, so the timing below
    # is the build itself, not lazy module loading.
    warm = BVHTree(3)
    wV0, wV1, wF, _ = scenes.folded_cloth(8)
    warm.update(wV0, wV1, wF)
    warm.traverse()
    del warm
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    e0.record(stream)
    tree.update(dV0, dV1a, dF)
    e1.record(stream)
    torch.cuda.synchronize()
    first_ms = e0.elapsed_time(e1)
    tree.traverse()
    V1s = [dV1b, dV1a]
    for i in range(args.warmup):
        tree.update(dV0, V1s[i % 2], dF)
        tree.traverse()
    clocks = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = tree.kernel_launches()
    step_ms, sten, stages = [], 0, []
    clocks.start()
    for i in range(args.steps):
        flush.zero_()                        # evict L2 between timed steps (outside the events)
        s0, s1 = ev(), ev()
        s0.record(stream)
        tree.update(dV0, V1s[i % 2], dF)
        tree.traverse()
        s1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(s0.elapsed_time(s1))
        c = tree.counts()
        sten += c["vf"] + c["ee"]
        stages.append(tree.stage_ms())
    clk = clocks.stop()
    launches = tree.kernel_launches() - launches0
    total_s = sum(step_ms) / 1e3
    total_max, sten_all = aggregate(dist, dev, total_s, sten)
    value = sten_all / total_max
    c = tree.counts()
    pstats = tree.precision_stats()
    stage = {k: float(np.median([s[k] for s in stages])) for k in stages[0]}

    # roofline of the dominant kernel.  The narrow phase is bound by the FP64
    # pipe: flops counted on the oracle / its device time against the FP64
    # peak; the other stages by memory: algorithmic bytes / time.
    tuning = tree.get_tuning()
    fused = prec == PREC_FP64 and tuning["narrow_fused"] == 1 and tuning["accd_rebin"] == 0
    ab = algorithmic_bytes(c, n, fused)
    kt = {"walk": stage["walk"], "expand": stage["expand"], "narrow": stage["narrow"], "refit": stage["refit"]}
    top = max(kt, key=kt.get)
    peak, src = measured_peaks()
    tr = measured_traffic(c, fused)
    try:
        from mclccd_b200.ccd import fp64_fma_rate
        fp64_measured = fp64_fma_rate(dev.index or 0)
    except Exception:
        fp64_measured = None
    fp = fp64_roofline(c, kt["narrow"], measured_tflops=fp64_measured)
    hbm = {k: {"ms": kt[k], "algorithmic_bytes": ab[k],
               "GB/s": ab[k] / (kt[k] / 1e3) / 1e9 if kt[k] > 0 else None,
               "frac": ab[k] / (kt[k] / 1e3) / 1e9 / peak if kt[k] > 0 else None,
               "traffic": tr.get(k)} for k in kt}
    if top == "narrow" and fp is not None:
        roof = {"bound": "fp64", "kernel": top, "achieved": fp["achieved"], "peak": fp["peak"], "unit": "TFLOP/s",
                "frac": fp["frac"], "traffic": tr.get(top), "peak_source": fp["peak_source"], "flops": fp["flops"],
                "flops_source": fp["flops_source"], "kernel_ms": kt[top]}
    else:
        roof = {"bound": "hbm", "kernel": top, "achieved": hbm[top]["GB/s"], "peak": peak, "unit": "GB/s",
                "frac": hbm[top]["frac"], "traffic": tr.get(top), "peak_source": src,
                "algorithmic_bytes": ab[top], "kernel_ms": kt[top]}
    roof.update({
        "narrow_form": "fused (expansion + discrete test + ACCD in one kernel)" if fused else "stencil lists",
        "traffic_source": "ncu dram bytes per unit (profiles/dram_traffic_per_unit.txt) x this run's units",
        "hbm_peak_gbs": peak, "hbm_peak_source": src, "stages_hbm": hbm, "narrow_fp64": fp})

    # end to end through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        pin = lambda a: torch.from_numpy(a).pin_memory()
        hV0, hV1a, hV1b, hF = pin(V0), pin(V1a), pin(V1b), pin(F)
        cap = int(c["hits"] * 1.5) + 1024
        hs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
        hv = torch.empty(cap, dtype=torch.uint8).pin_memory()
        ht = torch.empty(cap, dtype=torch.float64).pin_memory()
        hd = torch.empty((max(1024, int(c["discrete"] * 1.5)), 2), dtype=torch.int32).pin_memory()
        L = tree._L
        hV1s = [hV1b, hV1a]
        e_ms, h2d, d2h = [], 0, 0
        for i in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s0, s1 = ev(), ev()
            s0.record(stream)
            tree.update(hV0.numpy(), hV1s[i % 2].numpy(), hF.numpy())
            # traverse with the hits and discrete pairs delivered into the
            # page-locked host arrays; their copies overlap the step's compute
            nh, nd = tree.traverse_out(hs, hv, ht, hd)
            s1.record(stream)
            torch.cuda.synchronize()
            wall = (time.perf_counter() - t0) * 1e3
            if i >= args.warmup:
                e_ms.append(max(s0.elapsed_time(s1), wall))
                h2d = V0.nbytes + V1a.nbytes + F.nbytes
                d2h = nh * (16 + 1 + 8) + nd * 8
        e_total, _ = aggregate(dist, dev, sum(e_ms) / 1e3, 0)
        e2e = {"value": sten_all / e_total, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e_total * 1e3 / args.steps}

    dropin = None
    if rank == 0 and world == 1 and not args.no_e2e:
        dropin = measure_dropin(args, V0, V1a, V1b, F, eta, c)

    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        forms = measure_forms(args, tree, stage, dV0, V1s, dF, eta, flush, stream, dev, ev)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(V0, V1a, V1b, F, eta, c["vf"] + c["ee"])

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_max * 1e3 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == PREC_FP64 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": f"wavy cloth {args.n}x{args.n} ({n} tris), thickness 1e-4, refit-only "
                                   "update + traverse + ACCD per step (F unchanged, V1 alternates two seeded draws)",
                       "tris": n, "stencils_per_step": int(c["vf"] + c["ee"]), "vf": int(c["vf"]),
                       "ee": int(c["ee"]), "hits": int(c["hits"]), "discrete": int(c["discrete"]),
                       "leaf_pairs": int(c["leaf_pairs"]), "first_update_ms": first_ms,
                       "fp64_stencils": pstats[0], "toi_bound_hits": pstats[1],
                       "precision": args.precision, "parallelism": f"replicas x{world}",
                       "l2": "flushed between timed steps (512 MB write outside the timed events)",
                       "stage_ms_median": stage, "step_ms_all": step_ms},
            "gpu_launches": int(launches), "roofline": roof, "clocks": clk}
    if e2e is not None:
        line["e2e"] = e2e
    if dropin is not None:
        line["e2e_dropin"] = dropin
    if forms is not None:
        line["forms"] = forms
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)
    return 0


def measure_dropin(args, V0, V1a, V1b, F, eta, c):
    """End to end through the C++ drop-in (tests/cpp/dropin_bench.cpp):
    mcl::BVHTree<double, 3> with append_pair / append_discrete set, the
    reference's update(V0, V1, F, nf, 3) + traverse(V0, V1, F) on host arrays
    per step, hooks called for every hit; wall time per step."""
    exe_dir = tempfile.mkdtemp(prefix="mclccd_dropin_")
    try:
        exe = os.path.join(exe_dir, "dropin_bench")
        subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "dropin_bench.cpp"), "-L", os.path.join(ROOT, "mclccd_b200"),
                        "-lmclccd_b200", "-Wl,-rpath," + os.path.join(ROOT, "mclccd_b200"), "-o", exe], check=True)
        scene = os.path.join(exe_dir, "scene.bin")
        with open(scene, "wb") as f:
            f.write(np.array([len(V0), len(F)], np.int32).tobytes())
            f.write(np.array([eta], np.float64).tobytes())
            for a in (V0, V1a, V1b):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
            f.write(np.ascontiguousarray(F, np.int32).tobytes())
        out = subprocess.run([exe, scene, str(args.warmup), str(args.steps)], check=True, capture_output=True,
                             text=True).stdout
        r = json.loads(out.strip().splitlines()[-1])
    except Exception as e:   # reported, never fatal to the headline line
        return {"error": f"{type(e).__name__}: {e}"}
    finally:
        shutil.rmtree(exe_dir, ignore_errors=True)
    ms = float(np.mean(r["ms"]))
    sten = c["vf"] + c["ee"]
    return {"value": sten / (ms / 1e3), "unit": UNIT, "ms_per_step": ms, "step_ms_all": r["ms"],
            "h2d_bytes_per_step": int(V0.nbytes + V1a.nbytes + F.nbytes),
            "d2h_bytes_per_step": int(r["hits"] * (16 + 1 + 8) + r["discrete"] * 8),
            "hits_delivered": r["hits"], "discrete_delivered": r["discrete"],
            "api": "C++ mcl::BVHTree<double,3>: update(V0,V1,F,nf,3) + traverse(V0,V1,F) on host arrays, "
                   "append_pair / append_discrete called for every result (wall clock); options.threaded on, as "
                   "in the reference, so append_pair runs on all host threads (thread-local counting hook)",
            "host_threads": os.cpu_count()}


def measure_forms(args, tree, stage, dV0, V1s, dF, eta, flush, stream, dev, ev):
    """The other forms, on one GPU: the FP32-certified narrow phase on the
    same workload as the headline (other precision than the headline's), and
    the toi adjoint on the 256 x 256 folded cloth (forward = update +
    traverse + ACCD, backward = the VJP over all hits)."""
    import torch
    from mclccd_b200 import PREC_FP32_CERTIFIED, PREC_FP64, BVHTree, CCDError, scenes
    out = {}

    def timed(fn, k, w):
        for _ in range(w):
            fn()
        ms = []
        for _ in range(k):
            flush.zero_()
            a, b = ev(), ev()
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
        return float(np.median(ms)), ms

    # precision form: the other precision on the headline workload
    other = PREC_FP64 if tree.precision == PREC_FP32_CERTIFIED else PREC_FP32_CERTIFIED
    t2 = BVHTree(3, precision=other)
    t2.options.box_eta = t2.options.vf_ccd_eta = t2.options.ee_ccd_eta = eta
    t2.options.profile = True
    t2.set_stream(stream.cuda_stream)
    t2.update(dV0, V1s[1], dF)
    t2.traverse()
    it = [0]
    stg = []

    def step():
        t2.update(dV0, V1s[it[0] % 2], dF)
        t2.traverse()
        it[0] += 1
        stg.append(t2.stage_ms())

    ms, _ = timed(step, max(3, min(args.steps, 6)), 2)
    narrow2 = float(np.median([s["narrow"] for s in stg[2:]]))
    fp64_narrow, cert_narrow = (stage["narrow"], narrow2) if other == PREC_FP32_CERTIFIED else (narrow2, stage["narrow"])
    ps = t2.precision_stats() if other == PREC_FP32_CERTIFIED else tree.precision_stats()
    c2 = t2.counts()
    out["fp32_certified"] = {
        "workload": "headline workload, other precision than the headline line",
        "ms_per_step_" + ("fp32cert" if other == PREC_FP32_CERTIFIED else "fp64"): ms,
        "narrow_ms_fp64": fp64_narrow, "narrow_ms_fp32cert": cert_narrow,
        "narrow_speedup_fp32cert_vs_fp64": fp64_narrow / cert_narrow,
        "fp64_pass_stencils": ps[0], "toi_bound_hits": ps[1], "hits": int(c2["hits"]),
        "stencils": int(c2["vf"] + c2["ee"])}
    del t2

    try:
        out["certified_c2"] = measure_c2(args, stream, dev, ev)
    except CCDError as e:   # reported, never fatal to the headline line
        out["certified_c2"] = {"error": str(e)}
        torch.cuda.empty_cache()

    # differentiation form: 256 x 256 folded cloth, thickness 1e-3
    V0, V1, F, eta4 = scenes.folded_cloth(256)
    a0, a1, aF = (torch.from_numpy(x).to(dev) for x in (V0, V1, F))
    t3 = BVHTree(3, precision=PREC_FP64)
    t3.options.box_eta = t3.options.vf_ccd_eta = t3.options.ee_ccd_eta = eta4
    t3.set_stream(stream.cuda_stream)

    def fwd():
        t3.update(a0, a1, aF)
        t3.traverse()

    fwd()
    nh = t3.counts()["hits"]
    g = torch.randn(nh, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
    res = {}

    def bwd():
        res["v"] = t3.vjp_toi(g)

    f_ms, _ = timed(fwd, 5, 2)
    b_ms, _ = timed(bwd, 5, 2)
    out["adjoint"] = {"workload": f"folded cloth 256x256 ({len(F)} tris), thickness 1e-3, FP64",
                      "forward_ms": f_ms, "backward_ms": b_ms, "backward_to_forward": b_ms / f_ms,
                      "hits": int(nh), "hits_with_gradient": int(res["v"][2])}
    del t3
    if not args.no_batch:
        out["batch"] = measure_batch(args)
    return out


def measure_c2(args, stream, dev, ev, sample=10_000_000, subdiv=5):
    """Precision form on its own workload: 64 icospheres (radii U[0.05, 0.1],
    centres in the unit cube, per-sphere translation N(0, 0.05) plus
    N(0, 1e-3) per vertex), thickness 1e-3, in FP64 and in the FP32-certified
    form: step and narrow-phase times, hits.  Subdivision 5 (1,310,720 tris)
    is the largest that fits: the translation is 35x the edge length, so the
    swept boxes overlap hundreds of neighbours (subdivision 4: 34M stencils;
    5: 1.24G stencils, 1.08G hits, 72 GB of lists; 6, 5.2M tris, grows
    another 16-34x, past one GPU's memory for the lists and past host memory
    for the hits).  The toi of the certified form against FP64 on the first
    `sample` candidates of the FP64 tree and on the 100k constructed stress
    stencils (near-parallel EE, near-coplanar VF), through the bulk call in
    both precisions: hit/miss agreement, toi never later, relative error."""
    import ctypes
    import torch
    from mclccd_b200 import MEM_DEVICE, PREC_FP32_CERTIFIED, PREC_FP64, BVHTree, narrow_phase_bulk, scenes
    V0, V1, F, eta = scenes.icospheres(64, subdiv, seed=0)
    d0, d1, dF = (torch.from_numpy(x).to(dev) for x in (V0, V1, F))
    out = {"workload": f"64 icospheres, subdivision {subdiv} ({len(F)} tris), thickness 1e-3, seed 0"}
    cs = cv = None
    for name, prec in (("fp64", PREC_FP64), ("fp32cert", PREC_FP32_CERTIFIED)):
        t = BVHTree(3, precision=prec)
        t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
        t.options.profile = True
        t.set_stream(stream.cuda_stream)
        t.update(d0, d1, dF)
        t.traverse()
        ms, nar = [], []
        for _ in range(3):
            a, b = ev(), ev()
            a.record(stream)
            t.update(d0, d1, dF)
            t.traverse()
            b.record(stream)
            torch.cuda.synchronize()
            ms.append(a.elapsed_time(b))
            nar.append(t.stage_ms()["narrow"])
        c = t.counts()
        ps = t.precision_stats()
        out[name] = {"step_ms": float(np.median(ms)), "narrow_ms": float(np.median(nar)), "hits": int(c["hits"]),
                     "stencils": int(c["vf"] + c["ee"]), "leaf_pairs": int(c["leaf_pairs"]),
                     "fp64_pass_stencils": int(ps[0]), "toi_bound_hits": int(ps[1])}
        if prec == PREC_FP64:   # a prefix of the candidate list, on the device
            k = min(sample, int(c["vf"] + c["ee"]))
            cs = torch.empty((k, 4), dtype=torch.int32, device=dev)
            cv = torch.empty(k, dtype=torch.uint8, device=dev)
            t._L.mclccd_get_candidates(t._h, MEM_DEVICE, k, ctypes.c_void_p(cs.data_ptr()),
                                       ctypes.c_void_p(cv.data_ptr()))
        del t
        torch.cuda.empty_cache()
    out["narrow_speedup_fp32cert_vs_fp64"] = out["fp64"]["narrow_ms"] / out["fp32cert"]["narrow_ms"]
    out["same_hit_count"] = out["fp64"]["hits"] == out["fp32cert"]["hits"]

    def compare(a0, a1, s4, kind, e):
        t64, h64 = narrow_phase_bulk(a0, a1, s4, kind, e, precision=PREC_FP64)
        tc, hc, nfb = narrow_phase_bulk(a0, a1, s4, kind, e, precision=PREC_FP32_CERTIFIED, return_fallbacks=True)
        if not torch.is_tensor(t64):
            t64, h64, tc, hc = (torch.from_numpy(x) for x in (t64, h64, tc, hc))
        hit = h64 == 1
        rel = torch.where(hit & (t64 > 0), (t64 - tc) / t64, torch.zeros_like(t64))
        return {"stencils": int(len(h64)), "hits": int(hit.sum()), "hit_miss_identical": bool((h64 == hc).all()),
                "later_than_fp64": int((hit & (tc > t64)).sum()), "max_rel_toi_error": float(rel.abs().max()),
                "exact_toi": int((hit & (tc == t64)).sum()), "fp64_fallbacks": int(nfb)}

    out["sample"] = compare(d0, d1, cs, cv, eta)
    sV0, sV1, ssten, svf, seta = scenes.stress_stencils(100_000)
    out["stress"] = compare(sV0, sV1, ssten, svf, seta)
    return out


def measure_batch(args):
    """Batching form: 512 scenes (384 folded cloths, side log-uniform in
    [16, 384]; 128 2D annuli, ring resolution U[32, 2048]) per run, one CUDA
    graph.  The autotuner picks the form and launch knobs on a 64-scene
    sample (or --batch-tune fixes them); the full batch then runs once to
    capture and warm up and once timed, in FP64 and in the FP32-certified
    form."""
    from mclccd_b200 import PREC_FP32_CERTIFIED, PREC_FP64, scenes
    from mclccd_b200.autotune import tune_batch
    from mclccd_b200.batch import Batch
    n3d, n2d = (int(x) for x in args.batch_scenes.split(","))
    if args.batch_tune:
        best, table = {k: int(v) for k, v in (kv.split("=") for kv in args.batch_tune.split(","))}, []
    else:
        sample = [s for _, s in scenes.batch_scenes(n3d=48, n2d=16, seed=1)]
        tb = Batch()
        tb.set_scenes(sample)
        best, table = tune_batch(tb, space={"form": (0, 1), "block": (128, 256), "stack": (32, 64), "chunk": (1, 4),
                                            "leaf": (1, 2), "wave": (2048, 4096)}, repeats=1)
        del tb, sample
    full = [s for _, s in scenes.batch_scenes(n3d=n3d, n2d=n2d)]
    ns = len(full)
    tris = int(sum(len(s[2]) for s in full))
    b = Batch()
    b.set_scenes(full)
    b.set_tuning(**best)
    runs = {}
    for name, prec in (("fp64", PREC_FP64), ("fp32cert", PREC_FP32_CERTIFIED)):
        b.set_precision(prec)
        b.run()
        b.results()
        b.run()
        r = b.results()
        ms, d = r["batch_ms"], r["done_ms"]
        nst = int(r["n_stencils"].sum())
        runs[name] = {"batch_ms": ms, "scenes_per_s": ns / ms * 1e3, "stencils": nst,
                      "stencils_per_s": nst / ms * 1e3, "hits": int(r["n_hits"].sum()),
                      "waves_redos": list(b.wave_stats()),
                      "scene_latency_ms": {"p50": float(np.percentile(d, 50)), "p99": float(np.percentile(d, 99)),
                                           "max": float(d.max())}}
        if name == "fp64":
            ref = r
        else:
            runs[name]["same_hit_counts_as_fp64"] = bool(np.array_equal(r["n_hits"], ref["n_hits"]))
    out = {"workload": f"{ns} scenes: {n3d} folded cloths (side log-uniform [16, 384], thickness 1e-3) + {n2d} 2D "
                       "annuli (ring U[32, 2048]), one CUDA graph per run",
           "tris": tris, "tuning": best, "tuning_table": [[c, t] for c, t in table]}
    out.update(runs["fp64"])
    out["fp32cert"] = runs["fp32cert"]
    return out

def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_b200(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
