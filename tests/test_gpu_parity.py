"""GPU parity: the CUDA path (through the C ABI) against the reference's golden
fixtures and the oracle restatement on the same seeded inputs.

Bar: leaf boxes, representative flags, the canonical candidate-stencil set,
the discrete-pair set and hit/miss are bit-exact; toi is bit-exact too for the
FP64 path (same IEEE operations, no FMA), tested at 0 ulp."""
import os

import numpy as np
import pytest

from mclccd_b200 import PREC_FP64, BVHTree, CCDError, narrow_phase_bulk, scenes
from oracle.ref import Port, canonical_set, sort_rows

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
KATS = ["headon", "parallel", "shared", "static", "coplanar", "degenerate", "fold12", "spheres", "annulus48", "segments2d"]


@pytest.fixture(scope="module")
def port():
    return Port()


@pytest.fixture(scope="module")
def kats():
    z = np.load(os.path.join(GOLD, "kat_small.npz"))
    return {name: {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")} for name in z["names"]}


def run_gpu(V0, V1, F, eta, **opts):
    t = BVHTree(V0.shape[1])
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    for k, v in opts.items():
        setattr(t.options, k, v)
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    return t


def hit_map(sten, is_vf, toi):
    return {(int(v),) + tuple(int(x) for x in s): float(t) for s, v, t in zip(sten, is_vf, toi)}


def check_against_port(t, port, V0, V1, F, eta):
    p = port.run(V0, V1, F, eta)
    b, f = t.leaves(len(F))
    assert np.array_equal(b, p["leaf_boxes"])
    assert np.array_equal(f, p["leaf_flags"])
    cs, cv = t.candidates()
    assert np.array_equal(canonical_set(cs, cv), canonical_set(p["cand_sten"], p["cand_is_vf"]))
    assert np.array_equal(sort_rows(t.discrete()), sort_rows(p["discrete"]))
    hs, hv, ht = t.hits()
    # same orientation convention as the port (lower primitive first): exact maps
    got = hit_map(hs, hv, ht)
    want = hit_map(p["hit_sten"], p["hit_is_vf"], p["hit_toi"])
    assert got.keys() == want.keys()
    bad = [k for k in want if got[k] != want[k]]
    assert not bad, f"{len(bad)} toi mismatches, e.g. {bad[:3]}"
    return p


@pytest.mark.parametrize("name", KATS)
def test_kat_against_reference_golden(kats, name):
    g = kats[name]
    eta = float(g["eta"])
    t = run_gpu(g["V0"], g["V1"], g["F"], eta)
    b, f = t.leaves(len(g["F"]))
    assert np.array_equal(b, g["leaf_boxes"])
    flags = np.stack([(f >> j) & 1 for j in range(7)], axis=1)
    assert np.array_equal(flags, g["leaf_flags"])
    cs, cv = t.candidates()
    assert np.array_equal(canonical_set(cs, cv), g["cand"])
    assert np.array_equal(sort_rows(t.discrete()), g["discrete"])
    hs, hv, ht = t.hits()
    assert np.array_equal(canonical_set(hs, hv), g["hits"])
    m = (g["canon_hit"] == 1) & (g["canon_toi"] >= 0)
    want = hit_map(g["canon_sten"][m], g["canon_is_vf"][m], g["canon_toi"][m])
    assert hit_map(hs, hv, ht) == want


def test_cfg0_folded_cloth(port):
    V0, V1, F, eta = scenes.folded_cloth(64)
    t = run_gpu(V0, V1, F, eta)
    c = t.counts()
    assert (c["vf"], c["ee"], c["hits"], c["discrete"]) == (768841, 1711130, 2410926, 1061)
    check_against_port(t, port, V0, V1, F, eta)


def test_traverse_out_delivers_the_results(port):
    # mclccd_traverse_out: results streamed into caller arrays (host copies
    # overlapping the chunked step) equal the traverse + get_hits results
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=161, seed=9)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    p = check_against_port(t, port, V0, V1, F, eta)
    want = hit_map(*t.hits())
    wd = sort_rows(t.discrete())
    n = len(want)
    cap = n + 100
    hs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
    hv = torch.empty(cap, dtype=torch.uint8).pin_memory()
    ht = torch.empty(cap, dtype=torch.float64).pin_memory()
    hd = torch.empty((len(wd) + 10, 2), dtype=torch.int32).pin_memory()
    nh, nd = t.traverse_out(hs, hv, ht, hd, V0, V1, F)
    assert (nh, nd) == (n, len(wd))
    assert hit_map(hs[:nh].numpy(), hv[:nh].numpy(), ht[:nh].numpy()) == want
    assert np.array_equal(sort_rows(hd[:nd].numpy()), wd)
    # refit-only step, outputs on the device
    t.update(V0, V1, F)
    ds, dv, dt = (torch.empty_like(x, device="cuda") for x in (hs, hv, ht))
    nh2, _ = t.traverse_out(ds, dv, dt)
    assert nh2 == n and hit_map(ds[:n].cpu().numpy(), dv[:n].cpu().numpy(), dt[:n].cpu().numpy()) == want
    # a capacity below the count: a prefix, the full count reported
    small = n // 3
    nh3, _ = t.traverse_out(hs[:small], hv[:small], ht[:small])
    assert nh3 == n
    got = hit_map(hs[:small].numpy(), hv[:small].numpy(), ht[:small].numpy())
    assert len(got) == small and all(want[k] == v for k, v in got.items())


def test_traverse_out_overflow_retry(port):
    # a fresh handle's lists are sized for a few stencils per triangle; the
    # 64 x 64 fold has ~100 VF stencils per triangle, so the streamed step
    # overflows, regrows and runs again: the delivered results are exact
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.folded_cloth(64)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    cap = 2_500_000
    hs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
    hv = torch.empty(cap, dtype=torch.uint8).pin_memory()
    ht = torch.empty(cap, dtype=torch.float64).pin_memory()
    hd = torch.empty((2048, 2), dtype=torch.int32).pin_memory()
    nh, nd = t.traverse_out(hs, hv, ht, hd)
    assert (nh, nd) == (2410926, 1061)
    p = check_against_port(t, port, V0, V1, F, eta)
    assert hit_map(hs[:nh].numpy(), hv[:nh].numpy(), ht[:nh].numpy()) == hit_map(*t.hits())
    assert np.array_equal(sort_rows(hd[:nd].numpy()), sort_rows(p["discrete"]))


@pytest.mark.parametrize("case", ["small", "certified", "2d"])
def test_traverse_out_other_paths(case):
    # delivery after the step instead of streaming (a scene below the
    # chunking threshold, the certified form) and streaming in a 2D tree
    torch = pytest.importorskip("torch")
    from mclccd_b200 import PREC_FP32_CERTIFIED
    V0, V1, F, eta = {"small": lambda: scenes.folded_cloth(20, seed=3),
                      "certified": lambda: scenes.wavy_cloth(1025, rows=65, seed=4),
                      "2d": lambda: scenes.annulus_2d(900, seed=5)}[case]()
    t = BVHTree(V0.shape[1], precision=PREC_FP32_CERTIFIED if case == "certified" else PREC_FP64)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse()
    want = hit_map(*t.hits())
    wd = sort_rows(t.discrete())
    cap = len(want) + 16
    hs = torch.empty((cap, 4), dtype=torch.int32).pin_memory()
    hv = torch.empty(cap, dtype=torch.uint8).pin_memory()
    ht = torch.empty(cap, dtype=torch.float64).pin_memory()
    hd = torch.empty((len(wd) + 16, 2), dtype=torch.int32).pin_memory()
    nh, nd = t.traverse_out(hs, hv, ht, hd)
    assert (nh, nd) == (len(want), len(wd))
    assert hit_map(hs[:nh].numpy(), hv[:nh].numpy(), ht[:nh].numpy()) == want
    assert np.array_equal(sort_rows(hd[:nd].numpy()), wd)


@pytest.mark.parametrize("chunks", [2, 5])
@pytest.mark.parametrize("scene", ["wavy", "annulus"])
def test_overlapped_traverse_against_port(port, chunks, scene):
    # walk of one query chunk overlapped with the narrow phase of the previous
    # one: same candidates, hits (bit-identical toi) and discrete pairs
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=97, seed=7) if scene == "wavy" else scenes.annulus_2d(800, seed=8)
    t = BVHTree(V0.shape[1])
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(overlap=chunks)
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    check_against_port(t, port, V0, V1, F, eta)
    t.update(V0, V1, F)
    t.traverse()
    check_against_port(t, port, V0, V1, F, eta)


@pytest.mark.parametrize("window", [32, 128])
@pytest.mark.parametrize("scene", ["wavy", "annulus", "active"])
def test_walk_window_against_port(port, window, scene):
    # the Morton-window walk (shared-memory scan of the next W leaves, then
    # the tree beyond them) finds exactly the reference's leaf pairs
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=97, seed=5) if scene != "annulus" else scenes.annulus_2d(500, seed=6)
    t = BVHTree(V0.shape[1])
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(walk_window=window)
    if scene == "active":   # partial-mesh CCD: only a band of vertices active
        act = (np.arange(len(V0)) % 7 < 2).astype(np.int32)
        t.update(V0, V1, F, active=act)
        t.traverse(V0, V1, F)
        p = port.run(V0, V1, F, eta, active=act)
        cs, cv = t.candidates()
        assert np.array_equal(canonical_set(cs, cv), canonical_set(p["cand_sten"], p["cand_is_vf"]))
        return
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    check_against_port(t, port, V0, V1, F, eta)


def device_results(t):
    cs, cv = t.candidates()
    return canonical_set(cs, cv), hit_map(*t.hits()), sort_rows(t.discrete())


@pytest.mark.parametrize("window", [8, 16, 32])
@pytest.mark.parametrize("scene", ["wavy", "annulus", "active"])
def test_walk_buffer_matches_window_walk(window, scene):
    # the buffered walk (pairs collected per warp, written 32 at a time) finds
    # the same leaf pairs as the window walk
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=97, seed=5) if scene != "annulus" else scenes.annulus_2d(500, seed=6)
    act = (np.arange(len(V0)) % 7 < 2).astype(np.int32) if scene == "active" else None
    out = []
    for buf in (0, 1, 2):
        t = BVHTree(V0.shape[1])
        t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
        t.set_tuning(walk_window=window)
        t.set_tuning(walk_buffer=buf)
        t.update(V0, V1, F, active=act)
        t.traverse(V0, V1, F)
        out.append(device_results(t) + (t.counts()["leaf_pairs"],))
    for o in out[1:]:
        assert out[0][3] == o[3] > 0
        assert np.array_equal(out[0][0], o[0])
        assert out[0][1] == o[1]
        assert np.array_equal(out[0][2], o[2])


@pytest.mark.parametrize("window", [8, 16, 32])
@pytest.mark.parametrize("scene", ["wavy", "annulus", "active"])
def test_walk_refill_matches_window_walk(window, scene):
    # the refill walk (persistent warps, idle lanes refilled from a per-warp
    # query pool) finds the same leaf pairs as the window walk it reorders;
    # candidates, hits with toi and discrete pairs equal, in the full step and
    # in the streamed (query-chunked) step
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=97, seed=5) if scene != "annulus" else scenes.annulus_2d(500, seed=6)
    act = (np.arange(len(V0)) % 7 < 2).astype(np.int32) if scene == "active" else None
    out = []
    for refill in (0, 1):
        t = BVHTree(V0.shape[1])
        t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
        t.set_tuning(walk_window=window)
        t.set_tuning(walk_refill=refill)
        t.update(V0, V1, F, active=act)
        t.traverse(V0, V1, F)
        out.append(device_results(t) + (t.counts()["leaf_pairs"],))
    assert out[0][3] == out[1][3] > 0
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][2], out[1][2])
    if scene == "wavy":   # chunked queries through traverse_out
        n = len(out[0][1])
        hs = torch.empty((n + 64, 4), dtype=torch.int32).pin_memory()
        hv = torch.empty(n + 64, dtype=torch.uint8).pin_memory()
        ht = torch.empty(n + 64, dtype=torch.float64).pin_memory()
        nh, _ = t.traverse_out(hs, hv, ht)
        assert nh == n and hit_map(hs[:n].numpy(), hv[:n].numpy(), ht[:n].numpy()) == out[0][1]


@pytest.mark.parametrize("scene", ["fold", "annulus", "wavy"])
def test_fused_narrow_phase_against_port(port, scene):
    # the fused form (pairs -> stencils -> discrete test -> ACCD in one
    # kernel, candidate lists rebuilt on request) gives the reference's sets
    if scene == "fold":
        V0, V1, F, eta = scenes.folded_cloth(40, seed=8)
    elif scene == "annulus":
        V0, V1, F, eta = scenes.annulus_2d(300, seed=9)
    else:
        V0, V1, F, eta = scenes.wavy_cloth(1025, rows=49, seed=3)
    t = BVHTree(V0.shape[1])
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(narrow_fused=1)
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    check_against_port(t, port, V0, V1, F, eta)
    c = t.counts()
    p = port.run(V0, V1, F, eta)
    assert (c["vf"], c["ee"]) == (int(p["cand_is_vf"].sum()), int(len(p["cand_is_vf"]) - p["cand_is_vf"].sum()))


@pytest.mark.parametrize("form", ["walk_refill", "walk_buffer"])
def test_walk_forms_against_port(port, form):
    V0, V1, F, eta = scenes.folded_cloth(40, seed=7)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(**{form: 1})
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    check_against_port(t, port, V0, V1, F, eta)


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("dim", [3, 2])
def test_rebinned_accd_against_port(port, dim, form):
    # the re-binned ACCD forms (1: heads and tails in separate warp passes of
    # one kernel; 2: a head kernel and a tail kernel over a queue of the
    # stencils that go on) give the same bits as the one-stencil-per-thread form
    V0, V1, F, eta = scenes.folded_cloth(48, seed=21) if dim == 3 else scenes.annulus_2d(300, seed=22)
    t = BVHTree(dim)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(accd_rebin=form)
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    assert t.get_tuning()["accd_rebin"] == form
    check_against_port(t, port, V0, V1, F, eta)


@pytest.mark.parametrize("split", [1, 2])
@pytest.mark.parametrize("scene", ["fold", "annulus"])
def test_expand_split_against_port(port, scene, split):
    # the stencil expansion and the discrete test as two kernels (2: the
    # discrete test on lane-compacted pairs), with the split ACCD form: the
    # reference's sets
    V0, V1, F, eta = scenes.folded_cloth(40, seed=11) if scene == "fold" else scenes.annulus_2d(300, seed=12)
    t = BVHTree(V0.shape[1])
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.set_tuning(expand_split=split, accd_rebin=2)
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    check_against_port(t, port, V0, V1, F, eta)


def test_split_accd_full_size_step_equals_default():
    # the split form on the 2.1M-triangle cloth, streamed per query chunk
    # (the head kernel's queue is reset per chunk): the same hits and toi
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.wavy_cloth(1025, rows=257, seed=2)
    maps = []
    for form in (0, 2):
        t = BVHTree(3)
        t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
        t.set_tuning(accd_rebin=form, expand_split=form // 2)
        t.update(V0, V1, F)
        t.traverse(V0, V1, F)
        maps.append(hit_map(*t.hits()))
        n = len(maps[-1])
        hs = torch.empty((n + 64, 4), dtype=torch.int32).pin_memory()
        hv = torch.empty(n + 64, dtype=torch.uint8).pin_memory()
        ht = torch.empty(n + 64, dtype=torch.float64).pin_memory()
        nh, _ = t.traverse_out(hs, hv, ht)
        assert nh == n and hit_map(hs[:n].numpy(), hv[:n].numpy(), ht[:n].numpy()) == maps[-1]
    assert maps[0] == maps[1] and len(maps[0]) > 1_000_000


@pytest.mark.parametrize("scene", ["wavy129", "spheres", "annulus", "fold_big_motion"])
def test_scenes_against_port(port, scene):
    V0, V1, F, eta = {
        "wavy129": lambda: scenes.wavy_cloth(129, seed=3),
        "spheres": lambda: scenes.icospheres(12, 3, seed=5),
        "annulus": lambda: scenes.annulus_2d(400, seed=7),
        "fold_big_motion": lambda: scenes.folded_cloth(40, seed=9, noise=0.02),
    }[scene]()
    t = run_gpu(V0, V1, F, eta)
    check_against_port(t, port, V0, V1, F, eta)


def test_touching_boxes(port):
    """Boxes that touch exactly, or miss by one FP64 ulp: the FP32 brackets
    cannot decide these, so the exact FP64 test must."""
    rng = np.random.default_rng(5)
    tris, V = [], []
    for i in range(400):
        x0 = 0.3 * (i % 20)
        y0 = 0.3 * (i // 20)
        gap = [0.0, 5e-17, -5e-17, 1e-16][i % 4]
        base = len(V)
        V += [[x0, y0, 0.0], [x0 + 0.2 + gap, y0, 0.0], [x0, y0 + 0.2 - gap, 0.0]]
        tris.append([base, base + 1, base + 2])
    V0 = np.array(V, np.float64)
    V1 = V0 + rng.normal(0, 1e-9, V0.shape) * (rng.random(V0.shape) < 0.3)
    F = np.array(tris, np.int32)
    t = run_gpu(V0, V1, F, 0.05)
    p = check_against_port(t, port, V0, V1, F, 0.05)
    assert len(p["leaf_pairs"]) > 500


def test_refit_equals_rebuild(port):
    V0, V1, F, eta = scenes.wavy_cloth(97, seed=1)
    V1b = scenes.wavy_redraw(V0, 77)
    t = run_gpu(V0, V1, F, eta)
    t.update(V0, V1b, F)            # same F -> refit-only path
    t.traverse(V0, V1b, F)
    check_against_port(t, port, V0, V1b, F, eta)
    u = run_gpu(V0, V1b, F, eta, always_rebuild=True)
    for a, b in ((t.candidates(), u.candidates()),):
        assert np.array_equal(canonical_set(*a), canonical_set(*b))


def test_changed_topology_same_sizes_rebuilds(port):
    # same np, pdim and nv but a different P: the refit launched before the
    # comparison returns is followed by a full build, and the results are the
    # new topology's.  (reptri off: with np unchanged the reference keeps the
    # old representative flags, BVHTree.cpp:44-48, so only all-represented
    # flags mean the same for both topologies.)
    V0, V1, F, eta = scenes.wavy_cloth(97, seed=1)
    t = run_gpu(V0, V1, F, eta, reptri=False)
    assert t.build_stats()[0] == 1
    G = np.ascontiguousarray(np.random.default_rng(5).permutation(F)[:, [1, 2, 0]])
    p = port.run(V0, V1, G, eta, reptri=False)

    def check():
        assert np.array_equal(canonical_set(*t.candidates()), canonical_set(p["cand_sten"], p["cand_is_vf"]))
        assert np.array_equal(sort_rows(t.discrete()), sort_rows(p["discrete"]))
        assert hit_map(*t.hits()) == hit_map(p["hit_sten"], p["hit_is_vf"], p["hit_toi"])

    t.update(V0, V1, G)
    t.traverse(V0, V1, G)
    assert t.build_stats()[0] == 2
    check()
    t.update(V0, V1, G)             # unchanged again: refit only
    t.traverse(V0, V1, G)
    assert t.build_stats()[0] == 2
    check()


def test_quality_triggered_rebuild(port):
    # F never changes while 12 spheres drift apart along their own random
    # directions: every leaf box keeps its size, but the refit-only tree keeps
    # the grouping of the first positions, so its internal boxes stretch over
    # spheres now far apart; the quality trigger rebuilds it.  The results
    # stay those of a freshly built tree.
    V0, V1, F, eta = scenes.icospheres(12, 3, seed=5)
    nvs = len(V0) // 12
    vel = np.repeat(np.random.default_rng(6).normal(0.0, 0.15, (12, 3)), nvs, axis=0)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    X, Y = V0, V1
    for step in range(8):
        if step:
            X, Y = X + vel, Y + vel
        t.update(X, Y, F)
        t.traverse(X, Y, F)
        if step == 0:
            check_against_port(t, port, X, Y, F, eta)
    fresh = BVHTree(3)
    fresh.options.box_eta = fresh.options.vf_ccd_eta = fresh.options.ee_ccd_eta = eta
    fresh.update(X, Y, F)
    fresh.traverse(X, Y, F)
    assert np.array_equal(device_results(t)[0], device_results(fresh)[0])
    assert device_results(t)[1] == device_results(fresh)[1]
    builds, by_quality = t.build_stats()
    assert by_quality >= 1 and builds == 1 + by_quality
    t2 = BVHTree(3)
    t2.set_tuning(rebuild_ratio=0)
    t2.update(V0, V1, F)
    t2.update(V0 + vel, V1 + vel, F)
    assert t2.build_stats() == (1, 0)


def test_options(port):
    V0, V1, F, eta = scenes.folded_cloth(24, seed=4)
    # continuous off: no stencils; discrete off: no discrete pairs
    t = run_gpu(V0, V1, F, eta, continuous=False)
    c = t.counts()
    assert c["vf"] == c["ee"] == c["hits"] == 0 and c["discrete"] == len(port.run(V0, V1, F, eta)["discrete"])
    t = run_gpu(V0, V1, F, eta, discrete=False)
    assert t.counts()["discrete"] == 0
    # reptri off: every vertex / edge slot represented (BVHLeaf.hpp:45-49)
    t = run_gpu(V0, V1, F, eta, reptri=False)
    p = port.run(V0, V1, F, eta, reptri=False)
    cs, cv = t.candidates()
    assert np.array_equal(canonical_set(cs, cv), canonical_set(p["cand_sten"], p["cand_is_vf"]))
    # gaps above box_eta are clamped to it (BVHTree.cpp:39-40)
    t = BVHTree(3)
    t.options.box_eta, t.options.vf_ccd_eta, t.options.ee_ccd_eta = eta, 10 * eta, 10 * eta
    t.update(V0, V1, F)
    assert t.options.vf_ccd_eta == eta and t.options.ee_ccd_eta == eta
    t.traverse(V0, V1, F)
    q = port.run(V0, V1, F, eta)
    assert np.array_equal(canonical_set(*t.hits()[:2]), canonical_set(q["hit_sten"], q["hit_is_vf"]))


def test_active_mask(port):
    V0, V1, F, eta = scenes.folded_cloth(24, seed=6)
    rng = np.random.default_rng(0)
    active = (rng.random(len(V0)) < 0.1).astype(np.int32)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F, active=active)
    t.traverse(V0, V1, F)
    p = port.run(V0, V1, F, eta, active=active)
    cs, cv = t.candidates()
    assert np.array_equal(canonical_set(cs, cv), canonical_set(p["cand_sten"], p["cand_is_vf"]))
    b, f = t.leaves(len(F))
    assert np.array_equal(f, p["leaf_flags"])


def test_hooks_and_stop():
    V0, V1, F, eta = scenes.folded_cloth(32, seed=2)
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    got, disc = [], []
    t.append_pair = lambda s, v, toi: got.append((tuple(s), v, toi))
    t.append_discrete = lambda a, b: (disc.append((a, b)), True)[1]   # stop after the first
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    c = t.counts()
    assert len(got) == c["hits"] and all(toi >= 0 for _, _, toi in got)
    assert len(disc) == (1 if c["discrete"] else 0)
    # host filter_pair / narrow_phase hooks
    t2 = BVHTree(3)
    t2.options.box_eta = t2.options.vf_ccd_eta = t2.options.ee_ccd_eta = eta
    t2.filter_pair = lambda s, is_vf: not is_vf          # keep VF only
    t2.update(V0, V1, F)
    t2.traverse(V0, V1, F)
    hs, hv, ht = t2.hits()
    full = t.hits()
    assert np.all(hv == 1)
    assert len(hs) == int(np.sum(full[1] == 1))


def test_empty_single_and_errors():
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)
    t = BVHTree(3)
    t.update(V, V, np.zeros((0, 3), np.int32))
    t.traverse(V, V, np.zeros((0, 3), np.int32))
    assert t.counts()["hits"] == 0
    t.update(V, V + 0.1, np.array([[0, 1, 2]], np.int32))
    t.traverse(V, V + 0.1, np.array([[0, 1, 2]], np.int32))
    assert t.counts()["leaf_pairs"] == 0
    bad = BVHTree(3)
    with pytest.raises(CCDError) as e:
        bad.traverse(V, V, np.array([[0, 1, 2]], np.int32))
    assert e.value.status == 5   # STATE: traverse before update
    with pytest.raises(CCDError) as e:
        bad.update(V, V, np.array([[0, 1, 7], [0, 1, 2]], np.int32))
    assert e.value.status == 1   # index out of range


def test_bulk_narrow_phase_matches_port(port):
    rng = np.random.default_rng(3)
    n, nv = 20000, 4000
    V0 = rng.random((nv, 3))
    V1 = V0 + rng.normal(0, 0.05, V0.shape)
    sten = rng.integers(0, nv, (n, 4)).astype(np.int32)
    is_vf = (rng.random(n) < 0.5).astype(np.uint8)
    # degenerate stencils: repeated vertices, zero motion, parallel edges
    sten[:200, 1] = sten[:200, 0]
    V1[:50] = V0[:50]
    sten[200:300, 2:] = sten[200:300, :2]
    for eta in (1e-3, 0.05):
        toi, hit = narrow_phase_bulk(V0, V1, sten, is_vf, eta)
        h2, t2 = port.accd(V0, V1, sten, is_vf, eta)
        assert np.array_equal(hit, h2)
        # degenerate triangles (repeated vertex) give hit == 1 with toi = NaN
        # in the reference too; the pipeline's toi >= 0 gate drops them
        assert np.array_equal(toi, t2, equal_nan=True)
        assert np.isnan(toi).sum() == 2
    z = np.load(os.path.join(GOLD, "cfg0_sample.npz"))
    V0, V1, F, eta = scenes.folded_cloth(64)
    toi, hit = narrow_phase_bulk(V0, V1, z["sten"], z["is_vf"], eta)
    assert np.array_equal(hit, z["hit"]) and np.array_equal(toi, z["toi"])


def test_device_tensors(port):
    torch = pytest.importorskip("torch")
    V0, V1, F, eta = scenes.folded_cloth(48, seed=8)
    d = lambda a: torch.from_numpy(a).cuda()
    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(d(V0), d(V1), d(F))
    t.traverse(d(V0), d(V1), d(F))
    check_against_port(t, port, V0, V1, F, eta)
    t.traverse()   # NULL arrays: reuse the update's
    check_against_port(t, port, V0, V1, F, eta)


def test_float32_coordinates():
    # BVHTree<float, DIM>: float32 inputs (host arrays or CUDA tensors) give
    # the FP64 results for the same coordinates widened exactly to double
    torch = pytest.importorskip("torch")
    for V0, V1, F, eta in (scenes.folded_cloth(32, seed=41), scenes.annulus_2d(256, seed=42)):
        dim = V0.shape[1]
        f0, f1 = V0.astype(np.float32), V1.astype(np.float32)
        feta = float(np.float32(eta))
        ref_t = run_gpu(f0.astype(np.float64), f1.astype(np.float64), F, feta)
        want = hit_map(*ref_t.hits())
        for a0, a1, aF in ((f0, f1, F), tuple(torch.from_numpy(x).cuda() for x in (f0, f1, F))):
            t = BVHTree(dim)
            t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = feta
            t.update(a0, a1, aF)
            t.traverse(a0, a1, aF)
            assert hit_map(*t.hits()) == want
            assert np.array_equal(sort_rows(t.discrete()), sort_rows(ref_t.discrete()))
            t.update(a0, a1, aF)   # refit-only second step, traverse on the update's arrays
            t.traverse()
            assert hit_map(*t.hits()) == want


def test_fp64_fma_rate_is_a_b200_figure():
    # the measured denominator of the narrow phase's FP64 roofline: below the
    # nominal 148 SMs x 64 lanes x 2 flops x 1.965 GHz and well above zero
    from mclccd_b200.ccd import fp64_fma_rate
    r = fp64_fma_rate(0)
    assert 5.0 < r <= 148 * 64 * 2 * 1.965e9 / 1e12 * 1.02, r
