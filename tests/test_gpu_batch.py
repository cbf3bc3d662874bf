"""Batched path (mclccd_batch_*) against the single-scene path, scene by
scene: candidate, hit and discrete counts, the earliest toi and its stencil
(bit-identical in FP64); the FP32-certified form; every tuning; new
positions through the refit of an existing batch."""
import numpy as np
import pytest

from mclccd_b200 import PREC_FP32_CERTIFIED, PREC_FP64, BVHTree, scenes
from mclccd_b200.autotune import tune_batch
from mclccd_b200.batch import FORM_PERSISTENT, FORM_WAVES, Batch

pytestmark = pytest.mark.gpu


def small_batch(seed=0):
    out = []
    for i, side in enumerate((6, 9, 14, 21, 33, 48)):
        out.append(scenes.folded_cloth(side, seed=seed * 100 + i))
    for i, ring in enumerate((32, 57, 120, 260)):
        out.append(scenes.annulus_2d(ring, seed=seed * 100 + 50 + i))
    V0, V1, F, eta = scenes.folded_cloth(2, seed=seed)   # 2 triangles
    out.append((V0, V1, F, eta))
    out.append((V0, V1, F[:1], eta))                     # 1 triangle: no pairs
    return out


def expected(scene, precision=PREC_FP64):
    V0, V1, F, eta = scene
    t = BVHTree(V0.shape[1], precision=precision)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    c = t.counts()
    sten, is_vf, toi = t.hits()
    out = {"n_hits": c["hits"], "n_discrete": c["discrete"], "n_stencils": c["vf"] + c["ee"]}
    if len(toi):
        m = toi.min()
        cand = [(0 if v else 1, *map(int, s)) for s, v, x in zip(sten, is_vf, toi) if x == m]
        best = min(cand)
        out.update(min_toi=m, min_sten=best[1:], min_is_vf=1 - best[0])
    else:
        out.update(min_toi=-1.0, min_sten=(-1, -1, -1, -1), min_is_vf=0)
    return out


def check(res, exp, exact=True):
    for s, e in enumerate(exp):
        assert res["n_hits"][s] == e["n_hits"], s
        assert res["n_discrete"][s] == e["n_discrete"], s
        assert res["n_stencils"][s] == e["n_stencils"], s
        if exact:
            assert res["min_toi"][s] == e["min_toi"], (s, res["min_toi"][s], e["min_toi"])
            if e["n_hits"]:
                assert tuple(res["min_sten"][s]) == tuple(e["min_sten"]), s
                assert res["min_is_vf"][s] == e["min_is_vf"], s


def test_batch_fp64_matches_single_scene():
    sc = small_batch()
    b = Batch()
    b.set_scenes(sc)
    b.run()
    r = b.results()
    check(r, [expected(s) for s in sc])
    assert r["batch_ms"] > 0 and np.all(r["done_ms"] <= r["batch_ms"] * 1.5 + 1.0)


def test_batch_every_tuning_same_results():
    sc = small_batch(1)
    exp = [expected(s) for s in sc]
    b = Batch()
    b.set_scenes(sc)
    for form in (FORM_WAVES, FORM_PERSISTENT):
        for block in (128, 256):
            for stack in (32, 64):
                for knob in (1, 7):   # wave buffer (waves) or queue chunk (persistent)
                    for leaf in (1, 4):
                        b.set_tuning(form=form, block=block, stack=stack, leaf=leaf,
                                     **({"wave": knob} if form == FORM_WAVES else {"chunk": knob}))
                        b.run()
                        check(b.results(), exp)


def test_batch_waves_redo_on_overflow():
    # a 128 x 128 fold has far more leaf pairs than a 2^16-pair wave buffer
    # holds: the first waves overflow and are redone with fewer queries
    sc = [scenes.folded_cloth(128, seed=11), scenes.annulus_2d(700, seed=12), scenes.folded_cloth(20, seed=13)]
    exp = [expected(s) for s in sc]
    b = Batch()
    b.set_scenes(sc)
    b.set_tuning(form=FORM_WAVES, wave=1)
    b.run()
    check(b.results(), exp)
    waves, redos = b.wave_stats()
    assert redos > 0 and waves > 2, (waves, redos)
    b.run()   # the adapted wave size carries over: same results
    check(b.results(), exp)
    b.set_tuning(form=FORM_PERSISTENT)
    b.run()
    check(b.results(), exp)
    assert b.wave_stats() == (0, 0)


def test_batch_certified():
    sc = small_batch(2)
    exp = [expected(s) for s in sc]
    b = Batch(precision=PREC_FP32_CERTIFIED)
    b.set_scenes(sc)
    for form in (FORM_WAVES, FORM_PERSISTENT):
        b.set_tuning(form=form)
        b.run()
        r = b.results()
        check(r, exp, exact=False)
        for s, e in enumerate(exp):
            if e["n_hits"]:
                assert r["min_toi"][s] <= e["min_toi"] and r["min_toi"][s] >= e["min_toi"] * (1 - 1e-6)


def test_batch_new_positions_and_autotune():
    sc = small_batch(3)
    b = Batch()
    b.set_scenes(sc)
    rng = np.random.default_rng(4)
    V1s = [s[1] + rng.normal(0, 1e-3, s[1].shape) for s in sc]
    b.set_positions([s[0] for s in sc], V1s)
    best, table = tune_batch(b, space={"form": (0, 1), "block": (128,), "stack": (64,), "chunk": (1, 4), "leaf": (1, 2),
                                       "wave": (1, 512)}, repeats=1)
    assert len(table) == 8   # each form varies only its own knob
    assert best in [c for c, t in table if t is not None]
    b.run()
    check(b.results(), [expected((s[0], v1, s[2], s[3])) for s, v1 in zip(sc, V1s)])
