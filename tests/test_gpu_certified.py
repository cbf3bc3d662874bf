"""FP32-certified form against the FP64 path.

The bar: identical hit/miss; the reported toi is never later than
the FP64 toi and within 1e-6 relative of it (toi 0 stays exactly 0);
candidate and discrete sets unchanged."""
import numpy as np
import pytest

from mclccd_b200 import PREC_FP32_CERTIFIED, PREC_FP64, BVHTree, narrow_phase_bulk, scenes
from oracle.ref import Port, canonical_set, sort_rows

pytestmark = pytest.mark.gpu
TOI_REL = 1e-6


def check_toi(t_cert, t_fp64):
    t_cert = np.asarray(t_cert); t_fp64 = np.asarray(t_fp64)
    fin = np.isfinite(t_fp64)
    assert np.array_equal(np.isfinite(t_cert), fin)
    c, f = t_cert[fin], t_fp64[fin]
    miss = f < 0
    assert np.all(c[miss] == -1.0)
    c, f = c[~miss], f[~miss]
    assert np.all(c <= f), "certified toi later than FP64"
    assert np.all(c >= f - TOI_REL * f), f"max rel err {np.max((f - c) / np.maximum(f, 1e-300))}"
    assert np.all(c[f == 0] == 0)


def run(V0, V1, F, eta, precision):
    t = BVHTree(V0.shape[1], precision=precision)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    return t


def keyed(sten, is_vf, toi):
    return {(int(v),) + tuple(map(int, s)): float(x) for s, v, x in zip(sten, is_vf, toi)}


@pytest.mark.parametrize("scene", ["cfg0", "wavy129", "spheres", "annulus", "fold_big_motion"])
def test_certified_pipeline_matches_fp64(scene):
    V0, V1, F, eta = {
        "cfg0": lambda: scenes.folded_cloth(64),
        "wavy129": lambda: scenes.wavy_cloth(129, seed=3),
        "spheres": lambda: scenes.icospheres(12, 3, seed=5),
        "annulus": lambda: scenes.annulus_2d(400, seed=7),
        "fold_big_motion": lambda: scenes.folded_cloth(40, seed=9, noise=0.02),
    }[scene]()
    a = run(V0, V1, F, eta, PREC_FP64)
    b = run(V0, V1, F, eta, PREC_FP32_CERTIFIED)
    assert np.array_equal(canonical_set(*a.candidates()), canonical_set(*b.candidates()))
    assert np.array_equal(sort_rows(a.discrete()), sort_rows(b.discrete()))
    ka, kb = keyed(*a.hits()), keyed(*b.hits())
    assert ka.keys() == kb.keys()                    # identical hit/miss
    keys = list(ka)
    check_toi([kb[k] for k in keys], [ka[k] for k in keys])
    n_sten = a.counts()["vf"] + a.counts()["ee"]
    print(f"{scene}: {b.fp64_fallbacks()} of {n_sten} stencils evaluated in FP64")
    assert b.fp64_fallbacks() <= 0.25 * n_sten + 10


def test_certified_bulk_stress_stencils():
    V0, V1, sten, is_vf, eta = scenes.stress_stencils(100_000, seed=0)
    t64, h64 = narrow_phase_bulk(V0, V1, sten, is_vf, eta)
    tc, hc, nfb = narrow_phase_bulk(V0, V1, sten, is_vf, eta, precision=PREC_FP32_CERTIFIED, return_fallbacks=True)
    assert np.array_equal(h64, hc)
    check_toi(tc, t64)
    assert 0 < nfb < len(sten)        # the hard cases do reach FP64, the rest does not


def test_certified_bulk_random_and_degenerate():
    rng = np.random.default_rng(11)
    n, nv = 40000, 6000
    V0 = rng.random((nv, 3))
    V1 = V0 + rng.normal(0, 0.03, V0.shape)
    sten = rng.integers(0, nv, (n, 4)).astype(np.int32)
    is_vf = (rng.random(n) < 0.5).astype(np.uint8)
    sten[:100, 3] = sten[:100, 2]        # degenerate triangles / point edges
    V1[:40] = V0[:40]                    # no motion
    for eta in (1e-3, 2e-2):
        t64, h64 = narrow_phase_bulk(V0, V1, sten, is_vf, eta)
        tc, hc = narrow_phase_bulk(V0, V1, sten, is_vf, eta, precision=PREC_FP32_CERTIFIED)
        assert np.array_equal(h64, hc)
        nan = np.isnan(t64)
        assert np.array_equal(nan, np.isnan(tc))
        check_toi(tc[~nan], t64[~nan])


def test_certified_matches_oracle_port():
    """The certified toi brackets the oracle's FP64 toi too (not only ours)."""
    V0, V1, sten, is_vf, eta = scenes.stress_stencils(20_000, seed=3)
    h, t = Port().accd(V0, V1, sten, is_vf, eta)
    tc, hc = narrow_phase_bulk(V0, V1, sten, is_vf, eta, precision=PREC_FP32_CERTIFIED)
    assert np.array_equal(h, hc)
    check_toi(tc, np.where(h == 1, t, -1.0))
