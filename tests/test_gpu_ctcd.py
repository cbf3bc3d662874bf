"""One-sided VF narrow phase (vf_one_sided: CTCD with the wrong-side test).

Checked against the reference's own NarrowPhaseCTCD::query_ccd_vf and
BVHTree with vf_one_sided (oracle/_ref).  The device code follows the
reference's steps except the polynomial root finder (Aberth-Ehrlich here,
Jenkins-Traub there), so toi is compared within TOI_TOL.  Hit/miss and the
chosen time can differ only where interval ends of different polynomials
coincide exactly (closed intervals that touch), because then the last bits of
each root decide the overlap.  Generic scenes have none; the flat slide below
is built to have them: its grid vertices cross edge lines at exactly the same
instant (t = 10/87), and there a touching interval pair makes the reference's
vertex-face test miss and fall back to its vertex-edge test (t = 10/87 - eta /
speed), where this code's vertex-face test overlaps.  Such ties are counted
and bounded per scene."""
import numpy as np
import pytest

from mclccd_b200 import BVHTree, narrow_phase_bulk, scenes
from oracle.ref import DEFAULT_FLAGS, F_ONE_SIDED, F_RECORD_CAND, Reference

pytestmark = pytest.mark.gpu
TOI_TOL = 1e-9        # |toi - toi_ref| for stencils both call hits
MISMATCH_MAX = 2e-4   # hit/miss disagreements per stencil (root-boundary cases)


@pytest.fixture(scope="module")
def ref():
    return Reference()


def compare(hit, toi, rret, rtoi, what):
    rhit = rret == 1
    both = (hit == 1) & rhit
    dis = int(np.count_nonzero((hit == 1) != rhit))
    err = np.abs(toi[both] - rtoi[both])
    print(f"{what}: {len(hit)} stencils, {int(rhit.sum())} ref hits, {int(both.sum())} common, {dis} disagree, "
          f"max |dtoi| {err.max() if len(err) else 0:.2e}, wrong-side-only {int((rret == -1).sum())}")
    assert dis <= MISMATCH_MAX * len(hit) + 1, dis
    assert np.all(err <= TOI_TOL), err.max()
    return dis


def test_closed_form_cases(ref):
    eta = 1e-3
    V0 = np.array([[0.2, 0.2, 0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0],    # falls onto the face from above
                   [0.2, 0.2, -0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0],   # rises from below: wrong side
                   [0.2, 0.2, 0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0],    # moves parallel: no contact
                   [1.0, 1.0, 0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0]],   # falls outside the face
                  float)
    V1 = V0.copy()
    V1[0, 2] = -0.5
    V1[4, 2] = 0.5
    V1[8, 0] += 0.5
    V1[12, 2] = -0.5
    sten = np.arange(16, dtype=np.int32).reshape(4, 4)
    toi, hit = narrow_phase_bulk(V0, V1, sten, np.ones(4, np.uint8), eta, vf_one_sided=True)
    rret, rtoi = ref.ctcd_vf(V0, V1, sten, eta)
    assert list(rret) == [1, -1, 0, 0]
    assert list(hit) == [1, 0, 0, 0]
    assert abs(toi[0] - rtoi[0]) <= 1e-15 and abs(toi[0] - (0.5 - eta)) < 1e-12
    # 2D: a point crossing a segment, both directions
    P0 = np.array([[0.5, 0.5], [0, 0], [1, 0], [0.5, -0.5], [0, 0], [1, 0]], float)
    P1 = P0.copy()
    P1[0, 1] = -0.5
    P1[3, 1] = 0.5
    s2 = np.array([[0, 1, 2, -1], [3, 4, 5, -1]], np.int32)
    toi2, hit2 = narrow_phase_bulk(P0, P1, s2, np.ones(2, np.uint8), eta, vf_one_sided=True)
    r2, t2 = ref.ctcd_vf(P0, P1, s2, eta)
    assert list(hit2) == [int(r == 1) for r in r2]
    assert np.allclose(toi2[hit2 == 1], t2[r2 == 1], rtol=0, atol=1e-15)


def random_vf(rng, n, dim, coplanar=False):
    """n VF stencils: a point near a triangle (edge in 2D), both moving."""
    k = dim + 1
    base = rng.uniform(0, 1, (n, 1, dim))
    face = base + rng.normal(0, 0.1, (n, dim, dim))
    w = rng.dirichlet(np.ones(dim), n)[:, :, None]
    pt = (w * face).sum(1, keepdims=True) + rng.normal(0, 0.03, (n, 1, dim))
    x0 = np.concatenate([pt, face], axis=1)
    x1 = x0 + rng.normal(0, 0.05, (n, k, dim))
    if coplanar:   # everything starts in z = 0 (exact zero coefficients)
        x0[..., -1] = 0.0
    V0 = x0.reshape(-1, dim)
    V1 = x1.reshape(-1, dim)
    sten = np.arange(n * k, dtype=np.int32).reshape(n, k)
    if dim == 2:
        sten = np.concatenate([sten, -np.ones((n, 1), np.int32)], axis=1)
    return V0, V1, sten


@pytest.mark.parametrize("dim,coplanar", [(3, False), (3, True), (2, False)])
def test_bulk_random_against_reference(ref, dim, coplanar):
    rng = np.random.default_rng(11 + dim + 7 * coplanar)
    n = 20000
    V0, V1, sten = random_vf(rng, n, dim, coplanar)
    eta = 1e-3
    toi, hit = narrow_phase_bulk(V0, V1, sten, np.ones(n, np.uint8), eta, vf_one_sided=True)
    rret, rtoi = ref.ctcd_vf(V0, V1, sten, eta)
    assert (rret == 1).sum() > 200
    compare(hit, toi, rret, rtoi, f"bulk {dim}D{' coplanar' if coplanar else ''}")


def tree_hits(dim, V0, V1, F, eta):
    t = BVHTree(dim)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.options.vf_one_sided = True
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    return t.hits()


def canon(sten, is_vf):
    s = sten.copy()
    ee = is_vf == 0
    swap = ee & (np.minimum(s[:, 0], s[:, 1]) > np.minimum(s[:, 2], s[:, 3]))
    s[swap] = s[swap][:, [2, 3, 0, 1]]
    return [(int(v),) + tuple(int(x) for x in r) for r, v in zip(s, is_vf)]


@pytest.mark.parametrize("scene,tie_frac", [("fold", 0.0), ("flat_slide", 2e-3), ("annulus", 0.0)])
def test_tree_one_sided_against_reference(ref, scene, tie_frac):
    V0, V1, F, eta = {
        "fold": lambda: scenes.folded_cloth(40, seed=31),
        "flat_slide": lambda: flat_slide(30),
        "annulus": lambda: crumpled_annulus(200),
    }[scene]()
    dim = V0.shape[1]
    hs, hv, ht = tree_hits(dim, V0, V1, F, eta)
    r = ref.run(V0, V1, F, eta, flags=DEFAULT_FLAGS | F_RECORD_CAND | F_ONE_SIDED)
    got = dict(zip(canon(hs, hv), ht))
    want = dict(zip(canon(r["hit_sten"], r["hit_is_vf"]), r["hit_toi"]))
    # EE stays the bit-exact ACCD: same hit set, and the same toi as the
    # reference's own ACCD on this orientation of each edge pair (EE toi
    # depends on which edge comes first, and the reference's order follows
    # its Kd-tree)
    assert {k for k in got if k[0] == 0} == {k for k in want if k[0] == 0}
    ee = hv == 0
    if ee.any():
        rh, rt = ref.accd(V0, V1, hs[ee], hv[ee], eta)
        assert np.all(rh == 1) and np.array_equal(rt, ht[ee])
    vf_got = {k: v for k, v in got.items() if k[0] == 1}
    vf_want = {k: v for k, v in want.items() if k[0] == 1}
    cand = int((r["cand_is_vf"] == 1).sum())
    common = set(vf_got) & set(vf_want)
    ties = [k for k in set(vf_got) | set(vf_want) if k not in common or abs(vf_got[k] - vf_want[k]) > TOI_TOL]
    err = max((abs(vf_got[k] - vf_want[k]) for k in common if k not in ties), default=0.0)
    print(f"{scene}: {cand} VF candidates, {len(vf_want)} ref VF hits, {len(ties)} tie stencils, "
          f"max |dtoi| otherwise {err:.2e}")
    assert len(vf_want) > 0
    assert len(ties) <= tie_frac * len(vf_want)
    assert err <= TOI_TOL


def crumpled_annulus(ring):
    """A 2D annulus whose vertices move by about the edge length (points
    cross edges both ways), so that one-sided contacts occur."""
    V0, _, F, eta = scenes.annulus_2d(ring, seed=32)
    V1 = V0 + np.random.default_rng(33).normal(0.0, 0.01, V0.shape)
    return V0, V1, F, eta


def flat_slide(n):
    """A flat n x n cloth in z = 0 whose right half slides over the left in
    plane: every start position is exactly coplanar."""
    V0, _, F, eta = scenes.folded_cloth(n)
    V0 = V0.copy()
    V0[:, 2] = 0.0
    V1 = V0.copy()
    right = V0[:, 0] > 0.5
    V1[right, 0] -= 0.3
    V1[right, 2] = 1e-4 * np.sin(37 * V0[right, 1])
    return V0, V1, F, eta


def test_bulk_against_recorded_reference():
    # the device one-sided narrow phase against the reference's recorded
    # results (tests/golden/kat_ctcd.npz), with no reference build needed
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kat_ctcd.npz"))
    eta = float(z["eta"])
    for name in z["names"]:
        sten = z[f"{name}/sten"]
        toi, hit = narrow_phase_bulk(z[f"{name}/V0"], z[f"{name}/V1"], sten, np.ones(len(sten), np.uint8), eta,
                                     vf_one_sided=True)
        compare(hit, toi, z[f"{name}/ret"], z[f"{name}/toi"], f"recorded {name}")
