"""CPU tests of the oracle: the C restatement (oracle/port.c) against the
golden fixtures recorded from the reference's own code, and -- where the
reference build (oracle/_ref) is present -- against the reference directly."""
import hashlib
import json
import os

import numpy as np
import pytest

from mclccd_b200 import scenes
from oracle.ref import REF_SO, Port, Reference, canonical_set, sort_rows

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def port():
    return Port()


@pytest.fixture(scope="module")
def kats():
    z = np.load(os.path.join(GOLD, "kat_small.npz"))
    return {name: {k.split("/", 1)[1]: z[k] for k in z.files if k.startswith(name + "/")} for name in z["names"]}


def _flags_bits(pf):
    return np.stack([(pf >> j) & 1 for j in range(7)], axis=1)


def test_kat_scenes_present(kats):
    assert {"headon", "parallel", "shared", "static", "coplanar", "degenerate", "fold12", "spheres", "annulus48",
            "segments2d"} <= set(kats)


@pytest.mark.parametrize("name", ["headon", "parallel", "shared", "static", "coplanar", "degenerate", "fold12", "spheres",
                                  "annulus48", "segments2d"])
def test_port_matches_reference_golden(port, kats, name):
    g = kats[name]
    eta = float(g["eta"])
    p = port.run(g["V0"], g["V1"], g["F"], eta)
    assert np.array_equal(p["leaf_boxes"], g["leaf_boxes"])                 # bit-exact boxes
    assert np.array_equal(_flags_bits(p["leaf_flags"]), g["leaf_flags"])   # reptri + active
    assert np.array_equal(canonical_set(p["cand_sten"], p["cand_is_vf"]), g["cand"])
    assert np.array_equal(sort_rows(p["discrete"]), g["discrete"])
    assert np.array_equal(canonical_set(p["hit_sten"], p["hit_is_vf"]), g["hits"])
    hit, toi = port.accd(g["V0"], g["V1"], g["canon_sten"], g["canon_is_vf"], eta)
    assert np.array_equal(hit, g["canon_hit"])
    assert np.array_equal(toi, g["canon_toi"], equal_nan=True)              # bit-exact toi (NaN: degenerate)


def test_shared_vertex_and_static_semantics(kats):
    # Shared-vertex stencils never appear (BVHTree.cpp:333,356,384-386).
    g = kats["shared"]
    F = g["F"]
    for row in g["cand"]:
        is_vf, s = row[0], row[1:]
        if is_vf:
            assert s[0] not in s[1:]
        else:
            assert len({s[0], s[1]} & {s[2], s[3]}) == 0
    # No relative motion -> l_p == 0 -> never a CCD hit (NarrowPhase.cpp:671-673).
    assert len(kats["static"]["hits"]) == 0 and len(kats["static"]["cand"]) > 0
    assert F.shape == (3, 3)


def test_port_matches_cfg0_summary(port):
    with open(os.path.join(GOLD, "cfg0_summary.json")) as f:
        s = json.load(f)
    V0, V1, F, eta = scenes.folded_cloth(64)
    assert hashlib.sha256(V0.tobytes() + V1.tobytes() + F.tobytes()).hexdigest() == s["input_sha256"]
    p = port.run(V0, V1, F, eta)
    dig = lambda a: hashlib.sha256(np.ascontiguousarray(a, dtype=np.int64).tobytes()).hexdigest()
    cand = canonical_set(p["cand_sten"], p["cand_is_vf"])
    assert len(cand) == s["n_cand"] == 2479971
    assert dig(cand) == s["cand_sha256"]
    assert dig(canonical_set(p["hit_sten"], p["hit_is_vf"])) == s["hits_sha256"]
    assert dig(sort_rows(p["discrete"])) == s["discrete_sha256"]
    assert hashlib.sha256(np.ascontiguousarray(p["leaf_boxes"]).tobytes()).hexdigest() == s["leaf_boxes_sha256"]
    assert float(np.sum(p["hit_toi"])) == pytest.approx(s["canon_toi_sum"], rel=1e-12)
    z = np.load(os.path.join(GOLD, "cfg0_sample.npz"))
    hit, toi = port.accd(V0, V1, z["sten"], z["is_vf"], eta)
    assert np.array_equal(hit, z["hit"]) and np.array_equal(toi, z["toi"])


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", [11, 12])
def test_port_matches_reference_live(port, seed):
    R = Reference()
    for V0, V1, F, eta in (scenes.folded_cloth(20, seed=seed), scenes.annulus_2d(96, seed=seed),
                           scenes.icospheres(4, 2, seed=seed)):
        r = R.run(V0, V1, F, eta)
        p = port.run(V0, V1, F, eta)
        assert np.array_equal(r["leaf_boxes"], p["leaf_boxes"])
        assert np.array_equal(canonical_set(r["cand_sten"], r["cand_is_vf"]),
                              canonical_set(p["cand_sten"], p["cand_is_vf"]))
        assert np.array_equal(sort_rows(np.sort(r["discrete"], 1)), sort_rows(p["discrete"]))
        h, t = R.accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
        hp, tp = port.accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
        assert np.array_equal(h, hp) and np.array_equal(t, tp)


def test_port_edge_cases(port):
    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64)
    one = port.run(V, V + 0.1, np.array([[0, 1, 2]], np.int32), 1e-3)       # np == 1: nothing
    assert len(one["cand_sten"]) == 0 and len(one["discrete"]) == 0
    empty = port.run(V, V, np.zeros((0, 3), np.int32), 1e-3)                # np == 0
    assert len(empty["cand_sten"]) == 0
    # Degenerate triangle (repeated vertex) still gets a box and stencils.
    V2 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 0.1], [0.3, 0.2, 0.1]], np.float64)
    F2 = np.array([[0, 1, 2], [3, 4, 4]], np.int32)
    V2b = V2.copy()
    V2b[3:, 2] = -0.1                                                     # sweeps through triangle 0
    d = port.run(V2, V2b, F2, 1e-3)
    assert len(d["cand_sten"]) > 0 and len(d["hit_sten"]) > 0


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")
def test_reference_ctcd_one_sided_cases():
    # the reference's own one-sided VF narrow phase (the checker of the device
    # CTCD): a fall onto the face from above hits when the gap reaches eta, a
    # rise from below is a wrong-side contact, parallel or outside motion misses
    R = Reference()
    eta = 1e-3
    tri = [[0, 0, 0], [1, 0, 0], [0, 1, 0]]
    V0 = np.array([[0.2, 0.2, 0.5]] + tri + [[0.2, 0.2, -0.5]] + tri + [[0.2, 0.2, 0.5]] + tri + [[1, 1, 0.5]] + tri,
                  float)
    V1 = V0.copy()
    V1[0, 2], V1[4, 2], V1[8, 0], V1[12, 2] = -0.5, 0.5, 0.7, -0.5
    ret, toi = R.ctcd_vf(V0, V1, np.arange(16, dtype=np.int32).reshape(4, 4), eta)
    assert list(ret) == [1, -1, 0, 0]
    assert abs(toi[0] - (0.5 - eta)) < 1e-12


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")
def test_reference_rpoly_matches_eigenvalue_roots():
    # the reference's Jenkins-Traub root finder (the one the device CTCD's
    # Aberth iteration stands in for) agrees with companion-matrix eigenvalues
    # on well-separated roots, degrees 3-6
    R = Reference()
    rng = np.random.default_rng(5)
    for deg in range(3, 7):
        for _ in range(50):
            pairs = deg // 3   # complex-conjugate pairs, the rest real
            z = rng.uniform(-2, 2, pairs) + 1j * rng.uniform(0.2, 1.0, pairs)
            roots = np.concatenate([rng.uniform(-2, 2, deg - 2 * pairs), z, np.conj(z)])
            op = np.real(np.poly(roots))
            got = R.rpoly(op)
            want = np.roots(op)
            assert len(got) == deg
            assert all(np.min(np.abs(want - g)) < 1e-8 for g in got), (got, want)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference oracle not built")
def test_reference_reproduces_ctcd_fixture():
    # kat_ctcd.npz holds the reference's one-sided VF results; the oracle
    # build reproduces them bit for bit
    z = np.load(os.path.join(GOLD, "kat_ctcd.npz"))
    R = Reference()
    for name in z["names"]:
        ret, toi = R.ctcd_vf(z[f"{name}/V0"], z[f"{name}/V1"], z[f"{name}/sten"], float(z["eta"]))
        assert np.array_equal(ret, z[f"{name}/ret"]) and np.array_equal(toi, z[f"{name}/toi"]), name
