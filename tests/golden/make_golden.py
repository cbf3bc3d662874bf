"""Regenerates the golden fixtures in this folder from the reference itself.

Runs the reference's own, unmodified BVHTree / NarrowPhase code (the oracle
build in oracle/_ref, made with ``make -C oracle ref`` from the reference
checkout) on seeded scenes and stores what the reference's hooks received:
the candidate stencils (filter_pair), the hits with their toi (append_pair)
and the discrete pairs (append_discrete), together with leaf boxes and the
representative-triangle flags.

EE stencils and discrete pairs are stored canonicalised (the reference's
left/right order comes from its Kd-tree); hit/toi of every candidate is also
stored for the canonical orientation (lower primitive index first), by
calling the reference's NarrowPhaseACCD::query_ccd_* on it directly.

    python tests/golden/make_golden.py          # everything
    python tests/golden/make_golden.py ctcd     # only kat_ctcd.npz (one-sided VF)
    python tests/golden/make_golden.py cfg1     # only cfg1_digests.json (2.1M-triangle cloth)
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mclccd_b200 import scenes  # noqa: E402
from oracle.ref import Port, Reference, canonical_set, sort_rows  # noqa: E402
sys.path.insert(0, os.path.dirname(HERE))


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int64).tobytes()).hexdigest()


def kat_scenes():
    """Small hand-built and seeded scenes: (name, V0, V1, F, eta)."""
    out = []
    # Two triangles approaching head-on along z (VF and EE hits).
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0],
                   [0.1, 0.1, 0.5], [0.9, 0.2, 0.5], [0.2, 0.8, 0.5]], np.float64)
    V1 = V0.copy(); V1[3:, 2] = -0.5
    out.append(("headon", V0, V1, np.array([[0, 1, 2], [3, 4, 5]], np.int32), 1e-3))
    # Parallel edges: the two triangles' x-aligned edges stay parallel (EE denom == 0).
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0.5, -1, 0],
                   [0, 0, 0.3], [1, 0, 0.3], [0.5, 1, 0.3]], np.float64)
    V1 = V0.copy(); V1[3:, 2] = -0.1
    out.append(("parallel", V0, V1, np.array([[0, 1, 2], [3, 4, 5]], np.int32), 1e-3))
    # Shared vertex: a folding fan; shared-vertex stencils must be absent.
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.7, 0.7, 0.2]], np.float64)
    V1 = V0.copy(); V1[3] = [0.2, 0.2, -0.3]
    out.append(("shared", V0, V1, np.array([[0, 1, 2], [0, 1, 3], [1, 2, 3]], np.int32), 1e-3))
    # No relative motion (l_p == 0): overlapping but never a CCD hit.
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 0.0005], [0.8, 0.2, 0.0005], [0.2, 0.6, 0.0005]])
    out.append(("static", V0, V0.copy() + 0.25, np.array([[0, 1, 2], [3, 4, 5]], np.int32), 1e-3))
    # Coplanar overlapping triangles at t=1 (discrete coplanar branch).
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 0.3], [1.2, 0.2, 0.3], [0.2, 1.2, 0.3]])
    V1 = V0.copy(); V1[3:, 2] = 0.0
    out.append(("coplanar", V0, V1, np.array([[0, 1, 2], [3, 4, 5]], np.int32), 1e-3))
    # Degenerate triangle (repeated vertex) sweeping through another: its VF
    # stencils have NaN distance, ACCD reports hit with toi = NaN, and
    # collide() drops them (toi >= 0 gate, BVHTree.cpp:262).
    V0 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.2, 0.2, 0.1], [0.3, 0.25, 0.1]], np.float64)
    V1 = V0.copy(); V1[3:, 2] = -0.1
    out.append(("degenerate", V0, V1, np.array([[0, 1, 2], [3, 4, 4]], np.int32), 1e-3))
    out.append(("fold12", *scenes.folded_cloth(12, seed=5)))
    out.append(("spheres", *scenes.icospheres(3, 2, seed=4)))
    out.append(("annulus48", *scenes.annulus_2d(48, seed=2)))
    # 2D: crossing segments (discrete) and a point sweeping through an edge.
    V0 = np.array([[0, 0], [1, 0], [0.5, 0.5], [0.5, -0.5], [0.2, 0.3], [0.9, 0.3]], np.float64)
    V1 = V0.copy(); V1[4:, 1] = -0.2
    out.append(("segments2d", V0, V1, np.array([[0, 1], [2, 3], [4, 5]], np.int32), 1e-3))
    return out


def reference_record(R: Reference, P: Port, V0, V1, F, eta):
    r = R.run(V0, V1, F, eta)
    p = P.run(V0, V1, F, eta)
    h, t = R.accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
    return dict(
        cand=canonical_set(r["cand_sten"], r["cand_is_vf"]),
        hits=canonical_set(r["hit_sten"], r["hit_is_vf"]),
        discrete=sort_rows(np.sort(r["discrete"], axis=1)),
        leaf_boxes=r["leaf_boxes"], leaf_flags=r["leaf_flags"],
        canon_sten=p["cand_sten"], canon_is_vf=p["cand_is_vf"], canon_hit=h, canon_toi=t,
        ref_hit_sten=r["hit_sten"], ref_hit_is_vf=r["hit_is_vf"], ref_hit_toi=r["hit_toi"],
    )


def main():
    R, P = Reference(), Port()
    arrays = {}
    names = []
    for name, V0, V1, F, eta in kat_scenes():
        rec = reference_record(R, P, V0, V1, F, eta)
        names.append(name)
        arrays[f"{name}/V0"] = V0
        arrays[f"{name}/V1"] = V1
        arrays[f"{name}/F"] = F
        arrays[f"{name}/eta"] = np.array(eta)
        for k, v in rec.items():
            arrays[f"{name}/{k}"] = v
        print(f"{name}: tris={len(F)} cand={len(rec['cand'])} hits={len(rec['hits'])} disc={len(rec['discrete'])}")
    arrays["names"] = np.array(names)
    np.savez_compressed(os.path.join(HERE, "kat_small.npz"), **arrays)

    # Folded cloth 64x64 (4,096 verts / 7,938 tris), thickness 1e-3: digests of
    # the reference's full sets plus a 4,096-stencil sample with hit/toi.
    V0, V1, F, eta = scenes.folded_cloth(64)
    rec = reference_record(R, P, V0, V1, F, eta)
    rng = np.random.default_rng(123)
    idx = np.sort(rng.choice(len(rec["canon_sten"]), 4096, replace=False))
    summary = dict(
        scene="folded_cloth(64, seed=0)", eta=eta,
        input_sha256=hashlib.sha256(V0.tobytes() + V1.tobytes() + F.tobytes()).hexdigest(),
        n_cand=int(len(rec["cand"])), n_cand_vf=int((rec["cand"][:, 0] == 1).sum()),
        n_hits=int(len(rec["hits"])), n_hits_vf=int((rec["hits"][:, 0] == 1).sum()),
        n_discrete=int(len(rec["discrete"])),
        cand_sha256=digest(rec["cand"]), hits_sha256=digest(rec["hits"]),
        discrete_sha256=digest(rec["discrete"]),
        canon_toi_sum=float(np.sum(rec["canon_toi"][rec["canon_hit"] == 1])),
        leaf_boxes_sha256=hashlib.sha256(np.ascontiguousarray(rec["leaf_boxes"]).tobytes()).hexdigest(),
        leaf_flags_sha256=digest(rec["leaf_flags"]),
    )
    with open(os.path.join(HERE, "cfg0_summary.json"), "w") as f:
        json.dump(summary, f, indent=1)
    np.savez_compressed(os.path.join(HERE, "cfg0_sample.npz"), sten=rec["canon_sten"][idx],
                        is_vf=rec["canon_is_vf"][idx], hit=rec["canon_hit"][idx], toi=rec["canon_toi"][idx])
    print(json.dumps(summary, indent=1))


def vf_stencils(rng, n, dim, coplanar=False):
    """n VF stencils: a point near a triangle (an edge in 2D), all moving; with
    coplanar, every start position in z = 0 (exact zero coefficients)."""
    k = dim + 1
    base = rng.uniform(0, 1, (n, 1, dim))
    face = base + rng.normal(0, 0.1, (n, dim, dim))
    w = rng.dirichlet(np.ones(dim), n)[:, :, None]
    pt = (w * face).sum(1, keepdims=True) + rng.normal(0, 0.03, (n, 1, dim))
    x0 = np.concatenate([pt, face], axis=1)
    x1 = x0 + rng.normal(0, 0.05, (n, k, dim))
    if coplanar:
        x0[..., -1] = 0.0
    sten = np.arange(n * k, dtype=np.int32).reshape(n, k)
    if dim == 2:
        sten = np.concatenate([sten, -np.ones((n, 1), np.int32)], axis=1)
    return x0.reshape(-1, dim), x1.reshape(-1, dim), sten


def ctcd_fixture():
    """kat_ctcd.npz: the reference's one-sided VF narrow phase
    (NarrowPhaseCTCD::query_ccd_vf with the wrong-side test) on seeded
    stencils: its return code (1 hit, 0 none, -1 wrong side only) and toi."""
    R = Reference()
    arrays, eta = {}, 1e-3
    for name, dim, coplanar, seed in (("vf3", 3, False, 101), ("vf3_coplanar", 3, True, 102), ("vf2", 2, False, 103)):
        V0, V1, sten = vf_stencils(np.random.default_rng(seed), 1500, dim, coplanar)
        ret, toi = R.ctcd_vf(V0, V1, sten, eta)
        arrays.update({f"{name}/V0": V0, f"{name}/V1": V1, f"{name}/sten": sten, f"{name}/ret": ret,
                       f"{name}/toi": toi})
        print(f"{name}: {int((ret == 1).sum())} hits, {int((ret == -1).sum())} wrong-side only")
    arrays["names"] = np.array(["vf3", "vf3_coplanar", "vf2"])
    arrays["eta"] = np.array(eta)
    np.savez_compressed(os.path.join(HERE, "kat_ctcd.npz"), **arrays)


def cfg1_digests():
    """cfg1_digests.json: the full 2,097,152-triangle wavy cloth (1025 x 1025
    grid, thickness 1e-4) for both V1 draws of the timed step (seed 0, then the
    redraw with seed 1 over the same F, which the device takes through its
    refit-only path).  Per draw, order-independent digests (tests/digest.py)
    of the reference's candidate set (filter_pair), discrete-pair set
    (append_discrete) and hit set (append_pair), and of the hit/toi map in
    the device's orientation: the reference's own NarrowPhaseACCD::query_ccd_*
    called on every candidate in that orientation (the oracle restatement
    supplies the orientation; its candidate and hit sets are checked equal to
    the reference's first)."""
    import time
    from digest import hit_rows, set_digest, set_rows
    R, P = Reference(), Port()
    V0, V1a, F, eta = scenes.wavy_cloth(1025, seed=0)
    V1b = scenes.wavy_redraw(V0, 1)
    out = {"scene": "wavy_cloth(1025, seed=0); draw b = wavy_redraw(V0, 1)", "eta": eta, "tris": int(len(F)),
           "F_sha256": hashlib.sha256(F.tobytes()).hexdigest(),
           "V0_sha256": hashlib.sha256(V0.tobytes()).hexdigest(), "draws": {}}
    for name, V1 in (("a", V1a), ("b", V1b)):
        t0 = time.time()
        r = R.run(V0, V1, F, eta)
        ref_cand = set_digest(set_rows(r["cand_sten"], r["cand_is_vf"]))
        ref_hits = set_digest(set_rows(r["hit_sten"], r["hit_is_vf"]))
        ref_disc = set_digest(np.sort(r["discrete"], axis=1))
        del r
        t1 = time.time()
        p = P.run(V0, V1, F, eta)
        assert set_digest(set_rows(p["cand_sten"], p["cand_is_vf"])) == ref_cand
        assert set_digest(set_rows(p["hit_sten"], p["hit_is_vf"])) == ref_hits
        assert set_digest(np.asarray(p["discrete"])) == ref_disc
        hit, toi = R.accd(V0, V1, p["cand_sten"], p["cand_is_vf"], eta)
        m = (hit == 1) & (toi >= 0)   # collide() delivers only toi >= 0 (BVHTree.cpp:262)
        toi_map = set_digest(hit_rows(p["cand_sten"][m], p["cand_is_vf"][m], toi[m]))
        out["draws"][name] = {
            "V1_sha256": hashlib.sha256(V1.tobytes()).hexdigest(),
            "n_leaf_pairs": int(len(p["leaf_pairs"])),
            "n_vf": int(p["cand_is_vf"].sum()), "n_ee": int(len(p["cand_is_vf"]) - p["cand_is_vf"].sum()),
            "candidates": ref_cand, "hits": ref_hits, "discrete": ref_disc, "hit_toi": toi_map}
        print(f"draw {name}: reference {t1 - t0:.0f} s, oracle + reference ACCD {time.time() - t1:.0f} s: "
              f"{ref_cand[0]} candidates, {ref_hits[0]} hits, {ref_disc[0]} discrete", flush=True)
        del p, hit, toi
    with open(os.path.join(HERE, "cfg1_digests.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if sys.argv[1:] == ["ctcd"]:
        ctcd_fixture()
    elif sys.argv[1:] == ["cfg1"]:
        cfg1_digests()
    else:
        main()
        ctcd_fixture()
        cfg1_digests()
