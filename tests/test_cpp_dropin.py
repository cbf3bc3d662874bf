"""The C++ drop-in header (include/mclccd_b200/BVHTree.hpp): it compiles and
links against the library (CPU), and driven like reference code it delivers
the same hooks as the oracle (GPU)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "dropin_main.cpp")
LIBDIR = os.path.join(ROOT, "mclccd_b200")


def build_demo(tmp_path):
    exe = str(tmp_path / "dropin_main")
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lmclccd_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_demo(tmp_path))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["threaded", "serial"])
def test_dropin_hooks_match_oracle(tmp_path, mode):
    # threaded: append_pair on all host threads (the reference's default);
    # serial: options.threaded = false, on the calling thread
    from mclccd_b200 import scenes
    from oracle.ref import Port, canonical_set, sort_rows
    exe = build_demo(tmp_path)
    V0, V1, F, eta = scenes.folded_cloth(40, seed=21)
    scene = tmp_path / "scene.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V0), len(F), 3], np.int32).tobytes())
        f.write(np.array([eta], np.float64).tobytes())
        f.write(V0.tobytes()); f.write(V1.tobytes()); f.write(F.astype(np.int32).tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([exe, str(scene), str(out)] + (["serial"] if mode == "serial" else []), check=True)
    raw = out.read_bytes()
    nh, nd = np.frombuffer(raw[:16], np.int64)
    o = 16
    hs = np.frombuffer(raw[o:o + 16 * nh], np.int32).reshape(-1, 4); o += 16 * nh
    hv = np.frombuffer(raw[o:o + nh], np.uint8); o += nh
    ht = np.frombuffer(raw[o:o + 8 * nh], np.float64); o += 8 * nh
    ds = np.frombuffer(raw[o:o + 8 * nd], np.int32).reshape(-1, 2)
    p = Port().run(V0, V1, F, eta)
    assert np.array_equal(canonical_set(hs, hv), canonical_set(p["hit_sten"], p["hit_is_vf"]))
    got = {(int(v),) + tuple(map(int, s)): float(t) for s, v, t in zip(hs, hv, ht)}
    want = {(int(v),) + tuple(map(int, s)): float(t) for s, v, t in zip(p["hit_sten"], p["hit_is_vf"], p["hit_toi"])}
    assert got == want
    assert np.array_equal(sort_rows(ds), sort_rows(p["discrete"]))


@pytest.mark.gpu
def test_dropin_hook_exception_reaches_the_caller(tmp_path):
    # an exception thrown by append_pair on a dispatch thread is rethrown by
    # traverse() on the calling thread
    from mclccd_b200 import scenes
    exe = build_demo(tmp_path)
    V0, V1, F, eta = scenes.folded_cloth(40, seed=21)
    scene = tmp_path / "scene.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V0), len(F), 3], np.int32).tobytes())
        f.write(np.array([eta], np.float64).tobytes())
        f.write(V0.tobytes()); f.write(V1.tobytes()); f.write(F.astype(np.int32).tobytes())
    r = subprocess.run([exe, str(scene), str(tmp_path / "out.bin"), "throw"], capture_output=True, text=True)
    assert r.returncode == 3 and "hook failed" in r.stderr, (r.returncode, r.stderr)


@pytest.mark.gpu
def test_dropin_float_tree(tmp_path):
    """mcl::BVHTree<float, 3>: the FP64 results for the float coordinates
    (same sets; toi rounded down to float), compared with the reference's
    own float instantiation run on the same float coordinates."""
    from mclccd_b200 import scenes
    from oracle.ref import DEFAULT_FLAGS, F_FLOAT, F_RECORD_CAND, Port, Reference, canonical_set, sort_rows
    exe = build_demo(tmp_path)
    V0, V1, F, eta = scenes.folded_cloth(40, seed=22)
    scene = tmp_path / "scene.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V0), len(F), 3], np.int32).tobytes())
        f.write(np.array([eta], np.float64).tobytes())
        f.write(V0.tobytes()); f.write(V1.tobytes()); f.write(F.astype(np.int32).tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([exe, str(scene), str(out), "float"], check=True)
    raw = out.read_bytes()
    nh, nd = np.frombuffer(raw[:16], np.int64)
    o = 16
    hs = np.frombuffer(raw[o:o + 16 * nh], np.int32).reshape(-1, 4); o += 16 * nh
    hv = np.frombuffer(raw[o:o + nh], np.uint8); o += nh
    ht = np.frombuffer(raw[o:o + 8 * nh], np.float64); o += 8 * nh
    ds = np.frombuffer(raw[o:o + 8 * nd], np.int32).reshape(-1, 2)
    # the FP64 port on the float coordinates (and float eta), widened exactly
    W0, W1 = V0.astype(np.float32).astype(np.float64), V1.astype(np.float32).astype(np.float64)
    feta = float(np.float32(eta))
    p = Port().run(W0, W1, F, feta)
    assert np.array_equal(canonical_set(hs, hv), canonical_set(p["hit_sten"], p["hit_is_vf"]))
    assert np.array_equal(sort_rows(ds), sort_rows(p["discrete"]))
    want = {(int(v),) + tuple(map(int, s)): float(t) for s, v, t in zip(p["hit_sten"], p["hit_is_vf"], p["hit_toi"])}
    got = {(int(v),) + tuple(map(int, s)): float(t) for s, v, t in zip(hs, hv, ht)}
    for k, t in got.items():   # FP64 toi rounded down to float
        w = want[k]
        assert t <= w and float(np.float32(t)) == t
        assert float(np.nextafter(np.float32(t), np.float32(np.inf))) > w   # compared in float64
    # the reference's BVHTree<float, 3> (float arithmetic throughout)
    r = Reference().run(V0, V1, F, eta, flags=DEFAULT_FLAGS | F_RECORD_CAND | F_FLOAT)
    same = np.array_equal(canonical_set(hs, hv), canonical_set(r["hit_sten"], r["hit_is_vf"]))
    def key(s, v):   # EE edge pairs in canonical order (the reference's follows its Kd-tree)
        s = tuple(map(int, s))
        if not v and min(s[0], s[1]) > min(s[2], s[3]):
            s = s[2:] + s[:2]
        return (int(v),) + s
    rt = {key(s, v): float(t) for s, v, t in zip(r["hit_sten"], r["hit_is_vf"], r["hit_toi"])}
    got = {key(s, v): t for (v, *s), t in got.items()}
    common = set(rt) & set(got)
    rel = max(abs(got[k] - rt[k]) / max(rt[k], 1e-30) for k in common)
    print(f"float tree: {len(got)} hits; reference float instantiation {len(rt)} hits, same set {same}, "
          f"max rel toi difference {rel:.2e}")
    assert len(common) >= 0.999 * max(len(rt), len(got))


def build_cpp(tmp_path, name):
    exe = str(tmp_path / name)
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-L", LIBDIR, "-lmclccd_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_visitor_program_compiles(tmp_path):
    assert os.path.exists(build_cpp(tmp_path, "traverser_main"))


def point_in_triangle_brute(V, F, Q):
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    v0, v1 = b - a, c - a
    d00, d01, d11 = (v0 * v0).sum(1), (v0 * v1).sum(1), (v1 * v1).sum(1)
    out = []
    for p in Q:
        v2 = p - a
        d20, d21 = (v2 * v0).sum(1), (v2 * v1).sum(1)
        inv = 1.0 / (d00 * d11 - d01 * d01)
        s, t = (d11 * d20 - d01 * d21) * inv, (d00 * d21 - d01 * d20) * inv
        out.append(sorted(np.flatnonzero((s >= 0) & (t >= 0) & (1.0 - s - t >= 0)).tolist()))
    return out


@pytest.mark.gpu
def test_visitor_point_in_triangle_matches_brute_force(tmp_path):
    # BVHTree<double, 2>::traverse(BVHTraverse *) driven like the reference's
    # examples/traverser.cpp: every query finds exactly the triangles whose
    # barycentric test passes (the visitor descends into volumes containing
    # the point and checks each leaf it reaches)
    from mclccd_b200 import scenes
    exe = build_cpp(tmp_path, "traverser_main")
    V3, _, F, _ = scenes.folded_cloth(48, seed=3)
    rng = np.random.default_rng(5)
    V = np.ascontiguousarray(V3[:, :2] + rng.normal(0, 2e-3, (len(V3), 2)))
    Q = np.concatenate([rng.uniform(-0.05, 1.05, (400, 2)), V[rng.choice(len(V), 50)]])   # vertices: ties
    scene = tmp_path / "scene.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V), len(F), len(Q)], np.int32).tobytes())
        f.write(V.tobytes()); f.write(F.astype(np.int32).tobytes()); f.write(Q.tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([exe, str(scene), str(out)], check=True)
    raw = np.frombuffer(out.read_bytes(), np.int32)
    got, i = [], 0
    for _ in range(len(Q)):
        n = int(raw[i]); got.append(sorted(raw[i + 1:i + 1 + n].tolist())); i += 1 + n
    want = point_in_triangle_brute(V, F.astype(np.int64), Q)
    assert got == want
    assert sum(len(w) for w in want) > 300
