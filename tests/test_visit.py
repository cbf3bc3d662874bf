"""Device visitor traversal (include/mclccd_b200/visit.cuh, the form of the
reference's BVHTree::traverse(BVHTraverse*)): it compiles for sm_100a (CPU),
and the reference example's point-in-triangle query over a 2D mesh finds
exactly the (point, triangle) pairs a brute-force test finds (GPU)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "visit_main.cu")
LIBDIR = os.path.join(ROOT, "mclccd_b200")


def build(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "visit_main")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR, "-lmclccd_b200",
                    f"-Xlinker=-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_visit_header_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


def brute_force(V, F, Q):
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    v0, v1 = b - a, c - a
    d00 = (v0 * v0).sum(1); d01 = (v0 * v1).sum(1); d11 = (v1 * v1).sum(1)
    out = set()
    for q, p in enumerate(Q):
        v2 = p - a
        d20 = (v2 * v0).sum(1); d21 = (v2 * v1).sum(1)
        inv = 1.0 / (d00 * d11 - d01 * d01)
        r1 = (d11 * d20 - d01 * d21) * inv; r2 = (d00 * d21 - d01 * d20) * inv; r0 = 1.0 - r1 - r2
        for t in np.flatnonzero((r0 >= 0) & (r1 >= 0) & (r2 >= 0)):
            out.add((q, int(t)))
    return out


@pytest.mark.gpu
def test_point_in_triangle_matches_brute_force(tmp_path):
    from mclccd_b200 import scenes
    exe = build(tmp_path)
    V, F = scenes.grid(48)
    V = V[:, :2] + np.random.default_rng(3).normal(0, 2e-3, (len(V), 2))
    Q = np.random.default_rng(4).uniform(-0.05, 1.05, (3000, 2))
    scene = tmp_path / "mesh.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V), len(F), len(Q)], np.int32).tobytes())
        f.write(np.ascontiguousarray(V).tobytes()); f.write(F.astype(np.int32).tobytes())
        f.write(np.ascontiguousarray(Q).tobytes())
    out = tmp_path / "pairs.bin"
    subprocess.run([exe, str(scene), str(out)], check=True)
    raw = out.read_bytes()
    n = int(np.frombuffer(raw[:8], np.int64)[0])
    got = {tuple(map(int, p)) for p in np.frombuffer(raw[8:8 + 8 * n], np.int32).reshape(-1, 2)}
    want = brute_force(V, F, Q)
    assert len(want) > 2000 and got == want
