"""Device functors as filter_pair / narrow_phase (include/mclccd_b200/
device_hooks.cuh): the header compiles with nvcc for sm_100a (CPU), and on
the GPU a filter functor with the library ACCD, and a custom narrow-phase
functor, give exactly the hits the host-side definitions predict."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "device_hooks_main.cu")
LIBDIR = os.path.join(ROOT, "mclccd_b200")


def build(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = str(tmp_path / "device_hooks_main")
    subprocess.run([nvcc, "-std=c++17", "-O2", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), SRC, "-L", LIBDIR, "-lmclccd_b200",
                    f"-Xlinker=-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_device_hooks_header_compiles(tmp_path):
    assert os.path.exists(build(tmp_path))


def read_hits(raw, o, n):
    s = np.frombuffer(raw[o:o + 16 * n], np.int32).reshape(-1, 4); o += 16 * n
    v = np.frombuffer(raw[o:o + n], np.uint8); o += n
    t = np.frombuffer(raw[o:o + 8 * n], np.float64); o += 8 * n
    return {(int(a),) + tuple(map(int, b)): float(c) for b, a, c in zip(s, v, t)}, o


@pytest.mark.gpu
def test_device_hooks_match_host_definitions(tmp_path):
    from mclccd_b200 import BVHTree, scenes
    exe = build(tmp_path)
    V0, V1, F, eta = scenes.folded_cloth(40, seed=22)
    scene = tmp_path / "scene.bin"
    with open(scene, "wb") as f:
        f.write(np.array([len(V0), len(F), 3], np.int32).tobytes())
        f.write(np.array([eta], np.float64).tobytes())
        f.write(V0.tobytes()); f.write(V1.tobytes()); f.write(F.astype(np.int32).tobytes())
    out = tmp_path / "out.bin"
    subprocess.run([exe, str(scene), str(out)], check=True)
    raw = out.read_bytes()
    na, nb = np.frombuffer(raw[:16], np.int64)
    got_a, o = read_hits(raw, 16, int(na))
    got_b, o = read_hits(raw, o, int(nb))

    t = BVHTree(3)
    t.options.box_eta = t.options.vf_ccd_eta = t.options.ee_ccd_eta = eta
    t.update(V0, V1, F)
    t.traverse(V0, V1, F)
    hs, hv, ht = t.hits()
    want_a = {(int(v),) + tuple(map(int, s)): float(x) for s, v, x in zip(hs, hv, ht) if s[0] % 2 == 0}
    assert got_a == want_a and len(want_a) > 100
    cs, cv = t.candidates()
    want_b = {(1,) + tuple(map(int, s)): (int(s[0]) % 5) / 10.0 for s, v in zip(cs, cv) if v}
    assert got_b == want_b
