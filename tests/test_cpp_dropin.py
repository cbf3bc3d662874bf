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
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", LIBDIR, "-lmclccd_b200", f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def test_dropin_header_compiles_and_links(tmp_path):
    assert os.path.exists(build_demo(tmp_path))


@pytest.mark.gpu
def test_dropin_hooks_match_oracle(tmp_path):
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
    subprocess.run([exe, str(scene), str(out)], check=True)
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
