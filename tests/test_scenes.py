"""The seeded synthetic workloads (mclccd_b200/scenes.py) have the sizes and
construction rules the measurements are quoted on, and are deterministic."""
import math

import numpy as np

from mclccd_b200 import scenes


def test_folded_cloth_64():
    # 64 x 64 grid on the unit square, half x > 0.5 folded by 170 degrees
    # about x = 0.5, z = 0, plus N(0, 0.002) noise; thickness 1e-3
    V0, V1, F, eta = scenes.folded_cloth(64)
    assert V0.shape == V1.shape == (4096, 3) and F.shape == (7938, 3) and F.dtype == np.int32
    assert eta == 1e-3
    assert abs(V0[:, 2].std() - 0.01) < 1e-3
    right = V0[:, 0] > 0.5
    th = math.radians(170.0)
    dx, dz = V0[right, 0] - 0.5, V0[right, 2]
    x = 0.5 + math.cos(th) * dx - math.sin(th) * dz
    assert np.abs(V1[right, 0] - x).max() < 0.02   # the fold, up to the noise
    assert np.abs(V1[~right] - V0[~right]).std() < 0.003


def test_wavy_cloth_1025():
    # 1,025^2 vertices, 2,097,152 triangles, z = 0.05 sin(8 pi x) sin(8 pi y),
    # V1 compressed 30% toward x = 0.5 plus N(0, h/2) noise, h = 1/1024
    V0, V1, F, eta = scenes.wavy_cloth(1025)
    assert V0.shape == (1_050_625, 3) and F.shape == (2_097_152, 3) and eta == 1e-4
    z = 0.05 * np.sin(8 * np.pi * V0[:, 0]) * np.sin(8 * np.pi * V0[:, 1])
    assert np.allclose(V0[:, 2], z, atol=1e-12)
    h = 1.0 / 1024
    shift = V1[:, 0] - (0.5 + 0.7 * (V0[:, 0] - 0.5))
    assert abs(shift.mean()) < 1e-4 and abs(shift.std() - 0.5 * h) < 0.05 * h
    # the second draw of the refit-only step: same F, V1 re-drawn
    V1b = scenes.wavy_redraw(V0, 1)
    assert V1b.shape == V1.shape and not np.array_equal(V1b, V1)
    strip = scenes.wavy_cloth(1025, rows=257)
    assert len(strip[2]) == 2 * 1024 * 256


def test_icospheres_and_stress_stencils():
    V0, V1, F, eta = scenes.icospheres(64, 6)
    assert V0.shape == (64 * 40_962, 3) and F.shape == (64 * 81_920, 3)
    V0s, V1s, sten, is_vf, eta_s = scenes.stress_stencils(100_000)
    assert sten.shape == (100_000, 4) and int(is_vf.sum()) == 50_000


def test_batch_scenes():
    sc = scenes.batch_scenes()
    assert len(sc) == 512
    kinds = [k for k, _ in sc]
    assert kinds.count("cloth") == 384 and kinds.count("annulus") == 128
    sides = [int(round(math.sqrt(len(s[0])))) for k, s in sc if k == "cloth"]
    assert min(sides) >= 16 and max(sides) <= 384
    assert all(s[0].shape[1] == 2 and s[2].shape[1] == 2 for k, s in sc if k == "annulus")


def test_adjoint_fold_and_determinism():
    V0, V1, F, eta = scenes.folded_cloth(256)
    assert F.shape == (130_050, 3)
    a = scenes.folded_cloth(48, seed=7)
    b = scenes.folded_cloth(48, seed=7)
    assert all(np.array_equal(x, y) for x, y in zip(a[:3], b[:3]))
    c = scenes.annulus_2d(300, seed=3)
    d = scenes.annulus_2d(300, seed=3)
    assert all(np.array_equal(x, y) for x, y in zip(c[:3], d[:3]))
