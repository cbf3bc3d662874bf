"""CPU checks of the FP64 adjoint reference (oracle/adjoint_ref.c): its
implicit-function gradient against its own central finite differences and a
closed-form case, so the checker of the device adjoint is itself pinned."""
import numpy as np

from oracle.ref import Port


def test_head_on_closed_form():
    eta = 1e-3
    v0 = np.array([[0.2, 0.2, 0.5], [0, 0, 0], [1, 0, 0], [0, 1, 0]], float)
    v1 = v0.copy()
    v1[0, 2] = -0.5
    ts, st, rows = Port().vjp_rows(v0, v1, np.array([[0, 1, 2, 3]]), np.ones(1, np.uint8), np.array([0.4]), eta)
    assert st[0] == 0 and abs(ts[0] - (0.5 - eta)) < 1e-15
    r = rows[0].reshape(2, 4, 3)
    # t* = (z0 - eta) / (z0 - z1): d/dz0 = (eta - z1) / (z0 - z1)^2, d/dz1 = (z0 - eta) / (z0 - z1)^2
    assert abs(r[0, 0, 2] - (eta + 0.5)) < 1e-12
    assert abs(r[1, 0, 2] - (0.5 - eta)) < 1e-12
    # the triangle's vertices carry the opposite share by barycentric weight
    assert abs(r[0, 1:, 2].sum() + (eta + 0.5)) < 1e-12


def test_implicit_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    port = Port()
    eta = 1e-3
    checked = 0
    for trial in range(1200):
        is_vf = trial % 2
        v0 = rng.random((4, 3))
        if is_vf:   # point above a triangle, moving towards it
            v0[0] = v0[1:].mean(0) + rng.normal(0, 0.1, 3) + np.array([0, 0, 0.3])
        v1 = v0 + rng.normal(0, 0.3, (4, 3))
        out = port.vjp_rows(v0, v1, np.array([[0, 1, 2, 3]]), np.array([is_vf], np.uint8), np.array([1e-9]), eta)
        if out[1][0] != 0:
            continue
        st, fd = port.vjp_fd(v0, v1, is_vf, eta, 1e-9, 1e-7)
        if st != 0:
            continue
        rel = np.linalg.norm(out[2][0] - fd) / np.linalg.norm(fd)
        assert rel <= 1e-5, (trial, rel)
        checked += 1
    assert checked > 60
