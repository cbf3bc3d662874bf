"""The library's ACCD and distance code, built for the host (tests/cpp/accd_host.cu
includes mclccd_b200/csrc/geom.cuh unchanged), against the oracle restatement
(oracle/port.c, pinned to the reference by tests/test_oracle.py), bit for bit.

The device kernels run these same functions; what this checks on the CPU is
the arithmetic itself: each case of point_on_triangle / edge_to_edge with
its quotient selected before one division, l_p from the larger squared norm,
and the fast ACCD head (no threshold, no zero step divided out) resumed into
the reference loop.  Inputs: every case of the distance routines, degenerate
and non-finite stencils, and the candidate stencils of a folded cloth."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from mclccd_b200 import scenes
from oracle.ref import Port, _p

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "accd_host.cu")


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("accd_host") / "libaccd_host.so")
    subprocess.run(["nvcc", "-std=c++17", "-O2", "-x", "cu", "--shared", "-Xcompiler", "-fPIC,-ffp-contract=off",
                    "-Wno-deprecated-gpu-targets", "-o", so, SRC], check=True)
    L = C.CDLL(so)
    dp, ip, ucp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_ubyte)
    L.host_accd.argtypes = [C.c_int, C.c_int, dp, dp, ip, ucp, C.c_longlong, C.c_double, C.c_double, ip, dp, ip]
    L.host_distance.argtypes = [C.c_int, dp, ucp, C.c_longlong, dp]
    return L


@pytest.fixture(scope="module")
def port():
    P = Port()
    dp = C.POINTER(C.c_double)
    for f in ("port_vf_distance3", "port_ee_distance3"):
        getattr(P.L, f).argtypes = [dp, dp, dp, dp]
        getattr(P.L, f).restype = C.c_double
    P.L.port_vf_distance2.argtypes = [dp, dp, dp]
    P.L.port_vf_distance2.restype = C.c_double
    return P


def same_bits(a, b):
    a = np.ascontiguousarray(a, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    return np.array_equal(a.view(np.int64), b.view(np.int64)) or np.array_equal(a, b, equal_nan=True)


def host_accd(L, dim, form, V0, V1, sten, is_vf, vf_eta, ee_eta):
    V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
    s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4); v = np.ascontiguousarray(is_vf, np.uint8)
    n = len(s)
    hit = np.empty(n, np.int32); toi = np.empty(n); it = np.empty(n, np.int32)
    L.host_accd(dim, form, _p(V0, C.c_double), _p(V1, C.c_double), _p(s, C.c_int), _p(v, C.c_ubyte), n, vf_eta,
                ee_eta, _p(hit, C.c_int), _p(toi, C.c_double), _p(it, C.c_int))
    return hit, toi, it


def random_stencils(rng, n, dim, scale=1.0):
    """n stencils of dim + 1 vertices each, spread so that every case of the
    distance routines occurs, with a mix of slow and fast motion."""
    k = dim + 1
    x0 = rng.normal(0, scale, (n, k, dim))
    x0[n // 2:, 1:] = x0[n // 2:, :1] + rng.normal(0, 0.05 * scale, (n - n // 2, k - 1, dim))   # close pairs
    x1 = x0 + rng.normal(0, 1.0, (n, 1, 1)) * rng.normal(0, 0.1 * scale, (n, k, dim))
    return x0.reshape(-1, dim), x1.reshape(-1, dim), np.arange(n * k, dtype=np.int32).reshape(n, k)


def degenerate(rng, dim):
    """Repeated vertices, collinear triangles, parallel and zero-length edges,
    no motion, exact zeros, -0.0 coordinates and non-finite coordinates."""
    k = dim + 1
    out0, out1 = [], []
    for _ in range(400):
        x0 = rng.normal(0, 1, (k, dim))
        kind = rng.integers(0, 9)
        if kind == 0:
            x0[2] = x0[1]                                  # repeated vertex
        elif kind == 1 and dim == 3:
            x0[3] = x0[1] + 2.0 * (x0[2] - x0[1])          # collinear triangle / edge
        elif kind == 2 and dim == 3:
            x0[3] = x0[2] + (x0[1] - x0[0])                # parallel edges
        elif kind == 3:
            x0 = np.round(x0 * 4) / 4                       # exact grid values, exact zeros
        elif kind == 4:
            x0[:, -1] = -0.0                                # -0.0 coordinates
        x1 = x0.copy() if kind == 5 else x0 + rng.normal(0, 0.2, (k, dim))
        if kind == 6:
            x1 = x0 + 0.25                                 # rigid translation: no relative motion
        if kind == 7:
            x1[0, 0] = np.inf
        if kind == 8:
            x0[1, 1] = np.nan
        out0.append(x0); out1.append(x1)
    n = len(out0)
    return (np.concatenate(out0), np.concatenate(out1), np.arange(n * k, dtype=np.int32).reshape(n, k))


def pad4(sten):
    if sten.shape[1] == 4:
        return sten
    return np.concatenate([sten, -np.ones((len(sten), 4 - sten.shape[1]), np.int32)], axis=1)


@pytest.mark.parametrize("dim", [3, 2])
def test_distances_match_oracle(host, port, dim):
    rng = np.random.default_rng(7 + dim)
    V0, _, sten = random_stencils(rng, 20000, dim)
    D0, _, dsten = degenerate(rng, dim)
    X = np.concatenate([V0, D0]).reshape(-1, (dim + 1) * dim)
    n = len(X)
    X4 = np.zeros((n, 4 * dim))
    X4[:, :(dim + 1) * dim] = X
    kinds = [1] if dim == 2 else [1, 0]
    for vf in kinds:
        is_vf = np.full(n, vf, np.uint8)
        got = np.empty(n)
        host.host_distance(dim, _p(np.ascontiguousarray(X4), C.c_double), _p(is_vf, C.c_ubyte), n,
                           _p(got, C.c_double))
        want = np.empty(n)
        for i in range(n):
            pts = [np.ascontiguousarray(X[i, j * dim:(j + 1) * dim]) for j in range(dim + 1)]
            args = [_p(q, C.c_double) for q in pts]
            if dim == 2:
                want[i] = port.L.port_vf_distance2(*args)
            elif vf:
                want[i] = port.L.port_vf_distance3(*args)
            else:
                want[i] = port.L.port_ee_distance3(*args)
        assert same_bits(got, want)


@pytest.mark.parametrize("dim", [3, 2])
def test_accd_matches_oracle_random_and_degenerate(host, port, dim):
    rng = np.random.default_rng(100 + dim)
    parts = [random_stencils(rng, 20000, dim, 1.0), random_stencils(rng, 20000, dim, 1e-3), degenerate(rng, dim)]
    for V0, V1, sten in parts:
        sten = pad4(sten)
        n = len(sten)
        is_vf = (rng.random(n) < 0.5).astype(np.uint8) if dim == 3 else np.ones(n, np.uint8)
        for eta in (1e-3, 1e-6, 0.0):
            ph, pt = port.accd(V0, V1, sten, is_vf, eta, eta)
            for form in (0, 1):
                h, t, _ = host_accd(host, dim, form, V0, V1, sten, is_vf, eta, eta)
                assert np.array_equal(h, ph), (form, eta)
                m = ph == 1
                assert same_bits(t[m], pt[m]), (form, eta)


def test_accd_matches_oracle_on_fold_candidates(host, port):
    V0, V1, F, eta = scenes.folded_cloth(40, seed=3)
    p = port.run(V0, V1, F, eta)
    sten, is_vf = p["cand_sten"], p["cand_is_vf"]
    ph, pt = port.accd(V0, V1, sten, is_vf, eta, eta)
    assert len(sten) > 100000
    for form in (0, 1):
        h, t, it = host_accd(host, 3, form, V0, V1, sten, is_vf, eta, eta)
        assert np.array_equal(h, ph)
        assert same_bits(t[ph == 1], pt[ph == 1])
    # the fast head decides most stencils after one distance or resumes them
    assert np.mean(it <= 2) > 0.9
