"""Seeded synthetic CCD scenes (the benchmark workloads; no dataset involved).

Every generator returns plain numpy arrays: ``V0``/``V1`` float64 row-major
``nv x dim`` (positions at t=0 and t=1), ``F`` int32 ``np x dim`` (triangles in
3D, edges in 2D) and the thickness ``eta`` used for box padding and both ACCD
gaps.  The same seed always gives the same bytes.

Workloads
---------
* ``folded_cloth``  : n x n grid on the unit square, two triangles per quad;
  V0 gets z = z_sigma * N(0,1); V1 rotates the half x > 0.5 by ``fold_deg``
  about the line x = 0.5 (z = 0) in the xz-plane, then adds N(0, noise) to
  every coordinate.  n=64 -> 4,096 verts / 7,938 tris, thickness 1e-3.
* ``wavy_cloth``    : 1025 x 1025 grid (2,097,152 tris), h = 1/1024;
  V0 z = 0.05 sin(8 pi x) sin(8 pi y); V1 compresses x by 30% toward 0.5 and
  adds N(0, 0.5 h) per coordinate; thickness 1e-4.  ``redraw`` gives the
  second step's V1 (same F, new seed) for the refit-only update.
* ``icospheres``    : k icospheres (subdivision s) with radii U[0.05, 0.1],
  centres U[0,1]^3, per-sphere translation N(0, 0.05) and per-vertex
  N(0, 1e-3) noise.
* ``annulus_2d``    : triangulated annulus (r_in 0.3, r_out 0.5) as its unique
  edge list (2D edge mesh), random rigid motion plus N(0, 1e-3) noise.
"""
from __future__ import annotations

import math

import numpy as np


def grid(n: int, h: float | None = None):
    """n x n vertex grid on [0, (n-1) h]^2 (unit square by default), z = 0."""
    if h is None:
        h = 1.0 / (n - 1)
    xs = np.arange(n, dtype=np.float64) * h
    X, Y = np.meshgrid(xs, xs, indexing="xy")
    V = np.stack([X.ravel(), Y.ravel(), np.zeros(n * n)], axis=1)
    j, i = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    a = (j * n + i).ravel()
    b = a + 1
    c = a + n
    d = c + 1
    F = np.empty((2 * len(a), 3), dtype=np.int32)
    F[0::2] = np.stack([a, b, d], axis=1)
    F[1::2] = np.stack([a, d, c], axis=1)
    return V, F


def folded_cloth(n: int = 64, seed: int = 0, fold_deg: float = 170.0,
                 z_sigma: float = 0.01, noise: float = 0.002, eta: float = 1e-3):
    rng = np.random.default_rng(seed)
    V, F = grid(n)
    V0 = V.copy()
    V0[:, 2] = z_sigma * rng.standard_normal(len(V))
    V1 = V0.copy()
    m = V1[:, 0] > 0.5
    th = math.radians(fold_deg)
    dx = V1[m, 0] - 0.5
    dz = V1[m, 2]
    V1[m, 0] = 0.5 + math.cos(th) * dx - math.sin(th) * dz
    V1[m, 2] = math.sin(th) * dx + math.cos(th) * dz
    V1 += rng.normal(0.0, noise, V1.shape)
    return np.ascontiguousarray(V0), np.ascontiguousarray(V1), F, eta


def wavy_cloth(n: int = 1025, seed: int = 0, eta: float = 1e-4, rows: int | None = None):
    """``rows`` < n keeps only the first ``rows`` grid rows (a strip of the
    same cloth: same spacing, same motion field)."""
    h = 1.0 / (n - 1) if n == 1025 else 1.0 / 1024
    V, F = grid(n, h)
    if rows is not None and rows < n:
        V = V[: rows * n]
        F = F[: 2 * (n - 1) * (rows - 1)]
    V0 = V.copy()
    V0[:, 2] = 0.05 * np.sin(8 * np.pi * V[:, 0]) * np.sin(8 * np.pi * V[:, 1])
    V1 = wavy_redraw(V0, seed, h)
    return V0, V1, F, eta


def wavy_redraw(V0: np.ndarray, seed: int, h: float = 1.0 / 1024):
    """V1 for the wavy cloth: x compressed 30% toward 0.5, plus N(0, 0.5 h)."""
    rng = np.random.default_rng(seed + 1_000_003)
    V1 = V0.copy()
    V1[:, 0] = 0.5 + 0.7 * (V1[:, 0] - 0.5)
    V1 += rng.normal(0.0, 0.5 * h, V1.shape)
    return np.ascontiguousarray(V1)


def icosphere(subdiv: int):
    """Unit icosphere: 10 * 4^s + 2 vertices, 20 * 4^s triangles."""
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
             (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    V = np.array(verts, dtype=np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array(faces, dtype=np.int64)
    for _ in range(subdiv):
        e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        key = np.minimum(e[:, 0], e[:, 1]) * len(V) + np.maximum(e[:, 0], e[:, 1])
        uk, inv = np.unique(key, return_inverse=True)
        a = uk // len(V)
        b = uk % len(V)
        mid = V[a] + V[b]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(V)
        V = np.concatenate([V, mid])
        nf = len(F)
        m01 = base + inv[:nf]
        m12 = base + inv[nf:2 * nf]
        m20 = base + inv[2 * nf:]
        F = np.concatenate([
            np.stack([F[:, 0], m01, m20], 1), np.stack([F[:, 1], m12, m01], 1),
            np.stack([F[:, 2], m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return V, F.astype(np.int32)


def icospheres(k: int = 64, subdiv: int = 6, seed: int = 0, eta: float = 1e-3):
    rng = np.random.default_rng(seed)
    Vs, Fs = icosphere(subdiv)
    nv = len(Vs)
    V0 = np.empty((k * nv, 3))
    V1 = np.empty((k * nv, 3))
    F = np.empty((k * len(Fs), 3), dtype=np.int32)
    for s in range(k):
        r = rng.uniform(0.05, 0.1)
        c = rng.uniform(0.0, 1.0, 3)
        tr = rng.normal(0.0, 0.05, 3)
        p = Vs * r + c
        V0[s * nv:(s + 1) * nv] = p
        V1[s * nv:(s + 1) * nv] = p + tr + rng.normal(0.0, 1e-3, p.shape)
        F[s * len(Fs):(s + 1) * len(Fs)] = Fs + s * nv
    return V0, V1, F, eta


def annulus_2d(ring: int = 256, seed: int = 0, r_in: float = 0.3, r_out: float = 0.5,
               layers: int | None = None, eta: float = 1e-3):
    """2D triangulated annulus as an edge list (np x 2, int32)."""
    rng = np.random.default_rng(seed)
    if layers is None:
        layers = max(2, int(round(ring * (r_out - r_in) / (2 * math.pi * r_out))) + 1)
    rs = np.linspace(r_in, r_out, layers)
    th = np.arange(ring) * (2 * math.pi / ring)
    V = np.concatenate([np.stack([r * np.cos(th), r * np.sin(th)], 1) for r in rs])
    l, i = np.meshgrid(np.arange(layers - 1), np.arange(ring), indexing="ij")
    a = (l * ring + i).ravel()
    b = (l * ring + (i + 1) % ring).ravel()
    c = a + ring
    d = b + ring
    T = np.empty((2 * len(a), 3), dtype=np.int64)
    T[0::2] = np.stack([a, b, d], axis=1)
    T[1::2] = np.stack([a, d, c], axis=1)
    e = np.sort(np.concatenate([T[:, [0, 1]], T[:, [1, 2]], T[:, [2, 0]]]), axis=1)
    nvert = layers * ring
    key = np.unique(e[:, 0] * nvert + e[:, 1])          # sorted unique edges, row-major (lo, hi)
    e = np.stack([key // nvert, key % nvert], axis=1)
    ang = rng.uniform(-0.3, 0.3)
    R = np.array([[math.cos(ang), -math.sin(ang)], [math.sin(ang), math.cos(ang)]])
    shift = rng.normal(0.0, 0.05, 2)
    V0 = V + 0.5
    V1 = (V @ R.T) + 0.5 + shift + rng.normal(0.0, 1e-3, V.shape)
    return np.ascontiguousarray(V0), np.ascontiguousarray(V1), e.astype(np.int32), eta


def batch_scenes(n3d: int = 384, n2d: int = 128, seed: int = 0, max_side: int = 384, max_ring: int = 2048):
    """The batching workload: n3d folded cloths with side log-uniform in
    [16, max_side] and n2d annuli with ring resolution U[32, max_ring]."""
    rng = np.random.default_rng(seed)
    scenes = []
    for s in range(n3d):
        side = int(round(math.exp(rng.uniform(math.log(16), math.log(max_side)))))
        scenes.append(("cloth", folded_cloth(side, seed=seed * 7919 + s)))
    for s in range(n2d):
        ring = int(rng.integers(32, max_ring + 1))
        scenes.append(("annulus", annulus_2d(ring, seed=seed * 104729 + s)))
    return scenes


def stress_stencils(n: int = 100_000, seed: int = 0, eta: float = 1e-3):
    """Constructed hard stencils for the precision form: half near-parallel
    edge-edge pairs (angle <= 1e-7 rad), half near-coplanar vertex-face pairs
    (the point within the separation of the triangle's plane), separations
    log-uniform in [1e-8, 1e-2], each pair closing along its normal by a
    random fraction of up to twice the gap (some hit, some miss).
    Returns V0, V1 (4n x 3), sten (n x 4), is_vf (n), eta."""
    rng = np.random.default_rng(seed)
    sep = np.exp(rng.uniform(np.log(1e-8), np.log(1e-2), n))
    base = rng.uniform(0.0, 1.0, (n, 3))
    u = rng.normal(size=(n, 3)); u /= np.linalg.norm(u, axis=1, keepdims=True)
    w = rng.normal(size=(n, 3)); w -= (w * u).sum(1, keepdims=True) * u; w /= np.linalg.norm(w, axis=1, keepdims=True)
    nrm = np.cross(u, w)
    L = rng.uniform(1e-3, 5e-2, n)[:, None]
    V0 = np.empty((4 * n, 3)); V1 = np.empty((4 * n, 3))
    is_vf = (np.arange(n) % 2 == 0).astype(np.uint8)
    close = (eta + sep)[:, None] * rng.uniform(0.0, 2.0, (n, 1))
    # vertex-face: triangle (a, a+L u, a+L w); point above its interior (or
    # just outside) at height eta + sep, moving down by `close`.
    a = base
    off = rng.uniform(-0.1, 0.6, (n, 2))
    pt = a + L * (off[:, :1] * u + off[:, 1:] * w) + (eta + sep)[:, None] * nrm
    # edge-edge: edge (a, a + L u) and a copy tilted by <= 1e-7 rad, offset by
    # eta + sep along the normal, moving toward it by `close`.
    ang = rng.uniform(-1e-7, 1e-7, n)[:, None]
    dirb = u * np.cos(ang) + nrm * np.sin(ang)
    shift = rng.uniform(-0.5, 0.5, n)[:, None] * L
    q0 = a + shift * u + (eta + sep)[:, None] * nrm
    q1 = q0 + L * dirb
    vf = is_vf == 1
    V0[0::4] = np.where(vf[:, None], pt, a)
    V0[1::4] = np.where(vf[:, None], a, a + L * u)
    V0[2::4] = np.where(vf[:, None], a + L * u, q0)
    V0[3::4] = np.where(vf[:, None], a + L * w, q1)
    V1[:] = V0
    mv = close * nrm
    V1[0::4] -= np.where(vf[:, None], mv, 0.0)
    V1[2::4] -= np.where(vf[:, None], 0.0, mv)
    V1[3::4] -= np.where(vf[:, None], 0.0, mv)
    V1 += rng.normal(0.0, 1e-12, V1.shape)
    sten = (np.arange(4 * n, dtype=np.int32).reshape(n, 4))
    return V0, V1, sten, is_vf, eta
