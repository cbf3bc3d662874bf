"""mclccd_narrow_phase_bulk_static: the bulk narrow phase for callers that
cannot allocate device memory (fixed device-memory budgets, processes where
another allocator owns the device memory, plugins whose host forbids device
allocations).  It keeps its scratch in a fixed device array instead of
calling cudaMallocAsync.

Called through the C ABI, it must give exactly what mclccd_narrow_phase_bulk
gives (the same bit-exact bar as the other narrow-phase tests), on two calls
in a row -- the shared array keeps the previous call's contents -- for host
and for device arrays, and it must refuse host-memory calls whose staging
would not fit its fixed array.  This file is collected last and needs no
state from the other tests."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "mclccd_b200", "libmclccd_b200.so")
MEM_HOST, MEM_DEVICE = 0, 1
ERR_SCRATCH_LIMIT = 8
SCRATCH_BYTES = 32 << 20


def _lib():
    L = C.CDLL(LIB)
    sig = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_longlong, C.c_double,
           C.c_double, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    for name in ("mclccd_narrow_phase_bulk", "mclccd_narrow_phase_bulk_static"):
        getattr(L, name).argtypes = sig
        getattr(L, name).restype = C.c_int
    return L


def _scene(seed, n=30000, nv=5000):
    rng = np.random.default_rng(seed)
    V0 = rng.random((nv, 3))
    V1 = V0 + rng.normal(0, 0.04, V0.shape)
    sten = rng.integers(0, nv, (n, 4)).astype(np.int32)
    is_vf = (rng.random(n) < 0.4).astype(np.uint8)
    sten[:100, 3] = sten[:100, 2]            # degenerate triangles: hit with toi NaN
    return V0, V1, sten, is_vf


def _host_call(L, fn, V0, V1, sten, is_vf, eta):
    n = len(sten)
    toi = np.full(n, 7.0)
    hit = np.full(n, 7, np.int32)
    rc = getattr(L, fn)(3, V0.ctypes.data, V1.ctypes.data, len(V0), sten.ctypes.data, is_vf.ctypes.data, n,
                        eta, eta, toi.ctypes.data, hit.ctypes.data, MEM_HOST, None)
    return rc, toi, hit


def test_static_matches_allocating_host_twice():
    L = _lib()
    for seed, eta in ((1, 1e-3), (2, 2e-2)):       # two calls in a row, different data
        V0, V1, sten, is_vf = _scene(seed)
        rc_a, toi_a, hit_a = _host_call(L, "mclccd_narrow_phase_bulk", V0, V1, sten, is_vf, eta)
        rc_b, toi_b, hit_b = _host_call(L, "mclccd_narrow_phase_bulk_static", V0, V1, sten, is_vf, eta)
        assert rc_a == 0 and rc_b == 0
        assert np.array_equal(hit_a, hit_b)
        assert np.array_equal(toi_a, toi_b, equal_nan=True)
        assert hit_b.sum() > 0 and np.isnan(toi_b).any()


def test_static_matches_allocating_device_twice():
    torch = pytest.importorskip("torch")
    L = _lib()
    for seed, eta in ((3, 1e-3), (4, 5e-3)):
        V0, V1, sten, is_vf = (torch.from_numpy(a).cuda() for a in _scene(seed, n=50000))
        n = sten.shape[0]
        outs = []
        for fn in ("mclccd_narrow_phase_bulk", "mclccd_narrow_phase_bulk_static"):
            toi = torch.full((n,), 7.0, dtype=torch.float64, device="cuda")
            hit = torch.full((n,), 7, dtype=torch.int32, device="cuda")
            rc = getattr(L, fn)(3, V0.data_ptr(), V1.data_ptr(), V0.shape[0], sten.data_ptr(), is_vf.data_ptr(), n,
                                eta, eta, toi.data_ptr(), hit.data_ptr(), MEM_DEVICE, None)
            assert rc == 0
            outs.append((toi.cpu().numpy(), hit.cpu().numpy()))
        assert np.array_equal(outs[0][1], outs[1][1])
        assert np.array_equal(outs[0][0], outs[1][0], equal_nan=True)


def test_static_rejects_host_arrays_beyond_its_scratch():
    L = _lib()
    nv = SCRATCH_BYTES // (2 * 3 * 8) + 1024           # V0 + V1 alone exceed the fixed array
    V0 = np.zeros((nv, 3)); V1 = np.zeros((nv, 3))
    sten = np.zeros((4, 4), np.int32); is_vf = np.ones(4, np.uint8)
    rc, _, _ = _host_call(L, "mclccd_narrow_phase_bulk_static", V0, V1, sten, is_vf, 1e-3)
    assert rc == ERR_SCRATCH_LIMIT
    L.mclccd_status_string.restype = C.c_char_p
    assert b"fixed scratch" in L.mclccd_status_string(ERR_SCRATCH_LIMIT)
