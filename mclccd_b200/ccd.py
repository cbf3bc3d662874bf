"""Python mirror of mclccd's ``mcl::BVHTree<double, DIM>`` over the C ABI.

Same members and meaning as the reference (include/MCL/BVHTree.hpp):
``options`` (box_eta, vf_ccd_eta, ee_ccd_eta, reptri, threaded, discrete,
continuous, vf_one_sided, ee_robust), ``update(V0, V1, P, active=None)``,
``traverse(V0, V1, P)`` and the hooks ``append_pair(sten, is_vf, toi)`` and
``append_discrete(p0, p1) -> stop``.  The CCD work runs on the GPU; after
``traverse`` the results are also available as arrays (``hits()``,
``discrete()``, ``candidates()``).

``filter_pair`` and ``narrow_phase`` are honoured on the host: when set,
``traverse`` copies the candidate stencils out, drops those ``filter_pair``
rejects and scores the rest with ``narrow_phase`` (or the device ACCD when
only a filter is set).  Hooks are called from the calling thread.

Arrays may be numpy arrays (host) or CUDA torch tensors (device); there is
no CPU fallback: without the built library every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MCLCCD_B200_LIB") or os.path.join(_HERE, "libmclccd_b200.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_OVERFLOW, ERR_STATE, ERR_DEVICE, ERR_UNSUPPORTED = range(8)
MEM_HOST, MEM_DEVICE = 0, 1
OPT_REPTRI, OPT_THREADED, OPT_DISCRETE, OPT_CONTINUOUS = 1, 2, 4, 8
OPT_VF_ONE_SIDED, OPT_EE_ROBUST = 16, 32
BULK_VF_ONE_SIDED = 0x100
OPT_ALWAYS_REBUILD, OPT_PROFILE = 1 << 8, 1 << 9
PREC_FP64, PREC_FP32_CERTIFIED = 0, 1

_lib = None


class CCDError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"mclccd_b200 status {status}: {msg}")
        self.status = status


def lib():
    """Loads libmclccd_b200.so (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C mclccd_b200`")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip, ucp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_ubyte)
    llp = C.POINTER(C.c_longlong)
    sig = {
        "mclccd_create": ([C.c_int, C.POINTER(vp)], C.c_int),
        "mclccd_destroy": ([vp], C.c_int),
        "mclccd_set_options": ([vp, C.c_double, C.c_double, C.c_double, C.c_uint], C.c_int),
        "mclccd_get_options": ([vp, dp, dp, dp, C.POINTER(C.c_uint)], C.c_int),
        "mclccd_set_stream": ([vp, vp], C.c_int),
        "mclccd_set_precision": ([vp, C.c_int], C.c_int),
        "mclccd_update": ([vp, vp, vp, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int], C.c_int),
        "mclccd_traverse": ([vp, vp, vp, C.c_int, vp, C.c_int], C.c_int),
        "mclccd_update_f32": ([vp, vp, vp, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int], C.c_int),
        "mclccd_update_ex": ([vp, vp, vp, C.c_int, vp, C.c_int, C.c_int, vp, C.c_int, C.c_uint], C.c_int),
        "mclccd_traverse_ex": ([vp, vp, vp, C.c_int, vp, C.c_int, C.c_uint], C.c_int),
        "mclccd_traverse_out": ([vp, vp, vp, C.c_int, vp, C.c_int, vp, vp, vp, C.c_longlong, llp, vp, C.c_longlong, llp,
                                 C.c_int], C.c_int),
        "mclccd_traverse_f32": ([vp, vp, vp, C.c_int, vp, C.c_int], C.c_int),
        "mclccd_counts": ([vp, llp, llp, llp, llp, llp], C.c_int),
        "mclccd_get_hits": ([vp, C.c_int, C.c_longlong, vp, vp, vp], C.c_int),
        "mclccd_get_discrete": ([vp, C.c_int, C.c_longlong, vp], C.c_int),
        "mclccd_get_candidates": ([vp, C.c_int, C.c_longlong, vp, vp], C.c_int),
        "mclccd_get_leaves": ([vp, vp, vp], C.c_int),
        "mclccd_narrow_phase_bulk": ([C.c_int, vp, vp, C.c_int, vp, vp, C.c_longlong, C.c_double, C.c_double,
                                      vp, vp, C.c_int, vp], C.c_int),
        "mclccd_stage_ms": ([vp, C.POINTER(C.c_float), C.c_int], C.c_int),
        "mclccd_narrow_phase_bulk_ex": ([C.c_int, vp, vp, C.c_int, vp, vp, C.c_longlong, C.c_double, C.c_double,
                                         vp, vp, C.c_int, vp, C.c_int, llp], C.c_int),
        "mclccd_precision_stats": ([vp, llp, llp], C.c_int),
        "mclccd_vjp_toi": ([C.c_int, vp, vp, C.c_int, vp, vp, vp, vp, C.c_longlong, C.c_double, C.c_double, vp, vp,
                            vp, vp, vp, llp, C.c_int, vp], C.c_int),
        "mclccd_tree_vjp_toi": ([vp, vp, vp, vp, llp, C.c_int], C.c_int),
        "mclccd_set_tuning": ([vp, C.c_int, C.c_int], C.c_int),
        "mclccd_get_tuning": ([vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mclccd_kernel_launches": ([vp, llp], C.c_int),
        "mclccd_build_stats": ([vp, llp, llp], C.c_int),
        "mclccd_fp64_fma_rate": ([C.c_int, C.POINTER(C.c_double)], C.c_int),
        "mclccd_last_error": ([vp], C.c_char_p),
        "mclccd_status_string": ([C.c_int], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def fp64_fma_rate(device: int = 0) -> float:
    """Measured FP64 FMA throughput of a device in TFLOP/s
    (mclccd_fp64_fma_rate)."""
    out = C.c_double(0.0)
    rc = lib().mclccd_fp64_fma_rate(device, C.byref(out))
    if rc != 0:
        raise CCDError(rc, "mclccd_fp64_fma_rate failed")
    return out.value


def _is_torch_cuda(a) -> bool:
    return type(a).__module__.startswith("torch") and getattr(a, "is_cuda", False)


def _is_f32(a):
    """float32 coordinates (numpy array or CUDA tensor)."""
    if a is None:
        return False
    if _is_torch_cuda(a):
        import torch
        return a.dtype == torch.float32
    return getattr(a, "dtype", None) == np.float32


IN_F32, IN_V_COLMAJOR, IN_P_COLMAJOR = 1, 2, 4


def _colmajor(a, dtype):
    """True for a 2D column-major (Fortran-order) array of dtype: passed to
    the library as it is, with the layout flag, instead of a row-major copy."""
    if a is None:
        return False
    if _is_torch_cuda(a):
        import torch
        tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32}[dtype]
        return (a.dim() == 2 and a.dtype == tdt and a.shape[0] > 1 and a.shape[1] > 1
                and a.stride() == (1, a.shape[0]))
    return (isinstance(a, np.ndarray) and a.ndim == 2 and a.dtype == dtype and a.shape[0] > 1 and a.shape[1] > 1
            and a.flags.f_contiguous and not a.flags.c_contiguous)


def _arg_colmajor(a):
    """(pointer, mem_kind, keepalive, rows) of a column-major array."""
    if _is_torch_cuda(a):
        return C.c_void_p(a.data_ptr()), MEM_DEVICE, a, a.shape[0]
    return C.c_void_p(a.ctypes.data), MEM_HOST, a, a.shape[0]


def _arg(a, dtype, cols=None):
    """(pointer, mem_kind, keepalive, rows) for a numpy array or CUDA tensor."""
    if a is None:
        return None, None, None, 0
    if _is_torch_cuda(a):
        import torch
        tdt = {np.float64: torch.float64, np.float32: torch.float32, np.int32: torch.int32, np.uint8: torch.uint8}[dtype]
        if a.dtype != tdt:
            raise TypeError(f"expected {tdt}, got {a.dtype}")
        a = a.contiguous()
        return C.c_void_p(a.data_ptr()), MEM_DEVICE, a, (a.shape[0] if a.dim() else 0)
    arr = np.ascontiguousarray(a, dtype=dtype)
    if cols is not None and arr.ndim == 1:
        arr = arr.reshape(-1, cols)
    return C.c_void_p(arr.ctypes.data), MEM_HOST, arr, (arr.shape[0] if arr.ndim else 0)


@dataclass
class Options:
    """BVHTree::Options (BVHTree.hpp:42-64) with the reference defaults."""
    box_eta: float = 1e-6
    vf_ccd_eta: float = 1e-6
    ee_ccd_eta: float = 1e-6
    reptri: bool = True
    threaded: bool = True
    discrete: bool = True
    continuous: bool = True
    vf_one_sided: bool = False
    ee_robust: bool = True
    always_rebuild: bool = False
    profile: bool = False

    def flags(self) -> int:
        f = 0
        for name, bit in (("reptri", OPT_REPTRI), ("threaded", OPT_THREADED), ("discrete", OPT_DISCRETE),
                          ("continuous", OPT_CONTINUOUS), ("vf_one_sided", OPT_VF_ONE_SIDED),
                          ("ee_robust", OPT_EE_ROBUST), ("always_rebuild", OPT_ALWAYS_REBUILD),
                          ("profile", OPT_PROFILE)):
            if getattr(self, name):
                f |= bit
        return f


class BVHTree:
    """mcl::BVHTree<double, dim> on the GPU."""

    def __init__(self, dim: int = 3, precision: int = PREC_FP64):
        self._L = lib()
        self.dim = dim
        self._nv = 0
        h = C.c_void_p()
        self._check(self._L.mclccd_create(dim, C.byref(h)), None)
        self._h = h
        self.options = Options()
        self.append_pair = None
        self.append_discrete = None
        self.filter_pair = None
        self.narrow_phase = None
        self._keep = []
        self._last = None
        self.precision = PREC_FP64
        if precision != PREC_FP64:
            self.set_precision(precision)

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc, h):
        if rc != OK:
            L = self._L
            msg = (L.mclccd_last_error(h) if h is not None else b"") or L.mclccd_status_string(rc)
            raise CCDError(rc, msg.decode())

    def close(self):
        if getattr(self, "_h", None):
            self._L.mclccd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _push_options(self):
        o = self.options
        self._check(self._L.mclccd_set_options(self._h, o.box_eta, o.vf_ccd_eta, o.ee_ccd_eta, o.flags()), self._h)

    def _pull_options(self):
        b, v, e, f = C.c_double(), C.c_double(), C.c_double(), C.c_uint()
        self._L.mclccd_get_options(self._h, C.byref(b), C.byref(v), C.byref(e), C.byref(f))
        self.options.box_eta, self.options.vf_ccd_eta, self.options.ee_ccd_eta = b.value, v.value, e.value

    def set_precision(self, precision: int):
        self._check(self._L.mclccd_set_precision(self._h, precision), self._h)
        self.precision = precision

    TUNE_KEYS = {"expand_grid": 0, "accd_grid": 1, "walk_packet": 2, "accd_rebin": 3, "walk_window": 4, "overlap": 5,
                 "narrow_fused": 6, "fused_grid": 7, "walk_refill": 8, "expand_split": 9,
                 "rebuild_ratio": 10, "walk_buffer": 11}

    def set_tuning(self, **kv):
        """Launch-shape knobs (expand_grid, accd_grid, walk_packet, accd_rebin, walk_window, overlap,
        narrow_fused, fused_grid, walk_refill, expand_split, rebuild_ratio, walk_buffer); results
        never depend on them."""
        for k, v in kv.items():
            self._check(self._L.mclccd_set_tuning(self._h, self.TUNE_KEYS[k], int(v)), self._h)

    def get_tuning(self) -> dict:
        out = {}
        for k, key in self.TUNE_KEYS.items():
            v = C.c_int()
            self._check(self._L.mclccd_get_tuning(self._h, key, C.byref(v)), self._h)
            out[k] = v.value
        return out

    def set_stream(self, stream_handle: int | None):
        self._check(self._L.mclccd_set_stream(self._h, C.c_void_p(stream_handle or 0)), self._h)

    # -- the reference API --------------------------------------------------
    def update(self, V0, V1, P, active=None):
        """BVHTree::update (BVHTree.cpp:27-126).  float32 coordinates take
        the BVHTree<float, DIM> form (mclccd_update_f32: widened exactly to
        double on the device)."""
        f32 = _is_f32(V0)
        vt = np.float32 if f32 else np.float64
        vcol = _colmajor(V0, vt) and _colmajor(V1, vt)
        pcol = _colmajor(P, np.int32)
        pv0, k0, a0, nv = _arg_colmajor(V0) if vcol else _arg(V0, vt, self.dim)
        pv1, k1, a1, nv1 = _arg_colmajor(V1) if vcol else _arg(V1, vt, self.dim)
        pp, kp, ap, npr = _arg_colmajor(P) if pcol else _arg(P, np.int32)
        pa, ka, aa, _ = _arg(active, np.int32)
        if nv != nv1:   # BVHTree.hpp:160: silently ignored by the reference
            raise ValueError("V0 and V1 must have the same number of rows")
        kinds = {k for k in (k0, k1, kp, ka) if k is not None}
        if len(kinds) > 1:
            raise ValueError("V0, V1, P and active must all be host arrays or all CUDA tensors")
        pdim = ap.shape[1] if ap.ndim == 2 else self.dim
        flags = (IN_F32 if f32 else 0) | (IN_V_COLMAJOR if vcol else 0) | (IN_P_COLMAJOR if pcol else 0)
        self._push_options()
        rc = self._L.mclccd_update_ex(self._h, pv0, pv1, nv, pp, npr, pdim, pa, kinds.pop() if kinds else MEM_HOST,
                                      flags)
        self._pull_options()
        self._check(rc, self._h)
        self._keep = [a0, a1, ap, aa]
        self._nv = nv

    def traverse(self, V0=None, V1=None, P=None):
        """BVHTree::traverse (BVHTree.cpp:129-159), then the hooks."""
        f32 = _is_f32(V0)
        vt = np.float32 if f32 else np.float64
        vcol = _colmajor(V0, vt) and _colmajor(V1, vt)
        pcol = _colmajor(P, np.int32)
        pv0, k0, a0, nv = _arg_colmajor(V0) if vcol else _arg(V0, vt, self.dim)
        pv1, k1, a1, _ = _arg_colmajor(V1) if vcol else _arg(V1, vt, self.dim)
        pp, kp, ap, _ = _arg_colmajor(P) if pcol else _arg(P, np.int32)
        kind = k0 if k0 is not None else MEM_HOST
        flags = (IN_F32 if f32 else 0) | (IN_V_COLMAJOR if vcol else 0) | (IN_P_COLMAJOR if pcol else 0)
        self._push_options()
        self._check(self._L.mclccd_traverse_ex(self._h, pv0, pv1, nv, pp, kind, flags), self._h)
        if V0 is not None:
            self._nv = nv
        self._dispatch(V0, V1)

    def traverse_out(self, sten, is_vf, toi, discrete=None, V0=None, V1=None, P=None):
        """traverse with the results delivered into caller arrays
        (mclccd_traverse_out): sten (cap x 4 int32), is_vf (cap uint8), toi
        (cap float64), discrete (dcap x 2 int32), all host (numpy / CPU
        tensors, page-locked for overlap) or all CUDA tensors.  Host copies
        overlap the rest of the step.  Returns (n_hits, n_discrete), the
        full counts; the arrays receive a prefix up to their capacity.  The
        hooks are not called."""
        pv0, k0, a0, nv = _arg(V0, np.float64, self.dim)
        pv1, k1, a1, _ = _arg(V1, np.float64, self.dim)
        pp, kp, ap, _ = _arg(P, np.int32)
        kind = k0 if k0 is not None else MEM_HOST

        def ptr(a):
            if a is None:
                return None, None
            if hasattr(a, "data_ptr"):
                return C.c_void_p(a.data_ptr()), (MEM_DEVICE if a.is_cuda else MEM_HOST)
            return C.c_void_p(a.ctypes.data), MEM_HOST
        (ps, ks), (pv, kv), (pt, kt) = ptr(sten), ptr(is_vf), ptr(toi)
        pd, kd = ptr(discrete)
        kinds = {k for k in (ks, kv, kt, kd) if k is not None}
        if len(kinds) > 1:
            raise ValueError("output arrays must all be host arrays or all CUDA tensors")
        cap = min(len(x) for x in (sten, is_vf, toi) if x is not None) if any(x is not None for x in (sten, is_vf, toi)) else 0
        dcap = len(discrete) if discrete is not None else 0
        nh, nd = C.c_longlong(), C.c_longlong()
        self._push_options()
        self._check(self._L.mclccd_traverse_out(self._h, pv0, pv1, nv, pp, kind, ps, pv, pt, cap, C.byref(nh), pd, dcap,
                                                C.byref(nd), kinds.pop() if kinds else MEM_HOST), self._h)
        if V0 is not None:
            self._nv = nv
        return nh.value, nd.value

    def _dispatch(self, V0, V1):
        if self.filter_pair is not None or self.narrow_phase is not None:
            sten, is_vf = self.candidates()
            keep = np.ones(len(sten), bool)
            if self.filter_pair is not None:
                for i in range(len(sten)):
                    if self.filter_pair(sten[i], bool(is_vf[i])):
                        keep[i] = False
            sten, is_vf = sten[keep], is_vf[keep]
            if self.narrow_phase is not None:
                toi = np.array([self.narrow_phase(sten[i], bool(is_vf[i])) for i in range(len(sten))], np.float64)
            else:
                v0 = V0 if V0 is not None else self._keep[0]
                v1 = V1 if V1 is not None else self._keep[1]
                if _is_torch_cuda(v0):
                    v0, v1 = v0.cpu().numpy(), v1.cpu().numpy()
                toi, _ = narrow_phase_bulk(v0, v1, sten, is_vf, self.options.vf_ccd_eta, self.options.ee_ccd_eta)
            m = toi >= 0
            self._last = (sten[m], is_vf[m], toi[m])
            if self.append_pair is not None:
                for s, v, t in zip(*self._last):
                    self.append_pair(s, bool(v), float(t))
        elif self.append_pair is not None:
            for s, v, t in zip(*self.hits()):
                self.append_pair(s, bool(v), float(t))
        if self.append_discrete is not None and self.options.discrete:
            for a, b in self.discrete():
                if self.append_discrete(int(a), int(b)):
                    break

    # -- array access -----------------------------------------------------
    def counts(self) -> dict:
        v = [C.c_longlong() for _ in range(5)]
        self._check(self._L.mclccd_counts(self._h, *[C.byref(x) for x in v]), self._h)
        return dict(zip(("hits", "discrete", "vf", "ee", "leaf_pairs"), (x.value for x in v)))

    def hits(self):
        """(sten int32[n,4], is_vf uint8[n], toi float64[n]) of the last traverse."""
        if self._last is not None and (self.filter_pair is not None or self.narrow_phase is not None):
            return self._last
        n = self.counts()["hits"]
        s = np.empty((n, 4), np.int32); v = np.empty(n, np.uint8); t = np.empty(n, np.float64)
        self._check(self._L.mclccd_get_hits(self._h, MEM_HOST, n, s.ctypes.data, v.ctypes.data, t.ctypes.data), self._h)
        return s, v, t

    def discrete(self):
        n = self.counts()["discrete"]
        d = np.empty((n, 2), np.int32)
        self._check(self._L.mclccd_get_discrete(self._h, MEM_HOST, n, d.ctypes.data), self._h)
        return d

    def candidates(self):
        c = self.counts()
        n = c["vf"] + c["ee"]
        s = np.empty((n, 4), np.int32); v = np.empty(n, np.uint8)
        self._check(self._L.mclccd_get_candidates(self._h, MEM_HOST, n, s.ctypes.data, v.ctypes.data), self._h)
        return s, v

    def leaves(self, np_: int):
        b = np.empty((np_, 6, self.dim), np.float64); f = np.empty(np_, np.uint8)
        self._check(self._L.mclccd_get_leaves(self._h, b.ctypes.data, f.ctypes.data), self._h)
        return b, f

    def fp64_fallbacks(self) -> int:
        """Stencils the FP32-certified form evaluated in full FP64 (last traverse)."""
        return self.precision_stats()[0]

    def precision_stats(self):
        """(stencils the FP32-certified form handed to FP64, hits reported with the toi bound)."""
        n, m = C.c_longlong(), C.c_longlong()
        self._check(self._L.mclccd_precision_stats(self._h, C.byref(n), C.byref(m)), self._h)
        return n.value, m.value

    def vjp_toi(self, g_toi):
        """Adjoint of the last traverse's hits: (dL/dV0, dL/dV1, n_ok) for the
        upstream gradient g_toi (one entry per hit, in hits() order).  numpy
        in, numpy out; a CUDA tensor in gives CUDA tensors out."""
        n_ok = C.c_longlong()
        cnt = self.counts()
        if _is_torch_cuda(g_toi):
            import torch
            g = g_toi.to(torch.float64).contiguous()
            nv, dim = self._nv, self.dim
            dV0 = torch.empty((nv, dim), dtype=torch.float64, device=g.device)
            dV1 = torch.empty_like(dV0)
            self._check(self._L.mclccd_tree_vjp_toi(self._h, g.data_ptr(), dV0.data_ptr(), dV1.data_ptr(),
                                                    C.byref(n_ok), MEM_DEVICE), self._h)
            return dV0, dV1, n_ok.value
        g = np.ascontiguousarray(g_toi, np.float64).reshape(-1)
        if len(g) != cnt["hits"]:
            raise ValueError(f"g_toi has {len(g)} entries, the traverse had {cnt['hits']} hits")
        dV0 = np.zeros((self._nv, self.dim)); dV1 = np.zeros((self._nv, self.dim))
        self._check(self._L.mclccd_tree_vjp_toi(self._h, g.ctypes.data, dV0.ctypes.data, dV1.ctypes.data,
                                                C.byref(n_ok), MEM_HOST), self._h)
        return dV0, dV1, n_ok.value

    def stage_ms(self):
        a = (C.c_float * 7)()
        self._L.mclccd_stage_ms(self._h, a, 7)
        return dict(zip(("update", "build", "refit", "traverse", "walk", "expand", "narrow"), list(a)))

    def kernel_launches(self) -> int:
        n = C.c_longlong()
        self._L.mclccd_kernel_launches(self._h, C.byref(n))
        return n.value

    def build_stats(self):
        """(full hierarchy builds, of which caused by the tree-quality trigger)."""
        b, q = C.c_longlong(), C.c_longlong()
        self._check(self._L.mclccd_build_stats(self._h, C.byref(b), C.byref(q)), self._h)
        return b.value, q.value


def narrow_phase_bulk(V0, V1, sten, is_vf, vf_eta, ee_eta=None, stream: int | None = None,
                      precision: int = PREC_FP64, return_fallbacks: bool = False, vf_one_sided: bool = False):
    """NarrowPhaseACCD::query_ccd_vf/ee over a stencil array on the GPU.
    Returns (toi, hit); toi is -1 where hit == 0.  With
    precision=PREC_FP32_CERTIFIED and return_fallbacks, also the number of
    stencils that needed full FP64.  vf_one_sided: VF stencils take the
    one-sided CTCD narrow phase (NarrowPhaseCTCD::query_ccd_vf with the
    wrong-side test), as BVHTree does with options.vf_one_sided."""
    L = lib()
    ee_eta = vf_eta if ee_eta is None else ee_eta
    if vf_one_sided:
        precision |= BULK_VF_ONE_SIDED
    nfb = C.c_longlong()
    if _is_torch_cuda(V0):
        import torch
        n = sten.shape[0]
        dim = V0.shape[1]
        toi = torch.empty(n, dtype=torch.float64, device=V0.device)
        hit = torch.empty(n, dtype=torch.int32, device=V0.device)
        rc = L.mclccd_narrow_phase_bulk_ex(dim, V0.data_ptr(), V1.data_ptr(), V0.shape[0],
                                           sten.contiguous().data_ptr(), is_vf.contiguous().data_ptr(), n, vf_eta,
                                           ee_eta, toi.data_ptr(), hit.data_ptr(), MEM_DEVICE,
                                           C.c_void_p(stream or 0), precision, C.byref(nfb))
    else:
        V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
        s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        v = np.ascontiguousarray(is_vf, np.uint8).reshape(-1)
        n = len(s)
        toi = np.empty(n, np.float64); hit = np.empty(n, np.int32)
        rc = L.mclccd_narrow_phase_bulk_ex(V0.shape[1], V0.ctypes.data, V1.ctypes.data, V0.shape[0], s.ctypes.data,
                                           v.ctypes.data, n, vf_eta, ee_eta, toi.ctypes.data, hit.ctypes.data,
                                           MEM_HOST, C.c_void_p(stream or 0), precision, C.byref(nfb))
    if rc != OK:
        raise CCDError(rc, L.mclccd_status_string(rc).decode())
    return (toi, hit, nfb.value) if return_fallbacks else (toi, hit)


def vjp_toi(V0, V1, sten, is_vf, toi, g_toi=None, vf_eta=1e-6, ee_eta=None, want_rows: bool = False,
            stream: int | None = None):
    """Adjoint of the time of impact over a hit array (mclccd_vjp_toi).

    Returns a dict: t_star, status (MCLCCD_VJP_*), n_ok, and with g_toi the
    vector-Jacobian products dV0, dV1 (nv x dim); with want_rows the per-hit
    Jacobian rows (n x 2 (dim+1) dim: d(t*)/dV0 slots, then d(t*)/dV1 slots).
    numpy arrays in host memory (the device path is the C call with
    MCLCCD_MEM_DEVICE)."""
    L = lib()
    ee_eta = vf_eta if ee_eta is None else ee_eta
    V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
    nv, dim = V0.shape
    s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
    v = np.ascontiguousarray(is_vf, np.uint8).reshape(-1)
    t = np.ascontiguousarray(toi, np.float64).reshape(-1)
    n = len(s)
    g = None if g_toi is None else np.ascontiguousarray(g_toi, np.float64).reshape(-1)
    dV0 = np.zeros((nv, dim)) if g is not None else None
    dV1 = np.zeros((nv, dim)) if g is not None else None
    ts = np.empty(n); st = np.empty(n, np.int32)
    rows = np.empty((n, 2 * (dim + 1) * dim)) if want_rows else None
    n_ok = C.c_longlong()
    ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
    rc = L.mclccd_vjp_toi(dim, V0.ctypes.data, V1.ctypes.data, nv, s.ctypes.data, v.ctypes.data, t.ctypes.data,
                          ptr(g), n, vf_eta, ee_eta, ptr(dV0), ptr(dV1), ts.ctypes.data, st.ctypes.data, ptr(rows),
                          C.byref(n_ok), MEM_HOST, C.c_void_p(stream or 0))
    if rc != OK:
        raise CCDError(rc, L.mclccd_status_string(rc).decode())
    out = {"t_star": ts, "status": st, "n_ok": n_ok.value}
    if g is not None:
        out["dV0"], out["dV1"] = dV0, dV1
    if want_rows:
        out["rows"] = rows
    return out
