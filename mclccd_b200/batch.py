"""Batched CCD over many independent scenes (mclccd_batch_* in the C ABI).

Each scene is what one ``BVHTree(dim)`` would process with
box_eta = vf_ccd_eta = ee_ccd_eta = eta.  One ``run`` is a CUDA graph: a
segmented LBVH build over all scenes, then traversal and narrow phase in
one of two forms (tuning key ``form``): ``FORM_WAVES``, a device-driven
loop of waves (walk -> stencil expansion -> ACCD -> per-scene reductions)
in a conditional graph node, or ``FORM_PERSISTENT``, one persistent
traversal + narrow-phase kernel per group with a global work queue.  The
results are identical; the autotuner picks the faster.  Results are per scene:
hit / discrete / candidate counts, the earliest toi and its stencil, and
the device time at which the scene's last work finished.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .ccd import OK, MEM_HOST, PREC_FP64, CCDError, lib

TUNE_KEYS = {"block": 0, "stack": 1, "chunk": 2, "leaf": 3, "form": 4, "wave": 5}
FORM_WAVES, FORM_PERSISTENT = 0, 1


def _sig(L):
    if getattr(L, "_batch_sig", False):
        return L
    vp, llp = C.c_void_p, C.POINTER(C.c_longlong)
    sig = {
        "mclccd_batch_create": ([C.POINTER(vp)], C.c_int),
        "mclccd_batch_destroy": ([vp], C.c_int),
        "mclccd_batch_set_scenes": ([vp, C.c_int, vp, vp, vp, vp, vp, vp, vp, C.c_int], C.c_int),
        "mclccd_batch_set_positions": ([vp, vp, vp, C.c_int], C.c_int),
        "mclccd_batch_set_precision": ([vp, C.c_int], C.c_int),
        "mclccd_batch_set_tuning": ([vp, C.c_int, C.c_int], C.c_int),
        "mclccd_batch_get_tuning": ([vp, C.c_int, C.POINTER(C.c_int)], C.c_int),
        "mclccd_batch_wave_stats": ([vp, llp, llp], C.c_int),
        "mclccd_batch_run": ([vp, vp], C.c_int),
        "mclccd_batch_results": ([vp, vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "mclccd_batch_last_error": ([vp], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    L._batch_sig = True
    return L


class Batch:
    """Many scenes per step on one GPU."""

    def __init__(self, precision: int = PREC_FP64):
        self._L = _sig(lib())
        h = C.c_void_p()
        self._check(self._L.mclccd_batch_create(C.byref(h)), None)
        self._h = h
        self.n_scenes = 0
        self._dims = None
        self.set_precision(precision)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._L.mclccd_batch_destroy(h)
            self._h = None

    def _check(self, rc, h):
        if rc != OK:
            msg = self._L.mclccd_status_string(rc).decode()
            if h is not None:
                detail = self._L.mclccd_batch_last_error(h)
                if detail:
                    msg += ": " + detail.decode()
            raise CCDError(rc, msg)

    def set_precision(self, precision: int):
        self._check(self._L.mclccd_batch_set_precision(self._h, precision), self._h)
        self.precision = precision

    def set_tuning(self, **kv):
        for k, v in kv.items():
            self._check(self._L.mclccd_batch_set_tuning(self._h, TUNE_KEYS[k], int(v)), self._h)

    def get_tuning(self):
        out = {}
        for k, i in TUNE_KEYS.items():
            v = C.c_int()
            self._check(self._L.mclccd_batch_get_tuning(self._h, i, C.byref(v)), self._h)
            out[k] = v.value
        return out

    def wave_stats(self):
        """(waves, redos) of the last run in the waves form."""
        w, r = C.c_longlong(), C.c_longlong()
        self._check(self._L.mclccd_batch_wave_stats(self._h, C.byref(w), C.byref(r)), self._h)
        return w.value, r.value

    def set_scenes(self, scenes):
        """scenes: sequence of (V0, V1, P, eta); V0/V1 nv x dim float64, P
        np x dim int32 (edges in 2D, triangles in 3D), scene-local ids."""
        dims = np.array([np.asarray(s[0]).shape[1] for s in scenes], np.int32)
        nvs = np.array([np.asarray(s[0]).shape[0] for s in scenes], np.int32)
        nps = np.array([np.asarray(s[2]).reshape(-1, d).shape[0] for s, d in zip(scenes, dims)], np.int32)
        etas = np.array([float(s[3]) for s in scenes], np.float64)
        V0 = np.ascontiguousarray(np.concatenate([np.asarray(s[0], np.float64).ravel() for s in scenes]))
        V1 = np.ascontiguousarray(np.concatenate([np.asarray(s[1], np.float64).ravel() for s in scenes]))
        P = np.ascontiguousarray(np.concatenate([np.asarray(s[2], np.int32).ravel() for s in scenes]))
        rc = self._L.mclccd_batch_set_scenes(self._h, len(scenes), dims.ctypes.data, nvs.ctypes.data,
                                             nps.ctypes.data, V0.ctypes.data, V1.ctypes.data, P.ctypes.data,
                                             etas.ctypes.data, MEM_HOST)
        self._check(rc, self._h)
        self.n_scenes = len(scenes)
        self._dims = dims
        self._nv = nvs

    def set_positions(self, V0s, V1s):
        """New vertex positions for every scene (same topology)."""
        V0 = np.ascontiguousarray(np.concatenate([np.asarray(v, np.float64).ravel() for v in V0s]))
        V1 = np.ascontiguousarray(np.concatenate([np.asarray(v, np.float64).ravel() for v in V1s]))
        self._check(self._L.mclccd_batch_set_positions(self._h, V0.ctypes.data, V1.ctypes.data, MEM_HOST), self._h)

    def run(self, stream: int | None = None):
        self._check(self._L.mclccd_batch_run(self._h, C.c_void_p(stream or 0)), self._h)

    def results(self):
        n = self.n_scenes
        hits = np.zeros(n, np.int64); toi = np.zeros(n); sten = np.zeros((n, 4), np.int32)
        isvf = np.zeros(n, np.uint8); disc = np.zeros(n, np.int64); nst = np.zeros(n, np.int64)
        done = np.zeros(n); bms = C.c_double()
        rc = self._L.mclccd_batch_results(self._h, hits.ctypes.data, toi.ctypes.data, sten.ctypes.data,
                                          isvf.ctypes.data, disc.ctypes.data, nst.ctypes.data, done.ctypes.data,
                                          C.byref(bms))
        self._check(rc, self._h)
        return {"n_hits": hits, "min_toi": toi, "min_sten": sten, "min_is_vf": isvf, "n_discrete": disc,
                "n_stencils": nst, "done_ms": done, "batch_ms": bms.value}
