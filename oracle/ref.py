"""TEST INFRASTRUCTURE -- ctypes access to the oracle libraries.

* ``Reference``  : the reference's own unmodified BVHTree/NarrowPhase code
  (oracle/_ref/libmclccd_ref.so, built by ``make -C oracle ref``).
* ``Port``       : this project's C restatement of the same path
  (oracle/_build/liboracle_port.so, built by ``make -C oracle port``).

Only tests, the smoke check and bench.py's CPU-baseline leg use this module;
the product library never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libmclccd_ref.so")
PORT_SO = os.path.join(HERE, "_build", "liboracle_port.so")
FLOPS_SO = os.path.join(HERE, "_build", "liboracle_flops.so")

F_REPTRI, F_THREADED, F_DISCRETE, F_CONTINUOUS, F_RECORD_CAND, F_ONE_SIDED, F_FLOAT = 1, 2, 4, 8, 16, 32, 64
DEFAULT_FLAGS = F_REPTRI | F_THREADED | F_DISCRETE | F_CONTINUOUS


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


_dp, _ip, _ucp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_ubyte)


def canon_ee(sten: np.ndarray) -> np.ndarray:
    """EE stencil [a,b,c,d] vs [c,d,a,b]: keep the lexicographically smaller."""
    s = np.asarray(sten, dtype=np.int64).reshape(-1, 4)
    sw = s[:, [2, 3, 0, 1]]
    swap = (sw[:, 0] < s[:, 0]) | ((sw[:, 0] == s[:, 0]) & (
        (sw[:, 1] < s[:, 1]) | ((sw[:, 1] == s[:, 1]) & (
            (sw[:, 2] < s[:, 2]) | ((sw[:, 2] == s[:, 2]) & (sw[:, 3] < s[:, 3]))))))
    out = s.copy()
    out[swap] = sw[swap]
    return out


def sort_rows(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a)
    if len(a) == 0:
        return a
    idx = np.lexsort(a.T[::-1])
    return a[idx]


def canonical_set(sten: np.ndarray, is_vf: np.ndarray) -> np.ndarray:
    """Sorted (is_vf, s0..s3) rows with EE orientation canonicalised."""
    s = np.asarray(sten, dtype=np.int64).reshape(-1, 4).copy()
    v = np.asarray(is_vf).astype(np.int64).reshape(-1)
    ee = v == 0
    if ee.any():
        s[ee] = canon_ee(s[ee])
    return sort_rows(np.concatenate([v[:, None], s], axis=1))


class Reference:
    """The reference's mcl::BVHTree<double,DIM> behind a C ABI."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path} (make -C oracle ref)")
        L = C.CDLL(path)
        L.ref_run.argtypes = [C.c_int, _dp, _dp, _ip, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, _ip]
        L.ref_run.restype = C.c_int
        L.ref_count.argtypes = [C.c_int]
        L.ref_count.restype = C.c_longlong
        L.ref_copy_candidates.argtypes = [_ip, _ucp]
        L.ref_copy_hits.argtypes = [_ip, _ucp, _dp]
        L.ref_copy_discrete.argtypes = [_ip]
        L.ref_copy_leaves.argtypes = [_dp, _ip]
        L.ref_accd.argtypes = [C.c_int, _dp, _dp, _ip, _ucp, C.c_longlong, C.c_double, C.c_double, _ip, _dp]
        L.ref_discrete.argtypes = [C.c_int, _dp, _ip, _ip, C.c_longlong, _ip]
        L.ref_ctcd_vf.argtypes = [C.c_int, _dp, _dp, _ip, C.c_longlong, C.c_double, _ip, _dp]
        L.ref_rpoly.argtypes = [_dp, C.c_int, _dp, _dp]
        L.ref_rpoly.restype = C.c_int
        L.ref_time.argtypes = [C.c_int, _dp, _dp, _dp, _ip, C.c_int, C.c_int, C.c_double, C.c_int,
                               _dp, _dp, _dp, C.POINTER(C.c_longlong)]
        L.ref_time.restype = C.c_longlong
        L.ref_threads.restype = C.c_int
        L.ref_time_steps.argtypes = [C.c_int, _dp, _dp, _dp, _ip, C.c_int, C.c_int, C.c_double, C.c_int, _dp,
                                     C.POINTER(C.c_longlong)]
        self.L = L

    def run(self, V0, V1, F, box_eta, vf_eta=None, ee_eta=None, flags=DEFAULT_FLAGS | F_RECORD_CAND, active=None):
        V0 = np.ascontiguousarray(V0, np.float64)
        V1 = np.ascontiguousarray(V1, np.float64)
        F = np.ascontiguousarray(F, np.int32)
        dim = V0.shape[1]
        np_, pdim = F.shape
        act = None if active is None else np.ascontiguousarray(active, np.int32)
        vf_eta = box_eta if vf_eta is None else vf_eta
        ee_eta = box_eta if ee_eta is None else ee_eta
        rc = self.L.ref_run(dim, _p(V0, C.c_double), _p(V1, C.c_double), _p(F, C.c_int), np_, pdim,
                            box_eta, vf_eta, ee_eta, flags, _p(act, C.c_int))
        assert rc == 0
        nc, nh, nd = (self.L.ref_count(i) for i in range(3))
        cs = np.empty((nc, 4), np.int32); cv = np.empty(nc, np.uint8)
        hs = np.empty((nh, 4), np.int32); hv = np.empty(nh, np.uint8); ht = np.empty(nh, np.float64)
        dp = np.empty((nd, 2), np.int32)
        boxes = np.empty((np_, 6, dim), np.float64); fl = np.empty((np_, 7), np.int32)
        self.L.ref_copy_candidates(_p(cs, C.c_int), _p(cv, C.c_ubyte))
        self.L.ref_copy_hits(_p(hs, C.c_int), _p(hv, C.c_ubyte), _p(ht, C.c_double))
        self.L.ref_copy_discrete(_p(dp, C.c_int))
        self.L.ref_copy_leaves(_p(boxes, C.c_double), _p(fl, C.c_int))
        return dict(cand_sten=cs, cand_is_vf=cv, hit_sten=hs, hit_is_vf=hv, hit_toi=ht,
                    discrete=dp, leaf_boxes=boxes, leaf_flags=fl)

    def accd(self, V0, V1, sten, is_vf, vf_eta, ee_eta=None):
        V0 = np.ascontiguousarray(V0, np.float64)
        V1 = np.ascontiguousarray(V1, np.float64)
        s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        v = np.ascontiguousarray(is_vf, np.uint8).reshape(-1)
        n = len(s)
        hit = np.empty(n, np.int32); toi = np.empty(n, np.float64)
        self.L.ref_accd(V0.shape[1], _p(V0, C.c_double), _p(V1, C.c_double), _p(s, C.c_int), _p(v, C.c_ubyte), n,
                        vf_eta, vf_eta if ee_eta is None else ee_eta, _p(hit, C.c_int), _p(toi, C.c_double))
        return hit, toi

    def ctcd_vf(self, V0, V1, sten, eta):
        """The reference's NarrowPhaseCTCD::query_ccd_vf with the wrong-side
        test, per stencil: (ret, toi); ret 1 hit, 0 none, -1 wrong side only."""
        V0 = np.ascontiguousarray(V0, np.float64)
        V1 = np.ascontiguousarray(V1, np.float64)
        s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        n = len(s)
        ret = np.empty(n, np.int32); toi = np.empty(n, np.float64)
        self.L.ref_ctcd_vf(V0.shape[1], _p(V0, C.c_double), _p(V1, C.c_double), _p(s, C.c_int), n, eta,
                           _p(ret, C.c_int), _p(toi, C.c_double))
        return ret, toi

    def rpoly(self, op):
        """The reference's Jenkins-Traub root finder on op (descending
        powers): complex roots as a numpy array (root count it reports)."""
        c = np.array(op, np.float64)
        n = len(c) - 1
        re = np.zeros(n); im = np.zeros(n)
        k = self.L.ref_rpoly(_p(c, C.c_double), n, _p(re, C.c_double), _p(im, C.c_double))
        return (re + 1j * im)[:max(k, 0)]

    def discrete(self, V, F, pairs):
        V = np.ascontiguousarray(V, np.float64)
        F = np.ascontiguousarray(F, np.int32)
        pr = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        out = np.empty(len(pr), np.int32)
        self.L.ref_discrete(V.shape[1], _p(V, C.c_double), _p(F, C.c_int), _p(pr, C.c_int), len(pr), _p(out, C.c_int))
        return out

    def time(self, V0, V1, F, eta, V1b=None, threaded=True):
        V0 = np.ascontiguousarray(V0, np.float64)
        V1 = np.ascontiguousarray(V1, np.float64)
        V1b = None if V1b is None else np.ascontiguousarray(V1b, np.float64)
        F = np.ascontiguousarray(F, np.int32)
        a, b, c = C.c_double(), C.c_double(), C.c_double()
        nd = C.c_longlong()
        nh = self.L.ref_time(V0.shape[1], _p(V0, C.c_double), _p(V1, C.c_double), _p(V1b, C.c_double),
                             _p(F, C.c_int), F.shape[0], F.shape[1], eta, int(threaded),
                             C.byref(a), C.byref(b), C.byref(c), C.byref(nd))
        return dict(ms_update_first=a.value, ms_update_again=b.value, ms_traverse=c.value,
                    n_hits=nh, n_discrete=nd.value, threads=self.L.ref_threads())


    def time_steps(self, V0, V1a, V1b, F, eta, steps):
        """The benchmark step on the reference (ref_time_steps): per step the
        update + traverse ms and the candidate stencils, V1 alternating
        between V1b and V1a after an untimed first update with V1a."""
        V0, V1a, V1b = (np.ascontiguousarray(x, np.float64) for x in (V0, V1a, V1b))
        F = np.ascontiguousarray(F, np.int32)
        ms = np.zeros(steps); st = np.zeros(steps, np.int64)
        self.L.ref_time_steps(V0.shape[1], _p(V0, C.c_double), _p(V1a, C.c_double), _p(V1b, C.c_double),
                              _p(F, C.c_int), F.shape[0], F.shape[1], eta, steps, _p(ms, C.c_double),
                              st.ctypes.data_as(C.POINTER(C.c_longlong)))
        return {"ms": [float(x) for x in ms], "stencils": [int(x) for x in st], "threads": self.L.ref_threads()}


FLAG_ACTIVE = 1 << 6


class Port:
    """This project's C restatement of the same path (oracle/port.c)."""

    def __init__(self, path: str = PORT_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle port not built: {path} (make -C oracle port)")
        L = C.CDLL(path)
        L.port_leaf_boxes.argtypes = [C.c_int, _dp, _dp, _ip, C.c_int, C.c_int, C.c_double, _ip, _dp, _ucp]
        L.port_reptri.argtypes = [_ip, C.c_int, C.c_int, C.c_int, _ucp]
        L.port_reptri.restype = C.c_int
        L.port_leaf_pairs.argtypes = [C.c_int, _dp, _ucp, C.c_int, _ip, C.c_longlong]
        L.port_leaf_pairs.restype = C.c_longlong
        L.port_candidates.argtypes = [C.c_int, _ip, _ucp, _ip, C.c_longlong, _ip, _ucp, C.c_longlong]
        L.port_candidates.restype = C.c_longlong
        L.port_accd.argtypes = [C.c_int, _dp, _dp, _ip, _ucp, C.c_longlong, C.c_double, C.c_double, _ip, _dp, _ip]
        L.port_discrete.argtypes = [C.c_int, _dp, _ip, _ip, C.c_longlong, _ip]
        L.port_additive_ccd.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_int, _dp, _ip]
        L.port_additive_ccd.restype = C.c_int
        L.adj_ref_row.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, _dp, _dp]
        L.adj_ref_row.restype = C.c_int
        L.adj_ref_batch.argtypes = [C.c_int, _dp, _dp, _ip, _ucp, _dp, C.c_longlong, C.c_double, C.c_double, _dp,
                                    _ip, _dp]
        L.adj_ref_fd.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.adj_ref_fd.restype = C.c_int
        self.L = L

    def leaf_boxes(self, V0, V1, F, eta, active=None, flags=None):
        V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
        F = np.ascontiguousarray(F, np.int32)
        dim = V0.shape[1]
        np_, pdim = F.shape
        boxes = np.empty((np_, 6, dim), np.float64)
        flags = np.zeros(np_, np.uint8) if flags is None else np.ascontiguousarray(flags, np.uint8)
        act = None if active is None else np.ascontiguousarray(active, np.int32)
        self.L.port_leaf_boxes(dim, _p(V0, C.c_double), _p(V1, C.c_double), _p(F, C.c_int), np_, pdim, eta,
                               _p(act, C.c_int), _p(boxes, C.c_double), _p(flags, C.c_ubyte))
        return boxes, flags

    def reptri(self, F, nv, flags):
        F = np.ascontiguousarray(F, np.int32)
        assert self.L.port_reptri(_p(F, C.c_int), F.shape[0], F.shape[1], nv, _p(flags, C.c_ubyte)) == 0
        return flags

    def leaf_pairs(self, boxes, flags):
        np_, _, dim = boxes.shape
        cap = max(16, 8 * np_)
        while True:
            out = np.empty((cap, 2), np.int32)
            n = self.L.port_leaf_pairs(dim, _p(boxes, C.c_double), _p(flags, C.c_ubyte), np_, _p(out, C.c_int), cap)
            if n <= cap:
                return out[:n]
            cap = n

    def candidates(self, F, flags, pairs):
        F = np.ascontiguousarray(F, np.int32)
        pairs = np.ascontiguousarray(pairs, np.int32)
        cap = max(16, 15 * len(pairs))
        s = np.empty((cap, 4), np.int32); v = np.empty(cap, np.uint8)
        n = self.L.port_candidates(F.shape[1], _p(F, C.c_int), _p(flags, C.c_ubyte), _p(pairs, C.c_int), len(pairs),
                                   _p(s, C.c_int), _p(v, C.c_ubyte), cap)
        return s[:n], v[:n]

    def accd(self, V0, V1, sten, is_vf, vf_eta, ee_eta=None, want_iters=False):
        V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
        s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        v = np.ascontiguousarray(is_vf, np.uint8).reshape(-1)
        n = len(s)
        hit = np.empty(n, np.int32); toi = np.empty(n, np.float64)
        it = np.empty(n, np.int32) if want_iters else None
        self.L.port_accd(V0.shape[1], _p(V0, C.c_double), _p(V1, C.c_double), _p(s, C.c_int), _p(v, C.c_ubyte), n,
                         vf_eta, vf_eta if ee_eta is None else ee_eta, _p(hit, C.c_int), _p(toi, C.c_double),
                         _p(it, C.c_int))
        return (hit, toi, it) if want_iters else (hit, toi)

    def discrete(self, V, F, pairs):
        V = np.ascontiguousarray(V, np.float64); F = np.ascontiguousarray(F, np.int32)
        pr = np.ascontiguousarray(pairs, np.int32).reshape(-1, 2)
        out = np.empty(len(pr), np.int32)
        self.L.port_discrete(V.shape[1], _p(V, C.c_double), _p(F, C.c_int), _p(pr, C.c_int), len(pr), _p(out, C.c_int))
        return out

    def run(self, V0, V1, F, box_eta, vf_eta=None, ee_eta=None, reptri=True, discrete=True, continuous=True,
            active=None):
        """update + traverse restated; outputs in canonical orientation
        (lower primitive index first for EE stencils and discrete pairs)."""
        vf_eta = box_eta if vf_eta is None else min(vf_eta, box_eta)
        ee_eta = box_eta if ee_eta is None else min(ee_eta, box_eta)
        F = np.ascontiguousarray(F, np.int32)
        boxes, flags = self.leaf_boxes(V0, V1, F, box_eta, active)
        if reptri:
            self.reptri(F, len(V0), flags)
        else:
            flags |= 0x3F
        pairs = self.leaf_pairs(boxes, flags) if len(F) > 1 else np.zeros((0, 2), np.int32)
        out = dict(leaf_boxes=boxes, leaf_flags=flags, leaf_pairs=pairs)
        if continuous:
            cs, cv = self.candidates(F, flags, pairs)
            hit, toi = self.accd(V0, V1, cs, cv, vf_eta, ee_eta)
            m = (hit == 1) & (toi >= 0)   # collide() delivers only toi >= 0 (BVHTree.cpp:262)
            out.update(cand_sten=cs, cand_is_vf=cv, hit_sten=cs[m], hit_is_vf=cv[m], hit_toi=toi[m])
        else:
            e = np.zeros((0, 4), np.int32)
            out.update(cand_sten=e, cand_is_vf=e[:, 0].astype(np.uint8), hit_sten=e,
                       hit_is_vf=e[:, 0].astype(np.uint8), hit_toi=np.zeros(0))
        if discrete:
            d = self.discrete(V1, F, pairs)
            out["discrete"] = pairs[d == 1]
        else:
            out["discrete"] = np.zeros((0, 2), np.int32)
        return out

    # --- adjoint of the time of impact (oracle/adjoint_ref.c) ---
    def vjp_rows(self, V0, V1, sten, is_vf, toi, vf_eta, ee_eta=None):
        """Per hit: (t_star, status, rows) with rows = d(t*)/d(V0 slots, V1 slots)."""
        dim = V0.shape[1]
        ee_eta = vf_eta if ee_eta is None else ee_eta
        V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
        sten = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        is_vf = np.ascontiguousarray(is_vf, np.uint8); toi = np.ascontiguousarray(toi, np.float64)
        n = len(sten)
        ts = np.zeros(n); st = np.zeros(n, np.int32); rows = np.zeros((n, 2 * (dim + 1) * dim))
        self.L.adj_ref_batch(dim, _p(V0, C.c_double), _p(V1, C.c_double), _p(sten, C.c_int), _p(is_vf, C.c_ubyte),
                             _p(toi, C.c_double), n, vf_eta, ee_eta, _p(ts, C.c_double), _p(st, C.c_int),
                             _p(rows, C.c_double))
        return ts, st, rows

    def vjp_fd(self, v0, v1, is_vf, eta, toi, h=1e-7):
        """Central differences of t* over one stencil's coordinates (v0, v1: (dim+1) x dim)."""
        v0 = np.ascontiguousarray(v0, np.float64); v1 = np.ascontiguousarray(v1, np.float64)
        dim = v0.shape[1]
        out = np.zeros(2 * (dim + 1) * dim)
        st = self.L.adj_ref_fd(dim, int(is_vf), _p(v0, C.c_double), _p(v1, C.c_double), eta, toi, h,
                               _p(out, C.c_double))
        return st, out


class Flops:
    """FP64 flop count of the narrow phase on the oracle (oracle/flops.cpp):
    per kind, the reference loop's flops and the necessary flops (the
    device's form), with both forms' (hit, toi) for checking."""

    def __init__(self, path: str = FLOPS_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(f"flop counter not built: {path} (make -C oracle port)")
        L = C.CDLL(path)
        L.flops_accd.argtypes = [C.c_int, _dp, _dp, _ip, _ucp, C.c_longlong, C.c_double, C.c_double,
                                 C.POINTER(C.c_longlong), _ip, _dp, _ip, _dp]
        self.L = L

    def accd(self, V0, V1, sten, is_vf, vf_eta, ee_eta=None):
        V0 = np.ascontiguousarray(V0, np.float64); V1 = np.ascontiguousarray(V1, np.float64)
        s = np.ascontiguousarray(sten, np.int32).reshape(-1, 4)
        v = np.ascontiguousarray(is_vf, np.uint8).reshape(-1)
        n = len(s)
        out = np.zeros(8, np.int64)
        hit = np.empty(n, np.int32); toi = np.empty(n); hf = np.empty(n, np.int32); tf = np.empty(n)
        self.L.flops_accd(V0.shape[1], _p(V0, C.c_double), _p(V1, C.c_double), _p(s, C.c_int), _p(v, C.c_ubyte), n,
                          vf_eta, vf_eta if ee_eta is None else ee_eta, out.ctypes.data_as(C.POINTER(C.c_longlong)),
                          _p(hit, C.c_int), _p(toi, C.c_double), _p(hf, C.c_int), _p(tf, C.c_double))
        kinds = {}
        for name, k in (("ee", 0), ("vf", 1)):
            o = out[4 * k: 4 * k + 4]
            kinds[name] = {"stencils": int(o[0]), "reference_flops": int(o[1]), "necessary_flops": int(o[2]),
                           "reference_distances": int(o[3])}
        return kinds, (hit, toi), (hf, tf)
