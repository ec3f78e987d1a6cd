"""TEST INFRASTRUCTURE ONLY: ctypes bindings for the checker libraries.

* ``liboracle.so`` -- the plain-C restatement of the reference search path
  (sc_oracle.c).
* ``_ref/libscref.so`` -- the reference's own headers and sources compiled by
  oracle/Makefile, driven through ref_harness.cpp.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only to check or to time beside the CUDA library.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libscref.so")

IVFADC, IMI, SC, SC3 = 0, 1, 2, 3
ORDER_HEAP, ORDER_EXACT = 0, 1

_f32p = ctypes.POINTER(ctypes.c_float)
_i32p = ctypes.POINTER(ctypes.c_int)
_u8p = ctypes.POINTER(ctypes.c_ubyte)
_u16p = ctypes.POINTER(ctypes.c_ushort)


def build(ref=True):
    """Builds liboracle.so, and the reference harness when the reference tree
    is readable (oracle/Makefile decides: SCG_REFERENCE_TREE or its default;
    without the tree an existing _ref/libscref.so is kept as it is)."""
    targets = ["oracle"]
    if ref:
        targets.append("ref-if-present")
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def ref_available():
    return os.path.exists(REF_SO)


def _p(a, t):
    return a.ctypes.data_as(t)


class _OrcIndex(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("mc", ctypes.c_int), ("kc", ctypes.c_int),
                ("mp", ctypes.c_int), ("kp", ctypes.c_int), ("N", ctypes.c_int),
                ("cq", _f32p), ("pq", _f32p), ("norm_c", _f32p), ("norm_r", _f32p),
                ("dot_cr", _f32p), ("L", _i32p), ("pid", _i32p), ("codes", _u8p),
                ("raw", _f32p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.orc_search.restype = ctypes.c_int
        _lib.orc_distribution.restype = ctypes.c_int
        _lib.orc_distance_l2_square.restype = ctypes.c_double
        _lib.orc_rerank.restype = ctypes.c_int
    return _lib


def pre_compute1(cfg, cq, pq):
    """PQQuery::pre_compute1 (query.h:91-149)."""
    dim, mc, kc, mp, kp = cfg
    norm_c = np.zeros(mc * kc, np.float32)
    norm_r = np.zeros(mp * kp, np.float32)
    dot_cr = np.zeros(kc * kp * mp, np.float32)
    lib().orc_pre_compute1(dim, mc, kc, mp, kp, _p(cq, _f32p), _p(pq, _f32p),
                           _p(norm_c, _f32p), _p(norm_r, _f32p), _p(dot_cr, _f32p))
    return norm_c, norm_r, dot_cr


def pre_compute2(cfg, cq, pq, norm_c, norm_r, q):
    """PQQuery::pre_compute2 (query.h:154-184), intended sequencing."""
    dim, mc, kc, mp, kp = cfg
    dqc = np.zeros(mc * kc, np.float32)
    dqr = np.zeros(mp * kp, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    lib().orc_pre_compute2(dim, mc, kc, mp, kp, _p(cq, _f32p), _p(pq, _f32p),
                           _p(norm_c, _f32p), _p(norm_r, _f32p), _p(q, _f32p),
                           _p(dqc, _f32p), _p(dqr, _f32p))
    return dqc, dqr


class Index:
    """An index held the way the reference holds it (query.h:45-61)."""

    def __init__(self, dim, mc, kc, mp, kp, cq, pq, L, pid, codes, raw=None):
        self.dim, self.mc, self.kc, self.mp, self.kp = dim, mc, kc, mp, kp
        self.cq = np.ascontiguousarray(cq, np.float32).ravel()
        self.pq = np.ascontiguousarray(pq, np.float32).ravel()
        self.L = np.ascontiguousarray(L, np.int32)
        self.pid = np.ascontiguousarray(pid, np.int32)
        self.codes = np.ascontiguousarray(codes, np.uint8).ravel()
        self.N = int(self.pid.shape[0])
        self.raw = None if raw is None else np.ascontiguousarray(raw, np.float32).ravel()
        self.norm_c, self.norm_r, self.dot_cr = pre_compute1(self.cfg, self.cq, self.pq)
        self._s = _OrcIndex(dim, mc, kc, mp, kp, self.N,
                            _p(self.cq, _f32p), _p(self.pq, _f32p),
                            _p(self.norm_c, _f32p), _p(self.norm_r, _f32p),
                            _p(self.dot_cr, _f32p), _p(self.L, _i32p),
                            _p(self.pid, _i32p), _p(self.codes, _u8p),
                            _p(self.raw, _f32p) if self.raw is not None else None)

    @property
    def cfg(self):
        return (self.dim, self.mc, self.kc, self.mp, self.kp)

    def search_one(self, mode, q, w, T, order=ORDER_EXACT, real_dist=False, rank_limit=0):
        """All candidates of one query in visiting order plus the visited
        non-empty cells: dict(dist, ids, cells, sum, empty, max_rank).
        rank_limit > 0 confines the IMI / second-candidate walk to ranks
        0..rank_limit-1 of each sorted coarse list."""
        q = np.ascontiguousarray(q, np.float32)
        cap = self.N
        dist = np.zeros(max(cap, 1), np.float32)
        ids = np.zeros(max(cap, 1), np.int32)
        cells = np.zeros(max(cap, 1), np.int32)
        ncells = ctypes.c_int(0)
        s = ctypes.c_int(0)
        e = ctypes.c_int(0)
        lib().orc_set_rank_limit(int(rank_limit))
        try:
            rc = lib().orc_search(ctypes.byref(self._s), mode, order, _p(q, _f32p), w, T,
                                  1 if real_dist else 0, _p(dist, _f32p), _p(ids, _i32p), cap,
                                  _p(cells, _i32p), cap, ctypes.byref(ncells), ctypes.byref(s),
                                  ctypes.byref(e))
        finally:
            lib().orc_set_rank_limit(0)
        if rc != 0:
            raise RuntimeError("orc_search failed: %d" % rc)
        n = s.value
        return dict(dist=dist[:n].copy(), ids=ids[:n].copy(), cells=cells[:ncells.value].copy(),
                    sum=n, empty=e.value, max_rank=int(lib().orc_last_max_rank()))

    def search(self, mode, Q, R, w, T, order=ORDER_EXACT, real_dist=False, rank_limit=0):
        """Top-R per query (ascending distance; equal distances by id), the
        way the reference's top-R step orders them.  Returns
        (ids[nq,R] padded with -1, dist[nq,R] padded with +inf, sums[nq])."""
        Q = np.ascontiguousarray(Q, np.float32).reshape(-1, self.dim)
        nq = Q.shape[0]
        out_i = np.full((nq, R), -1, np.int32)
        out_d = np.full((nq, R), np.inf, np.float32)
        sums = np.zeros(nq, np.int32)
        for i in range(nq):
            r = self.search_one(mode, Q[i], w, T, order, real_dist, rank_limit)
            m = min(R, r["sum"])
            td = np.zeros(max(m, 1), np.float32)
            ti = np.zeros(max(m, 1), np.int32)
            lib().orc_topk(_p(r["dist"], _f32p), _p(r["ids"], _i32p), r["sum"], R,
                           _p(td, _f32p), _p(ti, _i32p))
            out_i[i, :m] = ti[:m]
            out_d[i, :m] = td[:m]
            sums[i] = r["sum"]
        return out_i, out_d, sums

    def rerank(self, Q, ids, R):
        """Shortlist re-rank (orc_rerank): ids[nq, L] (-1 = none) -> the R
        smallest exact distances per query, (ids[nq,R] padded with -1,
        dist[nq,R] padded with +inf)."""
        if self.raw is None:
            raise ValueError("raw vectors not given")
        Q = np.ascontiguousarray(Q, np.float32).reshape(-1, self.dim)
        ids = np.ascontiguousarray(ids, np.int32)
        nq, L = ids.shape
        out_i = np.full((nq, R), -1, np.int32)
        out_d = np.full((nq, R), np.inf, np.float32)
        ti = np.zeros(R, np.int32)
        td = np.zeros(R, np.float32)
        for i in range(nq):
            q = np.ascontiguousarray(Q[i])
            row = np.ascontiguousarray(ids[i])
            m = lib().orc_rerank(_p(self.raw, _f32p), self.dim, _p(q, _f32p), _p(row, _i32p), L, R,
                                 _p(ti, _i32p), _p(td, _f32p))
            out_i[i, :m] = ti[:m]
            out_d[i, :m] = td[:m]
        return out_i, out_d


def encode(cfg, cq, pq, X):
    """Encoder::encode<T> (encoder.h:69-192): (cid[n,mc] uint16, codes[n,mp])."""
    dim, mc, kc, mp, kp = cfg
    X = np.ascontiguousarray(X, np.float32)
    n = X.shape[0]
    cid = np.zeros((n, mc), np.uint16)
    codes = np.zeros((n, mp), np.uint8)
    lib().orc_encode(dim, mc, kc, mp, kp, _p(np.ascontiguousarray(cq, np.float32), _f32p),
                     _p(np.ascontiguousarray(pq, np.float32), _f32p), _p(X, _f32p),
                     ctypes.c_long(n), _p(cid, _u16p), _p(codes, _u8p))
    return cid, codes


def sc_encode(dim, kc, mp, kp, nc, cq, pq, X):
    """SCEncoder::encode<T> (sc_encoder.h:205-332, mc = 1)."""
    X = np.ascontiguousarray(X, np.float32)
    n = X.shape[0]
    cid = np.zeros((n, nc), np.uint16)
    codes = np.zeros((n, mp), np.uint8)
    lib().orc_sc_encode(dim, kc, mp, kp, nc, _p(np.ascontiguousarray(cq, np.float32), _f32p),
                        _p(np.ascontiguousarray(pq, np.float32), _f32p), _p(X, _f32p),
                        ctypes.c_long(n), _p(cid, _u16p), _p(codes, _u8p))
    return cid, codes


def distribution(mode, kc, mc, nc, cid, codes):
    """Encoder/SCEncoder::distribution + the CSR of load_encoded_data:
    (L inclusive prefix, pid, codes in cell order, non_empty)."""
    cid = np.ascontiguousarray(cid, np.uint16)
    codes = np.ascontiguousarray(codes, np.uint8)
    n, mp = codes.shape
    parts = nc if mode == SC else mc
    ncells = kc ** parts
    L = np.zeros(ncells, np.int32)
    pid = np.zeros(n, np.int32)
    co = np.zeros((n, mp), np.uint8)
    ne = lib().orc_distribution(mode, kc, mc, nc, mp, ctypes.c_long(n), _p(cid, _u16p),
                                _p(codes, _u8p), _p(L, _i32p), _p(pid, _i32p), _p(co, _u8p))
    return L, pid, co, ne


# --------------------------------------------------------------------------
# The reference itself (oracle/_ref/libscref.so)

_ref = None


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        _ref = ctypes.CDLL(REF_SO)
        _ref.ref_search_batch.restype = ctypes.c_int
        _ref.ref_search_batch_ex.restype = ctypes.c_int
        _ref.ref_search_one.restype = ctypes.c_int
        _ref.ref_encode.restype = ctypes.c_int
        _ref.ref_calc_recall.restype = ctypes.c_int
        _ref.ref_calc_comb_recall.restype = ctypes.c_int
    return _ref


def ref_tables(cfg, cq, pq, q):
    dim, mc, kc, mp, kp = cfg
    out = [np.zeros(mc * kc, np.float32), np.zeros(mp * kp, np.float32),
           np.zeros(kc * kp * mp, np.float32), np.zeros(mc * kc, np.float32),
           np.zeros(mp * kp, np.float32)]
    cq = np.ascontiguousarray(cq, np.float32)
    pq = np.ascontiguousarray(pq, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    ref().ref_tables(dim, mc, kc, mp, kp, _p(cq, _f32p), _p(pq, _f32p), _p(q, _f32p),
                     *[_p(a, _f32p) for a in out])
    return out


def _ref_index_args(ix):
    raw = _p(ix.raw, _f32p) if ix.raw is not None else None
    return (ix.dim, ix.mc, ix.kc, ix.mp, ix.kp, ix.N, _p(ix.cq, _f32p), _p(ix.pq, _f32p),
            _p(ix.L, _i32p), _p(ix.pid, _i32p), _p(ix.codes, _u8p), raw)


def ref_search_one(ix, mode, q, R, w, T, real_dist=False):
    """All `sum` (id, distance) pairs the reference leaves after one search."""
    q = np.ascontiguousarray(q, np.float32)
    cap = ix.N
    ids = np.zeros(max(cap, 1), np.int32)
    dist = np.zeros(max(cap, 1), np.float32)
    e = ctypes.c_int(0)
    s = ref().ref_search_one(mode, *_ref_index_args(ix), _p(q, _f32p), R, w, T,
                             1 if real_dist else 0, _p(ids, _i32p), _p(dist, _f32p), cap,
                             ctypes.byref(e))
    if s < 0:
        raise RuntimeError("capacity")
    return dict(ids=ids[:s].copy(), dist=dist[:s].copy(), sum=s, empty=e.value)


def ref_search_batch(ix, mode, Q, R, w, T, nthreads=0, real_dist=False, Tq=None, M=None):
    """Reference search over a query batch with OpenMP threads; Tq: optional
    per-query candidate targets; M: the coarse-list argument of search_multi2
    / search_mr_ivf (default kc).  Returns (ids[nq,R], dist[nq,R], sums[nq],
    seconds)."""
    Q = np.ascontiguousarray(Q, np.float32).reshape(-1, ix.dim)
    nq = Q.shape[0]
    ids = np.zeros((nq, R), np.int32)
    dist = np.zeros((nq, R), np.float32)
    sums = np.zeros(nq, np.int32)
    sec = ctypes.c_double(0.0)
    tq = None if Tq is None else np.ascontiguousarray(Tq, np.int32)
    rc = ref().ref_search_batch_ex(mode, *_ref_index_args(ix), _p(Q, _f32p), nq, R, w, T,
                                   _p(tq, _i32p) if tq is not None else None, ix.kc if M is None else M,
                                   1 if real_dist else 0, nthreads, _p(ids, _i32p),
                                   _p(dist, _f32p), _p(sums, _i32p), ctypes.byref(sec))
    if rc != 0:
        raise RuntimeError("ref_search_batch failed")
    return ids, dist, sums, sec.value


def ref_calc_recall(result, gt, R):
    """Evaluation::calc_recall of the reference: the count of queries whose
    ground truth is among the first R of result[N][R]."""
    result = np.ascontiguousarray(result, np.int32)
    gt = np.ascontiguousarray(gt, np.int32)
    return ref().ref_calc_recall(_p(result, _i32p), _p(gt, _i32p), R, result.shape[0])


def ref_calc_comb_recall(results, gt, R):
    """Evaluation::calc_comb_recall of the reference over S arrays [N][R]."""
    arrs = [np.ascontiguousarray(r, np.int32) for r in results]
    gt = np.ascontiguousarray(gt, np.int32)
    ptrs = (_i32p * len(arrs))(*[_p(a, _i32p) for a in arrs])
    return ref().ref_calc_comb_recall(ptrs, _p(gt, _i32p), R, arrs[0].shape[0], len(arrs))


def ref_encode(cq_path, pq_path, fvecs_path, nc, n, mc, mp, nthreads=0):
    cid = np.zeros((n, max(mc, nc)), np.uint16)
    codes = np.zeros((n, mp), np.uint8)
    got = ref().ref_encode(cq_path.encode(), pq_path.encode(), fvecs_path.encode(), nc,
                           nthreads, _p(cid, _u16p), _p(codes, _u8p), ctypes.c_long(n))
    if got != n:
        raise RuntimeError("ref_encode returned %d rows" % got)
    return cid, codes


def ref_build_edat(cq_path, pq_path, fvecs_path, nc, db_path, prefix):
    rc = ref().ref_build_edat(cq_path.encode(), pq_path.encode(), fvecs_path.encode(), nc,
                              db_path.encode(), prefix.encode())
    if rc != 0:
        raise RuntimeError("ref_build_edat failed")
