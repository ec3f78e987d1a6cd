"""Python binding of libscgpu.so (the C ABI in include/scg.h) via ctypes.

Used by the tests and by bench.py.  The library is built in-tree by
build.py; loading fails loudly when it cannot be built or loaded -- there is
no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# SCG_LIBRARY points at another build of the library (e.g. one compiled with
# different tuning defines); the default is the in-tree build.
LIB_PATH = os.environ.get("SCG_LIBRARY") or os.path.join(HERE, "libscgpu.so")

IVFADC, IMI, SC2, SC3 = 0, 1, 2, 3
FP32_EXACT, FAST, BF16, FP16 = 0, 1, 2, 3
ENC_EXACT, ENC_TENSOR = 0, 1

PENDING = 1

ERRORS = {-1: "SCG_ERR_ARG", -2: "SCG_ERR_OOM", -3: "SCG_ERR_IO", -4: "SCG_ERR_CUDA",
          -5: "SCG_ERR_CAP", -6: "SCG_ERR_STATE"}

EXPORTS = ["scg_last_error", "scg_index_create", "scg_index_destroy", "scg_load_codebooks",
           "scg_load_codebooks_file", "scg_load_csr", "scg_load_encoded_file", "scg_load_raw",
           "scg_precompute", "scg_search", "scg_search_device", "scg_set_query_targets",
           "scg_set_cell_budget", "scg_encode", "scg_sc_encode", "scg_encode_device",
           "scg_index_info", "scg_last_query_stats", "scg_last_timings",
           "scg_cell_counts", "scg_set_phase_counters", "scg_last_phase_counters",
           "scg_search_device_noalloc", "scg_query_tables_device", "scg_load_raw_u8",
           "scg_server_create", "scg_server_submit", "scg_server_wait", "scg_server_stats",
           "scg_server_destroy", "scg_autotune", "scg_set_scan_tuning",
           "scg_set_kernel_split", "scg_server_wait_times", "scg_set_encoder",
           "scg_train_codebooks", "scg_build_index", "scg_write_edat", "scg_search_graph",
           "scg_kmeans", "scg_exact_nn", "scg_set_rank_limit", "scg_autotune_ex",
           "scg_device_allocations", "scg_last_launches"]


def train_codebooks_device(dX_ptr, n, dim, mc, kc, mp, kp, iters, seed, d_cq, d_pq, device=0, stream=None):
    """k-means++ + Lloyd codebooks on the device (scg_train_codebooks)."""
    lib = load()
    _check(lib.scg_train_codebooks(ctypes.c_void_p(dX_ptr), ctypes.c_int64(n), dim, mc, kc, mp, kp, iters,
                                   ctypes.c_uint64(seed), ctypes.c_void_p(d_cq), ctypes.c_void_p(d_pq), device,
                                   ctypes.c_void_p(stream) if stream else None))



def exact_nn_device(dX_ptr, n, dQ_ptr, nq, dim, d_ids, d_dists=None, device=0, stream=None):
    """Exact nearest base row of each query, device buffers (scg_exact_nn)."""
    lib = load()
    _check(lib.scg_exact_nn(ctypes.c_void_p(dX_ptr), ctypes.c_int64(n), ctypes.c_void_p(dQ_ptr), nq, dim,
                            ctypes.c_void_p(d_ids), ctypes.c_void_p(d_dists) if d_dists else None, device,
                            ctypes.c_void_p(stream) if stream else None))


class ScgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (ERRORS.get(code, code), msg))
        self.code = code


class SearchParams(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("R", ctypes.c_int), ("w", ctypes.c_int),
                ("T", ctypes.c_int), ("precision", ctypes.c_int), ("rerank", ctypes.c_int)]


class TuneRecord(ctypes.Structure):
    """scg_tune_record (include/scg.h)."""
    _fields_ = [("upl", ctypes.c_int), ("upl_ms", ctypes.c_float * 3),
                ("prefix", ctypes.c_int), ("prefix_ms", ctypes.c_float * 4),
                ("split", ctypes.c_int), ("split_ms", ctypes.c_float * 2),
                ("shortlist", ctypes.c_int), ("shortlist_L", ctypes.c_int * 5),
                ("shortlist_ms", ctypes.c_float * 5), ("shortlist_agree", ctypes.c_float * 5)]


_lib = None


def load(build_if_missing=True):
    """Loads libscgpu.so, building it first when it is missing or stale."""
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and LIB_PATH == os.path.join(HERE, "libscgpu.so"):
        import importlib.util
        spec = importlib.util.spec_from_file_location("scg_build", os.path.join(HERE, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    _lib = ctypes.CDLL(LIB_PATH)
    for name in EXPORTS:
        getattr(_lib, name).restype = ctypes.c_int
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _check(rc):
    if rc != 0:
        buf = ctypes.create_string_buffer(1024)
        _lib.scg_last_error(buf, 1024)
        raise ScgError(rc, buf.value.decode(errors="replace"))


class Index:
    """One device-resident index (codebooks, CSR codes, tables)."""

    def __init__(self, device=0):
        lib = load()
        self._h = ctypes.c_void_p()
        _check(lib.scg_index_create(ctypes.byref(self._h), device))

    def close(self):
        if self._h:
            _lib.scg_index_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def load_codebooks(self, cq, kc, mc, pq, kp, mp, dim):
        cq = np.ascontiguousarray(cq, np.float32)
        pq = np.ascontiguousarray(pq, np.float32)
        _check(_lib.scg_load_codebooks(self._h, _ptr(cq), kc, mc, _ptr(pq), kp, mp, dim))
        self.dim, self.mc, self.kc, self.mp, self.kp = dim, mc, kc, mp, kp

    def load_codebooks_file(self, cq_path, pq_path):
        _check(_lib.scg_load_codebooks_file(self._h, cq_path.encode(), pq_path.encode()))
        self._refresh_info()

    def _refresh_info(self):
        v = [ctypes.c_int() for _ in range(5)]
        n = ctypes.c_int64()
        _check(_lib.scg_index_info(self._h, *[ctypes.byref(x) for x in v], ctypes.byref(n)))
        self.dim, self.mc, self.kc, self.mp, self.kp = (x.value for x in v)
        self.N = n.value

    def load_csr(self, L, pid, codes):
        L = np.ascontiguousarray(L, np.int32)
        pid = np.ascontiguousarray(pid, np.int32)
        codes = np.ascontiguousarray(codes, np.uint8)
        _check(_lib.scg_load_csr(self._h, _ptr(L), _ptr(pid), _ptr(codes),
                                 ctypes.c_int64(pid.shape[0]), ctypes.c_int64(L.shape[0])))
        self.N = pid.shape[0]

    def load_encoded_file(self, path, nc):
        _check(_lib.scg_load_encoded_file(self._h, path.encode(), nc))
        self._refresh_info()

    def load_raw(self, X):
        """Raw vectors for the shortlist re-rank: float32, or uint8 kept as uint8."""
        if X.dtype == np.uint8:
            X = np.ascontiguousarray(X)
            _check(_lib.scg_load_raw_u8(self._h, _ptr(X), ctypes.c_int64(X.shape[0])))
        else:
            X = np.ascontiguousarray(X, np.float32)
            _check(_lib.scg_load_raw(self._h, _ptr(X), ctypes.c_int64(X.shape[0])))

    def precompute(self):
        _check(_lib.scg_precompute(self._h))

    def set_cell_budget(self, n):
        _check(_lib.scg_set_cell_budget(self._h, n))

    def search(self, mode, Q, R, w, T, precision=FP32_EXACT, rerank=0, out=None):
        """Host-buffer search: returns (ids[nq,R], dists[nq,R], sums[nq]).
        `out` may hold caller-owned (ids, dists, sums) arrays to fill (e.g.
        in pinned memory)."""
        Q = np.ascontiguousarray(Q, np.float32).reshape(-1, self.dim)
        nq = Q.shape[0]
        if out is not None:
            ids, d, sums = out
            assert ids.shape == (nq, R) and d.shape == (nq, R) and sums.shape == (nq,)
            assert ids.flags.c_contiguous and d.flags.c_contiguous and sums.flags.c_contiguous
        else:
            ids = np.empty((nq, R), np.int32)
            d = np.empty((nq, R), np.float32)
            sums = np.empty(nq, np.int32)
        p = SearchParams(mode, R, w, T, precision, rerank)
        _check(_lib.scg_search(self._h, ctypes.byref(p), _ptr(Q), nq, _ptr(ids), _ptr(d), _ptr(sums)))
        return ids, d, sums

    def search_device(self, mode, dQ_ptr, nq, R, w, T, d_ids, d_d, d_sums, stream=None,
                      precision=FP32_EXACT, rerank=0):
        """Device-buffer search; arguments are raw device addresses (ints)."""
        p = SearchParams(mode, R, w, T, precision, rerank)
        _check(_lib.scg_search_device(self._h, ctypes.byref(p), ctypes.c_void_p(dQ_ptr), nq,
                                      ctypes.c_void_p(d_ids), ctypes.c_void_p(d_d),
                                      ctypes.c_void_p(d_sums),
                                      ctypes.c_void_p(stream) if stream else None))

    def search_graph(self, mode, dQ_ptr, nq, R, w, T, d_ids, d_d, d_sums, stream, precision=FP32_EXACT, rerank=0):
        """Device-buffer search replayed from a captured CUDA graph."""
        p = SearchParams(mode, R, w, T, precision, rerank)
        _check(_lib.scg_search_graph(self._h, ctypes.byref(p), ctypes.c_void_p(dQ_ptr), nq, ctypes.c_void_p(d_ids),
                                     ctypes.c_void_p(d_d), ctypes.c_void_p(d_sums), ctypes.c_void_p(stream)))

    def search_device_noalloc(self, mode, dQ_ptr, nq, R, w, T, d_ids, d_d, d_sums, stream=None,
                              precision=FP32_EXACT, rerank=0):
        """Device-buffer search that allocates nothing (scratch in a static
        device array); same arguments as search_device."""
        p = SearchParams(mode, R, w, T, precision, rerank)
        _check(_lib.scg_search_device_noalloc(self._h, ctypes.byref(p), ctypes.c_void_p(dQ_ptr), nq,
                                              ctypes.c_void_p(d_ids), ctypes.c_void_p(d_d),
                                              ctypes.c_void_p(d_sums),
                                              ctypes.c_void_p(stream) if stream else None))

    def query_tables_device(self, precision, dQ_ptr, nq, d_dqc, d_dqr, stream=None):
        """Batched per-query tables (diff_qc, diff_qr) into device buffers."""
        _check(_lib.scg_query_tables_device(self._h, precision, ctypes.c_void_p(dQ_ptr), nq,
                                            ctypes.c_void_p(d_dqc), ctypes.c_void_p(d_dqr),
                                            ctypes.c_void_p(stream) if stream else None))

    def autotune(self, mode, dQ_ptr, nq, R, w, T, d_ids, d_d, d_sums, precision=FP32_EXACT, rerank=0):
        """Times the scan variants on a device batch; returns (choice, ms[3])."""
        p = SearchParams(mode, R, w, T, precision, rerank)
        c = ctypes.c_int()
        ms = np.zeros(3, np.float32)
        _check(_lib.scg_autotune(self._h, ctypes.byref(p), ctypes.c_void_p(dQ_ptr), nq, ctypes.c_void_p(d_ids),
                                 ctypes.c_void_p(d_d), ctypes.c_void_p(d_sums), ctypes.byref(c), _ptr(ms)))
        return c.value, ms.tolist()

    def autotune_ex(self, mode, dQ_ptr, nq, R, w, T, d_ids, d_d, d_sums, precision=FP32_EXACT, rerank=0,
                    min_agree=0.99):
        """The wider autotuner (scg_autotune_ex): returns its record as a dict
        (each knob's candidates, their ms and the pick)."""
        p = SearchParams(mode, R, w, T, precision, rerank)
        r = TuneRecord()
        _check(_lib.scg_autotune_ex(self._h, ctypes.byref(p), ctypes.c_void_p(dQ_ptr), nq, ctypes.c_void_p(d_ids),
                                    ctypes.c_void_p(d_d), ctypes.c_void_p(d_sums), ctypes.c_float(min_agree),
                                    ctypes.byref(r)))
        out = {"candidates_per_lane": {"pick": r.upl, "ms_by_choice": dict(zip((2, 4, 8), list(r.upl_ms)))},
               "coarse_prefix": {"pick": r.prefix, "ms_by_choice": dict(zip((0, 128, 256, 512), list(r.prefix_ms)))},
               "kernel_split": {"pick": r.split, "ms_by_choice": {1: r.split_ms[0], 0: r.split_ms[1]}}}
        if rerank > 0:
            out["shortlist"] = {"pick": r.shortlist,
                                "by_length": {int(L): {"ms": float(m), "agree": float(a)}
                                              for L, m, a in zip(r.shortlist_L, r.shortlist_ms, r.shortlist_agree)
                                              if L > 0}}
        return out

    def build_index_device(self, dX_ptr, n, nc=0, stream=None):
        """Encodes device rows and loads the CSR built on the device."""
        _check(_lib.scg_build_index(self._h, ctypes.c_void_p(dX_ptr), ctypes.c_int64(n), nc,
                                    ctypes.c_void_p(stream) if stream else None))
        self.N = n

    def write_edat(self, path):
        _check(_lib.scg_write_edat(self._h, str(path).encode()))

    def set_encoder(self, method):
        _check(_lib.scg_set_encoder(self._h, method))

    def set_kernel_split(self, on):
        _check(_lib.scg_set_kernel_split(self._h, 1 if on else 0))

    def set_scan_tuning(self, precision, upl):
        _check(_lib.scg_set_scan_tuning(self._h, precision, upl))

    def set_query_targets(self, d_T_ptr):
        _check(_lib.scg_set_query_targets(self._h, ctypes.c_void_p(d_T_ptr) if d_T_ptr else None))

    def set_rank_limit(self, M):
        """Walk only ranks 0..M-1 of each sorted coarse list (0: all)."""
        _check(_lib.scg_set_rank_limit(self._h, int(M)))

    def last_query_stats(self, nq):
        nvis = np.empty(nq, np.int32)
        empty = np.empty(nq, np.int32)
        _check(_lib.scg_last_query_stats(self._h, _ptr(nvis), _ptr(empty), nq))
        return nvis, empty

    def set_phase_counters(self, on):
        _check(_lib.scg_set_phase_counters(self._h, 1 if on else 0))

    def last_phase_counters(self):
        out = np.zeros(16, np.int64)
        _check(_lib.scg_last_phase_counters(self._h, _ptr(out), 16))
        names = ["sort", "rounds", "cut", "compact", "scan", "final_merge", "pending", "deferred", "round_count",
                 "bisection_steps", "enumerated_cells", "full_sorts", "lut_fill", "warm_threshold", "bisection", "select_warp"]
        return {n: int(v) for n, v in zip(names, out) if n != "-"}

    def last_timings(self):
        """Device ms of the last search: (tables, selection + scan, re-rank,
        selection kernel, scan kernel) -- the last two 0 for the fused kernel."""
        ms = np.zeros(5, np.float32)
        _check(_lib.scg_last_timings(self._h, _ptr(ms), 5))
        return tuple(float(x) for x in ms)

    def last_launches(self):
        """Kernels the last search launched on the index's own stream."""
        c = ctypes.c_int()
        _check(_lib.scg_last_launches(self._h, ctypes.byref(c)))
        return c.value

    def encode(self, X):
        X = np.ascontiguousarray(X, np.float32)
        n = X.shape[0]
        cid = np.empty((n, self.mc), np.uint16)
        codes = np.empty((n, self.mp), np.uint8)
        _check(_lib.scg_encode(self._h, _ptr(X), ctypes.c_int64(n), _ptr(cid), _ptr(codes)))
        return cid, codes

    def sc_encode(self, X, nc=2):
        X = np.ascontiguousarray(X, np.float32)
        n = X.shape[0]
        cid = np.empty((n, nc), np.uint16)
        codes = np.empty((n, self.mp), np.uint8)
        _check(_lib.scg_sc_encode(self._h, _ptr(X), ctypes.c_int64(n), nc, _ptr(cid), _ptr(codes)))
        return cid, codes

    def encode_device(self, dX_ptr, n, nc, d_cid, d_codes, stream=None):
        _check(_lib.scg_encode_device(self._h, ctypes.c_void_p(dX_ptr), ctypes.c_int64(n), nc,
                                      ctypes.c_void_p(d_cid), ctypes.c_void_p(d_codes),
                                      ctypes.c_void_p(stream) if stream else None))


def device_allocations():
    """cudaMalloc calls the library has made for its own buffers so far."""
    load()
    c = ctypes.c_longlong()
    _check(_lib.scg_device_allocations(ctypes.byref(c)))
    return c.value


class Server:
    """Request loop with continuous batching over one Index (scg_server_*).

    submit() takes host arrays and returns a ticket; the arrays are kept
    alive here until wait() returns the results."""

    def __init__(self, index, slots=4, max_batch=4096, max_R=100, arena_bytes=1 << 30):
        self.index = index
        self._s = ctypes.c_void_p()
        _check(_lib.scg_server_create(index.handle, slots, max_batch, max_R, ctypes.c_size_t(arena_bytes),
                                      ctypes.byref(self._s)))
        self._live = {}

    def submit(self, mode, Q, R, w, T, precision=FP32_EXACT, rerank=0):
        Q = np.ascontiguousarray(Q, np.float32).reshape(-1, self.index.dim)
        nq = Q.shape[0]
        ids = np.empty((nq, R), np.int32)
        d = np.empty((nq, R), np.float32)
        sums = np.empty(nq, np.int32)
        p = SearchParams(mode, R, w, T, precision, rerank)
        t = ctypes.c_uint64()
        _check(_lib.scg_server_submit(self._s, ctypes.byref(p), _ptr(Q), nq, _ptr(ids), _ptr(d), _ptr(sums),
                                      ctypes.byref(t)))
        self._live[t.value] = (Q, ids, d, sums)
        return t.value

    def wait(self, ticket, timeout=-1.0, times=False):
        """(ids, dists, sums, latency_ms), or None if the timeout expired.
        With times=True the last item is (total, queued, service) in ms."""
        t = np.zeros(3, np.float64)
        rc = _lib.scg_server_wait_times(self._s, ctypes.c_uint64(ticket), ctypes.c_double(timeout), _ptr(t))
        if rc == PENDING:
            return None
        Q, ids, d, sums = self._live.pop(ticket)
        _check(rc)
        return ids, d, sums, (tuple(t.tolist()) if times else float(t[0]))

    def stats(self):
        c = ctypes.c_longlong()
        m = ctypes.c_int()
        q = ctypes.c_int()
        _check(_lib.scg_server_stats(self._s, ctypes.byref(c), ctypes.byref(m), ctypes.byref(q)))
        return {"completed": c.value, "max_inflight": m.value, "queued": q.value}

    def close(self):
        if self._s:
            _lib.scg_server_destroy(self._s)
            self._s = ctypes.c_void_p()
            self._live.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
