"""Benchmark of the batched search on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload C2] [--cache DIR]

A step is one batched search of the workload's whole query set, inputs
already resident on the device.  Default workload: the 10,000,000 x 128
inverted multi-index (2 x 1024 coarse centroids per half, residual PQ 8 x
256), 10,000 queries, T = 30,000 candidates, top-100 -- the configuration the
headline metric is quoted on.  Data is synthetic and seeded (see
second-candidate_b200/workloads.py); the workload is built with torch alone
and cached, so both arms search the same index.

Prints one JSON line (rank 0).  `value` is the whole-job QPS (all replicas)
of the BF16 batched form; `e2e` is the same metric through the public
host-buffer entry point with the host<->device copies inside the timed
region; `roofline` is for the ADC scan kernel.  After the detailed legs the
line ends with the compact comparison: `cpu_baseline` (the reference's own
search, compiled from its sources into oracle/_ref, on the host cores with all
threads on a bounded query sample, plus a 1-thread figure), `parity` (a
500-query sample: the FP32-exact form against the compiled reference, and
the distance error of every arithmetic form against float64) and `forms`
(QPS and recall@100 of every form beside the CPU figures).  The default run
also measures the plain-PQ 100k workload as `c1`.

`--impl reference` times only the reference's CPU search (rank 0; other
ranks exit at once) on the same workload and prints the same line with
"impl": "reference"; it loads none of this project's CUDA code.
"""
import argparse
import gc
import json
import os
import statistics
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "second-candidate_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "QPS at recall@100 (BF16 batched vs FP32 plain vs CPU); p50/p99 latency"
MODE_IDS = {"ivfadc": 0, "imi": 1, "sc": 2}
# name -> (C ABI precision, description)
PRECISIONS = {
    "fp32": (0, "fp32-exact: CUDA-core tables in the reference's float order, the reference's ADC adds"),
    "fast": (1, "bf16x3: tcgen05 BF16 hi/lo split tables (FP32 accumulation), fused per-vector term"),
    "bf16": (2, "bf16: tcgen05 one-product BF16 tables (FP32 accumulation), fused per-vector term"),
    "fp16": (3, "fp16: tcgen05 one-product FP16 tables (FP32 accumulation), fused per-vector term"),
}
FORM_NAMES = {"fast": "bf16x3", "fp32": "fp32_plain", "bf16": "bf16", "fp16": "fp16"}
L2_NOTE = ("GPU arm: L2 flushed before every timed step (256 MB device write); "
           "CPU reference arm: host caches left as they are")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


def per_query_targets(cfg, nq):
    """Per-query candidate targets of a config with a T range (log-uniform,
    seeded), else None."""
    if isinstance(cfg["T"], int):
        return None
    lo, hi = cfg["T"]
    return np.exp(np.random.default_rng(17).uniform(np.log(lo), np.log(hi), nq)).astype(np.int32)


def workload_desc(cfg):
    if cfg["mode"] == "imi":
        idx = "IMI 2x%d, residual PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    elif cfg["mode"] == "sc":
        idx = "second-candidate kc=%d, residual PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    elif cfg["kc"] == 1:
        idx = "plain PQ %dx%d (IVFADC, one zero coarse centroid)" % (cfg["mp"], cfg["kp"])
    else:
        idx = "IVFADC kc=%d, PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    return "%s: N=%d D=%d %s, Q=%d, T=%s, R=%d" % (cfg["name"], cfg["N"], cfg["D"], idx, cfg["nq"],
                                                    cfg["T"], cfg["R"])


def config_of(cfg):
    """The `config` object of both arms' lines (identical by construction)."""
    return {"workload": workload_desc(cfg), "queries_per_step": cfg["nq"], "l2": L2_NOTE}


class Clocks:
    """SM clock and clock-event (throttle) reasons sampled through NVML every
    few milliseconds by a thread, so that even a timed region of tens of
    milliseconds holds samples.  mark() brackets the timed region; stop()
    summarises the samples inside it (read-only NVML queries)."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, gpu, period=0.004):
        self.gpu, self.period = gpu, period
        self.samples, self.t0, self.t1 = [], None, None
        self.th, self.run, self.nv, self.err = None, False, None, None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception as ex:
            self.err = repr(ex)
            return
        self.run = True
        self.th = threading.Thread(target=self._loop, daemon=True)
        self.th.start()

    def _loop(self):
        nv = self.nv
        while self.run:
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception as ex:
                self.err = repr(ex)
            time.sleep(self.period)

    def mark(self, begin):
        if begin:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def stop(self):
        self.run = False
        if self.th:
            self.th.join(timeout=2)
        if not self.samples:
            return {"unavailable": self.err or "no samples"} if self.err else None
        t0 = self.t0 if self.t0 is not None else self.samples[0][0]
        t1 = self.t1 if self.t1 is not None else self.samples[-1][0]
        inside = [x for x in self.samples if t0 <= x[0] <= t1] or self.samples
        reasons = set()
        for _, _, rs in inside:
            for name, attr in self.REASONS:
                if rs & getattr(self.nv, attr, 0):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": self.max_mhz,
                "samples": len(inside), "reasons": sorted(reasons), "source": "NVML, %g ms period" % (1e3 * self.period)}


def cpu_reference(w, seconds_target=12.0, threads=None, nq_max=None):
    """Times the reference's own search (oracle/_ref/libscref.so: the
    unmodified search_ivfadc / search_multi2 / search_mr_ivf with OpenMP over
    queries, per-thread query objects sharing the index) on a bounded sample
    of the workload's queries: a probe sizes the sample to about
    `seconds_target` of work.  Falls back to the C restatement (one thread)
    when the reference build is not present."""
    import oracle as O
    from workloads import recall_at
    cfg = w["cfg"]
    threads = threads or os.cpu_count()
    mode = MODE_IDS[cfg["mode"]]
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    ix = O.Index(cfg["D"], mcp, cfg["kc"], cfg["mp"], cfg["kp"], w["cq"], w["pq"], w["L"], w["pid"],
                 w["codes"])
    Q = w["Q"]
    Ts = per_query_targets(cfg, Q.shape[0])
    T = cfg["T"] if Ts is None else int(Ts.max())
    R, wcap = cfg["R"], cfg["w"]
    if O.ref_available():
        kind = "reference"

        def run(a, b):
            ids, d, sums, sec = O.ref_search_batch(ix, mode, Q[a:b], R, wcap, T, nthreads=threads,
                                                   Tq=None if Ts is None else Ts[a:b])
            return ids, sec
    else:
        kind = "port"
        threads = 1

        def run(a, b):
            if Ts is not None:
                raise RuntimeError("per-query targets need the compiled reference")
            t0 = time.perf_counter()
            ids, d, sums = ix.search(mode, Q[a:b], R, wcap, T, order=O.ORDER_HEAP)
            return ids, time.perf_counter() - t0
    nmax = min(Q.shape[0], nq_max or Q.shape[0])
    probe = min(nmax, max(2 * threads, 16))
    _, sec = run(0, probe)
    per_q = sec / probe
    n = int(min(nmax, max(probe, seconds_target / max(per_q, 1e-9))))
    ids, sec = run(0, n)
    return {"value": n / sec, "unit": "queries/s", "cores": threads, "kind": kind,
            "sample": "first %d of %d queries, one batch, %s%s" % (
                n, Q.shape[0], "OpenMP over queries" if threads > 1 else "one thread",
                ", per-query T" if Ts is not None else ""),
            "seconds": sec, "recall@100": recall_at(ids, w["gt"][:n], min(100, R))}


def same_topk(ids_a, d_a, ids_b, d_b, n):
    """Two top-n lists agree: identical distances position by position and
    identical ids except inside runs of equal distance (compared as sets; a
    run cut by the n-th position may differ)."""
    ids_a, ids_b, d_a, d_b = ids_a[:n], ids_b[:n], d_a[:n], d_b[:n]
    if not np.array_equal(d_a, d_b):
        return False
    if n == 0:
        return True
    for v in np.unique(d_a):
        if v != d_a[n - 1] and set(ids_a[d_a == v].tolist()) != set(ids_b[d_a == v].tolist()):
            return False
    return True


def fp64_adc_dist(w, q, ids, pos_of_id, cell_of_pos):
    """Float64 ||q - c - r||^2 of database ids (the exact value of the ADC
    distance the reference sums from its tables): c = the coarse centroid(s)
    of the id's cell, r = the PQ centroids of its code."""
    cfg = w["cfg"]
    D, kc, mp, kp = cfg["D"], cfg["kc"], cfg["mp"], cfg["kp"]
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    cq = w["cq"].reshape(mcp, kc, D // mcp).astype(np.float64)
    pq = w["pq"].reshape(mp, kp, D // mp).astype(np.float64)
    pos = pos_of_id[ids]
    cell = cell_of_pos[pos]
    codes = w["codes"][pos]                                  # [n, mp]
    if cfg["mode"] == "imi":
        c = np.concatenate([cq[0][cell // kc], cq[1][cell % kc]], axis=1)
    elif cfg["mode"] == "sc":
        c = cq[0][cell // kc]                               # residual of the 1st nearest
    else:
        c = cq[0][cell]
    r = np.concatenate([pq[k][codes[:, k]] for k in range(mp)], axis=1)
    diff = q.astype(np.float64)[None, :] - c - r
    return (diff * diff).sum(1)


def parity_leg(ix, w, mode, nsample=500, threads=None):
    """On the first `nsample` queries: (1) the FP32-exact GPU form against the
    compiled reference's own search (oracle/_ref) -- the share of queries with
    the same candidate count, and with the same top-R ids and bit-identical
    distances (equal distances compared as sets of ids); (2) for every
    arithmetic form, the relative error of the returned top-R ADC distances
    against a float64 evaluation of ||q - c - r||^2 for the same codes."""
    import torch

    import oracle as O
    import scgpu
    cfg = w["cfg"]
    R, wcap = cfg["R"], cfg["w"]
    Q = w["Q"][:nsample]
    n = Q.shape[0]
    Ts = per_query_targets(cfg, w["Q"].shape[0])
    Ts = None if Ts is None else Ts[:n]
    T = cfg["T"] if Ts is None else int(Ts.max())
    dev = torch.device("cuda", torch.cuda.current_device())
    dQ = torch.from_numpy(np.ascontiguousarray(Q)).to(dev)
    d_ids = torch.empty(n * R, dtype=torch.int32, device=dev)
    d_d = torch.empty(n * R, dtype=torch.float32, device=dev)
    d_s = torch.empty(n, dtype=torch.int32, device=dev)
    d_T = None
    if Ts is not None:
        d_T = torch.from_numpy(Ts).to(dev)
        ix.set_query_targets(d_T.data_ptr())
    res = {}
    for name, (pv, _) in PRECISIONS.items():
        ix.search_device(mode, dQ.data_ptr(), n, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(), d_s.data_ptr(),
                         precision=pv, rerank=0)
        torch.cuda.synchronize()
        res[name] = (d_ids.view(n, R).cpu().numpy(), d_d.view(n, R).cpu().numpy(), d_s.cpu().numpy())
    if d_T is not None:
        ix.set_query_targets(None)
    out = {"queries": n, "what": "first %d queries of the workload, top-%d ADC results (no re-rank)" % (n, R)}
    # (1) against the compiled reference
    if O.ref_available():
        mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
        oix = O.Index(cfg["D"], mcp, cfg["kc"], cfg["mp"], cfg["kp"], w["cq"], w["pq"], w["L"], w["pid"],
                      w["codes"])
        rids, rd, rsums, _ = O.ref_search_batch(oix, mode, Q, R, wcap, T, nthreads=threads or os.cpu_count(),
                                                Tq=Ts)
        ids, d, sums = res["fp32"]
        same_sum = same_top = 0
        for i in range(n):
            if sums[i] != rsums[i]:
                continue
            same_sum += 1
            m = min(R, int(sums[i]))
            rid, rdi = rids[i][:m], rd[i][:m]
            o = np.lexsort((rid, rdi))
            if same_topk(ids[i], d[i], rid[o], rdi[o], m):
                same_top += 1
        out["vs_reference"] = {"form": "fp32_plain (SCG_FP32_EXACT)", "same_sum": same_sum / n,
                               "same_top": same_top / n,
                               "what": "share of queries whose candidate count / top-R ids and distances equal "
                                       "the reference's own search (oracle/_ref)"}
    else:
        out["vs_reference"] = {"unavailable": "oracle/_ref/libscref.so not built"}
    # (2) distance error against float64
    N = w["pid"].shape[0]
    pos_of_id = np.empty(N, np.int64)
    pos_of_id[w["pid"]] = np.arange(N)
    L = w["L"].astype(np.int64)
    cell_of_pos = np.repeat(np.arange(L.shape[0]), np.diff(np.concatenate([[0], L])))
    err = {}
    for name, (ids, d, sums) in res.items():
        rel = []
        for i in range(n):
            m = ids[i] >= 0
            if not m.any():
                continue
            d64 = fp64_adc_dist(w, Q[i], ids[i][m], pos_of_id, cell_of_pos)
            rel.append(np.abs(d[i][m].astype(np.float64) - d64) / np.maximum(np.abs(d64), 1e-30))
        rel = np.concatenate(rel) if rel else np.zeros(1)
        err[FORM_NAMES[name]] = {"max": float(rel.max()), "median": float(np.median(rel))}
    out["dist_err_fp64"] = err
    out["dist_err_what"] = ("relative error |d - d64| / d64 of the returned top-%d ADC distances, d64 = float64 "
                            "||q - c - r||^2 of the same codes" % R)
    return out


def serve_leg(scgpu, ix, w, mode, wcap, T, prec, seconds, load, seed=7, rerank=0):
    """A request stream through the server (scg_server_*): each request a
    batch of 1..4096 queries (log-uniform) drawn from the workload's queries,
    k in {1, 10, 100}.  First the server's capacity for this mix (requests
    kept 16 deep, as fast as it completes them), then Poisson arrivals at
    `load` x that capacity for `seconds`.  Latency = submit to results in
    host memory, per request."""
    import threading
    rng = np.random.default_rng(seed)
    Q = w["Q"]

    def mix(n):
        sizes = np.minimum(4096, np.exp(rng.uniform(0, np.log(4097), n)).astype(int))
        ks = rng.choice([1, 10, 100], n)
        starts = rng.integers(0, max(1, Q.shape[0] - 4096), n)
        return sizes, ks, starts

    srv = scgpu.Server(ix, slots=4, max_batch=4096, max_R=100, arena_bytes=8 << 30)

    def submit(q, k):
        return srv.submit(mode, q, k, wcap, T, precision=prec, rerank=max(rerank, k) if rerank else 0)

    for t in [submit(Q[:64], 10) for _ in range(8)]:
        srv.wait(t)
    # capacity (closed loop, 16 outstanding)
    n_cap = 600
    sizes, ks, starts = mix(n_cap)
    pending = []
    t0 = time.perf_counter()
    for i in range(n_cap):
        if len(pending) >= 16:
            srv.wait(pending.pop(0))
        pending.append(submit(Q[starts[i]:starts[i] + sizes[i]], int(ks[i])))
    for t in pending:
        srv.wait(t)
    capacity = float(sizes.sum() / (time.perf_counter() - t0))
    # open loop at `load` x capacity
    mean_batch = (4096 - 1) / np.log(4096)
    rate = load * capacity / mean_batch
    n = max(8, int(rate * seconds))
    gaps = rng.exponential(1.0 / rate, n)
    sizes, ks, starts = mix(n)
    tickets, done = [], []

    def waiter():
        i = 0
        while i < n:
            if i >= len(tickets):
                time.sleep(0.0002)
                continue
            done.append(srv.wait(tickets[i], times=True)[3])
            i += 1

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    nxt = t0
    for i in range(n):
        nxt += gaps[i]
        d = nxt - time.perf_counter()
        if d > 0:
            time.sleep(d)
        s0 = int(starts[i])
        tickets.append(submit(Q[s0:s0 + int(sizes[i])], int(ks[i])))
    th.join()
    span = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = np.array([x[0] for x in done])
    qd = np.array([x[1] for x in done])
    svc = np.array([x[2] for x in done])
    worst = np.argsort(lat)[-5:][::-1]
    return {"capacity_qps": capacity,
            "queued_ms": {"p50": float(np.percentile(qd, 50)), "p99": float(np.percentile(qd, 99))},
            "service_ms": {"p50": float(np.percentile(svc, 50)), "p99": float(np.percentile(svc, 99))},
            "slowest": [{"nq": int(sizes[i]), "k": int(ks[i]), "total_ms": float(lat[i]), "queued_ms": float(qd[i]),
                         "service_ms": float(svc[i])} for i in worst], "load": load, "qps": float(sizes.sum() / span), "requests": int(n),
            "queries": int(sizes.sum()), "offered_requests_per_s": float(rate),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "max_inflight": st["max_inflight"], "slots": 4,
            "what": "batches 1..4096 log-uniform, k in {1,10,100}; capacity = closed loop 16 deep; then Poisson "
                    "arrivals at load x capacity; continuous batching over 4 streams; latency = submit to "
                    "results in host memory"}


def encode_leg(scgpu, ix, cfg, rows, dev):
    """Encoder throughput on rows drawn like the workload's base (device
    buffers): the tensor-core encoder (tcgen05 distance tables + exact
    re-check) against the all-double kernel; both must give the same codes."""
    import torch
    import workloads as W
    X = W.mixture_sampler(cfg, 99, dev)(rows)
    nc = 2 if cfg["mode"] == "sc" else 0  # the second-candidate index: SCEncoder::encode<T>, two centroids
    mcp = nc if nc else cfg["mc"]
    out = {}
    codes = {}
    for name, method in (("tensor", scgpu.ENC_TENSOR), ("exact", scgpu.ENC_EXACT)):
        ix.set_encoder(method)
        cid = torch.empty(rows, mcp, dtype=torch.int16, device=dev)
        cod = torch.empty(rows, cfg["mp"], dtype=torch.uint8, device=dev)
        ix.encode_device(X[:65536].data_ptr(), 65536, nc, cid.data_ptr(), cod.data_ptr())  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ix.encode_device(X.data_ptr(), rows, nc, cid.data_ptr(), cod.data_ptr())
        e1.record()
        e1.synchronize()
        out[name + "_rows_per_s"] = rows / (e0.elapsed_time(e1) / 1e3)
        codes[name] = (cid.cpu().numpy(), cod.cpu().numpy())
    ix.set_encoder(scgpu.ENC_TENSOR)
    out["same_codes"] = bool(np.array_equal(codes["tensor"][0], codes["exact"][0]) and
                             np.array_equal(codes["tensor"][1], codes["exact"][1]))
    out["rows"] = rows
    out["what"] = ("%s codes of rows drawn from the workload's mixture: tcgen05 split-BF16 distance tables + "
                   "exact double re-check vs the all-double kernel"
                   % ("SCEncoder::encode<T> (two nearest coarse centroids)" if nc else "Encoder::encode<T> (IVF/IMI)"))
    return out


def time_steps(step, flush, stream, n):
    """Device time (ms, CUDA events on the launching stream) of n steps, the
    L2 flushed before each."""
    import torch
    out = []
    for _ in range(n):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        out.append(e0.elapsed_time(e1))
    return out


def run_workload(args, name, scgpu, dev, world, full=True):
    """Our arm on one workload: every arithmetic form (the chosen one timed
    over args.steps steps), roofline of the scan, and -- with `full` -- the
    CUDA-graph replay, the end-to-end host-buffer leg, the encoder and
    serving legs.  Returns the fields of the JSON line and the index."""
    import torch
    import replicas
    import workloads as W

    w = W.build_gpu_workload(name, cache_dir=args.cache, log=log)
    cfg = w["cfg"]
    mode = MODE_IDS[cfg["mode"]]
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    R, wcap = cfg["R"], cfg["w"]
    if args.queries and full:
        w["Q"] = w["Q"][: args.queries]
        w["gt"] = w["gt"][: args.queries]
    nq = w["Q"].shape[0]
    pname = args.precision if (full and args.precision) else cfg.get("precision", "fast")
    prec = PRECISIONS[pname][0]
    rerank = int(cfg.get("shortlist", 0))
    Ts = per_query_targets(cfg, nq)
    T = cfg["T"] if Ts is None else int(Ts.max())

    ix = scgpu.Index(dev.index)
    ix.load_codebooks(w["cq"], cfg["kc"], mcp, w["pq"], cfg["kp"], cfg["mp"], cfg["D"])
    ix.load_csr(w["L"], w["pid"], w["codes"])
    ix.precompute()
    if rerank:
        ix.load_raw(w["raw"])
        ix.set_cell_budget(1 << 19)  # long per-query lists of the large targets

    dQ = torch.from_numpy(w["Q"]).to(dev)
    d_ids = torch.empty(nq * R, dtype=torch.int32, device=dev)
    d_d = torch.empty(nq * R, dtype=torch.float32, device=dev)
    d_s = torch.empty(nq, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # per-query candidate targets first: the autotuner must time the batch
    # the steps search
    d_T = None
    if Ts is not None:
        d_T = torch.from_numpy(Ts).to(dev)
        ix.set_query_targets(d_T.data_ptr())

    # the scan's chunking picked by the library's autotuner on this batch, for
    # both scan forms (exact and fast)
    tuning = {}
    if args.upl:
        for pv in (prec, 0):
            ix.set_scan_tuning(pv, args.upl)
        tuning = {"fixed_candidates_per_lane": args.upl}
    if not (args.no_autotune or args.upl):
        # the main form: candidates per lane, coarse-prefix length, kernel
        # organisation (and the shortlist length with a re-rank); then the
        # exact form's candidates per lane
        tuning["main"] = ix.autotune_ex(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(),
                                        d_s.data_ptr(), precision=prec, rerank=rerank)
        choice, ms = ix.autotune(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(),
                                 d_s.data_ptr(), precision=0, rerank=rerank)
        tuning["fp32"] = {"candidates_per_lane": choice, "ms_by_choice": dict(zip((2, 4, 8), ms))}

    def step(p=None):
        ix.search_device(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(),
                         d_s.data_ptr(), stream=stream.cuda_stream, precision=prec if p is None else p,
                         rerank=rerank)

    # every other arithmetic form on the same queries (QPS at recall@100)
    forms = {}
    if not args.no_plain:
        for fname, (pv, desc) in PRECISIONS.items():
            if fname == pname:
                continue
            for _ in range(3):
                step(pv)
            torch.cuda.synchronize()
            pt = time_steps(lambda: step(pv), flush, stream, 3)
            pids = d_ids.view(nq, R).cpu().numpy()
            forms[fname] = {"value": nq / (statistics.mean(pt) / 1e3) * world, "unit": "queries/s",
                            "recall@100": W.recall_at(pids, w["gt"], min(100, R)),
                            "ms_per_step": statistics.mean(pt), "what": desc,
                            "kernels_ms": dict(zip(("tables_and_prefix", "select_scan", "rerank", "select", "scan"),
                                                   ix.last_timings()))}

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = Clocks(dev.index)
    clocks.start()
    replicas.barrier()
    torch.cuda.synchronize()
    clocks.mark(True)
    gc.collect()
    gc.disable()
    times, kern, launches = [], [], 0
    for _ in range(args.steps):
        times += time_steps(step, flush, stream, 1)
        kern.append(ix.last_timings())
        launches += ix.last_launches()  # this step's kernels, counted by the library
    torch.cuda.synchronize()
    gc.enable()
    clocks.mark(False)
    replicas.barrier()
    job_qps, total_ms = replicas.job_throughput(sum(times), nq * args.steps, device=dev)
    ck = clocks.stop()

    ids = d_ids.view(nq, R).cpu().numpy()
    sums = d_s.cpu().numpy()
    nvis, empty = ix.last_query_stats(nq)
    recall = W.recall_at(ids, w["gt"], min(100, R))

    # roofline of the dominant kernel, the ADC scan (the scan-only kernel when
    # selection and scan run as two kernels): algorithmic bytes = the codes of
    # every scanned candidate + 8 bytes of CSR offsets per visited cell + 4
    # bytes per returned id
    search_ms = statistics.mean(k[1] for k in kern)
    tables_ms = statistics.mean(k[0] for k in kern)
    select_ms = statistics.mean(k[3] for k in kern)
    scan_ms = statistics.mean(k[4] for k in kern)
    rerank_ms = statistics.mean(k[2] for k in kern)
    split = scan_ms > 0
    alg_bytes = float(sums.astype(np.int64).sum() * cfg["mp"] + 8 * nvis.astype(np.int64).sum() + 4 * nq * R)
    hbm, _, peak_kind = peaks()
    achieved = alg_bytes / ((scan_ms if split else search_ms) / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(("k_search_scan:" if split else "k_search:") + name)
        except Exception:
            traffic = None
    out = {
        "w": w, "cfg": cfg, "ix": ix, "mode": mode, "pname": pname, "job_qps": job_qps,
        "ms_per_step": total_ms / args.steps, "recall": recall, "rerank": rerank, "Ts": Ts,
        "forms": forms, "tuning": tuning, "clocks": ck, "times": times, "split": split,
        "kernels_ms": {"tables_and_prefix": tables_ms, "select_scan": search_ms, "select": select_ms,
                       "scan": scan_ms, "rerank": rerank_ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": ("k_search<.., 2> (ADC scan + top-R; selection runs as its own kernel)" if split
                                else "k_search (fused selection + ADC scan + top-R)"),
                     "alg_bytes_per_launch": alg_bytes, "scan_ms": scan_ms if split else search_ms},
        "candidates_per_query": float(sums.mean()), "cells_per_query": float(nvis.mean() + empty.mean()),
        "gpu_launches": launches,
    }
    if not full:
        if d_T is not None:
            ix.set_query_targets(None)
        return out

    # the same step replayed from a CUDA graph (captured once by the library)
    if Ts is None:
        gstream = torch.cuda.Stream(dev)
        gt_ = []
        for i in range(args.warmup + args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            g0 = torch.cuda.Event(enable_timing=True)
            g1 = torch.cuda.Event(enable_timing=True)
            g0.record(gstream)
            ix.search_graph(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(), d_s.data_ptr(),
                            gstream.cuda_stream, precision=prec, rerank=rerank)
            g1.record(gstream)
            g1.synchronize()
            if i >= args.warmup:
                gt_.append(g0.elapsed_time(g1))
        out["graph"] = {"value": nq / (statistics.mean(gt_) / 1e3) * world, "unit": "queries/s",
                        "ms_per_step": statistics.mean(gt_),
                        "what": "scg_search_graph: the step's launch sequence captured once, replayed as one "
                                "graph launch"}

    if args.phases:
        ix.set_phase_counters(True)
        step()
        ph = ix.last_phase_counters()
        ph["per_query_cycles"] = {k: ph[k] / nq for k in ("select_warp", "sort", "bisection", "rounds", "cut", "compact",
                                                          "lut_fill", "warm_threshold", "scan", "final_merge")}
        ph["per_query"] = {k: ph[k] / nq for k in ("pending", "deferred", "round_count", "bisection_steps",
                                                   "enumerated_cells", "full_sorts")}
        ix.set_phase_counters(False)
        out["phases"] = ph

    # end to end through the public host-buffer entry point
    if not args.no_e2e:
        # queries in and results out through pinned host buffers (the
        # caller's), reused every step
        Qh = torch.from_numpy(w["Q"]).pin_memory().numpy()
        outs = (torch.empty((nq, R), dtype=torch.int32).pin_memory().numpy(),
                torch.empty((nq, R), dtype=torch.float32).pin_memory().numpy(),
                torch.empty(nq, dtype=torch.int32).pin_memory().numpy())
        e2e_times = []
        if Ts is not None:
            # per-query targets ride on the device entry point: pinned
            # queries in, search, pinned results out, on one stream
            hq = torch.from_numpy(w["Q"]).pin_memory()
            hi = torch.empty(nq * R, dtype=torch.int32).pin_memory()
            hdd = torch.empty(nq * R, dtype=torch.float32).pin_memory()
            hs = torch.empty(nq, dtype=torch.int32).pin_memory()
        gc.collect()
        gc.disable()  # no collector pauses inside the timed calls
        for i in range(args.warmup + args.steps):
            flush.zero_()  # same cold-L2 start as the device-timed steps
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if Ts is None:
                hid, hd, hs_ = ix.search(mode, Qh, R, wcap, T, precision=prec, out=outs, rerank=rerank)
            else:
                dQ.copy_(hq, non_blocking=True)
                step()
                hi.copy_(d_ids, non_blocking=True)
                hdd.copy_(d_d, non_blocking=True)
                hs.copy_(d_s, non_blocking=True)
                torch.cuda.current_stream().synchronize()
                hid = hi.numpy().reshape(nq, R)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                e2e_times.append(dt)
        gc.enable()
        out["e2e"] = {"value": nq * len(e2e_times) / sum(e2e_times) * world, "unit": "queries/s",
                      "h2d_bytes_per_step": int(nq * cfg["D"] * 4), "d2h_bytes_per_step": int(nq * R * 8 + nq * 4),
                      "same_ids_as_device_path": bool(np.array_equal(hid, ids)),
                      "step_ms": {"mean": 1e3 * statistics.mean(e2e_times), "p50": 1e3 * statistics.median(e2e_times),
                                  "max": 1e3 * max(e2e_times)}}
    if d_T is not None:
        ix.set_query_targets(None)
    return out


def summary_forms(res, cpu=None, cpu1=None):
    """Compact QPS / recall@100 of every form (and the CPU reference)."""
    f = {FORM_NAMES[res["pname"]]: {"qps": res["job_qps"], "recall@100": res["recall"]}}
    for k, v in res["forms"].items():
        f[FORM_NAMES[k]] = {"qps": v["value"], "recall@100": v["recall@100"]}
    if cpu and "value" in cpu:
        f["cpu_reference_%dt" % cpu["cores"]] = {"qps": cpu["value"], "recall@100": cpu["recall@100"]}
    if cpu1 and "value" in cpu1:
        f["cpu_reference_1t"] = {"qps": cpu1["value"], "recall@100": cpu1["recall@100"]}
    return f


def cpu_legs(w, rank, world, args, one_thread_s=6.0):
    """The reference CPU figures (all threads and one thread), rank 0 at N=1."""
    if not (rank == 0 and world == 1 and not args.no_cpu_baseline):
        return None, None
    try:
        cpu = cpu_reference(w)
    except Exception as ex:  # reported, never silently dropped
        cpu = {"unavailable": repr(ex)}
    try:
        cpu1 = cpu_reference(w, seconds_target=one_thread_s, threads=1)
    except Exception as ex:
        cpu1 = {"unavailable": repr(ex)}
    return cpu, cpu1


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="C2")
    ap.add_argument("--extra", default="C1", help="comma-separated extra workloads measured after the main one "
                                                    "('' for none)")
    ap.add_argument("--cache", default="/tmp/scg_bench_cache")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the 500-query parity / FP64-error leg")
    ap.add_argument("--precision", default=None, choices=list(PRECISIONS),
                    help="arithmetic of the tables (default: the workload's; fast for the IMI 10M one)")
    ap.add_argument("--queries", type=int, default=0, help="use only the first N queries")
    ap.add_argument("--no-plain", action="store_true", help="skip the other arithmetic forms")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg")
    ap.add_argument("--phases", action="store_true", help="report per-phase cycle counters")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default scan chunking")
    ap.add_argument("--upl", type=int, default=0, choices=[0, 2, 4, 8],
                    help="fix the scan's candidates per lane for every form (skips the autotuner)")
    ap.add_argument("--encode-rows", type=int, default=2_000_000,
                    help="rows of the encoder leg (tensor-core vs exact encoder); 0 skips it")
    ap.add_argument("--serve-seconds", type=float, default=3.0,
                    help="length of the serving leg (Poisson request stream); 0 skips it")
    ap.add_argument("--serve-load", type=float, default=0.5,
                    help="offered load of the serving leg as a fraction of the server's measured capacity")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    import torch
    import workloads as W

    if args.impl == "reference":
        # the reference's CPU search alone: no module of this project's CUDA
        # library is imported on this path (the workload is built by torch)
        if rank != 0:
            return
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        w = W.build_gpu_workload(args.workload, cache_dir=args.cache, log=log)
        cfg = w["cfg"]
        vals = []
        for i in range(args.warmup + args.steps):
            r = cpu_reference(w, seconds_target=2.0)
            if i >= args.warmup:
                vals.append(r)
        qps = sum(v["value"] for v in vals) / len(vals)
        line = {"impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * statistics.mean(v["seconds"] for v in vals),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": config_of(cfg), "recall@100": vals[-1]["recall@100"],
                "parallelism": "host threads (OpenMP over queries)",
                "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": vals[-1]["cores"],
                                 "kind": vals[-1]["kind"], "sample": vals[-1]["sample"]},
                "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import scgpu
    import replicas
    torch.cuda.set_device(local)
    if world > 1:
        # replicas: every rank searches its own copy; only the timing is reduced
        replicas.init("nccl")
    dev = torch.device("cuda", local)

    res = run_workload(args, args.workload, scgpu, dev, world, full=True)
    w, cfg, ix, mode = res["w"], res["cfg"], res["ix"], res["mode"]
    Ts = res["Ts"]
    line = {
        "metric": METRIC, "value": res["job_qps"], "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp32": "f32", "fast": "bf16", "bf16": "bf16", "fp16": "f16"}[res["pname"]],
        "data": "synthetic", "config": config_of(cfg),
        "precision_form": PRECISIONS[res["pname"]][1],
        "parallelism": "replicas" if world > 1 else "1 GPU",
        "timing": "CUDA events per step on the launching stream",
        "recall@100": res["recall"],
        "rerank_shortlist": res["rerank"] or None,
        "per_query_T": None if Ts is None else {"min": int(Ts.min()), "median": int(np.median(Ts)),
                                                "max": int(Ts.max())},
        "phases": res.get("phases"),
        "latency_ms": {"p50": float(np.percentile(res["times"], 50)), "p99": float(np.percentile(res["times"], 99)),
                       "what": "whole batch of %d queries" % w["Q"].shape[0]},
        "batch_ms": {"p50": float(np.percentile(res["times"], 50)), "p99": float(np.percentile(res["times"], 99))},
        "kernels_ms": res["kernels_ms"],
        "roofline": res["roofline"],
        "e2e": res.get("e2e"),
        # per step: tensor-core tables, query norms, coarse prefixes,
        # selection, scan (the fused kernel replaces the last two), re-rank
        "gpu_launches": res["gpu_launches"],
        "autotune": res["tuning"],
        "graph": res.get("graph"),
        "clocks": res["clocks"],
        "candidates_per_query": res["candidates_per_query"], "cells_per_query": res["cells_per_query"],
        "other_forms": res["forms"],
    }
    if args.encode_rows > 0:
        line["encode"] = encode_leg(scgpu, ix, cfg, args.encode_rows, dev)
    if args.serve_seconds > 0:
        T = cfg["T"] if Ts is None else int(np.median(Ts))
        line["serving"] = serve_leg(scgpu, ix, w, mode, cfg["w"], T, PRECISIONS[res["pname"]][0],
                                    args.serve_seconds, args.serve_load, rerank=res["rerank"])
        line["latency_ms"] = {"p50": line["serving"]["p50_ms"], "p99": line["serving"]["p99_ms"],
                              "what": "per request of the serving leg"}
    parity = None
    if not args.no_parity and rank == 0:
        try:
            parity = parity_leg(ix, w, mode)
        except Exception as ex:
            parity = {"unavailable": repr(ex)}
    cpu, cpu1 = cpu_legs(w, rank, world, args)
    ix.close()
    # extra workloads (small): QPS / recall / roofline / CPU figures
    extras = {}
    for xname in [x for x in args.extra.split(",") if x and x != args.workload]:
        try:
            xr = run_workload(args, xname, scgpu, dev, world, full=False)
            xcpu, xcpu1 = cpu_legs(xr["w"], rank, world, args, one_thread_s=4.0)
            extras[xname.lower()] = {"config": config_of(xr["cfg"]), "value": xr["job_qps"], "unit": "queries/s",
                                     "ms_per_step": xr["ms_per_step"], "recall@100": xr["recall"],
                                     "precision_form": FORM_NAMES[xr["pname"]],
                                     "roofline": {k: xr["roofline"][k] for k in ("achieved", "peak", "frac", "unit",
                                                                                "scan_ms", "alg_bytes_per_launch")},
                                     "forms": summary_forms(xr, xcpu, xcpu1), "cpu_baseline": xcpu,
                                     "cpu_baseline_1t": xcpu1}
            xr["ix"].close()
        except Exception as ex:
            extras[xname.lower()] = {"unavailable": repr(ex)}
    line.update(extras)
    # the compact comparison last (the end of the line is what a tail shows)
    line["fp32_plain"] = res["forms"].get("fp32") and {k: res["forms"]["fp32"][k] for k in
                                                      ("value", "recall@100", "ms_per_step")}
    line["cpu_baseline"] = cpu
    line["cpu_baseline_1t"] = cpu1
    line["parity"] = parity
    line["forms"] = summary_forms(res, cpu, cpu1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.finish()


if __name__ == "__main__":
    main()
