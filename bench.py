"""Benchmark of the batched search on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload C2] [--cache DIR]

A step is one batched search of the workload's whole query set, inputs
already resident on the device.  Default workload: the 10,000,000 x 128
inverted multi-index (2 x 1024 coarse centroids per half, residual PQ 8 x
256), 10,000 queries, T = 30,000 candidates, top-100 -- the configuration the
headline metric is quoted on.  Data is synthetic and seeded (see
second-candidate_b200/workloads.py).

Prints one JSON line (rank 0).  `value` is the whole-job QPS (all replicas);
`e2e` is the same metric through the public host-buffer entry point with the
host<->device copies inside the timed region; `cpu_baseline` is the
reference's own search (compiled from its sources, oracle/_ref) on the host
cores with all threads on a bounded query sample; `roofline` is for the
fused selection + scan kernel.

`--impl reference` times only the reference's CPU search (rank 0; other
ranks exit at once) on the same workload and prints the same line with
"impl": "reference".
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


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], p["bf16_tflops"], "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


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


def cpu_reference(w, seconds_target=12.0, threads=None, mode=None):
    """Times the reference's own search (oracle/_ref/libscref.so, all host
    threads) on a bounded sample of the workload's queries.  Falls back to
    the C restatement when the reference build is not present."""
    import oracle as O
    cfg = w["cfg"]
    threads = threads or os.cpu_count()
    mode = MODE_IDS[cfg["mode"]] if mode is None else mode
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    ix = O.Index(cfg["D"], mcp, cfg["kc"], cfg["mp"], cfg["kp"], w["cq"], w["pq"], w["L"], w["pid"],
                 w["codes"])
    Q = w["Q"]
    T = cfg["T"] if isinstance(cfg["T"], int) else cfg["T"][0]
    R, wcap = cfg["R"], cfg["w"]
    if O.ref_available():
        kind = "reference"

        def run(qs):
            ids, d, sums, sec = O.ref_search_batch(ix, mode, qs, R, wcap, T, nthreads=threads)
            return ids, sec
    else:
        kind = "port"
        threads = 1

        def run(qs):
            t0 = time.perf_counter()
            ids, d, sums = ix.search(mode, qs, R, wcap, T, order=O.ORDER_HEAP)
            return ids, time.perf_counter() - t0
    probe = min(Q.shape[0], max(4 * threads, 32))
    _, sec = run(Q[:probe])
    per_q = sec / probe
    n = int(min(Q.shape[0], max(probe, seconds_target / max(per_q, 1e-9))))
    ids, sec = run(Q[:n])
    from workloads import recall_at
    return {"value": n / sec, "unit": "queries/s", "cores": threads, "kind": kind,
            "sample": "first %d of %d queries, one batch, %s" % (n, Q.shape[0], "OpenMP over queries"),
            "seconds": sec, "recall@100": recall_at(ids, w["gt"][:n], min(100, R))}


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
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    out = {}
    codes = {}
    for name, method in (("tensor", scgpu.ENC_TENSOR), ("exact", scgpu.ENC_EXACT)):
        ix.set_encoder(method)
        cid = torch.empty(rows, mcp, dtype=torch.int16, device=dev)
        cod = torch.empty(rows, cfg["mp"], dtype=torch.uint8, device=dev)
        ix.encode_device(X[:65536].data_ptr(), 65536, 0, cid.data_ptr(), cod.data_ptr())  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ix.encode_device(X.data_ptr(), rows, 0, cid.data_ptr(), cod.data_ptr())
        e1.record()
        e1.synchronize()
        out[name + "_rows_per_s"] = rows / (e0.elapsed_time(e1) / 1e3)
        codes[name] = (cid.cpu().numpy(), cod.cpu().numpy())
    ix.set_encoder(scgpu.ENC_TENSOR)
    out["same_codes"] = bool(np.array_equal(codes["tensor"][0], codes["exact"][0]) and
                             np.array_equal(codes["tensor"][1], codes["exact"][1]))
    out["rows"] = rows
    out["what"] = ("Encoder::encode<T> codes (IVF/IMI) of rows drawn from the workload's mixture: tcgen05 "
                   "split-BF16 distance tables + exact double re-check vs the all-double kernel")
    return out


def workload_desc(cfg):
    if cfg["mode"] == "imi":
        idx = "IMI 2x%d, residual PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    elif cfg["mode"] == "sc":
        idx = "second-candidate kc=%d, residual PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    else:
        idx = "IVFADC kc=%d, PQ %dx%d" % (cfg["kc"], cfg["mp"], cfg["kp"])
    return "%s: N=%d D=%d %s, Q=%d, T=%s, R=%d" % (cfg["name"], cfg["N"], cfg["D"], idx, cfg["nq"],
                                                    cfg["T"], cfg["R"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="C2")
    ap.add_argument("--cache", default="/tmp/scg_bench_cache")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default=None, choices=list(PRECISIONS),
                    help="arithmetic of the tables (default: the workload's; fast for the IMI 10M one)")
    ap.add_argument("--queries", type=int, default=0, help="use only the first N queries")
    ap.add_argument("--no-plain", action="store_true", help="skip the FP32 plain comparison")
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
        if rank != 0:
            return
        hbm, _, _ = peaks()
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
                "data": "synthetic", "recall@100": vals[-1]["recall@100"],
                "config": {"workload": workload_desc(cfg), "parallelism": "host threads"},
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

    w = W.build_gpu_workload(args.workload, cache_dir=args.cache, log=log)
    cfg = w["cfg"]
    mode = MODE_IDS[cfg["mode"]]
    mcp = 1 if cfg["mode"] == "sc" else cfg["mc"]
    R, wcap = cfg["R"], cfg["w"]
    T = cfg["T"] if isinstance(cfg["T"], int) else cfg["T"][0]
    if args.queries:
        w["Q"] = w["Q"][: args.queries]
        w["gt"] = w["gt"][: args.queries]
    nq = w["Q"].shape[0]
    if args.precision is None:
        args.precision = cfg.get("precision", "fast")
    rerank = int(cfg.get("shortlist", 0))
    # per-query candidate targets (log-uniform over the config's range, seeded)
    Ts = None
    if not isinstance(cfg["T"], int):
        lo, hi = cfg["T"]
        Ts = np.exp(np.random.default_rng(17).uniform(np.log(lo), np.log(hi), nq)).astype(np.int32)
        T = int(Ts.max())

    ix = scgpu.Index(local)
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

    prec = PRECISIONS[args.precision][0]

    # the scan's chunking picked by the library's autotuner on this batch, for
    # both scan forms (exact and fast)
    tuning = {}
    if args.upl:
        for pv in (prec, 0):
            ix.set_scan_tuning(pv, args.upl)
        tuning = {"fixed_candidates_per_lane": args.upl}
    for name, pv in ((("fast", prec), ("fp32", 0)) if not (args.no_autotune or args.upl) else ()):
        choice, ms = ix.autotune(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(),
                                 d_s.data_ptr(), precision=pv, rerank=rerank)
        tuning[name] = {"candidates_per_lane": choice, "ms_by_choice": dict(zip((2, 4, 8), ms))}

    d_T = None
    if Ts is not None:
        d_T = torch.from_numpy(Ts).to(dev)
        ix.set_query_targets(d_T.data_ptr())

    def step(p=None):
        ix.search_device(mode, dQ.data_ptr(), nq, R, wcap, T, d_ids.data_ptr(), d_d.data_ptr(),
                         d_s.data_ptr(), stream=stream.cuda_stream, precision=prec if p is None else p,
                         rerank=rerank)

    # every other arithmetic form on the same queries, for the comparison
    # (QPS at recall@100): a few timed steps each
    forms = {}
    if not args.no_plain:
        for name, (pv, desc) in PRECISIONS.items():
            if name == args.precision:
                continue
            for _ in range(3):
                step(pv)
            torch.cuda.synchronize()
            pt = []
            for _ in range(3):
                flush.zero_()
                e0p = torch.cuda.Event(enable_timing=True)
                e1p = torch.cuda.Event(enable_timing=True)
                e0p.record(stream)
                step(pv)
                e1p.record(stream)
                e1p.synchronize()
                pt.append(e0p.elapsed_time(e1p))
            pids = d_ids.view(nq, R).cpu().numpy()
            forms[name] = {"value": nq / (statistics.mean(pt) / 1e3), "unit": "queries/s",
                           "recall@100": W.recall_at(pids, w["gt"], min(100, R)),
                           "ms_per_step": statistics.mean(pt), "what": desc,
                           "kernels_ms": dict(zip(("tables_and_prefix", "select_scan", "rerank", "select", "scan"),
                                                  ix.last_timings()))}

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = Clocks(local)
    clocks.start()
    replicas.barrier()
    torch.cuda.synchronize()
    clocks.mark(True)
    times, kern = [], []
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    gc.collect()
    gc.disable()
    for _ in range(args.steps):
        flush.zero_()
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        kern.append(ix.last_timings())
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
            traffic = json.load(open(tpath)).get(("k_search_scan:" if split else "k_search:") + args.workload)
        except Exception:
            traffic = None

    # the same step replayed from a CUDA graph (captured once by the library)
    graph = None
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
        graph = {"value": nq / (statistics.mean(gt_) / 1e3) * world, "unit": "queries/s",
                 "ms_per_step": statistics.mean(gt_),
                 "what": "scg_search_graph: the step's launch sequence captured once, replayed as one graph launch"}

    phases = None
    if args.phases:
        ix.set_phase_counters(True)
        step()
        phases = ix.last_phase_counters()
        phases["per_query_cycles"] = {k: phases[k] / nq for k in
                                      ("sort", "rounds", "cut", "compact", "scan", "final_merge")}
        ix.set_phase_counters(False)

    # end to end through the public host-buffer entry point
    e2e_qps, same, e2e_ms = None, None, None
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
        e2e_qps = nq * len(e2e_times) / sum(e2e_times) * world
        e2e_ms = {"mean": 1e3 * statistics.mean(e2e_times), "p50": 1e3 * statistics.median(e2e_times),
                  "max": 1e3 * max(e2e_times)}
        same = bool(np.array_equal(hid, ids))

    line = {
        "metric": METRIC, "value": job_qps, "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp32": "f32", "fast": "bf16", "bf16": "bf16", "fp16": "f16"}[args.precision],
        "data": "synthetic",
        "config": {"workload": workload_desc(cfg),
                   "precision": PRECISIONS[args.precision][1],
                   "l2": "flushed between steps (256 MB write)", "parallelism": "replicas" if world > 1 else "1 GPU",
                   "timing": "CUDA events per step on the launching stream"},
        "recall@100": recall,
        "rerank_shortlist": rerank or None,
        "per_query_T": None if Ts is None else {"min": int(Ts.min()), "median": int(np.median(Ts)),
                                                "max": int(Ts.max())},
        "fp32_plain": forms.get("fp32"),
        "other_forms": {k: v for k, v in forms.items() if k != "fp32"},
        "phases": phases,
        "latency_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99)),
                       "what": "whole batch of %d queries" % nq},
        "batch_ms": {"p50": float(np.percentile(times, 50)), "p99": float(np.percentile(times, 99))},
        "kernels_ms": {"tables_and_prefix": tables_ms, "select_scan": search_ms, "select": select_ms,
                       "scan": scan_ms, "rerank": rerank_ms},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": ("k_search<.., 2> (ADC scan + top-R; selection runs as its own kernel)" if split
                                else "k_search (fused selection + ADC scan + top-R)"),
                     "alg_bytes_per_launch": alg_bytes},
        "e2e": {"value": e2e_qps, "unit": "queries/s", "h2d_bytes_per_step": int(nq * cfg["D"] * 4),
                "d2h_bytes_per_step": int(nq * R * 8 + nq * 4), "same_ids_as_device_path": same,
                "step_ms": e2e_ms},
        # per step: tensor-core tables, query norms, coarse prefixes,
        # selection, scan (the fused kernel replaces the last two)
        "gpu_launches": (5 if split else 4) * args.steps,
        "autotune": tuning,
        "graph": graph,
        "clocks": ck,
        "candidates_per_query": float(sums.mean()), "cells_per_query": float(nvis.mean() + empty.mean()),
    }
    if args.encode_rows > 0:
        line["encode"] = encode_leg(scgpu, ix, cfg, args.encode_rows, dev)
    if args.serve_seconds > 0:
        line["serving"] = serve_leg(scgpu, ix, w, mode, wcap, T if Ts is None else int(np.median(Ts)), prec,
                                    args.serve_seconds, args.serve_load, rerank=rerank)
        line["latency_ms"] = {"p50": line["serving"]["p50_ms"], "p99": line["serving"]["p99_ms"],
                              "what": "per request of the serving leg"}
    if d_T is not None:
        ix.set_query_targets(None)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if Ts is not None:
                raise RuntimeError("per-query candidate targets are not in the reference's CPU harness")
            line["cpu_baseline"] = cpu_reference(w)
        except Exception as ex:  # reported, never silently dropped
            line["cpu_baseline"] = {"unavailable": repr(ex)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    ix.close()
    replicas.finish()


if __name__ == "__main__":
    main()
