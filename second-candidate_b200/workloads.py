"""Seeded synthetic workloads for the search path.

The reference measures on TEXMEX SIFT files that are not available here; the
configurations below stand in for them with seeded Gaussian mixtures of the
same shapes, sizes and value ranges (no dataset items are reproduced):

* ``C1`` plain PQ exhaustive ADC (IVFADC with one zero coarse centroid):
  N=100,000, D=128, integer values in [0,255], M=8, K=256, Q=1,000.
* ``C2`` inverted multi-index (2 x 64-d halves x kc=1024) + residual PQ8:
  N=10,000,000, D=128, Q=10,000, T=30,000, top-100.
* ``C3`` second-candidate partition (one 128-d codebook, kc=1024, ordered
  pairs) on the C2 data, per-query T in [5k, 200k].
* ``C4`` D=960 in [0,1], IMI 2 x 480 x kc=256, M=32 (dsub=30), N=1,000,000.
* ``C5`` serving stream, N=100,000,000, D=96 unit-normalised, IMI 2 x 48 x
  kc=4096, M=16.

Codebooks are trained by k-means++ seeding plus Lloyd iterations with the
centroid means accumulated in float64 (the reference's own trainer stops after
one iteration and shifts centroid dimensions, so its codebooks are not used).
"""
import numpy as np

CONFIGS = {
    "C1": dict(name="plain-pq-100k-d128", N=100_000, D=128, mode="ivfadc", mc=1, kc=1,
               mp=8, kp=256, nq=1000, T=100_000, w=1, R=100, comps=64, sigma=20.0,
               train=50_000, iters=25),
    "C2": dict(name="imi-10m-d128", N=10_000_000, D=128, mode="imi", mc=2, kc=1024,
               mp=8, kp=256, nq=10_000, T=30_000, w=1 << 20, R=100, comps=64, sigma=20.0,
               train=100_000, iters=25),
    "C3": dict(name="sc-10m-d128", N=10_000_000, D=128, mode="sc", mc=1, kc=1024,
               mp=8, kp=256, nq=10_000, T=(5_000, 200_000), w=1 << 20, R=100, comps=64,
               sigma=20.0, train=100_000, iters=25, shortlist=1000, precision="bf16"),
    "C4": dict(name="imi-1m-d960", N=1_000_000, D=960, mode="imi", mc=2, kc=256,
               mp=32, kp=256, nq=1000, T=30_000, w=1 << 16, R=100, comps=32, sigma=0.08,
               train=50_000, iters=25, shortlist=1000, precision="fp16"),
    "C5": dict(name="imi-100m-d96", N=100_000_000, D=96, mode="imi", mc=2, kc=4096,
               mp=16, kp=256, nq=4096, T=30_000, w=1 << 24, R=100, comps=256, sigma=0.05,
               train=200_000, iters=15, precision="bf16"),
}


class Mixture:
    """Isotropic Gaussian mixture with equal weights.  ``kind`` selects the
    value treatment: "u8" rounds and clips to [0,255] (means ~ U[0,128]);
    "unit01" clips to [0,1] (means ~ U[0.2,0.8]); "sphere" normalises rows."""

    def __init__(self, D, comps, sigma, kind="u8", seed=0):
        rng = np.random.default_rng(seed)
        self.D, self.comps, self.sigma, self.kind = D, comps, sigma, kind
        if kind == "u8":
            self.means = rng.uniform(0.0, 128.0, (comps, D)).astype(np.float32)
        elif kind == "unit01":
            self.means = rng.uniform(0.2, 0.8, (comps, D)).astype(np.float32)
        else:
            m = rng.standard_normal((comps, D)).astype(np.float32)
            self.means = m / np.linalg.norm(m, axis=1, keepdims=True)

    def sample(self, n, seed):
        rng = np.random.default_rng(seed)
        comp = rng.integers(0, self.comps, n)
        X = self.means[comp] + self.sigma * rng.standard_normal((n, self.D), dtype=np.float32)
        if self.kind == "u8":
            X = np.clip(np.rint(X), 0, 255)
        elif self.kind == "unit01":
            X = np.clip(X, 0.0, 1.0)
        else:
            X /= np.maximum(np.linalg.norm(X, axis=1, keepdims=True), 1e-12)
        return X.astype(np.float32)


def _sqdist(X, C, Cn=None):
    Xn = (X.astype(np.float64) ** 2).sum(1)[:, None]
    if Cn is None:
        Cn = (C.astype(np.float64) ** 2).sum(1)[None, :]
    return Xn + Cn - 2.0 * (X.astype(np.float64) @ C.astype(np.float64).T)


def kmeans(X, k, iters, seed, chunk=16384):
    """k-means++ seeding, then `iters` Lloyd steps; centroid sums in float64.
    Empty clusters keep their previous centroid."""
    rng = np.random.default_rng(seed)
    X = np.ascontiguousarray(X, np.float32)
    n, d = X.shape
    if k >= n:
        C = np.zeros((k, d), np.float32)
        C[:n] = X
        return C
    C = np.empty((k, d), np.float32)
    C[0] = X[rng.integers(n)]
    closest = _sqdist(X, C[:1])[:, 0]
    for i in range(1, k):
        p = np.maximum(closest, 0)
        s = p.sum()
        idx = rng.integers(n) if s <= 0 else rng.choice(n, p=p / s)
        C[i] = X[idx]
        closest = np.minimum(closest, _sqdist(X, C[i : i + 1])[:, 0])
    for _ in range(iters):
        Cn = (C.astype(np.float64) ** 2).sum(1)[None, :]
        lab = np.empty(n, np.int64)
        for s in range(0, n, chunk):
            lab[s : s + chunk] = np.argmin(_sqdist(X[s : s + chunk], C, Cn), axis=1)
        sums = np.zeros((k, d), np.float64)
        np.add.at(sums, lab, X.astype(np.float64))
        cnt = np.bincount(lab, minlength=k).astype(np.float64)
        nz = cnt > 0
        C[nz] = (sums[nz] / cnt[nz, None]).astype(np.float32)
    return C


def train_codebooks(X, mc, kc, mp, kp, iters, seed, zero_coarse=False, sc=False):
    """Coarse codebook [mc][kc][D/mc] and residual PQ codebook [mp][kp][D/mp].
    With zero_coarse the coarse codebook is one all-zero centroid (plain PQ).
    The residual is taken w.r.t. the nearest coarse centroid of each part
    (the residual the encoder stores, encoder.h:155-160)."""
    n, D = X.shape
    bsc, bsp = D // mc, D // mp
    if zero_coarse:
        cq = np.zeros((mc, kc, bsc), np.float32)
    else:
        cq = np.stack([kmeans(X[:, i * bsc:(i + 1) * bsc], kc, iters, seed + 11 * i)
                       for i in range(mc)])
    resid = np.empty_like(X)
    for i in range(mc):
        part = X[:, i * bsc:(i + 1) * bsc]
        lab = np.argmin(_sqdist(part, cq[i]), axis=1)
        resid[:, i * bsc:(i + 1) * bsc] = part - cq[i][lab]
    pq = np.stack([kmeans(resid[:, j * bsp:(j + 1) * bsp], kp, iters, seed + 101 + 7 * j)
                   for j in range(mp)])
    return cq.astype(np.float32), pq.astype(np.float32)


def ground_truth_1nn(X, Q, chunk=4096):
    """Exact nearest neighbour of each query (float64 distances)."""
    best = np.full(Q.shape[0], np.inf)
    arg = np.zeros(Q.shape[0], np.int64)
    Qd = Q.astype(np.float64)
    Qn = (Qd ** 2).sum(1)[:, None]
    for s in range(0, X.shape[0], chunk):
        Xd = X[s:s + chunk].astype(np.float64)
        d = Qn + (Xd ** 2).sum(1)[None, :] - 2.0 * Qd @ Xd.T
        j = np.argmin(d, axis=1)
        v = d[np.arange(Q.shape[0]), j]
        better = v < best
        best[better] = v[better]
        arg[better] = j[better] + s
    return arg


def recall_at(ids, gt, R):
    """Evaluation::calc_recall (evaluation.h:58-92): the fraction of queries
    whose true nearest neighbour is among the first R returned ids."""
    ids = np.asarray(ids)[:, :R]
    return float((ids == np.asarray(gt)[:, None]).any(axis=1).mean())


def comb_recall_at(id_sets, gt, R):
    """Evaluation::calc_comb_recall (evaluation.h:103-140): the fraction of
    queries whose true nearest neighbour is among the first R ids of any of
    the result sets (each [N][>= R])."""
    g = np.asarray(gt)[:, None]
    hit = np.zeros(g.shape[0], bool)
    for ids in id_sets:
        hit |= (np.asarray(ids)[:, :R] == g).any(axis=1)
    return float(hit.mean())


# ---------------------------------------------------------------------------
# Full-size workloads, built on the GPU (data preparation for bench.py; the
# timed search never runs through this code).

def _torch_kmeans(X, k, iters, seed):
    """k-means++ seeding, then Lloyd steps (float32 distances, float64 means)
    on a CUDA tensor X [n, d]."""
    import torch
    g = torch.Generator(device=X.device).manual_seed(seed)
    n, d = X.shape
    C = torch.empty(k, d, device=X.device, dtype=torch.float32)
    C[0] = X[torch.randint(0, n, (1,), generator=g, device=X.device)]
    closest = ((X - C[0]) ** 2).sum(1)
    for i in range(1, k):
        p = closest.clamp_min(0)
        s = p.sum()
        if float(s) <= 0:
            j = torch.randint(0, n, (1,), generator=g, device=X.device)
        else:
            j = torch.multinomial(p / s, 1, generator=g)
        C[i] = X[j]
        closest = torch.minimum(closest, ((X - C[i]) ** 2).sum(1))
    Xn = (X * X).sum(1, keepdim=True)
    Xd = X.double()
    for _ in range(iters):
        dist = Xn + (C * C).sum(1)[None, :] - 2.0 * (X @ C.T)
        lab = dist.argmin(1)
        sums = torch.zeros(k, d, dtype=torch.float64, device=X.device).index_add_(0, lab, Xd)
        cnt = torch.bincount(lab, minlength=k)
        nz = cnt > 0
        C[nz] = (sums[nz] / cnt[nz, None].double()).float()
    return C


def _torch_nearest(X, C):
    import torch
    Xn = (X * X).sum(1, keepdim=True)
    out = torch.empty(X.shape[0], dtype=torch.long, device=X.device)
    for s in range(0, X.shape[0], 1 << 18):
        x = X[s:s + (1 << 18)]
        out[s:s + x.shape[0]] = (Xn[s:s + x.shape[0]] + (C * C).sum(1)[None] - 2.0 * x @ C.T).argmin(1)
    return out


def mixture_sampler(cfg, seed, dev):
    """The workload's generator on the device: `sample(n)` draws n rows
    (torch tensor) from the config's mixture -- "u8" rounded and clipped to
    [0,255] (means ~ U[0,128]), "unit01" clipped to [0,1] (means ~
    U[0.2,0.8]), or unit-normalised; successive calls continue one seeded
    stream."""
    import torch
    D = cfg["D"]
    g = torch.Generator(device=dev).manual_seed(seed)
    kind = "u8" if cfg["sigma"] >= 1 else ("unit01" if cfg["name"].startswith("imi-1m") else "sphere")
    if kind == "u8":
        means = torch.rand(cfg["comps"], D, generator=g, device=dev) * 128.0
    elif kind == "unit01":
        means = 0.2 + 0.6 * torch.rand(cfg["comps"], D, generator=g, device=dev)
    else:
        means = torch.randn(cfg["comps"], D, generator=g, device=dev)
        means /= means.norm(dim=1, keepdim=True)

    def sample(n):
        comp = torch.randint(0, cfg["comps"], (n,), generator=g, device=dev)
        x = means[comp] + cfg["sigma"] * torch.randn(n, D, generator=g, device=dev)
        if kind == "u8":
            x = x.round_().clamp_(0, 255)
        elif kind == "unit01":
            x = x.clamp_(0.0, 1.0)
        else:
            x /= x.norm(dim=1, keepdim=True).clamp_min(1e-12)
        return x.contiguous()

    sample.kind = kind
    return sample


def _nearest64(X, C, k=1, chunk=1 << 17):
    """Indices [n, k] of the k nearest rows of C (ascending distance) for each
    row of X, from float64 distances ||x||^2 + ||c||^2 - 2<x, c> on the device
    (torch); k = 1 takes the lowest index among equal distances."""
    import torch
    Cd = C.double()
    Cn = (Cd * Cd).sum(1)[None]
    out = torch.empty(X.shape[0], k, dtype=torch.long, device=X.device)
    for s in range(0, X.shape[0], chunk):
        x = X[s:s + chunk].double()
        d = (x * x).sum(1, keepdim=True) + Cn - 2.0 * (x @ Cd.T)
        if k == 1:
            out[s:s + x.shape[0], 0] = d.argmin(1)
        else:
            out[s:s + x.shape[0]] = torch.topk(d, k, dim=1, largest=False, sorted=True).indices
    return out


def _exact_nn64(X, Q, chunk=1 << 17):
    """Exact nearest row of X for each query (float64 distances, the lowest
    row among equal distances), torch on the device."""
    import torch
    Qd = Q.double()
    Qn = (Qd * Qd).sum(1)[:, None]
    best = torch.full((Q.shape[0],), float("inf"), dtype=torch.float64, device=Q.device)
    arg = torch.zeros(Q.shape[0], dtype=torch.long, device=Q.device)
    for s in range(0, X.shape[0], chunk):
        x = X[s:s + chunk].double()
        d = Qn + (x * x).sum(1)[None, :] - 2.0 * (Qd @ x.T)
        v, j = d.min(1)
        better = v < best
        best = torch.where(better, v, best)
        arg = torch.where(better, j + s, arg)
    return arg


def build_gpu_workload(name, seed=1234, cache_dir=None, log=print, device=None, overrides=None):
    """Generates config `name` on cuda:0 and returns a dict of host arrays:
    cq, pq (codebooks), L, pid, codes (CSR index in cell order), Q (queries),
    gt (exact nearest neighbour of each query), raw (the base rows, for
    configs with a re-rank shortlist) and the shape facts.

    Data preparation only, in torch on the device -- it loads none of this
    project's kernels, so that the reference's CPU arm and the GPU arm can
    share one cached workload.  The codes are those of Encoder::encode /
    SCEncoder::encode (nearest coarse centroid(s) per part, the float residual
    to the nearest, nearest PQ centroid per subspace), found with float64
    distances; rows are bucketed by cell id in row order (as
    Encoder::distribution does).  Ground truth: the exact nearest base row in
    float64 (exact for the integer-valued configs).  With cache_dir the result
    is kept as .npz and reused.  `device` (default cuda:0) and `overrides`
    (config keys replaced, e.g. a smaller N) serve the tests."""
    import hashlib
    import os
    import time

    import torch

    cfg = dict(CONFIGS[name])
    cfg.update(overrides or {})
    key = hashlib.sha1(repr((name, seed, sorted(cfg.items()), 6)).encode()).hexdigest()[:16]
    path = os.path.join(cache_dir, "%s_%s.npz" % (cfg["name"], key)) if cache_dir else None
    if path and os.path.exists(path):
        z = np.load(path)
        out = {k: z[k] for k in z.files}
        out.update(cfg=cfg)
        log("workload %s loaded from cache" % cfg["name"])
        return out

    t0 = time.time()
    dev = torch.device(device or "cuda:0")
    torch.backends.cuda.matmul.allow_tf32 = False
    N, D, mc, kc, mp, kp = cfg["N"], cfg["D"], cfg["mc"], cfg["kc"], cfg["mp"], cfg["kp"]
    sc = cfg["mode"] == "sc"
    sample = mixture_sampler(cfg, seed, dev)
    X = sample(N)
    Q = sample(cfg["nq"])
    log("generated %d x %d in %.1fs" % (N, D, time.time() - t0))
    # codebooks: coarse (k-means per part, or one zero centroid), residual PQ
    tr = X[: cfg["train"]]
    mcp = 1 if sc else mc
    bsc, bsp = D // mcp, D // mp
    if kc == 1:
        cq = torch.zeros(mcp, 1, bsc, device=dev)
    else:
        cq = torch.stack([_torch_kmeans(tr[:, i * bsc:(i + 1) * bsc].contiguous(), kc, cfg["iters"], seed + 11 * i)
                          for i in range(mcp)])
    resid = tr.clone()
    for i in range(mcp):
        part = tr[:, i * bsc:(i + 1) * bsc].contiguous()
        resid[:, i * bsc:(i + 1) * bsc] -= cq[i][_torch_nearest(part, cq[i])]
    pq = torch.stack([_torch_kmeans(resid[:, j * bsp:(j + 1) * bsp].contiguous(), kp, cfg["iters"], seed + 101 + 7 * j)
                      for j in range(mp)])
    del resid
    cq_h = cq.cpu().numpy().astype(np.float32).ravel()
    pq_h = pq.cpu().numpy().astype(np.float32).ravel()
    log("trained codebooks in %.1fs" % (time.time() - t0))
    # codes: nearest coarse centroid per part (second candidate: the two
    # nearest of the one codebook), float residual to the nearest, nearest PQ
    # centroid per subspace
    step = 1 << 22
    ncid = 2 if sc else mcp
    cid = torch.empty(N, ncid, dtype=torch.long, device=dev)
    codes = torch.empty(N, mp, dtype=torch.uint8, device=dev)
    for s in range(0, N, step):
        x = X[s:s + step]
        r = x.clone()
        for i in range(mcp):
            part = x[:, i * bsc:(i + 1) * bsc]
            nn = _nearest64(part, cq[i], 2 if sc else 1)
            cid[s:s + x.shape[0], i:i + nn.shape[1]] = nn
            r[:, i * bsc:(i + 1) * bsc] -= cq[i][nn[:, 0]]
        for j in range(mp):
            codes[s:s + x.shape[0], j] = _nearest64(r[:, j * bsp:(j + 1) * bsp], pq[j])[:, 0].to(torch.uint8)
        del r
    if dev.type == "cuda":
        torch.cuda.synchronize()
    log("encoded in %.1fs" % (time.time() - t0))
    cell = cid[:, 0] * kc + cid[:, 1] if ncid == 2 else cid[:, 0]
    ncells = kc * kc if (sc or mc == 2) else kc
    cell_sorted, perm = torch.sort(cell, stable=True)
    counts = torch.bincount(cell, minlength=ncells)
    L = counts.cumsum(0).to(torch.int32)
    codes_sorted = codes[perm]
    gt = _exact_nn64(X, Q)
    log("index + ground truth in %.1fs" % (time.time() - t0))
    out = dict(cq=cq_h, pq=pq_h, L=L.cpu().numpy(), pid=perm.to(torch.int32).cpu().numpy(),
               codes=codes_sorted.cpu().numpy(), Q=Q.cpu().numpy(), gt=gt.to(torch.int32).cpu().numpy())
    if cfg.get("shortlist"):
        # raw vectors for the exact re-rank (uint8 when the data are bytes)
        out["raw"] = (X.to(torch.uint8) if sample.kind == "u8" else X).cpu().numpy()
    del X, codes, cid, cell, perm, codes_sorted
    if dev.type == "cuda":
        torch.cuda.empty_cache()
    if path:
        os.makedirs(cache_dir, exist_ok=True)
        tmp = path + ".%d.tmp.npz" % os.getpid()
        np.savez(tmp, **out)
        os.replace(tmp, path)
    out.update(cfg=cfg)
    return out
