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
               sigma=20.0, train=100_000, iters=25, shortlist=1000),
    "C4": dict(name="imi-1m-d960", N=1_000_000, D=960, mode="imi", mc=2, kc=256,
               mp=32, kp=256, nq=1000, T=30_000, w=1 << 16, R=100, comps=32, sigma=0.08,
               train=50_000, iters=25),
    "C5": dict(name="imi-100m-d96", N=100_000_000, D=96, mode="imi", mc=2, kc=4096,
               mp=16, kp=256, nq=4096, T=30_000, w=1 << 24, R=100, comps=256, sigma=0.05,
               train=200_000, iters=15),
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
