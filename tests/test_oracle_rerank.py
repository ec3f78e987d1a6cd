"""The oracle's shortlist re-rank (orc_rerank) against its real_dist branch,
which is pinned to the compiled reference (test_oracle_vs_ref.py): re-ranking
ALL candidates of a query must give the real_dist branch's top-R."""
import numpy as np

import oracle as O
import workloads as W


def test_rerank_of_all_candidates_equals_real_dist(oracle_mod):
    D, mc, kc, mp, kp = 32, 2, 16, 4, 64
    mix = W.Mixture(D, 8, 20.0, "u8", seed=90)
    X = mix.sample(6000, seed=91)
    Q = mix.sample(12, seed=92)
    cq, pq = W.train_codebooks(X[:2000], mc, kc, mp, kp, 3, seed=93)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co, raw=X.astype(np.float32))
    R, T = 25, 700
    ri, rd, _ = ix.search(O.IMI, Q, R, 1 << 20, T, real_dist=True)
    for i in range(Q.shape[0]):
        c = ix.search_one(O.IMI, Q[i], 1 << 20, T)
        oi, od = ix.rerank(Q[i:i + 1], c["ids"][None, :], R)
        m = min(R, c["sum"])
        assert np.array_equal(oi[0, :m], ri[i, :m]) and np.array_equal(od[0, :m], rd[i, :m])
