"""The coarse-list argument M of search_multi2 / search_mr_ivf with M < kc,
against the compiled reference.

The reference sorts only the M smallest coarse keys of each list
(nth_element_id + sort_id, multi_query.h:125-128, sc_query.h:105-106), which
leaves ranks 0..M in sorted order and the tail in std::nth_element's
unspecified order; its multi-sequence is bounded by kc, not M
(multi_query.h:176,191; sc_query.h:160,173), so a walk that pops a cell
(empty ones included) past rank M - 1 reads that unspecified order.
Whenever every popped cell lies within ranks 0..M-1 of both lists, the
result is the one of M = kc, and the one of the library's rank limit M (the
walk confined to ranks 0..M-1).  This test pins that statement on the
reference itself and records how often it applies."""
import numpy as np
import pytest

import oracle as O
import workloads as W


def _max_rank(ix, mode, q, w, T):
    """Largest rank of either list among the cells the reference's own walk
    (the heap order, restated bit for bit by the oracle) pops, empty cells
    included: a popped rank past M lets the unsorted tail into the heap."""
    return ix.search_one(mode, q, w, T, order=O.ORDER_HEAP)["max_rank"]


@pytest.mark.parametrize("mode,mc,kc", [(O.IMI, 2, 32), (O.SC, 1, 32)])
def test_m_below_kc_equals_full_sort_within_the_prefix(oracle_mod, mode, mc, kc):
    if not O.ref_available():
        pytest.skip("reference harness not built")
    D, mp, kp = 32, 4, 64
    mix = W.Mixture(D, 16, 20.0, "u8", seed=300 + mode)
    X = mix.sample(20000, seed=301)
    Q = mix.sample(40, seed=302)
    cq, pq = W.train_codebooks(X[:4000], mc, kc, mp, kp, 3, seed=303)
    if mode == O.SC:
        cid, codes = O.sc_encode(D, kc, mp, kp, 2, cq, pq, X)
        L, pid, co, _ = O.distribution(O.SC, kc, 1, 2, cid, codes)
    else:
        cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        L, pid, co, _ = O.distribution(mode, kc, mc, 0, cid, codes)
    ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co)
    R, w = 20, 1 << 20
    applies = 0
    for T in (200, 1500):
        full = O.ref_search_batch(ix, mode, Q, R, w, T, nthreads=1)
        for M in (kc // 4, kc // 2):
            part = O.ref_search_batch(ix, mode, Q, R, w, T, nthreads=1, M=M)
            for i in range(Q.shape[0]):
                # ranks 0..M are sorted; a cell popped at rank M - 1 pushes
                # rank M, still in the sorted part
                if _max_rank(ix, mode, Q[i], w, T) + 1 <= M:
                    applies += 1
                    assert part[2][i] == full[2][i]
                    m = min(R, int(full[2][i]))
                    assert np.array_equal(np.sort(part[1][i][:m]), np.sort(full[1][i][:m]))
    assert applies >= 40


@pytest.mark.parametrize("mode,mc,kc", [(O.IMI, 2, 32), (O.SC, 1, 32), (O.SC3, 1, 12)])
def test_rank_limit_confines_the_walk(oracle_mod, mode, mc, kc):
    """The oracle's rank limit (the library's scg_set_rank_limit): every
    popped cell has ranks below M, a walk that never passed M - 1 without
    the limit is unchanged, and a target beyond N ends once the M-grid is
    exhausted (each cell visited once, fewer candidates than the whole
    grid)."""
    D, mp, kp = 32, 4, 64
    mix = W.Mixture(D, 16, 20.0, "u8", seed=400 + mode)
    X = mix.sample(20000, seed=401)
    Q = mix.sample(16, seed=402)
    cq, pq = W.train_codebooks(X[:4000], mc, kc, mp, kp, 3, seed=403)
    if mode in (O.SC, O.SC3):
        nc = 2 if mode == O.SC else 3
        cid, codes = O.sc_encode(D, kc, mp, kp, nc, cq, pq, X)
        L, pid, co, _ = O.distribution(O.SC, kc, 1, nc, cid, codes)
    else:
        cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        L, pid, co, _ = O.distribution(mode, kc, mc, 0, cid, codes)
    ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co)
    w = 1 << 20
    for M in (kc // 4, kc // 2):
        for T in (200, 1500, 10 ** 7):
            for q in Q:
                full = ix.search_one(mode, q, w, T)
                lim = ix.search_one(mode, q, w, T, rank_limit=M)
                assert lim["max_rank"] < M
                if full["max_rank"] < M:
                    assert lim["sum"] == full["sum"]
                    assert np.array_equal(lim["cells"], full["cells"])
                if T == 10 ** 7:
                    assert lim["sum"] <= full["sum"]
                    assert len(set(lim["cells"].tolist())) == len(lim["cells"])
