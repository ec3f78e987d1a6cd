"""Shortlist re-rank (scg_search_params.rerank = L) through the C ABI.

The ADC search keeps the top-L of each query, then every shortlisted id gets
the exact distance of the reference's real_dist branch (query.h:307-312:
distance_l2_square, float differences summed in double) and the R smallest
remain.  With the exact arithmetic form the shortlist equals the oracle's, so
ids and distances must be identical to the oracle's re-rank (orc_rerank).
"""
import numpy as np
import pytest

import helpers
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu

MODES = {O.IVFADC: 0, O.IMI: 1, O.SC: 2}


def _build(mode, mc, kc, D, kind, seed, mp=8):
    kp = 256
    if kind == "u8":
        mix = W.Mixture(D, 16, 20.0, "u8", seed=seed)
        X = mix.sample(30000, seed=seed + 1)
        Q = mix.sample(40, seed=seed + 2)
    else:
        rng = np.random.default_rng(seed)
        means = rng.normal(0, 1, (16, D))
        X = (means[rng.integers(0, 16, 30000)] + 0.3 * rng.normal(0, 1, (30000, D))).astype(np.float32)
        Q = (means[rng.integers(0, 16, 40)] + 0.3 * rng.normal(0, 1, (40, D))).astype(np.float32)
    cq, pq = W.train_codebooks(X[:4000], mc, kc, mp, kp, 4, seed=seed + 3)
    if mode == O.SC:
        cid, codes = O.sc_encode(D, kc, mp, kp, 2, cq, pq, X)
        L, pid, co, _ = O.distribution(O.SC, kc, 1, 2, cid, codes)
    else:
        cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        L, pid, co, _ = O.distribution(mode, kc, mc, 0, cid, codes)
    ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co, raw=X.astype(np.float32))
    return X, Q, cq, pq, L, pid, co, ix, (D, mc, kc, mp, kp)


@pytest.mark.parametrize("mode,mc,kc,kind", [(O.IMI, 2, 32, "u8"), (O.SC, 1, 32, "f32"), (O.IVFADC, 1, 64, "f32")])
def test_rerank_matches_oracle(oracle_mod, mode, mc, kc, kind):
    import scgpu
    X, Q, cq, pq, L, pid, co, ix, (D, mc, kc, mp, kp) = _build(mode, mc, kc, 48, kind, 60 + mode)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    g.load_raw(X.astype(np.float32))
    w = kc if mode == O.IVFADC else 1 << 20
    for Lsl, R, T in ((200, 20, 3000), (64, 64, 500), (1000, 100, 8000)):
        ids, d, sums = g.search(MODES[mode], Q, R, w, T, rerank=Lsl)
        si, sd, ssum = ix.search(mode, Q, Lsl, w, T, order=O.ORDER_EXACT)
        assert np.array_equal(sums, ssum)
        ri, rd = ix.rerank(Q, si, R)
        for i in range(Q.shape[0]):
            assert helpers.same_topk(ids[i], d[i], ri[i], rd[i], R), (Lsl, R, T, i)
        # sorted ascending, unused slots (+inf) last
        assert (np.diff(np.where(np.isinf(d), np.float32(3e38), d), axis=1) >= 0).all()
    if kind == "u8":
        # uint8 raw vectors give the same exact distances as their float copies
        ids32, d32, _ = g.search(MODES[mode], Q, 50, w, 3000, rerank=300)
        g.load_raw(X.astype(np.uint8))
        ids8, d8, _ = g.search(MODES[mode], Q, 50, w, 3000, rerank=300)
        assert np.array_equal(ids32, ids8) and np.array_equal(d32, d8)
    g.close()


@pytest.mark.parametrize("mode,mc,kc,kind,D,mp", [(O.IMI, 2, 16, "u8", 40, 8), (O.IVFADC, 1, 32, "f32", 30, 6)])
def test_rerank_unaligned_rows(oracle_mod, mode, mc, kc, kind, D, mp):
    """Rows whose length is not a multiple of 16 bytes (uint8 D = 40, float
    D = 30) take the element-by-element path of the re-rank kernel; it must
    give the same ids and bit-identical distances as the oracle's re-rank."""
    import scgpu
    X, Q, cq, pq, L, pid, co, ix, (D, mc, kc, mp, kp) = _build(mode, mc, kc, D, kind, 80 + mode, mp=mp)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    g.load_raw(X.astype(np.uint8) if kind == "u8" else X.astype(np.float32))
    w = kc if mode == O.IVFADC else 1 << 20
    for Lsl, R, T in ((200, 20, 3000), (1000, 100, 8000)):
        ids, d, sums = g.search(MODES[mode], Q, R, w, T, rerank=Lsl)
        si, sd, ssum = ix.search(mode, Q, Lsl, w, T, order=O.ORDER_EXACT)
        assert np.array_equal(sums, ssum)
        ri, rd = ix.rerank(Q, si, R)
        for i in range(Q.shape[0]):
            assert helpers.same_topk(ids[i], d[i], ri[i], rd[i], R), (Lsl, R, T, i)
    g.close()


@pytest.mark.parametrize("mode,mc,kc,kind,D,mp", [(O.IMI, 2, 32, "u8", 48, 8), (O.SC, 1, 32, "f32", 48, 8),
                                                  (O.IVFADC, 1, 64, "f32", 30, 6), (O.IMI, 2, 16, "u8", 40, 8)])
def test_exact_distance_every_candidate(oracle_mod, mode, mc, kc, kind, D, mp):
    """rerank = -1, the reference's real_dist branch (query.h:307-312,
    multi_query.h:255-259, sc_query.h:232-236): every candidate of the visited
    cells gets its exact distance and the R smallest are returned -- the same
    candidate counts, ids and bit-identical distances as the oracle's
    real_dist search in the exact order (the fast form's coarse tables may
    move a boundary cell of a few queries), split and fused kernels alike."""
    import scgpu
    X, Q, cq, pq, L, pid, co, ix, (D, mc, kc, mp, kp) = _build(mode, mc, kc, D, kind, 90 + mode, mp=mp)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    g.load_raw(X.astype(np.uint8) if kind == "u8" else X.astype(np.float32))
    w = kc if mode == O.IVFADC else 1 << 20
    for R, T in ((20, 3000), (100, 12000), (1, 50)):
        oi, od, osum = ix.search(mode, Q, R, w, T, order=O.ORDER_EXACT, real_dist=True)
        for prec in (scgpu.FP32_EXACT, scgpu.FAST):
            for split in (True, False):
                g.set_kernel_split(split)
                ids, d, sums = g.search(MODES[mode], Q, R, w, T, precision=prec, rerank=-1)
                same = [sums[i] == osum[i] and helpers.same_topk(ids[i], d[i], oi[i], od[i], R)
                        for i in range(Q.shape[0])]
                if prec == scgpu.FP32_EXACT:
                    assert all(same), (R, T, split, np.nonzero(~np.array(same)))
                else:
                    # the fast form's coarse tables may move a boundary cell
                    assert np.mean(same) >= 0.9, (R, T, split, np.mean(same))
    g.close()


def test_rerank_errors(oracle_mod):
    import scgpu
    X, Q, cq, pq, L, pid, co, ix, (D, mc, kc, mp, kp) = _build(O.IMI, 2, 16, 32, "u8", 70)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    with pytest.raises(scgpu.ScgError) as e:      # no raw vectors yet
        g.search(1, Q, 10, 1 << 20, 500, rerank=100)
    assert e.value.code == -6
    with pytest.raises(scgpu.ScgError) as e:      # every-candidate branch without raw vectors
        g.search(1, Q, 10, 1 << 20, 500, rerank=-1)
    assert e.value.code == -6
    g.load_raw(X)
    for bad in (5, 2000, -2):                    # L < R, L > 1024, no such mode
        with pytest.raises(scgpu.ScgError) as e:
            g.search(1, Q, 10, 1 << 20, 500, rerank=bad)
        assert e.value.code == -1
    # fewer candidates than L: unused slots stay -1 / +inf
    ids, d, sums = g.search(1, Q, 10, 1 << 20, 1, rerank=100)
    for i in range(Q.shape[0]):
        m = min(10, int(sums[i]))
        assert (ids[i, m:] == -1).all() and np.isinf(d[i, m:]).all()
    g.close()
