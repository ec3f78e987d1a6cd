"""The C restatement against the compiled reference on fresh seeded inputs
(skipped where the reference tree is not present to build it)."""
import os
import tempfile

import numpy as np
import pytest

import formats
import oracle as O
import workloads as W



@pytest.fixture(scope="module")
def refbuilt(oracle_mod):
    if not O.ref_available():
        pytest.skip("reference harness not built")
    return True


def _index(mode, D, N, mc, kc, mp, kp, seed):
    mix = W.Mixture(D, 8, 20.0, "u8", seed=seed)
    X = mix.sample(N, seed=seed + 1)
    Q = mix.sample(16, seed=seed + 2)
    cq, pq = W.train_codebooks(X[:2000], mc, kc, mp, kp, 4, seed=seed + 3)
    if mode == O.SC:
        cid, codes = O.sc_encode(D, kc, mp, kp, 2, cq, pq, X)
        L, pid, co, _ = O.distribution(O.SC, kc, 1, 2, cid, codes)
    else:
        cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        L, pid, co, _ = O.distribution(mode, kc, mc, 0, cid, codes)
    return O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co, raw=X), Q, X, cq, pq


@pytest.mark.parametrize("mode,mc,kc", [(O.IVFADC, 1, 32), (O.IMI, 2, 24), (O.SC, 1, 24)])
@pytest.mark.parametrize("real_dist", [False, True])
def test_search_matches_reference(refbuilt, mode, mc, kc, real_dist):
    ix, Q, X, cq, pq = _index(mode, 48, 6000, mc, kc, 6, 128, seed=7 + mode)
    w = kc if mode == O.IVFADC else 1 << 20
    for T in (1, 500, 2500):
        for i in range(Q.shape[0]):
            a = ix.search_one(mode, Q[i], w, T, order=O.ORDER_HEAP, real_dist=real_dist)
            b = O.ref_search_one(ix, mode, Q[i], 10, w, T, real_dist=real_dist)
            assert a["sum"] == b["sum"]
            assert sorted(zip(a["ids"].tolist(), a["dist"].tolist())) == \
                sorted(zip(b["ids"].tolist(), b["dist"].tolist()))


def test_encoders_match_reference(refbuilt):
    for mode, mc, kc, nc in [(O.IMI, 2, 32, 0), (O.IVFADC, 1, 40, 0), (O.SC, 1, 32, 2), (O.SC, 1, 32, 3)]:
        D, mp, kp = 32, 4, 64
        mix = W.Mixture(D, 8, 20.0, "u8", seed=3)
        X = mix.sample(3000, seed=4)
        cq, pq = W.train_codebooks(X[:1500], mc, kc, mp, kp, 3, seed=5)
        with tempfile.TemporaryDirectory() as td:
            cqp, pqp, xp = (os.path.join(td, f) for f in ("cq.ctr_", "pq.ctr_", "x.fvecs"))
            formats.write_ctr(cqp, cq, kc, mc, D)
            formats.write_ctr(pqp, pq, kp, mp, D)
            formats.write_vecs(xp, X)
            cid_r, codes_r = O.ref_encode(cqp, pqp, xp, nc, X.shape[0], mc, mp)
        if nc:
            cid, codes = O.sc_encode(D, kc, mp, kp, nc, cq, pq, X)
        else:
            cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        assert np.array_equal(cid, cid_r[:, :cid.shape[1]])
        assert np.array_equal(codes, codes_r)


def test_edat_writer_matches_reference(refbuilt):
    D, mc, kc, mp, kp = 32, 2, 8, 4, 32
    mix = W.Mixture(D, 8, 20.0, "u8", seed=9)
    X = mix.sample(1500, seed=10)
    cq, pq = W.train_codebooks(X, mc, kc, mp, kp, 3, seed=11)
    with tempfile.TemporaryDirectory() as td:
        cqp, pqp, xp = (os.path.join(td, f) for f in ("cq.ctr_", "pq.ctr_", "x.fvecs"))
        formats.write_ctr(cqp, cq, kc, mc, D)
        formats.write_ctr(pqp, pq, kp, mp, D)
        formats.write_vecs(xp, X)
        O.ref_build_edat(cqp, pqp, xp, 0, td, "t")
        ref_bytes = open(os.path.join(td, "t_ivf.edat_"), "rb").read()
        cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
        L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
        mine = os.path.join(td, "mine.edat_")
        formats.write_edat(mine, L, pid, co)
        assert open(mine, "rb").read() == ref_bytes[:len(open(mine, "rb").read())]
        L2, pid2, co2, ne = formats.read_edat(mine, kc * kc, mp)
        assert np.array_equal(L2, L) and np.array_equal(pid2, pid) and np.array_equal(co2, co)
