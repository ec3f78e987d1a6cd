"""The fast form's scan on the rotated, bank-private LUT (kp = 256, mp = 8,
16, 32) through the C ABI: split and fused kernels and the allocation-free
entry point give identical results (the sum order depends on the candidate
only), returned distances agree with a float64 evaluation of ||q - c - r||^2
of the same codes within the fast form's error, and the candidate counts and
top-R match the oracle's exact order except at rare boundary ties."""
import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def _fp64(cq, pq, D, mc, kc, mp, L, pid, codes, q, ids):
    N = pid.shape[0]
    pos_of_id = np.empty(N, np.int64)
    pos_of_id[pid] = np.arange(N)
    cell_of_pos = np.repeat(np.arange(L.shape[0]), np.diff(np.concatenate([[0], L.astype(np.int64)])))
    pos = pos_of_id[ids]
    cell = cell_of_pos[pos]
    cqr = cq.reshape(mc, kc, D // mc).astype(np.float64)
    pqr = pq.reshape(mp, 256, D // mp).astype(np.float64)
    c = np.concatenate([cqr[0][cell // kc], cqr[1][cell % kc]], axis=1)
    r = np.concatenate([pqr[k][codes[pos, k]] for k in range(mp)], axis=1)
    diff = q.astype(np.float64)[None, :] - c - r
    return (diff * diff).sum(1)


@pytest.mark.parametrize("mp", [8, 16, 32])
def test_rotated_lut_scan(oracle_mod, mp):
    import torch

    import scgpu
    D, mc, kc, kp = 64, 2, 32, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=100 + mp)
    X = mix.sample(40000, seed=101)
    Q = mix.sample(64, seed=102)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=103)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    nq, w = Q.shape[0], 1 << 20
    for R, T in ((50, 3000), (10, 200), (100, 9000)):
        g.set_kernel_split(True)
        a = g.search(1, Q, R, w, T, precision=scgpu.FAST)
        g.set_kernel_split(False)
        b = g.search(1, Q, R, w, T, precision=scgpu.FAST)
        g.set_kernel_split(True)
        for x, y in zip(a, b):
            assert np.array_equal(x, y), (R, T)
        dQ = torch.from_numpy(np.ascontiguousarray(Q)).cuda()
        di = torch.empty(nq * R, dtype=torch.int32, device="cuda")
        dd = torch.empty(nq * R, dtype=torch.float32, device="cuda")
        ds = torch.empty(nq, dtype=torch.int32, device="cuda")
        g.search_device_noalloc(1, dQ.data_ptr(), nq, R, w, T, di.data_ptr(), dd.data_ptr(), ds.data_ptr(),
                                precision=scgpu.FAST)
        torch.cuda.synchronize()
        assert np.array_equal(di.cpu().numpy().reshape(nq, R), a[0])
        assert np.array_equal(dd.cpu().numpy().reshape(nq, R), a[1])
        assert np.array_equal(ds.cpu().numpy(), a[2])
        ids, d, sums = a
        ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co)
        oi, od, osum = ix.search(O.IMI, Q, R, w, T, order=O.ORDER_EXACT)
        same = sums == osum
        assert same.mean() >= 0.95
        for i in range(nq):
            m = ids[i] >= 0
            d64 = _fp64(cq, pq, D, mc, kc, mp, L, pid, co, Q[i], ids[i][m])
            assert np.allclose(d[i][m], d64, rtol=1e-4, atol=1e-2), i
            if same[i]:
                k = min(R, int(sums[i]))
                assert len(set(ids[i, :k].tolist()) & set(oi[i, :k].tolist())) >= k - 2
    g.close()
