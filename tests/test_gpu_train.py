"""Codebook training on the GPU (scg_train_codebooks): k-means++ seeding and
Lloyd steps with FP64 centroid means, for the coarse parts and the residual
PQ subspaces.  Checked: determinism for a seed, the plain-PQ zero centroid,
that Lloyd steps lower the quantisation error, and that the result is as
good as an independent float64 k-means (workloads.train_codebooks) on the
same sample."""
import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def _train(X, mc, kc, mp, kp, iters, seed):
    import torch
    import scgpu
    dX = torch.from_numpy(np.ascontiguousarray(X, np.float32)).cuda()
    D = X.shape[1]
    cq = torch.empty(kc * D, device="cuda")
    pq = torch.empty(kp * D, device="cuda")
    torch.cuda.synchronize()
    scgpu.train_codebooks_device(dX.data_ptr(), X.shape[0], D, mc, kc, mp, kp, iters, seed, cq.data_ptr(),
                                 pq.data_ptr())
    torch.cuda.synchronize()
    return cq.cpu().numpy(), pq.cpu().numpy()


def _mse(X, cq, pq, mc, kc, mp, kp):
    """Mean squared quantisation error of X under (cq, pq) with the
    reference encoder's codes (oracle)."""
    D = X.shape[1]
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    C = cq.reshape(mc, kc, D // mc)
    P = pq.reshape(mp, kp, D // mp)
    rec = np.concatenate([C[i][cid[:, i]] for i in range(mc)], 1)
    rec += np.concatenate([P[j][codes[:, j]] for j in range(mp)], 1)
    return float(((X.astype(np.float64) - rec) ** 2).sum(1).mean())


@pytest.mark.parametrize("mc,kc,mp,kp", [(2, 64, 8, 256), (1, 128, 8, 64), (1, 1, 8, 256)])
def test_train_codebooks(oracle_mod, mc, kc, mp, kp):
    D = 64
    mix = W.Mixture(D, 16, 20.0, "u8", seed=3)
    X = mix.sample(12000, seed=4)
    cq, pq = _train(X, mc, kc, mp, kp, 8, 1234)
    assert np.isfinite(cq).all() and np.isfinite(pq).all()
    cq2, pq2 = _train(X, mc, kc, mp, kp, 8, 1234)
    assert np.array_equal(cq, cq2) and np.array_equal(pq, pq2)  # deterministic
    if kc == 1:
        assert (cq == 0).all()  # plain PQ: the zero coarse centroid
    e8 = _mse(X[:3000], cq, pq, mc, kc, mp, kp)
    c0, p0 = _train(X, mc, kc, mp, kp, 0, 1234)
    e0 = _mse(X[:3000], c0, p0, mc, kc, mp, kp)
    assert e8 < e0  # Lloyd steps lower the error of the seeding
    rc, rp = W.train_codebooks(X, mc, kc, mp, kp, 8, seed=5, zero_coarse=kc == 1)
    er = _mse(X[:3000], np.asarray(rc, np.float32).ravel(), np.asarray(rp, np.float32).ravel(), mc, kc, mp, kp)
    assert e8 <= 1.05 * er, (e8, er)
