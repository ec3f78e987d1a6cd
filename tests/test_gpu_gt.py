"""Exact nearest neighbour on the GPU (scg_exact_nn) through the C ABI.

The ground truth that Evaluation::calc_recall (evaluation.h:58-92) scores
against is the brute-force nearest base row of each query under
distance_l2_square (float differences, squared and summed in double).  The
GPU result must be that argmin exactly -- ties to the lowest row index -- and
its distance the float of that double sum.  Cases: uint8-valued data (the
SIFT-like workloads), float data, and duplicated base rows that force ties,
with row counts that span several chunks and leave a ragged last chunk.
"""
import numpy as np
import pytest

import workloads as W

pytestmark = pytest.mark.gpu


def _brute(X, Q):
    ids = np.empty(Q.shape[0], np.int64)
    ds = np.empty(Q.shape[0], np.float32)
    for i, q in enumerate(Q):
        diff = (q[None, :] - X).astype(np.float64)  # float differences, as the reference
        d = (diff * diff).sum(1)
        j = int(np.argmin(d))  # first minimum: lowest row index
        ids[i] = j
        ds[i] = np.float32(d[j])
    return ids, ds


def _data(kind, n, nq, D, seed):
    rng = np.random.default_rng(seed)
    if kind == "u8":
        mix = W.Mixture(D, 16, 20.0, "u8", seed=seed)
        return mix.sample(n, seed=seed + 1).astype(np.float32), mix.sample(nq, seed=seed + 2).astype(np.float32)
    if kind == "ties":
        base = rng.integers(0, 4, (n // 8, D)).astype(np.float32)
        X = base[rng.integers(0, base.shape[0], n)]
        Q = rng.integers(0, 4, (nq, D)).astype(np.float32)
        return X, Q
    X = rng.normal(0, 1, (n, D)).astype(np.float32)
    Q = (X[rng.integers(0, n, nq)] + 0.05 * rng.normal(0, 1, (nq, D))).astype(np.float32)
    return X, Q


@pytest.mark.parametrize("kind,n,nq,D", [("u8", 20000, 300, 128), ("f32", 7777, 65, 96),
                                         ("ties", 5000, 129, 8), ("f32", 300, 3000000 // 10000, 960)])
def test_exact_nn_matches_brute_force(oracle_mod, kind, n, nq, D):
    import torch
    import scgpu
    X, Q = _data(kind, n, nq, D, 11 + n)
    dX = torch.from_numpy(X).cuda()
    dQ = torch.from_numpy(Q).cuda()
    ids = torch.full((nq,), -7, dtype=torch.int32, device="cuda")
    ds = torch.full((nq,), float("nan"), device="cuda")
    torch.cuda.synchronize()
    scgpu.exact_nn_device(dX.data_ptr(), n, dQ.data_ptr(), nq, D, ids.data_ptr(), ds.data_ptr())
    gi, gd = ids.cpu().numpy(), ds.cpu().numpy()
    ri, rd = _brute(X, Q)
    assert np.array_equal(gi, ri), np.nonzero(gi != ri)[0][:5]
    assert np.array_equal(gd, rd)


def test_exact_nn_many_chunks(oracle_mod):
    # nq large enough that a chunk holds only 2^28 / nq rows: many chunks
    import torch
    import scgpu
    n, nq, D = 12000, 40000, 16
    X, Q = _data("u8", n, nq, D, 5)
    dX = torch.from_numpy(X).cuda()
    dQ = torch.from_numpy(Q).cuda()
    ids = torch.empty((nq,), dtype=torch.int32, device="cuda")
    scgpu.exact_nn_device(dX.data_ptr(), n, dQ.data_ptr(), nq, D, ids.data_ptr())
    sel = np.arange(0, nq, 97)
    ri, _ = _brute(X, Q[sel])
    assert np.array_equal(ids.cpu().numpy()[sel], ri)


def test_exact_nn_errors(oracle_mod):
    import scgpu
    with pytest.raises(scgpu.ScgError) as e:
        scgpu.exact_nn_device(0, 10, 0, 1, 4, 0)
    assert e.value.code == -1
