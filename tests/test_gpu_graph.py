"""scg_search_graph: the batched search captured once in a CUDA graph and
replayed.  Replays must equal scg_search_device on the same inputs, follow
new buffer contents (the graph reads the buffers at each launch), and a
change of arguments must re-capture."""
import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def test_graph_replay_equals_device_path(oracle_mod):
    import torch
    import scgpu
    D, mc, kc, mp, kp = 64, 2, 64, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=111)
    X = mix.sample(50000, seed=112)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=113)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    stream = torch.cuda.Stream()
    R = 30
    for prec in (scgpu.FAST, scgpu.FP32_EXACT):
        for nq in (300, 77):
            dQ = torch.empty((nq, D), device="cuda")
            gi = torch.empty(nq * R, dtype=torch.int32, device="cuda")
            gd = torch.empty(nq * R, dtype=torch.float32, device="cuda")
            gs = torch.empty(nq, dtype=torch.int32, device="cuda")
            di, dd, ds = torch.empty_like(gi), torch.empty_like(gd), torch.empty_like(gs)
            for rep in range(3):
                Q = mix.sample(nq, seed=200 + rep + nq)
                dQ.copy_(torch.from_numpy(Q))
                torch.cuda.synchronize()
                g.search_graph(1, dQ.data_ptr(), nq, R, 1 << 20, 1500, gi.data_ptr(), gd.data_ptr(), gs.data_ptr(),
                               stream.cuda_stream, precision=prec)
                g.search_device(1, dQ.data_ptr(), nq, R, 1 << 20, 1500, di.data_ptr(), dd.data_ptr(),
                                ds.data_ptr(), precision=prec)
                torch.cuda.synchronize()
                assert torch.equal(gi, di) and torch.equal(gd, dd) and torch.equal(gs, ds), (prec, nq, rep)
    g.close()


def test_launch_count_of_a_search(oracle_mod):
    """scg_last_launches counts the kernels of the last search: the split
    organisation runs more kernels than the fused one, a re-rank adds one,
    and the first fast-form search also builds the per-vector term."""
    import torch
    import scgpu
    D, mc, kc, mp, kp = 64, 2, 64, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=121)
    X = mix.sample(40000, seed=122)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=123)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    g.load_raw(X.astype(np.uint8))
    nq, R = 200, 20
    dQ = torch.from_numpy(mix.sample(nq, seed=124)).cuda()
    di = torch.empty(nq * 100, dtype=torch.int32, device="cuda")
    dd = torch.empty(nq * 100, dtype=torch.float32, device="cuda")
    ds = torch.empty(nq, dtype=torch.int32, device="cuda")

    def count(prec, rerank=0):
        g.search_device(1, dQ.data_ptr(), nq, R, 1 << 20, 2000, di.data_ptr(), dd.data_ptr(), ds.data_ptr(),
                        precision=prec, rerank=rerank)
        torch.cuda.synchronize()
        return g.last_launches()

    first = count(scgpu.FAST)
    split = count(scgpu.FAST)
    assert first == split + 1  # the per-vector term, once
    assert 5 <= split <= 7, split  # tables, norms, prefixes, selection(s), scan, merge
    assert count(scgpu.FAST, rerank=100) >= split  # the merge gives way to the re-rank
    g.set_kernel_split(False)
    fused = count(scgpu.FAST)
    assert 3 <= fused <= 4 and fused < split, (fused, split)
    assert count(scgpu.FAST, rerank=100) == fused + 1
    g.close()
