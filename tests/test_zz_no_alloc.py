"""The allocation-free search entry point (scg_search_device_noalloc).

Callers that cannot allocate device memory at search time -- a memory pool
that forbids cudaMalloc, or an allocator owned by another component -- use
this entry point; its scratch is a fixed device array inside the library.
This test calls it through the C ABI and checks that two calls in a row give
exactly the output of the allocating entry point, scg_search_device (both run
the same kernels, so the tolerance is zero).  The file is named to be
collected last and must pass both alone and after the rest of the suite.
"""
import os

import numpy as np
import pytest

import helpers
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def _index(scgpu, D, mc, kc, mp, kp, cq, pq, L, pid, codes):
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, codes)
    g.precompute()
    return g


def _cases():
    c = helpers.load_case(os.path.join(helpers.GOLDEN, "imi_d32.npz"))
    yield ("golden", int(c["D"]), int(c["mc"]), int(c["kc"]), int(c["mp"]), int(c["kp"]), c["cq"], c["pq"],
           c["L"], c["pid"], c["icodes"], c["Q"], 1, 300)
    D, mc, kc, mp, kp = 64, 2, 64, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=77)
    X = mix.sample(50000, seed=78)
    Q = mix.sample(300, seed=79)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=80)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    yield ("random", D, mc, kc, mp, kp, cq, pq, L, pid, co, Q, 1, 3000)


def test_noalloc_matches_allocating_search(oracle_mod):
    import torch

    import scgpu
    for name, D, mc, kc, mp, kp, cq, pq, L, pid, codes, Q, mode, T in _cases():
        g = _index(scgpu, D, mc, kc, mp, kp, cq, pq, L, pid, codes)
        dQ = torch.from_numpy(np.ascontiguousarray(Q, np.float32)).cuda()
        nq, R, w = dQ.shape[0], 50, 1 << 20

        def bufs():
            return (torch.empty(nq * R, dtype=torch.int32, device="cuda"),
                    torch.empty(nq * R, dtype=torch.float32, device="cuda"),
                    torch.empty(nq, dtype=torch.int32, device="cuda"))

        for precision in (scgpu.FP32_EXACT, scgpu.FAST):
            ri, rd, rs = bufs()
            g.search_device(mode, dQ.data_ptr(), nq, R, w, T, ri.data_ptr(), rd.data_ptr(), rs.data_ptr(),
                            precision=precision)
            torch.cuda.synchronize()
            for call in range(2):
                ai, ad, as_ = bufs()
                g.search_device_noalloc(mode, dQ.data_ptr(), nq, R, w, T, ai.data_ptr(), ad.data_ptr(),
                                        as_.data_ptr(), precision=precision)
                torch.cuda.synchronize()
                assert torch.equal(as_, rs), (name, precision, call)
                assert torch.equal(ai, ri), (name, precision, call)
                assert torch.equal(ad, rd), (name, precision, call)
        g.close()
