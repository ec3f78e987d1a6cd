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


def test_noalloc_limits(oracle_mod):
    """The scratch's batch limit is the one the error message names: one
    query more is refused with SCG_ERR_CAP, exactly that many run.  The
    tensor-core forms are refused (SCG_ERR_STATE) until an allocating call
    has built their per-vector term."""
    import re

    import torch

    import scgpu
    c = helpers.load_case(os.path.join(helpers.GOLDEN, "imi_d32.npz"))
    D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    g = _index(scgpu, D, mc, kc, mp, kp, c["cq"], c["pq"], c["L"], c["pid"], c["icodes"])
    R, w, T = 10, 1 << 20, 300
    nq0 = c["Q"].shape[0]
    dQ0 = torch.from_numpy(np.ascontiguousarray(c["Q"], np.float32)).cuda()
    o = [torch.empty(nq0 * R, dtype=torch.int32, device="cuda"),
         torch.empty(nq0 * R, dtype=torch.float32, device="cuda"),
         torch.empty(nq0, dtype=torch.int32, device="cuda")]
    with pytest.raises(scgpu.ScgError) as e:
        g.search_device_noalloc(1, dQ0.data_ptr(), nq0, R, w, T, *(t.data_ptr() for t in o), precision=scgpu.FAST)
    assert e.value.code == -6
    # find the limit: a batch far beyond it names it (buffers of its full
    # size, so that even a wrong admission stays within them)
    big = 1 << 18
    bq = torch.zeros(big, D, dtype=torch.float32, device="cuda")
    bo = [torch.empty(big * R, dtype=torch.int32, device="cuda"),
          torch.empty(big * R, dtype=torch.float32, device="cuda"),
          torch.empty(big, dtype=torch.int32, device="cuda")]
    with pytest.raises(scgpu.ScgError) as e:
        g.search_device_noalloc(1, bq.data_ptr(), big, R, w, T, *(t.data_ptr() for t in bo))
    assert e.value.code == -5
    del bq, bo
    maxq = int(re.search(r"at most (\d+) queries", str(e.value)).group(1))
    assert 0 < maxq < big
    reps = (maxq + 1 + nq0 - 1) // nq0
    dQ = dQ0.repeat(reps, 1)[: maxq + 1].contiguous()
    ids = torch.empty((maxq + 1) * R, dtype=torch.int32, device="cuda")
    ds = torch.empty((maxq + 1) * R, dtype=torch.float32, device="cuda")
    sums = torch.empty(maxq + 1, dtype=torch.int32, device="cuda")
    with pytest.raises(scgpu.ScgError) as e:
        g.search_device_noalloc(1, dQ.data_ptr(), maxq + 1, R, w, T, ids.data_ptr(), ds.data_ptr(), sums.data_ptr())
    assert e.value.code == -5
    g.search_device_noalloc(1, dQ.data_ptr(), maxq, R, w, T, ids.data_ptr(), ds.data_ptr(), sums.data_ptr())
    torch.cuda.synchronize()
    # every repeated query gives its original's result
    ri, rd, rs = g.search(1, c["Q"], R, w, T)
    got_i = ids[: maxq * R].view(maxq, R).cpu().numpy()
    got_s = sums[:maxq].cpu().numpy()
    for i in range(maxq):
        assert got_s[i] == rs[i % nq0] and np.array_equal(got_i[i], ri[i % nq0])
    g.close()
