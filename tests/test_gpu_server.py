"""The request loop (scg_server_*): continuous batching of mixed requests.

Requests of mixed size, k, arithmetic form and re-rank are submitted from
two threads at once; the server admits them as slots and arena memory free
up and runs them concurrently.  Each result must be identical to the same
request run alone through scg_search (the same kernels on the same inputs:
tolerance zero), requests must have overlapped on the device, and admission
must respect the arena (a request larger than it is refused, a small arena
still completes everything one request at a time).
"""
import threading

import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def index(oracle_mod):
    import scgpu
    D, mc, kc, mp, kp = 64, 2, 64, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=101)
    X = mix.sample(60000, seed=102)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=103)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    g.load_raw(X.astype(np.uint8))
    yield g, mix
    g.close()


def _requests(mix, n, seed):
    import scgpu
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nq = int(np.exp(rng.uniform(0, np.log(400))))
        R = int(rng.choice([1, 10, 100]))
        prec = int(rng.choice([scgpu.FAST, scgpu.FP32_EXACT, scgpu.BF16]))
        rerank = int(rng.choice([0, 0, 200])) if R <= 100 else 0
        T = int(rng.choice([500, 2000, 6000]))
        out.append((mix.sample(nq, seed=seed * 1000 + i), R, T, prec, rerank))
    return out


def test_mixed_requests_equal_alone(index):
    import scgpu
    g, mix = index
    reqs = _requests(mix, 36, 7)
    srv = scgpu.Server(g, slots=3, max_batch=512, max_R=100, arena_bytes=256 << 20)
    tickets = [None] * len(reqs)

    def submit(part):
        for i in part:
            Q, R, T, prec, rr = reqs[i]
            tickets[i] = srv.submit(1, Q, R, 1 << 20, T, precision=prec, rerank=rr)

    th = [threading.Thread(target=submit, args=(range(k, len(reqs), 2),)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    results = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs)
    assert st["max_inflight"] >= 2, st  # requests overlapped on the device
    for (Q, R, T, prec, rr), (ids, d, sums, lat) in zip(reqs, results):
        ai, ad, asum = g.search(1, Q, R, 1 << 20, T, precision=prec, rerank=rr)
        assert np.array_equal(ids, ai) and np.array_equal(d, ad) and np.array_equal(sums, asum)
        assert lat > 0


def test_admission_by_memory(index):
    import scgpu
    g, mix = index
    Q = mix.sample(300, seed=5)
    srv = scgpu.Server(g, slots=4, max_batch=512, max_R=100, arena_bytes=2 << 20)
    # larger than the whole arena: refused at submit
    with pytest.raises(scgpu.ScgError) as e:
        srv.submit(1, Q, 100, 1 << 20, 2000, precision=scgpu.FAST)
    assert e.value.code == -5
    # requests that fit only one or two at a time still all complete
    small = [mix.sample(60, seed=20 + i) for i in range(8)]
    ts = [srv.submit(1, q, 10, 1 << 20, 2000, precision=scgpu.FAST) for q in small]
    for q, t in zip(small, ts):
        ids, d, sums, _ = srv.wait(t)
        ai, ad, _ = g.search(1, q, 10, 1 << 20, 2000, precision=scgpu.FAST)
        assert np.array_equal(ids, ai) and np.array_equal(d, ad)
    # invalid requests are refused like scg_search refuses them
    with pytest.raises(scgpu.ScgError):
        srv.submit(2, small[0], 10, 1 << 20, 2000)
    srv.close()


def test_requests_make_no_device_allocation(index):
    """The server reserves every per-slot device buffer when it starts, so
    requests of up to max_batch queries, of any size, k and arithmetic form,
    make no cudaMalloc: growing a workspace inside the request loop means a
    cudaFree, which waits for the work of every slot."""
    import scgpu
    g, mix = index
    srv = scgpu.Server(g, slots=2, max_batch=1024, max_R=100, arena_bytes=256 << 20)
    before = scgpu.device_allocations()
    forms = [scgpu.FAST, scgpu.FP32_EXACT, scgpu.BF16]
    tickets = []
    for i, nq in enumerate([1, 7, 64, 333, 1024, 1024, 500, 1000, 12]):
        Q = mix.sample(nq, seed=900 + i)
        tickets.append(srv.submit(scgpu.IMI, Q, [1, 10, 100][i % 3], 1 << 20, 4000, precision=forms[(i // 3) % 3]))
    for t in tickets:
        assert srv.wait(t) is not None
    after = scgpu.device_allocations()
    srv.close()
    assert after == before, (before, after)
