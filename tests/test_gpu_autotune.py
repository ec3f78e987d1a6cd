"""The autotuners: scg_autotune (the scan's candidates per lane) and
scg_autotune_ex (also the coarse-prefix length, the kernel organisation and
the re-rank shortlist).  Every knob leaves the search results unchanged, the
record lists every candidate with its time, and the picks are applied."""
import numpy as np
import pytest

import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


def _index(scgpu, raw=False, kc=64):
    D, mc, mp, kp = 64, 2, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=131)
    X = mix.sample(40000 if kc <= 64 else 120000, seed=132)
    cq, pq = W.train_codebooks(X[:5000], mc, kc, mp, kp, 3, seed=133)
    cid, codes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    L, pid, co, _ = O.distribution(O.IMI, kc, mc, 0, cid, codes)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.load_csr(L, pid, co)
    g.precompute()
    if raw:
        g.load_raw(X)
    return g, mix, D


@pytest.mark.parametrize("prec,kc", [("FAST", 64), ("FP32_EXACT", 64), ("FAST", 1024)])
def test_autotune_ex_keeps_results_and_reports_every_choice(prec, kc):
    """kc = 1024: the coarse-prefix lengths tried (the density rule, 128,
    256, 512) are all shorter than the lists."""
    import torch
    import scgpu
    g, mix, D = _index(scgpu, kc=kc)
    pv = getattr(scgpu, prec)
    nq, R, T = 400, 50, 3000
    Q = mix.sample(nq, seed=140)
    ref_i, ref_d, ref_s = g.search(1, Q, R, 1 << 20, T, precision=pv)
    dQ = torch.from_numpy(Q).cuda()
    di = torch.empty(nq * R, dtype=torch.int32, device="cuda")
    dd = torch.empty(nq * R, dtype=torch.float32, device="cuda")
    ds = torch.empty(nq, dtype=torch.int32, device="cuda")
    rec = g.autotune_ex(1, dQ.data_ptr(), nq, R, 1 << 20, T, di.data_ptr(), dd.data_ptr(), ds.data_ptr(), precision=pv)
    assert rec["candidates_per_lane"]["pick"] in (2, 4, 8)
    assert rec["coarse_prefix"]["pick"] in (0, 128, 256, 512)
    assert rec["kernel_split"]["pick"] in (0, 1)
    fell_back = False
    for knob in ("candidates_per_lane", "coarse_prefix", "kernel_split"):
        ms = rec[knob]["ms_by_choice"]
        assert all(0 < v < 1e4 for v in ms.values()), (knob, ms)
        if knob == "kernel_split" and rec[knob]["pick"] == 0 and ms[1] < ms[0]:
            # the split runs' visited lists outgrew the pool and the fused
            # kernel searched the batch again, so the split's time is that
            # of the second search alone: such a split never wins
            fell_back = True
        else:
            assert ms[rec[knob]["pick"]] == min(ms.values())
    # the outputs of the tuning runs and of searches after it (with the
    # picks applied) are the untuned results
    assert np.array_equal(ds.cpu().numpy(), ref_s)
    assert np.array_equal(dd.view(nq, R).cpu().numpy(), ref_d)
    i2, d2, s2 = g.search(1, Q, R, 1 << 20, T, precision=pv)
    assert np.array_equal(s2, ref_s) and np.array_equal(d2, ref_d) and np.array_equal(i2, ref_i)
    if fell_back:
        # a split search of this batch does end in the fused kernel: no
        # selection or scan kernel time of a split search is recorded
        g.set_kernel_split(True)
        g.search_device(1, dQ.data_ptr(), nq, R, 1 << 20, T, di.data_ptr(), dd.data_ptr(), ds.data_ptr(),
                        precision=pv)
        torch.cuda.synchronize()
        assert g.last_timings()[3] == 0.0 and g.last_timings()[4] == 0.0
    g.close()


def test_autotune_ex_shortlist():
    import torch
    import scgpu
    g, mix, D = _index(scgpu, raw=True)
    nq, R, T, L = 300, 20, 3000, 320
    Q = mix.sample(nq, seed=150)
    dQ = torch.from_numpy(Q).cuda()
    di = torch.empty(nq * R, dtype=torch.int32, device="cuda")
    dd = torch.empty(nq * R, dtype=torch.float32, device="cuda")
    ds = torch.empty(nq, dtype=torch.int32, device="cuda")
    rec = g.autotune_ex(1, dQ.data_ptr(), nq, R, 1 << 20, T, di.data_ptr(), dd.data_ptr(), ds.data_ptr(),
                        precision=scgpu.FAST, rerank=L, min_agree=0.9)
    sl = rec["shortlist"]
    assert sorted(sl["by_length"]) == [20, 40, 80, 160, 320]
    # the caller's own length agrees with itself; the pick meets the bar
    assert sl["by_length"][L]["agree"] == 1.0
    assert sl["by_length"][sl["pick"]]["agree"] >= 0.9
    ok = [Lx for Lx, v in sl["by_length"].items() if v["agree"] >= 0.9]
    assert sl["by_length"][sl["pick"]]["ms"] == min(sl["by_length"][Lx]["ms"] for Lx in ok)
    g.close()


def test_autotune_ex_arguments():
    import scgpu
    g, mix, D = _index(scgpu)
    with pytest.raises(scgpu.ScgError):
        g.autotune_ex(1, 0, 0, 10, 1 << 20, 100, 0, 0, 0)
    g.close()
