"""The bench workloads' index build (workloads.build_gpu_workload, torch
only, run here on the CPU at a reduced size) against the oracle's encoder
and bucketing (pinned to the reference's Encoder / SCEncoder): the same CSR
offsets, row order and codes, and the same ground truth as a float64 brute
force."""
import numpy as np
import pytest

import oracle as O
import workloads as W


@pytest.mark.parametrize("name", ["C1", "C2", "C3", "C4"])
def test_workload_index_equals_oracle_encoder(oracle_mod, name):
    import torch
    small = {"C1": dict(N=20000, nq=20, train=8000, iters=2),
             "C2": dict(N=30000, nq=30, kc=24, train=10000, iters=2),
             "C3": dict(N=30000, nq=30, kc=24, train=10000, iters=2),
             "C4": dict(N=6000, nq=10, kc=12, train=4000, iters=2)}[name]
    w = W.build_gpu_workload(name, device="cpu", overrides=small, log=lambda *a: None)
    cfg = w["cfg"]
    X = W.mixture_sampler(cfg, 1234, torch.device("cpu"))(cfg["N"]).numpy()
    D, kc, mp, kp = cfg["D"], cfg["kc"], cfg["mp"], cfg["kp"]
    if cfg["mode"] == "sc":
        cid, codes = O.sc_encode(D, kc, mp, kp, 2, w["cq"], w["pq"], X)
        L, pid, co, _ = O.distribution(O.SC, kc, 1, 2, cid, codes)
    else:
        mode = O.IMI if cfg["mode"] == "imi" else O.IVFADC
        cid, codes = O.encode((D, cfg["mc"], kc, mp, kp), w["cq"], w["pq"], X)
        L, pid, co, _ = O.distribution(mode, kc, cfg["mc"], 0, cid, codes)
    assert np.array_equal(L, w["L"])
    assert np.array_equal(pid, w["pid"])
    assert np.array_equal(co, w["codes"])
    assert np.array_equal(W.ground_truth_1nn(X, w["Q"]), w["gt"])
