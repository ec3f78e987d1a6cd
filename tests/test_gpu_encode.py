"""The CUDA encoders reproduce the reference's codes bit for bit."""
import os

import numpy as np
import pytest

import helpers
import oracle as O
import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", helpers.golden_cases(), ids=lambda p: os.path.basename(p)[:-4])
def test_encoder_golden(oracle_mod, path):
    import scgpu
    c = helpers.load_case(path)
    D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    g = scgpu.Index(0)
    g.load_codebooks(c["cq"], kc, mc, c["pq"], kp, mp, D)
    X = c["X"].astype(np.float32)
    if int(c["mode"]) == O.SC:
        cid, codes = g.sc_encode(X, 2)
    else:
        cid, codes = g.encode(X)
    assert np.array_equal(cid, c["cid"])
    assert np.array_equal(codes, c["codes"])
    g.close()


@pytest.mark.parametrize("mc,kc,nc", [(2, 256, 0), (1, 512, 0), (1, 256, 2), (1, 128, 3)])
def test_encoder_random(oracle_mod, mc, kc, nc):
    import scgpu
    D, mp, kp = 64, 8, 256
    mix = W.Mixture(D, 16, 20.0, "u8", seed=5)
    X = mix.sample(20000, seed=6)
    cq, pq = W.train_codebooks(X[:4000], mc, kc, mp, kp, 3, seed=7)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    if nc:
        cid, codes = g.sc_encode(X, nc)
        ocid, ocodes = O.sc_encode(D, kc, mp, kp, nc, cq, pq, X)
    else:
        cid, codes = g.encode(X)
        ocid, ocodes = O.encode((D, mc, kc, mp, kp), cq, pq, X)
    assert np.array_equal(cid, ocid)
    assert np.array_equal(codes, ocodes)
    g.close()
