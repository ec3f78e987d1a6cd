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
    if int(c["mode"]) in (O.SC, O.SC3):
        cid, codes = g.sc_encode(X, 2 if int(c["mode"]) == O.SC else 3)
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


def _enc_case(kind, D, mc, kc, mp, kp, n, seed):
    rng = np.random.default_rng(seed)
    if kind == "u8":
        mix = W.Mixture(D, 16, 20.0, "u8", seed=seed)
        X = mix.sample(n, seed=seed + 1)
        cq, pq = W.train_codebooks(X[:4000], mc, kc, mp, kp, 2, seed=seed + 2)
    elif kind == "unit01":
        mix = W.Mixture(D, 8, 0.08, "unit01", seed=seed)
        X = mix.sample(n, seed=seed + 1)
        cq, pq = W.train_codebooks(X[:3000], mc, kc, mp, kp, 2, seed=seed + 2)
    else:
        # integer data and centroids with duplicates: exact distance ties
        X = rng.integers(0, 4, (n, D)).astype(np.float32)
        cq = rng.integers(0, 4, (mc * kc * (D // mc))).astype(np.float32)
        cq.reshape(mc, kc, -1)[:, 1::2] = cq.reshape(mc, kc, -1)[:, 0::2][:, : kc // 2]
        pq = rng.integers(-1, 2, (mp * kp * (D // mp))).astype(np.float32)
    return X, cq, pq


@pytest.mark.parametrize("kind,D,mc,kc,mp,kp", [("u8", 64, 2, 256, 8, 256), ("u8", 128, 1, 300, 8, 256),
                                               ("unit01", 960, 2, 32, 32, 256), ("ties", 32, 2, 64, 4, 16)])
def test_tensor_encoder_is_exact(oracle_mod, kind, D, mc, kc, mp, kp):
    """The tensor-core encoder (tcgen05 distance tables + exact re-check of
    every centroid within the tables' error margin) gives the reference's
    codes: identical to the double-precision kernel and to the oracle,
    including exact ties (first minimum) and D = 960."""
    import scgpu
    n = 6000 if D < 960 else 1500
    X, cq, pq = _enc_case(kind, D, mc, kc, mp, kp, n, 11 + D)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.set_encoder(scgpu.ENC_TENSOR)
    cid_t, codes_t = g.encode(X)
    g.set_encoder(scgpu.ENC_EXACT)
    cid_e, codes_e = g.encode(X)
    g.close()
    assert np.array_equal(cid_t, cid_e) and np.array_equal(codes_t, codes_e)
    m = min(n, 600)
    ocid, ocodes = O.encode((D, mc, kc, mp, kp), cq, pq, X[:m])
    assert np.array_equal(cid_t[:m], ocid) and np.array_equal(codes_t[:m], ocodes)


@pytest.mark.parametrize("kind,D,kc,mp,kp,nc", [("u8", 64, 256, 8, 256, 2), ("u8", 128, 300, 8, 256, 3),
                                                ("unit01", 960, 64, 32, 256, 2), ("ties", 32, 64, 4, 16, 2),
                                                ("ties", 32, 64, 4, 16, 3)])
def test_tensor_sc_encoder_is_exact(oracle_mod, kind, D, kc, mp, kp, nc):
    """The second-candidate encoder on the tensor cores (nc nearest coarse
    centroids from the candidates within the tables' margin of the nc-th
    smallest, float-rounded comparisons) gives the reference's codes:
    identical to the double-precision kernel and to the oracle, including
    exact ties (equal distances by centroid id) and D = 960."""
    import scgpu
    n = 6000 if D < 960 else 1500
    X, cq, pq = _enc_case(kind, D, 1, kc, mp, kp, n, 23 + D + nc)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, 1, pq, kp, mp, D)
    g.set_encoder(scgpu.ENC_TENSOR)
    cid_t, codes_t = g.sc_encode(X, nc)
    g.set_encoder(scgpu.ENC_EXACT)
    cid_e, codes_e = g.sc_encode(X, nc)
    g.close()
    assert np.array_equal(cid_t, cid_e) and np.array_equal(codes_t, codes_e)
    m = min(n, 600)
    ocid, ocodes = O.sc_encode(D, kc, mp, kp, nc, cq, pq, X[:m])
    assert np.array_equal(cid_t[:m], ocid) and np.array_equal(codes_t[:m], ocodes)
