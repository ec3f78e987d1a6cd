"""Per-query tables (batched pre_compute2, query.h:154-184) through the C ABI.

SCG_FP32_EXACT must be bit-identical to the reference's tables (golden
vectors).  The tensor-core forms are checked against a float64 evaluation of
the same tables, with error bounds stated per form, on shapes that exercise
partial tiles (kc, kp not multiples of 256; nq not a multiple of 128) and K
padding (segment lengths not multiples of 16).
"""
import os

import numpy as np
import pytest

import helpers
import workloads as W

pytestmark = pytest.mark.gpu


def _tables(g, precision, Q):
    import torch
    nq = Q.shape[0]
    dQ = torch.from_numpy(np.ascontiguousarray(Q, np.float32)).cuda()
    dqc = torch.full((nq, g.mc * g.kc), float("nan"), device="cuda")
    dqr = torch.full((nq, g.mp * g.kp), float("nan"), device="cuda")
    torch.cuda.synchronize()
    g.query_tables_device(precision, dQ.data_ptr(), nq, dqc.data_ptr(), dqr.data_ptr())
    torch.cuda.synchronize()
    return dqc.cpu().numpy(), dqr.cpu().numpy()


def _f64_tables(Q, cq, pq, D, mc, kc, mp, kp):
    Q = Q.astype(np.float64)
    C = cq.astype(np.float64).reshape(mc, kc, D // mc)
    P = pq.astype(np.float64).reshape(mp, kp, D // mp)
    dqc, dqr, bc, br = [], [], [], []
    # scale of each entry: 2 sum |q_t c_t| for the dot product, plus a share
    # of ||c||^2 for its FP32 rounding
    for i in range(mc):
        q = Q[:, i * (D // mc):(i + 1) * (D // mc)]
        n = (C[i] ** 2).sum(1)[None, :]
        dqc.append(n - 2 * q @ C[i].T)
        bc.append(2 * np.abs(q) @ np.abs(C[i]).T + n * 2.0 ** -18)
    for k in range(mp):
        q = Q[:, k * (D // mp):(k + 1) * (D // mp)]
        n = (P[k] ** 2).sum(1)[None, :]
        dqr.append(n - 2 * q @ P[k].T)
        br.append(2 * np.abs(q) @ np.abs(P[k]).T + n * 2.0 ** -18)
    return np.concatenate(dqc, 1), np.concatenate(dqr, 1), np.concatenate(bc, 1), np.concatenate(br, 1)


def test_exact_tables_match_golden(oracle_mod):
    import scgpu
    for name in ("ivf_d32", "plainpq_d32", "imi_d32", "sc_d32"):
        c = helpers.load_case(os.path.join(helpers.GOLDEN, name + ".npz"))
        D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
        g = scgpu.Index(0)
        g.load_codebooks(c["cq"], kc, mc, c["pq"], kp, mp, D)
        g.precompute()
        dqc, dqr = _tables(g, scgpu.FP32_EXACT, c["Q"])
        assert np.array_equal(dqc[0], c["dqc0"]), name
        assert np.array_equal(dqr[0], c["dqr0"]), name
        g.close()


# (D, mc, kc, mp, kp, nq, value kind)
SHAPES = [
    (128, 2, 1024, 8, 256, 300, "u8"),   # the IMI 10M workload's table shapes
    (64, 1, 300, 8, 100, 130, "u8"),     # partial entry tiles
    (96, 2, 48, 16, 256, 1, "unit"),     # segment length 6 -> K padded to 16
    (960, 2, 64, 32, 256, 129, "unit01"),  # segment lengths 480 and 30
]

# max |error| / (2 sum |q_t c_t|) per form.  One BF16 product: 2u, u = 2^-8;
# one FP16 product: 2u, u = 2^-11; the hi/lo split drops lo*lo and the
# second rounding residues: 3u^2 = 3 * 2^-16.  Each bound has a factor-2 margin.
BOUNDS = {"FAST": 2.0 ** -13, "BF16": 2.0 ** -6, "FP16": 2.0 ** -9}


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "D%d_mc%d_kc%d_mp%d" % s[:4])
def test_tensor_core_tables(oracle_mod, shape):
    import scgpu
    D, mc, kc, mp, kp, nq, kind = shape
    rng = np.random.default_rng(D + kc + nq)
    if kind == "u8":
        mix = W.Mixture(D, 8, 20.0, "u8", seed=5)
        Q = mix.sample(nq, seed=6)
        cq = rng.uniform(0, 255, (mc * kc * (D // mc))).astype(np.float32)
        pq = rng.normal(0, 15, (mp * kp * (D // mp))).astype(np.float32)
    else:
        Q = rng.normal(0, 1, (nq, D)).astype(np.float32)
        if kind == "unit01":
            Q = np.abs(Q) / 4
        else:
            Q /= np.linalg.norm(Q, axis=1, keepdims=True)
        cq = rng.normal(0, 0.1, mc * kc * (D // mc)).astype(np.float32)
        pq = rng.normal(0, 0.05, mp * kp * (D // mp)).astype(np.float32)
    g = scgpu.Index(0)
    g.load_codebooks(cq, kc, mc, pq, kp, mp, D)
    g.precompute()
    rc, rr, bc, br = _f64_tables(Q, cq, pq, D, mc, kc, mp, kp)
    ec, er = _tables(g, scgpu.FP32_EXACT, Q)
    for form in ("FAST", "BF16", "FP16"):
        tc, tr = _tables(g, getattr(scgpu, form), Q)
        assert np.isfinite(tc).all() and np.isfinite(tr).all(), form
        errc = np.abs(tc - rc) / (bc + 1e-30)
        errr = np.abs(tr - rr) / (br + 1e-30)
        assert errc.max() <= BOUNDS[form] and errr.max() <= BOUNDS[form], (form, errc.max(), errr.max())
    # the exact FP32 form is within FP32 rounding of float64
    assert (np.abs(ec - rc) / bc).max() <= 2.0 ** -12
    assert (np.abs(er - rr) / br).max() <= 2.0 ** -12
    g.close()
