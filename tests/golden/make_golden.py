"""Generates the golden fixtures in this directory by running the REFERENCE
itself (its own headers and sources compiled by oracle/Makefile into
oracle/_ref/libscref.so) on small seeded synthetic inputs.

    python tests/golden/make_golden.py [case ...]   (default: every case)

Needs the reference tree (only readable where the sources live).  Each
fixture ``<name>.npz`` holds the inputs (codebooks in .ctr_ layout, uint8
base vectors, queries), the reference encoder's output, the CSR index read
back from the reference's own .edat_ writer, and per query the reference's
candidate count, empty-cell count and full candidate (id, distance) set, plus
the top-R ids and distances of its batched entry point.
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "second-candidate_b200"))

import formats  # noqa: E402
import oracle as O  # noqa: E402
import workloads as W  # noqa: E402

# T never exceeds N for IMI/SC: the reference loops forever once its heap
# empties (multi_query.h:151, sc_query.h:130).
CASES = [
    # name, mode, D, N, mc, kc, mp, kp, nq, (T, w) pairs
    ("ivf_d32", O.IVFADC, 32, 2000, 1, 16, 4, 64, 10, [(300, 16), (50, 3), (0, 16), (3000, 16)]),
    ("plainpq_d32", O.IVFADC, 32, 2000, 1, 1, 8, 64, 10, [(2000, 1)]),
    ("imi_d32", O.IMI, 32, 3000, 2, 16, 4, 64, 10, [(300, 1 << 20), (120, 40), (0, 100), (2990, 1 << 20)]),
    ("sc_d32", O.SC, 32, 3000, 1, 16, 4, 64, 10, [(300, 1 << 20), (150, 12)]),
    # SCQuery::search_mr_ivf3: three nearest centroids per cell, kc^3 cells
    ("sc3_d32", O.SC3, 32, 4000, 1, 10, 4, 64, 12, [(300, 1 << 20), (120, 9), (0, 100)]),
]
R = 20


def make_case(name, mode, D, N, mc, kc, mp, kp, nq, rules, seed):
    mix = W.Mixture(D, 8, 20.0, "u8", seed=seed)
    X = mix.sample(N, seed=seed + 1).astype(np.uint8)
    Q = mix.sample(nq, seed=seed + 2).astype(np.float32)
    Xf = X.astype(np.float32)
    cq, pq = W.train_codebooks(Xf[:1500], mc, kc, mp, kp, 6, seed=seed + 3,
                               zero_coarse=(kc == 1))
    nc = {O.SC: 2, O.SC3: 3}.get(mode, 0)
    with tempfile.TemporaryDirectory() as td:
        cqp, pqp, xp = (os.path.join(td, f) for f in ("cq.ctr_", "pq.ctr_", "x.fvecs"))
        formats.write_ctr(cqp, cq, kc, mc, D)
        formats.write_ctr(pqp, pq, kp, mp, D)
        formats.write_vecs(xp, Xf)
        cid, codes = O.ref_encode(cqp, pqp, xp, nc, N, mc, mp)
        O.ref_build_edat(cqp, pqp, xp, nc, td, "g")
        edat = os.path.join(td, "g_mr%d_ivf.edat_" % nc if nc else "g_ivf.edat_")
        ncells = kc ** (nc or mc)
        L, pid, co, ne = formats.read_edat(edat, ncells, mp)
    ix = O.Index(D, mc, kc, mp, kp, cq, pq, L, pid, co, raw=Xf)
    out = dict(mode=mode, D=D, N=N, mc=mc, kc=kc, mp=mp, kp=kp, R=R,
               cq=cq.ravel(), pq=pq.ravel(), X=X, Q=Q, cid=cid[:, : (nc or mc)], codes=codes,
               L=L, pid=pid, icodes=co, rules=np.array(rules, np.int64))
    norm_c, norm_r, dot_cr, dqc, dqr = O.ref_tables(ix.cfg, ix.cq, ix.pq, Q[0])
    out.update(norm_c=norm_c, norm_r=norm_r, dot_cr=dot_cr, dqc0=dqc, dqr0=dqr)
    for ri, (T, w) in enumerate(rules):
        sums, empt, cand_ids, cand_d, offs = [], [], [], [], [0]
        for i in range(nq):
            r = O.ref_search_one(ix, mode, Q[i], R, w, T)
            order = np.lexsort((r["dist"], r["ids"]))
            cand_ids.append(r["ids"][order])
            cand_d.append(r["dist"][order])
            offs.append(offs[-1] + r["sum"])
            sums.append(r["sum"])
            empt.append(r["empty"])
        ids, d, s2, _ = O.ref_search_batch(ix, mode, Q, R, w, T, nthreads=1)
        assert np.array_equal(s2, np.array(sums))
        out["r%d_sum" % ri] = np.array(sums, np.int32)
        out["r%d_empty" % ri] = np.array(empt, np.int32)
        out["r%d_cand_ids" % ri] = np.concatenate(cand_ids).astype(np.int32)
        out["r%d_cand_d" % ri] = np.concatenate(cand_d).astype(np.float32)
        out["r%d_cand_off" % ri] = np.array(offs, np.int64)
        out["r%d_top_ids" % ri] = ids
        out["r%d_top_d" % ri] = d
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "written")


def main():
    O.build(ref=True)
    only = set(sys.argv[1:])
    for k, c in enumerate(CASES):
        if not only or c[0] in only:
            make_case(*c, seed=100 + 17 * k)


if __name__ == "__main__":
    main()
