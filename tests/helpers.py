"""Shared helpers of the test suite (fixtures on disk, comparisons)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Golden queries (over all (T, w) rules of a case) whose exact-order result --
# candidate count, top-R ids and distances -- equals the compiled reference's.
# IVFADC / IMI / plain PQ: all of them.  Second candidate: the reference heap
# orders the exactly tied cells (a,b) / (b,a) arbitrarily, so 3 of 20 differ
# by one tied boundary cell.  Three nearest centroids: the six rank
# permutations of a centroid triple tie (up to rounding) and only one of them
# holds vectors, so the reference heap's arbitrary order among them moves the
# cut on 12 of 36 queries.
GOLDEN_SAME_AS_REF = {"imi_d32": 40, "ivf_d32": 40, "plainpq_d32": 10, "sc_d32": 17, "sc3_d32": 24}


def same_as_reference(c, ri, ids, d, sums):
    """Queries of rule ri whose result equals the reference's golden one."""
    R = int(c["R"])
    n = 0
    for i in range(c["Q"].shape[0]):
        if sums[i] == c["r%d_sum" % ri][i]:
            m = min(R, int(sums[i]))
            rid, rd = c["r%d_top_ids" % ri][i][:m], c["r%d_top_d" % ri][i][:m]
            o = np.lexsort((rid, rd))
            if same_topk(ids[i], d[i], rid[o], rd[o], m):
                n += 1
    return n


def golden_cases():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_case(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def oracle_index(O, g):
    D, mc, kc, mp, kp = (int(g[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    return O.Index(D, mc, kc, mp, kp, g["cq"], g["pq"], g["L"], g["pid"], g["icodes"],
                   raw=g["X"].astype(np.float32))


def same_topk(ids_a, d_a, ids_b, d_b, n):
    """True when two top-n lists agree: identical distances position by
    position, and identical ids except inside runs of equal distance (where
    the ids must agree as sets, and a run cut by the n-th position may differ)."""
    ids_a, ids_b = np.asarray(ids_a)[:n], np.asarray(ids_b)[:n]
    d_a, d_b = np.asarray(d_a)[:n], np.asarray(d_b)[:n]
    if not np.array_equal(d_a, d_b):
        return False
    if n == 0:
        return True
    last = d_a[n - 1]
    for v in np.unique(d_a):
        m = d_a == v
        if v == last:
            continue
        if set(ids_a[m].tolist()) != set(ids_b[m].tolist()):
            return False
    return True
