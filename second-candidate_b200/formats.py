"""On-disk formats of the reference, read and written with numpy.

* TEXMEX ``.fvecs`` / ``.bvecs`` / ``.ivecs``: every row is an int32 dimension
  followed by that many float32 / uint8 / int32 values (read by
  ``load_data`` / ``load_and_convert_data``, sc_utilities.h:817-886,
  :1078-1143, with a 4-byte row header).
* ``.ctr_`` codebooks: float32 header {k, m, dim} then k*dim float32 values
  laid out [m][k][dim/m] (written by ``PQQuantizer::output``,
  quantizer.h:370-431; read by ``load_codebook``, sc_utilities.h:897-980).
* ``.edat_`` encoded databases: int32 non_empty, int32 N, then for every
  cell in id order int32 L, int32 pid[L], uint8 codes[L*mp] (written by
  ``Encoder::output``, encoder.cpp:207-305, and ``SCEncoder::output``,
  sc_encoder.cpp:83-182; read into CSR by ``PQQuery::load_encoded_data``,
  query.cpp:82-165).
"""
import numpy as np


def write_vecs(path, X):
    X = np.ascontiguousarray(X)
    n, d = X.shape
    if X.dtype == np.float32 or X.dtype == np.int32:
        rows = np.empty((n, d + 1), X.dtype)
        rows[:, 0] = np.array([d], np.int32).view(X.dtype)[0]
        rows[:, 1:] = X
        rows.tofile(path)
    elif X.dtype == np.uint8:
        rows = np.empty((n, d + 4), np.uint8)
        rows[:, :4] = np.frombuffer(np.int32(d).tobytes(), np.uint8)
        rows[:, 4:] = X
        rows.tofile(path)
    else:
        raise TypeError(X.dtype)


def read_vecs(path, dtype):
    raw = np.fromfile(path, np.uint8)
    d = int(raw[:4].view(np.int32)[0])
    item = np.dtype(dtype).itemsize
    row = 4 + d * item
    n = raw.size // row
    rows = raw[: n * row].reshape(n, row)
    return np.ascontiguousarray(rows[:, 4:]).view(dtype).reshape(n, d)


def write_ctr(path, centers, k, m, dim):
    c = np.ascontiguousarray(centers, np.float32).ravel()
    if c.size != k * dim:
        raise ValueError("codebook holds %d values, expected %d" % (c.size, k * dim))
    np.concatenate([np.array([k, m, dim], np.float32), c]).tofile(path)


def read_ctr(path):
    a = np.fromfile(path, np.float32)
    k, m, dim = int(a[0]), int(a[1]), int(a[2])
    return a[3 : 3 + k * dim].copy(), k, m, dim


def write_edat(path, L, pid, codes):
    """L is the inclusive prefix count per cell (the CSR the reference loads)."""
    L = np.asarray(L, np.int64)
    counts = np.diff(np.concatenate([[0], L]))
    mp = codes.shape[1]
    pid = np.ascontiguousarray(pid, np.int32)
    codes = np.ascontiguousarray(codes, np.uint8)
    with open(path, "wb") as f:
        f.write(np.array([int((counts > 0).sum()), pid.shape[0]], np.int32).tobytes())
        start = 0
        nz = np.nonzero(counts)[0]
        prev = 0
        for c in nz:
            if c > prev:
                f.write(np.zeros(c - prev, np.int32).tobytes())
            l = int(counts[c])
            f.write(np.int32(l).tobytes())
            f.write(pid[start : start + l].tobytes())
            f.write(codes[start : start + l].tobytes())
            start += l
            prev = c + 1
        if prev < L.size:
            f.write(np.zeros(L.size - prev, np.int32).tobytes())


def read_edat(path, ncells, mp):
    """Returns (L inclusive prefix int32, pid, codes[N, mp], non_empty)."""
    raw = np.fromfile(path, np.uint8)
    non_empty, N = (int(v) for v in raw[:8].view(np.int32))
    L = np.zeros(ncells, np.int32)
    pid = np.zeros(N, np.int32)
    codes = np.zeros((N, mp), np.uint8)
    pos, base, acc = 8, 0, 0
    for c in range(ncells):
        l = int(raw[pos : pos + 4].view(np.int32)[0])
        pos += 4
        if l > 0:
            pid[base : base + l] = raw[pos : pos + 4 * l].view(np.int32)
            pos += 4 * l
            codes[base : base + l] = raw[pos : pos + l * mp].reshape(l, mp)
            pos += l * mp
            base += l
        acc += l
        L[c] = acc
    return L, pid, codes, non_empty
