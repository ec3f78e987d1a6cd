import numpy as np

import formats


def test_round_trips(tmp_path):
    rng = np.random.default_rng(0)
    X = rng.integers(0, 255, (50, 12)).astype(np.uint8)
    formats.write_vecs(tmp_path / "a.bvecs", X)
    assert np.array_equal(formats.read_vecs(tmp_path / "a.bvecs", np.uint8), X)
    F = rng.standard_normal((40, 7)).astype(np.float32)
    formats.write_vecs(tmp_path / "a.fvecs", F)
    assert np.array_equal(formats.read_vecs(tmp_path / "a.fvecs", np.float32), F)
    C = rng.standard_normal((2, 16, 4)).astype(np.float32)
    formats.write_ctr(tmp_path / "c.ctr_", C, 16, 2, 8)
    c, k, m, d = formats.read_ctr(tmp_path / "c.ctr_")
    assert (k, m, d) == (16, 2, 8) and np.array_equal(c, C.ravel())
    counts = np.array([0, 3, 0, 0, 2, 1, 0], np.int64)
    L = np.cumsum(counts).astype(np.int32)
    pid = rng.permutation(6).astype(np.int32)
    codes = rng.integers(0, 255, (6, 3)).astype(np.uint8)
    formats.write_edat(tmp_path / "e.edat_", L, pid, codes)
    L2, pid2, codes2, ne = formats.read_edat(tmp_path / "e.edat_", 7, 3)
    assert ne == 3 and np.array_equal(L2, L) and np.array_equal(pid2, pid) and np.array_equal(codes2, codes)
