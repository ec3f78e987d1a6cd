"""Index arithmetic of the fast form's bank-private LUT (search_impl.cuh,
scan_chunks / scan_cells / rot_lut_sum), restated in numpy: the bank each
lane reads at each step, the table that bank holds, the code byte that the
lane's word permutation and byte selector give at that step, and the float
the tree over steps sums to.  Every step of a warp must touch 32 different
banks (no shared-memory bank conflicts), read, for each lane, the entry of
table k = s ^ x at the candidate's k-th code byte, and sum to the same float
as the tree over k (so identical codes give identical distances on every
lane)."""
import numpy as np
import pytest


def permute_words(words, xw):
    """Word i moved to i ^ xw, by log steps of swaps on the bits of xw (the
    kernel's permute_words)."""
    r = list(words)
    b = 1
    while b < len(words):
        if xw & b:
            r = [r[i ^ b] for i in range(len(r))]
        b <<= 1
    return r


def byte_select(word, j, x):
    """__byte_perm(word, 0, 0x4440 | (j ^ (x & 3))): byte j ^ (x & 3) of the
    word in the low byte, zeros above."""
    return (int(word) >> (8 * ((j ^ (x & 3)) & 3))) & 0xFF


def tree(v):
    """Pairwise sum v[k] + v[k + s] for s = 1, 2, 4, ... in float32."""
    v = [np.float32(t) for t in v]
    s = 1
    while s < len(v):
        for k in range(0, len(v) - s, 2 * s):
            v[k] = np.float32(v[k] + v[k + s])
        s <<= 1
    return v[0]


@pytest.mark.parametrize("mp", [8, 16, 32])
def test_bank_private_lut_is_conflict_free_and_reads_the_right_table(mp):
    rng = np.random.default_rng(mp)
    lanes = np.arange(32)
    x = lanes & (mp - 1)
    # LUT fill: word c * 32 + b holds table (b mod mp) at code c
    table_of_bank = np.arange(32) & (mp - 1)
    for _ in range(4):
        codes = rng.integers(0, 256, (32, mp), dtype=np.uint8)   # candidate of each lane
        got = np.zeros((32, mp), np.int64)
        for s in range(mp):
            banks = (lanes - x) + (s ^ x)
            assert len(set(banks.tolist())) == 32                # 32 lanes, 32 banks
            for lane in range(32):
                xl = int(x[lane])
                words = np.frombuffer(codes[lane].tobytes(), np.uint32)
                pw = permute_words(words, xl >> 2)
                cb = byte_select(pw[s >> 2], s & 3, xl)
                k = int(table_of_bank[banks[lane]])
                assert k == s ^ xl
                assert cb == codes[lane][k]                      # the code byte of table k
                got[lane, k] += 1
        assert (got == 1).all()                                  # every table once per candidate


@pytest.mark.parametrize("mp", [8, 16, 32])
def test_tree_over_steps_equals_tree_over_tables(mp):
    rng = np.random.default_rng(100 + mp)
    for _ in range(200):
        v = (rng.standard_normal(mp) * rng.choice([1e-3, 1.0, 1e3], mp)).astype(np.float32)
        ref = tree(v)
        for x in range(mp):
            assert tree([v[s ^ x] for s in range(mp)]) == ref


def test_permute_words_is_xor_of_the_index():
    words = list(range(8))
    for xw in range(8):
        assert permute_words(words, xw) == [i ^ xw for i in range(8)]

