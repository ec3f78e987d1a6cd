"""Index arithmetic of the fast form's rotated LUT (search_impl.cuh,
scan_chunks), restated in numpy: the bank each lane reads at each step, the
table that bank holds, and the code byte the lane's rotated code word gives
at that step.  Every step of a warp must touch 32 different banks (no
shared-memory bank conflicts) and read, for each lane, the entry of table k
at the candidate's k-th code byte."""
import numpy as np
import pytest


def rotate_code(code, rb):
    """Byte s of the result is byte (s + rb) mod len(code) of code (the
    kernel's rotate_code: word rotation, then funnel shifts)."""
    n = len(code) // 4
    w = np.frombuffer(np.asarray(code, np.uint8).tobytes(), np.uint32)
    qw = rb >> 2
    t = np.array([w[(i + qw) % n] for i in range(n)], np.uint64)
    sh = (rb & 3) * 8
    r = [((int(t[(i + 1) % n]) << 32 | int(t[i])) >> sh) & 0xFFFFFFFF for i in range(n)]
    return np.frombuffer(np.array(r, np.uint32).tobytes(), np.uint8)


@pytest.mark.parametrize("mp", [8, 16, 32])
def test_rotated_lut_is_conflict_free_and_reads_the_right_table(mp):
    rng = np.random.default_rng(mp)
    # LUT fill: word c * 32 + b holds table (b mod mp) at code c
    table_of_bank = np.arange(32) & (mp - 1)
    for base in (0, 32, 4096, 96 * 7):
        codes = rng.integers(0, 256, (32, mp), dtype=np.uint8)  # candidate of lane l: flat base + l
        got = np.zeros((32, mp), np.int64)
        for s in range(mp):
            banks = (np.arange(32) & ~(mp - 1)) + ((np.arange(32) + s) & (mp - 1))
            assert len(set(banks.tolist())) == 32  # 32 lanes, 32 banks
            for lane in range(32):
                rot = rotate_code(codes[lane], lane & (mp - 1))
                k = table_of_bank[banks[lane]]
                flat = base + lane
                assert k == (flat + s) % mp  # the order depends on the candidate only
                assert rot[s] == codes[lane][k]  # the code byte of table k
                got[lane, k] += 1
        assert (got == 1).all()  # every table once per candidate


@pytest.mark.parametrize("n", [2, 4, 8])
def test_rotate_code_matches_byte_rotation(n):
    rng = np.random.default_rng(n)
    code = rng.integers(0, 256, 4 * n, dtype=np.uint8)
    for rb in range(4 * n):
        assert np.array_equal(rotate_code(code, rb), np.roll(code, -rb))
