"""recall@R of the drop-in Evaluation (C++), of workloads.recall_at /
comb_recall_at (Python, used by the bench) and of the reference's own
Evaluation::calc_recall / calc_comb_recall (evaluation.h:58-140, compiled in
oracle/_ref) on the same seeded results: identical counts."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def eval_driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("ev") / "eval_driver")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "second-candidate_b200", "cpp"),
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "eval_driver.cpp"),
                    "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("N,R,S", [(200, 100, 1), (300, 10, 3), (50, 1, 4), (0, 5, 2)])
def test_recall_counts_agree(oracle_mod, eval_driver, N, R, S):
    rng = np.random.default_rng(N + R + S)
    gt = rng.integers(0, 1000, N).astype(np.int32)
    sets = []
    for s in range(S):
        ids = rng.integers(0, 1000, (N, R)).astype(np.int32)
        # plant the ground truth at random ranks in some queries, -1 padding in others
        hit = rng.random(N) < 0.3
        ids[hit, rng.integers(0, R, N)[hit]] = gt[hit]
        ids[rng.random(N) < 0.1, R // 2:] = -1
        sets.append(ids)
    text = "%d %d %d\n" % (N, R, S) + "\n".join(" ".join(map(str, a.ravel())) for a in sets) + "\n" + \
        " ".join(map(str, gt)) + "\n"
    out = subprocess.run([eval_driver], input=text, capture_output=True, text=True, check=True).stdout.split()
    drop, drop_comb = int(out[0]), int(out[1])
    py = round(W.recall_at(sets[0], gt, R) * N) if N else 0
    py_comb = round(W.comb_recall_at(sets, gt, R) * N) if N else 0
    assert drop == py and drop_comb == py_comb
    if O.ref_available() and N:
        assert O.ref_calc_recall(sets[0], gt, R) == drop
        assert O.ref_calc_comb_recall(sets, gt, R) == drop_comb
