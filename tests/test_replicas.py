"""The replica timing of bench.py --gpus N (second-candidate_b200/replicas.py)
with two gloo ranks on the CPU: the job time is the slowest rank's and the
throughput counts both ranks' queries."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    r, w = replicas.init("gloo", timeout_s=60)
    replicas.barrier()
    qps, slowest = replicas.job_throughput(10.0 + 5.0 * r, 1000)
    out.put((r, w, qps, slowest))
    replicas.finish()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    for _, _, qps, slowest in res:
        assert slowest == 15.0  # the slower rank's time on both ranks
        assert abs(qps - 2 * 1000 / 0.015) < 1e-6
