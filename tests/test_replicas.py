"""The multi-GPU path is replicas (no exchange between GPUs): two gloo ranks on
the CPU check the host-side coordination bench.py uses for N > 1 -- process
group from the environment, barrier, maximum over ranks of the timed region,
and the whole-job rate over all ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "WORLD_SIZE": str(world),
                       "RANK": str(rank), "LOCAL_RANK": str(rank)})
    from dogqc_b200 import replicas
    w, r, local = replicas.setup(timeout_s=60)
    replicas.barrier(w)
    ms = 10.0 + 5.0 * r               # rank 1 is the slower one
    ms_max = replicas.max_over_ranks(ms, w)
    rate = replicas.whole_job_rate(1000, ms_max, w)
    replicas.barrier(w)
    replicas.teardown(w)
    q.put((r, w, local, ms_max, rate))


def test_two_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    for r, w, local, ms_max, rate in out:
        assert w == 2 and local == r
        assert ms_max == pytest.approx(15.0)
        assert rate == pytest.approx(1000 * 2 / 0.015)


def test_one_rank_needs_no_process_group():
    from dogqc_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    w, r, local = replicas.setup()
    assert (w, r, local) == (1, 0, 0)
    assert replicas.max_over_ranks(3.5, w) == 3.5
    assert replicas.whole_job_rate(10, 2.0, w) == pytest.approx(5000.0)
