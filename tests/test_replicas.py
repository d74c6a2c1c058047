"""The N > 1 path of bench.py (replicas only): two gloo ranks on CPU, each
timing different local work; the job's time is the slowest rank's and its
throughput counts the units of both ranks. One rank that raises makes the
other's next collective end with an error within the group's timeout."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out, fail):
    import torch.distributed as dist

    from solarsystemsimulator_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if fail and rank == 1:
            raise RuntimeError("planted failure on rank 1")
        rate, t = replicas.job_rate(100.0, 1.0 + rank)
        out.put((rank, rate, t))
    except RuntimeError as e:
        out.put((rank, "error", str(e)[:80]))
    finally:
        if not (fail and rank == 1):
            dist.destroy_process_group()


def _run(fail):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out, fail)) for r in range(2)]
    for p in procs:
        p.start()
    res = [out.get(timeout=60) for _ in procs]
    for p in procs:
        p.join(timeout=60)
    return sorted(res, key=lambda r: r[0])


def test_two_replicas_max_and_sum():
    res = _run(fail=False)
    for rank, rate, t in res:
        assert t == pytest.approx(2.0)            # the slower rank's time
        assert rate == pytest.approx(100.0)       # 2 ranks x 100 units / 2 s


def test_a_failing_rank_ends_the_others_collective():
    res = _run(fail=True)
    assert res[1][1] == "error"
    assert res[0][1] == "error"                   # rank 0's all_reduce fails instead of hanging


def test_single_process_without_group():
    from solarsystemsimulator_b200 import replicas
    assert replicas.job_rate(50.0, 2.0) == (25.0, 2.0)
