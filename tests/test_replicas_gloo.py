"""The multi-GPU path of bench.py runs independent replicas (no collective on
the data path); its only cross-rank steps are the barrier and the max/sum
reductions of the timing.  Checked here with two gloo ranks on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    barrier, maxred, sumred = bench.make_reducers(torch, world, "cpu")
    barrier()
    ms = 100.0 + 50.0 * rank          # each replica's device time
    pushes = 1_000_000 * (rank + 1)   # each replica's particle pushes
    t = maxred(ms)
    n = sumred(pushes)
    q.put((rank, t, n, n / (t * 1e-3)))
    dist.destroy_process_group()


def test_two_replicas_time_is_max_and_work_is_sum():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, n, rate in res:
        assert t == 150.0 and n == 3_000_000
        assert rate == pytest.approx(3_000_000 / 0.150)


def test_single_rank_reducers_are_identity():
    import bench
    barrier, maxred, sumred = bench.make_reducers(torch, 1, "cpu")
    barrier()
    assert maxred(3.5) == 3.5 and sumred(7) == 7
