"""The replica path of several GPUs, on CPU with gloo (world size 2): every rank
gets the maximum of the ranks' times, and the whole-job rate counts the units of
all ranks over that maximum."""
import os

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from suguru_b200 import replicas as R
    t = R.max_over_ranks(1.0 + rank)  # rank 1 is the slow one
    q.put((rank, R.world(), t, R.whole_job_rate(1000, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_rate():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2, 2]
    assert [o[2] for o in out] == [2.0, 2.0]
    assert [o[3] for o in out] == [1000.0, 1000.0]  # 2 ranks x 1000 units / 2 s


def test_single_rank():
    from suguru_b200 import replicas as R
    assert R.world() == 1 and R.max_over_ranks(3.5) == 3.5 and R.whole_job_rate(10, 2.0) == 5.0
