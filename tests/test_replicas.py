"""The multi-GPU form is replicas only (pixels and requests are independent,
the scene is read-only): N processes each render their own frame, the job's
time is the slowest rank's and its throughput every rank's units over that
time.  This checks that host logic with two gloo ranks on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = torch.multiprocessing


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    r, w, local = bench.dist_info()
    # rank 1 is the slow one in the first timing, rank 0 in the second
    times = bench.max_over_ranks([10.0 + 5.0 * r, 7.0 - 3.0 * r], "cpu", w)
    rate = bench.whole_job_rate(1e6, 10, w, times[0])
    queue.put((r, w, local, times, rate))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank_and_the_whole_job():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(i, 2, port, queue)) for i in range(2)]
    for p in procs:
        p.start()
    got = sorted(queue.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, world, local, times, rate) in enumerate(got):
        assert (rank, world, local) == (r, 2, r)
        assert times == [15.0, 7.0]
        # 2 ranks x 10 steps x 1e6 units in 15 ms
        assert rate == pytest.approx(2 * 10 * 1e6 / 0.015 / 1e6)
