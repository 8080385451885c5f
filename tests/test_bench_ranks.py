"""bench.py's multi-rank host logic on CPU: two gloo ranks (the same
all-reduce the GPU ranks run over NCCL) agree on the slowest rank's time,
compute the same whole-job frames/s, and detect distinct frames."""
import datetime
import multiprocessing as mp
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    fps = bench.job_frames_per_s(world, 4, 8, t)
    pool = bench.make_pool(rank, 2)
    q.put((rank, t, fps, pool[0].tobytes()[::9973]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_job_rate():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=240) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, f0, s0), (r1, t1, f1, s1) = got
    assert (r0, r1) == (0, 1)
    assert t0 == t1 == 15.0  # the slowest rank's time on every rank
    assert f0 == f1 == 2 * 4 * 8 / 0.015
    assert s0 != s1  # each rank detects its own frames


def test_one_rank_is_its_own_time():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.job_frames_per_s(1, 20, 32, 100.0) == 6400.0
