"""The N-rank (replicas) path of bench.py on the CPU: two processes joined by
a gloo process group over 127.0.0.1.

Each rank solves its own seeded problem (different coefficients, update patch
and right-hand sides per rank, the same on every run), and the whole-job
figure is the sum of the ranks' work over the slowest rank's time, identical
on every rank.
"""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms, fl = [120.0, 300.0][rank], [2e12, 5e12][rank]
        rate, mx, tot = bench.whole_job(ms, fl, "cpu")
        w = bench.WORKLOADS["3d-63"]
        a1, a2, A1, A2, mod, b, _ = bench.make_problem(w, rank)
        again = bench.make_problem(w, rank)
        same = bool(np.array_equal(a1, again[0]) and np.array_equal(b, again[5]))
        q.put((rank, rate, mx, tot, float(np.sum(a1)), tuple(mod[:5]), same))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_whole_job_and_per_rank_problems():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        res = sorted(q.get(timeout=240) for _ in procs)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert [p.exitcode for p in procs] == [0, 0]
    for rank, rate, mx, tot, _, _, same in res:
        assert mx == 300.0 and tot == 7e12            # slowest rank; work of both
        assert abs(rate - 7e12 / 0.3 / 1e12) < 1e-9     # TFLOP/s of the whole job
        assert same                                     # seeded: the same on every run
    assert res[0][4] != res[1][4] and res[0][5] != res[1][5]   # a different problem per rank
