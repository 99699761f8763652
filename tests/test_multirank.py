"""The multi-GPU bench path on CPU: two `gloo` ranks run bench.py's host logic (torchrun-style env,
barrier, max-over-ranks time, whole-job rate, the reference arm's rank rule) without a GPU. The
rendering itself is per-rank and has no collective (replicas, weak scaling)."""
import contextlib
import io
import multiprocessing as mp
import os
import socket
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    w, r, local = bench.dist_info()
    dist = bench.init_dist(w, local, backend="gloo")
    try:
        bench.barrier(dist)
        # Each rank's own step time; the job's time is the slowest rank's.
        slowest = bench.reduce_max(dist, 10.0 * (r + 1), local)
        rate = bench.whole_job_rate(w, 5, 2_000_000, slowest)
        # The reference arm: ranks other than 0 exit 0 without work or output.
        out = io.StringIO()
        rc = None
        if r != 0:
            with contextlib.redirect_stdout(out):
                rc = bench.run_reference(types.SimpleNamespace(steps=1, warmup=0), w, r)
        bench.barrier(dist)
        q.put((r, w, slowest, rate, rc, out.getvalue()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_max_time_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, slowest, rate, rc, out in res:
        assert w == 2
        assert slowest == 20.0                                  # max over ranks, seen by every rank
        assert abs(rate - 2 * 5 * 2_000_000 / 20.0 / 1e6) < 1e-12  # whole job: both ranks' units
    assert res[1][4] == 0 and res[1][5] == ""                   # rank 1 of the reference arm
