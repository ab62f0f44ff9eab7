"""The benchmark's multi-rank bookkeeping on CPU (gloo, two ranks).

The timed region of every mode ends in a barrier and the maximum of the
per-rank times (with --replicas the rate is the units of all copies over the
slowest rank's time), and the reference arm runs on rank 0 alone.  Both run
here without a GPU.
"""
import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + rank, "cpu")
        rate = bench.whole_job_rate(1000, 4, t, world)
        # the reference arm: ranks other than 0 do no work and succeed
        ref_rc = bench.run_reference(None) if rank != 0 else 0
        out.put((rank, t, rate, ref_rc))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]
    assert all(abs(r[2] - 2 * 1000 * 4 / 11.0) < 1e-9 for r in res)
    assert res[1][3] == 0


def test_single_rank_max_is_identity():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(3.5, "cpu") == 3.5
    assert bench.whole_job_rate(10, 2, 4.0, 1) == 5.0



def test_host_kick_drift_times_every_particle():
    """The reference arm's O(N) step part runs over all particles in any
    split of the host threads (more threads than particles included)."""
    sys.path.insert(0, REPO)
    import bench
    from treepm import ics
    box = ics.lattice_box(4, 100.0, 1.0, 3)  # 64 particles
    for threads in (1, 3, 100):
        assert bench.cpu_kick_drift(box, threads) > 0.0
