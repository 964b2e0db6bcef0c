"""The N > 1 host logic of bench.py, on world-size-2 gloo process groups on the CPU.

Multi-GPU here is replicas only: each rank runs its own independent session on its own seeded
frames, with no collective in the data path.  The only collectives are a barrier around the
timed region and the max over ranks of the measured times, taken outside it.  These tests
check that logic (distinct per-rank work, the max over ranks, the whole-job rate, the
reference arm running on rank 0 alone) without a GPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, local = bench.dist_setup()
    seconds = 0.5 + rank                       # per-rank device time of K steps
    slowest = bench.reduce_max(seconds, dist, "cpu")
    # the reference arm: rank 0 alone does work; other ranks return at once
    ref_ran = bench.run_reference(None, w, r) if r != 0 else "rank0"
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, local, bench.rank_seed(r), slowest, bench.aggregate_rate(w, 100, slowest), ref_ran))


def test_two_ranks_gloo():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    rows = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in rows] == [0, 1] and all(r[1] == 2 for r in rows)
    assert rows[0][3] != rows[1][3]                          # each rank its own seeded session
    assert rows[0][4] == rows[1][4] == pytest.approx(1.5)    # max over ranks
    assert rows[0][5] == pytest.approx(2 * 100 / 1.5)        # whole-job frames/s
    assert rows[1][6] is None                                # rank 1 skips the reference arm
