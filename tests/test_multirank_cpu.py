"""The N > 1 bench path on the CPU: two ``gloo`` ranks (the same process-group
calls the NCCL run makes).  Every rank gets its own object (distinct seeds,
weak scaling, no data-path collective) and the timing reduction returns the
maximum over ranks on every rank."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    w, r, local = bench.dist_env()
    dist = bench.init_dist(w, "gloo")
    try:
        seen = bench.max_over_ranks(10.0 + 5.0 * r, dist, "cpu")
        out.put((r, seen, bench.instance_seed(r)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [15.0, 15.0]       # max over ranks, on every rank
    assert got[0][2] != got[1][2]                    # independent objects per rank
