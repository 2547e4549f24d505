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


def _sharded_rank(rank, world, port, out):
    """bench.py's fdk-sharded step on one gloo rank, the library's local
    operators replaced by the FP64 oracle (projection, filter and
    backprojection) so that the check is the workload's split: this rank's
    views, projected, then reconstructed with one sum over the ranks."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import numpy as np
    import torch

    import bench
    from dgc_b200 import sharded
    from oracle import oracle as O

    w, r, _ = bench.dist_env()
    dist = bench.init_dist(w, "gloo")
    try:
        A, U, V, shape = 13, 12, 10, (6, 7, 8)
        bench.WORKLOAD.clear()
        bench.WORKLOAD.update(bench.WORKLOADS["fdk-sharded"], D=shape[0], H=shape[1], W=shape[2],
                              A=A, U=U, V=V, sid=300.0, sod=180.0)
        wl = bench.WORKLOAD
        rng = np.random.default_rng(4)  # the same object on every rank
        vol = rng.random(shape).astype(np.float32)
        cols = [np.arange(A) * (2 * np.pi / A), np.full(A, wl["sid"]), np.full(A, wl["sod"]),
                np.full(A, (U - 1) / 2), np.full(A, (V - 1) / 2), rng.normal(0, 1, A),
                rng.normal(0, 1, A), rng.normal(0, 1, A)]
        geom = np.stack(cols).astype(np.float32)
        mine = sharded.view_shard(A, w, r)
        local = [torch.from_numpy(geom[k, mine.start:mine.stop].copy()) for k in range(8)]

        def project(volume, *args):
            g = np.stack([t.numpy() for t in args[:8]])
            return torch.from_numpy(O.project(volume.numpy(), g, wl["pixel"], U, V, wl["step"],
                                              wl["voxel"], mode=1).astype(np.float32))

        def partial(p, geometry, pixel, vshape, voxel, offset, a, scale, frame=None):
            g = np.stack([t.numpy() for t in geometry])
            f = O.fdk_filter(p.numpy(), pixel, g[2], g[1], a)
            return torch.from_numpy(O.backproject(f, g, pixel, vshape, voxel, offset) * scale)

        sharded.project = project
        sharded._partial_volume = partial
        sharded._clamp = lambda v: v.clamp_min_(0.0)
        proj, recon = bench.sharded_step(torch.from_numpy(vol), local)
        full = O.project(vol, geom, wl["pixel"], U, V, wl["step"], wl["voxel"], mode=1)
        full = full.astype(np.float32)
        truth = O.reconstruct_fdk(full, geom, wl["pixel"], shape, wl["voxel"], alpha=wl["alpha"])
        out.put((r, (mine.start, mine.stop), tuple(proj.shape),
                 float(np.abs(proj.numpy() - full[mine.start:mine.stop]).max()),
                 float(np.linalg.norm(recon.numpy() - truth) / np.linalg.norm(truth))))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_fdk_sharded_workload_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sharded_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert [g[1] for g in got] == [(0, 7), (7, 13)]           # the views split, none twice
    assert [g[2][0] for g in got] == [7, 6]
    assert max(g[3] for g in got) == 0.0                      # each rank projects its own views
    assert max(g[4] for g in got) < 1e-6                      # the summed reconstruction is whole
