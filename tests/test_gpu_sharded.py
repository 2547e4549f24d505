"""View-sharded operators on one GPU: the native partial reconstruction
(dgc_reconstruct_fdk_partial, then dgc_clamp_volume) of two view shards summed
as an all-reduce would sum them, against reconstruct_fdk and the FP64 oracle;
with one rank the sharded functions are the single-device operators.  The
collective itself is covered by the two-rank gloo test."""

import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _scan(A, U, V, seed):
    rng = np.random.default_rng(seed)
    proj = torch.tensor(rng.random((A, U, V)) * 4, dtype=torch.float32, device="cuda")
    cols = [np.arange(A) * (2 * np.pi / A), np.full(A, 300.0), np.full(A, 180.0),
            np.full(A, (U - 1) / 2 + 0.3), np.full(A, (V - 1) / 2 - 0.2), rng.normal(0, 1, A),
            rng.normal(0, 1, A), rng.normal(0, 1, A)]
    geom = [torch.tensor(c, dtype=torch.float32, device="cuda") for c in cols]
    return proj, geom


def test_two_view_shards_sum_to_the_reconstruction(oracle):
    from dgc_b200 import _ops, reconstruct_fdk
    from dgc_b200.sharded import view_shard

    A, U, V, shape, off = 37, 48, 40, (20, 24, 22), (0.4, -0.3, 0.2)
    proj, geom = _scan(A, U, V, 9)
    full = reconstruct_fdk(proj, *geom, 1.0, shape, 1.0, volume_offset=off)
    acc = torch.zeros(shape, dtype=torch.float32, device="cuda")
    parts = []
    for r in range(2):
        s = view_shard(A, 2, r)
        part = _ops.reconstruct_fdk_partial(proj[s.start:s.stop], [g[s.start:s.stop] for g in geom],
                                            1.0, shape, 1.0, off, 0.8, None, math.pi / A)
        parts.append(part)
        acc += part
    assert bool((torch.stack(parts) < 0).any())  # partial volumes are not clamped
    _ops.clamp_volume(acc)
    torch.cuda.synchronize()
    assert rel_l2(acc.cpu(), full.cpu()) < 1e-5
    truth = oracle.reconstruct_fdk(proj.cpu().numpy(), np.stack([g.cpu().numpy() for g in geom]),
                                   1.0, shape, 1.0, off, 0.8)
    assert rel_l2(acc.cpu(), truth) < 1e-5


def test_two_view_shards_offset_preweight():
    """The unclamped partial reconstruction with the offset-aware preweight
    (dgc_reconstruct_fdk_ex, clamp off) of two view shards, summed and
    clamped, against reconstruct_fdk(offset_preweight=True)."""
    from dgc_b200 import _ops, reconstruct_fdk
    from dgc_b200.filtering import preweight_frame
    from dgc_b200.sharded import view_shard

    A, U, V, shape, off = 33, 44, 38, (18, 22, 20), (0.2, 0.3, -0.1)
    proj, geom = _scan(A, U, V, 21)
    full = reconstruct_fdk(proj, *geom, 1.0, shape, 1.0, volume_offset=off,
                           offset_preweight=True)
    acc = torch.zeros(shape, dtype=torch.float32, device="cuda")
    for r in range(2):
        s = view_shard(A, 2, r)
        mine = [g[s.start:s.stop] for g in geom]
        acc += _ops.reconstruct_fdk_ex(proj[s.start:s.stop], mine, 1.0, shape, 1.0, off, 0.8,
                                       preweight_frame(*mine, 1.0), None, math.pi / A,
                                       clamp=False)
    _ops.clamp_volume(acc)
    torch.cuda.synchronize()
    assert rel_l2(acc.cpu(), full.cpu()) < 1e-5


def test_depth_slabs_are_the_reconstruction():
    """Depth-slab sharding on one device: without a process group the slab is
    the whole volume (bit for bit), and each of three slabs, reconstructed as
    a sub-volume at its slab_offset, is the same rows of the whole volume (up
    to the float rounding of the voxel centres)."""
    from cbct_backprojector import reconstruct_fdk
    from dgc_b200.sharded import reconstruct_fdk_slab, slab_offset, slab_shard

    A, U, V, shape, off = 30, 40, 36, (19, 20, 18), (0.3, -0.2, 0.45)
    proj, geom = _scan(A, U, V, 17)
    full = reconstruct_fdk(proj, *geom, 1.0, shape, 1.0, volume_offset=off)
    whole, rows = reconstruct_fdk_slab(proj, *geom, 1.0, shape, 1.0, volume_offset=off)
    assert rows == range(0, shape[0]) and torch.equal(whole, full)
    for r in range(3):
        s = slab_shard(shape[0], 3, r)
        part = reconstruct_fdk(proj, *geom, 1.0, (len(s),) + shape[1:], 1.0,
                               volume_offset=slab_offset(shape, 1.0, off, s))
        assert rel_l2(part.cpu(), full[s.start:s.stop].cpu()) < 1e-5, r


def test_one_rank_is_the_single_device_operator():
    from cbct_backprojector import backproject, project, reconstruct_fdk
    from dgc_b200.sharded import (backproject_sharded, project_sharded,
                                            reconstruct_fdk_sharded)

    A, U, V, shape = 24, 32, 28, (16, 18, 20)
    proj, geom = _scan(A, U, V, 4)
    a = reconstruct_fdk_sharded(proj, *geom, 1.0, shape, 1.0)
    b = reconstruct_fdk(proj, *geom, 1.0, shape, 1.0)
    assert torch.equal(a, b)
    vol = torch.rand(shape, device="cuda")
    outs = []
    for fn in (project_sharded, project):
        v = vol.clone().requires_grad_()
        p = fn(v, *geom, 1.0, U, V, 0.5, 1.0)
        p.square().sum().backward()
        outs.append((p.detach(), v.grad))
    assert torch.equal(outs[0][0], outs[1][0])
    assert rel_l2(outs[0][1].cpu(), outs[1][1].cpu()) < 1e-6  # float atomics
    outs = []
    for fn in (backproject_sharded, backproject):
        q = proj.clone().requires_grad_()
        vb = fn(q, *geom, 1.0, shape, 1.0)
        vb.sum().backward()
        outs.append((vb.detach(), q.grad))
    assert torch.equal(outs[0][0], outs[1][0])
    assert rel_l2(outs[0][1].cpu(), outs[1][1].cpu()) < 1e-6


def _nccl_rank(port, out):
    import os
    from datetime import timedelta

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        from cbct_backprojector import reconstruct_fdk
        from dgc_b200.sharded import reconstruct_fdk_sharded, total_views

        A, U, V, shape = 30, 40, 36, (16, 20, 18)
        proj, geom = _scan(A, U, V, 12)
        n = total_views(A, proj.device)
        a = reconstruct_fdk_sharded(proj, *geom, 1.0, shape, 1.0)
        b = reconstruct_fdk(proj, *geom, 1.0, shape, 1.0)
        torch.cuda.synchronize()
        out.put((n, bool(torch.equal(a, b))))
    finally:
        dist.destroy_process_group()


def test_one_rank_nccl_group():
    """The sharded reconstruction through a real NCCL process group (one
    rank: the all-reduces run, the result is the single-device one)."""
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_rank, args=(port, q))
    p.start()
    p.join(120)
    assert p.exitcode == 0, p.exitcode
    assert q.get(timeout=5) == (30, True)
