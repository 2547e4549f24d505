"""View-sharded operators on the CPU: two ``gloo`` ranks (the process-group
calls an NCCL run makes).  Each rank's local operator is replaced by a CPU
stand-in -- the FP64 oracle's filter and backprojection for the FDK
reconstruction, fixed random linear maps for ``project`` / ``backproject`` --
so what is checked is the sharding: the view ranges, the sum of the partial
volumes before the clamp, the pi / (views of the whole scan) factor, and
where autograd sums gradients over the ranks."""

import os
import socket
from datetime import timedelta

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_view_shard_ranges():
    from dgc_b200.sharded import view_shard

    for views in (0, 1, 7, 360):
        for world in (1, 2, 3, 8):
            got = [view_shard(views, world, r) for r in range(world)]
            assert [v for r in got for v in r] == list(range(views))
            assert max(map(len, got)) - min(map(len, got)) <= 1
    with pytest.raises(ValueError):
        view_shard(4, 2, 2)


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import numpy as np
    import torch
    import torch.distributed as dist

    from dgc_b200 import sharded
    from oracle import oracle as O

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        res = {}
        A, U, V, shape, px, vox, off, alpha = 11, 12, 10, (6, 7, 8), 1.0, 1.0, (0.3, -0.2, 0.1), 0.8
        rng = np.random.default_rng(3)  # the same scan on every rank
        proj = (rng.random((A, U, V)) * 4).astype(np.float32)
        angles = np.arange(A) * (2 * np.pi / A)
        cols = [angles, np.full(A, 300.0), np.full(A, 180.0), np.full(A, (U - 1) / 2),
                np.full(A, (V - 1) / 2), rng.normal(0, 1, A), rng.normal(0, 1, A),
                rng.normal(0, 1, A)]
        geom = np.stack(cols).astype(np.float32)
        mine = sharded.view_shard(A, world, rank)
        res["views"] = (mine.start, mine.stop)
        res["total"] = sharded.total_views(len(mine), "cpu")

        # FDK: oracle filter + backprojection as the rank's partial volume
        def partial(p, geometry, pixel, vshape, voxel, offset, a, scale, frame=None):
            g = np.stack([t.numpy() for t in geometry])
            fr = None if frame is None else [t.numpy() for t in frame]
            f = O.fdk_filter(p.numpy(), pixel, g[2], g[1], a, fr)
            return torch.from_numpy(O.backproject(f, g, pixel, vshape, voxel, offset) * scale)

        sharded._partial_volume = partial
        sharded._clamp = lambda v: v.clamp_min_(0.0)
        local = [torch.from_numpy(geom[k, mine.start:mine.stop].copy()) for k in range(8)]
        vol = sharded.reconstruct_fdk_sharded(
            torch.from_numpy(proj[mine.start:mine.stop].copy()), *local, px, shape, vox,
            volume_offset=off, alpha=alpha)
        truth = O.reconstruct_fdk(proj, geom, px, shape, vox, off, alpha)
        res["fdk_err"] = float(np.linalg.norm(vol.numpy() - truth) / np.linalg.norm(truth))
        res["fdk_negative_clamped"] = bool((vol >= 0).all())
        # the offset-aware preweight: each rank's frames from its own views
        vol = sharded.reconstruct_fdk_sharded(
            torch.from_numpy(proj[mine.start:mine.stop].copy()), *local, px, shape, vox,
            volume_offset=off, alpha=alpha, offset_preweight=True)
        truth = O.reconstruct_fdk(proj, geom, px, shape, vox, off, alpha, offset_preweight=True)
        res["fdk_frame_err"] = float(np.linalg.norm(vol.numpy() - truth) / np.linalg.norm(truth))

        # project: linear stand-in p_a = M_a vol; loss = 0.5 sum over this rank's p^2
        n = shape[0] * shape[1] * shape[2]
        M = torch.from_numpy(rng.standard_normal((A, U * V, n)))
        v0 = torch.from_numpy(rng.standard_normal(shape))
        sharded.project = lambda volume, *rest: torch.einsum(
            "apk,k->ap", M[mine.start:mine.stop], volume.reshape(-1)).reshape(-1, U, V)
        v = v0.clone().requires_grad_()
        p = sharded.project_sharded(v, *local, px, U, V, group=None)
        (0.5 * p.square().sum()).backward()
        vf = v0.clone().requires_grad_()
        (0.5 * torch.einsum("apk,k->ap", M, vf.reshape(-1)).square().sum()).backward()
        res["project_grad_err"] = float((v.grad - vf.grad).norm() / vf.grad.norm())

        # backproject: linear stand-in vol = sum_a M_a^T p_a; loss = <vol, c>
        c = torch.from_numpy(rng.standard_normal(n))
        pr = torch.from_numpy(rng.standard_normal((A, U, V)))
        sharded.backproject = lambda q, *rest: torch.einsum(
            "apk,ap->k", M[mine.start:mine.stop], q.reshape(q.shape[0], -1)).reshape(shape)
        q = pr[mine.start:mine.stop].clone().requires_grad_()
        b = sharded.backproject_sharded(q, *local, px, shape, vox)
        (b.reshape(-1) * c).sum().backward()
        full = torch.einsum("apk,ap->k", M, pr.reshape(A, -1))
        res["bp_value_err"] = float((b.detach().reshape(-1) - full).norm() / full.norm())
        gfull = torch.einsum("apk,k->ap", M, c).reshape(A, U, V)[mine.start:mine.stop]
        res["bp_grad_err"] = float((q.grad - gfull).norm() / gfull.norm())
        out.put((rank, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_sharded_views():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got[0]["views"] == (0, 6) and got[1]["views"] == (6, 11)
    for r in (0, 1):
        res = got[r]
        assert res["total"] == 11
        assert res["fdk_err"] < 1e-6 and res["fdk_negative_clamped"], res
        assert res["fdk_frame_err"] < 1e-6, res
        assert res["project_grad_err"] < 1e-12, res
        assert res["bp_value_err"] < 1e-12 and res["bp_grad_err"] < 1e-12, res


def _calib_standins(monkeypatch_target):
    """CPU stand-ins for the projection losses: a view's 'measurement' row
    holds its true eight parameters and the loss is the masked squared
    parameter mismatch, so every view's offsets only see their own view."""
    import torch

    def terms(volume, geometry, measured, scan, mask=None):
        r = (torch.stack(list(geometry), 1) - measured).square() * mask
        return r.sum(), mask.sum()

    def fused(volume, geometry, measured, scan, mask=None, denom=None):
        return terms(volume, geometry, measured, scan, mask)[0] / denom

    monkeypatch_target._loss_terms = terms
    monkeypatch_target._fused_loss = fused
    monkeypatch_target._loss = lambda *a, **k: (lambda s, c: s / c)(*terms(*a, **k))


def _calib_problem():
    import numpy as np
    import torch

    rng = np.random.default_rng(8)
    A = 13
    nominal = [torch.tensor(x, dtype=torch.float32) for x in (
        np.arange(A) * (2 * np.pi / A), np.full(A, 300.0), np.full(A, 180.0), np.full(A, 20.0),
        np.full(A, 16.0), np.zeros(A), np.zeros(A), np.zeros(A))]
    scale = np.array([3e-3, 2.0, 2.0, 1.0, 1.0, 0.5, 0.5, 0.5])
    true = [g + torch.tensor(rng.normal(0, s, A), dtype=torch.float32)
            for g, s in zip(nominal, scale)]
    measured = torch.stack(true, 1)
    mask = torch.tensor(rng.random((A, 8)) > 0.1, dtype=torch.float32)
    return nominal, true, measured, mask


def _calib_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch
    import torch.distributed as dist

    from dgc_b200 import calibration, sharded
    from dgc_b200.calibration import ScanSetup

    _calib_standins(calibration)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        nominal, true, measured, mask = _calib_problem()
        v = sharded.view_shard(nominal[0].numel(), world, rank)
        sl = slice(v.start, v.stop)
        pts = calibration.lattice_points((8, 8, 8), device="cpu", n=3)
        res = sharded.calibrate_sharded(
            torch.zeros(1), measured[sl], [g[sl] for g in nominal], ScanSetup(U=8, V=8),
            iterations=60, true_geometry=[g[sl] for g in true], points=pts, mask=mask[sl],
            target_px=0.75)
        out.put((rank, [d.detach().numpy().copy() for d in res.delta],  # by value
                 [(e["reproj_px"], e["angle_err_deg"], e["loss"]) for e in res.history],
                 res.iterations_to_target, res.final_loss))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_sharded_calibration(monkeypatch):
    """Each rank's offsets equal one calibration over all views, restricted to
    its views, bit for bit; the metrics, loss and iteration to target agree."""
    import math

    import torch

    from dgc_b200 import calibration
    from dgc_b200.calibration import ScanSetup

    for name in ("_loss_terms", "_fused_loss", "_loss"):
        monkeypatch.setattr(calibration, name, getattr(calibration, name))
    _calib_standins(calibration)
    nominal, true, measured, mask = _calib_problem()
    pts = calibration.lattice_points((8, 8, 8), device="cpu", n=3)
    whole = calibration.calibrate(torch.zeros(1), measured, nominal, ScanSetup(U=8, V=8),
                                  iterations=60, true_geometry=true, points=pts, mask=mask,
                                  target_px=0.75)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_calib_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = {r: rest for r, *rest in (q.get(timeout=5) for _ in range(2))}
    from dgc_b200.sharded import view_shard

    for r in range(2):
        delta, hist, it_target, final = got[r]
        v = view_shard(13, 2, r)
        for d, w in zip(delta, whole.delta):
            assert torch.equal(torch.from_numpy(d), w.detach()[v.start:v.stop])
        assert it_target == whole.iterations_to_target is not None
        assert math.isclose(final, whole.final_loss, rel_tol=1e-6)
        for (rp, ang, loss), e in zip(hist, whole.history):
            assert math.isclose(rp, e["reproj_px"], rel_tol=1e-9)
            assert math.isclose(ang, e["angle_err_deg"], rel_tol=1e-9)
            assert (math.isnan(loss) and math.isnan(e["loss"])) or \
                math.isclose(loss, e["loss"], rel_tol=1e-5)


def _slab_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import numpy as np
    import torch
    import torch.distributed as dist

    from dgc_b200 import filtering, sharded
    from oracle import oracle as O

    def oracle_fdk(projections, *args, volume_offset=(0.0, 0.0, 0.0), alpha=0.8,
                   offset_preweight=False, **_):
        geometry, (pixel, vshape, voxel) = args[:8], args[8:11]
        g = np.stack([t.numpy() for t in geometry])
        vol = O.reconstruct_fdk(projections.numpy(), g, pixel, vshape, voxel, volume_offset,
                                alpha, offset_preweight)
        return torch.from_numpy(vol).to(projections.dtype)  # float32, as the library's

    filtering.reconstruct_fdk = oracle_fdk  # this rank's process only
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        A, U, V, px, vox, off, alpha = 9, 12, 10, 1.0, 1.0, (0.3, -0.2, 0.45), 0.8
        rng = np.random.default_rng(5)  # the same scan on every rank
        proj = (rng.random((A, U, V)) * 4).astype(np.float32)
        cols = [np.arange(A) * (2 * np.pi / A), np.full(A, 300.0), np.full(A, 180.0),
                np.full(A, (U - 1) / 2 + 0.4), np.full(A, (V - 1) / 2 - 0.3),
                rng.normal(0, 1, A), rng.normal(0, 1, A), rng.normal(0, 1, A)]
        geom = [torch.from_numpy(c.astype(np.float32)) for c in cols]
        res = {}
        for shape in ((7, 6, 8), (1, 5, 5)):
            slab, rows = sharded.reconstruct_fdk_slab(torch.from_numpy(proj), *geom, px, shape,
                                                      vox, volume_offset=off, alpha=alpha,
                                                      offset_preweight=True)
            whole = sharded.gather_slabs(slab, shape[0])
            g32 = np.stack([c.astype(np.float32) for c in cols])  # the ranks' geometry
            truth = O.reconstruct_fdk(proj, g32, px, shape, vox, off, alpha, True)
            res[shape] = ((rows.start, rows.stop), tuple(slab.shape),
                          float(np.abs(slab.numpy() - truth[rows.start:rows.stop]).max(
                              initial=0.0)),
                          float(np.abs(whole.numpy() - truth).max()), float(np.abs(truth).max()))
        out.put((rank, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_slab_sharded_reconstruction():
    """Depth-slab sharding: each rank's slab (the FP64 oracle as its
    reconstruction, on the slab's shifted volume offset, rounded to float32
    as the library's output is) equals the same rows of the whole volume, and
    gathering the slabs gives the whole volume, also when a rank has no
    rows."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_slab_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(q.get(timeout=5) for _ in range(2))
    assert got[0][(7, 6, 8)][:2] == ((0, 4), (4, 6, 8))
    assert got[1][(7, 6, 8)][:2] == ((4, 7), (3, 6, 8))
    assert got[1][(1, 5, 5)][:2] == ((1, 1), (0, 5, 5))
    for r in (0, 1):
        for shape, (_, _, slab_err, whole_err, scale) in got[r].items():
            assert slab_err <= 1e-6 * scale and whole_err <= 1e-6 * scale, (r, shape)
    from dgc_b200.sharded import slab_offset

    # row z of the slab sits where row start + z of the whole volume does
    assert slab_offset((10, 4, 4), 1.0, (0.0, 0.0, 0.5), range(3, 6)) == (0.0, 0.0, 0.0)
    assert slab_offset((8, 4, 4), 0.5, (1.0, 2.0, 3.0), range(0, 8)) == (1.0, 2.0, 3.0)
