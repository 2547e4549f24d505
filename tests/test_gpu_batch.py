"""Batched forward projection + backward (ProjectionBatch) on the GPU.

Each problem of an uneven batch must give what a plain ``project`` call and
its autograd backward give for the same problem: projections bitwise, the
geometry gradients bitwise where the backward tile matches the single-call
default (8 columns) and to 1e-6 otherwise (the per-CTA FP64 partial sums then
group the rays differently), the volume gradient to 1e-6 (float atomics).
A CUDA-graph replay must reproduce the eager step, and one problem is
checked against the FP64 oracle at the parity bar (rel-L2 1e-5 / 1e-4).
"""

import math

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def make_problems(seed=0):
    from dgc_b200.batch import Problem

    rng = np.random.default_rng(seed)
    specs = [  # (D, H, W), A, U, V, px, vox, step, offset, tiles
        ((24, 20, 16), 12, 40, 36, 1.0, 1.0, 0.5, (0.0, 0.0, 0.0), (8, 8)),
        ((9, 31, 27), 7, 33, 65, 0.9, 0.75, 0.4, (0.3, -0.2, 0.1), (4, 4)),
        ((40, 12, 22), 19, 17, 70, 1.2, 1.5, 0.6, (0.0, 0.0, 0.0), (2, 8)),
        ((16, 16, 16), 1, 300, 3, 0.5, 1.0, 0.5, (0.0, 0.0, -0.4), (8, 4)),
        ((5, 7, 6), 33, 12, 9, 2.0, 2.0, 1.0, (0.0, 0.0, 0.0), (4, 8)),
    ]
    problems = []
    for (D, H, W), A, U, V, px, vox, step, off, tiles in specs:
        vol = torch.tensor(rng.random((D, H, W)), dtype=torch.float32, device="cuda")
        angles = np.arange(A) * 2 * math.pi / A + rng.normal(0, 0.01, A)
        sod = 4.0 * max(D, H, W) * vox
        geom = [angles, sod * 1.5 + rng.normal(0, 1, A), sod + rng.normal(0, 0.5, A),
                (U - 1) / 2 + rng.normal(0, 1, A), (V - 1) / 2 + rng.normal(0, 1, A),
                rng.normal(0, 0.4, A), rng.normal(0, 0.4, A), rng.normal(0, 0.4, A)]
        geom = [torch.tensor(g, dtype=torch.float32, device="cuda") for g in geom]
        problems.append(Problem(vol, geom, px, U, V, step, vox, off, tiles=tiles))
    return problems


def plain(pr):
    from cbct_backprojector import project

    vol = pr.volume.clone().requires_grad_()
    geom = [g.clone().requires_grad_() for g in pr.geometry]
    p = project(vol, *geom, pr.pixel_size, pr.U, pr.V, step_size=pr.step_size,
                voxel_size=pr.voxel_size, off_x=pr.offset[0], off_y=pr.offset[1],
                off_z=pr.offset[2])
    grads = torch.autograd.grad(p, [vol, *geom], grad_outputs=p.detach())
    return p.detach(), grads[0], torch.stack(grads[1:])


def test_batch_matches_plain_calls():
    """Batched launches against per-problem calls."""
    from dgc_b200.batch import ProjectionBatch

    problems = make_problems()
    batch = ProjectionBatch(problems)
    batch.step()
    torch.cuda.synchronize()
    for i, pr in enumerate(problems):
        p, gv, gg = plain(pr)
        assert torch.equal(batch.projections[i], p), i
        assert rel_l2(batch.grad_volumes[i].cpu(), gv.cpu()) < 1e-6, i
        if pr.tiles[1] == 8:
            assert torch.equal(batch.grad_geometry[i], gg), i
        else:
            for k in range(8):
                assert rel_l2(batch.grad_geometry[i][k].cpu(), gg[k].cpu()) < 1e-6, (i, k)


def test_batch_against_reference_and_oracle(oracle, ref_native):
    """Parity bar on one problem: projections and the volume gradient against
    the FP64 oracle, all nine gradients against the reference's CUDA kernels
    (the geometry gradients of a random geometry meet sample-cell boundaries,
    where FP32 and FP64 take different one-sided derivatives; the reference's
    FP32 kernels take the same side)."""
    from dgc_b200.batch import ProjectionBatch

    ref_fp, _ = ref_native
    pr = make_problems(1)[1]  # non power-of-two voxel size, ROI offset, 4-column tiles
    batch = ProjectionBatch([pr])
    batch.step()
    torch.cuda.synchronize()
    geom = [g.cpu().numpy() for g in pr.geometry]
    vol = pr.volume.cpu().numpy()
    truth = oracle.project(vol, geom, pr.pixel_size, pr.U, pr.V, pr.step_size, pr.voxel_size,
                           pr.offset, mode=1)
    assert rel_l2(batch.projections[0].cpu(), truth) < 1e-5
    gv, _ = oracle.project_backward(batch.projections[0].cpu().numpy(), vol, geom, pr.pixel_size,
                                    pr.step_size, pr.voxel_size, pr.offset, mode=1)
    assert rel_l2(batch.grad_volumes[0].cpu(), gv) < 1e-4
    ref_p = ref_fp.forward(pr.volume, *pr.geometry, pr.pixel_size, pr.U, pr.V, pr.step_size,
                           pr.voxel_size, *pr.offset)
    ref = ref_fp.backward(batch.projections[0], pr.volume, *pr.geometry, pr.pixel_size,
                          pr.step_size, pr.voxel_size, True, *pr.offset)
    torch.cuda.synchronize()
    assert rel_l2(batch.projections[0].cpu(), ref_p.cpu()) < 1e-5
    assert rel_l2(batch.grad_volumes[0].cpu(), ref[0].cpu()) < 1e-4
    for k in range(8):
        assert rel_l2(batch.grad_geometry[0][k].cpu(), ref[k + 1].cpu()) < 1e-4, k


def test_graph_replay_and_rebuild():
    from dgc_b200.batch import ProjectionBatch

    problems = make_problems(2)
    batch = ProjectionBatch(problems, grad_volume=False)
    batch.step()
    torch.cuda.synchronize()
    want_p = [p.clone() for p in batch.projections]
    want_g = [g.clone() for g in batch.grad_geometry]
    assert all(g is None for g in batch.grad_volumes)
    batch.capture()
    for p in batch.projections:
        p.zero_()
    for g in batch.grad_geometry:
        g.zero_()
    batch.replay()
    batch.replay()
    torch.cuda.synchronize()
    for i in range(len(problems)):
        assert torch.equal(batch.projections[i], want_p[i]), i
        assert torch.equal(batch.grad_geometry[i], want_g[i]), i
    # a new volume, re-packed by the backward itself
    problems[0].volume.mul_(2.0)
    batch.backward(rebuild_quads=True)
    torch.cuda.synchronize()
    assert torch.equal(batch.grad_geometry[0], 2.0 * want_g[0])


def test_autotuner_on_gpu(tmp_path):
    from dgc_b200.autotune import Autotuner

    problems = make_problems(3)[:2]
    tuner = Autotuner(cache_path=tmp_path / "tiles.json")
    tiles = tuner.choose(problems)
    assert all(t[0] in (8, 4, 2) and t[1] in (8, 4) for t in tiles)
    assert (tmp_path / "tiles.json").exists() and len(tuner.measured) == 2
    again = Autotuner(cache_path=tmp_path / "tiles.json", measure=lambda *a: 1 / 0)
    assert again.choose(problems) == tiles
