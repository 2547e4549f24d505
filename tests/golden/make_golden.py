"""Generate the golden fixtures in ``tests/golden/`` from the reference's own CPU code.

Run in a container where the reference project (TomSHINING/diff-geoCali) is
checked out::

    python tests/golden/make_golden.py [--reference DIR]

The checkout is ``--reference``, else ``DGC_REFERENCE_DIR``, else this
script's default location ``/root/reference``.

It imports, unmodified and read-only, the reference's FP64 CPU oracles

* ``examples/check_operator.py``         (``make_case``, ``reference_backproject``,
  ``scalar_loss``) for the backprojector,
* ``examples/check_forward_operator.py`` (``make_case``, ``reference_project``)
  for the forward projector,
* ``cbct_backprojector/filtering.py``    (``fdk_filter`` on CPU float32, and
  its autograd gradients),

evaluates them on the reference's own test cases and on the config-1 operator
case (16x20x24 volume, 24 views, 48x40 detector), and stores inputs, outputs
and autograd gradients as compressed ``.npz`` files.  The fixtures are what the
CPU test-suite pins the C oracle against; this script is not needed at test
time and nothing imports it.
"""

import argparse
import os
import math
import sys
import time
from pathlib import Path

import numpy as np
import torch

HERE = Path(__file__).resolve().parent
NAMES9 = ("data", "angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")


def _np(t):
    return t.detach().cpu().numpy()


def bp_check_case(cop):
    params, upstream = cop.make_case(torch.float64)
    out = cop.reference_backproject(params)
    loss = (out * upstream).sum()
    grads = torch.autograd.grad(loss, params)
    scalar = cop.scalar_loss(params, upstream)
    d = {
        "pixel_size": cop.PIXEL_SIZE, "voxel_size": cop.VOXEL_SIZE,
        "volume_shape": np.array(cop.VOLUME_SHAPE), "volume_offset": np.array(cop.VOLUME_OFFSET),
        "upstream": _np(upstream.contiguous()), "output": _np(out), "scalar_loss": scalar,
    }
    for n, p, g in zip(NAMES9, params, grads):
        d["in_" + n] = _np(p.contiguous())
        d["grad_" + n] = _np(g)
    np.savez_compressed(HERE / "bp_check_case.npz", **d)


def fp_check_case(fop):
    params, upstream = fop.make_case(torch.float64)
    out, traces = fop.reference_project(params)
    grads = torch.autograd.grad((out * upstream).sum(), params)
    d = {
        "pixel_size": fop.PIXEL_SIZE, "voxel_size": fop.VOXEL_SIZE, "step_size": fop.STEP_SIZE,
        "detector": np.array([fop.DETECTOR_U, fop.DETECTOR_V]),
        "volume_offset": np.array(fop.VOLUME_OFFSET),
        "upstream": _np(upstream.contiguous()), "output": _np(out),
        "counts": np.array([t[1] for t in traces]).reshape(out.shape),
        "entry_axis": np.array([t[0] for t in traces]).reshape(out.shape),
    }
    for n, p, g in zip(NAMES9, params, grads):
        d["in_" + n] = _np(p.contiguous())
        d["grad_" + n] = _np(g)
    np.savez_compressed(HERE / "fp_check_case.npz", **d)


def config1_geometry(dtype=torch.float64):
    A, U, V = 24, 48, 40
    angles = torch.arange(A, dtype=torch.float32) * (2 * math.pi / A)
    full = lambda x: torch.full((A,), x, dtype=torch.float32)  # noqa: E731
    # detector_centers(0, 0, U, V, 1.0) = ((U-1)/2, (V-1)/2)
    geometry = [angles, full(180.0), full(120.0), full((U - 1) / 2.0), full((V - 1) / 2.0),
                full(0.0), full(0.0), full(0.0)]
    return [g.to(dtype) for g in geometry], (A, U, V)


def fp_config1(fop):
    torch.manual_seed(0)
    volume32 = torch.rand(16, 20, 24, dtype=torch.float32)
    geometry, (A, U, V) = config1_geometry()
    fop.DETECTOR_U, fop.DETECTOR_V = U, V
    fop.PIXEL_SIZE, fop.VOXEL_SIZE, fop.STEP_SIZE = 1.0, 1.0, 0.5
    fop.VOLUME_OFFSET = (0.0, 0.0, 0.0)
    params = [volume32.to(torch.float64).requires_grad_()] + [g.requires_grad_() for g in geometry]
    t0 = time.time()
    out, traces = fop.reference_project(params)
    loss = out.square().mean()
    grads = torch.autograd.grad(loss, params)
    print(f"config-1 forward oracle: {time.time() - t0:.1f}s")
    d = {
        "pixel_size": 1.0, "voxel_size": 1.0, "step_size": 0.5, "detector": np.array([U, V]),
        "volume_offset": np.zeros(3), "output": _np(out),
        "counts": np.array([t[1] for t in traces]).reshape(out.shape),
    }
    d["in_data"] = _np(volume32)
    for n, p, g in zip(NAMES9, params, grads):
        if n != "data":
            d["in_" + n] = _np(p).astype(np.float32)
        d["grad_" + n] = _np(g)
    np.savez_compressed(HERE / "fp_config1.npz", **d)
    return out.detach()


def bp_config1(cop, projections):
    geometry, (A, U, V) = config1_geometry()
    cop.PIXEL_SIZE, cop.VOXEL_SIZE = 1.0, 1.0
    cop.VOLUME_SHAPE, cop.VOLUME_OFFSET = (16, 20, 24), (0.0, 0.0, 0.0)
    proj32 = projections.to(torch.float32)
    params = [proj32.to(torch.float64).requires_grad_()] + [g.requires_grad_() for g in geometry]
    out = cop.reference_backproject(params)
    upstream = torch.linspace(-0.7, 1.3, out.numel(), dtype=torch.float64).reshape(out.shape)
    grads = torch.autograd.grad((out * upstream).sum(), params)
    d = {"pixel_size": 1.0, "voxel_size": 1.0, "volume_shape": np.array(cop.VOLUME_SHAPE),
         "volume_offset": np.zeros(3), "upstream": _np(upstream), "output": _np(out),
         "in_data": _np(proj32)}
    for n, p, g in zip(NAMES9, params, grads):
        if n != "data":
            d["in_" + n] = _np(p).astype(np.float32)
        d["grad_" + n] = _np(g)
    np.savez_compressed(HERE / "bp_config1.npz", **d)


def fdk_cases(filtering):
    gen = torch.Generator().manual_seed(7)
    cases = [
        dict(shape=(3, 9, 7), pixel=0.9, sod=[12.0, 12.4, 11.8], sid=[18.0, 18.7, 17.8], alpha=0.8),
        dict(shape=(4, 48, 40), pixel=1.0, sod=120.0, sid=180.0, alpha=0.8),
        dict(shape=(2, 17, 5), pixel=0.75, sod=[600.0, 610.0], sid=[1000.0, 990.0], alpha=1.0),
        dict(shape=(2, 1, 3), pixel=1.0, sod=600.0, sid=1000.0, alpha=0.5),
    ]
    d = {}
    for i, c in enumerate(cases):
        p = torch.rand(c["shape"], generator=gen, dtype=torch.float32) * 3.0
        out = filtering.fdk_filter(p, c["pixel"], c["sod"], c["sid"], c["alpha"])
        d[f"c{i}_in"] = _np(p)
        d[f"c{i}_out"] = _np(out)
        d[f"c{i}_pixel"] = c["pixel"]
        d[f"c{i}_alpha"] = c["alpha"]
        d[f"c{i}_sod"] = np.broadcast_to(np.asarray(c["sod"], np.float64), (c["shape"][0],)).copy()
        d[f"c{i}_sid"] = np.broadcast_to(np.asarray(c["sid"], np.float64), (c["shape"][0],)).copy()
    d["n_cases"] = len(cases)
    np.savez_compressed(HERE / "fdk_filter.npz", **d)


def fdk_grad_cases(filtering):
    """Autograd gradients of the reference's torch fdk_filter for the
    projections and per-view sod / sid tensors, under a random upstream
    gradient."""
    gen = torch.Generator().manual_seed(11)
    cases = [
        dict(shape=(3, 9, 7), pixel=0.9, sod=[12.0, 12.4, 11.8], sid=[18.0, 18.7, 17.8], alpha=0.8),
        dict(shape=(2, 40, 33), pixel=1.0, sod=[120.0, 121.0], sid=[180.0, 178.5], alpha=0.8),
        dict(shape=(2, 17, 5), pixel=0.75, sod=[600.0, 610.0], sid=[1000.0, 990.0], alpha=1.0),
    ]
    d = {}
    for i, c in enumerate(cases):
        p = (torch.rand(c["shape"], generator=gen, dtype=torch.float32) * 3.0).requires_grad_()
        sod = torch.tensor(c["sod"], dtype=torch.float32, requires_grad=True)
        sid = torch.tensor(c["sid"], dtype=torch.float32, requires_grad=True)
        g = torch.rand(c["shape"], generator=gen, dtype=torch.float32) - 0.5
        out = filtering.fdk_filter(p, c["pixel"], sod, sid, c["alpha"])
        gp, gsod, gsid = torch.autograd.grad(out, [p, sod, sid], grad_outputs=g)
        d[f"c{i}_in"] = _np(p)
        d[f"c{i}_up"] = _np(g)
        d[f"c{i}_out"] = _np(out)
        d[f"c{i}_pixel"] = c["pixel"]
        d[f"c{i}_alpha"] = c["alpha"]
        d[f"c{i}_sod"] = _np(sod)
        d[f"c{i}_sid"] = _np(sid)
        d[f"c{i}_grad_in"] = _np(gp)
        d[f"c{i}_grad_sod"] = _np(gsod)
        d[f"c{i}_grad_sid"] = _np(gsid)
    d["n_cases"] = len(cases)
    np.savez_compressed(HERE / "fdk_filter_grad.npz", **d)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=os.environ.get("DGC_REFERENCE_DIR", "/root/reference"))
    ap.add_argument("--only", nargs="*", default=None,
                    help="fixture groups to write (bp_check fp_check fdk fdk_grad config1)")
    args = ap.parse_args(argv)
    sys.path.insert(0, args.reference)
    torch.set_num_threads(max(1, torch.get_num_threads()))
    from examples import check_forward_operator as fop
    from examples import check_operator as cop
    from cbct_backprojector import filtering

    want = set(args.only or ("bp_check", "fp_check", "fdk", "fdk_grad", "config1"))
    if "bp_check" in want:
        bp_check_case(cop)
    if "fp_check" in want:
        fp_check_case(fop)
    if "fdk" in want:
        fdk_cases(filtering)
    if "fdk_grad" in want:
        fdk_grad_cases(filtering)
    if "config1" in want:
        proj = fp_config1(fop)
        bp_config1(cop, proj)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
