"""Run the reference's own Python wrappers on this library's native-module shims.

The reference's ``cbct_backprojector`` package (TomSHINING/diff-geoCali,
unmodified: its pip installation, or its checkout) imports its native
extensions by module name (``cbct_backprojector/operator.py:20-29``,
``cbct_backprojector/source_only_forward_projector.py:17-27``).  This script
loads that package under its own name, puts only this repository's shim
directory (``diff-geocali_b200``: ``src_cbct_forwardprojector_cuda``,
``src_cbct_backprojector_cuda``) on ``sys.path``, and then

* ``--mode routing`` (no GPU needed): checks that the reference's
  ``_native()`` lookups return the shims, that the shims' functions are
  ``dgc_b200._ops``', that this repository's own ``cbct_backprojector`` was
  never imported, and that a call through the reference's autograd classes
  reaches ``dgc_b200._ops`` (whose argument checks reject CPU tensors);
* ``--mode cuda``: does what the reference's ``check_cuda()`` functions do
  (``examples/check_operator.py:180-205``,
  ``examples/check_forward_operator.py:197-226``) through the reference's
  ``project`` / ``backproject`` on their own test cases, with non-contiguous
  inputs and the same tolerances, against the FP64 CPU results stored as
  golden fixtures (``tests/golden/*_check_case.npz``, written by
  ``tests/golden/make_golden.py`` from those very check scripts), plus the
  config-1 operator case.

Test infrastructure, run by ``tests/test_dropin_reference_wrappers.py`` in a
fresh interpreter so that the reference's package never shares a process with
this repository's package of the same name.  Prints ``PASS`` lines; exits
non-zero on the first failure.
"""

import argparse
import importlib
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
SHIMS = ROOT / "diff-geocali_b200"
GOLDEN = ROOT / "tests" / "golden"
GEOM = ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")


def load_reference_package(pkg_dir: Path):
    sys.path.insert(0, str(SHIMS))
    spec = importlib.util.spec_from_file_location(
        "cbct_backprojector", pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    module = importlib.util.module_from_spec(spec)
    sys.modules["cbct_backprojector"] = module
    spec.loader.exec_module(module)
    for name in ("operator", "source_only_forward_projector", "filtering"):
        sub = importlib.import_module(f"cbct_backprojector.{name}")
        if Path(sub.__file__).resolve().parent != pkg_dir.resolve():
            raise AssertionError(f"cbct_backprojector.{name} is not the reference's module")
    return module


def check_routing(ref):
    import torch

    import dgc_b200._ops as ops

    fp_native = ref.source_only_forward_projector._native()
    bp_native = ref.operator._native()
    for native, stem, fwd, bwd in ((fp_native, "src_cbct_forwardprojector_cuda", ops.fp_forward,
                                    ops.fp_backward),
                                   (bp_native, "src_cbct_backprojector_cuda", ops.bp_forward,
                                    ops.bp_backward)):
        if Path(native.__file__).resolve() != (SHIMS / f"{stem}.py").resolve():
            raise AssertionError(f"{stem} resolved to {native.__file__}")
        if native.forward is not fwd or native.backward is not bwd:
            raise AssertionError(f"{stem} does not expose dgc_b200._ops")
    if sys.modules["cbct_backprojector"] is not ref:
        raise AssertionError("this repository's cbct_backprojector replaced the reference's")
    print("routing: the reference's _native() lookups return this library's shims: PASS")

    A, U, V = 2, 4, 3
    proj = torch.zeros((A, U, V))
    geom = [torch.zeros(A) for _ in GEOM]
    try:
        ref.backproject(proj, *geom, 1.0, (2, 2, 2), 1.0)
    except ValueError as error:
        if "CUDA float32" not in str(error):
            raise
    else:
        raise AssertionError("the reference's backproject accepted CPU tensors")
    try:
        ref.operator._Backproject.apply(proj, *geom, 1.0, (2, 2, 2), 1.0, (0.0, 0.0, 0.0))
    except RuntimeError as error:
        if "CUDA" not in str(error):
            raise
    else:
        raise AssertionError("the native call accepted CPU tensors")
    try:
        ref.source_only_forward_projector.DifferentiableSourceOnlyForwardProjector.apply(
            torch.zeros((2, 2, 2)), *[torch.zeros(1) for _ in GEOM], 1.0, 2, 2, 0.5, 1.0)
    except ValueError as error:  # the reference's own validation runs first
        if "CUDA float32" not in str(error):
            raise
    print("routing: calls through the reference's autograd classes reach dgc_b200._ops: PASS")


def noncontig(t):
    out = t.transpose(-1, -2).contiguous().transpose(-1, -2)
    assert not out.is_contiguous()
    return out


def check_cuda(ref):
    import torch

    dev = torch.device("cuda")

    def cuda32(x):
        return torch.as_tensor(np.asarray(x), dtype=torch.float32, device=dev)

    # examples/check_operator.py check_cuda(): backprojection and nine gradients
    d = np.load(GOLDEN / "bp_check_case.npz")
    params = [noncontig(cuda32(d["in_data"])).requires_grad_()]
    params += [cuda32(d["in_" + n]).requires_grad_() for n in GEOM]
    upstream = noncontig(cuda32(d["upstream"]))
    shape = tuple(int(x) for x in d["volume_shape"])
    out = ref.backproject(*params, float(d["pixel_size"]), shape, float(d["voxel_size"]),
                          volume_offset=tuple(float(x) for x in d["volume_offset"]))
    grads = torch.autograd.grad(out, params, grad_outputs=upstream)
    torch.cuda.synchronize()
    torch.testing.assert_close(out.detach().double().cpu(), torch.from_numpy(d["output"]),
                               rtol=2e-5, atol=2e-5)
    for name, g in zip(("data",) + GEOM, grads):
        torch.testing.assert_close(g.double().cpu(), torch.from_numpy(d["grad_" + name]),
                                   rtol=3e-4, atol=3e-5, msg=name)
    print("cuda: reference backproject wrapper, check_operator case, value and nine gradients: PASS")

    # examples/check_forward_operator.py check_cuda(): projection and nine gradients
    d = np.load(GOLDEN / "fp_check_case.npz")
    U, V = (int(x) for x in d["detector"])
    off = [float(x) for x in d["volume_offset"]]
    params = [noncontig(cuda32(d["in_data"])).requires_grad_()]
    params += [cuda32(d["in_" + n]).requires_grad_() for n in GEOM]
    upstream = noncontig(cuda32(d["upstream"]))

    def run(values):
        return ref.project(*values, float(d["pixel_size"]), U, V, step_size=float(d["step_size"]),
                           voxel_size=float(d["voxel_size"]), off_x=off[0], off_y=off[1],
                           off_z=off[2])

    out = run(params)
    grads = torch.autograd.grad(out, params, grad_outputs=upstream)
    torch.cuda.synchronize()
    torch.testing.assert_close(out.detach().double().cpu(), torch.from_numpy(d["output"]),
                               rtol=5e-5, atol=5e-5)
    for name, g in zip(("data",) + GEOM, grads):
        if not torch.isfinite(g).all().item():
            raise AssertionError(f"{name} gradient is non-finite")
        torch.testing.assert_close(g.double().cpu(), torch.from_numpy(d["grad_" + name]),
                                   rtol=1e-3, atol=1e-4, msg=name)
    with torch.no_grad():
        other = params[0].flip(-1)
        combined = run([1.3 * params[0] - 0.4 * other, *params[1:]])
        torch.testing.assert_close(combined, 1.3 * out.detach() - 0.4 * run([other, *params[1:]]),
                                   rtol=5e-5, atol=5e-5)
    print("cuda: reference project wrapper, check_forward_operator case, value, nine gradients "
          "and linearity: PASS")

    # config 1 (16x20x24 volume, 24 views, 48x40 detector): values and volume gradient
    d = np.load(GOLDEN / "fp_config1.npz")
    U, V = (int(x) for x in d["detector"])
    vol = cuda32(d["in_data"]).requires_grad_()
    geom = [cuda32(d["in_" + n]) for n in GEOM]
    out = ref.project(vol, *geom, 1.0, U, V, step_size=0.5, voxel_size=1.0)
    loss = (out.double() ** 2).mean()
    (gvol,) = torch.autograd.grad(loss, [vol])
    torch.cuda.synchronize()

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    e_out = rel(out.detach().double().cpu().numpy(), d["output"])
    e_gv = rel(gvol.double().cpu().numpy(), d["grad_data"])
    if not (e_out < 1e-5 and e_gv < 1e-4):
        raise AssertionError(f"config 1 through the reference wrapper: rel-L2 {e_out:.2e}, "
                             f"volume gradient {e_gv:.2e}")
    print(f"cuda: reference project wrapper, config 1: rel-L2 {e_out:.2e}, volume gradient "
          f"{e_gv:.2e}: PASS")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--package", required=True, type=Path,
                    help="the reference's cbct_backprojector package directory")
    ap.add_argument("--mode", choices=("routing", "cuda"), required=True)
    args = ap.parse_args(argv)
    ref = load_reference_package(args.package)
    check_routing(ref)
    if args.mode == "cuda":
        check_cuda(ref)
    if "dgc_b200" not in sys.modules:
        raise AssertionError("dgc_b200 was never loaded")
    return 0


if __name__ == "__main__":
    sys.exit(main())
