"""The module-name drop-in: the reference's own wrappers over this library.

The reference's ``cbct_backprojector`` package finds its native extensions by
module name (``cbct_backprojector/operator.py:20-29``,
``cbct_backprojector/source_only_forward_projector.py:17-27``).  A user who
keeps that package and puts ``diff-geocali_b200`` on ``sys.path`` gets this
library's kernels under those names.  These tests load the reference's
package, unmodified, from its pip installation under ``baseline/_ref`` (or,
in a container holding the reference's checkout, from that checkout) in a
fresh interpreter (``tests/reference_wrappers_check.py``):

* on the CPU, that the lookups resolve to the shims and the calls reach
  ``dgc_b200._ops``;
* on the GPU, the reference's ``check_cuda()`` checks of both operators,
  through its own ``project`` / ``backproject``, at its own tolerances, plus
  config 1.
"""

import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
CHECK = Path(__file__).resolve().parent / "reference_wrappers_check.py"


def reference_package():
    installed = ROOT / "baseline" / "_ref" / "cbct_backprojector"
    if (installed / "__init__.py").is_file():
        return installed
    sys.path.insert(0, str(ROOT))
    from oracle.build_ref import DEFAULT_REFERENCE

    checkout = Path(os.environ.get("DGC_REFERENCE_DIR", DEFAULT_REFERENCE)) / "cbct_backprojector"
    if (checkout / "__init__.py").is_file():
        return checkout
    pytest.skip("the reference's cbct_backprojector package is not installed here")


def run_check(mode):
    env = {k: v for k, v in os.environ.items() if k != "PYTHONPATH"}
    r = subprocess.run([sys.executable, str(CHECK), "--package", str(reference_package()),
                        "--mode", mode], cwd=str(ROOT), env=env, capture_output=True, text=True,
                       timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_reference_wrappers_route_to_this_library():
    out = run_check("routing")
    assert out.count("PASS") == 2


@pytest.mark.gpu
def test_reference_check_cuda_through_the_shims():
    out = run_check("cuda")
    assert out.count("PASS") == 5
