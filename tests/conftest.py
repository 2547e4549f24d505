"""Shared fixtures: import paths, the ``gpu`` marker, golden fixtures, the oracle."""

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "diff-geocali_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"
REF_DIR = ROOT / "oracle" / "_ref"

for p in (str(PKG), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GEOM_NAMES = ("angles", "sid", "sod", "det_u0", "det_v0", "src_x", "src_y", "src_z")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_cuda = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_cuda = False
    if has_cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this process")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.build()
    return o


def load_golden(name):
    with np.load(GOLDEN / name) as d:
        return {k: d[k] for k in d.files}


@pytest.fixture(scope="session")
def golden():
    return load_golden


def golden_geometry(d, dtype=np.float64):
    return [np.asarray(d["in_" + n], dtype=dtype) for n in GEOM_NAMES]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


@pytest.fixture(scope="session")
def ref_native():
    """The reference's own CUDA operators built by ``oracle/build_ref.py`` (or skip)."""
    fp = REF_DIR / "ref_src_cbct_forwardprojector_cuda.so"
    bp = REF_DIR / "ref_src_cbct_backprojector_cuda.so"
    if not (fp.exists() and bp.exists()):
        pytest.skip("reference CUDA build (oracle/_ref) not present")
    import torch  # noqa: F401  (the extensions link against torch)

    if str(REF_DIR) not in sys.path:
        sys.path.insert(0, str(REF_DIR))
    return (importlib.import_module("ref_src_cbct_forwardprojector_cuda"),
            importlib.import_module("ref_src_cbct_backprojector_cuda"))
