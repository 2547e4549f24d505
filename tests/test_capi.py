"""The C ABI without a GPU: the library loads, exports every symbol that
include/dgc.h declares, answers workspace queries, computes filter taps on the
host and rejects invalid arguments with the reference's messages (argument
checks run before any CUDA call)."""

import ctypes
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    text = (ROOT / "include" / "dgc.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dgc_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from dgc_b200 import _native

    return _native.lib()


def test_exports_every_declared_symbol(lib):
    from dgc_b200 import _native

    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _native.SIGNATURES, f"{name} has no ctypes signature"
    assert lib.dgc_abi_version() == 1


def test_workspace_queries(lib):
    a = lib.dgc_project_workspace_bytes(256, 256, 256, 360, 384, 384)
    assert a == 16 * 258 * 257 * 257 + (-(16 * 258 * 257 * 257) % 256) + 256  # quads + status word
    assert lib.dgc_project_workspace_bytes(0, 1, 1, 1, 1, 1) == 0
    b0 = lib.dgc_project_backward_workspace_bytes(64, 64, 64, 90, 128, 128, 0)
    b1 = lib.dgc_project_backward_workspace_bytes(64, 64, 64, 90, 128, 128, 1)
    assert b1 > b0 > 0
    assert lib.dgc_backproject_workspace_bytes(360, 384, 384, 256, 256, 256) >= 16 * 360 * 383 * 383
    assert lib.dgc_reconstruct_fdk_workspace_bytes(360, 384, 384, 256, 256, 256) > \
        lib.dgc_backproject_workspace_bytes(360, 384, 384, 256, 256, 256)
    assert lib.dgc_backproject_workspace_bytes(1, 1, 5, 1, 1, 1) == 0


def test_filter_taps_on_host(lib, oracle):
    for U, px, alpha in [(9, 0.9, 0.8), (384, 1.0, 0.8), (768, 1.0, 0.8), (17, 0.75, 1.0)]:
        buf = (ctypes.c_double * U)()
        assert lib.dgc_fdk_filter_taps(U, px, alpha, buf) == 0
        np.testing.assert_allclose(np.array(buf), oracle.fdk_taps(U, px, alpha), rtol=1e-9,
                                   atol=1e-15)
    buf = (ctypes.c_double * 4)()
    assert lib.dgc_fdk_filter_taps(4, 1.0, 1.5, buf) == 1
    assert b"alpha" in lib.dgc_last_error()


def _geom_ptrs():
    return [ctypes.c_void_p(16)] * 8  # never dereferenced: checks fail first


def test_invalid_arguments_return_status(lib):
    g = _geom_ptrs()
    # forward projector (fp.cu:585-611)
    rc = lib.dgc_project(None, 0, 4, 4, *g, 3, 1.0, 4, 4, 0.5, 1.0, 0.0, 0.0, 0.0, None, None, 0,
                         None)
    assert rc == 1 and lib.dgc_last_error() == b"every volume dimension must be positive"
    rc = lib.dgc_project(None, 4, 4, 4, *g, 3, 1.0, 0, 4, 0.5, 1.0, 0.0, 0.0, 0.0, None, None, 0,
                         None)
    assert rc == 1 and lib.dgc_last_error() == b"U and V must be positive"
    rc = lib.dgc_project(None, 4, 4, 4, *g, 3, 1.0, 4, 4, 0.0, 1.0, 0.0, 0.0, 0.0, None, None, 0,
                         None)
    assert rc == 1 and b"must be positive" in lib.dgc_last_error()
    rc = lib.dgc_project(None, 4, 4, 4, *g, 0, 1.0, 4, 4, 0.5, 1.0, 0.0, 0.0, 0.0, None, None, 0,
                         None)
    assert rc == 1 and lib.dgc_last_error() == b"angles must contain at least one view"
    # workspace too small is reported before any launch
    rc = lib.dgc_project(ctypes.c_void_p(16), 4, 4, 4, *g, 3, 1.0, 4, 4, 0.5, 1.0, 0.0, 0.0, 0.0,
                         ctypes.c_void_p(16), None, 0, None)
    assert rc == 3 and b"workspace too small" in lib.dgc_last_error()
    # backprojector (bp.cu:298-383)
    rc = lib.dgc_backproject(None, 2, 1, 4, *g, 1.0, 4, 4, 4, 1.0, 0.0, 0.0, 0.0, None, None, 0,
                             None)
    assert rc == 1 and b"U,V >= 2" in lib.dgc_last_error()
    rc = lib.dgc_backproject(None, 2, 4, 4, *g, 1.0, 8 * 65535 + 1, 1, 1, 1.0, 0.0, 0.0, 0.0, None,
                             None, 0, None)
    assert rc == 1 and b"grid limits" in lib.dgc_last_error()
    rc = lib.dgc_backproject(None, 2, 4, 4, *g, 1.0, 4, 4, 4, 1.0, float("nan"), 0.0, 0.0, None,
                             None, 0, None)
    assert rc == 1 and lib.dgc_last_error() == b"sizes and ROI offsets must be finite"
    rc = lib.dgc_fdk_filter(None, 2, 4, 4, -1.0, None, None, 0.8, None, None, 0, None)
    assert rc == 1 and b"pixel_size" in lib.dgc_last_error()


def test_preprocess_argument_checks(lib):
    p = ctypes.c_void_p(256)
    assert lib.dgc_preprocess(None, None, None, 1, 4, 4, 1, 1e-6, p, None) == 1
    assert b"non-null" in lib.dgc_last_error()
    assert lib.dgc_preprocess(p, None, None, 1, 0, 4, 1, 1e-6, ctypes.c_void_p(512), None) == 1
    assert lib.dgc_preprocess(p, None, None, 1, 4, 4, 1, 0.0, ctypes.c_void_p(512), None) == 1
    assert b"min_ratio" in lib.dgc_last_error()
    assert lib.dgc_preprocess(p, None, None, 1, 4, 4, 1, 1e-6, p, None) == 1
    assert b"alias" in lib.dgc_last_error()


def test_sharding_entries_check_arguments(lib):
    """dgc_reconstruct_fdk_partial and dgc_clamp_volume reject bad arguments
    before any CUDA call; an empty clamp is a no-op."""
    g = _geom_ptrs()
    for scale in (0.0, -1.0, float("inf")):
        rc = lib.dgc_reconstruct_fdk_partial(None, 4, 8, 8, *g, 1.0, 4, 4, 4, 1.0, 0.0, 0.0, 0.0,
                                             0.8, None, scale, None, None, 0, None)
        assert rc == 1 and b"angle_scale" in lib.dgc_last_error()
    assert lib.dgc_clamp_volume(None, -1, None) == 1
    assert b"non-negative" in lib.dgc_last_error()
    assert lib.dgc_clamp_volume(None, 5, None) == 1
    assert lib.dgc_clamp_volume(None, 0, None) == 0


def test_frame_entries_check_arguments(lib):
    """The preweight-frame entries reject bad arguments before any CUDA call:
    a frame gradient without its frame array, a bad alpha, a bad angular
    factor, a short scan of one view; the backward's scratch holds four FP64
    sums per (view, filter tile)."""
    g = _geom_ptrs()
    p = ctypes.c_void_p(256)
    for k in range(3):  # grad_frame_dist / _u / _v without frame_dist / _u / _v
        grads = [None, None, None]
        grads[k] = p
        frames = [p, p, p]
        frames[k] = None
        rc = lib.dgc_fdk_filter_backward_ex(p, p, p, 2, 8, 8, 1.0, p, p, *frames, 0.8, None, None,
                                            None, *grads, None, 0, None)
        assert rc == 1 and b"frame gradient" in lib.dgc_last_error(), k
    rc = lib.dgc_fdk_filter_ex(p, 2, 8, 8, 1.0, p, p, None, None, None, 1.5, p, None, 0, None)
    assert rc == 1 and b"alpha" in lib.dgc_last_error()
    for scale in (0.0, float("nan")):
        rc = lib.dgc_reconstruct_fdk_ex(None, 4, 8, 8, *g, 1.0, 4, 4, 4, 1.0, 0.0, 0.0, 0.0, 0.8,
                                        None, None, None, None, scale, 1, None, None, 0, None)
        assert rc == 1 and b"angle_scale" in lib.dgc_last_error()
    assert lib.dgc_parker_weights_ex(p, p, None, None, 1, 8, 1.0, p, None) == 1
    assert b"A >= 2" in lib.dgc_last_error()
    A, U, V = 360, 384, 384
    tiles = -(-V // 128) * -(-U // 128)
    assert lib.dgc_fdk_filter_backward_workspace_bytes(A, U, V) >= 4 * 8 * A * tiles + 4 * U


def test_header_is_c99_and_links_from_c(tmp_path):
    """include/dgc.h compiles as strict C99 and a C program links against
    libdgc.so and calls it (host-only entry points, no GPU)."""
    import shutil
    import subprocess
    from pathlib import Path

    from dgc_b200 import _native

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    root = Path(__file__).resolve().parents[1]
    libdir = Path(_native.LIB_PATH).parent
    src = tmp_path / "use_dgc.c"
    src.write_text(
        '#include "dgc.h"\n'
        "#include <stdio.h>\n"
        "int main(void) {\n"
        "    double taps[16];\n"
        "    if (dgc_abi_version() != DGC_ABI_VERSION) return 1;\n"
        "    if (dgc_fdk_filter_taps(16, 1.0, 0.8, taps) != DGC_OK) return 2;\n"
        "    if (dgc_fdk_filter_taps(16, 1.0, 2.0, taps) != DGC_ERR_INVALID_ARGUMENT) return 3;\n"
        '    printf("%s\\n", dgc_last_error());\n'
        "    return taps[0] > 0.0 ? 0 : 4;\n"
        "}\n")
    exe = tmp_path / "use_dgc"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                    f"-I{root / 'include'}", str(src), f"-L{libdir}", "-ldgc",
                    f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0, (run.returncode, run.stdout, run.stderr)
    assert "alpha" in run.stdout
