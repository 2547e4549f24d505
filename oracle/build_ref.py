"""Compile the reference's own CUDA operators into ``oracle/_ref/`` (test infrastructure only).

The two reference sources (``csrc/src_cbct_forwardprojector_cuda.cu`` and
``csrc/src_cbct_backprojector_cuda.cu``) are compiled where they lie, unmodified,
with ``torch.utils.cpp_extension.load``; the reference's own ``setup.py`` is not
run.  Each module is built under a distinct name (``ref_`` prefix, passed as
``TORCH_EXTENSION_NAME``) so that the reference kernels and this project's
drop-in modules can be imported in one process and compared on the same
inputs.  Output goes only to ``oracle/_ref/`` (git-ignored; it travels to GPU
machines with the working tree).  Nothing in the product imports this.

Usage: ``python oracle/build_ref.py [--reference DIR]``.  The reference's
checkout is ``--reference``, else the environment variable
``DGC_REFERENCE_DIR``, else this recipe's default location
``/root/reference`` (where the development container mounts it read-only).
Exits 0 with a message when the sources are absent.
"""

import argparse
import os
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
DEFAULT_REFERENCE = "/root/reference"
OUT = HERE / "_ref"

MODULES = {
    "ref_src_cbct_forwardprojector_cuda": "csrc/src_cbct_forwardprojector_cuda.cu",
    "ref_src_cbct_backprojector_cuda": "csrc/src_cbct_backprojector_cuda.cu",
}


def main(argv=None):
    parser = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    parser.add_argument("--reference", default=os.environ.get("DGC_REFERENCE_DIR", DEFAULT_REFERENCE))
    args = parser.parse_args(argv)
    ref = Path(args.reference)
    if not all((ref / src).is_file() for src in MODULES.values()):
        print(f"reference sources not found under {ref}; oracle/_ref not rebuilt")
        return 0
    # The reference is built for plain sm_100, as its own docs describe
    # (TORCH_CUDA_ARCH_LIST selects the -gencode flags of cpp_extension).
    os.environ["TORCH_CUDA_ARCH_LIST"] = "10.0"
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils.cpp_extension import load

    OUT.mkdir(parents=True, exist_ok=True)
    for name, src in MODULES.items():
        build_dir = OUT / ("build_" + name)
        build_dir.mkdir(parents=True, exist_ok=True)
        load(
            name=name,
            sources=[str(ref / src)],
            extra_cflags=["-O3"],
            extra_cuda_cflags=["-O3"],
            build_directory=str(build_dir),
            verbose=False,
        )
        built = build_dir / f"{name}.so"
        shutil.copy2(built, OUT / f"{name}.so")
        print(f"built {OUT / (name + '.so')}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
