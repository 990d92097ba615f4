"""Build recipe of the in-tree CUDA library ``jno_b200/libfemk.so`` (sm_100a only).

``python -m jno_b200._build`` (or ``__graft_entry__.build()``) compiles every ``csrc/*.cu`` with
nvcc for ``-gencode arch=compute_100a,code=sm_100a`` and links one shared library next to this
file; ``--bounds`` builds ``libfemk_bounds.so`` from the same sources with ``-DFEMK_BOUNDS_CHECK``. The CUDA runtime is linked statically, so the library loads without a CUDA toolkit on the
library path; streams created by PyTorch are plain driver streams and are accepted as ``void*``.
"""

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libfemk.so")
# the same sources with -DFEMK_BOUNDS_CHECK: every checked index returns FEMK_EBOUNDS instead of faulting
LIB_BOUNDS = os.path.join(HERE, "libfemk_bounds.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr"]


def _nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the B200 kernels cannot be built")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def build(verbose=False, extra=(), bounds=False):
    """Compile every source into LIB (or, with ``bounds``, the bounds-checked LIB_BOUNDS)."""
    nvcc = _nvcc()
    objdir = os.path.join(ROOT, "_build", "bounds") if bounds else os.path.join(ROOT, "_build")
    extra = tuple(extra) + (("-DFEMK_BOUNDS_CHECK",) if bounds else ())
    lib = LIB_BOUNDS if bounds else LIB
    os.makedirs(objdir, exist_ok=True)
    objs = []
    inc = ["-I", os.path.join(ROOT, "include")]
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
        deps = [src] + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "femk.h")]
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in deps):
            cmd = [nvcc, *ARCH, *FLAGS, *inc, *extra, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = lib + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, bounds="--bounds" in sys.argv))
