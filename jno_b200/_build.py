"""Build recipe of the in-tree CUDA library ``jno_b200/libfemk.so`` (sm_100a only).

``python -m jno_b200._build`` (or ``__graft_entry__.build()``) compiles every ``csrc/*.cu`` with
nvcc for ``-gencode arch=compute_100a,code=sm_100a`` and links one shared library next to this
file; ``--bounds`` builds ``libfemk_bounds.so`` from the same sources with ``-DFEMK_BOUNDS_CHECK``. The CUDA runtime is linked statically, so the library loads without a CUDA toolkit on the
library path; streams created by PyTorch are plain driver streams and are accepted as ``void*``.
"""

import fcntl
import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

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
    """Compile every source into LIB (or, with ``bounds``, the bounds-checked LIB_BOUNDS).

    Sources compile in parallel; an object is rebuilt when it is older than its source, any
    ``csrc/*.cuh`` or ``include/femk.h``. A lock on the object directory keeps two builds from
    interleaving (an object written by an older build after a newer one would look up to date)."""
    nvcc = _nvcc()
    objdir = os.path.join(ROOT, "_build", "bounds") if bounds else os.path.join(ROOT, "_build")
    extra = tuple(extra) + (("-DFEMK_BOUNDS_CHECK",) if bounds else ())
    lib = LIB_BOUNDS if bounds else LIB
    os.makedirs(objdir, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include")]
    with open(os.path.join(objdir, ".lock"), "w") as lock:
        fcntl.flock(lock, fcntl.LOCK_EX)
        jobs, objs = [], []
        headers = glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "femk.h")]
        for src in sources():
            obj = os.path.join(objdir, os.path.basename(src).replace(".cu", ".o"))
            if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(d) for d in [src] + headers):
                jobs.append([nvcc, *ARCH, *FLAGS, *inc, *extra, "-c", src, "-o", obj])
            objs.append(obj)

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)

        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
            list(pool.map(run, jobs))
        tmp = lib + ".tmp"
        run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-cudart", "static"])
        os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, bounds="--bounds" in sys.argv))
