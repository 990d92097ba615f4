"""Build recipe and ctypes binding of ``femcpu.c`` (the C/OpenMP CPU restatement of the P1/P2 path).

``build()`` compiles it with gcc into ``oracle/_ref/libfemcpu.so`` (a built artefact: ignored by git,
shipped with the tree). :class:`FemCpu` wraps a P1 or P2 tetrahedral mesh: the pattern, incidence and
Dirichlet set as setup, then ``assemble`` / ``jacobi`` / ``pcg`` / ``step`` on all host threads.
Test and benchmark infrastructure only.
"""

import ctypes
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "femcpu.c")
LIB = os.path.join(HERE, "_ref", "libfemcpu.so")


def build(verbose=False):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler: the CPU baseline cannot be built")
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = [cc, "-O3", "-fopenmp", "-fPIC", "-shared", SRC, "-o", LIB + ".tmp", "-lm"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_P = ctypes.c_void_p
_I64 = ctypes.c_int64


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


class FemCpu:
    """Tets ``cells`` i32[T, nd] (nd = 4: P1, 10: P2 in basix order, the first 4 DOFs the vertices)
    over the P1 vertex coordinates ``points`` f64[nv, 3], with Dirichlet DOFs ``dirichlet`` (ids)."""

    def __init__(self, points, cells, dirichlet, threads=None):
        lib = ctypes.CDLL(build())
        lib.femcpu_pattern.restype = ctypes.c_int64
        lib.femcpu_pcg.restype = ctypes.c_int
        self.lib = lib
        self.threads = int(threads or os.cpu_count() or 1)
        lib.femcpu_set_threads(self.threads)
        self.xyz = np.ascontiguousarray(points, dtype=np.float64)
        self.tets = np.ascontiguousarray(cells, dtype=np.int32)
        T, self.nd = self.tets.shape
        if self.nd not in (4, 10):
            raise ValueError("femcpu takes P1 (4) or P2 (10) tetrahedra")
        self.nv = int(self.tets.max()) + 1  # DOFs (rows)
        nd = ctypes.c_int(self.nd)
        self.ptr = np.empty(self.nv + 1, dtype=np.int32)
        self.inc = np.empty(self.nd * T, dtype=np.int32)
        if lib.femcpu_incidence(_I64(self.nv), _I64(T), nd, _ptr(self.tets), _ptr(self.ptr), _ptr(self.inc)):
            raise MemoryError("femcpu_incidence")
        self.indptr = np.empty(self.nv + 1, dtype=np.int32)
        nnz = lib.femcpu_pattern(_I64(self.nv), nd, _ptr(self.tets), _ptr(self.ptr), _ptr(self.inc),
                                 _ptr(self.indptr), None)
        if nnz < 0:
            raise ValueError("femcpu_pattern: a row has more than 512 columns")
        self.indices = np.empty(int(nnz), dtype=np.int32)
        lib.femcpu_pattern(_I64(self.nv), nd, _ptr(self.tets), _ptr(self.ptr), _ptr(self.inc), _ptr(self.indptr),
                           _ptr(self.indices))
        self.dmask = np.zeros(self.nv, dtype=np.uint8)
        self.dmask[np.asarray(dirichlet, dtype=np.int64)] = 1
        self.vals = np.empty(int(nnz), dtype=np.float64)
        self.b = np.empty(self.nv, dtype=np.float64)
        self.inv = np.empty(self.nv, dtype=np.float64)
        self.x = np.empty(self.nv, dtype=np.float64)
        self.work = np.empty(4 * self.nv, dtype=np.float64)

    def assemble(self, logk, f=1.0):
        lk = np.ascontiguousarray(logk, dtype=np.float64)
        self.lib.femcpu_assemble(_I64(self.nv), ctypes.c_int(self.nd), _ptr(self.xyz), _ptr(self.tets), _ptr(self.ptr),
                                 _ptr(self.inc), _ptr(self.indptr), _ptr(self.indices), _ptr(self.dmask), _ptr(lk),
                                 ctypes.c_double(f), _ptr(self.vals), _ptr(self.b))
        return self.vals, self.b

    def jacobi(self):
        self.lib.femcpu_jacobi(_I64(self.nv), _ptr(self.indptr), _ptr(self.indices), _ptr(self.vals), _ptr(self.inv))
        return self.inv

    def pcg(self, tol=1e-8, atol=0.0, maxiter=20_000):
        """From x0 = 0: (x, iterations, relres)."""
        self.x[:] = 0.0
        rel = ctypes.c_double(0.0)
        it = self.lib.femcpu_pcg(_I64(self.nv), _ptr(self.indptr), _ptr(self.indices), _ptr(self.vals), _ptr(self.b),
                                 _ptr(self.inv), _ptr(self.x), ctypes.c_double(tol), ctypes.c_double(atol),
                                 ctypes.c_int(maxiter), _ptr(self.work), ctypes.byref(rel))
        return self.x, int(it), rel.value

    def step(self, logk, tol=1e-8):
        """One benchmark step: assembly, Jacobi inverse, PCG to tol from zero. Returns (iterations, relres)."""
        self.assemble(logk)
        self.jacobi()
        _, it, rel = self.pcg(tol)
        return it, rel
