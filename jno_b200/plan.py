"""Device-resident assembly plan and the CSR operator it produces (host side of the C ABI).

A :class:`FemPlan` owns one ``femk_plan``: the P1/P2 DOF numbering, the compress-plan CSR
pattern, the element -> slot map, the Dirichlet set and the solver workspace, all in HBM. Every
method launches CUDA kernels through ``libfemk.so`` on the current torch stream; inputs and outputs
are CUDA tensors. Nothing here computes on the CPU.
"""

import ctypes

import numpy as np
import torch

from . import _lib


def _device_tensor(a, dtype):
    if isinstance(a, torch.Tensor):
        t = a.to(device="cuda", dtype=dtype)
    else:
        t = torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)
    return t.contiguous()


class FemPlan:
    """P1/P2 simplex assembly plan on the current CUDA device.

    ``points`` f64[nv, 3] with ``tets`` int[T, 4] (tetrahedra), or ``points`` f64[nv, 2] with
    int[T, 3] triangles, describe the P1 mesh; ``order`` 2 adds the edge midpoint DOFs in the
    reference's first-encounter numbering. ``dirichlet_mask`` (bool/uint8 per DOF) overrides the
    default Dirichlet set (every node on a boundary facet). ``options`` maps fields of
    ``femk_plan_options`` (include/femk.h) to values; unnamed fields keep the library defaults.
    """

    def __init__(self, points, tets, order=1, dirichlet_mask=None, options=None):
        if not torch.cuda.is_available():
            raise RuntimeError("jno_b200 needs a CUDA device (B200, sm_100a); there is no CPU path")
        lib = _lib.load()
        self._lib = lib
        t = np.asarray(tets.cpu().numpy() if isinstance(tets, torch.Tensor) else tets)
        nv = int(points.shape[0])
        dim = int(points.shape[1]) if len(points.shape) == 2 else 0
        if dim not in (2, 3):
            raise ValueError("points must be [nv, 3] (tetrahedra) or [nv, 2] (triangles)")
        kind = "tets" if dim == 3 else "triangles"
        if t.ndim != 2 or t.shape[1] != dim + 1 or t.size == 0:
            raise ValueError(f"{kind} must be a non-empty [T, {dim + 1}] array for [nv, {dim}] points")
        if t.min() < 0 or t.max() >= nv:
            raise ValueError(f"{kind} reference vertices outside [0, {nv})")
        srt = np.sort(t, axis=1)
        if np.any(srt[:, 1:] == srt[:, :-1]):
            raise ValueError(f"an element of the {kind} repeats a vertex")
        xyz = _device_tensor(points, torch.float64)
        cells = _device_tensor(t, torch.int32)
        mask = None if dirichlet_mask is None else _device_tensor(dirichlet_mask, torch.uint8)
        opts = _lib.PlanOptions()
        lib.femk_plan_options_default(ctypes.byref(opts))
        for key, value in (options or {}).items():
            if key == "size" or key not in dict(_lib.PlanOptions._fields_):
                raise ValueError(f"unknown plan option {key!r}")
            setattr(opts, key, value)
        handle = ctypes.c_void_p()
        _lib.check(
            lib.femk_plan_create_ex(
                _lib.ptr(xyz), dim, xyz.shape[0], _lib.ptr(cells), cells.shape[0], int(order), _lib.ptr(mask),
                ctypes.byref(opts), _lib.stream_handle(), ctypes.byref(handle),
            )
        )
        self._h = handle
        info = _lib.PlanInfo()
        _lib.check(lib.femk_plan_get_info(self._h, ctypes.byref(info)))
        self.order = info.order
        self.dim = info.dim
        self.nd = info.ndof_local
        self.ntet = info.ntet
        self.nvert = info.nvert
        self.n = info.n
        self.nnz = info.nnz
        self.n_dirichlet = info.n_dirichlet
        self.cols16 = bool(info.cols16)
        self.sell_nnz = int(info.sell_nnz)
        self.sell_col_units = int(info.sell_col_units)
        self.device = torch.device("cuda", info.device)
        self._pattern = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.femk_plan_destroy(h)
            except Exception:
                pass
            self._h = None

    @property
    def handle(self):
        return self._h

    # ---------------------------------------------------------------- pattern export
    def pattern(self):
        """(indptr i32[n+1], indices i32[nnz]) of the canonical CSR, cached on the device."""
        if self._pattern is None:
            indptr = torch.empty(self.n + 1, dtype=torch.int32, device=self.device)
            indices = torch.empty(self.nnz, dtype=torch.int32, device=self.device)
            _lib.check(self._lib.femk_plan_export(self._h, _lib.ptr(indptr), _lib.ptr(indices), None, None, None,
                                                  None, None, _lib.stream_handle()))
            self._pattern = (indptr, indices)
        return self._pattern

    def export(self):
        """Every plan array as CUDA tensors (dict)."""
        d = self.device
        out = {
            "slot": torch.empty(self.ntet * self.nd * self.nd, dtype=torch.int32, device=d),
            "cells": torch.empty(self.ntet * self.nd, dtype=torch.int32, device=d),
            "points": torch.empty(self.n * 3, dtype=torch.float64, device=d),
            "dirichlet_mask": torch.empty(self.n, dtype=torch.uint8, device=d),
            "diag_slot": torch.empty(self.n, dtype=torch.int32, device=d),
        }
        indptr, indices = self.pattern()
        _lib.check(self._lib.femk_plan_export(
            self._h, None, None, _lib.ptr(out["slot"]), _lib.ptr(out["cells"]), _lib.ptr(out["points"]),
            _lib.ptr(out["dirichlet_mask"]), _lib.ptr(out["diag_slot"]), _lib.stream_handle()))
        out["indptr"], out["indices"] = indptr, indices
        out["slot"] = out["slot"].view(self.ntet, self.nd, self.nd)
        out["cells"] = out["cells"].view(self.ntet, self.nd)
        out["points"] = out["points"].view(self.n, 3)[:, : self.dim]  # a 2-D plan stores z = 0
        return out

    # ---------------------------------------------------------------- kernels
    def assemble(self, param=None, mode=_lib.COEF_EXP, scale=1.0, f=1.0, g=None, vals=None, b=None):
        """(vals f64[nnz], b f64[n]) of ``k_e grad u . grad v - f v`` with Dirichlet ``u = g``."""
        if mode != _lib.COEF_CONST:
            param = _device_tensor(param, torch.float64)
            want = self.nvert if mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR) else self.ntet
            if param.numel() != want:
                kind = "nodal P1" if want == self.nvert else "P0"
                raise ValueError(f"a {kind} parameter needs {want} values, got {param.numel()}")
        g = None if g is None else _device_tensor(g, torch.float64)
        vals = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if vals is None else vals
        b = torch.empty(self.n, dtype=torch.float64, device=self.device) if b is None else b
        _lib.check(self._lib.femk_assemble(self._h, _lib.ptr(param), int(mode), float(scale), float(f), _lib.ptr(g),
                                           _lib.ptr(vals), _lib.ptr(b), _lib.stream_handle()))
        return vals, b

    def load(self, param=None, mode=_lib.COEF_EXP, scale=1.0, f=1.0, g=None, b=None):
        """The load ``b`` of :meth:`assemble` alone (no values): what a matrix-free solve needs."""
        if mode != _lib.COEF_CONST:
            param = _device_tensor(param, torch.float64)
        g = None if g is None else _device_tensor(g, torch.float64)
        b = torch.empty(self.n, dtype=torch.float64, device=self.device) if b is None else b
        _lib.check(self._lib.femk_assemble(self._h, _lib.ptr(param), int(mode), float(scale), float(f), _lib.ptr(g),
                                           None, _lib.ptr(b), _lib.stream_handle()))
        return b

    def assemble_vjp(self, param, grad_vals=None, grad_b=None, mode=_lib.COEF_EXP, scale=1.0, g=None):
        """d(vals, b)/dparam applied to the cotangents (grad_vals f64[nnz], grad_b f64[n], either
        may be None): f64[ntet] for P0 modes, f64[nvert] for nodal modes (``femk_assemble_vjp``)."""
        param = _device_tensor(param, torch.float64)
        g = None if g is None else _device_tensor(g, torch.float64)
        nodal = mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR)
        out = torch.empty(self.nvert if nodal else self.ntet, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.femk_assemble_vjp(self._h, _lib.ptr(param), int(mode), float(scale), _lib.ptr(g),
                                               _lib.ptr(grad_vals), _lib.ptr(grad_b), _lib.ptr(out),
                                               _lib.stream_handle()))
        return out

    def compact(self, vals):
        """(indptr i32[n+1], indices i32[m], data f64[m]): the entries of ``vals`` with ``|v| > 0``
        in CSR order (``compress_eager``, jno/utils/solver/fem_utils.py:4063-4091)."""
        indptr = torch.empty(self.n + 1, dtype=torch.int32, device=self.device)
        indices = torch.empty(self.nnz, dtype=torch.int32, device=self.device)
        data = torch.empty(self.nnz, dtype=torch.float64, device=self.device)
        m = ctypes.c_int64(-1)
        _lib.check(self._lib.femk_compact(self._h, _lib.ptr(vals), _lib.ptr(indptr), _lib.ptr(indices), _lib.ptr(data),
                                          self.nnz, ctypes.byref(m), _lib.stream_handle()))
        return indptr, indices[: m.value], data[: m.value]

    def element_matrices(self):
        khat = torch.empty(self.ntet, self.nd, self.nd, dtype=torch.float64, device=self.device)
        fhat = torch.empty(self.ntet, self.nd, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.femk_element_matrices(self._h, _lib.ptr(khat), _lib.ptr(fhat), _lib.stream_handle()))
        return khat, fhat

    def lumped_mass(self):
        m = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.femk_lumped_mass(self._h, _lib.ptr(m), _lib.stream_handle()))
        return m

    def jacobi(self, vals, out=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_jacobi(self._h, _lib.ptr(vals), _lib.ptr(out), _lib.stream_handle()))
        return out

    def jacobi_matfree(self, param=None, mode=_lib.COEF_EXP, scale=1.0, out=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_jacobi_matfree(self._h, _lib.ptr(param), int(mode), float(scale), _lib.ptr(out),
                                                 _lib.stream_handle()))
        return out

    def spmv(self, vals, x, out=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_spmv(self._h, _lib.ptr(vals), _lib.ptr(x), _lib.ptr(out), _lib.stream_handle()))
        return out

    def prepare_operator(self, vals):
        """Gather CSR values into the plan's sliced-ELL solver copy (what each CG iteration uses)."""
        _lib.check(self._lib.femk_prepare_operator(self._h, _lib.ptr(vals), _lib.stream_handle()))

    def spmv_prepared(self, x, out=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_spmv_prepared(self._h, _lib.ptr(x), _lib.ptr(out), _lib.stream_handle()))
        return out

    def set_profiling(self, on=True):
        _lib.check(self._lib.femk_set_profiling(self._h, 1 if on else 0))

    def profile(self):
        """(step SpMV ms, update ms, p-update ms, iterations) accumulated while profiling is on."""
        v = [ctypes.c_double(0.0) for _ in range(3)]
        it = ctypes.c_int64(0)
        _lib.check(self._lib.femk_get_profile(self._h, *[ctypes.byref(x) for x in v], ctypes.byref(it)))
        return v[0].value, v[1].value, v[2].value, it.value

    def spmv_matfree(self, param, x, mode=_lib.COEF_EXP, scale=1.0, out=None):
        out = torch.empty(self.n, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_spmv_matfree(self._h, _lib.ptr(param), int(mode), float(scale), _lib.ptr(x),
                                               _lib.ptr(out), _lib.stream_handle()))
        return out

    def pcg(self, vals, b, x=None, inv_diag=None, tol=1e-8, atol=0.0, maxiter=20_000, relres=True):
        """Jacobi-PCG (jax cg semantics). Returns (x, iterations, relres, status)."""
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = ctypes.c_int32(0)
        rr = ctypes.c_double(float("nan"))
        st = self._lib.femk_pcg(self._h, _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv_diag), float(tol),
                                float(atol), int(maxiter), ctypes.byref(it), ctypes.byref(rr) if relres else None,
                                _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        return x, it.value, rr.value, st

    def pcg_matfree(self, param, b, x=None, inv_diag=None, mode=_lib.COEF_EXP, scale=1.0, tol=1e-8, atol=0.0,
                    maxiter=20_000, relres=True):
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = ctypes.c_int32(0)
        rr = ctypes.c_double(float("nan"))
        st = self._lib.femk_pcg_matfree(self._h, _lib.ptr(param), int(mode), float(scale), _lib.ptr(b), _lib.ptr(x),
                                        _lib.ptr(inv_diag), float(tol), float(atol), int(maxiter), ctypes.byref(it),
                                        ctypes.byref(rr) if relres else None, _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        return x, it.value, rr.value, st

    def bicgstab(self, vals, b, x=None, inv_diag=None, tol=1e-8, atol=0.0, maxiter=20_000):
        """Jacobi-BiCGStab (jax bicgstab semantics). Returns (x, iterations, relres, status);
        a breakdown is reported as FEMK_BREAKDOWN with x as the iteration left it."""
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = ctypes.c_int32(0)
        rr = ctypes.c_double(float("nan"))
        st = self._lib.femk_bicgstab(self._h, _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv_diag), float(tol),
                                     float(atol), int(maxiter), ctypes.byref(it), ctypes.byref(rr),
                                     _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED, _lib.FEMK_BREAKDOWN))
        return x, it.value, rr.value, st

    def pcg_mixed(self, vals, b, inv_diag, x=None, tol=1e-8, atol=0.0, maxiter=20_000, mode=_lib.MIXED_RELIABLE):
        """FP32-inner / FP64-refined PCG. Returns (x, inner iterations, outer updates, relres, status)."""
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        inner = ctypes.c_int32(0)
        outer = ctypes.c_int32(0)
        rr = ctypes.c_double(float("nan"))
        st = self._lib.femk_pcg_mixed(self._h, _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv_diag),
                                      float(tol), float(atol), int(maxiter), int(mode), ctypes.byref(inner),
                                      ctypes.byref(outer), ctypes.byref(rr), _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        return x, inner.value, outer.value, rr.value, st

    def pcg_batched(self, row_off, vals, b, x=None, inv_diag=None, tol=1e-8, atol=0.0, maxiter=20_000,
                    tile_rows=2048, blocks_per_sm=2):
        """Independent Jacobi-PCGs of the problems owning rows [row_off[k], row_off[k+1]).

        Returns (x, iterations i32[nprob], relres f64[nprob], status i32[nprob], return status)."""
        ro = np.ascontiguousarray(np.asarray(row_off, dtype=np.int64))
        nprob = ro.size - 1
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = np.zeros(nprob, dtype=np.int32)
        rel = np.zeros(nprob, dtype=np.float64)
        stv = np.zeros(nprob, dtype=np.int32)
        c = ctypes.c_void_p
        st = self._lib.femk_pcg_batched(self._h, nprob, c(ro.ctypes.data), _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x),
                                        _lib.ptr(inv_diag), float(tol), float(atol), int(maxiter), int(tile_rows),
                                        int(blocks_per_sm), c(it.ctypes.data), c(rel.ctypes.data), c(stv.ctypes.data),
                                        _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        info = _lib.PlanInfo()
        _lib.check(self._lib.femk_plan_get_info(self._h, ctypes.byref(info)))
        self.batch_graph = bool(info.batch_graph)
        return x, it, rel, stv, st

    def pcg_batched_mixed(self, row_off, vals, b, inv_diag, x=None, tol=1e-8, atol=0.0, maxiter=20_000,
                          tile_rows=2048, blocks_per_sm=2):
        """Mixed-precision form of :meth:`pcg_batched` (FP32 inner CG, FP64 reliable updates).

        Returns (x, FP32 iterations i32[nprob], FP64 updates i32[nprob], relres f64[nprob],
        status i32[nprob], return status)."""
        ro = np.ascontiguousarray(np.asarray(row_off, dtype=np.int64))
        nprob = ro.size - 1
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = np.zeros(nprob, dtype=np.int32)
        outer = np.zeros(nprob, dtype=np.int32)
        rel = np.zeros(nprob, dtype=np.float64)
        stv = np.zeros(nprob, dtype=np.int32)
        c = ctypes.c_void_p
        st = self._lib.femk_pcg_batched_mixed(
            self._h, nprob, c(ro.ctypes.data), _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv_diag),
            float(tol), float(atol), int(maxiter), int(tile_rows), int(blocks_per_sm), c(it.ctypes.data),
            c(outer.ctypes.data), c(rel.ctypes.data), c(stv.ctypes.data), _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        info = _lib.PlanInfo()
        _lib.check(self._lib.femk_plan_get_info(self._h, ctypes.byref(info)))
        self.batch_graph = bool(info.batch_graph)
        return x, it, outer, rel, stv, st

    def adjoint_grad(self, param, u, lam, mode=_lib.COEF_EXP, scale=1.0, out=None):
        nodal = mode in (_lib.COEF_NODAL_EXP, _lib.COEF_NODAL_LINEAR)
        size = self.nvert if nodal else self.ntet
        out = torch.empty(size, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_adjoint_grad(self._h, _lib.ptr(param), int(mode), float(scale), _lib.ptr(u),
                                               _lib.ptr(lam), _lib.ptr(out), _lib.stream_handle()))
        return out

    # ---------------------------------------------------------------- transient
    def mass_matrix(self, zero_dirichlet=False, out=None):
        """Consistent mass f64[nnz] in the canonical CSR (Dirichlet rows/columns zeroed on request)."""
        out = torch.empty(self.nnz, dtype=torch.float64, device=self.device) if out is None else out
        _lib.check(self._lib.femk_mass_matrix(self._h, 1 if zero_dirichlet else 0, _lib.ptr(out),
                                              _lib.stream_handle()))
        return out

    def assemble_theta(self, param=None, mode=_lib.COEF_EXP, scale=1.0, f=1.0, g=None, theta=1.0, dt=1.0,
                       dirichlet=_lib.DIRICHLET_ROWS):
        """(step_vals, rhs_vals, q) of the theta step: S = M' + theta dt A', R = M' - (1 - theta) dt A',
        q = dt (c' + f') on the canonical CSR."""
        if mode != _lib.COEF_CONST:
            param = _device_tensor(param, torch.float64)
        g = None if g is None else _device_tensor(g, torch.float64)
        S = torch.empty(self.nnz, dtype=torch.float64, device=self.device)
        R = torch.empty(self.nnz, dtype=torch.float64, device=self.device)
        q = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.femk_assemble_theta(self._h, _lib.ptr(param), int(mode), float(scale), float(f),
                                                 _lib.ptr(g), float(theta), float(dt), int(dirichlet), _lib.ptr(S),
                                                 _lib.ptr(R), _lib.ptr(q), _lib.stream_handle()))
        return S, R, q

    def theta_march(self, step_vals, rhs_vals, q, u, nsteps, tol=1e-10, maxiter=20_000, traj=None,
                    step_check=1e-9, with_rescue=False):
        """Advance u (in place) by nsteps theta steps (Jacobi-BiCGStab per step). Returns (u,
        iterations i32[nsteps], worst BiCGStab step residual), plus the GMRES rescue's Arnoldi steps
        i32[nsteps] when with_rescue; traj f64[nsteps, n] receives every state when given. A step
        whose relative residual is not below step_check (<= 0: no check) is re-solved by GMRES."""
        it = np.zeros(max(int(nsteps), 1), dtype=np.int32)
        gm = np.zeros(max(int(nsteps), 1), dtype=np.int32)
        worst = ctypes.c_double(0.0)
        _lib.check(self._lib.femk_theta_march(
            self._h, _lib.ptr(step_vals), _lib.ptr(rhs_vals), _lib.ptr(q), _lib.ptr(u), int(nsteps), float(tol),
            int(maxiter), float(step_check), _lib.ptr(traj), ctypes.c_void_p(it.ctypes.data),
            ctypes.c_void_p(gm.ctypes.data), ctypes.byref(worst), _lib.stream_handle()))
        if with_rescue:
            return u, it[: int(nsteps)], worst.value, gm[: int(nsteps)]
        return u, it[: int(nsteps)], worst.value

    def gmres(self, vals, b, x=None, inv_diag=None, tol=1e-8, atol=0.0, restart=30, maxiter=None):
        """Restarted Jacobi-GMRES (jax gmres, solve_method="batched"). Returns (x, Arnoldi steps,
        restart cycles, relres, status); maxiter None is jax's 10 n restart cycles, 0 runs none.
        1 <= restart <= 64 (the library's largest Krylov basis)."""
        x = torch.zeros(self.n, dtype=torch.float64, device=self.device) if x is None else x
        it = ctypes.c_int32(0)
        cyc = ctypes.c_int32(0)
        rr = ctypes.c_double(float("nan"))
        st = self._lib.femk_gmres(self._h, _lib.ptr(vals), _lib.ptr(b), _lib.ptr(x), _lib.ptr(inv_diag), float(tol),
                                  float(atol), int(restart), -1 if maxiter is None else int(maxiter), ctypes.byref(it),
                                  ctypes.byref(cyc), ctypes.byref(rr), _lib.stream_handle())
        _lib.check(st, allow=(_lib.FEMK_NOT_CONVERGED,))
        return x, it.value, cyc.value, rr.value, st
