#!/usr/bin/env python
"""Benchmark: P1 128^3 Kuhn-tet Poisson, FP64 assembly + Jacobi-PCG to 1e-8, DOF/s on B200.

One step = assemble the CSR operator for one of 20 seeded log-conductivity fields, build the Jacobi
inverse, run PCG from x0 = 0 to the 1e-8 relative stop rule and evaluate the eager residual guard
(one more SpMV), with the mesh, plan and k fields resident in HBM. ``value`` = DOFs / step time
(all ranks' DOFs over the max-over-ranks time). Variants (mixed precision, matrix-free), the SpMV
roofline, the end-to-end number through the public ``jno_b200`` API with host buffers, SM clocks,
a CPU baseline (full steps of the path restated in C on all host threads) and full-size parity
against that restatement ride on the same JSON line.

``--impl reference`` times that CPU restatement (jNO itself cannot be imported on this image) on
the same workload instead, full steps on all host threads.
"""

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "assemble+CG DOF/s at 1e-8 rel err, mixed vs FP64 (1 B200); SpMV HBM GB/s"
N_FIELDS = 20
FIELD_SEED0 = 1000


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="hexes per cube side")
    ap.add_argument("--order", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--solver", choices=["fp64", "mixed", "matfree"], default="fp64",
                    help="solver of the timed step (fp64 is the headline; the others serve profiling runs)")
    ap.add_argument("--profile-step", action="store_true",
                    help="kernel profiling: after the warm-up run ONE step of --solver between cudaProfilerStart "
                         "and cudaProfilerStop (for ncu --profile-from-start off), print a short line and exit")
    ap.add_argument("--path", choices=["tri", "theta", "batched"], default=None,
                    help="time a secondary workload instead of the headline (kernel profiling): 'tri' = 2-D P1 "
                         "triangles, n^2 rectangles (--n, default 1024), FP64 assemble + PCG; 'theta' = the P1 "
                         "n^3 transient march (--n, default 128), step-operator assembly + 10 backward-Euler steps; "
                         "'batched' = the 256-problem batch, assemble + one batched FP64 PCG launch")
    return ap.parse_args()


def run_path(args):
    """One secondary workload, K timed steps after W warm-up on cuda:0 (CUDA events, inputs resident);
    prints one JSON line. Serves the ncu launch lists of the 2-D and transient paths."""
    import torch

    from jno_b200 import _lib
    from jno_b200.domain import jitter_interior_2d, rect_points_tris
    from jno_b200.plan import FemPlan

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    info = {}
    if args.path == "batched":
        from jno_b200.batch import BatchedPoisson, batched_workload
        from jno_b200.tuner import batched_schedule

        sides, probs = batched_workload(256)
        batch = BatchedPoisson([(p, t) for p, t, _ in probs])
        plan = batch.plan
        logk = torch.as_tensor(np.concatenate([lk for _, _, lk in probs]), device=dev)
        vals, b = plan.assemble(logk)
        inv = plan.jacobi(vals)
        sched = batched_schedule(batch, vals, b, inv, 1e-8)

        mixed = args.solver == "mixed"

        def step(i):
            plan.assemble(logk, vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            if mixed:
                out = plan.pcg_batched_mixed(batch.row_off, vals, b, inv, None, 1e-8, 0.0, 20_000,
                                             sched["tile_rows"], sched["blocks_per_sm"])
            else:
                out = plan.pcg_batched(batch.row_off, vals, b, None, inv, 1e-8, 0.0, 20_000, sched["tile_rows"],
                                       sched["blocks_per_sm"])
            info.setdefault("iters", []).append(float(out[1].max()))

        workload = (f"256 P1 problems, sides {int(sides.min())}..{int(sides.max())} hexes ({plan.n:,} DOF), "
                    f"assemble + batched {'mixed-precision ' if mixed else ''}Jacobi-PCG to 1e-8, schedule "
                    f"{sched['tile_rows']} rows x {sched['blocks_per_sm']} blocks/SM")
        metric, units = "DOF/s", plan.n
    elif args.path == "tri":
        n = 1024 if args.n == 128 else args.n
        pts, tris = rect_points_tris(n, n)
        plan = FemPlan(jitter_interior_2d(pts, n, n, seed=0)[:, :2], tris, 1)
        fields = [torch.as_tensor(f, device=dev) for f in logk_fields(plan.ntet, 3)]
        vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
        b = torch.empty(plan.n, dtype=torch.float64, device=dev)
        inv = torch.empty(plan.n, dtype=torch.float64, device=dev)
        x = torch.empty(plan.n, dtype=torch.float64, device=dev)

        def step(i):
            plan.assemble(fields[i % 3], vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            x.zero_()
            info.setdefault("iters", []).append(plan.pcg(vals, b, x, inv, tol=1e-8)[1])

        workload = f"P1 {n}^2 triangles ({plan.ntet:,} triangles, {plan.n:,} DOF), FP64 assemble + Jacobi-PCG to 1e-8"
        metric, units = "DOF/s", plan.n
    else:
        n = args.n
        pts, tets = make_mesh(n)
        plan = FemPlan(pts, tets, 1)
        fields = [torch.as_tensor(f, device=dev) for f in logk_fields(plan.ntet, 3)]
        p = plan.export()["points"]
        u0 = torch.sin(np.pi * p[:, 0]) * torch.sin(np.pi * p[:, 1]) * torch.sin(np.pi * p[:, 2])
        u = torch.empty_like(u0)

        def step(i):
            S, R, q = plan.assemble_theta(fields[i % 3], f=1.0, theta=1.0, dt=1e-3, dirichlet=_lib.DIRICHLET_ROWS)
            u.copy_(u0)
            it = plan.theta_march(S, R, q, u, 10)[1]
            info.setdefault("iters", []).append(float(np.mean(it)))

        workload = f"P1 {n}^3 transient heat, backward Euler, dt=1e-3, 10 steps per march ({plan.n:,} DOF)"
        metric, units = "DOF-steps/s", plan.n * 10
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        step(args.warmup + i)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    print(json.dumps({"path": args.path, "metric": metric, "value": units / (ms / 1e3), "ms_per_step": ms,
                      "steps": args.steps, "warmup": args.warmup, "config": {"workload": workload},
                      "iters": float(np.mean(info["iters"])), "gpu_launches_total": int(_lib.load().femk_kernel_launches())}))


def workload_desc(n, order, T, ndof, nnz):
    return (f"P{order} {n}^3 Kuhn tets ({T:,} tets, {ndof:,} DOF, {nnz:,} CSR nnz), jittered +-0.1h, "
            f"k=exp(N(0,0.5^2)) per tet, u=0 on the boundary, FP64 assembly to CSR + Jacobi-PCG to 1e-8, "
            f"{N_FIELDS} seeded k fields")


def make_mesh(n):
    from jno_b200.domain import box_points_tets, jitter_interior

    pts, tets = box_points_tets(n, n, n)
    return jitter_interior(pts, n, n, n, seed=0), tets


def logk_fields(T, count=N_FIELDS):
    return [np.random.default_rng(FIELD_SEED0 + i).normal(0.0, 0.5, T) for i in range(count)]


# ------------------------------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.rows = []
        self.proc = None
        self.dev = device_index

    def start(self):
        try:
            ident = self._ident()
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={ident}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _ident(self):
        import torch

        try:
            return "GPU-" + str(torch.cuda.get_device_properties(self.dev).uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
            return vis.split(",")[self.dev] if vis else str(self.dev)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sm, mx, reasons = [], [], set()
        for r in self.rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for nm, v in zip(names, r[4:8]):
                    if v.lower().startswith("active"):
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------ CPU restatement
class CpuPath:
    """The path on the host: oracle/femcpu.c (C, OpenMP, FP64) -- the compress-plan pattern, the
    row-gather assembly, the Jacobi inverse and jax-cg PCG -- on all host threads. Setup (mesh,
    boundary set, incidence, pattern) is untimed; a step is a full assembly + Jacobi + PCG to 1e-8
    from zero, nothing sampled or extrapolated."""

    def __init__(self, n, order=1, cells=None, threads=None):
        from oracle import build_cpu
        from oracle import mesh as om

        self.n_h, self.order = n, order
        pf, cf, tets, p1 = om.kuhn_cube(n, order=1, seed=0)
        if order == 2:
            cf = np.asarray(cells)  # the P2 numbering exported by the device plan (pinned at small sizes)
        self.bnd = om.boundary_nodes(cf, order)
        self.cpu = build_cpu.FemCpu(p1, cf, self.bnd, threads=threads)
        self.ndof, self.ntet = self.cpu.nv, cf.shape[0]
        self.threads = self.cpu.threads

    def step(self, logk):
        t0 = time.perf_counter()
        it, rel = self.cpu.step(logk)
        return time.perf_counter() - t0, it, rel


def cpu_steps(cpu, fields, steps, warmup=0):
    """(mean seconds per full step, iterations) of `steps` timed steps after `warmup` untimed ones."""
    times, iters = [], []
    for i in range(warmup + steps):
        t, it, rel = cpu.step(fields[i % len(fields)])
        if not rel <= 1e-4:
            raise RuntimeError(f"CPU PCG did not solve (relres {rel})")
        if i >= warmup:
            times.append(t)
            iters.append(it)
    return float(np.mean(times)), float(np.mean(iters))


def run_reference(args):
    """The reference arm: jNO's own path cannot run on this image (no jax), so the C/OpenMP
    restatement of the path (oracle/femcpu.c) times full steps of the same workload on all host
    threads. Rank 0 alone runs it; other ranks exit without work."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cpu = CpuPath(args.n)
    fields = logk_fields(cpu.ntet, N_FIELDS)
    sec, iters = cpu_steps(cpu, fields, args.steps, args.warmup)
    value = cpu.ndof / sec
    desc = (f"oracle/femcpu.c (C, OpenMP, FP64) on {cpu.threads} host threads: {args.steps} full steps of P1 "
            f"{args.n}^3 (assembly + Jacobi + PCG to 1e-8 from zero, {iters:.1f} iterations), after {args.warmup} "
            f"warm-up steps; nothing sampled or extrapolated")
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded jittered Kuhn cube, lognormal P0 k)",
        "config": {"workload": workload_desc(args.n, 1, cpu.ntet, cpu.ndof, cpu.cpu.indices.size),
                   "iterations": iters, "parallelism": f"cpu, {cpu.threads} threads (OpenMP)"},
        "cpu_baseline": {"value": value, "unit": "DOF/s", "cores": cpu.threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "DOF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "jNO (JAX) cannot be imported on this image; its path restated in C stands in for its CPU path",
    }
    print(json.dumps(out), flush=True)


def parity_full_size(plan, fields_h, dev, cpu=None):
    """The device path against the CPU restatement at the benchmark size, field 0: CSR pattern
    bit-exact, values and load within 1e-12 of the largest entry, PCG iterations and solution."""
    import torch

    cpu = cpu or CpuPath(round(plan.ntet ** (1 / 3) / 6 ** (1 / 3)), plan.order,
                         cells=plan.export()["cells"].cpu().numpy() if plan.order == 2 else None)
    ip, ind = plan.pattern()
    same_pattern = bool(np.array_equal(ip.cpu().numpy(), cpu.cpu.indptr) and
                        np.array_equal(ind.cpu().numpy(), cpu.cpu.indices))
    same_dirichlet = bool(np.array_equal(np.flatnonzero(plan.export()["dirichlet_mask"].cpu().numpy()), cpu.bnd))
    lk = fields_h[0]
    vals, b = plan.assemble(torch.as_tensor(lk, device=dev))
    vc, bc = cpu.cpu.assemble(lk)
    v_err = float(np.abs(vals.cpu().numpy() - vc).max() / np.abs(vc).max())
    b_err = float(np.abs(b.cpu().numpy() - bc).max() / np.abs(bc).max())
    out = {"workload": f"P{plan.order} ({plan.ntet:,} tets, {plan.n:,} DOF, {plan.nnz:,} nnz), k field 0",
           "pattern_bit_exact": same_pattern, "dirichlet_bit_exact": same_dirichlet,
           "max_val_err_rel": v_err, "max_b_err_rel": b_err}
    if plan.order == 1:
        inv = plan.jacobi(vals)
        x, it, rel, st = plan.pcg(vals, b, inv_diag=inv, tol=1e-8)
        cpu.cpu.jacobi()
        xc, itc, relc = cpu.cpu.pcg(1e-8)
        out.update({"iterations": it, "iterations_cpu": itc, "relres": rel,
                    "x_err_rel": float(np.linalg.norm(x.cpu().numpy() - xc) / np.linalg.norm(xc))})
    out["bars"] = ("pattern and Dirichlet set bit-exact; values and b <= 1e-12 of max; iterations within 1; "
                   "x within 1e-7")
    out["met"] = bool(same_pattern and same_dirichlet and v_err <= 1e-12 and b_err <= 1e-12 and
                      (plan.order == 2 or (abs(out["iterations"] - out["iterations_cpu"]) <= 1 and
                                           out["x_err_rel"] <= 1e-7)))
    return out


# ------------------------------------------------------------------------------------------ replicas
def replica_field(i, rank):
    """k field of step i on `rank`: ranks start at different fields (independent problems)."""
    return (i + rank) % N_FIELDS


def max_over_ranks(ms, world, device=None):
    """The job's time: the slowest rank's (an all-reduce MAX; one rank returns its own)."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(ndof, world, ms_step):
    """DOF/s of the whole job: every rank solves its own ndof-DOF problem per step."""
    return world * ndof / (ms_step / 1e3)


# ------------------------------------------------------------------------------------------ ours
def peak_hbm_gbs():
    """(HBM copy bandwidth in GB/s, its source): MEASURED_PEAKS.json's hbm_gbs when the file exists,
    else the earlier copy-bandwidth measurement on this pool (6650 GB/s)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return float(json.load(open(path))["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            pass
    return 6650.0, "fallback (no MEASURED_PEAKS.json): 6.65 TB/s"


def roofline_traffic():
    """DRAM bytes per SpMV launch from the committed ncu summary, if one exists."""
    path = os.path.join(ROOT, "profiles", "sell_spmv_fp64_p1_128.md")
    if not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None



def p2_variants(args, world, dev, timed, parity=False):
    """P2 tets at 64^3 hexes (2.15M DOF): FP64 and mixed assemble + solve, 3 steps each (and, with
    ``parity``, the values against the CPU restatement: returned under "parity")."""
    import torch

    from jno_b200.plan import FemPlan

    pts, tets = make_mesh(64)
    plan = FemPlan(pts, tets, 2)
    fields = [torch.as_tensor(f, device=dev) for f in logk_fields(plan.ntet, 3)]
    vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
    b = torch.empty(plan.n, dtype=torch.float64, device=dev)
    inv = torch.empty(plan.n, dtype=torch.float64, device=dev)
    x = torch.empty(plan.n, dtype=torch.float64, device=dev)
    info = {"it": [], "inner": []}

    def s64(i):
        plan.assemble(fields[i % 3], vals=vals, b=b)
        plan.jacobi(vals, out=inv)
        x.zero_()
        info["it"].append(plan.pcg(vals, b, x, inv, tol=1e-8)[1])

    def s32(i):
        plan.assemble(fields[i % 3], vals=vals, b=b)
        plan.jacobi(vals, out=inv)
        x.zero_()
        info["inner"].append(plan.pcg_mixed(vals, b, inv, x, tol=1e-8)[1])

    def smf(i):
        plan.load(fields[i % 3], b=b)
        plan.jacobi_matfree(fields[i % 3], out=inv)
        x.zero_()
        info["mf"].append(plan.pcg_matfree(fields[i % 3], b, x, inv, tol=1e-8)[1])

    info["mf"] = []
    ms64 = timed(s64, 3, 1) / 3
    ms32 = timed(s32, 3, 1) / 3
    msmf = timed(smf, 3, 1) / 3
    x_ref = torch.zeros_like(x)
    plan.assemble(fields[0], vals=vals, b=b)
    plan.jacobi(vals, out=inv)
    plan.pcg(vals, b, x_ref, inv, tol=1e-12, relres=False)
    x.zero_()
    plan.pcg_mixed(vals, b, inv, x, tol=1e-8)
    err = (torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref)).item()
    base = {"workload": f"P2 64^3 Kuhn tets ({plan.ntet:,} tets, {plan.n:,} DOF, {plan.nnz:,} nnz)"}
    out_parity = parity_full_size(plan, [f.cpu().numpy() for f in fields], dev) if parity else None
    return out_parity, {
        "p2_64_fp64": {**base, "value": world * plan.n / (ms64 / 1e3), "unit": "DOF/s", "ms_per_step": ms64,
                       "iters": float(np.mean(info["it"]))},
        "p2_64_mixed": {**base, "value": world * plan.n / (ms32 / 1e3), "unit": "DOF/s", "ms_per_step": ms32,
                        "inner_iters": float(np.mean(info["inner"])), "speedup_vs_fp64": ms64 / ms32,
                        "err_vs_fp64_tight": err},
        "p2_64_matrix_free": {**base, "value": world * plan.n / (msmf / 1e3), "unit": "DOF/s", "ms_per_step": msmf,
                              "iters": float(np.mean(info["mf"])), "speedup_vs_assembled_fp64": ms64 / msmf,
                              "note": "load-only assembly + matrix-free Jacobi + PCG to 1e-8, the operator "
                                      "recomputed per element from the coordinates in every CG step"},
    }


def tri_variants(world, dev, timed, n1=1024, n2=512):
    """2-D triangles: P1 on 1024^2 rectangles (1.05M DOF), P2 on 512^2 (1.05M DOF); jittered +-0.1h,
    k = exp(N(0, 0.5^2)) per triangle, FP64 assemble + Jacobi-PCG to 1e-8, 3 steps. (The mixed solver
    is not run here: at this condition number its FP32 inner CG needs more than 5x the FP64
    iterations and misses the 20,000-iteration cap.)"""
    import torch

    from jno_b200.domain import jitter_interior_2d, rect_points_tris
    from jno_b200.plan import FemPlan

    out = {}
    for order, nh in ((1, n1), (2, n2)):
        pts, tris = rect_points_tris(nh, nh)
        pts = jitter_interior_2d(pts, nh, nh, seed=0)[:, :2]
        plan = FemPlan(pts, tris, order)
        fields = [torch.as_tensor(f, device=dev) for f in logk_fields(plan.ntet, 3)]
        vals = torch.empty(plan.nnz, dtype=torch.float64, device=dev)
        b = torch.empty(plan.n, dtype=torch.float64, device=dev)
        inv = torch.empty(plan.n, dtype=torch.float64, device=dev)
        x = torch.empty(plan.n, dtype=torch.float64, device=dev)
        info = {"it": []}

        def s64(i):
            plan.assemble(fields[i % 3], vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            x.zero_()
            info["it"].append(plan.pcg(vals, b, x, inv, tol=1e-8)[1])

        base = {"workload": f"P{order} {nh}^2 triangles ({plan.ntet:,} triangles, {plan.n:,} DOF, {plan.nnz:,} nnz)"}
        ms64 = timed(s64, 3, 1) / 3
        out[f"tri_p{order}_{nh}_fp64"] = {**base, "value": world * plan.n / (ms64 / 1e3), "unit": "DOF/s",
                                          "ms_per_step": ms64, "iters": float(np.mean(info["it"]))}
        del plan
    return out


def theta_variant(plan, fields, dev, timed, dt=1e-3, nsteps=10):
    """Transient heat on the headline mesh (P1 128^3): the parametric route (k = exp(logk), rows
    replaced), backward Euler, dt = 1e-3, u0 = sin(pi x) sin(pi y) sin(pi z): one step-operator
    assembly + 10 Jacobi-BiCGStab steps to 1e-10 per march."""
    import torch

    from jno_b200 import _lib

    pts = plan.export()["points"]
    u0 = torch.sin(np.pi * pts[:, 0]) * torch.sin(np.pi * pts[:, 1]) * torch.sin(np.pi * pts[:, 2])
    u = torch.empty_like(u0)
    info = {}

    def march(i):
        S, R, q = plan.assemble_theta(fields[i % len(fields)], f=1.0, theta=1.0, dt=dt, dirichlet=_lib.DIRICHLET_ROWS)
        u.copy_(u0)
        _, iters, worst = plan.theta_march(S, R, q, u, nsteps)
        info.setdefault("it", []).append(float(np.mean(iters)))
        info.setdefault("res", []).append(worst)

    ms = timed(march, 3, 1) / 3
    return {"workload": f"P1 128^3 heat, backward Euler, dt={dt}, {nsteps} steps", "ms_per_march": ms,
            "ms_per_step": ms / nsteps, "value": plan.n * nsteps / (ms / 1e3), "unit": "DOF-steps/s",
            "bicgstab_iters_per_step": float(np.mean(info["it"])), "max_step_residual": float(np.max(info["res"]))}


def batched_variant(dev, count=256, reps=3):
    """256 independent P1 problems, sides log-uniform in [8, 48] hexes (master seed 42), own jitter
    and lognormal k each: one assembly launch over the disjoint union + one persistent batched-PCG
    launch to 1e-8 with the autotuned schedule."""
    import torch

    from jno_b200.batch import BatchedPoisson, batched_workload
    from jno_b200.tuner import batched_schedule

    sides, probs = batched_workload(count)
    batch = BatchedPoisson([(p, t) for p, t, _ in probs])
    logk = torch.as_tensor(np.concatenate([lk for _, _, lk in probs]), device=dev)
    vals, b = batch.plan.assemble(logk)
    inv = batch.plan.jacobi(vals)
    sched = batched_schedule(batch, vals, b, inv, 1e-8)
    # one untimed call with the chosen schedule first: the tuner's last trial leaves another
    # schedule's graph and tile tables in place, and their rebuild is not part of a solve
    batch.plan.pcg_batched(batch.row_off, vals, b, None, inv, 1e-8, 0.0, 20_000, sched["tile_rows"],
                           sched["blocks_per_sm"])
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        batch.plan.assemble(logk, vals=vals, b=b)
        batch.plan.jacobi(vals, out=inv)
        x, it, rel, stv, st = batch.plan.pcg_batched(batch.row_off, vals, b, None, inv, 1e-8, 0.0, 20_000,
                                                     sched["tile_rows"], sched["blocks_per_sm"])
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    x64 = x.clone()
    # the same batch in mixed precision (FP32 inner CG, per-problem FP64 reliable updates); one
    # untimed call first (its graph capture and FP32 buffers)
    batch.plan.pcg_batched_mixed(batch.row_off, vals, b, inv, None, 1e-8, 0.0, 20_000, sched["tile_rows"],
                                 sched["blocks_per_sm"])
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        batch.plan.assemble(logk, vals=vals, b=b)
        batch.plan.jacobi(vals, out=inv)
        xm, itm, outm, relm, stvm, stm = batch.plan.pcg_batched_mixed(
            batch.row_off, vals, b, inv, None, 1e-8, 0.0, 20_000, sched["tile_rows"], sched["blocks_per_sm"])
    e1.record()
    torch.cuda.synchronize()
    ms_m = e0.elapsed_time(e1) / reps
    err = max(float(torch.linalg.norm(xm[r0:r1] - x64[r0:r1]) / max(torch.linalg.norm(x64[r0:r1]).item(), 1e-300))
              for r0, r1 in zip(batch.row_off[:-1], batch.row_off[1:]) if r1 > r0)
    # algorithmic bytes of the FP64 batch: per problem and iteration the CSR product (12 nnz + 20 n)
    # and the vector phases (x, r read + written, p, q, D^-1 read, z written: 64 n; p = z + beta p: 24 n)
    ip = batch.plan.pattern()[0].cpu().numpy().astype(np.int64)
    ro = np.asarray(batch.row_off, dtype=np.int64)
    nk, nnzk = np.diff(ro), ip[ro[1:]] - ip[ro[:-1]]
    it_np = np.asarray(it.cpu() if hasattr(it, "cpu") else it, dtype=np.float64)
    sum_bytes = float(np.sum(it_np * (12.0 * nnzk + 108.0 * nk)))
    return {"workload": f"{count} P1 problems, sides {int(sides.min())}..{int(sides.max())} hexes "
                        f"({batch.plan.ntet:,} tets, {batch.plan.n:,} DOF in total)",
            "value": batch.plan.n / (ms / 1e3), "unit": "DOF/s", "ms_per_batch": ms,
            "iters_min": int(it.min()), "iters_max": int(it.max()), "max_relres": float(rel.max()),
            "sum_iteration_bytes": sum_bytes, "GB/s": sum_bytes / (ms / 1e3) / 1e9,
            "frac_of_hbm": sum_bytes / (ms / 1e3) / 1e9 / peak_hbm_gbs()[0],
            "status_ok": bool(st == 0), "schedule": {k: sched[k] for k in ("tile_rows", "blocks_per_sm")},
            "one_graph_launch": bool(getattr(batch.plan, "batch_graph", False)), "precision": "fp64",
            "mixed": {"value": batch.plan.n / (ms_m / 1e3), "unit": "DOF/s", "ms_per_batch": ms_m,
                      "speedup_vs_fp64": ms / ms_m, "inner_iters_max": int(itm.max()),
                      "fp64_updates_max": int(outm.max()), "max_relres": float(relm.max()),
                      "status_ok": bool(stm == 0), "max_err_vs_fp64_batched": err}}


def adjoint_variant(dev, n=64, n_fd=32, check=True):
    """Adjoint config: J = 1/2 sum_i M_ii (u_i - u*_i)^2 at P1 64^3, dJ/dlogk by the adjoint (forward
    solve + transposed solve + element contraction). Checked (``check``) against the adjoint computed
    on the host by the C restatement (every element) and against central differences on n_fd random
    elements, evaluated without cancellation (jno_b200.autograd.central_difference)."""
    import torch

    from jno_b200.autograd import central_difference, solve_p0
    from jno_b200.plan import FemPlan

    pts, tets = make_mesh(n)
    plan = FemPlan(pts, tets, 1)
    logk_h = np.random.default_rng(FIELD_SEED0).normal(0, 0.5, plan.ntet)
    lk_star_h = np.random.default_rng(2000).normal(0, 0.5, plan.ntet)
    logk = torch.as_tensor(logk_h, device=dev)
    m = plan.lumped_mass()
    with torch.no_grad():
        ustar = solve_p0(plan, torch.as_tensor(lk_star_h, device=dev), tol=1e-13)

    def grad_once(tol=1e-10):
        lk = logk.clone().requires_grad_(True)
        u = solve_p0(plan, lk, tol=tol)
        J = 0.5 * torch.sum(m * (u - ustar) ** 2)
        (g,) = torch.autograd.grad(J, lk)
        return g

    grad_once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 3
    e0.record()
    for _ in range(reps):
        grad_once()
    e1.record()
    torch.cuda.synchronize()
    out = {"workload": f"P1 {n}^3 ({plan.ntet:,} tets), gradient of a lumped-mass misfit w.r.t. per-element log k",
           "ms_per_gradient": e0.elapsed_time(e1) / reps, "timing_tol": 1e-10}
    if not check:
        return out
    g = grad_once(tol=1e-13).cpu().numpy()
    gmax = float(np.abs(g).max())
    # the adjoint on the host (C restatement: assembly + PCG to 1e-13 for u and lambda; numpy contraction)
    from oracle import element as oe

    cpu = CpuPath(n)
    us_h = ustar.cpu().numpy()
    mass_h = m.cpu().numpy()
    cpu.cpu.assemble(logk_h)
    cpu.cpu.jacobi()
    u_h = cpu.cpu.pcg(1e-13)[0].copy()
    cpu.cpu.b[:] = mass_h * (u_h - us_h)
    lam_h = cpu.cpu.pcg(1e-13)[0].copy()
    free = 1.0 - cpu.cpu.dmask.astype(np.float64)
    K, _ = oe.element_matrices(oe.vertices(cpu.cpu.xyz, cpu.cpu.tets.astype(np.int64)), 1)
    cells = cpu.cpu.tets.astype(np.int64)
    g_h = -np.exp(logk_h) * np.einsum("ta,tab,tb->t", (free * lam_h)[cells], K, (free * u_h)[cells])
    idx = np.random.default_rng(7).choice(plan.ntet, n_fd, replace=False)
    eps = 1e-6
    fd = central_difference(plan, logk_h, us_h, mass_h, idx, eps=eps)
    big = np.abs(g[idx]) > 1e-3 * gmax
    out.update({
        "max_err_vs_host_adjoint_rel_max_grad": float(np.abs(g - g_h).max() / gmax),
        "fd_checked_elements": n_fd, "fd_step": eps,
        "max_err_vs_fd_rel_max_grad": float(np.abs(fd - g[idx]).max() / gmax),
        "max_rel_err_vs_fd_where_g_gt_1e-3_max": float(np.max(np.abs(fd - g[idx])[big] / np.abs(g[idx])[big]))
        if big.any() else None,
        "fd_method": ("(J(+eps) - J(-eps)) / 2 eps with J(+) - J(-) = sum M d (u- + d/2 - u*), d solving "
                      "A(+) d = (A(-) - A(+)) u-: no subtractive cancellation; truncation O(eps^2), solves to 1e-13"),
        "target": "1e-6 relative to FD and to jax.grad; jax.grad cannot run here, the host adjoint stands in",
    })
    return out


def summary_of(out):
    """The key figures of a bench line in one small object (variants, parity, baselines)."""
    v = out.get("variants") or {}

    def pick(key, *fields):
        d = v.get(key) or {}
        return {f: d.get(f) for f in fields if f in d} or None

    par = out.get("parity") or {}
    return {
        "fp64_DOF_per_s": out["value"], "ms_per_step": out["ms_per_step"],
        "spmv_frac_of_hbm": (out.get("roofline") or {}).get("frac"),
        "mixed_vs_fp64": pick("mixed_fp32_fp64_reliable", "speedup_vs_fp64", "ms_per_step", "inner_iters",
                              "err_vs_fp64_tight"),
        "mixed_1e-10": pick("mixed_1e-10_vs_fp64_1e-10", "speedup_vs_fp64", "err_vs_fp64_tight"),
        "p2_64": {"fp64_ms": (v.get("p2_64_fp64") or {}).get("ms_per_step"),
                  "mixed_ms": (v.get("p2_64_mixed") or {}).get("ms_per_step"),
                  "mixed_speedup": (v.get("p2_64_mixed") or {}).get("speedup_vs_fp64"),
                  "matrix_free_ms": (v.get("p2_64_matrix_free") or {}).get("ms_per_step")} if "p2_64_fp64" in v else None,
        "adjoint_p1_64": pick("adjoint_p1_64", "ms_per_gradient", "max_err_vs_host_adjoint_rel_max_grad",
                              "max_err_vs_fd_rel_max_grad", "max_rel_err_vs_fd_where_g_gt_1e-3_max"),
        "matrix_free_ms": (v.get("matrix_free_fp64") or {}).get("ms_per_step"),
        "batched_ms": (v.get("batched_256") or {}).get("ms_per_batch"),
        "parity_met": {k: p.get("met") for k, p in par.items()} or None,
        "e2e_DOF_per_s": (out.get("e2e") or {}).get("value"),
        "cpu_baseline_DOF_per_s": (out.get("cpu_baseline") or {}).get("value"),
        "cpu_threads": (out.get("cpu_baseline") or {}).get("cores"),
    }


def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    import jno_b200 as jno
    from jno_b200 import _lib
    from jno_b200.plan import FemPlan

    lib = _lib.load()
    pts, tets = make_mesh(args.n)
    t0 = time.perf_counter()
    plan = FemPlan(pts, tets, args.order)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    T, ndof, nnz = plan.ntet, plan.n, plan.nnz
    fields_h = logk_fields(T)
    fields = [torch.as_tensor(f, device=dev) for f in fields_h]
    vals = torch.empty(nnz, dtype=torch.float64, device=dev)
    b = torch.empty(ndof, dtype=torch.float64, device=dev)
    inv = torch.empty(ndof, dtype=torch.float64, device=dev)
    x = torch.empty(ndof, dtype=torch.float64, device=dev)
    iters_seen = []
    rel_seen = []
    phase = {"asm": [], "solve": []}

    def step(i, record=False):
        lk = fields[replica_field(i, rank)]
        if record:
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
        plan.assemble(lk, vals=vals, b=b)
        plan.jacobi(vals, out=inv)
        if record:
            e1.record()
        x.zero_()
        if args.solver == "mixed":
            _, it, _, rel, st = plan.pcg_mixed(vals, b, inv, x, tol=1e-8)
        elif args.solver == "matfree":
            plan.jacobi_matfree(lk, out=inv)
            _, it, rel, st = plan.pcg_matfree(lk, b, x, inv, tol=1e-8)
        else:
            _, it, rel, st = plan.pcg(vals, b, x, inv, tol=1e-8)
        if record:
            e2.record()
            phase["pending"] = (e0, e1, e2)
        iters_seen.append(it)
        rel_seen.append(rel)
        if st != 0 or rel > 1e-4:
            raise RuntimeError(f"solve failed: status {st}, relres {rel}")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps, warmup):
        for i in range(warmup):
            fn(i)
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for i in range(steps):
            fn(warmup + i)
        end.record()
        barrier()
        return max_over_ranks(start.elapsed_time(end), world, dev)

    # ---- headline: FP64 CSR
    for i in range(args.warmup):
        step(i)
    if args.profile_step:
        barrier()
        torch.cuda.profiler.start()
        step(args.warmup)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"profile_step": args.solver, "workload": workload_desc(args.n, args.order, T, ndof, nnz),
                              "iters": iters_seen[-1], "relres": rel_seen[-1]}))
        return
    iters_seen.clear()
    rel_seen.clear()
    clocks = ClockSampler(dev.index)
    clocks.start()
    time.sleep(0.3)
    launches0 = lib.femk_kernel_launches()
    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for i in range(args.steps):
        step(args.warmup + i)
    end.record()
    barrier()
    launches = lib.femk_kernel_launches() - launches0
    clk = clocks.stop()
    ms_total = max_over_ranks(start.elapsed_time(end), world, dev)
    ms_step = ms_total / args.steps
    value = whole_job_value(ndof, world, ms_step)
    iters_mean = float(np.mean(iters_seen))

    # phase split (separate short run with events between phases)
    asm_ms, solve_ms = [], []
    for i in range(3):
        step(i, record=True)
        e0, e1, e2 = phase.pop("pending")
        torch.cuda.synchronize()
        asm_ms.append(e0.elapsed_time(e1))
        solve_ms.append(e1.elapsed_time(e2))

    # ---- dominant kernel: the sliced-ELL SpMV every CG iteration runs (CUDA events, same stream)
    xr = torch.randn(ndof, dtype=torch.float64, device=dev)
    yr = torch.empty_like(xr)
    plan.prepare_operator(vals)

    def time_launches(fn, reps=50):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record()
        for _ in range(reps):
            fn()
        s1.record()
        torch.cuda.synchronize()
        return s0.elapsed_time(s1) / reps

    sell_standalone_ms = time_launches(lambda: plan.spmv_prepared(xr, yr))
    csr_ms = time_launches(lambda: plan.spmv(vals, xr, yr))
    # the same kernel as it runs inside the CG loop: library-recorded CUDA events around every
    # step SpMV of two profiled solves (graph replay is off while profiling)
    plan.set_profiling(True)
    for i in range(2):
        plan.assemble(fields[i], vals=vals, b=b)
        plan.jacobi(vals, out=inv)
        x.zero_()
        plan.pcg(vals, b, x, inv, tol=1e-8)
    step_ms_tot, upd_ms_tot, pup_ms_tot, prof_iters = plan.profile()
    plan.set_profiling(False)
    if prof_iters <= 0 or step_ms_tot <= 0.0:
        raise RuntimeError("the profiled FP64 solves recorded no SpMV timings")
    sell_ms = step_ms_tot / max(prof_iters, 1)
    col_bytes = 2 if plan.cols16 else 4
    nsl = (ndof + 31) // 32
    tables = plan.cols16 and plan.sell_col_units != plan.sell_nnz
    # bytes the kernel must move: every stored sliced-ELL value, the column entries it streams (per-slice
    # tables: a slice whose rows share one offset sequence stores it once), slice offsets (and table
    # offsets), x read once, y written once
    sell_bytes = (plan.sell_nnz * 8 + plan.sell_col_units * col_bytes + 8 * (nsl + 1) * (2 if tables else 1)
                  + 16 * ndof)
    csr_bytes = 12 * nnz + 20 * ndof + 4
    peak, peak_src = peak_hbm_gbs()
    achieved = sell_bytes / (sell_ms / 1e3) / 1e9
    # the bulk-copy ring runs on int16 column offsets and rows of at most 32 entries (3-D P2 rows are
    # wider); the committed ncu traffic figure is for the P1 128^3 workload only
    bulk = plan.cols16 and not (plan.dim == 3 and plan.order == 2)
    profiled = plan.dim == 3 and plan.order == 1 and ndof == 129 ** 3
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": roofline_traffic() if profiled else None,
                "kernel": ((f"k_sell_bulk (FP64 sliced-ELL CG-step SpMV, bulk-copy ring, " if bulk else
                            "k_sell (FP64 sliced-ELL CG-step SpMV, thread per row, ")
                           + f"{'int16' if plan.cols16 else 'int32'} column offsets"
                           + f"{', per-slice column tables' if tables else ''})"),
                "bytes_per_launch": sell_bytes, "ms_per_launch": sell_ms, "peak_source": peak_src,
                "column_entries": plan.sell_col_units, "stored_entries": plan.sell_nnz,
                "timing": f"CUDA events around each CG-step SpMV inside {prof_iters} profiled iterations",
                "in_loop_ms": {"step_spmv": sell_ms, "update": upd_ms_tot / max(prof_iters, 1),
                               "p_update": pup_ms_tot / max(prof_iters, 1)},
                "standalone_ms": sell_standalone_ms,
                "csr_equivalent_GBps": csr_bytes / (sell_ms / 1e3) / 1e9,
                "canonical_csr_kernel": {"ms": csr_ms, "GB/s": csr_bytes / (csr_ms / 1e3) / 1e9,
                                         "bytes_per_launch": csr_bytes}}

    variants = {}
    p2_parity = None
    if not args.no_variants:
        # FP64 tight reference solution for error reporting
        plan.assemble(fields[0], vals=vals, b=b)
        plan.jacobi(vals, out=inv)
        x_ref = torch.zeros_like(x)
        plan.pcg(vals, b, x_ref, inv, tol=1e-12, relres=False)
        ref_norm = torch.linalg.norm(x_ref).item()
        # mixed precision, reliable updates
        mixed_info = {}

        def mstep(i):
            lk = fields[i % N_FIELDS]
            plan.assemble(lk, vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            x.zero_()
            _, inner, outer, rel, st = plan.pcg_mixed(vals, b, inv, x, tol=1e-8)
            mixed_info.setdefault("inner", []).append(inner)
            mixed_info.setdefault("outer", []).append(outer)
            mixed_info.setdefault("rel", []).append(rel)

        vsteps = min(args.steps, N_FIELDS)
        ms = timed(mstep, vsteps, 2) / vsteps
        mstep(N_FIELDS * 10)  # field 0 again for the error check
        err = (torch.linalg.norm(x - x_ref).item() / ref_norm)
        variants["mixed_fp32_fp64_reliable"] = {
            "value": world * ndof / (ms / 1e3), "unit": "DOF/s", "ms_per_step": ms,
            "speedup_vs_fp64": ms_step / ms, "inner_iters": float(np.mean(mixed_info["inner"])),
            "fp64_updates": float(np.mean(mixed_info["outer"])), "max_relres": float(np.max(mixed_info["rel"])),
            "err_vs_fp64_tight": err}
        # the plain FP64 method: the same assemble + Jacobi-PCG with every CG-step SpMV on the
        # canonical CSR kernel (no sliced-ELL operator), on a second plan of the same mesh
        plan_csr = FemPlan(pts, tets, args.order, options={"solver_layout": 0})
        csr_info = {}

        def cstep(i):
            lk = fields[i % N_FIELDS]
            plan_csr.assemble(lk, vals=vals, b=b)
            plan_csr.jacobi(vals, out=inv)
            x.zero_()
            _, it, rel, st = plan_csr.pcg(vals, b, x, inv, tol=1e-8)
            if st != 0 or rel > 1e-4:
                raise RuntimeError(f"CSR solve failed: status {st}, relres {rel}")
            csr_info.setdefault("it", []).append(it)
            csr_info.setdefault("rel", []).append(rel)

        csteps = min(args.steps, 5)
        ms_csr = timed(cstep, csteps, 2) / csteps
        variants["fp64_plain_csr"] = {
            "value": world * ndof / (ms_csr / 1e3), "unit": "DOF/s", "ms_per_step": ms_csr,
            "iters": float(np.mean(csr_info["it"])), "max_relres": float(np.max(csr_info["rel"])),
            "mixed_speedup_vs_plain_csr": ms_csr / ms,
            "note": "FP64 assemble + Jacobi-PCG with the canonical-CSR SpMV kernel in every CG step"}
        del plan_csr
        torch.cuda.synchronize()
        # the mixed-precision config's 1e-10 refinement target, against FP64 CG at the same tolerance
        m10 = {}

        def m10step(i, mixed):
            lk = fields[i % N_FIELDS]
            plan.assemble(lk, vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            x.zero_()
            if mixed:
                out = plan.pcg_mixed(vals, b, inv, x, tol=1e-10)
                m10.setdefault("inner", []).append(out[1])
                m10.setdefault("rel", []).append(out[3])
            else:
                m10.setdefault("it64", []).append(plan.pcg(vals, b, x, inv, tol=1e-10)[1])

        k10 = min(args.steps, 5)
        ms10_64 = timed(lambda i: m10step(i, False), k10, 1) / k10
        ms10_m = timed(lambda i: m10step(i, True), k10, 1) / k10
        m10step(N_FIELDS * 10, True)
        variants["mixed_1e-10_vs_fp64_1e-10"] = {
            "value": world * ndof / (ms10_m / 1e3), "unit": "DOF/s", "ms_per_step": ms10_m, "fp64_ms_per_step": ms10_64,
            "speedup_vs_fp64": ms10_64 / ms10_m, "inner_iters": float(np.mean(m10["inner"])),
            "fp64_iters": float(np.mean(m10["it64"])), "max_relres": float(np.max(m10["rel"])),
            "err_vs_fp64_tight": torch.linalg.norm(x - x_ref).item() / ref_norm}
        # matrix-free FP64
        mf_info = {}

        def fstep(i):
            lk = fields[i % N_FIELDS]
            plan.load(lk, b=b)
            plan.jacobi_matfree(lk, out=inv)
            x.zero_()
            _, it, rel, st = plan.pcg_matfree(lk, b, x, inv, tol=1e-8)
            mf_info.setdefault("it", []).append(it)

        fsteps = min(args.steps, 5)
        ms_f = timed(fstep, fsteps, 1) / fsteps
        variants["matrix_free_fp64"] = {"value": world * ndof / (ms_f / 1e3), "unit": "DOF/s", "ms_per_step": ms_f,
                                        "iters": float(np.mean(mf_info["it"]))}
        # Jacobi-BiCGStab (the reference's steady fem.solve() default) on the same systems
        bi_info = {}

        def bstep(i):
            lk = fields[i % N_FIELDS]
            plan.assemble(lk, vals=vals, b=b)
            plan.jacobi(vals, out=inv)
            x.zero_()
            _, it, rel, st = plan.bicgstab(vals, b, x, inv, tol=1e-8)
            if st != 0 or rel > 1e-4:
                raise RuntimeError(f"BiCGStab failed: status {st}, relres {rel}")
            bi_info.setdefault("it", []).append(it)
            bi_info.setdefault("rel", []).append(rel)

        bsteps = min(args.steps, 10)
        ms_b = timed(bstep, bsteps, 2) / bsteps
        variants["bicgstab_fp64"] = {"value": world * ndof / (ms_b / 1e3), "unit": "DOF/s", "ms_per_step": ms_b,
                                     "iters": float(np.mean(bi_info["it"])), "max_relres": float(np.max(bi_info["rel"])),
                                     "note": "2 SpMVs per iteration; stop rule <r, r> <= tol^2 <b, b>"}
        variants["spmv_csr_fp64"] = {"GB/s": csr_bytes / (csr_ms / 1e3) / 1e9, "ms": csr_ms}
        # compress_eager export of the non-parametric route (count + scan + fill, one host read)
        plan.assemble(fields[0], vals=vals, b=b)
        ip_c, ind_c, dat_c = plan.compact(vals)
        m_c = ind_c.numel()
        ms_c = time_launches(lambda: plan.compact(vals), reps=10)
        variants["compact_export"] = {"ms": ms_c, "nnz_in": nnz, "nnz_out": int(m_c),
                                      "GB/s": (20 * nnz + 12 * m_c + 40 * ndof) / (ms_c / 1e3) / 1e9,
                                      "note": "bytes: values read twice + columns + kept entries + row arrays"}
        variants["spmv_sell_fp64"] = {"GB/s": achieved, "frac_of_peak": achieved / peak, "ms_in_loop": sell_ms,
                                      "ms_standalone": sell_standalone_ms}
        p2_parity, p2 = p2_variants(args, world, dev, timed, parity=rank == 0 and world == 1 and not args.no_cpu_baseline)
        variants.update(p2)
        variants.update(tri_variants(world, dev, timed))
        variants["theta_p1_128"] = theta_variant(plan, fields, dev, timed)
        variants["adjoint_p1_64"] = adjoint_variant(dev, check=rank == 0 and world == 1 and not args.no_cpu_baseline)
        variants["batched_256"] = batched_variant(dev)

    # ---- end to end through the public API with host buffers
    d = jno.domain.from_mesh(pts, tets)
    u, v = d.fem_symbols(order=args.order)
    _r, s = d.fem_symbols(space="P0", names=("r", "s"))
    xi, yi, zi = d.variable("interior")
    xb, yb, zb = d.variable("boundary")
    ui, vi = u.bind(x=xi, y=yi, z=zi), v.bind(x=xi, y=yi, z=zi)
    logk_sym = jno.np.parameter(s, name="logk")
    fem = jno.fem([jno.np.exp(logk_sym) * (ui.x * vi.x + ui.y * vi.y + ui.z * vi.z) - 1.0 * vi, u(xb, yb, zb) - 0.0])
    system = fem.operator
    solver = jno.solve.cg(tol=1e-8)
    host_fields = [torch.as_tensor(f).pin_memory() for f in fields_h]
    out_host = torch.empty(ndof, dtype=torch.float64).pin_memory()

    def estep(i):
        lk = host_fields[replica_field(i, rank)].to(dev, non_blocking=True)
        A, bb = system.evaluate({"logk": lk})
        xs = solver(A, bb, M=jno.precond.jacobi())
        out_host.copy_(xs, non_blocking=True)

    esteps = min(args.steps, N_FIELDS)
    ms_serial = timed(estep, esteps, 2) / esteps

    # the same calls with double-buffered copies: step i+1's k field goes up on one copy stream and
    # step i's solution comes down on another while step i assembles and solves
    copy_in, copy_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    staged = {}

    def stage(i):
        with torch.cuda.stream(copy_in):
            t = host_fields[replica_field(i, rank)].to(dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(copy_in)
        staged[i] = (t, ev)

    def estep_pipe(i):
        if i not in staged:
            stage(i)
        lk, ev = staged.pop(i)
        cur = torch.cuda.current_stream()
        cur.wait_event(ev)
        lk.record_stream(cur)
        stage(i + 1)
        A, bb = system.evaluate({"logk": lk})
        xs = solver(A, bb, M=jno.precond.jacobi())
        done = torch.cuda.Event()
        done.record(cur)
        copy_out.wait_event(done)
        with torch.cuda.stream(copy_out):
            out_host.copy_(xs, non_blocking=True)
        xs.record_stream(copy_out)

    def timed_pipe(steps, warmup):
        for i in range(warmup):
            estep_pipe(i)
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for i in range(steps):
            estep_pipe(warmup + i)
        # every copy issued inside the region (steps H2D, steps D2H) ends before the end event
        cur = torch.cuda.current_stream()
        cur.wait_stream(copy_in)
        cur.wait_stream(copy_out)
        end.record()
        barrier()
        staged.clear()
        return max_over_ranks(start.elapsed_time(end), world, dev)

    ms_pipe = timed_pipe(esteps, 2) / esteps
    e2e = {"value": world * ndof / (ms_serial / 1e3), "unit": "DOF/s", "h2d_bytes_per_step": 8 * T,
           "d2h_bytes_per_step": 8 * ndof, "ms_per_step": ms_serial,
           "copies": "pinned host buffers; each step's H2D and D2H on the compute stream, in series with its "
                     "assembly and solve",
           "pipelined": {"value": world * ndof / (ms_pipe / 1e3), "ms_per_step": ms_pipe,
                         "copies": "the same calls with step i+1's H2D and step i's D2H on two copy streams, "
                                   "overlapping step i's assembly and solve (double buffering)"},
           "path": "jno_b200.fem(...).operator.evaluate({'logk'}) + jno_b200.solve.cg(tol=1e-8)(A, b, M=jacobi())"}

    cpu_baseline = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = CpuPath(args.n, args.order, cells=plan.export()["cells"].cpu().numpy() if args.order == 2 else None)
        parity = {f"p{args.order}_{args.n}": parity_full_size(plan, fields_h, dev, cpu)}
        if p2_parity is not None:
            parity["p2_64"] = p2_parity
        k_cpu = 3
        sec, it_cpu = cpu_steps(cpu, fields_h, k_cpu)
        cpu_baseline = {"value": cpu.ndof / sec, "unit": "DOF/s", "cores": cpu.threads, "kind": "port",
                        "sample": (f"oracle/femcpu.c (C, OpenMP, FP64) on {cpu.threads} host threads: {k_cpu} full "
                                   f"steps of the same workload (assembly + Jacobi + PCG to 1e-8 from zero, "
                                   f"{it_cpu:.1f} iterations, fields 0-{k_cpu - 1}), {sec * 1e3:.0f} ms per step"),
                        "host_cpus": os.cpu_count()}

    if world > 1:
        dist.barrier()
    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": "DOF/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded jittered Kuhn cube, lognormal P0 k)",
            "config": {"workload": workload_desc(args.n, args.order, T, ndof, nnz), "order": args.order,
                       "solver": args.solver,
                       "n_hex_side": args.n, "ntet": T, "dofs": ndof, "nnz": nnz, "tol": 1e-8,
                       "iterations_mean": iters_mean, "max_relres": float(np.max(rel_seen)),
                       "assemble_ms": float(np.mean(asm_ms)), "solve_ms": float(np.mean(solve_ms)),
                       "plan_setup_s": setup_s,
                       "l2": "inputs larger than L2 (381 MB CSR stream per SpMV vs 126 MB L2)",
                       "parallelism": f"replicas x{world} (independent problems per GPU, no collective)"},
            "variants": variants, "roofline": roofline, "cpu_baseline": cpu_baseline, "e2e": e2e, "parity": parity,
            "gpu_launches": int(launches), "clocks": clk,
        }
        out["summary"] = summary_of(out)  # last key: the end of the line carries the key figures
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.path:
        run_path(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
