"""Benchmark: time to true relative residual 1e-8 on the 192^3 heterogeneous
7-point diffusion system, plain FP64 drop-in path, one B200 per rank.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--n 192] [--method ilu0|jacobi|cheb3_saad_power20|cheb3_saad_lanczos20]

Workload (per rank): 192^3 cells, log10 k = seeded Gaussian random field
(std 1, smoothing length 4 cells), harmonic-mean faces, Dirichlet faces,
b = A x_true with x_true ~ U[-1,1] (seeds: rank).  CSR + sliced ELL-32, FP64.
A step is one complete solve: preconditioner set-up + the CG loop to
||r||/||b|| < 1e-8 (Alien's stop test), with the matrix and b already
resident in HBM.  e2e repeats the step through the C ABI from HOST arrays:
matrix upload + set-up + b upload + solve + x download.

Each rank solves its own system (weak scaling, no collective on the data
path).  Timing: CUDA events on libab2's stream, barrier + synchronize around
the K timed steps, max over ranks.  The matrix (>600 MB) is larger than L2,
so no explicit flush is needed between steps.

--impl reference times the reference's own CPU path for the same workload:
Alien's CG.h + ILU0Preconditioner.h templates over the SimpleCSR-restating
algebra (oracle/_ref), one host core (SimpleCSR and its ILU(0) sweeps are
sequential per rank).  It builds the system with the host-only build of the
same seeded generator (oracle/_build/libab2_inputs.so) and loads no CUDA
code.  Each warm-up step is a bounded sample (set-up + 2 and 8 iterations,
whose per-iteration time cross-checks the complete solves); each timed step
is one COMPLETE solve to convergence, as many of the requested K as fit in
--ref-budget seconds (at least one); the line reports the counts that ran.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

# Plain FP64 forms timed on the same system (CG to ||r||/||b|| < 1e-8).
# "ilu0" is the headline (the configuration names CG+ILU0 first); the others
# are reported beside it under "methods".
METHODS = {
    "ilu0": dict(precond="ilu0"),
    "jacobi": dict(precond="diag"),
    "cheb3_saad_power20": dict(precond="cheb", cheb_saad=True, poly_order=3, poly_factor_max_iter=20),
    "cheb3_saad_lanczos20": dict(precond="cheb", cheb_saad=True, cheb_lanczos=True, poly_order=3,
                                 poly_factor_max_iter=20),
}

# The reference's other two preconditioners, measured where they converge
# (bench `preconditioners` section): on the heterogeneous headline system
# unscaled Neumann stalls (rows with small coefficients barely move) and
# BiCGStab + FILU0 diverges, as the reference's own templates do.
OTHER_METHODS = {
    # NeumannPolyPreconditioner.h (omega = 1 / power-method estimate, 20 steps)
    "neumann3_power20": dict(precond="neumann", poly_order=3, poly_factor_max_iter=20),
    # FILU0Preconditioner.h: exact ILU(0) factor, 3 Jacobi sweeps per triangle
    # (the krylov example's defaults); not symmetric, so with BiCGStab
    "bicgstab_filu0_3": dict(solver="bicgs", precond="filu0", filu_factor_iter=0, filu_solver_iter=3),
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_init():
    from alien_b200 import dist

    return dist.init("nccl")


def barrier(world):
    from alien_b200 import dist

    dist.barrier(world)


def max_over_ranks(world, value: float) -> float:
    from alien_b200 import dist

    return dist.reduce_max(world, value)


def spmv_bytes(info, n: int) -> int:
    """Sliced-ELL SpMV algorithmic bytes: stored (value + column) + slice
    offsets + x read once + y written once."""
    return int(info.ell_stored * 12 + 4 * (n // 32 + 1) + 16 * n)


def ilu_bytes(n: int, nnz: int) -> int:
    """ILU0 apply (both sweeps), B_LU: the LU factor's values and column
    indices, its row pointers and one n-vector of 8-byte values."""
    return int(12 * nnz + 4 * (n + 1) + 8 * n)


def ilu_stencil_min_bytes(n: int, nnz: int) -> int:
    """ILU0 apply (both sweeps), the least any schedule on a 7-point matrix
    must move: every factor value read once (no column indices: the stencil
    fixes them), y read once, x written once."""
    return int(8 * nnz + 16 * n)


def iteration_bytes(method: str, n: int, nnz: int) -> int:
    """Fused-schedule lower bound of one PCG iteration (FP64), from the CSR
    SpMV bytes B = 12 nnz + 4(n+1) + 16 n: Jacobi B + 104 n; ILU0
    B + B_LU + 120 n with B_LU = 12 nnz + 4(n+1) + 8 n; Chebyshev(3)
    4 B + 200 n; Neumann(k) (k+1) B + (24 k + 104) n; BiCGStab + FILU0(S)
    twice (B + S B_sweeps + 100 n), B_sweeps = 12 (nnz - n) + 56 n (the strict
    triangles' slots and one L and one U sweep's vectors)."""
    b_spmv = 12 * nnz + 4 * (n + 1) + 16 * n
    m = METHODS[method] if method in METHODS else OTHER_METHODS[method]
    pc = m["precond"]
    if pc == "diag":
        return b_spmv + 104 * n
    if pc == "ilu0":
        return b_spmv + (12 * nnz + 4 * (n + 1) + 8 * n) + 120 * n
    if pc == "neumann":
        k = m["poly_order"]
        return (k + 1) * b_spmv + (24 * k + 104) * n
    if pc == "filu0":
        return 2 * (b_spmv + m["filu_solver_iter"] * (12 * (nnz - n) + 56 * n) + 100 * n)
    return 4 * b_spmv + 200 * n


def load_traffic():
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return {}
    return {}


# ----------------------------------------------------------------------------- reference arm
def reference_method(method: str) -> tuple[dict, str]:
    """The reference configuration that times `method` on the CPU: the same
    preconditioner through Alien's own templates.  Lanczos bounds have no
    reference counterpart; its nearest reference form (power-method bounds,
    same Saad recurrence) stands in and the sample says so."""
    kw = dict(poly_factor=0.0, poly_order=3, poly_factor_max_iter=20, cheb_saad=False)
    m = METHODS[method]
    kw["precond"] = m["precond"]
    kw["solver"] = m.get("solver", "cg")
    if m["precond"] == "cheb":
        kw["cheb_saad"] = True
        kw["poly_order"] = m["poly_order"]
        kw["poly_factor_max_iter"] = m["poly_factor_max_iter"]
    if m["precond"] == "filu0":
        kw["filu_factor_iter"] = m["filu_factor_iter"]
        kw["filu_solver_iter"] = m["filu_solver_iter"]
    if m["precond"] == "neumann":
        kw["poly_order"] = m["poly_order"]
    label = {"ilu0": "ILU0Preconditioner.h", "diag": "DiagPreconditioner.h",
             "cheb": "ChebyshevPreconditioner<.., true>.h (power-method bounds)",
             "filu0": "BiCGStab.h + FILU0Preconditioner.h",
             "neumann": "NeumannPolyPreconditioner.h (omega = 1/Gershgorin bound: its own estimate "
                        "seeds from std::random_device)"}[m["precond"]]
    return kw, label


def reference_sample(P, method: str, iterations_hint: int | None, sample_iters=(2, 8)):
    """Alien's own templates (oracle/_ref) on one host core: set-up + a few
    iterations, extrapolated to `iterations_hint` (the iteration count this
    solve takes; the templates and the GPU agree on it to +-2).  A bounded
    sample: the complete solve is timed by reference_solve."""
    from oracle import oracle as O

    kw = reference_kwargs(P, method)
    times = []
    for m in sample_iters:
        t = time.perf_counter()
        r = O.solve(P.row_ptr, P.cols, P.vals, P.b, tol=1e-8, max_iter=m, which="ref", **kw)
        times.append((r.iterations, time.perf_counter() - t))
    (i1, t1), (i2, t2) = times
    per_iter = (t2 - t1) / max(i2 - i1, 1)
    setup = max(t1 - i1 * per_iter, 0.0)
    iters = iterations_hint if iterations_hint else i2
    return setup + per_iter * iters, setup, per_iter, sum(t for _, t in times)


def reference_kwargs(P, method: str) -> dict:
    kw, _ = reference_method(method)
    if kw["precond"] == "neumann":
        kw["poly_factor"] = 1.0 / float(np.add.reduceat(np.abs(P.vals), P.row_ptr[:-1]).max())
    return kw


def reference_solve(P, method: str, max_iter: int):
    """One complete solve by Alien's own templates (oracle/_ref) on one host
    core, set-up included: (seconds, result)."""
    from oracle import oracle as O

    kw = reference_kwargs(P, method)
    t = time.perf_counter()
    r = O.solve(P.row_ptr, P.cols, P.vals, P.b, tol=1e-8, max_iter=max_iter, which="ref", **kw)
    return time.perf_counter() - t, r


def all_cores_sample(P, method: str, iterations: int, sample_iters=(2, 8)) -> dict:
    """The all-cores CPU baseline: this repo's restatement of the SimpleCSR
    algebra with its SpMV and BLAS-1 loops on every host thread
    (oracle/_build/libab2_oracle_threads.so), running `method` (Jacobi or
    Chebyshev CG, whose loops parallelise; ILU(0)'s sweeps do not) --
    set-up + 2 and 8 iterations, scaled to `iterations`.  A restatement, not
    the reference."""
    from oracle import oracle as O

    kw, label = reference_method(method)
    times = []
    for m in sample_iters:
        t = time.perf_counter()
        r = O.solve(P.row_ptr, P.cols, P.vals, P.b, tol=1e-8, max_iter=m, which="threads", **kw)
        times.append((r.iterations, time.perf_counter() - t))
    (i1, t1), (i2, t2) = times
    per_iter = (t2 - t1) / max(i2 - i1, 1)
    setup = max(t1 - i1 * per_iter, 0.0)
    threads = int(os.environ.get("AB2_CPU_THREADS", os.cpu_count() or 1))
    return {"value": round(setup + per_iter * iterations, 4), "unit": "s", "cores": threads, "kind": "port",
            "method": method, "iterations": iterations, "extrapolated": True, **host_info(),
            "sample": f"restatement, not reference: CG + {label} with the SimpleCSR SpMV and BLAS-1 loops on "
                      f"{threads} host threads; set-up + 2 and 8 iterations ({t1 + t2:.1f} s), scaled to "
                      f"{iterations} iterations (set-up {setup:.2f} s, {per_iter * 1e3:.1f} ms/iteration)"}


def host_info() -> dict:
    """The host the CPU legs ran on: logical cores and the CPU model."""
    model = None
    try:
        for ln in Path("/proc/cpuinfo").read_text().splitlines():
            if ln.lower().startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "cpu_model": model}


def solution_digest(x: np.ndarray) -> dict:
    """Size-independent figures of a solution, printed by both arms so that
    their solutions can be compared across processes: 2-norm, plain sum and
    the dot with a fixed +-1 pattern."""
    w = np.where(np.arange(x.size) % 3 == 0, 1.0, -1.0)
    return {"norm2": float(np.linalg.norm(x)), "sum": float(np.sum(x)), "dot_pm1": float(np.dot(w, x))}


def reference_main(a, world: int, rank: int, P, config: dict) -> int:
    """--impl reference: Alien's templates on the host cores (rank 0 only)."""
    if rank != 0:
        return 0
    from oracle import oracle as O

    _, label = reference_method(a.method)
    t_start = time.perf_counter()
    samples = []
    for _ in range(a.warmup):  # bounded samples; their per-iteration time cross-checks the complete solves
        samples.append(reference_sample(P, a.method, None))
    steps, res = [], None
    t0 = time.perf_counter()
    while len(steps) < max(a.steps, 1):
        dt, res = reference_solve(P, a.method, a.max_iter)
        steps.append(dt)
        if time.perf_counter() - t0 + dt > a.ref_budget:
            break
    value = float(np.median(steps))
    r_true = P.b - O.spmv(P.row_ptr, P.cols, P.vals, res.x)
    true_rel = float(np.linalg.norm(r_true) / np.linalg.norm(P.b))
    cross = None
    if samples:
        _, setup, per_iter, _ = samples[-1]
        cross = {"sample_setup_s": round(setup, 4), "sample_ms_per_iteration": round(per_iter * 1e3, 3),
                 "extrapolated_s": round(setup + per_iter * res.iterations, 3),
                 "note": "set-up + 2 and 8 iterations (a warm-up step), scaled to the complete solve's iterations"}
    host = host_info()
    # Beside it, one complete Jacobi-CG solve by the all-cores restatement
    # (its loops parallelise; the reference's ILU(0) sweeps do not).
    cpu_all = None
    if a.method == "ilu0":
        kw, lab = reference_method("jacobi")
        t = time.perf_counter()
        rj = O.solve(P.row_ptr, P.cols, P.vals, P.b, tol=1e-8, max_iter=a.max_iter, which="threads", **kw)
        tj = time.perf_counter() - t
        threads = int(os.environ.get("AB2_CPU_THREADS", os.cpu_count() or 1))
        cpu_all = {"jacobi": {"value": round(tj, 4), "unit": "s", "cores": threads, "kind": "port",
                              "iterations": rj.iterations, "converged": bool(rj.converged), **host,
                              "sample": f"restatement, not reference: one complete CG + {lab} solve with the "
                                        f"SimpleCSR SpMV and BLAS-1 loops on {threads} host threads"}}
    line = {"metric": "time_to_true_rel_residual_1e-8", "value": value, "unit": "s", "n_gpus": a.gpus,
            "steps": len(steps), "warmup": len(samples), "requested": {"steps": a.steps, "warmup": a.warmup},
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded generator, host-only build)", "impl": "reference",
            "config": config, "iterations": res.iterations, "converged": bool(res.converged),
            "true_rel_residual": true_rel,
            "rel_error_vs_x_true": float(np.linalg.norm(res.x - P.x_true) / np.linalg.norm(P.x_true)),
            "solution_digest": solution_digest(res.x), "step_times_s": [round(t, 4) for t in steps],
            "cross_check": cross,
            "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference", **host,
                             "sample": f"Alien CG.h + {label} (oracle/_ref) on 1 host core, {len(steps)} complete "
                                       f"solve(s) to convergence ({res.iterations} iterations), set-up included; "
                                       f"SimpleCSR and its ILU(0) sweeps are sequential per rank"},
            "cpu_all_cores": cpu_all,
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": round(time.perf_counter() - t_start, 2)}
    print(json.dumps(line), flush=True)
    return 0


def timed_solve(torch, stream, make, run, reps=3):
    """One warm pass, then `reps` timed (set-up + solve) passes on the
    library's stream; returns the median time and the median pass's result."""
    obj = make()
    run(obj)
    obj.close()
    runs = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        obj = make()
        res = run(obj)
        e1.record(stream)
        e1.synchronize()
        hist = obj.history() if hasattr(obj, "history") else None
        obj.close()
        runs.append((e0.elapsed_time(e1) / 1e3, res, hist))
    runs.sort(key=lambda v: v[0])
    return runs[len(runs) // 2]


MIXED_METHODS = {  # mixed-precision forms of the FP64 methods, same system, same 1e-8 true residual
    "ilu0": dict(precond="ilu0"),
    "jacobi": dict(precond="diag"),  # AUTO: the scaled Jacobi form on the 7-point bands
    "jacobi_plain": dict(precond="diag", jacobi_form="plain"),
    "cheb3_saad_lanczos20": dict(precond="cheb", cheb_saad=True, cheb_lanczos=True, poly_order=3,
                                 poly_factor_max_iter=20),
}


def mixed_section(abi, ctx, stream, A, P, b, x, methods, a):
    """Mixed precision (FP32 inner Krylov, FP64 refinement): the 192^3
    system to true relative residual 1e-8 beside each FP64 method, and the
    128^3 convection-diffusion system (BiCGStab + ILU0 inner, 1e-10) with its
    error against an FP64 BiCGStab solution."""
    import torch

    out = {"diffusion3d_192": {}, "note": "time = set-up + solve on the device (CUDA events); "
                                         "speedups against the FP64 solver on the same system; errors "
                                         "against an FP64 CG+ILU0 solution to 1e-12"}
    x_fp64 = x.download()  # the FP64 headline solution (CG + ILU0, 1e-8)
    S = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-12, max_iter=a.max_iter)
    ctx.assign(x, 0.0)
    S.solve(b, x)
    S.close()
    x_ref = x.download()
    out["fp64_cg_ilu0_1e-8_rel_error"] = float(np.linalg.norm(x_fp64 - x_ref) / np.linalg.norm(x_ref))
    fp64_best = min(v["s"] for v in methods.values()) if methods else None
    for m, kw in MIXED_METHODS.items():
        def make(kw=kw):
            return abi.Mixed(ctx, A, solver="cg", tol=1e-8, max_outer=20, inner_tol=1e-4, inner_max_iter=5000,
                             use_graph=not a.host_loop, **kw)

        def run(M):
            ctx.assign(x, 0.0)
            return M.solve(b, x)

        t, st, hist = timed_solve(torch, stream, make, run)
        xs = x.download()
        entry = {"s": round(t, 5), "converged": bool(st.succeeded), "true_rel_residual": st.true_residual,
                 "outer_iterations": st.outer_iterations, "inner_iterations": st.inner_iterations,
                 "setup_ms": round(st.setup_ms, 3), "solve_ms": round(st.solve_ms, 3),
                 "rel_error_vs_fp64_1e-12": float(np.linalg.norm(xs - x_ref) / np.linalg.norm(x_ref)),
                 "residual_history": [float(h) for h in hist]}
        entry["jacobi_scaled"] = bool(st.jacobi_scaled)
        if st.jacobi_scaled and st.inner_iterations:
            # FP32 inner CG on the scaled operator: 3 bands + 11 vectors of 4 bytes per row and iteration
            entry["inner_bytes_per_iteration"] = 56 * P.n
        base = m if m in methods else m.split("_")[0]
        if base in methods:
            entry["speedup_vs_fp64_same_precond"] = round(methods[base]["s"] / t, 3)
        if "ilu0" in methods:
            entry["speedup_vs_fp64_cg_ilu0"] = round(methods["ilu0"]["s"] / t, 3)
        if fp64_best:
            entry["speedup_vs_fastest_fp64"] = round(fp64_best / t, 3)
        out["diffusion3d_192"][m] = entry
    ctx.assign(x, 0.0)

    # 128^3 convection-diffusion, nonsymmetric: mixed BiCGStab + ILU0 to 1e-10 vs FP64 BiCGStab + ILU0.
    n3 = 128 if a.n >= 128 else a.n
    Q = abi.convdiff(n3, n3, n3, peclet=10.0, modes=8, seed=0)
    AQ = ctx.matrix(Q.row_ptr, Q.cols, Q.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32 | abi.FMT_STENCIL)
    bq, xq = ctx.vector(Q.b), ctx.vector(Q.n)

    def run_q(S):
        ctx.assign(xq, 0.0)
        return S.solve(bq, xq)

    t64, st64, _ = timed_solve(torch, stream, lambda: abi.Solver(ctx, AQ, solver="bicgs", precond="ilu0", tol=1e-10,
                                                                 max_iter=5000, use_graph=not a.host_loop), run_q)
    tm, stm, hist = timed_solve(torch, stream, lambda: abi.Mixed(ctx, AQ, solver="bicgs", precond="ilu0", tol=1e-10,
                                                                 max_outer=20, inner_tol=1e-4, inner_max_iter=5000,
                                                                 use_graph=not a.host_loop), run_q)
    xm = xq.download()
    # the FP64 BiCGStab solution the error is stated against: tightened to 1e-12
    S = abi.Solver(ctx, AQ, solver="bicgs", precond="ilu0", tol=1e-12, max_iter=5000)
    ctx.assign(xq, 0.0)
    S.solve(bq, xq)
    S.close()
    x64 = xq.download()
    out[f"convdiff3d_{n3}"] = {
        "workload": f"convdiff3d_{n3}^3_peclet10_modes8_bicgstab_ilu0_tol1e-10", "rows": Q.n, "nnz": Q.nnz,
        "mixed": {"s": round(tm, 5), "converged": bool(stm.succeeded), "true_rel_residual": stm.true_residual,
                  "outer_iterations": stm.outer_iterations, "inner_iterations": stm.inner_iterations,
                  "residual_history": [float(h) for h in hist],
                  "rel_error_vs_fp64_bicgstab_1e-12": float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))},
        "fp64": {"s": round(t64, 5), "converged": bool(st64.succeeded), "iterations": st64.iterations,
                 "true_rel_residual": st64.true_residual},
        "speedup": round(t64 / tm, 3)}
    for o in (bq, xq, AQ):
        o.close()
    return out


def fmt_name(variant: int, slice_rows: int, lanes: int) -> str:
    """The batched solver's inner SpMV format: ell<rows per slice> or csr_l<lanes per row>."""
    return f"ell{slice_rows}" if variant == 3 else f"csr_l{lanes}" if variant == 1 else str(variant)


def batch_section(abi, ctx, stream, a):
    """The batched form: 512 independent SPD systems (2-D 5-point or 3-D
    7-point heterogeneous diffusion, log10 k ~ smoothed N(0,1), per-system
    seed, rows log-uniform in [2,000, 200,000]) solved in one persistent
    launch to per-system true relative residual 1e-8 (FP32 Jacobi-CG inside
    FP64 refinement); the configuration picked by the autotuner."""
    import torch

    t = time.perf_counter()
    B = abi.batch_problem(nsys=a.batch_systems, min_rows=2000, max_rows=200000, seed=0, sigma=1.0, smooth=2.0)
    gen_s = time.perf_counter() - t
    Q = B.problem
    A = ctx.matrix(Q.row_ptr, Q.cols, Q.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32)
    bq, xq = ctx.vector(Q.b), ctx.vector(Q.n)
    S = abi.Batch(ctx, A, B.sys_offsets, tol=1e-8, max_outer=20, inner_tol=1e-4, inner_max_iter=20000)
    info = S.info
    times = []
    for i in range(3):
        ctx.assign(xq, 0.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = S.solve(bq, xq)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1) / 1e3)
    conv, outer, inner, res = S.results()
    xs = xq.download()
    err = []
    for s_ in range(0, B.nsys, max(1, B.nsys // 16)):
        lo, hi = B.sys_offsets[s_], B.sys_offsets[s_ + 1]
        err.append(float(np.linalg.norm(xs[lo:hi] - Q.x_true[lo:hi]) / np.linalg.norm(Q.x_true[lo:hi])))
    sizes = np.diff(B.sys_offsets)
    # Inner FP32 Jacobi-PCG bytes per iteration of each system, the fused-schedule
    # lower bound B_SpMV + 52 n with 4-byte values (B_SpMV = 8 nnz + 4 (n + 1) + 8 n).
    nnz_s = np.diff(Q.row_ptr[B.sys_offsets]).astype(np.float64)
    bytes_it = 8 * nnz_s + 4 * (sizes + 1) + 8 * sizes + 52 * sizes
    inner_bytes = float(np.sum(inner.astype(np.float64) * bytes_it))
    pk, pk_kind = peaks()
    out = {"workload": f"{B.nsys} systems, 2-D 5-pt / 3-D 7-pt heterogeneous diffusion, rows log-uniform 2k-200k, "
                       f"cg_jacobi fp32 inner + fp64 refinement, per-system tol 1e-8",
           "systems": B.nsys, "rows": int(Q.n), "nnz": int(Q.nnz), "rows_min_max": [int(sizes.min()), int(sizes.max())],
           "systems_3d": int(sum(1 for d in B.dims if d[2] > 1)),
           "s": round(min(times), 5), "s_runs": [round(v, 5) for v in times],
           "systems_converged": int(conv.sum()), "max_true_rel_residual": float(res.max()),
           "inner_iterations_total": int(inner.sum()), "inner_iterations_max": int(inner.max()),
           "outer_steps_max": int(outer.max()),
           "rows_per_s": round(Q.n / min(times), 1),
           "inner_bytes": inner_bytes,
           "inner_gbs": round(inner_bytes / min(times) / 1e9, 1),
           "inner_frac": round(inner_bytes / min(times) / 1e9 / pk["hbm_gbs"], 4), "peak_source": pk_kind,
           "inner_bytes_note": "sum over systems of inner iterations x (8 nnz + 4 (n + 1) + 60 n): the FP32 "
                               "Jacobi-PCG fused-schedule lower bound; systems of up to ~20 MB run from L2",
           "config": {"spmv_variant": fmt_name(info.spmv_variant, info.ell_slice, info.lanes_per_row),
                      "cluster_size": info.cluster_size, "threads": info.threads, "autotuned": bool(info.tuned)},
           "autotune_ms": round(info.tune_ms, 2), "setup_ms": round(info.setup_ms, 2),
           "trials": [{"spmv": fmt_name(v, sl, lpr), "cluster": c, "threads": th, "ms": round(ms, 3)}
                      for v, c, th, ms, sl, lpr in S.trials()],
           "rel_error_vs_x_true_sample": err, "generate_s": round(gen_s, 2)}
    S.close()
    for o in (bq, xq, A):
        o.close()
    return out


def preconditioner_section(abi, ctx, stream, A, P, a):
    """Every preconditioner of the path: one application at the headline size
    (time and GB/s of its algorithmic bytes), and the two the headline system
    does not suit solved where they converge -- BiCGStab + FILU0 against
    BiCGStab + ILU0 on the 128^3 convection-diffusion system, CG + Neumann
    against CG + Jacobi on the 192^3 constant-coefficient Poisson system."""
    import torch

    n, nnz = P.n, P.nnz
    b_spmv = 12 * nnz + 4 * (n + 1) + 16 * n
    sweeps = 12 * (nnz - n) + 56 * n
    kinds = {"diag": (dict(kind="diag"), 24 * n),
             "ilu0": (dict(kind="ilu0"), ilu_bytes(n, nnz)),
             "cheb3_saad": (dict(kind="cheb", cheb_saad=True, poly_order=3, poly_factor_max_iter=20),
                            3 * b_spmv + 5 * 8 * n),
             "filu0_3": (dict(kind="filu0", filu_factor_iter=0, filu_solver_iter=3), 3 * sweeps),
             "neumann3": (dict(kind="neumann", poly_order=3, poly_factor_max_iter=20), 3 * (b_spmv + 16 * n))}
    pk, pk_kind = peaks()
    vx, vy = ctx.vector(P.b), ctx.vector(n)
    out = {"apply": {}, "note": "algorithmic bytes per application: diag 24n; ILU0 B_LU = 12 nnz + 4 (n + 1) + 8 n; Chebyshev(3) "
                                 "3 B_spmv + 40 n; FILU0(3 sweeps) 3 (12 (nnz - n) + 56 n); Neumann(3) 3 (B_spmv + 16 n)"}
    for name, (kw, nbytes) in kinds.items():
        pc = abi.Precond(ctx, A, **kw)
        for _ in range(3):
            pc.apply(vx, vy)
        k0 = torch.cuda.Event(enable_timing=True)
        k1 = torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(20):
            pc.apply(vx, vy)
        k1.record(stream)
        k1.synchronize()
        ms = k0.elapsed_time(k1) / 20
        out["apply"][name] = {"ms": round(ms, 4), "algorithmic_bytes": int(nbytes),
                              "gbs": round(nbytes / ms / 1e6, 1), "frac": round(nbytes / ms / 1e6 / pk["hbm_gbs"], 4)}
        pc.close()
    for v in (vx, vy):
        v.close()
    out["peak_source"] = pk_kind

    def solve_pair(Q, label, pairs):
        AQ = ctx.matrix(Q.row_ptr, Q.cols, Q.vals)
        bq, xq = ctx.vector(Q.b), ctx.vector(Q.n)
        res = {"rows": Q.n, "nnz": Q.nnz}

        def run(S):
            ctx.assign(xq, 0.0)
            return S.solve(bq, xq)

        for name, kw in pairs:
            t, st, _ = timed_solve(torch, stream, lambda kw=kw: abi.Solver(ctx, AQ, tol=1e-8, max_iter=5000,
                                                                            use_graph=not a.host_loop, **kw), run)
            res[name] = {"s": round(t, 5), "iterations": st.iterations, "converged": bool(st.succeeded),
                         "true_rel_residual": st.true_residual}
        for o in (bq, xq, AQ):
            o.close()
        out[label] = res

    m = 128 if a.n >= 128 else a.n
    solve_pair(abi.convdiff(m, m, m, peclet=10.0, modes=8, seed=0), f"convdiff3d_{m}",
               [(f"bicgstab_filu0_{k}", dict(solver="bicgs", precond="filu0", filu_factor_iter=0, filu_solver_iter=k))
                for k in (3, 6, 10)] + [("bicgstab_ilu0", dict(solver="bicgs", precond="ilu0"))])
    solve_pair(abi.poisson(a.n, a.n, a.n, seed=0), f"poisson3d_{a.n}",
               [("cg_neumann3_power20", dict(solver="cg", precond="neumann", poly_order=3, poly_factor_max_iter=20)),
                ("cg_jacobi", dict(solver="cg", precond="diag"))])
    return out


def small_section(abi, ctx, stream, a):
    """The plain method at the small size: 3-D 7-point constant-coefficient
    Poisson on 32^3 (32,768 rows), b = A x_true, Jacobi-CG to 1e-8, max 1000
    iterations -- the case the reference runs on its CPU path.  The matrix
    (3.3 MB) lives in L2: a latency-bound case, reported but not a roofline
    figure.  Beside it the reference's own CG.h + DiagPreconditioner.h
    (oracle/_ref) solving the same system on one host core."""
    import torch

    Q = abi.poisson(32, 32, 32, seed=0)
    A = ctx.matrix(Q.row_ptr, Q.cols, Q.vals)
    b, x = ctx.vector(Q.b), ctx.vector(Q.n)

    def run(S):
        ctx.assign(x, 0.0)
        return S.solve(b, x)

    t, st, _ = timed_solve(torch, stream, lambda: abi.Solver(ctx, A, solver="cg", precond="diag", tol=1e-8,
                                                              max_iter=1000, use_graph=not a.host_loop), run)
    out = {"workload": "poisson3d_32^3_cg_jacobi_tol1e-8", "rows": Q.n, "nnz": Q.nnz, "s": round(t, 6),
           "iterations": st.iterations, "converged": bool(st.succeeded), "true_rel_residual": st.true_residual,
           "note": "set-up + solve on the device, median of three; the matrix lives in L2 (latency-bound)"}
    if not a.no_cpu:
        from oracle import oracle as O

        if O.ref_available():
            runs = []
            for _ in range(3):
                t0 = time.perf_counter()
                r = O.solve(Q.row_ptr, Q.cols, Q.vals, Q.b, solver="cg", precond="diag", tol=1e-8, max_iter=1000,
                            which="ref")
                runs.append(time.perf_counter() - t0)
            out["cpu_reference"] = {"s": round(sorted(runs)[1], 6), "iterations": r.iterations, "cores": 1,
                                    "kind": "reference",
                                    "sample": "Alien CG.h + DiagPreconditioner.h (oracle/_ref), whole solve, median "
                                              "of three"}
    for o in (b, x, A):
        o.close()
    return out


def rowblock_section(abi, stream, P, x_single, iters_single, a):
    """The row-block distribution (include/ab2_dist.h) on the headline system:
    the device-resident distributed CG + ILU0 with one rank over NCCL (its
    solution must equal the single-GPU solver's bit for bit), and 2, 4, 8
    ranks of a local group SHARING this one GPU -- the iteration counts of
    block-Jacobi ILU(0) as the slabs shrink and the cost of the distributed
    machinery; their times are not a scaling measurement."""
    import threading

    out = {"note": "1 rank over NCCL, then R ranks sharing one GPU (threads of one process, host barriers): "
                   "times of shared-GPU runs are not multi-GPU scaling"}
    n = P.n
    plane = a.n * a.n

    def solve_rank(ctx, comm, off, r, res):
        t0 = time.perf_counter()
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        S = abi.DistSolver(ctx, comm, A, solver="cg", precond="ilu0", tol=1e-8, max_iter=a.max_iter)
        b, x = A.vector(P.b[off[r]:off[r + 1]]), A.vector()
        t1 = time.perf_counter()
        st = S.solve(b, x)
        res[r] = (st, x.download() if r == 0 or len(off) == 2 else None, t1 - t0, time.perf_counter() - t1)
        S.close(), A.close(), b.close(), x.close()

    try:
        uid = abi.Comm.nccl_unique_id()
        ctx = abi.Context(0)
        comm = abi.Comm.nccl(ctx, uid, 0, 1)
        off = np.asarray([0, n], np.int32)
        res = [None]
        solve_rank(ctx, comm, off, 0, res)  # warm
        solve_rank(ctx, comm, off, 0, res)
        st, xr, setup_s, solve_s = res[0]
        out["nccl_1"] = {"iterations": st.iterations, "converged": bool(st.succeeded), "solve_ms": round(st.solve_ms, 2),
                         "setup_s": round(setup_s, 3), "true_rel_residual": st.true_residual,
                         "identical_to_single_gpu_solver": bool(np.array_equal(xr, x_single)
                                                                and st.iterations == iters_single)}
        comm.close()
        ctx.close()
    except abi.AB2Error as e:
        out["nccl_1"] = {"unavailable": str(e)}

    for k in (2, 4, 8):
        off = abi.row_offsets(n, k, plane)
        ctxs = [abi.Context(0) for _ in range(k)]
        comms = abi.Comm.local_group(ctxs, timeout_s=600.0)
        res = [None] * k
        ts = [threading.Thread(target=solve_rank, args=(ctxs[r], comms[r], off, r, res)) for r in range(k)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()
        if any(v is None for v in res):
            out[f"local_{k}"] = {"error": "a rank failed"}
            continue
        st = res[0][0]
        out[f"local_{k}"] = {"ranks": k, "planes_per_rank": a.n // k, "iterations": st.iterations,
                             "converged": bool(st.succeeded), "true_rel_residual": st.true_residual,
                             "solve_ms_max_over_ranks": round(max(v[0].solve_ms for v in res), 2),
                             "iterations_vs_one_rank": round(st.iterations / iters_single, 3)}
        for c in comms:
            c.close()
    return out


def rowblock_main(a, world, rank, local) -> int:
    """--rowblock: ONE 192^3 system split across the N ranks by z-slabs
    (include/ab2_dist.h over NCCL: halo per SpMV, rank-ordered sums, block-Jacobi
    ILU(0) for N > 1) -- strong scaling.  Every rank builds the same global
    system and keeps its block; the solve is the device-resident distributed
    CG, timed with CUDA events on each rank's stream, max over ranks."""
    import torch

    from alien_b200 import abi

    pc = METHODS[a.method]["precond"]
    if pc not in ("ilu0", "diag"):
        raise SystemExit("--rowblock runs CG with ilu0 or jacobi")
    n1 = a.n
    P = abi.diffusion(n1, n1, n1, sigma=1.0, smooth=4.0, seed=0)
    off = abi.row_offsets(P.n, world, n1 * n1)
    torch.cuda.set_device(local)
    ctx = abi.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    if world > 1:
        import torch.distributed as tdist

        box = [abi.Comm.nccl_unique_id() if rank == 0 else None]
        tdist.broadcast_object_list(box, src=0)
        uid = box[0]
    else:
        uid = abi.Comm.nccl_unique_id()
    comm = abi.Comm.nccl(ctx, uid, rank, world)
    lo, hi = int(off[rank]), int(off[rank + 1])
    kw = dict(solver="cg", precond=pc, tol=1e-8, max_iter=a.max_iter)

    def e2e_step():
        t = time.perf_counter()
        A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
        b, x = A.vector(P.b[lo:hi]), A.vector()
        S = abi.DistSolver(ctx, comm, A, **kw)
        S.solve(b, x)
        x.download()
        v = time.perf_counter() - t
        S.close(), A.close(), b.close(), x.close()
        return v

    A = abi.DistMatrix.from_global(ctx, comm, off, P.row_ptr, P.cols, P.vals)
    b, x = A.vector(P.b[lo:hi]), A.vector()

    def step():
        S = abi.DistSolver(ctx, comm, A, **kw)
        ctx.assign(x, 0.0)
        st = S.solve(b, x)
        S.close()
        return st

    for _ in range(a.warmup):
        step()
    ctx.synchronize()
    launches0 = ctx.launches
    barrier(world)
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            st = step()
        e1.record(stream)
        e1.synchronize()
    barrier(world)
    launches = ctx.launches - launches0
    ms = max_over_ranks(world, e0.elapsed_time(e1) / a.steps)
    e2e = None if a.no_e2e else max_over_ranks(world, min(e2e_step() for _ in range(2)))
    if rank == 0:
        print(json.dumps({
            "metric": "time_to_true_rel_residual_1e-8", "value": round(ms / 1e3, 5), "unit": "s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, one system)",
            "config": {"workload": f"diffusion3d_{n1}^3_grf_sigma1_len4_cg_{a.method}_tol1e-8", "rows": P.n,
                       "nnz": P.nnz, "solver": "cg", "method": a.method, "tol": 1e-8,
                       "parallelism": f"row blocks x{world} (z-slabs; NCCL halo + rank-ordered sums; "
                                      f"{'block-Jacobi ' if world > 1 and pc == 'ilu0' else ''}{pc})",
                       "l2": "inputs larger than L2 (no flush)"},
            "iterations": st.iterations, "converged": bool(st.succeeded), "true_rel_residual": st.true_residual,
            "e2e": None if e2e is None else {"value": round(e2e, 4), "unit": "s",
                                             "h2d_bytes_per_step": int(P.row_ptr.nbytes + P.cols.nbytes
                                                                       + P.vals.nbytes + P.b.nbytes),
                                             "d2h_bytes_per_step": int(P.n * 8),
                                             "note": "per rank: block set-up from host arrays + solve + x "
                                                     "download, wall clock, max over ranks"},
            "roofline": None, "cpu_baseline": None, "gpu_launches": int(launches), "clocks": clk.summary()}),
            flush=True)
    for o in (b, x, A, comm):
        o.close()
    from alien_b200 import dist

    dist.finish(world)
    return 0


GNN_WEIGHTS = ROOT / "alien_b200" / "gnn_weights.npy"


def long_row_matrix(n: int, mean: int, seed: int = 0):
    """Synthetic long-row CSR system: row i holds L_i entries (L_i uniform in
    [mean/4, 7 mean/4]) at columns i + j (n // L_i) mod n, diagonal first,
    sorted; values uniform in [-1, 1].  The shape on which one thread per
    row stalls and a warp per row does not."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(mean // 4, 7 * mean // 4 + 1, n).astype(np.int64)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    row = np.repeat(np.arange(n, dtype=np.int64), lens)
    j = np.arange(rp[-1], dtype=np.int64) - rp[row]
    col = (row + j * (n // lens[row])) % n
    order = np.argsort(row * n + col, kind="stable")
    return rp.astype(np.int32), col[order].astype(np.int32), rng.uniform(-1, 1, rp[-1])


def spmv_variant_section(abi, ctx, timed, A, P, a):
    """Every SpMV variant timed alone on the headline matrix and on a
    long-row matrix; GB/s over the CSR algorithmic bytes (value + column per
    entry, row pointers, x and y once), which the ELL variant also moves at
    slice width 7."""
    names = {abi.SPMV_CSR_SCALAR: "csr_scalar", abi.SPMV_CSR_STAGED: "csr_staged",
             abi.SPMV_CSR_VECTOR: "csr_warp_per_row", abi.SPMV_ELL: "ell32", abi.SPMV_STENCIL: "stencil_bands"}
    pk, _ = peaks()

    def table(M, n, nnz, variants):
        x, y = ctx.vector(np.random.default_rng(5).uniform(-1, 1, n)), ctx.vector(n)
        nbytes = 12 * nnz + 4 * (n + 1) + 16 * n
        out = {}
        for v in variants:
            ms = timed(lambda v=v: ctx.mult(M, x, y, v), 30)
            out[names[v]] = {"us": round(ms * 1e3, 1), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1)}
            if v == abi.SPMV_STENCIL:
                own = M.info.stencil_bands * 8 * n + 16 * n  # the bands, x once, y once
                out[names[v]].update({"own_bytes": own, "own_gbs": round(own / (ms * 1e-3) / 1e9, 1),
                                      "own_frac": round(own / (ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4),
                                      "bands": M.info.stencil_bands})
        return out

    head = list(names) if A.info.stencil_bands else [v for v in names if v != abi.SPMV_STENCIL]
    res = {"bytes": "12 nnz + 4 (n + 1) + 16 n (CSR); stencil_bands also by its own bytes: bands x 8 n + 16 n",
           "headline": table(A, P.n, P.nnz, head)}
    names.pop(abi.SPMV_STENCIL)
    rp, ci, v = long_row_matrix(a.long_rows, 256)
    L = ctx.matrix(rp, ci, v, abi.FMT_CSR | abi.FMT_ELL)
    res["long_rows"] = {"n": a.long_rows, "nnz": int(rp[-1]), "row_len": "uniform 64..448",
                        **table(L, a.long_rows, int(rp[-1]), list(names))}
    L.close()
    return res


def gnn_apply_bytes(n: int, nbw: int, layer: str = "gather") -> int:
    """Algorithmic bytes of one network application: scale (r, 1/sqrt(a_ii)
    read, x_r written), encoder (x_r, log a_ii read, h1 written), three layers
    (h read once, the graph, h written) and the last layer (h and the graph
    read, x_r and 1/sqrt(a_ii) read, z written).  The graph per node: the
    gather layer's nbw-slot neighbour table (column + feature, 8 bytes a
    slot); the grid layer's six direction features (24 bytes)."""
    g = 24 if layer == "grid" else 8 * nbw
    per_node = (8 + 4 + 4) + (4 + 4 + 128) + 3 * (128 + g + 128) + (128 + g + 4 + 4 + 8)
    return n * per_node


def learned_section(abi, ctx, stream, a):
    """The learned preconditioner: flexible CG (FCG(8)) on held-out
    heterogeneous fields (128^3, log10 k ~ smoothed N(0, 1.5^2), smoothing
    length drawn in [2, 8] cells; training used other seeds) to relative
    residual 1e-8: the trained network alone; the network with ILU(0) for the
    step after each network step that does not reduce the residual; the
    network with its learned part removed (only its Jacobi skip: the method
    without it); ILU(0) alone; and the plain FP64 CG + ILU(0) / CG + Jacobi
    solvers.  Errors against the plain solver's converged solution (CG + ILU(0)
    to 1e-12)."""
    import torch

    from alien_b200 import gnn_train

    if not GNN_WEIGHTS.exists():
        return {"unavailable": "no trained weights: python -m alien_b200.gnn_train"}
    side = 128 if a.n >= 128 else a.n
    seeds = (5_000_017, 5_000_018)
    meta = json.loads(GNN_WEIGHTS.with_suffix(".json").read_text()) if GNN_WEIGHTS.with_suffix(".json").exists() else {}
    out = {"training": meta, "fields": [],
           "note": "time = set-up (network binding / ILU0 factor) + solve, CUDA events on the library stream; "
                   "flexible CG keeps 8 directions"}
    for seed in seeds:
        out["fields"].append(learned_field(abi, ctx, stream, a, gnn_train.field(side, seed),
                                           f"diffusion3d_{side}^3_grf_sigma1.5_len2-8_heldout_seed{seed}_tol1e-8"))
    f0 = out["fields"][0]
    out["apply_ms"] = f0.pop("apply_ms")
    out["network_roofline"] = f0.pop("network_roofline")
    out["fields"][-1].pop("apply_ms", None)
    out["fields"][-1].pop("network_roofline", None)
    return out


def learned_field(abi, ctx, stream, a, P, workload):
    import torch

    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_STENCIL)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    S = abi.Solver(ctx, A, solver="cg", precond="ilu0", tol=1e-12, max_iter=a.max_iter)
    S.solve(b, x)
    S.close()
    xs = x.download()

    def err():
        v = x.download()
        return float(np.linalg.norm(v - xs) / np.linalg.norm(xs))

    out = {"workload": workload, "rows": P.n, "nnz": P.nnz}

    def run_solver(S):
        ctx.assign(x, 0.0)
        return S.solve(b, x)

    for name, pc in (("cg_ilu0", "ilu0"), ("cg_jacobi", "diag")):
        t, st, _ = timed_solve(torch, stream, lambda pc=pc: abi.Solver(ctx, A, solver="cg", precond=pc, tol=1e-8,
                                                                       max_iter=a.max_iter), run_solver)
        out[name] = {"s": round(t, 5), "iterations": st.iterations, "converged": bool(st.succeeded),
                     "true_rel_residual": st.true_residual, "rel_error": err()}

    w = np.load(GNN_WEIGHTS)
    trained = abi.Gnn(ctx, w)
    w_skip = w.copy()
    w_skip[192 + 4 * 8192 + 264:192 + 4 * 8192 + 329] = 0.0  # decoder wd, bd: only the Jacobi skip is left
    skip_only = abi.Gnn(ctx, w_skip)

    class Fcg:
        def __init__(self, net, fallback):
            self.net, self.pc = net, None
            if net is not None:
                net.bind(A)
            if fallback:
                self.pc = abi.Precond(ctx, A, "ilu0")

        def close(self):
            if self.pc is not None:
                self.pc.close()

    def run_fcg(F, cap=3000, ratio=1.0):
        ctx.assign(x, 0.0)
        return abi.fcg_solve(ctx, A, b, x, gnn=F.net, fallback=F.pc, tol=1e-8, max_iter=cap, fallback_ratio=ratio)

    # fallback_ratio: ILU(0) takes the next step when a network step's residual
    # reduction |r_new| / |r_old| is not below it -- 1.0 (no reduction) and the
    # configuration's 0.5
    for name, net, fb, ratio in (("fcg_ilu0", None, True, 1.0), ("fcg_gnn_ilu0_fallback", trained, True, 1.0),
                                 ("fcg_gnn_ilu0_fallback_ratio0.5", trained, True, 0.5),
                                 ("fcg_gnn", trained, False, 1.0), ("fcg_network_skip_only", skip_only, False, 1.0)):
        t, st, _ = timed_solve(torch, stream, lambda net=net, fb=fb: Fcg(net, fb),
                               lambda F, ratio=ratio: run_fcg(F, ratio=ratio))
        out[name] = {"s": round(t, 5), "iterations": st.iterations, "converged": bool(st.succeeded),
                     "fallback_ratio": ratio,
                     "network_steps": st.gnn_steps, "ilu0_steps": st.fallback_steps, "switched_at": st.switched_at,
                     "true_rel_residual": st.true_residual, "rel_error": err(), "solve_ms": round(st.solve_ms, 3)}
    # one network application and one ILU(0) application, alone
    trained.bind(A)
    pc = abi.Precond(ctx, A, "ilu0")
    vz = ctx.vector(P.n)

    def per_call(f, reps=20):
        for _ in range(3):
            f()
        k0 = torch.cuda.Event(enable_timing=True)
        k1 = torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(reps):
            f()
        k1.record(stream)
        k1.synchronize()
        return k0.elapsed_time(k1) / reps

    layer = trained.layer
    g_ms = per_call(lambda: trained.apply(b, vz))
    i_ms = per_call(lambda: pc.apply(b, vz))
    # the same network on the gather layer kernel (indexed neighbour rows, mma.sync)
    gather = abi.Gnn(ctx, w)
    gather.set_layer("gather")
    gather.bind(A)
    gg_ms = per_call(lambda: gather.apply(b, vz))
    gather.close()
    nbw = max(2, (int(np.diff(P.row_ptr).max()) - 1 + 1) // 2 * 2)
    gb = gnn_apply_bytes(P.n, nbw, layer)
    pk, pk_kind = peaks()
    out["apply_ms"] = {"network": round(g_ms, 4), "network_layer": layer, "network_gather_layer": round(gg_ms, 4),
                       "ilu0": round(i_ms, 4)}
    out["network_roofline"] = {"bound": "hbm", "kernel": f"network application, {layer} layer",
                               "algorithmic_bytes": int(gb), "achieved": round(gb / g_ms / 1e6, 1),
                               "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": round(gb / g_ms / 1e6 / pk["hbm_gbs"], 4),
                               "peak_source": pk_kind}
    out["speedup_vs_cg_ilu0"] = {k: round(out["cg_ilu0"]["s"] / out[k]["s"], 3)
                                 for k in ("fcg_ilu0", "fcg_gnn_ilu0_fallback", "fcg_gnn_ilu0_fallback_ratio0.5",
                                           "fcg_gnn")}
    for o in (pc, vz, trained, skip_only, b, x, A):
        o.close()
    return out


def profile_case(a) -> int:
    """--profile-case: one piece of the workload on the --n system, run twice
    (the second run is the steady one), for ncu launch lists and captures."""
    from alien_b200 import abi

    n1 = a.n
    P = abi.diffusion(n1, n1, n1, sigma=1.0, smooth=4.0, seed=0)
    ctx = abi.Context(0)
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32 | abi.FMT_STENCIL)
    b, x = ctx.vector(P.b), ctx.vector(P.n)
    graph = not a.host_loop
    for _ in range(2):
        ctx.assign(x, 0.0)
        if a.profile_case == "spmv_bands":
            ctx.mult(A, b, x, abi.SPMV_STENCIL)
            st = None
        elif a.profile_case.startswith("gnn"):
            # one application of the committed network, grid or gather layer kernel
            net = abi.Gnn(ctx, np.load(GNN_WEIGHTS))
            net.set_layer(a.profile_case[4:])
            net.bind(A)
            net.apply(b, x)
            st = net.layer
            net.close()
        elif a.profile_case.startswith("mixed"):
            form = "plain" if a.profile_case.endswith("plain") else "auto"
            M = abi.Mixed(ctx, A, solver="cg", precond="diag", tol=1e-8, max_outer=20, inner_tol=1e-4,
                          inner_max_iter=5000, use_graph=graph, jacobi_form=form)
            st = M.solve(b, x)
            M.close()
        else:
            pc = "diag" if a.profile_case == "fp64_jacobi" else "ilu0"
            S = abi.Solver(ctx, A, solver="cg", precond=pc, tol=1e-8, max_iter=a.max_iter, use_graph=graph)
            st = S.solve(b, x)
            S.close()
        ctx.synchronize()
    print(f"profile case {a.profile_case} at {n1}^3 done: {st}", flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=192)
    ap.add_argument("--method", default="ilu0", choices=sorted(METHODS))
    ap.add_argument("--max-iter", type=int, default=20000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-methods", action="store_true", help="time the headline method only")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision measurements")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-systems measurement")
    ap.add_argument("--batch-systems", type=int, default=512)
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-preconditioner measurement")
    ap.add_argument("--no-precond", action="store_true", help="skip the per-preconditioner measurements")
    ap.add_argument("--no-rowblock", action="store_true", help="skip the row-block distribution measurements")
    ap.add_argument("--no-small", action="store_true", help="skip the 32^3 Jacobi-CG case")
    ap.add_argument("--no-variants", action="store_true", help="skip the per-variant SpMV table")
    ap.add_argument("--long-rows", type=int, default=262144, help="rows of the long-row SpMV matrix")
    ap.add_argument("--rowblock", action="store_true",
                    help="strong scaling instead: one system split across the N ranks by z-slabs (NCCL), "
                         "distributed CG")
    ap.add_argument("--profile-case", choices=["mixed_jacobi", "mixed_jacobi_plain", "fp64_jacobi", "fp64_ilu0",
                                               "gnn_grid", "gnn_gather", "spmv_bands"],
                    help="run one small piece of the workload and exit (for profilers): the solve, the SpMV or "
                         "one network application, twice, on the --n system, no timing or JSON line")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="--impl reference: seconds of complete solves to fit the timed steps into")
    ap.add_argument("--host-loop", action="store_true",
                    help="drive the Krylov loop from the host instead of the CUDA graph (same kernels; for "
                         "profilers that do not see kernels inside conditional graph nodes)")
    a = ap.parse_args()

    n1 = a.n
    head_solver = METHODS[a.method].get("solver", "cg")
    workload = f"diffusion3d_{n1}^3_grf_sigma1_len4_{'cg_' if head_solver == 'cg' else ''}{a.method}_tol1e-8"

    def make_config(P):
        return {"workload": workload, "rows": P.n, "nnz": P.nnz, "precision": "fp64", "solver": head_solver,
                "method": a.method, "tol": 1e-8, "formats": "csr+ell32", "l2": "inputs larger than L2 (no flush)",
                "parallelism": f"independent systems x{world}"}

    if a.impl == "reference":
        # No process group, no CUDA: rank 0 alone times the host path, the others exit.
        from alien_b200 import dist
        from oracle import oracle as O

        world, rank, local = dist.ranks()
        if rank != 0:
            return 0
        P = O.problem_diffusion(n1, n1, n1, sigma=1.0, smooth=4.0, seed=rank)
        return reference_main(a, world, rank, P, make_config(P))

    if a.profile_case:
        return profile_case(a)
    world, rank, local = dist_init()
    if a.rowblock:
        return rowblock_main(a, world, rank, local)
    from alien_b200 import abi

    P = abi.diffusion(n1, n1, n1, sigma=1.0, smooth=4.0, seed=rank)
    config = make_config(P)

    import torch

    torch.cuda.set_device(local)
    ctx = abi.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    # CSR + BEllPack-32 as the configuration names them, the FP32 copies for the
    # mixed forms, and the 7-point bands that AUTO then picks for every SpMV
    A = ctx.matrix(P.row_ptr, P.cols, P.vals, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_F32 | abi.FMT_STENCIL)
    b = ctx.vector(P.b)
    x = ctx.vector(P.n)

    def solver_kw(method):
        kw = dict(solver="cg", tol=1e-8, max_iter=a.max_iter, poly_factor=0.0, use_graph=not a.host_loop)
        kw.update(METHODS[method])
        return kw

    kw = solver_kw(a.method)

    def step(kw=kw):
        S = abi.Solver(ctx, A, **kw)
        ctx.assign(x, 0.0)
        st = S.solve(b, x)
        S.close()
        return st

    for _ in range(a.warmup):
        st = step()
    ctx.synchronize()
    launches0 = ctx.launches
    barrier(world)
    torch.cuda.synchronize()
    sts = []
    with Clocks(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            sts.append(step())
        e1.record(stream)
        e1.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    launches = ctx.launches - launches0
    ms = e0.elapsed_time(e1) / a.steps
    ms = max_over_ranks(world, ms)
    st = sts[-1]
    xs = x.download()
    err = float(np.linalg.norm(xs - P.x_true) / np.linalg.norm(P.x_true))

    # Every plain-FP64 method on the same system: one warm + three timed solves each, the median kept.
    methods = {}
    for m in ([] if a.no_methods else sorted(METHODS)):
        mkw = solver_kw(m)
        step(mkw)
        ctx.synchronize()
        runs = []
        for _ in range(3):
            m0 = torch.cuda.Event(enable_timing=True)
            m1 = torch.cuda.Event(enable_timing=True)
            m0.record(stream)
            mst = step(mkw)
            m1.record(stream)
            m1.synchronize()
            runs.append((m0.elapsed_time(m1) / 1e3, mst))
        runs.sort(key=lambda v: v[0])
        s, mst = runs[1]
        methods[m] = {"s": round(s, 5), "iterations": mst.iterations, "converged": bool(mst.succeeded),
                      "true_rel_residual": mst.true_residual, "setup_ms": round(mst.setup_ms, 3),
                      "solve_ms": round(mst.solve_ms, 3),
                      "solver_gbs": round(mst.iterations * iteration_bytes(m, P.n, P.nnz) / (mst.solve_ms * 1e-3)
                                          / 1e9, 1)}

    mixed = None if a.no_mixed else mixed_section(abi, ctx, stream, A, P, b, x, methods, a)
    batched = None if a.no_batch else batch_section(abi, ctx, stream, a)
    learned = None if a.no_learned else learned_section(abi, ctx, stream, a)
    preconds = None if a.no_precond else preconditioner_section(abi, ctx, stream, A, P, a)
    small = None if a.no_small else small_section(abi, ctx, stream, a)
    rowblock = None if (a.no_rowblock or a.method != "ilu0" or world > 1) else \
        rowblock_section(abi, stream, P, xs, st.iterations, a)

    pk, pk_kind = peaks()
    traffic = load_traffic()

    def timed(f, reps):
        for _ in range(3):
            f()
        k0 = torch.cuda.Event(enable_timing=True)
        k1 = torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(reps):
            f()
        k1.record(stream)
        k1.synchronize()
        return k0.elapsed_time(k1) / reps

    def roof(kernel, nbytes, ms, key):
        g = nbytes / (ms * 1e-3) / 1e9
        return {"bound": "hbm", "kernel": kernel, "achieved": round(g, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(g / pk["hbm_gbs"], 4), "peak_source": pk_kind, "algorithmic_bytes": int(nbytes),
                "launch_us": round(ms * 1e3, 2), "traffic": traffic.get(key)}

    # The sliced-ELL SpMV, timed alone with events on the same stream.
    info = A.info
    vy = ctx.vector(P.n)
    spmv_ms = timed(lambda: ctx.mult(A, b, vy, abi.SPMV_ELL), 50)
    ell_roof = roof("k_spmv_ell (sliced ELL-32 FP64 SpMV)", spmv_bytes(info, P.n), spmv_ms, f"spmv_ell_{n1}")
    # the SpMV every solver on this matrix runs (AUTO: the 7-point bands), by its own bytes
    if info.stencil_bands:
        band_ms = timed(lambda: ctx.mult(A, b, vy, abi.SPMV_STENCIL), 50)
        spmv_roof = roof(f"k_spmv_view<StencilView> (7-point bands x{info.stencil_bands}, FP64 SpMV)",
                         info.stencil_bands * 8 * P.n + 16 * P.n, band_ms, f"spmv_bands_{n1}")
        spmv_roof["ell32"] = ell_roof
    else:
        spmv_roof = ell_roof
    achieved = spmv_roof["achieved"]
    variants = None if a.no_variants else spmv_variant_section(abi, ctx, timed, A, P, a)

    # The headline step's dominant kernel: for ILU0 the two triangular sweeps
    # (one precond apply), else the SpMV.
    if METHODS[a.method]["precond"] == "ilu0":
        pc = abi.Precond(ctx, A, "ilu0")
        ilu_ms = timed(lambda: pc.apply(b, vy), 20)
        roofline = roof("k_walk_gather_t + k_walk_sweep_cl<L> + k_walk_sweep_cl<U> + k_walk_scatter_t (ILU0 apply, tile walk in 2x2-tile clusters)",
                        ilu_bytes(P.n, P.nnz), ilu_ms, f"ilu0_apply_{n1}")
        roofline["bytes_formula"] = "B_LU = 12 nnz + 4 (n + 1) + 8 n"
        smin = ilu_stencil_min_bytes(P.n, P.nnz)
        roofline["stencil_min"] = {"bytes": smin, "formula": "8 nnz + 16 n",
                                   "frac": round(smin / (ilu_ms * 1e-3) / 1e9 / pk["hbm_gbs"], 4)}
        pc.close()
    else:
        roofline = spmv_roof

    # End to end through the C ABI from host arrays.
    e2e = None
    if not a.no_e2e:
        h2d = P.row_ptr.nbytes + P.cols.nbytes + P.vals.nbytes + P.b.nbytes
        d2h = P.n * 8

        def pinned(arr):
            t = torch.empty(arr.size, dtype=torch.from_numpy(arr[:1]).dtype, pin_memory=True)
            t.numpy()[:] = arr
            return t

        # the step's inputs and its result live in pinned host memory, as a caller's would
        keep = [pinned(np.ascontiguousarray(v)) for v in (P.row_ptr, P.cols, P.vals, P.b, np.zeros(P.n))]
        rp, ci, vv, bh, xh = (t.numpy() for t in keep)
        t_e2e = []
        for i in range(2):
            torch.cuda.synchronize()
            t = time.perf_counter()
            A2 = ctx.matrix(rp, ci, vv, abi.FMT_CSR | abi.FMT_ELL | abi.FMT_STENCIL)
            b2 = ctx.vector(bh)
            x2 = ctx.vector(P.n)
            S2 = abi.Solver(ctx, A2, **kw)
            S2.solve(b2, x2)
            x2.download(out=xh)
            t_e2e.append(time.perf_counter() - t)
            S2.close(), A2.close(), b2.close(), x2.close()
        v = max_over_ranks(world, min(t_e2e))
        e2e = {"value": round(v, 4), "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "note": "wall clock of matrix upload + set-up + b upload + solve + x download, host arrays "
                       "in pinned memory"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        from oracle import oracle as O

        if O.ref_available():
            v, setup, per_iter, spent = reference_sample(P, a.method, st.iterations)
            _, label = reference_method(a.method)
            cpu = {"value": round(v, 3), "unit": "s", "cores": 1, "kind": "reference", **host_info(),
                   "extrapolated": True,
                   "sample": f"Alien CG.h + {label} (oracle/_ref) on 1 host core: set-up + 2 and 8 "
                             f"iterations of the same system ({spent:.1f} s), scaled to {st.iterations} iterations "
                             f"(set-up {setup:.2f} s, {per_iter*1e3:.1f} ms/iteration); complete solves are timed "
                             f"by --impl reference"}

    cpu_all = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu_all = {m: all_cores_sample(P, m, methods[m]["iterations"]) for m in ("jacobi", "cheb3_saad_power20")
                   if m in methods}

    if rank == 0:
        line = {"metric": "time_to_true_rel_residual_1e-8", "value": round(ms / 1e3, 5), "unit": "s",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms, 3),
                "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded generator, per-rank seed)", "config": config,
                "iterations": st.iterations, "converged": bool(st.succeeded),
                "true_rel_residual": st.true_residual, "rel_error_vs_x_true": err,
                "solution_digest": solution_digest(xs),
                "setup_ms": round(st.setup_ms, 3), "solve_ms": round(st.solve_ms, 3),
                "solver_gbs": round(st.iterations * iteration_bytes(a.method, P.n, P.nnz) / (st.solve_ms * 1e-3)
                                    / 1e9, 1),
                "spmv_gbs": achieved, "roofline": roofline, "spmv_roofline": spmv_roof, "spmv_variants": variants, "methods": methods, "mixed": mixed, "batched": batched,
                "learned": learned, "preconditioners": preconds, "rowblock": rowblock, "small": small,
                "cpu_baseline": cpu, "cpu_all_cores": cpu_all, "e2e": e2e, "gpu_launches": int(launches),
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    from alien_b200 import dist

    dist.finish(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
