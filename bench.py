"""Headline benchmark: Helmholtz solves/s, C192 x 70, to 1e-8, mixed vs FP64.

One step = one complete solve of the seeded C192 x 70 W3 Helmholtz system
(GCR(10) preconditioned by a 4-level multigrid V-cycle, C192/96/48/24,
block-Jacobi column smoother 2+2 sweeps) from a zero initial guess to a
relative FP64 residual of 1e-8, in the mixed-precision form (FP32 inner
GCR + multigrid, FP64 residual and refinement).  The plain FP64 solve is
timed beside it.  Inputs (operators, right-hand side) are resident in HBM;
the e2e figure adds, every step, the host->device copy of the right-hand
side from pinned host memory and the device->host copy of the solution,
through the C ABI.

--impl reference times the CPU restatement of the same solver (the oracle;
the Fortran reference cannot be compiled here) on the host cores.

Multi-GPU: the path does not shard (the whole mesh is resident on one GPU);
--gpus N runs N independent replicas and reports their total throughput.
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

METRIC = "Helmholtz solves/s C192x70L to 1e-8: mixed vs FP64 on 1 B200; HBM GB/s"
N_FINE, NLAYERS, MG_LEVELS, SEED = 192, 70, 4, 3
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lfg", choices=["lfg", "reference"])
    ap.add_argument("--n", type=int, default=N_FINE, help=argparse.SUPPRESS)
    # profiling aids: only the batched workload, at a chosen size and launch shape
    ap.add_argument("--batched-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--kernels", action="store_true", help=argparse.SUPPRESS)
    # small cases for ncu captures of one kernel family
    ap.add_argument("--case", choices=["lma", "coarse", "cma"], help=argparse.SUPPRESS)
    ap.add_argument("--batch-rhs", type=int, default=64, help=argparse.SUPPRESS)
    ap.add_argument("--batch-uneven", type=int, default=32, help=argparse.SUPPRESS)
    ap.add_argument("--batch-shape", type=int, nargs=2, default=(0, 0), help=argparse.SUPPRESS)
    return ap.parse_args()


def max_over_ranks(value: float, world: int, device: str = "cuda") -> float:
    """The largest value over all ranks (device times are reported as the
    slowest rank's); the identity on one rank."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx, self.rows, self.proc = gpu_index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi takes a few hundred ms to start: wait for its first
            # row so that the samples cover the timed region from its start
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 5.0:
                time.sleep(0.01)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[4 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def measured_hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


_CPU = {}


def cpu_oracle(n: int):
    """The seeded C_n x 70 problem and the oracle's view of it on the -O3
    -march=native -fopenmp build (built on this host); set-up is not timed."""
    from lfric_core_b200.problems import helmholtz_problem
    from oracle.oracle import Helmholtz as OraHelm
    if n not in _CPU:
        p = helmholtz_problem(n, NLAYERS, seed=SEED, mg_levels=MG_LEVELS)
        _CPU[n] = (p, OraHelm(p, native=True))
    return _CPU[n]


def cpu_solve(n: int, threads: int, form: str = "mixed"):
    """One complete solve of the C_n x 70 system by the oracle on `threads`
    OpenMP threads, from zero to 1e-8: the mixed form (FP32 inner GCR(10) +
    multigrid, FP64 refinement) or the plain FP64 GCR(10) + multigrid.
    Returns (seconds, threads used)."""
    p, ora = cpu_oracle(n)
    used = ora.L.ora_threads(threads)
    t0 = time.perf_counter()
    if form == "mixed":
        _, st, _ = ora.mixed_solve(p.rhs)
    else:
        _, st, _ = ora.gcr_mg_solve(p.rhs)
    dt = time.perf_counter() - t0
    if st != 0:
        raise RuntimeError(f"CPU {form} solve on C{n} ended with status {st}")
    return dt, used


def cpu_baselines(n: int, n_all: int) -> dict:
    """The CPU path on the full C_n x 70 workload: `n_all` mixed solves and
    one FP64 solve on all host threads, and one mixed solve on one thread."""
    threads = host_threads()
    _, used = cpu_solve(n, threads)                    # first touch of the work arrays
    t_all = [cpu_solve(n, threads)[0] for _ in range(n_all)]
    t64, _ = cpu_solve(n, threads, "fp64")
    t1, _ = cpu_solve(n, 1)
    lib_note = "oracle C restatement built -O3 -march=native -fopenmp on this host"
    return {
        "all_threads": {"value": n_all / sum(t_all), "unit": "solves/s", "cores": used,
                        "sample": f"{n_all} mixed solves on C{n}x{NLAYERS}, {used} OpenMP threads "
                                  f"({lib_note}), {sum(t_all):.1f} s"},
        "fp64_all_threads": {"value": 1.0 / t64, "unit": "solves/s", "cores": used,
                             "sample": f"1 FP64 GCR(10)+MG solve on C{n}x{NLAYERS}, "
                                       f"{used} threads, {t64:.1f} s"},
        "one_thread": {"value": 1.0 / t1, "unit": "solves/s", "cores": 1,
                       "sample": f"1 mixed solve on C{n}x{NLAYERS}, 1 thread, {t1:.1f} s"},
    }


def run_reference(args, rank, world):
    """CPU reference arm: rank 0 alone times the oracle's mixed solve on the
    full C192 x 70 workload on all host threads (the Fortran reference
    cannot be compiled here, so the restatement stands in for it)."""
    if rank != 0:
        return
    threads = host_threads()
    for _ in range(args.warmup):
        cpu_solve(args.n, threads)
    times, used = [], threads
    for _ in range(args.steps):
        dt, used = cpu_solve(args.n, threads)
        times.append(dt)
    t = float(np.sum(times))
    value = args.steps / t
    t1, _ = cpu_solve(args.n, 1)
    sample = (f"one full mixed solve per step on C{args.n}x{NLAYERS} (oracle C restatement built "
              f"-O3 -march=native -fopenmp on this host, {used} OpenMP threads)")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"helmholtz_c{args.n}x{NLAYERS}_gcr10_mg{MG_LEVELS}_mixed_to_1e-8",
                   "sample": f"C{args.n}x{NLAYERS}"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": used, "kind": "port",
                         "sample": sample},
        "one_thread": {"value": 1.0 / t1, "unit": "solves/s", "cores": 1,
                       "sample": f"1 mixed solve on C{args.n}x{NLAYERS}, 1 thread, {t1:.1f} s"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measure_batched(ctx, stream, steps: int, warmup: int, n_rhs: int = 64, n_uneven: int = 32,
                    shape=(0, 0), world: int = 1) -> dict:
    """The batched workload: 64 seeded right-hand sides on one C48 x 30
    operator plus 32 problems with n in 12..96 and 10..70 levels, all solved
    to 1e-8 in one persistent launch (lfg_batch_*).  Device-resident timing
    replays the captured graph; e2e adds every problem's host->device rhs
    copy and device->host solution copy (pinned buffers) to each step."""
    import torch
    from lfric_core_b200 import api
    from lfric_core_b200.problems import batch_workload
    wl = batch_workload(n_rhs=n_rhs, n_uneven=n_uneven)
    ops = [api.Helmholtz(ctx, api.R_DOUBLE, api.Mesh(ctx, p.links), p.nlayers, p.cm, p.hf)
           for p in wl.operators]
    B = api.BatchedHelmholtz(ctx, [ops[j] for j in wl.problem_op], tile_cols=shape[0],
                             blocks_per_sm=shape[1])
    rhs_f, sol_f = B.rhs, B.sol
    rhs_views = [rhs_f[i] for i in range(len(B))]
    sol_views = [sol_f[i] for i in range(len(B))]
    pinned_b = [torch.from_numpy(np.ascontiguousarray(r)).pin_memory().numpy() for r in wl.rhs]
    pinned_x = [torch.empty(r.size, dtype=torch.float64).pin_memory().numpy() for r in wl.rhs]
    for v, r in zip(rhs_views, pinned_b):
        v.import_(r)
    B.solve()                                   # autotune + graph capture
    for _ in range(warmup):
        B.launch()
    B.wait()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = ctx.kernel_launches()
    e0.record(stream)
    for _ in range(steps):
        B.launch()
    e1.record(stream)
    nfailed = B.wait()
    launches = (ctx.kernel_launches() - n0) / steps
    ms = max_over_ranks(e0.elapsed_time(e1), world) / steps
    res = [B.result(i) for i in range(len(B))]

    def e2e_step():
        for v, r in zip(rhs_views, pinned_b):
            v.import_(r)
        B.launch()
        B.wait()
        for v, x in zip(sol_views, pinned_x):
            v.export_into(x)

    e2e_step()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), world) / steps
    # algorithmic bytes per problem dof: RESID 96 (FP64 x, b, operator; FP32
    # r, e, z written, sub, inv, c' read), APPLY 44, UPDATE 40, CORRECT 20
    nbytes = 0.0
    for i, r in enumerate(res):
        op = wl.operators[wl.problem_op[i]]
        n = op.ncol * op.nlayers
        nbytes += n * (96 * (r.outer_iterations + 1) + 84 * r.inner_iterations
                       + 20 * r.outer_iterations)
    # the same with each operator's arrays counted once per phase for all the
    # problems that share it (operator bytes per dof: RESID 68 = FP64 bands
    # and couplings + FP32 sub, inv, c'; APPLY 28 = FP32 bands and
    # couplings; UPDATE 12 = FP32 sub, inv, c'; the rest are vector bytes)
    nbytes_shared = 0.0
    by_op = {}
    for i, r in enumerate(res):
        op = wl.operators[wl.problem_op[i]]
        n = op.ncol * op.nlayers
        nbytes_shared += n * (28 * (r.outer_iterations + 1) + 44 * r.inner_iterations
                              + 20 * r.outer_iterations)
        g = by_op.setdefault(wl.problem_op[i], [n, 0, 0])
        g[1] = max(g[1], r.outer_iterations + 1)
        g[2] = max(g[2], r.inner_iterations)
    for n, resid_phases, inner in by_op.values():
        nbytes_shared += n * (68 * resid_phases + 40 * inner)
    tune = B.tuning()
    return {
        "workload": f"{n_rhs} rhs on C48x30 + {n_uneven} problems n~U{{12..96}}, "
                    f"L~U{{10..70}} (seeds 5+i), mixed CG + column solve to 1e-8",
        "problems": len(B), "ndof": wl.ndof, "ms_per_batch": ms,
        "problems_per_s": len(B) / (ms * 1e-3), "nfailed": nfailed,
        "max_rel_residual": max(r.rel_residual for r in res),
        "outer": sorted({r.outer_iterations for r in res}),
        "inner_min_max": [min(r.inner_iterations for r in res),
                          max(r.inner_iterations for r in res)],
        "gpu_launches_per_batch": launches, "tuning": tune,
        "algorithmic_bytes": nbytes, "algorithmic_GB/s": nbytes / (ms * 1e-3) / 1e9,
        "bytes_note": "each problem's own operator counted; the 64 right-hand sides share "
                      "one C48x30 operator that stays in L2",
        "algorithmic_bytes_shared_operator_once": nbytes_shared,
        "algorithmic_GB/s_shared_operator_once": nbytes_shared / (ms * 1e-3) / 1e9,
        "e2e": {"ms_per_batch": ms_e2e, "problems_per_s": len(B) / (ms_e2e * 1e-3),
                "h2d_bytes_per_step": wl.ndof * 8, "d2h_bytes_per_step": wl.ndof * 8},
    }


def _cpu_time(fn, threads: int, lib, reps: int = 1) -> float:
    """Seconds per call of fn() on `threads` OpenMP threads (mean of reps)."""
    lib.ora_threads(threads)
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    return (time.perf_counter() - t0) / reps


def measure_configs(ctx, stream, steps: int, peak: float, cpu: bool) -> dict:
    """The other workloads, each GPU figure beside the oracle's CPU time
    (the -O3 -march=native -fopenmp build, all host threads and one thread):
    config1_cg_w0, config2_line_solve, config4_adjoint and the CPU side of
    the batched workload."""
    import torch
    from lfric_core_b200 import api
    from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field, field_from
    from lfric_core_b200.problems import w0_problem, helmholtz_problem, batch_workload
    threads = host_threads()
    out = {}

    def gpu_ms(fn, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def gpu_ms_cold(fn, n):
        """Each launch timed alone after a 256 MB read has replaced L2 (for
        inputs smaller than L2; a read leaves no dirty lines for the timed
        launch to write back)."""
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(n)]
        sink = torch.empty((), dtype=torch.int64, device="cuda")
        for a, b in ev:
            sink.copy_(flush_buf.sum(dtype=torch.int64))
            a.record(stream)
            fn()
            b.record(stream)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in ev) / n

    # ---- config 1: C24 x 20 W0 mass + stiffness, Jacobi-CG FP64 to 1e-8
    p = w0_problem(24, 20, seed=1, top=20e3)
    A = p.matrix()
    nent, nlev = p.nvert, p.nlayers + 1
    lma = api.LocalOperator(ctx, R_DOUBLE, p.ncell, p.nlayers, A, p.map, nent, nlev)
    diag = Field(ctx, R_DOUBLE, nent, nlev)
    lma.diagonal(diag)
    sol = api.IterativeSolver(api.LinearOperator.from_lma(lma), api.Preconditioner.diagonal(diag),
                              diag, "cg", r_tol=1e-8, max_iter=2000)
    B, X = field_from(ctx, p.rhs, nent, nlev), Field(ctx, R_DOUBLE, nent, nlev)
    res = {}

    def cg_once():
        X.set_scalar(0.0)
        res["r"] = sol.apply(X, B)

    for _ in range(3):
        cg_once()
    ms = gpu_ms(cg_once, max(5, steps))
    c1 = {"workload": "C24x20 W0 mass+stiffness (kappa 1), Jacobi-preconditioned CG FP64 to 1e-8",
          "ndof": p.ndof, "iterations": res["r"].iterations, "ms_per_solve": ms,
          "solves_per_s": 1e3 / ms,
          "note": "the reference's monitor_convergence tests the residual norm after every "
                  "iteration; the solver reads the norms of 8 iterations at a time (the "
                  "batch replayed from a CUDA graph) and rolls x back to the one that "
                  "converged (same iterations and bits); about 8 small kernels per "
                  "iteration: latency-bound at this size"}
    if cpu:
        from oracle.oracle import W0 as OraW0
        o = OraW0(p, A, native=True)
        o.cg_solve(p.rhs)
        t_all = _cpu_time(lambda: o.cg_solve(p.rhs), threads, o.L, 5)
        t_one = _cpu_time(lambda: o.cg_solve(p.rhs), 1, o.L, 5)
        c1["cpu"] = {"all_threads": {"solves_per_s": 1 / t_all, "cores": threads},
                     "one_thread": {"solves_per_s": 1 / t_one, "cores": 1},
                     "kind": "port", "sample": "5 solves each; the LMA apply (GH_INC scatter) "
                                               "runs serially in the restatement"}
    out["config1_cg_w0"] = c1
    del sol, lma, diag, B, X

    # ---- config 2: C96 x 70 CMA tridiagonal line solve, FP64 and FP32 + FP64 refinement
    p = helmholtz_problem(96, NLAYERS, seed=2, mg_levels=1)
    ncol, nl = p.ncol, p.nlayers
    n = ncol * nl
    ind = np.arange(1, nl + 1, dtype=np.int32)
    A64 = api.ColumnwiseOperator(ctx, R_DOUBLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, p.cm)
    A32 = api.ColumnwiseOperator(ctx, R_SINGLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind, p.cm)
    B = field_from(ctx, p.rhs, ncol, nl)
    X, X2, R = (Field(ctx, R_DOUBLE, ncol, nl) for _ in range(3))
    R32, E32 = Field(ctx, R_SINGLE, ncol, nl), Field(ctx, R_SINGLE, ncol, nl)
    nref = 3

    def refine():
        # FP32 Thomas on the residual, FP64 update and residual (nref corrections)
        X2.set_scalar(0.0)
        R.copy(B)
        for _ in range(nref):
            R32.copy(R)
            A32.apply_inverse(E32, R32)
            X2.axpy(1.0, E32)
            R.copy(B)
            R.scale(-1.0)
            A64.apply(R, X2)
            R.scale(-1.0)

    for _ in range(3):
        A64.apply_inverse(X, B)
        refine()
    ms64 = gpu_ms_cold(lambda: A64.apply_inverse(X, B), 20)
    B32 = Field(ctx, R_SINGLE, ncol, nl)
    B32.copy(B)
    ms32 = gpu_ms_cold(lambda: A32.apply_inverse(E32, B32), 20)
    msref = gpu_ms(refine, 10)
    x64, xr = X.export(), X2.export()
    # the same solves back to back, as the per-kernel rows are timed: four
    # copies of the system taken in turn (310 MB FP32, 620 MB FP64), so
    # each launch's arrays were last touched three launches before and come
    # from HBM, with no flush between the launches
    rot = []
    for _ in range(4):
        b64r = field_from(ctx, p.rhs, ncol, nl)
        b32r = Field(ctx, R_SINGLE, ncol, nl)
        b32r.copy(b64r)
        rot.append((api.ColumnwiseOperator(ctx, R_DOUBLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind,
                                           p.cm), Field(ctx, R_DOUBLE, ncol, nl), b64r,
                    api.ColumnwiseOperator(ctx, R_SINGLE, ncol, nl, nl, 3, 1, 1, 1, 1, ind, ind,
                                           p.cm), Field(ctx, R_SINGLE, ncol, nl), b32r))

    def rot64():
        for a, x, b, *_ in rot:
            a.apply_inverse(x, b)

    def rot32():
        for *_, a, x, b in rot:
            a.apply_inverse(x, b)

    for _ in range(3):
        rot64()
        rot32()
    ms64b = gpu_ms(rot64, 5) / len(rot)
    ms32b = gpu_ms(rot32, 5) / len(rot)
    assert np.array_equal(rot[0][1].export(), x64)
    del rot
    c2 = {"workload": "C96x70 W3 tridiagonal (diagonal ratio U(1.5,3)), seeded rhs; solves "
                      "timed alone after an L2-replacing read, and back to back over four "
                      "copies of the system (inputs larger than L2)",
          "ndof": n,
          "fp64_solve": {"us": ms64 * 1e3, "algorithmic_bytes": 5 * n * 8,
                         "GB/s": 5 * n * 8 / (ms64 * 1e-3) / 1e9,
                         "frac": 5 * n * 8 / (ms64 * 1e-3) / 1e9 / peak},
          "fp32_solve": {"us": ms32 * 1e3, "algorithmic_bytes": 5 * n * 4,
                         "GB/s": 5 * n * 4 / (ms32 * 1e-3) / 1e9,
                         "frac": 5 * n * 4 / (ms32 * 1e-3) / 1e9 / peak},
          "fp64_solve_back_to_back": {"us": ms64b * 1e3,
                                      "frac": 5 * n * 8 / (ms64b * 1e-3) / 1e9 / peak},
          "fp32_solve_back_to_back": {"us": ms32b * 1e3,
                                      "frac": 5 * n * 4 / (ms32b * 1e-3) / 1e9 / peak},
          "fp32_plus_fp64_refinement": {
              "us": msref * 1e3, "corrections": nref,
              "rel_diff_to_fp64": float(np.linalg.norm(xr - x64) / np.linalg.norm(x64))}}
    if cpu:
        from oracle.oracle import lib as olib, ptr
        L = olib(True)
        cmc = np.ascontiguousarray(p.cm)
        cm32 = cmc.astype(np.float32)
        b64 = np.ascontiguousarray(p.rhs)
        b32 = b64.astype(np.float32)
        y64, y32 = np.zeros(n), np.zeros(n, dtype=np.float32)
        f64 = lambda: L.ora_cma_appinv_mesh_d(ncol, nl, ptr(cmc), ptr(b64), ptr(y64))
        f32 = lambda: L.ora_cma_appinv_mesh_f(ncol, nl, ptr(cm32), ptr(b32), ptr(y32))
        f64()
        c2["cpu"] = {"fp64_solve": {"all_threads_us": 1e6 * _cpu_time(f64, threads, L, 10),
                                    "one_thread_us": 1e6 * _cpu_time(f64, 1, L, 5)},
                     "fp32_solve": {"all_threads_us": 1e6 * _cpu_time(f32, threads, L, 10),
                                    "one_thread_us": 1e6 * _cpu_time(f32, 1, L, 5)},
                     "cores": threads, "kind": "port",
                     "sample": "columnwise_op_appinv over all 55296 columns, 10 (all threads) "
                               "and 5 (one thread) calls"}
    out["config2_line_solve"] = c2
    del A64, A32, B, X, X2, R, R32, E32, B32

    # ---- config 4: gradients of J = 0.5 ||u - u_obs||^2 through the C48 x 30
    # W0 diffusion solve (log-normal kappa, sigma 0.5), FP64, solves to 1e-13
    from lfric_core_b200.autograd import DiffusionSolve, W0Diffusion
    p = w0_problem(48, 30, seed=4, top=30e3, kappa_sigma=0.5, kappa_scale=1e6)
    nl = p.nlayers
    sysm = W0Diffusion(ctx, p, r_tol=1e-13, max_iter=5000)
    dev = torch.device("cuda")
    lm = lambda a, nc_, nv_: torch.tensor(np.ascontiguousarray(
        np.asarray(a).reshape(nc_, nv_).T), dtype=torch.float64, device=dev).reshape(-1)
    f = lm(p.rhs, p.nvert, nl + 1)
    kap = lm(p.kappa.ravel(), p.ncell, nl)
    rng = np.random.default_rng(7)
    with torch.no_grad():
        u_nom = DiffusionSolve.apply(f, kap, sysm)
        uobs = u_nom + 0.1 * u_nom.std() * torch.tensor(rng.standard_normal(p.ndof),
                                                        dtype=torch.float64, device=dev)

    def forward():
        with torch.no_grad():
            return DiffusionSolve.apply(f, kap, sysm)

    def gradient():
        ff, kk = f.clone().requires_grad_(True), kap.clone().requires_grad_(True)
        u = DiffusionSolve.apply(ff, kk, sysm)
        (0.5 * torch.sum((u - uobs) ** 2)).backward()
        return ff.grad, kk.grad

    def fd16():
        h = 1e-6
        for _ in range(16):
            with torch.no_grad():
                DiffusionSolve.apply(f + h * f, kap, sysm)
                DiffusionSolve.apply(f - h * f, kap, sysm)

    def host_ms(fn, n):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / n

    for _ in range(2):
        forward()
        gradient()
    fwd_ms = host_ms(forward, 3)
    grad_ms = host_ms(gradient, 3)
    fd_ms = host_ms(fd16, 1)
    c4 = {"workload": "C48x30 W0 diffusion, log-normal kappa (sigma 0.5), CG to 1e-13, "
                      "gradient of J w.r.t. rhs and kappa",
          "ndof": p.ndof, "forward_solve_ms": fwd_ms,
          "adjoint_gradient_ms": grad_ms, "fd_16_directions_ms": fd_ms,
          "gradient_over_forward": grad_ms / fwd_ms, "fd_over_gradient": fd_ms / grad_ms,
          "note": "timed on the host clock around device-synchronised calls (the solves read "
                  "their residual norms on the host)"}
    if cpu:
        from oracle.oracle import W0 as OraW0
        o = OraW0(p, native=True)
        t1 = _cpu_time(lambda: o.cg_solve(p.rhs, r_tol=1e-13, max_iter=5000), threads, o.L, 1)
        c4["cpu"] = {"forward_solve_s": t1, "fd_16_directions_s": 32 * t1,
                     "cores": threads, "kind": "port",
                     "sample": "one Jacobi-CG forward solve timed; the central-difference "
                               "gradient over 16 directions costs 32 such solves"}
    out["config4_adjoint"] = c4
    del sysm
    ctx.set_stream(stream.cuda_stream)        # W0Diffusion ran the library on its own stream

    # ---- config 5, CPU side: the oracle's refinement + CG + column solve on a sample
    if cpu:
        from oracle.oracle import Helmholtz as OraHelm
        wl = batch_workload()
        pick = [0, 1, 2, 3] + [64 + j for j in range(4)]
        ndof, t = 0, 0.0
        L = None
        for i in pick:
            op = wl.operators[wl.problem_op[i]]
            o = OraHelm(op, native=True)
            L = o.L
            L.ora_threads(threads)
            t0 = time.perf_counter()
            _, st, _ = o.mixed_cg_col_solve(wl.rhs[i])
            t += time.perf_counter() - t0
            ndof += op.ncol * op.nlayers
        out["config5_batched_cpu"] = {
            "problems": len(pick), "ndof": ndof, "seconds": t, "Mdof_per_s": ndof / t / 1e6,
            "problems_per_s": len(pick) / t, "cores": threads, "kind": "port",
            "sample": "problems 0-3 (C48x30, shared operator) and 64-67 (uneven) of the "
                      "batched workload, one after another, each on all threads"}
    return out


def cma_assembly_cases(ctx):
    """The CMA assembly and product workloads on C96 x 70 columns, FP64
    (columnwise_op_asm W3 <- Wtheta, columnwise_op_mul Wtheta <- W3 <-
    Wtheta, columnwise_op_asm_diag_hmht on W3, columnwise_op_asm_m2v_lumped_inv
    on W2v): a list of (kernel label, call, algorithmic bytes of one call)."""
    from lfric_core_b200 import api
    from lfric_core_b200.api import R_DOUBLE
    from lfric_core_b200.problems import banded_dofmap, cma_prod_size, cma_size
    ncell, nl, w = 6 * 96 * 96, NLAYERS, 8
    rng = np.random.default_rng(6)
    p3t = cma_size(nl, 1, 2, 0, 1, 1, 0)           # W3 <- Wtheta
    pt3 = cma_size(nl, 2, 1, 1, 0, 0, 1)           # Wtheta <- W3
    ptt = cma_prod_size(pt3, p3t)                  # Wtheta <- Wtheta
    ls = rng.standard_normal((ncell * nl, 1, 2))
    mt = np.array([[c * nl] for c in range(ncell)])            # W3 dofmap, (cell, 1)
    mf = np.array([[c * (nl + 1), c * (nl + 1) + 1] for c in range(ncell)])  # Wtheta, (cell, 2)
    lma = api.LocalOperator(ctx, R_DOUBLE, ncell, nl, np.asfortranarray(ls).ravel(order="F"),
                            mt, ncell, nl, mf, ncell, nl + 1)

    def cma(pp, bands=None):
        return api.ColumnwiseOperator(ctx, R_DOUBLE, ncell, pp["nrow"], pp["ncol"], pp["bw"],
                                      pp["alpha"], pp["beta"], pp["gm"], pp["gp"],
                                      np.arange(1, pp["nrow"] + 1), np.arange(1, pp["ncol"] + 1),
                                      bands)
    cases = []
    A = cma(p3t)
    cb_to, cb_from = banded_dofmap(nl, 1, 1, 0), banded_dofmap(nl, 2, 0, 1)
    cases.append(("k_cma_asm_rows (columnwise_op_asm, W3 <- Wtheta)",
                  lambda: A.assemble(lma, cb_to, cb_from),
                  (ncell * nl * 2 + p3t["bw"] * p3t["nrow"] * ncell) * w))
    At = cma(pt3, rng.standard_normal((pt3["bw"], pt3["nrow"], ncell)).ravel(order="F"))
    Bt = cma(p3t, rng.standard_normal((p3t["bw"], p3t["nrow"], ncell)).ravel(order="F"))
    Ct = cma(ptt, np.zeros((ptt["bw"], ptt["nrow"], ncell)).ravel(order="F"))
    cases.append(("k_cma_mul_u (columnwise_op_mul, Wtheta <- W3 <- Wtheta, C += A B)",
                  lambda: Ct.multiply(At, Bt),
                  (pt3["bw"] * pt3["nrow"] + p3t["bw"] * p3t["nrow"] + 2 * ptt["bw"] * ptt["nrow"])
                  * ncell * w))
    # diag(Dh M2h^-1 Dh^T) on W3 (columnwise_op_asm_diag_hmht) and the lumped
    # inverse of a W2v mass matrix (columnwise_op_asm_m2v_lumped_inv)
    p33 = cma_size(nl, 1, 1, 0, 1, 0, 1)
    dh_ls = rng.standard_normal((ncell * nl, 1, 4))
    m2h_ls = rng.standard_normal((ncell * nl, 4, 4))
    for d in range(4):
        m2h_ls[:, d, d] = 1.0 + rng.random(ncell * nl)
    m3 = np.array([[c * nl] for c in range(ncell)])
    m2h_map = np.array([[(c * 4 + d) * nl for d in range(4)] for c in range(ncell)])
    Dh = api.LocalOperator(ctx, R_DOUBLE, ncell, nl, np.asfortranarray(dh_ls).ravel(order="F"),
                           m3, ncell, nl, m2h_map, ncell * 4, nl)
    M2h = api.LocalOperator(ctx, R_DOUBLE, ncell, nl,
                            np.asfortranarray(m2h_ls).ravel(order="F"), m2h_map, ncell * 4, nl,
                            m2h_map, ncell * 4, nl)
    Hc = cma(p33)
    cb3 = banded_dofmap(nl, 1, 1, 0)
    cases.append(("k_cma_hmht_rows (columnwise_op_asm_diag_hmht, W3)",
                  lambda: Hc.assemble_diag_hmht(Dh, M2h, cb3),
                  (ncell * nl * (4 + 4) + p33["bw"] * p33["nrow"] * ncell) * w))
    pvv = cma_size(nl, 2, 2, 1, 0, 1, 0)
    mv_ls = np.abs(rng.standard_normal((ncell * nl, 2, 2))) + 0.1
    mvm = np.array([[c * (nl + 1), c * (nl + 1) + 1] for c in range(ncell)])
    Mv = api.LocalOperator(ctx, R_DOUBLE, ncell, nl, np.asfortranarray(mv_ls).ravel(order="F"),
                           mvm, ncell, nl + 1, mvm, ncell, nl + 1)
    Lc = cma(pvv)
    cbv = banded_dofmap(nl, 2, 0, 1)
    cases.append(("k_cma_asm_rows<inverse> (columnwise_op_asm_m2v_lumped_inv, W2v)",
                  lambda: Lc.assemble_m2v_lumped_inv(Mv, cbv),
                  (ncell * nl * 2 + pvv["bw"] * pvv["nrow"] * ncell) * w))
    return cases


def measure_next_rows(ctx, stream, peak: float, cpu: bool) -> dict:
    """The rows past the hot path (their parity is tested in tests/), timed
    on the GPU beside the oracle where it runs whole solves: the Krylov
    variants with the multigrid preconditioner on the C96 x 70 Helmholtz
    problem (FP64, to 1e-8), GCR(10) with the W2 (vector-space) multigrid on
    a C48 x 4 W2 hierarchy, and the CMA assembly and product kernels on
    C96 x 70 columns (GPU only: the oracle restates them one column per
    call)."""
    import ctypes as C
    import torch
    from lfric_core_b200 import api
    from lfric_core_b200.problems import helmholtz_problem, w2_hierarchy
    threads = host_threads()
    out = {}

    def host_ms(fn, reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps * 1e3

    # ---- Krylov variants (sci_iterative_solver_mod.f90:645-1940)
    p = helmholtz_problem(96, NLAYERS, seed=SEED, mg_levels=3)
    S = api.HelmholtzSystem(ctx, p, mixed=False)
    B, X = S.op64.field(p.rhs), S.op64.field()
    kry = {"workload": "C96x70 W3 Helmholtz, FP64, 3-level multigrid preconditioner, "
                       "r_tol 1e-8, restart length 10, x0 = 0", "ndof": p.ndof}
    for method in ("gcr", "bicgstab", "gmres", "fgmres"):
        sol = api.IterativeSolver(api.LinearOperator.from_helmholtz(S.op64), S.mg64, S.x64,
                                  method, r_tol=1e-8, max_iter=60, gcrk=10,
                                  fail_on_non_converged=False)
        res = {}

        def run():
            X.set_scalar(0.0)
            res["r"] = sol.apply(X, B)
        run()
        ms = host_ms(run, 3)
        kry[method] = {"ms_per_solve": ms, "iterations": res["r"].iterations,
                       "final_err": res["r"].final_err, "status": res["r"].status}
    if cpu:
        from oracle.oracle import Helmholtz as OraHelm, SolveInfo, ptr
        ora = OraHelm(p, native=True)
        L = ora.L
        op, mg = ora.op(0), ora.mg(nlevels=3)
        n = p.ndof
        b = np.ascontiguousarray(p.rhs)
        cb_a = C.cast(L.ora_helm_apply_cb_d, C.c_void_p)
        cb_p = C.cast(L.ora_mg_apply_cb_d, C.c_void_p)
        cpu_k = {"cores": threads, "kind": "port",
                 "sample": "one solve each on all threads (-O3 -march=native -fopenmp build)"}
        for method in ("bicgstab", "gmres"):
            x = np.zeros(n)
            info = SolveInfo()
            if method == "bicgstab":
                work = np.zeros(8 * n)
                fn = lambda: L.ora_bicgstab_solve_d(n, cb_a, C.byref(op), cb_p, C.byref(mg),
                                                    1e-8, 0.0, 60, 1, ptr(x), ptr(b), ptr(work),
                                                    C.byref(info))
            else:
                work = np.zeros(25 * n)
                fn = lambda: L.ora_gmres_solve_d(n, cb_a, C.byref(op), cb_p, C.byref(mg), 10,
                                                 1e-8, 0.0, 60, 1, ptr(x), ptr(b), ptr(work),
                                                 C.byref(info))
            sec = _cpu_time(fn, threads, L)
            cpu_k[method] = {"ms_per_solve": sec * 1e3, "iterations": info.iterations}
        kry["cpu"] = cpu_k
    out["krylov_variants"] = kry
    del S, B, X

    # ---- GCR(10) with the W2 multigrid (sci_hierarchical_preconditioner_mod.f90:22-38)
    H = w2_hierarchy(48, 4, 3, seed=1, top=4e5, tau=1e9, radius=1.2742e6)
    W = api.W2System(ctx, H)
    sol = api.IterativeSolver(api.LinearOperator.from_lma(W.ops[0]), W.prec, W.field(), "gcr",
                              r_tol=1e-8, max_iter=100, gcrk=10)
    Bw, Xw = W.field(H.rhs), W.field()
    res = {}

    def run_w2():
        Xw.set_scalar(0.0)
        res["r"] = sol.apply(Xw, Bw)
    run_w2()
    w2 = {"workload": "C48x4 W2 (RT0 mass + div-div, tau 1e9, radius 1.2742e6 m), 3-level W2 "
                      "multigrid (weighted Jacobi 2+2, 8 coarse), GCR(10) to 1e-8",
          "ndof": int(H.levels[0].flat_ndof), "ms_per_solve": host_ms(run_w2, 3),
          "iterations": res["r"].iterations}
    if cpu:
        from oracle.oracle import W2Multigrid
        ora2 = W2Multigrid(H, omega=0.6, native=True)
        info2 = {}

        def cpu_w2():
            info2["i"] = ora2.gcr_solve(H.rhs, gcrk=10, r_tol=1e-8, max_iter=100)[2]
        sec = _cpu_time(cpu_w2, threads, ora2.L)
        w2["cpu"] = {"ms_per_solve": sec * 1e3, "iterations": info2["i"].iterations,
                     "cores": threads, "kind": "port",
                     "sample": "one solve on all threads (-O3 -march=native -fopenmp build; "
                               "its LMA applies, GH_INC scatters, run serially)"}
    out["w2_multigrid"] = w2
    del W, sol, Bw, Xw

    # ---- CMA assembly and product on C96 x 70 columns (columnwise_op_asm,
    # columnwise_op_mul; components/science/source/kernel/columnwise_operators)
    def ev_ms(fn, n=10):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    rows = []
    for label, fn, nb in cma_assembly_cases(ctx):
        ms = ev_ms(fn)
        rows.append({"kernel": label, "us": ms * 1e3, "algorithmic_bytes": nb,
                     "frac_of_measured_hbm": nb / (ms * 1e-3) / 1e9 / peak})
    out["cma_assembly"] = {"workload": "C96x70 columns (55,296), FP64", "kernels": rows}
    return out


def measure_kernels(ctx, stream, peak: float) -> list:
    """Every hot-path kernel timed alone (CUDA events on the library's
    stream, 3 warm-up + 20 timed launches, inputs larger than L2 where the
    workload allows) against its algorithmic bytes: each array read once
    and written once at its stored precision."""
    import torch
    from lfric_core_b200 import api
    from lfric_core_b200.api import R_DOUBLE, R_SINGLE, Field
    from lfric_core_b200.problems import helmholtz_problem, w0_problem
    rows = []

    def time(fn, n=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    def add(name, workload, nbytes, ms):
        gbs = nbytes / (ms * 1e-3) / 1e9
        rows.append({"kernel": name, "workload": workload, "algorithmic_bytes": nbytes,
                     "us": ms * 1e3, "GB/s": gbs, "frac_of_measured_hbm": gbs / peak})

    prob = helmholtz_problem(N_FINE, NLAYERS, seed=SEED, mg_levels=2)
    N = prob.ndof
    mesh = api.Mesh(ctx, prob.links)
    ig = api.Intergrid(ctx, prob.mg_child[0], prob.ncol)
    nc = prob.mg_child[0].shape[0]
    for kind, w, tag in ((R_SINGLE, 4, "FP32"), (R_DOUBLE, 8, "FP64")):
        H = api.Helmholtz(ctx, kind, mesh, NLAYERS, prob.cm, prob.hf)
        x, b, y = H.field(), H.field(), H.field()
        x.import_(prob.rhs)
        b.import_(prob.rhs)
        wl = f"C{N_FINE}x{NLAYERS} {tag}"
        # couplings: 2 words per dof for FP64 operators (symmetric, each face
        # read through one side), 4 for FP32 ones (per-side reads)
        hw = 2 if kind == R_DOUBLE else 4
        add("k_helm_apply (y = A x)", wl, (5 + hw) * N * w, time(lambda: H.apply(y, x)))
        add("k_helm_rhs (r = b + H_off x)", wl, (3 + hw) * N * w,
            time(lambda: H.sweep_rhs(x, b, y)))
        Cb = Field(ctx, kind, nc, NLAYERS)
        add("k_helm_resid_restrict (restrict_mass_w3(b - A x))",
            f"C{N_FINE}->C{N_FINE // 2}x{NLAYERS} {tag}", (5 + hw) * N * w + nc * NLAYERS * w,
            time(lambda: H.residual_restrict(ig, x, b, Cb)))
        add("substitution from zero (k_subst_tma_reg)", wl, 5 * N * w,
            time(lambda: H.smooth(0.8, None, b, y)))
        add("smoother sweep (k_helm_rhs + substitution)", wl, (9 + hw) * N * w,
            time(lambda: H.smooth(0.8, x, b, y)))
        add("k_axpy (y = y + a x)", wl, 3 * N * w, time(lambda: y.axpy(0.5, x)))
        add("k_axpby (z = a x + b y)", wl, 3 * N * w, time(lambda: y.axpby(0.5, x, 0.25, b)))
        dres = torch.zeros(1, dtype=torch.float64, device="cuda")
        add("k_dot (<x, y>, FP64 accumulation, result left on the device)", wl, 2 * N * w,
            time(lambda: x.dot_into(b, dres.data_ptr())))
        del H, x, b, y, Cb
    # intergrid C192 -> C96 (FP64): restrict_mass_w3 and prolong_scalar_unweighted
    F = Field(ctx, R_DOUBLE, prob.ncol, NLAYERS)
    Cc = Field(ctx, R_DOUBLE, nc, NLAYERS)
    F.set_scalar(1.0)
    Cc.set_scalar(1.0)
    add("k_restrict (restrict_mass_w3)", f"C{N_FINE}->C{N_FINE // 2}x{NLAYERS} FP64",
        (N + nc * NLAYERS) * 8, time(lambda: ig.restrict(api.RESTRICT_MASS_W3, Cc, F)))
    add("k_prolong (prolong_scalar_unweighted)", f"C{N_FINE // 2}->C{N_FINE}x{NLAYERS} FP64",
        (2 * N + nc * NLAYERS) * 8, time(lambda: ig.prolong(F, Cc)))
    # CMA tridiagonal (W3 -> W3) app and appinv on C192 x 70, whose arrays
    # are larger than L2 (the C96 line solve of config 2 is timed with L2
    # replaced before each launch in the bench line)
    ncma = 6 * N_FINE * N_FINE
    rng = np.random.default_rng(2)
    sub = -rng.random((ncma, NLAYERS))
    sup = -rng.random((ncma, NLAYERS))
    diag = (np.abs(sub) + np.abs(sup)) * (1.5 + 1.5 * rng.random((ncma, NLAYERS)))
    cm = np.stack([sub, diag, sup], axis=-1).ravel()
    ind = np.arange(1, NLAYERS + 1)
    for kind, w, tag in ((R_DOUBLE, 8, "FP64"), (R_SINGLE, 4, "FP32")):
        A = api.ColumnwiseOperator(ctx, kind, ncma, NLAYERS, NLAYERS, 3, 1, 1, 1, 1, ind, ind, cm)
        X = Field(ctx, kind, ncma, NLAYERS)
        Y = Field(ctx, kind, ncma, NLAYERS)
        X.set_scalar(1.0)
        Y.set_scalar(0.0)
        n = ncma * NLAYERS
        add("k_cma_app_v (columnwise_op_app)", f"C{N_FINE}x{NLAYERS} {tag}", 6 * n * w,
            time(lambda: A.apply(Y, X)))
        add("k_subst_tma_reg (columnwise_op_appinv)", f"C{N_FINE}x{NLAYERS} {tag}", 5 * n * w,
            time(lambda: A.apply_inverse(Y, X)))
        del A, X, Y
    # LMA W0 apply (matrix_vector, gather form) on the C48 x 30 W0 problem
    wp = w0_problem(48, 30, seed=4, top=30e3)
    L = api.LocalOperator(ctx, R_DOUBLE, wp.ncell, wp.nlayers, wp.matrix(), wp.map, wp.nvert,
                          wp.nlayers + 1)
    X = Field(ctx, R_DOUBLE, wp.nvert, wp.nlayers + 1)
    Y = Field(ctx, R_DOUBLE, wp.nvert, wp.nlayers + 1)
    X.set_scalar(1.0)
    Y.set_scalar(0.0)
    ncell3 = wp.ncell * wp.nlayers
    add("k_lma_local + k_lma_gather_tab (matrix_vector)", "C48x30 W0 FP64",
        (64 * ncell3 + 3 * wp.ndof) * 8, time(lambda: L.apply(api.LMA_INC, Y, X)))
    add("k_lma_local + k_lma_gather_tab (transpose_matrix_vector)", "C48x30 W0 FP64",
        (64 * ncell3 + 3 * wp.ndof) * 8, time(lambda: L.apply(api.LMA_TRANSPOSE, Y, X)))
    return rows


def profile_case(ctx, case: str):
    """A small workload for an ncu capture of one kernel family: "lma" makes
    the C48x30 W0 operator and runs three forward then three transposed
    applies (k_lma_local, k_lma_local_tsplit, k_lma_gather_tab); "coarse"
    makes the C96x70 hierarchy (FP32) and runs four sweeps on its C24 level,
    then four on its C48 level (k_helm_sweep_seg); "cma" runs each of the
    C96 x 70 CMA assembly and product calls three times (k_cma_asm_rows,
    k_cma_mul_u, k_cma_hmht_rows)."""
    from lfric_core_b200 import api
    from lfric_core_b200.api import R_DOUBLE, Field
    from lfric_core_b200.problems import helmholtz_problem, w0_problem
    if case == "lma":
        wp = w0_problem(48, 30, seed=4, top=30e3)
        L = api.LocalOperator(ctx, R_DOUBLE, wp.ncell, wp.nlayers, wp.matrix(), wp.map,
                              wp.nvert, wp.nlayers + 1)
        X = Field(ctx, R_DOUBLE, wp.nvert, wp.nlayers + 1)
        Y = Field(ctx, R_DOUBLE, wp.nvert, wp.nlayers + 1)
        X.set_scalar(1.0)
        Y.set_scalar(0.0)
        for mode in (api.LMA_INC, api.LMA_TRANSPOSE):
            for _ in range(3):
                L.apply(mode, Y, X)
    elif case == "cma":
        for _, fn, _ in cma_assembly_cases(ctx):
            for _ in range(3):
                fn()
    else:
        p = helmholtz_problem(96, NLAYERS, seed=SEED, mg_levels=3)
        S = api.HelmholtzSystem(ctx, p, fp64=False)
        for lev in (S.levels32[2], S.levels32[1]):
            x, b, y = lev.field(), lev.field(), lev.field()
            x.set_scalar(1.0)
            b.set_scalar(1.0)
            for _ in range(4):
                lev.smooth(0.8, x, b, y)
    ctx.synchronize()


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from lfric_core_b200 import api
    from lfric_core_b200.problems import helmholtz_problem

    if args.case:
        ctx = api.Context(dev)
        profile_case(ctx, args.case)
        ctx.close()
        return

    if args.kernels:
        ctx = api.Context(dev)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx.set_stream(stream.cuda_stream)
        peak, kind = measured_hbm_peak()
        rows = measure_kernels(ctx, stream, peak)
        if rank == 0:
            print(json.dumps({"kernels": rows, "peak_GB/s": peak, "peak_source": kind}),
                  flush=True)
        ctx.close()
        return

    if args.batched_only:
        ctx = api.Context(dev)
        stream = torch.cuda.Stream()
        torch.cuda.set_stream(stream)
        ctx.set_stream(stream.cuda_stream)
        out = measure_batched(ctx, stream, args.steps, args.warmup, args.batch_rhs,
                              args.batch_uneven, tuple(args.batch_shape))
        if rank == 0:
            print(json.dumps({"batched": out}), flush=True)
        ctx.close()
        return

    prob = helmholtz_problem(args.n, NLAYERS, seed=SEED + rank, mg_levels=MG_LEVELS)
    ctx = api.Context(dev)
    # one explicit stream for the library's kernels and the timing events
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    system = api.HelmholtzSystem(ctx, prob)
    system.b64.import_(prob.rhs)
    N = prob.ndof

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
            torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0, b0 = ctx.kernel_launches(), ctx.algorithmic_bytes()
        e0.record(stream)
        last = None
        for _ in range(steps):
            last = fn()
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1), world)
        timed.bytes = (ctx.algorithmic_bytes() - b0) / steps
        return ms, ctx.kernel_launches() - n0, last

    # ---- warm-up (both forms)
    for _ in range(args.warmup):
        system.solve_mixed()
        system.solve_fp64()

    b_host = torch.from_numpy(prob.rhs.astype(np.float64)).pin_memory()
    x_host = torch.empty(N, dtype=torch.float64).pin_memory()
    b_np, x_np = b_host.numpy(), x_host.numpy()

    def e2e_step():
        system.b64.import_(b_np)
        r = system.mixed.apply(system.x64, system.b64)
        system.x64.export_into(x_np)
        return r

    e2e_step()
    # the clocks are sampled over the three timed regions
    with ClockSampler(dev) as clk:
        # ---- mixed (headline, device-resident inputs)
        torch.cuda.nvtx.range_push("timed_mixed")
        ms_mixed, launches, res_m = timed(system.solve_mixed, args.steps)
        bytes_mixed = timed.bytes
        torch.cuda.nvtx.range_pop()
        # ---- plain FP64 drop-in
        torch.cuda.nvtx.range_push("timed_fp64")
        ms_fp64, launches64, res_64 = timed(system.solve_fp64, args.steps)
        bytes_fp64 = timed.bytes
        torch.cuda.nvtx.range_pop()
        # ---- e2e through the ABI with host buffers (pinned)
        ms_e2e, _, _ = timed(e2e_step, args.steps)

    # true residual of the last mixed solve, in FP64 on the device
    system.solve_mixed()
    R = system.op64.field()
    system.op64.apply(R, system.x64)
    R.aypx(-1.0, system.b64)
    true_rel = R.norm() / system.b64.norm()

    # ---- roofline of the dominant kernel: the sweep right-hand side
    # r = b + H_off x (k_helm_rhs<float>, the largest single share of the
    # mixed solve's time), on the C192 level, FP32; the substitution from
    # zero (one launch of the TMA substitution) and the whole sweep from a
    # nonzero guess (k_helm_rhs + the substitution) are timed beside it
    op32 = system.levels32[0]
    xs, bs, ys = op32.field(), op32.field(), op32.field()
    xs.copy(system.x64)
    bs.copy(system.b64)
    nrep = 20

    def time_loop(fn):
        for _ in range(3):
            fn(0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(nrep):
            fn(i)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / nrep

    torch.cuda.nvtx.range_push("smoother_roofline")
    rhs_ms = time_loop(lambda i: op32.sweep_rhs(xs, bs, ys))
    subst_ms = time_loop(lambda i: op32.smooth(0.8, None, bs, ys if i % 2 == 0 else xs))
    sweep_ms = time_loop(lambda i: op32.smooth(0.8, xs if i % 2 == 0 else ys, bs,
                                               ys if i % 2 == 0 else xs))
    torch.cuda.nvtx.range_pop()
    rhs_bytes = 7 * N * 4              # x, b, the 4 per-side couplings read; r written
    subst_bytes = 5 * N * 4            # b, sub, inv, c' read; x written (FP32)
    sweep_bytes = 13 * N * 4           # rhs: x, b, 4 couplings, r; subst: r, inv, sub, c', x_in, x
    peak, peak_kind = measured_hbm_peak()
    traffic = {}
    tp = ROOT / "profiles" / "roofline_traffic.json"
    if tp.exists():
        for name, t in json.loads(tp.read_text()).get("kernels", {}).items():
            traffic[name] = t["dram_bytes_per_launch"] * N / t["dofs"]

    # ---- batched persistent solves (every rank: replicas)
    torch.cuda.nvtx.range_push("batched")
    batched = measure_batched(ctx, stream, max(1, args.steps), max(1, args.warmup), world=world)
    torch.cuda.nvtx.range_pop()

    # ---- the other workloads (configs 1, 2 and 4; the CPU side of the batched one)
    torch.cuda.nvtx.range_push("configs")
    configs = measure_configs(ctx, stream, args.steps, measured_hbm_peak()[0],
                              cpu=(rank == 0 and world == 1))
    torch.cuda.nvtx.range_pop()

    # ---- the rows past the hot path (rank 0 only; a minute at most)
    nxt = None
    if rank == 0:
        torch.cuda.nvtx.range_push("next_rows")
        nxt = measure_next_rows(ctx, stream, measured_hbm_peak()[0], cpu=(world == 1))
        torch.cuda.nvtx.range_pop()

    # ---- CPU baseline (rank 0, N=1 only): the oracle on the same workload
    cpu = None
    if rank == 0 and world == 1:
        cb = cpu_baselines(args.n, 3)
        cpu = dict(cb["all_threads"], kind="port", one_thread=cb["one_thread"],
                   fp64_all_threads=cb["fp64_all_threads"])

    value = world * args.steps / (ms_mixed * 1e-3)
    fp64_value = world * args.steps / (ms_fp64 * 1e-3)
    e2e_value = world * args.steps / (ms_e2e * 1e-3)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"helmholtz_c{args.n}x{NLAYERS}_gcr10_mg{MG_LEVELS}_mixed_to_1e-8",
                       "ndof": N, "mg": "C192/96/48/24 block-Jacobi column smoother 2+2, 8 coarse",
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (FP64 operator 0.87 GB, FP32 0.43 GB)"},
            "fp64": {"value": fp64_value, "unit": "solves/s", "ms_per_step": ms_fp64 / args.steps,
                     "iterations": res_64.iterations, "final_err": res_64.final_err,
                     "gpu_launches": launches64},
            "mixed_over_fp64": value / fp64_value,
            "mixed": {"outer": res_m.outer_iterations, "inner": res_m.inner_iterations,
                      "rel_residual": res_m.rel_residual, "true_rel_residual": true_rel},
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": N * 8,
                    "d2h_bytes_per_step": N * 8},
            "gpu_launches": launches,
            # every kernel of a solve: the algorithmic bytes the library
            # counts per launch (each array read once, written once) over
            # the solve's time, against the measured copy bandwidth
            "solve_level": {
                form: {"algorithmic_bytes_per_solve": nb, "GB/s": nb / (ms * 1e-3 / args.steps) / 1e9,
                       "frac": nb / (ms * 1e-3 / args.steps) / 1e9 / peak}
                for form, nb, ms in (("mixed", bytes_mixed, ms_mixed), ("fp64", bytes_fp64, ms_fp64))},
            "roofline": {"bound": "hbm",
                         "kernel": "k_helm_rhs<float> sweep right-hand side r = b + H_off x, C192x70",
                         "achieved": rhs_bytes / (rhs_ms * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": rhs_bytes / (rhs_ms * 1e-3) / 1e9 / peak,
                         "peak_source": peak_kind, "traffic": traffic.get("k_helm_rhs"),
                         "algorithmic_bytes": rhs_bytes, "ms_per_launch": rhs_ms},
            "substitution": {"kernel": "k_subst_tma_reg<float,0,5> zero-start column "
                                       "substitution (TMA-staged, d' in registers), C192x70",
                             "ms": subst_ms, "algorithmic_bytes": subst_bytes,
                             "GB/s": subst_bytes / (subst_ms * 1e-3) / 1e9,
                             "frac": subst_bytes / (subst_ms * 1e-3) / 1e9 / peak,
                             "traffic": traffic.get("k_subst_tma_reg")},
            "smoother_sweep": {"kernels": "k_helm_rhs + k_subst_tma_reg<float,1,5>, FP32, C192x70",
                               "ms": sweep_ms, "algorithmic_bytes": sweep_bytes,
                               "GB/s": sweep_bytes / (sweep_ms * 1e-3) / 1e9,
                               "frac": sweep_bytes / (sweep_ms * 1e-3) / 1e9 / peak},
            "batched": dict(batched, problems_Mdof_per_s=batched["ndof"] /
                            (batched["ms_per_batch"] * 1e-3) / 1e6),
            **configs,
            "next_rows": nxt,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
