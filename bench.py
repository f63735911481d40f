"""Benchmark: tau00 solves/s at N = 2160 (complex), mixed precision vs plain FP64.

Workload (one step): one atom's fcc LIZ of 135 sites (a = 6.82 bohr, lmax 3, N = 2160,
kkrsz_ns = 16, binary alloy t-matrices from seeded phase shifts) solved at every point of a
31-point semicircle energy contour (-0.3 .. 0.7 Ry): 31 tau00 solves = build M = 1 - t G0, block
elimination, refinement, tau00_l.  Each rank (GPU) solves its own atom's contour (independent
atoms, no data-path collective: weak scaling).  Inputs are synthetic (seeded), see
lsms_b200/workloads.py.

JSON keys beyond the driver contract:
  value        mixed-precision solves/s (refined to <= 1e-10 of FP64), all ranks
  fp64         the plain-FP64 path on the same workload (solves/s), and the mixed/FP64 ratio
  err_mixed_vs_fp64   max relative tau00 difference between the two paths on this workload
  roofline     the dominant kernel (trailing update of the block elimination), algorithmic
               FLOPs / CUDA-event device time, against the peak named in `peak_source`
  e2e          the same metric through the public API with host buffers (tmatStore and LIZ
               uploaded from pinned host memory and tau00_l copied back every step)
  cpu_baseline the reference's own calculateTauMatrix (oracle/_ref) on the host cores

--impl reference times the reference's CPU implementation (oracle/_ref/libtauref.so, build
0x2000 + solver 0x2005, OpenBLAS on all host threads) on the same workload, one solve per step.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "tau00 solves/s at N=2160 c128: mixed vs plain FP64 at <=1e-10 rel err; %peak"
N_ENERGIES = 31
DATA = "synthetic (seeded phase-shift t-matrices, fcc LIZ)"
CONFIG = {"workload": "fcc LIZ 135 sites a=6.82, lmax 3, N=2160, kkrsz_ns 16, 31-point semicircle contour "
                      "-0.3..0.7 Ry, one atom per GPU"}
# DRAM bytes (read + write) of the trailing update per trailing-block entry and pass, from ncu
# captures on this workload: 18.7 B for a paired-step pass (24 jobs, trailing block 1776^2, K = 128
# complex; the FP32 read-modify-write of the block once for two steps) and 17.4 B for a single-step
# pass.  Not measured by this run (a kernel under ncu is not timed).
BYTES_PER_ENTRY_PAIR = 18.7
BYTES_PER_ENTRY_SINGLE = 17.4


def update_traffic_per_step(n, b, jobs, min_rest):
    """Average DRAM bytes of the trailing update per 64-column elimination step, over the schedule
    the library runs at paired-steps threshold min_rest (pairs while the block after the second
    step keeps >= min_rest columns): 434.9 MB at N = 2160, 31 jobs and the default 768."""
    nelim, k, total, steps = n - b, 0, 0.0, 0
    while k < nelim:
        k2 = k + 64
        if min_rest > 0 and k2 + 64 < nelim and n - k2 - 64 >= min_rest:
            total, k, steps = total + (n - k2 - 64) ** 2 * BYTES_PER_ENTRY_PAIR * jobs, k + 128, steps + 2
        else:
            total, k, steps = total + max(0, n - k - 64) ** 2 * BYTES_PER_ENTRY_SINGLE * jobs, k + 64, steps + 1
    return total / steps


def algorithmic_flops(N: int, b: int, L: int) -> float:
    """F = 8/3 n^3 + 8 n^2 b + 8 n b^2 + 8/3 b^3 + 8 b^3 + 8 b^3 L (L-1), n = N - b."""
    n = N - b
    return (8.0 / 3.0 * n ** 3 + 8.0 * n * n * b + 8.0 * n * b * b + 8.0 / 3.0 * b ** 3 + 8.0 * b ** 3
            + 8.0 * b ** 3 * L * (L - 1))


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running.

    Started before the warm-up (nvidia-smi's own start-up queries the driver); only the samples
    taken between mark_start() and mark_stop() count."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.samples = []
        self._stop = threading.Event()
        self._proc = None
        self._window = [None, None]

    def mark_start(self):
        self._window[0] = time.perf_counter()

    def mark_stop(self):
        self._window[1] = time.perf_counter()

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append((time.perf_counter(), parts))

    def __exit__(self, *a):
        if self._proc:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        t0, t1 = self._window
        inside = [p for t, p in self.samples if (t0 is None or t >= t0) and (t1 is None or t <= t1 + 0.25)]
        samples = inside or [p for _, p in self.samples[-2:]]
        return self._summarize(samples)

    @staticmethod
    def _summarize(samples):
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def rank_max(x, dist=None, device="cpu"):
    """The largest of every rank's x (one all-reduce over the process group `dist`; x itself
    without one): per-step times are reported as the slowest rank's."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, world, ms_max):
    """Units per second of the whole job: every rank processes units_per_rank (replicas over
    independent atoms) in the slowest rank's ms_max."""
    return world * units_per_rank / (ms_max * 1e-3)


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f), "MEASURED_PEAKS.json"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def run_reference(args, world, rank):
    """Reference CPU implementation timed on the host cores (rank 0 only): the reference's own
    calculateTauMatrix (oracle/_ref, build 0x2000 + zblock_lu 0x2005) on the same workload as the
    GPU arm.  A step is the whole 31-point contour when --steps K of them fit about two and a half
    minutes, else the first energies of the contour that do (every step the same sample)."""
    if rank != 0:
        return
    from lsms_b200 import workloads as W
    from oracle import reflib
    if not reflib.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtauref.so was not built"}))
        return
    cores = os.cpu_count() or 1
    reflib.set_num_threads(cores)
    prob = W.config_n2160(seed=2, npts=N_ENERGIES)
    t0 = time.perf_counter()
    reflib.calculate_tau(prob, 0, 0, reflib.ZBLOCKLU_CPP)  # one solve: the time of a solve
    t_solve = time.perf_counter() - t0
    per_step = int(min(N_ENERGIES, max(1, 150.0 / max(1, args.steps + args.warmup) / max(t_solve, 1e-3))))

    def step():
        for i in range(per_step):
            reflib.calculate_tau(prob, i, 0, reflib.ZBLOCKLU_CPP)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = (time.perf_counter() - t0) / args.steps
    value = per_step / dt
    sample = (f"the {per_step} first of the 31 contour solves at N=2160 per step, one after another, "
              f"OpenBLAS on {cores} threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": DATA,
        "config": dict(CONFIG, solver="reference calculateTauMatrix build 0x2000 + zblocklu_cpp 0x2005",
                       solves_per_step=per_step),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def cpu_baseline(prob, seconds_budget=20.0):
    """The reference's calculateTauMatrix on the host cores over the contour (within the budget);
    returns the baseline entry and the reference's tau00_l of the energies it solved."""
    from oracle import reflib
    if not reflib.available():
        return None, []
    cores = os.cpu_count() or 1
    reflib.set_num_threads(cores)
    reflib.calculate_tau(prob, 0, 0, reflib.ZBLOCKLU_CPP)  # warm-up
    outs = []
    n, t0 = 0, time.perf_counter()
    while n < 3 or (time.perf_counter() - t0 < seconds_budget and n < N_ENERGIES):
        outs.append(reflib.calculate_tau(prob, n % N_ENERGIES, 0, reflib.ZBLOCKLU_CPP))
        n += 1
        if time.perf_counter() - t0 > seconds_budget:
            break
    dt = time.perf_counter() - t0
    return ({"value": n / dt, "unit": "solves/s", "cores": cores, "kind": "reference",
             "sample": f"{n} of the 31 contour solves at N=2160, one after another, OpenBLAS on {cores} threads"},
            outs)


def cusolver_comparator(s, prob, ne, local, steps=3):
    """The reference GPU path's library solve (cuSOLVER zgetrf + zgetrs, as the reference's solver
    0x13 calls it, linearSolvers_CUDA.cu:316-322) on the same KKR matrices, via torch.linalg.solve:
    factor + solve of the ne built matrices with kkrsz_ns right-hand sides (no build, no tau00
    post-processing), device time per step of ne solves."""
    import torch
    N, b = prob.nrmat_ns, prob.kkrsz_ns
    dev = f"cuda:{local}"
    ms = torch.empty(ne, N, N, dtype=torch.complex128, device=dev)
    rhs = torch.zeros(ne, N, b, dtype=torch.complex128, device=dev)
    for i in range(ne):
        ms[i] = torch.from_numpy(s.build_kkr(0, i, 0, prob.energies[i], N))
        rhs[i, :b] = torch.from_numpy(prob.t_block(int(prob.liz_store_idx[0]), i))
    torch.linalg.solve(ms, rhs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        x = torch.linalg.solve(ms, rhs)
    e1.record()
    e1.synchronize()
    t = e0.elapsed_time(e1) / steps
    del ms, rhs, x
    torch.cuda.empty_cache()
    return {"value": ne / (t * 1e-3), "unit": "solves/s", "ms_per_step": t,
            "note": "cuSOLVER batched LU + solve (torch.linalg.solve) of the same 31 KKR matrices, "
                    "16 right-hand sides, factor and solve only"}


WORKLOADS = {
    "batched": "256 atoms x 32 energies, random fcc alloy with 5% vacancies, LIZ sizes 43..135 "
               "(N=688..2160), lmax 3, FP64 (and mixed) in one batched call",
    "noncollinear": "64 atoms x 16 energies, non-collinear kkrsz_ns=32, fcc LIZ 135 sites (N=4320), "
                    "mixed vs FP64",
    "adjoint": "64 atoms x 16 energies, fcc LIZ 87 sites (N=1392): tau00 plus d tau00/d t and "
               "d ln det M/d t for every LIZ site (b200tau_solve_vjp, FP64)",
    "comparators": "library baselines on this GPU: cuSOLVER batched zgetrf+zgetrs (torch.linalg.solve) on "
                   "the headline's 31 KKR matrices (N=2160, 16 right-hand sides), and cuBLAS "
                   "DGEMM / ZGEMM / SGEMM peaks",
}


def run_comparators(args, local):
    """The reference GPU comparator of the benchmark table (cuSOLVER LU on the same M) and the
    FP64 / FP32 library GEMM rates used as roofline context."""
    import torch
    from lsms_b200 import tau as T
    from lsms_b200 import workloads as W
    torch.cuda.set_device(local)
    prob = W.config_n2160(npts=N_ENERGIES)
    N, b = prob.nrmat_ns, prob.kkrsz_ns
    s = T.TauSolver(prob.lmax, prob.n_spin_cant, prob.n_spin_pola, device=local)
    s.load_problem(prob)
    ms = torch.empty(N_ENERGIES, N, N, dtype=torch.complex128, device=f"cuda:{local}")
    rhs = torch.zeros(N_ENERGIES, N, b, dtype=torch.complex128, device=f"cuda:{local}")
    for i in range(N_ENERGIES):
        ms[i] = torch.from_numpy(s.build_kkr(0, i, 0, prob.energies[i], N))
        rhs[i, :b] = torch.from_numpy(prob.t_block(int(prob.liz_store_idx[0]), i))
    s.close()

    def events(fn, reps):
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    sol = {}
    t_lu = events(lambda: sol.update(x=torch.linalg.solve(ms, rhs)), max(1, args.steps))
    del ms, rhs, sol

    def gemm_tflops(dtype, n):
        a = torch.randn(n, n, dtype=dtype, device=f"cuda:{local}")
        bb = torch.randn(n, n, dtype=dtype, device=f"cuda:{local}")
        t = events(lambda: a @ bb, 10)
        return (8 if dtype.is_complex else 2) * n ** 3 / (t * 1e-3) / 1e12

    line = {"metric": "comparators", "config": {"workload": WORKLOADS["comparators"]},
            "cusolver_zgesv": {"value": N_ENERGIES / (t_lu * 1e-3), "unit": "solves/s", "ms_per_step": t_lu,
                               "note": "factor + solve of the built M only (no build, no tau00 post-processing)"},
            "cublas_dgemm_tflops": gemm_tflops(torch.float64, 8192),
            "cublas_zgemm_tflops": gemm_tflops(torch.complex128, 4096),
            "cublas_sgemm_tflops": gemm_tflops(torch.float32, 8192)}
    print(json.dumps(line))


def run_workload(args, world, rank, local):
    """The other configurations of the benchmark's table, one JSON line each (not the headline):
    one step = every job of the configuration in one batched call."""
    line = workload_line(args.workload, args.steps, args.warmup, world, rank, local, args.autotune_by_size)
    print(json.dumps(line))


def workload_line(kind, steps, warmup, world, rank, local, autotune=False):
    import torch
    from lsms_b200 import tau as T
    from lsms_b200 import workloads as W
    torch.cuda.set_device(local)
    wl = {"batched": W.config_batched, "noncollinear": W.config_noncollinear_batch,
          "adjoint": W.config_adjoint_batch}[kind](seed=3 + rank)
    b = wl.kkrsz_ns
    s = T.TauSolver(wl.lmax, wl.n_spin_cant, wl.n_spin_pola, device=local)
    s.upload_tmat(wl.tmat_store)
    for a, at in enumerate(wl.atoms):
        s.set_atom(a, at.liz_pos, at.liz_lmax, at.liz_store_idx, at.ubr, at.ubrd)
    nspin = 2 if wl.n_spin_pola != wl.n_spin_cant else 1
    specs = [(a, iie, sp, e) for a in range(len(wl.atoms)) for iie, e in enumerate(wl.energies)
             for sp in range(nspin)]
    jobs = T.make_jobs(specs)
    nj = len(specs)
    flops = sum(algorithmic_flops(wl.nrmat_ns(a), b, wl.atoms[a].num_liz) for a, _, _, _ in specs)
    stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{local}")
    steps, warmup = max(1, steps), max(1, min(warmup, 1))

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    line = {"metric": f"{kind}: tau00 solves/s", "unit": "solves/s", "n_gpus": world, "steps": steps,
            "warmup": warmup, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": WORKLOADS[kind], "jobs_per_step": nj}}
    if kind == "adjoint":
        rng = np.random.default_rng(7)
        tb = rng.normal(size=(nj, b, b)) + 1j * rng.normal(size=(nj, b, b))
        Ls = [wl.atoms[a].num_liz for a, _, _, _ in specs]
        res = {}

        def vjp():
            res["out"] = s.solve_vjp(jobs, tb, Ls)
        ms = timed(vjp)
        tau = res["out"][0]
        fwd = s.solve_jobs(jobs, T.PREC_FP64)
        t0 = np.stack([wl.tmat_store[wl.atoms[a].liz_store_idx[0], iie, :b * b].reshape(b, b).T
                       for a, iie, _, _ in specs])
        fwd = fwd.reshape(nj, b, b).transpose(0, 2, 1) + t0
        line.update({"metric": "adjoint: tau00 + gradients per site, solves/s", "value": nj / (ms * 1e-3),
                     "ms_per_step": ms, "dtype": "c128",
                     "tau00_vs_forward_fp64": float(np.abs(tau - fwd).max() / np.abs(fwd).max()),
                     "note": "host buffers in and out (taubar, tau00, L gradient blocks per job)"})
        s.close()
        return line
    out = torch.empty(nj * b * b * 2, dtype=torch.float64, device=f"cuda:{local}")
    res = {}
    fallbacks = 0
    phases = {}
    tune = None
    if autotune:
        # untimed: the paired-steps threshold per size bucket, timed on a sample of each bucket's jobs
        mixed_default_ms = timed(lambda: s.solve_jobs_device(jobs, out.data_ptr(), T.PREC_MIXED))
        table = s.autotune_paired_steps_by_size(jobs)
        tune = {"paired_steps_min_rest_by_n": {str(k): v[0] for k, v in table.items()},
                "mixed_at_default_768": {"value": nj / (mixed_default_ms * 1e-3), "ms_per_step": mixed_default_ms}}
    for name, prec in (("fp64", T.PREC_FP64), ("mixed", T.PREC_MIXED)):
        ms = timed(lambda: s.solve_jobs_device(jobs, out.data_ptr(), prec))
        s.sync()
        res[name] = (ms, out.cpu().numpy().view(np.complex128).reshape(nj, -1).copy())
        if name == "mixed":
            fallbacks = s.last_fallback_count
        # device time per phase of one more step (CUDA events on the library stream)
        s.set_profiling(True)
        s.solve_jobs_device(jobs, out.data_ptr(), prec)
        s.sync()
        phases[name] = s.profile_phases()
        s.set_profiling(False)
    f, m = res["fp64"][1], res["mixed"][1]
    err = float(max(np.abs(m[j] - f[j]).max() / np.abs(f[j]).max() for j in range(nj)))
    head = "mixed" if kind == "noncollinear" else "fp64"
    ms = res[head][0]
    line.update({"value": nj / (res[head][0] * 1e-3), "ms_per_step": ms,
                 "dtype": "c64 trailing updates + c128 refinement" if head == "mixed" else "c128",
                 "fp64": {"value": nj / (res["fp64"][0] * 1e-3), "ms_per_step": res["fp64"][0],
                          "effective_tflops": flops / (res["fp64"][0] * 1e-3) / 1e12},
                 "mixed": {"value": nj / (res["mixed"][0] * 1e-3), "ms_per_step": res["mixed"][0],
                           "effective_tflops": flops / (res["mixed"][0] * 1e-3) / 1e12},
                 "err_mixed_vs_fp64_on_tau00_l": err,
                 "mixed_jobs_resolved_in_fp64": fallbacks,
                 "phase_ms_per_step": phases,
                 "algorithmic_flops_per_step": flops,
                 "autotune": tune or "off (paired-steps threshold 768)"})
    s.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the cuSOLVER comparator and the batched / non-collinear keys of the line")
    ap.add_argument("--workload", default="contour2160", choices=["contour2160", *WORKLOADS],
                    help="contour2160 = the headline line; the others print their own line")
    ap.add_argument("--energies", type=int, default=N_ENERGIES,
                    help="contour points solved per step (31 = the benchmark; fewer for small profiling cases)")
    ap.add_argument("--no-graphs", action="store_true",
                    help="launch each wave's kernels one by one instead of replaying its CUDA graph "
                         "(for profilers, which do not see into graphs with conditional nodes)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default paired-steps threshold instead of timing the candidates "
                         "on the headline workload before the warm-up")
    ap.add_argument("--autotune-by-size", action="store_true",
                    help="batched / non-collinear lines: tune the threshold per size bucket on a "
                         "64-job sample of each before timing (off: the default threshold)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world, rank, local = dist_setup()

    if args.impl == "reference":
        run_reference(args, world, rank)
        return
    if args.workload == "comparators":
        if rank == 0:
            run_comparators(args, local)
        return
    if args.workload != "contour2160":
        run_workload(args, world, rank, local)
        return

    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist

    from lsms_b200 import tau as T
    from lsms_b200 import workloads as W

    # each rank its own atom (seed) -> independent solves
    prob = W.config_n2160(seed=2 + rank, npts=N_ENERGIES)
    ne = max(1, min(args.energies, N_ENERGIES))
    N, b, L = prob.nrmat_ns, prob.kkrsz_ns, prob.num_liz
    flops_per_solve = algorithmic_flops(N, b, L)
    s = T.TauSolver(prob.lmax, prob.n_spin_cant, prob.n_spin_pola, device=local)
    s.load_problem(prob)
    if args.no_graphs:
        s.set_graphs(False)
    jobs = T.make_jobs([(0, i, 0, prob.energies[i]) for i in range(ne)])
    # untimed: the paired-steps threshold that is fastest on this workload becomes the setting
    tune = None
    if not args.no_autotune:
        chosen, tune_ms = s.autotune_paired_steps(jobs, reps=2)
        tune = {"paired_steps_min_rest": chosen, "ms_per_candidate": tune_ms}
    out = torch.empty(ne * b * b * 2, dtype=torch.float64, device=f"cuda:{local}")
    stream = torch.cuda.ExternalStream(s.stream, device=f"cuda:{local}")

    def barrier():
        if pg is not None:
            pg.barrier()

    def max_over_ranks(x: float) -> float:
        return rank_max(x, pg, f"cuda:{local}")

    def timed(prec, steps, warmup, sampler=None):
        cm = sampler if sampler is not None else _Null()
        with cm:  # the sampler starts before the warm-up, and counts the timed window only
            for _ in range(warmup):
                s.solve_jobs_device(jobs, out.data_ptr(), prec)
            s.sync()
            torch.cuda.synchronize()
            barrier()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            launches = 0
            if sampler is not None:
                sampler.mark_start()
            e0.record(stream)
            for _ in range(steps):
                s.solve_jobs_device(jobs, out.data_ptr(), prec)
                launches += s.last_launch_count
            e1.record(stream)
            s.sync()
            if sampler is not None:
                sampler.mark_stop()
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return max_over_ranks(ms), launches

    # --- mixed precision (the headline), device-resident inputs -------------------------------
    sampler = ClockSampler(local)
    ms_mixed, launches = timed(T.PREC_MIXED, args.steps, args.warmup, sampler)
    mixed_out = out.clone()
    # --- plain FP64 on the same workload ---------------------------------------------------------
    ms_fp64, _ = timed(T.PREC_FP64, max(2, args.steps // 2), 1)
    fp64_out = out.clone()
    a = mixed_out.cpu().numpy().view(np.complex128).reshape(ne, -1)
    f = fp64_out.cpu().numpy().view(np.complex128).reshape(ne, -1)
    t0l = np.stack([prob.t_block(int(prob.liz_store_idx[0]), i).T.reshape(-1) for i in range(ne)])
    err = float(max(np.abs(a[i] - f[i]).max() / np.abs(f[i] + t0l[i]).max() for i in range(ne)))

    # --- roofline of the dominant kernel (trailing update), CUDA events on the library stream ---
    s.set_profiling(True)
    for _ in range(2):
        s.solve_jobs_device(jobs, out.data_ptr(), T.PREC_MIXED)
    s.sync()
    k_ms, k_launches, k_flops = s.profile_read()
    phases = {k: v / 2.0 for k, v in s.profile_phases().items()}
    s.set_profiling(False)
    peaks, peak_src = measured_peaks()
    achieved = k_flops / (k_ms * 1e-3) / 1e12 if k_ms > 0 else None
    tf32_peak = float(peaks.get("bf16_tflops", 1590.0)) / 2.0

    # --- end to end through the public API with host buffers ------------------------------------
    tm_host = torch.from_numpy(np.ascontiguousarray(prob.tmat_store).view(np.float64)).pin_memory()
    tm_np = tm_host.numpy().view(np.complex128).reshape(prob.tmat_store.shape)
    h2d = tm_np.nbytes + prob.liz_pos.nbytes + prob.liz_lmax.nbytes + prob.liz_store_idx.nbytes
    d2h = ne * b * b * 16
    for _ in range(2):
        s.upload_tmat(tm_np)
        s.set_atom(0, prob.liz_pos, prob.liz_lmax, prob.liz_store_idx, prob.ubr, prob.ubrd)
        s.solve_jobs(jobs, T.PREC_MIXED)
    barrier()
    # each step timed on its own; the median over at least 20 steps (a host stall of the VM moves
    # one step, not the figure)
    e2e_steps = max(20, args.steps)
    e2e_times = []
    for _ in range(e2e_steps):
        t0 = time.perf_counter()
        s.upload_tmat(tm_np)
        s.set_atom(0, prob.liz_pos, prob.liz_lmax, prob.liz_store_idx, prob.ubr, prob.ubrd)
        s.solve_jobs(jobs, T.PREC_MIXED)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.median(e2e_times))

    # --- config 2 as the reference runs it: FP64, one energy per call -------------------------
    one = [T.make_jobs([(0, i, 0, prob.energies[i])]) for i in range(ne)]
    for i in range(ne):
        s.solve_jobs_device(one[i], out.data_ptr(), T.PREC_FP64)
    s.sync()
    # the fastest of three windows of ne host-enqueued calls (a host stall while enqueuing idles
    # the device and would otherwise land in the figure)
    one_ms = None
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(ne):
            s.solve_jobs_device(one[i], out.data_ptr() + 16 * b * b * i, T.PREC_FP64)
        e1.record(stream)
        s.sync()
        w_ms = e0.elapsed_time(e1) / ne
        one_ms = w_ms if one_ms is None else min(one_ms, w_ms)
    one_ms = max_over_ranks(one_ms)

    cpu, ref_outs = None, []
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, ref_outs = cpu_baseline(prob)
    err_ref = None
    if ref_outs:  # the GPU outputs against the reference's own tau00_l, on tau00 (+ t0)
        def rel(x, want):
            return float(np.abs(x - want).max() / np.abs(want).max())
        errs_m = [rel(a[i] + t0l[i], ref_outs[i] + t0l[i]) for i in range(len(ref_outs))]
        errs_f = [rel(f[i] + t0l[i], ref_outs[i] + t0l[i]) for i in range(len(ref_outs))]
        err_ref = {"mixed": max(errs_m), "fp64": max(errs_f), "energies": len(ref_outs),
                   "tolerance": {"mixed": 1e-10, "fp64": 1e-12},
                   "metric": "max |tau00 - tau00_ref| / max |tau00_ref| per energy, max over energies"}

    extras = {}
    if rank == 0 and world == 1 and not args.no_extras:
        extras["cusolver_zgesv"] = cusolver_comparator(s, prob, ne, local)
        for kind in ("batched", "noncollinear"):
            wlne = workload_line(kind, 1, 1, world, rank, local, args.autotune_by_size)
            extras[kind] = {k: wlne[k] for k in ("config", "value", "fp64", "mixed", "err_mixed_vs_fp64_on_tau00_l",
                                                 "mixed_jobs_resolved_in_fp64", "phase_ms_per_step", "autotune")}

    value = whole_job_rate(ne, world, ms_mixed)
    fp64_value = whole_job_rate(ne, world, ms_fp64)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 trailing updates + c128 refinement",
            "data": DATA,
            "config": {**CONFIG,
                       "solves_per_step": ne, "l2": "inputs larger than L2 "
                       f"({ne} x {N * N * 16 / 1e6:.0f} MB KKR matrices per step)",
                       "refinement_steps_mixed": "up to 10, per job until the correction estimate < 1e-12",
                       "refinement_steps_fp64": 1,
                       "autotune": tune or "off (paired-steps threshold 768)"},
            "fp64": {"value": fp64_value, "unit": "solves/s", "ms_per_step": ms_fp64,
                     "mixed_over_fp64": value / fp64_value},
            "fp64_one_energy_per_call": {"value": world / (one_ms * 1e-3), "unit": "solves/s",
                                         "ms_per_solve": one_ms,
                                         "note": "the reference's calling pattern: one b200tau call per "
                                                 "(atom, energy), FP64, inputs resident; fastest of three "
                                                 "windows of the 31 calls"},
            "err_mixed_vs_fp64": err,
            "err_vs_reference": err_ref,
            "phase_ms_per_step_mixed": phases,
            "flops_per_solve": flops_per_solve,
            "effective_tflops_mixed": value * flops_per_solve / 1e12,
            "roofline": {"kernel": "tc_update_kernel + tc_pack_kernel (trailing update A22 -= A21 W, "
                                   "tcgen05 kind::tf32, 3 hi/lo passes)",
                         "bound": "tensor",
                         "achieved": achieved, "unit": "TFLOP/s",
                         "peak": tf32_peak, "frac": (achieved / tf32_peak) if achieved else None,
                         "executed_frac": (3.0 * achieved / tf32_peak) if achieved else None,
                         "traffic": update_traffic_per_step(N, b, ne, tune["paired_steps_min_rest"] if tune else 768),
                         "traffic_unit": "bytes per elimination step",
                         "traffic_source": "ncu capture of the trailing-update kernel (dram__bytes_read.sum + "
                                           "dram__bytes_write.sum), scaled to this workload; not measured in "
                                           "this run",
                         "launches_timed": k_launches, "device_ms": k_ms, "algorithmic_flops": k_flops,
                         "flops_note": "algorithmic complex FLOPs 8 m n kb; the tensor pipe executes 3x "
                                       "that (hi*hi + hi*lo + lo*hi)",
                         "peak_source": f"TF32 dense = bf16_tflops / 2 of {peak_src} (measured bf16 "
                                        f"{peaks.get('bf16_tflops')} TF/s)"},
            "e2e": {"value": world * ne / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                    "ms_per_step_median": e2e_s * 1e3,
                    "ms_per_step_mean": statistics.mean(e2e_times) * 1e3,
                    "ms_per_step_min": min(e2e_times) * 1e3,
                    "timing": "wall clock per step (upload_tmat + set_atom + b200tau_solve with host "
                              "buffers), median over the steps"},
            "gpu_launches": int(launches),
            "clocks": sampler.summary(),
            "cpu_baseline": cpu,
            "configs": extras or None,
        }
        print(json.dumps(line))
    s.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
