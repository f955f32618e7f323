#!/usr/bin/env python3
"""Benchmark: one CheFSI pass (the eigensolver part of an SCF iteration) on Si216.

Workload (the configuration the headline metric is quoted on): Si216, 3x3x3 conventional
diamond supercell (30.78 Bohr cube), 90^3 grid (729,000 points), 520 states, FD order 12,
Chebyshev degree 20, Gamma point, atoms displaced by seeded N(0, 0.02 Bohr).  The
pseudopotential is the Si-like synthetic psp8 of lynx_b200.pseudo and V_eff a seeded
synthetic potential (no converged Si216 potential or Si psp8 is available), so `data` is
"synthetic".

A step = one CheFSI pass = Chebyshev filter (20 H-applies) + H*Y + Rayleigh-Ritz
(overlap, projected H, Cholesky, subspace eigensolve, rotation) on device-resident
orbitals; value = seconds per pass (lower is better).  With --gpus N each rank runs its
own replica (the path has no exchange step: replicas only); the timing is the max over
ranks.  `--impl reference` times the reference's own CPU code (oracle/_ref) on a bounded
sample of the same workload on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "s/SCF-iter Si216 CheFSI: mixed vs plain FP64 on B200 at ΔE≤1e-5 Ha/atom; HBM GB/s"
METRIC_NOTE = ("value = seconds per CheFSI pass at fixed V_eff (filter + H*Y + Rayleigh-Ritz), the "
               "eigensolver part of an SCF iteration; scf_iteration adds the Fermi level, the density and "
               "the V_eff build (GGA-PBE + Poisson) of that pass; density mixing is not included")

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one cheb_pipe_kernel launch per
# grid-point x state update, from an ncu capture of the Si64 case (60^3 grid, 160 states, the
# launch shape the autotuner picks there): 440.3 MB (FP32) and 864.1 MB (FP64) per launch.
# Whole planes stream through the same band geometry at every size, so the traffic of a launch
# scales with the updates it processes.
TRAFFIC_PER_UPDATE = {"mixed": 440.271e6 / (216000 * 160), "fp64": 864.076e6 / (216000 * 160)}
# The same for the launch the pass runs, with the fused nonlocal term: 482.0 MB per FP32 launch at
# Si64 (dram__bytes_read.sum 369.85 MB + dram__bytes_write.sum 112.16 MB, mean of three launches).
TRAFFIC_PER_UPDATE_FUSED = {"mixed": 482.0e6 / (216000 * 160), "fp64": None}

CONFIGS = {
    # name: (reps, grid, nstates, degree, displace)
    "si216": (3, 90, 520, 20, 0.02),
    "si64": (2, 60, 160, 20, 0.0),
    "si8": (1, 30, 24, 20, 0.0),
}
# Batched workload: primitive FCC Si2 on a 4x4x4 Monkhorst-Pack grid (36 reduced k-points, complex
# Bloch orbitals, 20^3 grid, 16 states) plus 32 Si8 cells with seeded isotropic strain
# uniform(+-3%) on grids drawn from {24,26,28,30,32}^3 (24 states); degree 20.  A step is one
# CheFSI pass over all 68 problems.
BATCH_CONFIG = "kpt_ensemble"
BATCH_METRIC = "s per CheFSI pass over a batch: Si2 FCC 4x4x4 k-points + 32 strained Si8 cells"


def workload_config(config, cl, nst, degree, natom, world):
    """The `config` dict of both arms (the same workload for the GPU arm and the reference arm)."""
    from lynx_b200 import cell as C
    return {"workload": f"{config} CheFSI pass at fixed V_eff", "grid": cl.shape[0], "nstates": nst,
            "degree": degree, "fd_order": 12, "natom": natom,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs larger than L2 (FP32 orbital blocks of %.2f GB)" % (4 * cl.nd * nst / 1e9)}


def converged_accuracy(solver, ctx, es, psi, Vd, lc, emin, hi, degree, nocc, natom, max_passes=60):
    """Mixed vs FP64 at convergence (see main).  Leaves psi as it found it."""
    import torch
    start = psi.clone()
    out = {}
    npass = None
    for prec in ("fp64", "mixed"):
        psi.copy_(start)
        l, e = lc, emin
        prev, last = None, None
        n = 0
        while True:
            _, eig = es.solve(psi, Vd, l, e, hi, degree, precision=prec)
            eig = np.asarray(eig).copy()
            l, e = es.lambda_cutoff(), float(eig[0])
            n += 1
            if prev is not None:
                last = float(np.abs(eig[:nocc] - prev[:nocc]).max())
            prev = eig
            if prec == "fp64" and ((last is not None and last < 1e-9) or n >= max_passes):
                npass = n
                break
            if prec == "mixed" and n >= npass:
                break
        nel = 4.0 * natom
        ef = solver.fermi_level(eig, 2.0 * np.ones(len(eig)), nel, 1000.0)
        occ = solver.occupations(eig, ef, 1000.0)
        f, _ = solver.NonlocalProjector(ctx).force(psi, occ, occfac=2.0)
        out[prec] = (eig, np.asarray(f), last)
    psi.copy_(start)
    torch.cuda.synchronize()
    e64, f64, last64 = out["fp64"]
    em, fm, _ = out["mixed"]
    return {"passes": npass, "fp64_last_change_occ_Ha": last64,
            "max_abs_dE_occ_Ha": float(np.abs(em[:nocc] - e64[:nocc]).max()),
            "band_energy_dE_per_atom_Ha": float(abs(2.0 * (em[:nocc] - e64[:nocc]).sum()) / natom),
            "max_abs_dF_nonlocal_Ha_per_Bohr": float(np.abs(fm - f64).max()),
            "max_abs_F_nonlocal_Ha_per_Bohr": float(np.abs(f64).max()),
            "how": "FP64 passes from the state after the timed passes until the occupied Ritz values move "
                   "< 1e-9 Ha, the same number of mixed passes from the same state; forces: nonlocal, "
                   "Fermi-Dirac occupations at 0.001 Ha"}


def replica_seed(rank: int) -> int:
    """Seed of a replica's start orbitals: with --gpus N every rank solves its own problem."""
    return 1234 + rank


def max_over_ranks(seconds: float, world: int, device) -> float:
    """The job's time is the slowest replica's: an all-reduce MAX over the ranks (no-op at N=1)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([seconds], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="lynx", choices=["lynx", "reference"])
    p.add_argument("--config", default="si216", choices=sorted(CONFIGS) + [BATCH_CONFIG])
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-scf", action="store_true", help="skip the SCF-iteration summary (pass + density + V_eff)")
    p.add_argument("--no-batch", action="store_true", help="skip the batched k-point + ensemble summary")
    p.add_argument("--profile-pass", action="store_true",
                   help="bracket the first timed pass with cudaProfilerStart/Stop, so that "
                        "`ncu --profile-from-start off` captures exactly one pass")
    return p.parse_args()


def build_system(config, seed=2024):
    from lynx_b200 import cell as C
    from lynx_b200 import pseudo as P
    reps, grid, nst, degree, disp = CONFIGS[config]
    cl, pos = C.diamond_si(reps, grid, displace=disp, seed=seed)
    psp_path = os.path.join("/tmp", f"lynx_b200_si_synthetic_{os.getpid()}.psp8")
    P.synthetic_si_psp8(psp_path)
    psp = P.read_psp8(psp_path)
    tab = P.nonlocal_tables(cl, pos, psp)
    V = veff_separable(cl, pos, noise=1e-3, seed=seed)
    return cl, pos, psp_path, tab, V, nst, degree


def veff_separable(cl, pos, depth=1.2, width=1.1, noise=0.0, seed=0):
    """The synthetic potential of lynx_b200.cell.synthetic_veff, evaluated separably."""
    from lynx_b200 import cell as C
    return C.synthetic_veff_separable(cl, pos, depth=depth, width=width, noise=noise, seed=seed)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    except Exception:
        return 6650.0, 1590.0, "fallback"


class RefSample:
    """Reference CPU CheFSI time per pass, estimated from a bounded sample.

    filter: the reference chebyshev_filter on `cols` of the columns, scaled by nstates/cols
    (the filter is column-independent);  Rayleigh-Ritz: the reference orthogonalize +
    project + diag + rotate on all nstates columns of a 1/8-size grid (45^3 for Si216), the
    grid-proportional part scaled by 8 and the N^3 eigensolve counted once.  The set-up
    (projector tables, Lanczos bounds) is done once; run() times one sample."""

    def __init__(self, cl, pos, psp_path, V, nstates, degree, cols=8):
        from lynx_b200 import cell as C
        from lynx_b200.cell import Cell
        from oracle import ref
        self.ref = ref
        self.nthreads = os.cpu_count() or 1
        ref.set_threads(self.nthreads)
        self.cl, self.pos, self.psp_path, self.V = cl, pos, psp_path, V
        self.nstates, self.degree, self.cols = nstates, degree, cols
        R = ref.RefLynx(cl, pos, psp_path)
        self.lo, self.hi = R.lanczos(V, maxit=60)
        self.nd = R.nd
        self.X = C.random_orbitals(R.nd, cols, seed=7)
        self.g = tuple(max(13, n // 2) for n in cl.shape)
        self.cs = Cell(cl.latvec, self.g, True, (0, 0, 0), cl.fd_order)
        self.scale = float(np.prod(cl.shape)) / float(np.prod(self.g))
        self.Vs = veff_separable(self.cs, pos)
        self.Y = None
        self.sample = (f"reference CPU CheFSI (oracle/_ref, OpenMP {self.nthreads} threads): filter degree {degree} on "
                       f"{cols}/{nstates} columns of the {cl.shape[0]}^3 grid scaled x{nstates / cols:.1f}; "
                       f"Rayleigh-Ritz on all {nstates} states of a {self.g[0]}^3 grid, grid-proportional part "
                       f"scaled x{self.scale:.2f}, eigensolve once")

    def run(self):
        from lynx_b200 import cell as C
        ref = self.ref
        R = ref.RefLynx(self.cl, self.pos, self.psp_path)
        lc = 0.5 * (self.lo + self.hi)
        t0 = time.perf_counter()
        R.chebyshev_filter(self.X, self.V, lc, self.lo, self.hi, self.degree)
        t_filter = (time.perf_counter() - t0) * self.nstates / self.cols
        Rs = ref.RefLynx(self.cs, self.pos, self.psp_path)
        Y = C.random_orbitals(Rs.nd, self.nstates, seed=8)
        t0 = time.perf_counter()
        Yo = Rs.orthogonalize(Y)
        Hs = Rs.project(Yo, self.Vs)
        t1 = time.perf_counter()
        eig, Q = Rs.diag(Hs)
        t2 = time.perf_counter()
        Rs.rotate(Yo, Q)
        t3 = time.perf_counter()
        t_rr = ((t1 - t0) + (t3 - t2)) * self.scale + (t2 - t1)
        ref.lib().ref_free()
        return t_filter + t_rr, {"filter_s": t_filter, "rr_s": t_rr}


def cpu_baseline_sample(cl, pos, psp_path, V, nstates, degree, cols=8):
    """One RefSample: (seconds per pass, threads, sample description, parts)."""
    S = RefSample(cl, pos, psp_path, V, nstates, degree, cols)
    t, parts = S.run()
    return t, S.nthreads, S.sample, parts


def sample_check(psp_path):
    """The sampled estimate of cpu_baseline_sample checked against one whole reference pass, at
    the Si64 workload (60^3 grid, 160 states, degree 20), where a whole pass takes seconds:
    returns both times and their ratio."""
    from lynx_b200 import cell as C
    from oracle import ref
    reps, grid, nst, degree, disp = CONFIGS["si64"]
    cl, pos = C.diamond_si(reps, grid, displace=disp, seed=2024)
    V = veff_separable(cl, pos, noise=1e-3, seed=2024)
    est, cores, _, _ = cpu_baseline_sample(cl, pos, psp_path, V, nst, degree)
    ref.set_threads(cores)
    R = ref.RefLynx(cl, pos, psp_path)
    lo, hi = R.lanczos(V, maxit=60)
    X = C.random_orbitals(R.nd, nst, seed=9)
    t0 = time.perf_counter()
    R.solve(X, V, 0.5 * (lo + hi), lo, hi, degree)
    full = time.perf_counter() - t0
    ref.lib().ref_free()
    return {"workload": "si64 CheFSI pass at fixed V_eff (60^3, 160 states, degree 20)", "whole_pass_s": full,
            "sampled_estimate_s": est, "whole_over_estimate": full / est, "cores": cores}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_lynx.so not built"}))
        return
    cl, pos, psp_path, tab, V, nst, degree = build_system(args.config)
    # each step is one bounded sample (one column of the filter, the Rayleigh-Ritz on the coarse
    # grid), so that --warmup W --steps K stays within minutes; the set-up is done once
    S = RefSample(cl, pos, psp_path, V, nst, degree, cols=1)
    times = []
    for i in range(args.warmup + args.steps):
        t, parts = S.run()
        if i >= args.warmup:
            times.append(t)
    v = float(np.mean(times))
    cores, sample = S.nthreads, S.sample
    line = {
        "metric": METRIC, "metric_note": METRIC_NOTE, "value": v, "unit": "s/iter", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": workload_config(args.config, cl, nst, degree, len(pos), world),
        "cpu_baseline": {"value": v, "unit": "s/iter", "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if args.config != "si64":
        line["sample_check"] = sample_check(psp_path)
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.config == BATCH_CONFIG:
            return run_reference_batch(args, rank, world)
        return run_reference(args, rank, world)
    if args.config == BATCH_CONFIG:
        return run_batch(args, rank, world, local)

    import torch
    import torch.distributed as dist
    from lynx_b200 import _lib
    from lynx_b200 import solver

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    cl, pos, psp_path, tab, V, nst, degree = build_system(args.config)
    ctx = solver.Context(cl, device=local)
    ctx.set_nonlocal(tab)
    lib = ctx.lib
    Vd = torch.from_numpy(V).cuda()
    es = solver.EigenSolver(ctx, args.precision)
    lo, hi = es.lanczos_bounds(Vd)
    lc, emin = 0.5 * (lo + hi), lo
    gen = torch.Generator(device="cuda").manual_seed(replica_seed(rank))
    psi = (torch.rand((nst, ctx.nd), generator=gen, device="cuda", dtype=torch.float64) - 0.5).contiguous()

    def one_pass(precision):
        nonlocal lc, emin
        _, eig = es.solve(psi, Vd, lc, emin, hi, degree, precision=precision)
        lc = es.lambda_cutoff()
        emin = float(eig[0])
        return eig

    for _ in range(args.warmup):
        one_pass(args.precision)
    # the other precision's first pass runs the stencil autotuner for its own types: keep it out of
    # the timed passes
    other = "fp64" if args.precision == "mixed" else "mixed"
    one_pass(other)
    natom = len(pos)
    nocc = 2 * natom  # 4 valence electrons per Si, 2 per state

    # FP64 timing (the plain-FP64 GPU CheFSI the mixed path is compared against)
    def timed(precision, k, profile=False):
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for i in range(k):
            if profile and i == 0:
                torch.cuda.profiler.start()
            one_pass(precision)
            if profile and i == 0:
                torch.cuda.synchronize()
                torch.cuda.profiler.stop()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / k

    t_other = timed(other, max(1, min(2, args.steps)))

    lib.lynx_launch_count(1)
    with ClockSampler(local) as clk:
        t_main = timed(args.precision, args.steps, args.profile_pass)
    launches = int(lib.lynx_launch_count(1))
    t_main = max_over_ranks(t_main, world, "cuda")

    # Converged accuracy: from the state after the timed passes, FP64 passes until the occupied
    # Ritz values stop moving, and the same number of mixed passes from the same state; then the
    # occupied Ritz values and the nonlocal forces (Fermi-Dirac, 0.001 Ha) of both.  Untimed.
    acc = converged_accuracy(solver, ctx, es, psi, Vd, lc, emin, hi, degree, nocc, natom)

    # Roofline of the dominant kernel: the stencil kernel as the pass runs it (nonlocal term fused),
    # each launch timed alone with CUDA events on the context's stream.
    import ctypes
    prec_id = _lib.PREC_MIXED if args.precision == "mixed" else _lib.PREC_FP64
    ctx.sync_stream()
    ms_k = ctypes.c_double()
    _lib.check(lib.lynx_time_filter_step(ctx.handle, ctypes.c_void_p(Vd.data_ptr()), nst, prec_id, 2, 10,
                                         ctypes.byref(ms_k)))
    ms = ctypes.c_double()
    _lib.check(lib.lynx_time_filter_step(ctx.handle, ctypes.c_void_p(Vd.data_ptr()), nst, prec_id, 0, 10,
                                         ctypes.byref(ms)))
    ms_nl = ctypes.c_double()
    _lib.check(lib.lynx_time_filter_step(ctx.handle, ctypes.c_void_p(Vd.data_ptr()), nst, prec_id, 1, 5,
                                         ctypes.byref(ms_nl)))
    wsize = 4 if args.precision == "mixed" else 8
    step_bytes = wsize * ctx.nd * (3 * nst + 1)  # x, xold, out per update + V per point
    n_pts = int(np.unique(np.asarray(tab.gpos)).size)  # distinct sphere points: the fused term reads
    fused_bytes = step_bytes + wsize * n_pts * nst   # one (chi alpha) value per sphere point and state
    hbm, bf16, peak_kind = measured_peaks()
    achieved = fused_bytes / (ms_k.value * 1e-3) / 1e9
    updates = ctx.nd * nst * degree

    scf = None
    if rank == 0 and not args.no_scf:
        scf = scf_iteration_summary(ctx, es, psi, Vd, lc, emin, hi, degree, natom)

    e2e = None
    if not args.no_e2e:
        host_psi = torch.empty((nst, ctx.nd), dtype=torch.float64, pin_memory=True)
        host_psi.copy_(psi)
        hv = torch.from_numpy(V).pin_memory()
        eig = np.zeros(nst)
        lc_out = ctypes.c_double()
        hp = host_psi.numpy()
        hvn = hv.numpy()
        _lib.check(lib.lynx_eigensolver_solve_host(ctx.handle, _lib.dptr(hp), _lib.dptr(eig), _lib.dptr(hvn), nst,
                                                   ctx.nd, lc, emin, hi, degree, prec_id, ctypes.byref(lc_out)))
        torch.cuda.synchronize()
        k = max(1, min(3, args.steps))
        t0 = time.perf_counter()
        for _ in range(k):
            _lib.check(lib.lynx_eigensolver_solve_host(ctx.handle, _lib.dptr(hp), _lib.dptr(eig), _lib.dptr(hvn),
                                                       nst, ctx.nd, lc_out.value, float(eig[0]), hi, degree,
                                                       prec_id, ctypes.byref(lc_out)))
        torch.cuda.synchronize()
        te = (time.perf_counter() - t0) / k
        e2e = {"value": te, "unit": "s/iter", "h2d_bytes_per_step": int(8 * ctx.nd * (nst + 1)),
               "d2h_bytes_per_step": int(8 * (ctx.nd * nst + nst)), "api": "lynx_eigensolver_solve_host"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            v, cores, sample, parts = cpu_baseline_sample(cl, pos, psp_path, V, nst, degree)
            cpu = {"value": v, "unit": "s/iter", "cores": cores, "kind": "reference", "sample": sample}

    if rank == 0:
        line = {
            "metric": METRIC, "metric_note": METRIC_NOTE, "value": t_main, "unit": "s/iter", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_main * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == "mixed" else "f64",
            "data": "synthetic", "config": workload_config(args.config, cl, nst, degree, natom, world),
            "updates_per_s": world * updates / t_main,
            "fp64_s_per_iter" if args.precision == "mixed" else "mixed_s_per_iter": t_other,
            "speedup_vs_fp64" if args.precision == "mixed" else "speedup_vs_mixed": t_other / t_main,
            "accuracy": acc,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": (TRAFFIC_PER_UPDATE_FUSED[args.precision] * ctx.nd * nst
                                     if TRAFFIC_PER_UPDATE_FUSED[args.precision] else None),
                         "traffic_source": "ncu capture of the Si64 case scaled by updates per launch",
                         "kernel": "cheb_pipe_kernel with the fused nonlocal term (stencil + Veff + a*chi*alpha + "
                                   "three-term recurrence), as the pass runs it",
                         "algorithmic_bytes": fused_bytes, "ms_per_launch": ms_k.value,
                         "plain_step": {"ms_per_launch": ms.value, "algorithmic_bytes": step_bytes,
                                        "frac": step_bytes / (ms.value * 1e-3) / 1e9 / hbm},
                         "whole_degree_step": {"ms": ms_nl.value, "frac_of_3_word_floor":
                                               step_bytes / (ms_nl.value * 1e-3) / 1e9 / hbm},
                         "peak_kind": peak_kind},
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "scf_iteration": scf,
        }
        if not args.no_batch:
            line["batch"] = batch_summary()
        print(json.dumps(line))
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    try:
        os.remove(psp_path)
    except OSError:
        pass


def build_batch(seed=2024):
    from lynx_b200 import ensemble as E
    from lynx_b200 import pseudo as P
    psp_path = os.path.join("/tmp", f"lynx_b200_si_synthetic_{os.getpid()}.psp8")
    P.synthetic_si_psp8(psp_path)
    psp = P.read_psp8(psp_path)
    probs = E.kpoint_problems(psp, (4, 4, 4), grid=20, nband=16, seed=seed)
    probs += E.strained_ensemble(psp, 32, (24, 26, 28, 30, 32), 0.03, nband=24, seed=seed)
    return probs, psp_path


def batch_filter_bytes(probs, precision, degree):
    """Algorithmic bytes of the filter steps of one pass: per update, x, xold and out in the
    filter's storage type, plus V per point, `degree` steps per problem."""
    tot = 0
    for pb in probs:
        w = (4 if precision == "mixed" else 8) * (2 if pb.complex else 1)
        tot += degree * (w * pb.cell.nd * 3 * pb.nband + 8 * pb.cell.nd)
    return tot


def reference_batch_pass(probs, psp_path, degree, nthreads):
    """The reference CPU CheFSI pass over every problem of the batch, one after another (as
    SCF::solve_eigenproblem loops over k-points), timed per problem and summed."""
    from lynx_b200 import cell as C
    from oracle import ref
    ref.set_threads(nthreads)
    total = 0.0
    for i, pb in enumerate(probs):
        R = ref.RefLynx(pb.cell, pb.positions, psp_path)
        lo, hi = R.lanczos(pb.veff, maxit=60, kpt=pb.kcart)
        lc = 0.5 * (lo + hi)
        X = C.random_orbitals(R.nd, pb.nband, seed=300 + i, complex_=pb.complex)
        t0 = time.perf_counter()
        if pb.complex:
            R.solve_kpt(X, pb.veff, lc, lo, hi, degree, pb.kcart)
        else:
            R.solve(X, pb.veff, lc, lo, hi, degree)
        total += time.perf_counter() - t0
    ref.lib().ref_free()
    return total


def run_reference_batch(args, rank, world):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref_lynx.so not built"}))
        return
    probs, psp_path = build_batch()
    nthreads = os.cpu_count() or 1
    times = [reference_batch_pass(probs, psp_path, 20, nthreads) for _ in range(args.warmup + args.steps)]
    v = float(np.mean(times[args.warmup:]))
    sample = (f"reference CPU CheFSI (oracle/_ref, OpenMP {nthreads} threads): the full pass over all "
              f"{len(probs)} problems, one after another")
    print(json.dumps({
        "metric": BATCH_METRIC, "value": v, "unit": "s/iter", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": "batched CheFSI pass: 36 k-points Si2 FCC 20^3 N=16 + 32 strained Si8 "
                               "24-32^3 N=24", "degree": 20, "fd_order": 12, "parallelism": "replicas"},
        "cpu_baseline": {"value": v, "unit": "s/iter", "cores": nthreads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "s/iter", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    try:
        os.remove(psp_path)
    except OSError:
        pass


class BatchRun:
    """The batched workload on this process's GPU: every problem on its own context; passes over
    all of them through solve_batch (lynx_eigensolver_solve_batch), or one after another."""

    def __init__(self, rank, degree=20):
        import torch
        from lynx_b200 import solver
        self.solver = solver
        self.degree = degree
        self.probs, self.psp_path = build_batch()
        self.solvers, self.lo_hi, self.psis, self.Vs = [], [], [], []
        gen = torch.Generator(device="cuda").manual_seed(replica_seed(rank))
        for pb in self.probs:
            ctx = solver.Context(pb.cell, device=torch.cuda.current_device())
            ctx.set_nonlocal(pb.tables)
            if pb.complex:
                ctx.set_kpoint(pb.kcart)
            es = solver.EigenSolver(ctx, "mixed")
            V = torch.from_numpy(pb.veff).cuda()
            lo, hi = es.lanczos_bounds(V, kpt=pb.complex)
            self.solvers.append(es)
            self.lo_hi.append([0.5 * (lo + hi), lo, hi])
            self.Vs.append(V)
            x = torch.rand((pb.nband, ctx.nd), generator=gen, device="cuda", dtype=torch.float64) - 0.5
            if pb.complex:
                y = torch.rand((pb.nband, ctx.nd), generator=gen, device="cuda", dtype=torch.float64) - 0.5
                x = torch.complex(x, y)
            self.psis.append(x.contiguous())
        self.kflags = [pb.complex for pb in self.probs]

    def batched(self, precision, host=None):
        res = self.solver.solve_batch(self.solvers, host if host is not None else self.psis, self.Vs,
                                      [b[0] for b in self.lo_hi], [b[1] for b in self.lo_hi], [b[2] for b in self.lo_hi],
                                      self.degree, precision=precision, kpt=self.kflags)
        for b, es, (_, eig) in zip(self.lo_hi, self.solvers, res):
            b[0] = es.lambda_cutoff()
            b[1] = float(eig[0])
        return res

    def sequential(self, precision):
        for pb, es, b, p, V in zip(self.probs, self.solvers, self.lo_hi, self.psis, self.Vs):
            fn = es.solve_kpt if pb.complex else es.solve
            _, eig = fn(p, V, b[0], b[1], b[2], self.degree, precision=precision)
            b[0] = es.lambda_cutoff()
            b[1] = float(eig[0])

    def close(self):
        for es in self.solvers:
            es.ctx.close()
        try:
            os.remove(self.psp_path)
        except OSError:
            pass


def timed_device(fn, k, world=1):
    """Seconds per call of fn over k calls, CUDA events on torch's current stream."""
    import torch
    import torch.distributed as dist
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(k):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / k


def batch_summary():
    """The batched k-point + strained-ensemble workload, measured beside the headline: s per pass
    over all problems through solve_batch, mixed and FP64, and the mixed passes one after another."""
    B = BatchRun(0)
    try:
        for _ in range(2):
            B.batched("mixed")
        B.batched("fp64")
        B.sequential("mixed")
        t_mixed = timed_device(lambda: B.batched("mixed"), 3)
        t_fp64 = timed_device(lambda: B.batched("fp64"), 2)
        t_seq = timed_device(lambda: B.sequential("mixed"), 2)
        return {"workload": "batched CheFSI pass: 36 k-points Si2 FCC 20^3 N=16 (complex) + 32 strained Si8 "
                            "24-32^3 N=24, degree 20", "problems": len(B.probs), "mixed_s_per_pass": t_mixed,
                "fp64_s_per_pass": t_fp64, "speedup_vs_fp64": t_fp64 / t_mixed,
                "sequential_mixed_s_per_pass": t_seq, "speedup_vs_sequential": t_seq / t_mixed,
                "api": "lynx_eigensolver_solve_batch (one host thread and stream per problem)"}
    finally:
        B.close()


def scf_iteration_summary(ctx, es, psi, Vd, lc, emin, hi, degree, natom, reps=2):
    """One SCF iteration at fixed V_eff as the device runs it: the CheFSI pass with the Fermi level
    (Fermi-Dirac, 0.001 Ha), occupations and density of the new orbitals
    (lynx_eigensolver_solve_density; in the mixed pass the density is accumulated by the
    tensor-core rotation), then V_eff = V_xc + phi of that density (GGA-PBE; the periodic cell's
    Poisson equation solved by FFT, lynx_effective_potential's default).  The new potential is not
    fed back (no mixing, and the synthetic V_eff has no pseudocharge), so every iteration solves
    the same eigenproblem.  Mixing is not included."""
    import torch
    from lynx_b200 import potential as Pm
    pot = Pm.EffectivePotential(ctx)
    nel = 4.0 * natom
    st = {"lc": lc, "emin": emin}
    rho = torch.empty(ctx.nd, dtype=torch.float64, device="cuda")
    iters = []

    def one(prec):
        _, eig, _, _ = es.solve_density(psi, Vd, st["lc"], st["emin"], hi, degree, nelectron=nel, beta=1000.0,
                                        rho=rho, precision=prec)
        st["lc"] = es.lambda_cutoff()
        st["emin"] = float(eig[0])
        iters.append(pot.compute(rho, poisson_tol=1e-8).poisson_iters)

    t0 = time.perf_counter()
    one("mixed")  # the first V_eff build solves Poisson from phi = 0
    torch.cuda.synchronize()
    cold = {"s": time.perf_counter() - t0, "poisson_iters": iters[-1]}
    out = {"note": "CheFSI pass + Fermi level + density + V_eff build (GGA-PBE; Poisson of the periodic cell "
                   "solved by FFT); V_eff not fed back, mixing not included",
           "first_iteration_cold_poisson": cold}
    for prec in ("mixed", "fp64"):
        one(prec)
        t = timed_device(lambda: one(prec), reps)
        out[f"{prec}_s_per_iter"] = t
    out["veff_build_s"] = timed_device(lambda: pot.compute(rho, poisson_tol=1e-8), 2)
    out["poisson_iters_warm"] = iters[-1]
    out["speedup_vs_fp64"] = out["fp64_s_per_iter"] / out["mixed_s_per_iter"]
    return out


def run_batch(args, rank, world, local):
    """The batched workload as the headline: every problem on its own context, one pass over all
    of them per step through solve_batch (lynx_eigensolver_solve_batch), against the same passes
    run one after another."""
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    B = BatchRun(rank)
    probs, psp_path, psis, degree = B.probs, B.psp_path, B.psis, B.degree
    batched, sequential = B.batched, B.sequential

    for _ in range(args.warmup):
        batched(args.precision)
    sequential(args.precision)
    lib = B.solvers[0].ctx.lib
    t_seq = timed_device(lambda: sequential(args.precision), max(1, min(2, args.steps)), world)
    lib.lynx_launch_count(1)
    with ClockSampler(local) as clk:
        t_main = timed_device(lambda: batched(args.precision), args.steps, world)
    launches = int(lib.lynx_launch_count(1))
    t_main = max_over_ranks(t_main, world, "cuda")

    e2e = None
    if not args.no_e2e:
        host = []
        for p in psis:
            a = p.cpu().numpy().T
            host.append(np.asfortranarray(a))
        batched(args.precision, host)
        torch.cuda.synchronize()
        k = max(1, min(3, args.steps))
        t0 = time.perf_counter()
        for _ in range(k):
            batched(args.precision, host)
        torch.cuda.synchronize()
        te = (time.perf_counter() - t0) / k
        h2d = sum(p.numel() * p.element_size() + 8 * pb.cell.nd for p, pb in zip(psis, probs))
        d2h = sum(p.numel() * p.element_size() + 8 * pb.nband for p, pb in zip(psis, probs))
        e2e = {"value": te, "unit": "s/iter", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "api": "lynx_b200.solver.solve_batch (host numpy orbitals)"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import ref
        if ref.available():
            nthreads = os.cpu_count() or 1
            v = reference_batch_pass(probs, psp_path, degree, nthreads)
            cpu = {"value": v, "unit": "s/iter", "cores": nthreads, "kind": "reference",
                   "sample": f"the full pass over all {len(probs)} problems, one after another"}

    if rank == 0:
        hbm, _, peak_kind = measured_peaks()
        fb = batch_filter_bytes(probs, args.precision, degree)
        achieved = fb / t_main / 1e9
        nbytes = sum(p.numel() * p.element_size() for p in psis)
        print(json.dumps({
            "metric": BATCH_METRIC, "value": t_main, "unit": "s/iter", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_main * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": f"batched CheFSI pass ({args.precision}): 36 k-points Si2 FCC 20^3 N=16 + "
                                   f"32 strained Si8 24-32^3 N=24", "problems": len(probs), "degree": degree,
                       "fd_order": 12, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 in total (orbitals %.2f GB)" % (nbytes / 1e9)},
            "sequential_s_per_iter": t_seq, "speedup_vs_sequential": t_seq / t_main,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None, "kernel": "whole batched pass (filter bytes / pass time); "
                         "per-problem blocks fit in L2, so the pass is launch- and latency-bound",
                         "peak_kind": peak_kind},
            "clocks": clk.summary(),
            "gpu_launches": launches,
            "e2e": e2e,
            "cpu_baseline": cpu,
        }))
    B.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
