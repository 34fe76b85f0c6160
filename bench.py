#!/usr/bin/env python
"""Benchmark: HISQ multishift CG to a per-shift true relative residual of 1e-10 on one B200 per rank.

Workload (one step = one complete multishift solve of one system):
  32^4 lattice, thin links U = exp(i*0.3*H) (seeded Gaussian traceless Hermitian H), staggered phases folded in,
  fat = 9/8 U, long = -1/24 U U U, mass m = 0.05, 12 shifts sigma_i log-spaced 1e-4..1 (absolute shifts
  m^2 + sigma_i), Gaussian even-site source.  Synthetic data generated on the device from a seed.

  value : solves/s over all ranks, inputs resident in HBM (kq_solve_multishift_device)
  e2e   : the same through the reference-facing call kuqcd_solve_multishift with host (pinned) buffers,
          host<->device copies inside the timed region
  roofline : the dominant kernel (the dslash of the solver's precision), algorithmic bytes / CUDA-event time
  cpu_baseline : the reference's own CPU solver (oracle/_ref, all host cores) on a bounded sample of the solve

`--impl reference` times the reference CPU implementation alone (rank 0) and prints its own JSON line.
Multi-GPU: every rank solves an independent system (different seed): weak scaling, no data-path collective.
"""
from __future__ import annotations

import argparse
import ctypes as C
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

METRIC = "HISQ dslash GFLOP/s + HBM GB/s; multishift CG time to 1e-10, mixed vs plain FP64"
REL_RES = 1e-10
DSLASH_FLOPS = 1146          # per output site
DSLASH_BYTES = {8: 2400, 4: 1200, 2: 608}   # compulsory bytes per output site: 16 links + 1 in + 1 out spinor
# Bytes an FP64 dslash moves per output site in its storage: with the long links compressed (two rows + 1/s,
# 104 B) 8 x 144 + 8 x 104 + 96 = 2080; with full storage the compulsory 2400.
DSLASH_FP64_STORAGE_BYTES = {1: 2080, 0: 2400}
# DRAM traffic of one FP64 dslash_kernel launch per output site, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum at 32^4, Vh = 524,288: 1.073 GB compressed, profiles/dslash_fp64_recon_32x32x32x32.txt;
# 1.238 GB full storage, profiles/dslash_fp64_32x32x32x32.txt), scaled by sites
DSLASH_FP64_TRAFFIC_PER_SITE = {1: 1.073e9 / 524288, 0: 1.238e9 / 524288}
# Workloads.  "32": 32^4, eps 0.3, m 0.05, 12 shifts 1e-4..1 (the default).  "48": 48^3x96, eps 0.4, m 0.02,
# 16 shifts 1e-5..1.  ref_iters: iterations the reference CGM (inverter_cgm.cpp:17-87) needs on the workload
# (seed 1000, tol (1e-10)^2 |b|^2, reference-semantics shifts): for 32^4 counted by running oracle/ref_iterations.py
# to convergence; for 48^3x96 (hours on a CPU) the count of the GPU solver that reproduces the reference's
# recurrences in kernel order (KQ_SOLVER_CGM, same count as the reference on every tested lattice).
CONFIGS = {
    "32": dict(dims=(32, 32, 32, 32), eps=0.3, mass=0.05, nshift=12, smin=1e-4, ref_iters=295),
    "48": dict(dims=(48, 48, 48, 96), eps=0.4, mass=0.02, nshift=16, smin=1e-5, ref_iters=None),
}
DIMS, EPS, MASS, NSHIFT, SMIN, REF_ITERS = (32, 32, 32, 32), 0.3, 0.05, 12, 1e-4, 295


def select_config(name):
    global DIMS, EPS, MASS, NSHIFT, SMIN, REF_ITERS
    c = CONFIGS[name]
    DIMS, EPS, MASS, NSHIFT, SMIN, REF_ITERS = c["dims"], c["eps"], c["mass"], c["nshift"], c["smin"], c["ref_iters"]


def shifts_abs():
    return list(MASS * MASS + np.logspace(np.log10(SMIN), 0, NSHIFT))


def workload_name(dims):
    return (f"multishift CG {'x'.join(map(str, dims))}, {NSHIFT} shifts {SMIN:g}..1, m={MASS}, eps={EPS}, "
            f"per-shift true residual {REL_RES}")


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
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
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist

    import kuqcd_b200 as K

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))
    dims = tuple(args.dims)
    V = int(np.prod(dims))
    Vh = V // 2
    seed = 1000 + rank
    ctx = K.Context(dims, device=local)
    dfat = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    dlng = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    ctx.make_links(EPS, seed, dfat, dlng)
    hfat, hlng = dfat.cpu().numpy(), dlng.cpu().numpy()
    del dfat, dlng
    ctx.load_links(K.KUQCD_FAT_LINK, hfat)
    ctx.load_links(K.KUQCD_LONG_LINK, hlng)
    db = torch.empty(Vh * 6, dtype=torch.float64, device="cuda")
    ctx.make_source(0, seed, db)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    d_b = torch.empty(vb, dtype=torch.uint8, device="cuda")
    ctx.upload(K.KUQCD_DOUBLE, db.cpu().numpy(), d_b)
    d_x = torch.empty(vb * NSHIFT, dtype=torch.uint8, device="cuda")
    sig = shifts_abs()
    hb = db.cpu().numpy()
    bnorm2 = float(hb @ hb)

    sloppy = {"mixed": K.KUQCD_SINGLE, "mixed-half": K.KUQCD_HALF}

    def solver_kw(name):
        if name in ("fp64", "fp64w"):
            # plain CGM stopping rule tol = (rel * |b|)^2 on the recursive residual of every shift; "fp64" keeps the
            # reference's kernel order, "fp64w" defers the shift updates over windows of 16 iterations
            return dict(parity=0, solver=K.KQ_SOLVER_CGM if name == "fp64" else K.KQ_SOLVER_CGM_WINDOWED,
                        prec=K.KUQCD_DOUBLE, max_iter=100000, tol=(REL_RES ** 2) * bnorm2, shift_mode=1)
        return dict(parity=0, solver=K.KQ_SOLVER_MIXED, prec=sloppy[name], max_iter=100000, rel_residual=REL_RES,
                    shift_mode=1)

    def timed(name, clock=None):
        """W warm-up solves, then K timed solves.  The solver runs on the context's stream and times itself there
        with CUDA events (info.seconds); every solve returns after its stream has drained, and the wall clock
        around the loop is reported beside the device time."""
        kw = solver_kw(name)
        for _ in range(args.warmup):
            ctx.solve_device(d_b, d_x, sig, **kw)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        iters, refine, dev_s, launches = [], [], 0.0, 0
        with (clock or ClockSampler(local)) as clk:
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            for _ in range(args.steps):
                info = ctx.solve_device(d_b, d_x, sig, **kw)
                iters.append(info.iter)
                refine.append(info.iter_refine)
                dev_s += info.seconds
                launches += info.kernel_launches
            torch.cuda.synchronize()
            wall_s = time.perf_counter() - w0
        ms_step = dev_s * 1e3 / args.steps
        true_res = ctx.true_residuals(0, sig, d_b, d_x)
        if world > 1:
            t = torch.tensor([ms_step], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_step = float(t.item())
            dist.barrier()
        return dict(ms=ms_step, wall_ms=wall_s * 1e3 / args.steps, iters=iters[-1], refine=refine[-1],
                    launches=launches, true_res=max(true_res), sloppy_res=info.sloppy_residual, clocks=clk.summary())

    plain = timed("fp64") if args.solver != "fp64" else None
    plain_w = timed("fp64w") if args.solver not in ("fp64", "fp64w") else None
    main_run = timed(args.solver)
    ms_step, iters, true_res = main_run["ms"], [main_run["iters"]], [main_run["true_res"]]
    wall_s = main_run["wall_ms"] * 1e-3 * args.steps

    # ---------------- dslash roofline: the solver's dominant kernel, CUDA events on the launching stream
    dsl = {}
    # a dedicated (non-default) torch stream: the kernels run where the events are recorded
    stream = torch.cuda.Stream()
    long_recon = ctx.long_links_compressed(K.KUQCD_DOUBLE)
    for name, prec in [("fp64", K.KUQCD_DOUBLE), ("fp32", K.KUQCD_SINGLE), ("half", K.KUQCD_HALF)]:
        nbp = ctx.spinor_bytes(prec)
        a = torch.zeros(nbp, dtype=torch.uint8, device="cuda")
        o = torch.zeros(nbp, dtype=torch.uint8, device="cuda")
        ctx.convert(d_b, K.KUQCD_DOUBLE, a, prec, stream.cuda_stream)
        for _ in range(3):
            ctx.dslash(prec, a, o, 1, stream.cuda_stream)
        reps = 20
        s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for r in range(reps):
            ctx.dslash(prec, a if r % 2 == 0 else o, o if r % 2 == 0 else a, 1 - (r % 2), stream.cuda_stream)
        s1.record(stream)
        torch.cuda.synchronize()
        t_launch = s0.elapsed_time(s1) / reps * 1e-3
        dsl[name] = {"ms": t_launch * 1e3, "gflops": DSLASH_FLOPS * Vh / t_launch / 1e9,
                     "gbs": DSLASH_BYTES[prec] * Vh / t_launch / 1e9}
    ctx.close()  # free its links and workspace before the API path loads its own copy

    # ---------------- e2e: reference-facing call with pinned host buffers
    hb_pin = torch.from_numpy(hb).pin_memory()
    hx_pin = [torch.empty(Vh * 6, dtype=torch.float64).pin_memory() for _ in range(NSHIFT)]
    os.environ["KUQCD_SOLVER"] = args.solver
    K.kuqcd_gauge_free()
    K.kuqcd_init()
    gp = K.KuQCDGaugeParam()
    gp.lat[:] = dims
    gp.halo_depth, gp.od, gp.site_subset = 0, K.KUQCD_TZYX_ORDER, K.KUQCD_ALL
    gp.gauge_order, gp.prec, gp.recon = K.KUQCD_NORMAL_ORDER, K.KUQCD_DOUBLE, K.KUQCD_GAUGE_RECON_NO
    gp.link_type = K.KUQCD_FAT_LINK
    assert K.kuqcd_load_gaugefield(hfat, gp) == 0
    gp.link_type = K.KUQCD_LONG_LINK
    assert K.kuqcd_load_gaugefield(hlng, gp) == 0
    refsh = [sig[0]] + [s - sig[0] for s in sig[1:]]
    shc = (C.c_double * NSHIFT)(*refsh)
    ip = K.KuQCDInvertParam(dslash_type=K.KUQCD_HISQPC_DIRAC, inverter_type=K.KUQCD_CGM,
                            matpc_type=K.KUQCD_EVEN_EVEN, prec=K.KUQCD_DOUBLE, num_shift=NSHIFT, max_iter=100000,
                            iter=0, tol=(REL_RES ** 2) * bnorm2, shifts=C.cast(shc, C.POINTER(C.c_double)))
    xs_np = [x.numpy() for x in hx_pin]
    b_np = hb_pin.numpy()
    with quiet_stdout():
        for _ in range(max(1, args.warmup)):
            assert K.kuqcd_solve_multishift(xs_np, b_np, ip) == 0
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            assert K.kuqcd_solve_multishift(xs_np, b_np, ip) == 0
        e2e_s = (time.perf_counter() - t0) / args.steps
    K.kuqcd_gauge_free()
    if world > 1:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())

    # the FP64 operator dominates every solver (the relaxed schedule runs it while |r| > rho32 |b|)
    dom = "fp64"
    peaks = {}
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = peaks.get("hbm_gbs")
    peak_note = "measured" if peak else "fallback"
    peak = peak or 6650.0
    achieved = dsl[dom]["gbs"]  # the compulsory 2400 B per site (18 reals per link)
    storage_gbs = DSLASH_FP64_STORAGE_BYTES[long_recon] * Vh / (dsl[dom]["ms"] * 1e-3) / 1e9

    result = None
    if rank == 0:
        cpu = (cpu_baseline_sample(args, plain["iters"] if plain else None)
               if (world == 1 and not args.no_cpu_baseline) else None)
        launches = main_run["launches"]
        plain_info = None
        if plain is not None:
            plain_info = {"ms_per_step": plain["ms"], "iterations": plain["iters"],
                          "max_true_residual": plain["true_res"], "solves_per_s": world * 1000.0 / plain["ms"],
                          "speedup_of_headline": plain["ms"] / ms_step}
            if plain_w is not None:
                plain_info["windowed"] = {"ms_per_step": plain_w["ms"], "iterations": plain_w["iters"],
                                          "max_true_residual": plain_w["true_res"],
                                          "speedup_of_headline": plain_w["ms"] / ms_step}
        result = {
            "metric": METRIC,
            "value": world * 1000.0 / ms_step,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp64w": "f64", "mixed": "f64+f32", "mixed-half": "f64+f32+f16(int16+norm)"}[
                args.solver],
            "data": "synthetic (seeded on device: exp(i eps H) thin links, Gaussian source)",
            "config": {"workload": workload_name(dims),
                       "solver": args.solver, "lattice": list(dims), "shifts": NSHIFT,
                       "iterations": iters[-1], "refine_iterations": main_run["refine"],
                       "max_true_residual": max(true_res), "sloppy_phase_residual": main_run["sloppy_res"],
                       "l2": "inputs larger than L2 (links 1.2 GB FP64)", "parallelism": f"replicas x{world}"},
            "plain_fp64": plain_info,
            "e2e": {"value": world / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": Vh * 6 * 8,
                    "d2h_bytes_per_step": NSHIFT * Vh * 6 * 8},
            "roofline": {"bound": "hbm", "kernel": f"dslash_kernel<{dom}>", "achieved": achieved, "peak": peak,
                         "peak_source": peak_note, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": DSLASH_FP64_TRAFFIC_PER_SITE[long_recon] * Vh,
                         "traffic_source": "ncu DRAM bytes of one launch at 32^4, scaled by output sites",
                         "algorithmic_bytes": DSLASH_BYTES[8] * Vh,
                         "bytes_per_site": DSLASH_BYTES[8 if dom == 'fp64' else 4],
                         "long_links_compressed": bool(long_recon),
                         "storage_bytes_per_site": DSLASH_FP64_STORAGE_BYTES[long_recon],
                         "storage_gbs": storage_gbs, "storage_frac": storage_gbs / peak},
            "dslash": dsl,
            "cpu_baseline": cpu,
            "gpu_launches": launches,
            "clocks": main_run["clocks"],
            "wall_ms_per_step": wall_s * 1e3 / args.steps,
        }
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


# ---------------------------------------------------------------------------------------------- CPU reference
def ref_iterations_needed():
    return REF_ITERS


class quiet_stdout:
    """Send the C libraries' printf output (the reference's "CGM: # iterations" lines) to stderr, so that stdout
    carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


_REF_FIELDS = {}


def ref_cpu_time_per_iter(dims, sample_iters, seed=1000):
    """Seconds per CGM iteration of the reference (oracle/_ref, all host cores) on the bench workload: the time of a
    (1 + sample_iters)-iteration solve minus that of a 1-iteration solve, so that gauge loading, neighbour-table
    construction and field copies (paid once per solve call) cancel."""
    from oracle import oracle as O

    key = (tuple(dims), seed)
    if key not in _REF_FIELDS:
        fat, lng = O.make_links(dims, EPS, seed)
        _REF_FIELDS.clear()
        _REF_FIELDS[key] = (fat, lng, O.make_source(dims, 0, seed))
    fat, lng, b = _REF_FIELDS[key]
    sig = shifts_abs()
    refsh = [sig[0]] + [s - sig[0] for s in sig[1:]]
    tol = (REL_RES ** 2) * float(b @ b)
    t = []
    with quiet_stdout():
        for n in (1, 1 + sample_iters):
            t0 = time.perf_counter()
            st, xs, it = O.ref_solve(dims, fat, lng, b, refsh, tol, n)
            t.append(time.perf_counter() - t0)
            assert st == 0 and it == n
    per_iter = (t[1] - t[0]) / sample_iters
    if per_iter <= 0.0:
        # on a lattice so small that timer noise exceeds the iterations' cost: charge the whole longer solve
        per_iter = t[1] / (1 + sample_iters)
    return per_iter


def ref_cpu_dslash_seconds(dims, reps=10, seed=1000):
    """Seconds per FP64 DiracHISQ::Dslash of the reference (oracle/_ref, all host cores) on the bench's fields: a call
    applying it 1 + reps times minus a call applying it once (field set-up and neighbour tables cancel)."""
    from oracle import oracle as O

    key = (tuple(dims), seed)
    if key not in _REF_FIELDS:
        fat, lng = O.make_links(dims, EPS, seed)
        _REF_FIELDS.clear()
        _REF_FIELDS[key] = (fat, lng, O.make_source(dims, 0, seed))
    fat, lng, b = _REF_FIELDS[key]
    t = []
    with quiet_stdout():
        for n in (1, 1 + reps):
            t0 = time.perf_counter()
            O.ref_dslash(dims, fat, lng, b, 1, reps=n)
            t.append(time.perf_counter() - t0)
    return max(t[1] - t[0], 0.0) / reps or t[1] / (1 + reps)


def cpu_baseline_sample(args, iters_hint=None):
    from oracle import oracle as O

    if not O.ref_available():
        return None
    dims = tuple(args.dims)
    sample = args.cpu_sample_iters
    t_it = ref_cpu_time_per_iter(dims, sample)
    iters = ref_iterations_needed() or iters_hint or 0
    solve_s = t_it * iters if iters else None
    t_d = ref_cpu_dslash_seconds(dims)
    vh = int(np.prod(dims)) // 2
    return {"value": (1.0 / solve_s) if solve_s else None, "unit": "solves/s", "cores": os.cpu_count(),
            "kind": "reference", "seconds_per_iteration": t_it,
            "dslash_ms": t_d * 1e3, "dslash_gbs": 2400.0 * vh / t_d / 1e9,
            "sample": f"{sample} CGM iterations of the reference on the same workload, extrapolated to "
                      f"{iters} iterations (its iteration count to convergence); FP64 dslash: mean of 10 "
                      f"applications (compulsory 2400 B per output site)"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return None
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkuqcd_ref.so was not built"}))
        return None
    dims = tuple(args.dims)
    sample = args.cpu_sample_iters
    for _ in range(args.warmup):
        ref_cpu_time_per_iter(dims, max(1, sample // 4))
    times = [ref_cpu_time_per_iter(dims, sample) for _ in range(args.steps)]
    t_it = float(np.mean(times))
    iters = ref_iterations_needed()
    solve_s = t_it * iters
    v = 1.0 / solve_s
    t_d = ref_cpu_dslash_seconds(dims)
    res = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": workload_name(dims), "solver": "reference CGM (CPU)"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
                         "seconds_per_iteration": t_it, "dslash_ms": t_d * 1e3,
                         "dslash_gbs": 2400.0 * (int(np.prod(dims)) // 2) / t_d / 1e9,
                         "sample": f"{sample} CGM iterations per step, extrapolated to {iters} iterations; FP64 "
                                   f"dslash: mean of 10 applications"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(res))
    return res


def run_batch(args):
    """Batched multi-system workload: 24 independent systems, 8 each on 16^4, 24^3x48 and 32^4, own gauge field
    (eps ~ U[0.2,0.4]), mass (m ~ U[0.01,0.1]), 8-16 shifts log-spaced 1e-4..1 and Gaussian source, all seeded.
    One step = all 24 solved to per-shift true residual 1e-10 by kq_batch_solve (persistent launches over every
    system's tiles, CUDA graphs, autotuned shape); compared with the same 24 solved one after another."""
    import torch

    import kuqcd_b200 as K

    torch.cuda.set_device(0)
    rng = np.random.default_rng(4242)
    lattices = [(16, 16, 16, 16)] * 8 + [(24, 24, 24, 48)] * 8 + [(32, 32, 32, 32)] * 8
    systems = []
    for i, dims in enumerate(lattices):
        eps, mass, ns = rng.uniform(0.2, 0.4), rng.uniform(0.01, 0.1), int(rng.integers(8, 17))
        V, Vh = int(np.prod(dims)), int(np.prod(dims)) // 2
        ctx = K.Context(dims)
        dfat = torch.empty(V * 72, dtype=torch.float64, device="cuda")
        dlng = torch.empty(V * 72, dtype=torch.float64, device="cuda")
        ctx.make_links(eps, 5000 + i, dfat, dlng)
        ctx.load_links(K.KUQCD_FAT_LINK, dfat.cpu().numpy())
        ctx.load_links(K.KUQCD_LONG_LINK, dlng.cpu().numpy())
        del dfat, dlng
        db = torch.empty(Vh * 6, dtype=torch.float64, device="cuda")
        ctx.make_source(0, 5000 + i, db)
        vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
        d_b = torch.empty(vb, dtype=torch.uint8, device="cuda")
        ctx.upload(K.KUQCD_DOUBLE, db.cpu().numpy(), d_b)
        d_x = torch.empty(vb * ns, dtype=torch.uint8, device="cuda")
        sig = list(mass * mass + np.logspace(-4, 0, ns))
        systems.append((ctx, d_b, d_x, sig, dims))
    prec = K.KUQCD_HALF if args.solver == "mixed-half" else K.KUQCD_SINGLE

    # the batch object is built once and re-solved every step, as the single-system contexts keep their
    # workspaces between solves
    bobj = K.Batch()
    for ctx, d_b, d_x, sig, dims in systems:
        bobj.add(ctx, d_b, d_x, sig, solver=K.KQ_SOLVER_MIXED, prec=prec, rel_residual=REL_RES)

    def batched():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        info = bobj.solve()
        t = time.perf_counter() - t0
        worst = max(max(bobj.system_info(i).true_residual[:len(systems[i][3])]) for i in range(len(systems)))
        return t, info, worst

    def sequential():
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        worst, iters = 0.0, 0
        for ctx, d_b, d_x, sig, dims in systems:
            inf = ctx.solve_device(d_b, d_x, sig, solver=K.KQ_SOLVER_MIXED, prec=prec, rel_residual=REL_RES)
            worst = max(worst, max(inf.true_residual[:len(sig)]))
            iters = max(iters, inf.iter)
        return time.perf_counter() - t0, worst, iters

    for _ in range(args.warmup):
        batched()
    with ClockSampler(0) as clk:
        bt = [batched() for _ in range(args.steps)]
    sequential()
    st = [sequential() for _ in range(args.steps)]
    t_b = float(np.median([x[0] for x in bt]))
    t_s = float(np.median([x[0] for x in st]))
    info = bt[-1][1]
    res = {
        "metric": METRIC, "value": len(systems) / t_b, "unit": "systems/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_b * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32" + ("+f16(int16+norm)" if prec == K.KUQCD_HALF else ""),
        "data": "synthetic (seeded on device)",
        "config": {"workload": "24 systems: 8 x 16^4, 8 x 24^3x48, 8 x 32^4; eps U[0.2,0.4], m U[0.01,0.1], 8-16 "
                               "shifts 1e-4..1, per-shift true residual 1e-10", "solver": "kq_batch_solve (mixed)",
                   "tile": info.tile, "ctas_per_sm": info.ctas_per_sm, "max_iterations": info.iterations,
                   "refined_systems": info.refined_systems, "max_true_residual": bt[-1][2]},
        "sequential": {"ms_per_step": t_s * 1e3, "max_true_residual": st[-1][1], "speedup_of_batched": t_s / t_b},
        "gpu_launches": int(info.kernel_launches), "clocks": clk.summary(),
    }
    print(json.dumps(res))
    bobj.close()
    for ctx, *_ in systems:
        ctx.close()
    return res


def run_learned(args):
    """Learned-preconditioner workload: 32^4, eps 0.45, m 0.01, 12 shifts 1e-4..1.  The preconditioner M = N^dag N
    of a 2-layer, 8-channel parallel-transport chain N is trained on residual/error pairs from the plain solver over
    20 seeded gauge fields and evaluated on 5 held-out seeds: multishift CG to 1e-6 then per-shift FCG polish to
    1e-10 (with the network on the shifts <= --learned-net-max-shift), against the plain FP64 multishift CG to 1e-10
    and against the same polish without the network."""
    import torch

    import kuqcd_b200 as K
    from kuqcd_b200 import learned as LN

    torch.cuda.set_device(0)
    dims = tuple(args.dims) if args.dims else (32, 32, 32, 32)
    eps, mass, ns = 0.45, 0.01, 12
    sig = list(mass * mass + np.logspace(-4, 0, ns))
    ntrain, ntest = args.learned_train, args.learned_test
    V, Vh = int(np.prod(dims)), int(np.prod(dims)) // 2

    def field_ctx(seed):
        ctx = K.Context(dims)
        f = torch.empty(V * 72, dtype=torch.float64, device="cuda")
        l = torch.empty_like(f)
        ctx.make_links(eps, seed, f, l)
        ctx.load_links(K.KUQCD_FAT_LINK, f.cpu().numpy())
        ctx.load_links(K.KUQCD_LONG_LINK, l.cpu().numpy())
        return ctx

    t0 = time.perf_counter()
    train_ctx = [field_ctx(7000 + s) for s in range(ntrain)]
    data = [(c, LN.make_pairs(c, sig[0], args.learned_pairs, 100 * i)) for i, c in enumerate(train_ctx)]
    t_data = time.perf_counter() - t0
    chans = (1, 8, 8)
    net = K.Net(train_ctx[0], chans)
    c0 = float(np.mean([np.sqrt(e2 / float((r.view(torch.float64) ** 2).sum())) for c, ps in data
                        for r, e, e2 in ps]))
    net.weights = LN.init_weights(chans, c0)
    loss0 = LN.eval_loss(net, data)
    t0 = time.perf_counter()
    losses = LN.train(net, data, steps=args.learned_steps, lr=5e-3, batch=4)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    for c in train_ctx:
        c.close()

    rows = []
    for s in range(ntest):
        ctx = field_ctx(9000 + s)
        db = LN.gaussian_source(ctx, 0, 9000 + s)
        vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
        bh = ctx.download(K.KUQCD_DOUBLE, db)
        bb = float(bh @ bh)
        dx = torch.zeros(ns * vb, dtype=torch.uint8, device="cuda")
        row = {}
        for name in ("plain", "polish_net", "polish_cg"):
            torch.cuda.synchronize()
            t = time.perf_counter()
            if name == "plain":
                inf = ctx.solve_device(db, dx, sig, solver=K.KQ_SOLVER_CGM_WINDOWED, tol=REL_RES ** 2 * bb)
                its = inf.iter
            else:
                ms, pol = LN.solve_with_polish(ctx, net if name == "polish_net" else None, db, dx, sig,
                                               target=REL_RES, net_max_shift=args.learned_net_max_shift)
                its = (ms.iter, pol.iter_refine, pol.iter)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t
            res = max(ctx.true_residuals(0, sig, db, dx))
            row[name] = {"seconds": dt, "iterations": its, "max_true_residual": res}
        rows.append(row)
        ctx.close()
    mean = lambda k: float(np.mean([r[k]["seconds"] for r in rows]))
    res = {
        "metric": METRIC, "value": 1.0 / mean("polish_net"), "unit": "solves/s", "n_gpus": 1,
        "steps": ntest, "warmup": 0, "ms_per_step": 1e3 * mean("polish_net"), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (+bf16/f32 network)", "data": "synthetic (seeded)",
        "config": {"workload": f"learned preconditioner {'x'.join(map(str, dims))}, eps {eps}, m {mass}, {ns} shifts "
                               "1e-4..1: multishift to 1e-6 + per-shift FCG to 1e-10",
                   "train_fields": ntrain, "test_fields": ntest, "pairs_per_field": args.learned_pairs,
                   "train_steps": args.learned_steps, "net_max_shift": args.learned_net_max_shift,
                   "channels": list(chans), "loss_before": loss0, "loss_after": float(np.mean(losses[-10:])),
                   "data_seconds": t_data, "train_seconds": t_train},
        "plain_fp64_seconds": mean("plain"), "polish_without_net_seconds": mean("polish_cg"),
        "per_field": rows,
    }
    print(json.dumps(res))
    net.close()
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--solver", choices=["mixed", "mixed-half", "fp64", "fp64w"], default="mixed-half")
    ap.add_argument("--config", choices=list(CONFIGS) + ["batch", "learned"], default="32")
    ap.add_argument("--learned-train", type=int, default=20)
    ap.add_argument("--learned-test", type=int, default=5)
    ap.add_argument("--learned-pairs", type=int, default=2)
    ap.add_argument("--learned-net-max-shift", type=float, default=0.01)
    ap.add_argument("--learned-steps", type=int, default=300)
    ap.add_argument("--dims", type=int, nargs=4, default=None, help="override the lattice of --config")
    ap.add_argument("--cpu-sample-iters", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.config == "learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no preconditioned solver"}))
        else:
            run_learned(args)
        return
    if args.config == "batch":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched workload has no reference "
                                                                  "counterpart; run the reference per system"}))
        else:
            run_batch(args)
        return
    select_config(args.config)
    if args.dims is None:
        args.dims = list(DIMS)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
