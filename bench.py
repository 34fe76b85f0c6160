#!/usr/bin/env python
"""Benchmark: HISQ multishift CG to a per-shift true relative residual of 1e-10 on one B200 per rank.

Workload (one step = one complete multishift solve of one system), default `--config 48`:
  48^3x96 lattice (Vh = 5,308,416 sites per parity), thin links U = exp(i*0.4*H) (seeded Gaussian traceless
  Hermitian H), staggered phases folded in, fat = 9/8 U, long = -1/24 U U U, mass m = 0.02, 16 shifts sigma_i
  log-spaced 1e-5..1 (absolute shifts m^2 + sigma_i), Gaussian even-site source.  Synthetic data generated on the
  device from a seed.  `--config 32` is the 32^4 case (eps 0.3, m 0.05, 12 shifts 1e-4..1); the default line also
  carries the 32^4 numbers under "lattice_32".

  value : solves/s over all ranks, inputs resident in HBM (kq_solve_multishift_device, relaxed-precision solver)
  plain_fp64 : the plain FP64 GPU multishift CG (the reference's recurrences) on the same system
  e2e   : the same metric through the reference-facing call kuqcd_solve_multishift with host (pinned) buffers,
          host<->device copies inside the timed region
  dslash : the FP64 / FP32 / HALF dslash, GFLOP/s at 1146 flop per site and GB/s
  roofline : the FP64 dslash (the solver's dominant kernel), bytes its storage moves / CUDA-event time
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
# Bytes a dslash moves per output site in its storage.  FP64: with the long links compressed (two rows + 1/s,
# 104 B) 8 x 144 + 8 x 104 + 96 = 2080, with full storage the compulsory 2400.  FP32: 8 x 72 + 8 x 52 + 48 = 1040
# or 1200.  HALF (no compression): 608.
DSLASH_STORAGE_BYTES = {(8, 1): 2080, (8, 0): 2400, (4, 1): 1040, (4, 0): 1200, (2, 1): 608, (2, 0): 608}
# DRAM traffic of one FP64 dslash_kernel launch per output site, from ncu (dram__bytes_read.sum +
# dram__bytes_write.sum at 32^4, Vh = 524,288: 1.073 GB compressed, profiles/dslash_fp64_recon_32x32x32x32.txt;
# 1.238 GB full storage, profiles/dslash_fp64_32x32x32x32.txt), scaled by output sites
DSLASH_FP64_TRAFFIC_PER_SITE = {1: 1.073e9 / 524288, 0: 1.238e9 / 524288}
# Workloads.  ref_iters: iterations the reference CGM (inverter_cgm.cpp:17-87) needs to converge on the workload
# (seed 1000, tol (1e-10)^2 |b|^2, reference-semantics shifts), counted by running the reference library
# (oracle/_ref) to convergence with oracle/ref_iterations.py: 295 at 32^4, 1057 at 48^3x96.
CONFIGS = {
    "32": dict(dims=(32, 32, 32, 32), eps=0.3, mass=0.05, nshift=12, smin=1e-4, ref_iters=295),
    "48": dict(dims=(48, 48, 48, 96), eps=0.4, mass=0.02, nshift=16, smin=1e-5, ref_iters=1057),
}
SEED = 1000


def shifts_abs(cfg):
    return list(cfg["mass"] ** 2 + np.logspace(np.log10(cfg["smin"]), 0, cfg["nshift"]))


def ref_shifts(cfg):
    """The reference's shift semantics: shifts[0] absolute, shifts[j >= 1] relative to it (inverter_cgm.cpp:51-56)."""
    sig = shifts_abs(cfg)
    return [sig[0]] + [s - sig[0] for s in sig[1:]]


def workload_name(cfg):
    return (f"multishift CG {'x'.join(map(str, cfg['dims']))}, {cfg['nshift']} shifts {cfg['smin']:g}..1, "
            f"m={cfg['mass']}, eps={cfg['eps']}, per-shift true residual {REL_RES}")


def workload_config(cfg, world):
    """The `config` object of both arms: what the workload is, nothing about how an arm solves it."""
    vh = int(np.prod(cfg["dims"])) // 2
    return {"workload": workload_name(cfg), "lattice": list(cfg["dims"]), "shifts": cfg["nshift"],
            "mass": cfg["mass"], "eps": cfg["eps"], "rel_residual": REL_RES,
            "l2": f"inputs larger than L2 (FP64 links {vh * 2 * 4 * 144 * 2 / 1e9:.1f} GB)",
            "parallelism": f"replicas x{world}"}


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


def measured_peak():
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
    except Exception:
        peaks = {}
    if peaks.get("hbm_gbs"):
        return float(peaks["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------------------------- our arm
def run_lattice(cfg, args, rank, world, local, steps, warmup, plain_steps, e2e_steps, clocks=True,
                windowed=False):
    """Everything measured on one lattice: the headline solver, the plain FP64 multishift, the dslash in three
    precisions and the end-to-end reference-facing call.  Returns a dict (rank 0) of the numbers."""
    import torch
    import torch.distributed as dist

    import kuqcd_b200 as K

    dims = tuple(cfg["dims"])
    V = int(np.prod(dims))
    Vh = V // 2
    nshift = cfg["nshift"]
    seed = SEED + rank
    sig = shifts_abs(cfg)
    ctx = K.Context(dims, device=local)
    dfat = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    dlng = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    ctx.make_links(cfg["eps"], seed, dfat, dlng)
    hfat, hlng = dfat.cpu().numpy(), dlng.cpu().numpy()
    del dfat, dlng
    ctx.load_links(K.KUQCD_FAT_LINK, hfat)
    ctx.load_links(K.KUQCD_LONG_LINK, hlng)
    db = torch.empty(Vh * 6, dtype=torch.float64, device="cuda")
    ctx.make_source(0, seed, db)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    d_b = torch.empty(vb, dtype=torch.uint8, device="cuda")
    hb = db.cpu().numpy()
    del db
    ctx.upload(K.KUQCD_DOUBLE, hb, d_b)
    d_x = torch.empty(vb * nshift, dtype=torch.uint8, device="cuda")
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

    def max_over_ranks(v):
        if world > 1:
            t = torch.tensor([v], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return v

    def timed(name, nsteps, nwarm, sample_clocks):
        """nwarm warm-up solves, then nsteps timed solves.  The solver runs on the context's stream and times
        itself there with CUDA events (info.seconds, between a barrier + synchronize on both sides); every solve
        returns after its stream has drained, and the wall clock around the loop is reported beside it."""
        kw = solver_kw(name)
        for _ in range(nwarm):
            ctx.solve_device(d_b, d_x, sig, **kw)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        iters, refine, dev_s, launches = [], [], 0.0, 0
        clk = ClockSampler(local) if sample_clocks else None
        if clk:
            clk.__enter__()
        try:
            torch.cuda.synchronize()
            w0 = time.perf_counter()
            for _ in range(nsteps):
                info = ctx.solve_device(d_b, d_x, sig, **kw)
                iters.append(info.iter)
                refine.append(info.iter_refine)
                dev_s += info.seconds
                launches += info.kernel_launches
            torch.cuda.synchronize()
            wall_s = time.perf_counter() - w0
        finally:
            if clk:
                clk.__exit__()
        if world > 1:
            dist.barrier()
        ms_step = max_over_ranks(dev_s * 1e3 / nsteps)
        true_res = ctx.true_residuals(0, sig, d_b, d_x)
        return dict(ms=ms_step, wall_ms=wall_s * 1e3 / nsteps, iters=iters[-1], refine=refine[-1],
                    launches=launches, true_res=max(true_res), sloppy_res=info.sloppy_residual, steps=nsteps,
                    clocks=clk.summary() if clk else None)

    # ---------------- dslash in three precisions: CUDA events on the (non-default) stream the kernels run on.  Timed
    # alone, before the solves (compared with the burst copy peak), with the SM clocks sampled meanwhile.
    dsl = {}
    stream = torch.cuda.Stream()
    peak, _ = measured_peak()
    dclk = ClockSampler(local) if clocks else None
    if dclk:
        dclk.__enter__()
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
        t = s0.elapsed_time(s1) / reps * 1e-3
        rc = ctx.long_links_compressed(prec)
        moved = DSLASH_STORAGE_BYTES[(prec, 1 if rc == 1 else 0)]
        dsl[name] = {"us": t * 1e6, "gflops": DSLASH_FLOPS * Vh / t / 1e9,
                     "gbs": moved * Vh / t / 1e9, "frac_of_measured_hbm": moved * Vh / t / 1e9 / peak,
                     "bytes_per_site": moved, "compulsory_bytes_per_site": DSLASH_BYTES[prec],
                     "compulsory_gbs": DSLASH_BYTES[prec] * Vh / t / 1e9, "long_links_compressed": bool(rc == 1)}
        del a, o
    if dclk:
        dclk.__exit__(None, None, None)
        dsl["clocks"] = dclk.summary()

    main_run = timed(args.solver, steps, warmup, clocks)
    plain = timed("fp64", plain_steps, 1, False) if args.solver != "fp64" else None
    plain_w = timed("fp64w", plain_steps, 1, False) if windowed and args.solver not in ("fp64", "fp64w") else None

    long_recon = ctx.long_links_compressed(K.KUQCD_DOUBLE)
    ctx.close()  # free its links and workspace before the API path loads its own copy
    del d_b, d_x
    torch.cuda.empty_cache()

    # ---------------- e2e: reference-facing call with pinned host buffers
    hb_pin = torch.from_numpy(hb).pin_memory()
    hx_pin = [torch.empty(Vh * 6, dtype=torch.float64).pin_memory() for _ in range(nshift)]
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
    refsh = ref_shifts(cfg)
    shc = (C.c_double * nshift)(*refsh)
    ip = K.KuQCDInvertParam(dslash_type=K.KUQCD_HISQPC_DIRAC, inverter_type=K.KUQCD_CGM,
                            matpc_type=K.KUQCD_EVEN_EVEN, prec=K.KUQCD_DOUBLE, num_shift=nshift, max_iter=100000,
                            iter=0, tol=(REL_RES ** 2) * bnorm2, shifts=C.cast(shc, C.POINTER(C.c_double)))
    xs_np = [x.numpy() for x in hx_pin]
    b_np = hb_pin.numpy()
    with quiet_stdout():
        for _ in range(1):
            assert K.kuqcd_solve_multishift(xs_np, b_np, ip) == 0
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            assert K.kuqcd_solve_multishift(xs_np, b_np, ip) == 0
        e2e_s = (time.perf_counter() - t0) / e2e_steps
    K.kuqcd_gauge_free()
    e2e_s = max_over_ranks(e2e_s)
    del hx_pin, hb_pin, xs_np, b_np
    torch.cuda.empty_cache()

    fp64 = dsl["fp64"]
    roofline = {"bound": "hbm", "kernel": "dslash_kernel<fp64>",
                "achieved": fp64["gbs"], "peak": peak, "peak_source": measured_peak()[1], "unit": "GB/s",
                "frac": fp64["frac_of_measured_hbm"],
                "bytes_per_site": fp64["bytes_per_site"],
                "bytes_note": ("bytes the FP64 storage moves per output site: 8 fat links x 144 B + 8 long links x "
                               + ("104 B (two rows + 1/s)" if long_recon == 1 else "144 B") +
                               " + 48 B in + 48 B out"),
                "algorithmic_bytes_per_launch": fp64["bytes_per_site"] * Vh,
                "compulsory_bytes_per_site": 2400, "compulsory_gbs": fp64["compulsory_gbs"],
                "compulsory_frac": fp64["compulsory_gbs"] / peak,
                "traffic": DSLASH_FP64_TRAFFIC_PER_SITE[1 if long_recon == 1 else 0] * Vh,
                "traffic_source": "ncu DRAM bytes of one launch at 32^4 (profiles/), scaled by output sites",
                "long_links_compressed": bool(long_recon == 1)}
    out = {"main": main_run, "plain": plain, "plain_w": plain_w, "dslash": dsl, "roofline": roofline,
           "e2e_s": e2e_s, "e2e_steps": e2e_steps, "hfat": hfat, "hlng": hlng, "hb": hb, "Vh": Vh,
           "nshift": nshift}
    return out


def plain_info(r, ms_step, world):
    if r is None:
        return None
    return {"ms_per_step": r["ms"], "steps": r["steps"], "iterations": r["iters"],
            "max_true_residual": r["true_res"], "solves_per_s": world * 1000.0 / r["ms"],
            "speedup_of_headline": r["ms"] / ms_step}


def run_ours(args):
    import torch
    import torch.distributed as dist

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=600))
    cfg = dict(CONFIGS[args.config])
    if args.dims:
        cfg["dims"] = tuple(args.dims)
    big = int(np.prod(cfg["dims"])) > 4 * 32 ** 4
    # auxiliary comparisons (plain FP64 solver, end-to-end call) take fewer steps on the large lattice, where one
    # plain FP64 solve takes seconds
    r = run_lattice(cfg, args, rank, world, local, args.steps, args.warmup,
                    plain_steps=min(args.steps, 3 if big else 10), e2e_steps=min(args.steps, 5 if big else 10),
                    windowed=not big)
    small = None
    if args.config == "48" and not args.dims and not args.no_extra:
        small = run_lattice(CONFIGS["32"], args, rank, world, local, args.steps, args.warmup,
                            plain_steps=min(args.steps, 10), e2e_steps=min(args.steps, 10), clocks=False,
                            windowed=True)
    main_run = r["main"]
    ms_step = main_run["ms"]
    Vh, nshift = r["Vh"], r["nshift"]

    result = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample(cfg, r["hfat"], r["hlng"], r["hb"], args.cpu_sample_iters)
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
            "config": workload_config(cfg, world),
            "solver": {"name": args.solver, "iterations": main_run["iters"], "refine_iterations": main_run["refine"],
                       "max_true_residual": main_run["true_res"], "sloppy_phase_residual": main_run["sloppy_res"]},
            "plain_fp64": plain_info(r["plain"], ms_step, world),
            "e2e": {"value": world / r["e2e_s"], "unit": "solves/s", "h2d_bytes_per_step": Vh * 6 * 8,
                    "d2h_bytes_per_step": nshift * Vh * 6 * 8, "steps": r["e2e_steps"], "warmup": 1,
                    "call": "kuqcd::kuqcd_solve_multishift (C twin), pinned host b and x"},
            "roofline": r["roofline"],
            "dslash": r["dslash"],
            "cpu_baseline": cpu,
            "gpu_launches": main_run["launches"],
            "clocks": main_run["clocks"],
            "wall_ms_per_step": main_run["wall_ms"],
        }
        if r["plain_w"] is not None:
            result["plain_fp64"]["windowed"] = plain_info(r["plain_w"], ms_step, world)
        if small is not None:
            sm = small["main"]
            result["lattice_32"] = {
                "config": workload_config(CONFIGS["32"], world), "value": world * 1000.0 / sm["ms"],
                "unit": "solves/s", "ms_per_step": sm["ms"], "steps": sm["steps"], "iterations": sm["iters"],
                "refine_iterations": sm["refine"], "max_true_residual": sm["true_res"],
                "plain_fp64": plain_info(small["plain"], sm["ms"], world),
                "e2e": {"value": world / small["e2e_s"], "unit": "solves/s", "steps": small["e2e_steps"],
                        "h2d_bytes_per_step": small["Vh"] * 6 * 8,
                        "d2h_bytes_per_step": small["nshift"] * small["Vh"] * 6 * 8},
                "dslash": small["dslash"], "gpu_launches": sm["launches"]}
            if small["plain_w"] is not None:
                result["lattice_32"]["plain_fp64"]["windowed"] = plain_info(small["plain_w"], sm["ms"], world)
        if small is not None and world == 1:
            # the batched workloads (24 systems on three lattices): two warm-up steps (the first tunes the launch
            # shape), the median of three timed steps; their own lines come from --config batch / batch-rhs
            bargs = argparse.Namespace(**vars(args))
            bargs.steps, bargs.warmup = 3, 2
            for name, shared in (("batch", False), ("batch_rhs", True)):
                b = run_batch(bargs, shared=shared, emit=False)
                result[name] = {k: b[k] for k in ("value", "unit", "ms_per_step", "steps", "warmup", "config",
                                                  "sequential", "gpu_launches", "clocks")}
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


# ---------------------------------------------------------------------------------------------- CPU reference
class RefSolver:
    """The reference library (oracle/_ref, all host cores) with the workload's gauge field loaded once; each solve()
    is one kuqcd_solve_multishift call (its own field set-up, neighbour tables and CGM iterations, as a caller of the
    reference pays them per solve)."""

    def __init__(self, cfg, fat, lng, b):
        from oracle import oracle as O

        self.O, self.L = O, O.ref()
        self.cfg, self.b = cfg, b
        self.lat = (C.c_uint * 4)(*cfg["dims"])
        self.L.kqref_gauge_free()
        with quiet_stdout():
            assert self.L.kqref_load_gaugefield(O._p(fat), self.lat, 8, 0, 1, 2, 0) == 0
            assert self.L.kqref_load_gaugefield(O._p(lng), self.lat, 8, 0, 2, 2, 0) == 0
        n = cfg["nshift"]
        self.xs = [np.zeros_like(b) for _ in range(n)]
        self.xp = (C.c_void_p * n)(*[x.ctypes.data for x in self.xs])
        self.sh = (C.c_double * n)(*ref_shifts(cfg))
        self.tol = (REL_RES ** 2) * float(b @ b)

    def solve(self, max_iter):
        it = C.c_int()
        with quiet_stdout():
            t0 = time.perf_counter()
            st = self.L.kqref_solve_multishift(self.xp, self.O._p(self.b), 3, 0, 8, self.cfg["nshift"], max_iter,
                                               self.tol, self.sh, C.byref(it))
            t = time.perf_counter() - t0
        assert st == 0
        return t, it.value

    def close(self):
        self.L.kqref_gauge_free()


def ref_fields(cfg):
    """The workload's fields for the reference, generated on the host by the oracle's generator (the device
    generator implements the same algorithm)."""
    from oracle import oracle as O

    fat, lng = O.make_links(cfg["dims"], cfg["eps"], SEED)
    return fat, lng, O.make_source(cfg["dims"], 0, SEED)


def ref_dslash_seconds(cfg, fat, lng, b, reps=10):
    """Seconds per FP64 DiracHISQ::Dslash of the reference on the workload's fields: a call applying it 1 + reps
    times minus a call applying it once (field set-up and neighbour tables cancel)."""
    from oracle import oracle as O

    t = []
    with quiet_stdout():
        for n in (1, 1 + reps):
            t0 = time.perf_counter()
            O.ref_dslash(cfg["dims"], fat, lng, b, 1, reps=n)
            t.append(time.perf_counter() - t0)
    return max(t[1] - t[0], 0.0) / reps or t[1] / (1 + reps)


def ref_sample(rs, cfg, sample_iters):
    """Extrapolated time of one complete reference solve from a bounded sample: t(1) (one solve call stopped after
    its first iteration: set-up plus one iteration) and t(1 + n) give the per-iteration cost; a complete solve of N
    iterations costs t(1) + (N - 1) (t(1 + n) - t(1)) / n."""
    t1, it1 = rs.solve(1)
    tn, itn = rs.solve(1 + sample_iters)
    assert it1 == 1 and itn == 1 + sample_iters
    per_iter = max(tn - t1, 0.0) / sample_iters or tn / (1 + sample_iters)
    return t1 + (cfg["ref_iters"] - 1) * per_iter, t1, per_iter


def cpu_baseline_sample(cfg, fat, lng, b, sample_iters):
    from oracle import oracle as O

    if not O.ref_available():
        return None
    rs = RefSolver(cfg, fat, lng, b)
    solve_s, t1, per_iter = ref_sample(rs, cfg, sample_iters)
    rs.close()
    t_d = ref_dslash_seconds(cfg, fat, lng, b)
    vh = int(np.prod(cfg["dims"])) // 2
    return {"value": 1.0 / solve_s, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
            "extrapolated": True, "seconds_per_solve": solve_s, "seconds_first_iteration": t1,
            "seconds_per_iteration": per_iter, "iterations_to_converge": cfg["ref_iters"],
            "dslash_ms": t_d * 1e3, "dslash_gbs": 2400.0 * vh / t_d / 1e9,
            "dslash_gflops": DSLASH_FLOPS * vh / t_d / 1e9,
            "sample": f"EXTRAPOLATED: reference kuqcd_solve_multishift calls stopped after 1 and {1 + sample_iters} "
                      f"iterations on the same workload (FP64, {os.cpu_count()} OpenMP threads), scaled to the "
                      f"{cfg['ref_iters']} iterations the reference needs to converge; FP64 dslash: mean of 10 "
                      f"applications (compulsory 2400 B per output site)"}


def run_reference(args):
    """The reference arm: the reference's own CPU library (oracle/_ref, unmodified sources, all host cores) on the
    workload of the default arm.  On 32^4 every timed step is one complete kuqcd_solve_multishift (about 15 s); on
    48^3x96, where a complete solve takes about 10 minutes, every step is a bounded sample extrapolated to the
    reference's iteration count (labelled so), and the line also carries one complete, timed 32^4 solve."""
    rank, world, local = dist_env()
    if rank != 0:
        return None
    from oracle import oracle as O

    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkuqcd_ref.so was not built"}))
        return None
    cfg = dict(CONFIGS[args.config])
    if args.dims:
        cfg["dims"] = tuple(args.dims)
    complete = int(np.prod(cfg["dims"])) <= 32 ** 4
    fat, lng, b = ref_fields(cfg)
    rs = RefSolver(cfg, fat, lng, b)
    if complete:
        for _ in range(args.warmup):
            rs.solve(1)  # warm-up: one solve call stopped after one iteration (a complete solve per step follows)
        runs = [rs.solve(100000) for _ in range(args.steps)]
        solve_s = float(np.mean([t for t, _ in runs]))
        iters = runs[-1][1]
        xs_res = None
        sample = (f"{args.steps} complete reference kuqcd_solve_multishift solves to convergence ({iters} "
                  f"iterations each), FP64, {os.cpu_count()} OpenMP threads; warm-up: solves stopped after one "
                  f"iteration")
        extra = {"extrapolated": False, "iterations": iters}
        tol_ok = [O.true_residual(cfg["dims"], fat, lng, 0, s, b, x) for s, x in zip(shifts_abs(cfg), rs.xs)]
        extra["max_true_residual"] = max(tol_ok)
    else:
        for _ in range(args.warmup):
            rs.solve(1)
        samples = [ref_sample(rs, cfg, args.cpu_sample_iters) for _ in range(args.steps)]
        solve_s = float(np.mean([s[0] for s in samples]))
        sample = (f"EXTRAPOLATED: each step times reference kuqcd_solve_multishift calls stopped after 1 and "
                  f"{1 + args.cpu_sample_iters} iterations (FP64, {os.cpu_count()} OpenMP threads) and scales them "
                  f"to the {cfg['ref_iters']} iterations the reference needs to converge on this workload (counted "
                  f"by running the reference to convergence)")
        extra = {"extrapolated": True, "iterations_to_converge": cfg["ref_iters"],
                 "seconds_first_iteration": float(np.mean([s[1] for s in samples])),
                 "seconds_per_iteration": float(np.mean([s[2] for s in samples]))}
    rs.close()
    t_d = ref_dslash_seconds(cfg, fat, lng, b)
    vh = int(np.prod(cfg["dims"])) // 2
    v = 1.0 / solve_s
    res = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded on the host, same generator algorithm)",
        "config": workload_config(cfg, world),
        "solver": dict({"name": "reference CGM (CPU, oracle/_ref)"}, **extra),
        "cpu_baseline": dict({"value": v, "unit": "solves/s", "cores": os.cpu_count(), "kind": "reference",
                              "sample": sample, "dslash_ms": t_d * 1e3, "dslash_gbs": 2400.0 * vh / t_d / 1e9,
                              "dslash_gflops": DSLASH_FLOPS * vh / t_d / 1e9}, **extra),
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    del fat, lng
    if not complete and not args.dims and not args.no_extra:
        c32 = CONFIGS["32"]
        f32, l32, b32 = ref_fields(c32)
        rs = RefSolver(c32, f32, l32, b32)
        t, it = rs.solve(100000)
        rs.close()
        res["lattice_32"] = {"config": workload_config(c32, world), "value": 1.0 / t, "unit": "solves/s",
                             "seconds_per_solve": t, "iterations": it, "extrapolated": False,
                             "sample": "one complete reference kuqcd_solve_multishift solve to convergence, FP64, "
                                       f"{os.cpu_count()} OpenMP threads"}
    print(json.dumps(res))
    return res


def run_batch(args, shared=False, emit=True):
    """Batched multi-system workload: 24 systems, 8 each on 16^4, 24^3x48 and 32^4, own gauge field
    (eps ~ U[0.2,0.4]), own mass (m ~ U[0.01,0.1]), 8-16 shifts log-spaced 1e-4..1 and Gaussian source, all seeded.
    With shared=True (--config batch-rhs) the 8 systems of a lattice are 8 sources on one gauge field with one mass
    and shift set (the multi-right-hand-side case: propagators of several sources on one configuration), so the
    grouped dslash loads each link once for all of them.
    One step = all 24 solved to per-shift true residual 1e-10 by kq_batch_solve (persistent launches over every
    system's tiles, CUDA graphs, autotuned shape); compared with the same 24 solved one after another."""
    import torch

    import kuqcd_b200 as K

    torch.cuda.set_device(0)
    rng = np.random.default_rng(4242)
    lattices = [(16, 16, 16, 16)] * 8 + [(24, 24, 24, 48)] * 8 + [(32, 32, 32, 32)] * 8
    systems = []
    field_ctx = {}
    per_field = {}
    for i, dims in enumerate(lattices):
        eps, mass, ns = rng.uniform(0.2, 0.4), rng.uniform(0.01, 0.1), int(rng.integers(8, 17))
        if shared:  # one mass and shift set per gauge field
            eps, mass, ns = per_field.setdefault(dims, (eps, mass, ns))
        V, Vh = int(np.prod(dims)), int(np.prod(dims)) // 2
        if shared and dims in field_ctx:
            ctx = field_ctx[dims]
        else:
            ctx = K.Context(dims)
            dfat = torch.empty(V * 72, dtype=torch.float64, device="cuda")
            dlng = torch.empty(V * 72, dtype=torch.float64, device="cuda")
            ctx.make_links(eps, 5000 + i, dfat, dlng)
            ctx.load_links(K.KUQCD_FAT_LINK, dfat.cpu().numpy())
            ctx.load_links(K.KUQCD_LONG_LINK, dlng.cpu().numpy())
            del dfat, dlng
            field_ctx[dims] = ctx
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
        worst, iters, refine = 0.0, 0, 0
        for ctx, d_b, d_x, sig, dims in systems:
            inf = ctx.solve_device(d_b, d_x, sig, solver=K.KQ_SOLVER_MIXED, prec=prec, rel_residual=REL_RES)
            worst = max(worst, max(inf.true_residual[:len(sig)]))
            iters = max(iters, inf.iter)
            refine += inf.iter_refine
        return time.perf_counter() - t0, worst, iters, refine

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
        "config": {"workload": ("24 systems: 8 x 16^4, 8 x 24^3x48, 8 x 32^4; "
                                + ("8 sources on one gauge field per lattice (eps, m, shift set per field: "
                                   "eps U[0.2,0.4], m U[0.01,0.1], 8-16 shifts 1e-4..1)"
                                   if shared else "eps U[0.2,0.4], own gauge field each, m U[0.01,0.1], 8-16 "
                                                  "shifts 1e-4..1")
                                + ", per-shift true residual 1e-10"),
                   "solver": "kq_batch_solve (mixed)", "gauge_fields": len(set(id(c) for c, *_ in systems)),
                   "tile": info.tile, "ctas_per_sm": info.ctas_per_sm, "rhs_per_cta": info.rhs_per_cta,
                   "sites_per_thread": info.sites_per_thread, "fp64_rhs_per_pass": info.fp64_rhs_per_pass,
                   "groups": info.groups,
                   "max_iterations": info.iterations, "refined_systems": info.refined_systems,
                   "refine_iterations": info.refine_iterations,
                   "batched_phase_ms": info.batched_seconds * 1e3, "check_refine_ms": info.check_seconds * 1e3,
                   "max_true_residual": bt[-1][2]},
        "sequential": {"ms_per_step": t_s * 1e3, "max_true_residual": st[-1][1], "refine_iterations": st[-1][3],
                       "speedup_of_batched": t_s / t_b},
        "gpu_launches": int(info.kernel_launches), "clocks": clk.summary(),
    }
    if emit:
        print(json.dumps(res))
    bobj.close()
    for ctx in set(c for c, *_ in systems):
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
    ap.add_argument("--config", choices=list(CONFIGS) + ["batch", "batch-rhs", "learned"], default="48")
    ap.add_argument("--learned-train", type=int, default=20)
    ap.add_argument("--learned-test", type=int, default=5)
    ap.add_argument("--learned-pairs", type=int, default=2)
    ap.add_argument("--learned-net-max-shift", type=float, default=0.01)
    ap.add_argument("--learned-steps", type=int, default=300)
    ap.add_argument("--dims", type=int, nargs=4, default=None, help="override the lattice of --config")
    ap.add_argument("--cpu-sample-iters", type=int, default=None,
                    help="iterations of the reference's sampled solves (default 4 on 48^3x96, 10 otherwise)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="48^3x96: skip the 32^4 numbers of the same line")
    args = ap.parse_args()
    if args.config == "learned":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no preconditioned solver"}))
        else:
            run_learned(args)
        return
    if args.config in ("batch", "batch-rhs"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the batched workload has no reference "
                                                                  "counterpart; run the reference per system"}))
        else:
            run_batch(args, shared=args.config == "batch-rhs")
        return
    if args.cpu_sample_iters is None:
        dims = args.dims or CONFIGS[args.config]["dims"]
        args.cpu_sample_iters = 4 if int(np.prod(dims)) > 4 * 32 ** 4 else 10
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
