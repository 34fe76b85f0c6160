"""Stand-alone HISQ dslash driver: applies the even-odd dslash `--reps` times on synthetic fields and prints the
achieved rate (1146 flop per output site; compulsory bytes 2400 / 1200 / 608 per site for DOUBLE / SINGLE /
HALF).  Used for profiling the dslash kernels in isolation.  With --ptc it applies the learned preconditioner
M = N^dag N (N: 1 -> 8 -> 8 channels, random weights) instead, four tensor-core PTC layers per application.

    python -m kuqcd_b200.dslash_bench --dims 32 32 32 32 --prec double --reps 20
    python -m kuqcd_b200.dslash_bench --dims 32 32 32 32 --ptc --reps 5

With --batch-sources N it solves N seeded sources on the one gauge field together with kq_batch_solve (mixed
solver, 12 shifts, per-shift true residual 1e-10; shape from KUQCD_BATCH_SHAPE or the tuner): the grouped
multi-right-hand-side dslash kernels in isolation from the rest of the batched workload.

    KUQCD_BATCH_SHAPE=256,8,4,2,0 python -m kuqcd_b200.dslash_bench --dims 24 24 24 48 --batch-sources 4
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

import kuqcd_b200 as K

PRECS = {"double": K.KUQCD_DOUBLE, "single": K.KUQCD_SINGLE, "half": K.KUQCD_HALF}
BYTES = {K.KUQCD_DOUBLE: 2400, K.KUQCD_SINGLE: 1200, K.KUQCD_HALF: 608}


def batch_sources(ctx, dims, n):
    """n seeded sources (parity 0, mass 0.03, 12 shifts 1e-4..1) solved together by kq_batch_solve."""
    Vh = int(np.prod(dims)) // 2
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    sig = list(0.03 ** 2 + np.logspace(-4, 0, 12))
    batch = K.Batch()
    keep = []
    for s in range(n):
        db = torch.empty(Vh * 6, dtype=torch.float64, device="cuda")
        ctx.make_source(0, 100 + s, db)
        d_b = torch.empty(vb, dtype=torch.uint8, device="cuda")
        ctx.upload(K.KUQCD_DOUBLE, db.cpu().numpy(), d_b)
        d_x = torch.empty(vb * len(sig), dtype=torch.uint8, device="cuda")
        batch.add(ctx, d_b, d_x, sig, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF, rel_residual=1e-10)
        keep.append((d_b, d_x))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    info = batch.solve()
    t = time.perf_counter() - t0
    print(json.dumps({"dims": list(dims), "batch_sources": n, "seconds": t,
                      "batched_ms": info.batched_seconds * 1e3, "iterations": info.iterations,
                      "shape": [info.tile, info.ctas_per_sm, info.rhs_per_cta, info.sites_per_thread,
                                info.fp64_rhs_per_pass], "max_true_residual": info.max_true_residual}))
    batch.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=4, default=[32, 32, 32, 32])
    ap.add_argument("--prec", choices=list(PRECS), nargs="+", default=["double"])
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--eps", type=float, default=0.3)
    ap.add_argument("--ptc", action="store_true", help="time the learned preconditioner's application instead")
    ap.add_argument("--batch-sources", type=int, default=0,
                    help="solve this many sources on the field with kq_batch_solve instead")
    args = ap.parse_args()
    dims = tuple(args.dims)
    V = int(np.prod(dims))
    Vh = V // 2
    ctx = K.Context(dims)
    dfat = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    dlng = torch.empty(V * 72, dtype=torch.float64, device="cuda")
    ctx.make_links(args.eps, 1, dfat, dlng)
    ctx.load_links(K.KUQCD_FAT_LINK, dfat.cpu().numpy())
    ctx.load_links(K.KUQCD_LONG_LINK, dlng.cpu().numpy())
    del dfat, dlng
    if args.batch_sources > 0:
        batch_sources(ctx, dims, args.batch_sources)
        return
    db = torch.empty(Vh * 6, dtype=torch.float64, device="cuda")
    ctx.make_source(1, 2, db)
    hb = db.cpu().numpy()
    if args.ptc:
        net = K.Net(ctx, (1, 8, 8))
        net.weights = (0.3 * np.random.default_rng(0).standard_normal(net.nw)).astype(np.float32)
        a = torch.zeros(ctx.spinor_bytes(K.KUQCD_DOUBLE), dtype=torch.uint8, device="cuda")
        o = torch.zeros_like(a)
        ctx.upload(K.KUQCD_DOUBLE, hb, a)
        for _ in range(args.warmup):
            net.apply(a, o, 1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.reps):
            net.apply(a, o, 1)  # returns after its stream has drained
        t = (time.perf_counter() - t0) / args.reps
        print(json.dumps({"dims": list(dims), "ptc_apply_ms": t * 1e3, "layers": 4}))
        net.close()
        return
    stream = torch.cuda.Stream()
    out = {}
    for name in args.prec:
        prec = PRECS[name]
        ctx.prepare(prec)
        a = torch.zeros(ctx.spinor_bytes(prec), dtype=torch.uint8, device="cuda")
        o = torch.zeros_like(a)
        ctx.upload(prec, hb, a)
        for _ in range(args.warmup):
            ctx.dslash(prec, a, o, 0, stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for r in range(args.reps):
            src, dst = (a, o) if r % 2 == 0 else (o, a)
            ctx.dslash(prec, src, dst, r % 2, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / args.reps * 1e-3
        out[name] = {"us": t * 1e6, "gflops": 1146 * Vh / t / 1e9, "gbs": BYTES[prec] * Vh / t / 1e9}
    print(json.dumps({"dims": list(dims), "dslash": out}))


if __name__ == "__main__":
    main()
