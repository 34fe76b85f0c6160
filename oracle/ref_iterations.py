"""ORACLE / TEST INFRASTRUCTURE ONLY — runs the reference CGM (oracle/_ref) to convergence on the bench workload
and prints its iteration count and per-shift FP64 true residuals.  bench.py records the count it prints, so that
its CPU-baseline legs can time a bounded sample of iterations and extrapolate to a full solve.

    python -m oracle.ref_iterations 32          # 32^4, eps 0.3, m 0.05, 12 shifts 1e-4..1
    python -m oracle.ref_iterations 48          # 48^3x96, eps 0.4, m 0.02, 16 shifts 1e-5..1 (about 33 GB of RAM)
"""
import sys
import time

import numpy as np

from oracle import oracle as O


CONFIGS = {
    "32": dict(dims=(32, 32, 32, 32), eps=0.3, mass=0.05, nshift=12, smin=1e-4),
    "48": dict(dims=(48, 48, 48, 96), eps=0.4, mass=0.02, nshift=16, smin=1e-5),
}


def main(dims, eps=0.3, mass=0.05, nshift=12, smin=1e-4, rel=1e-10, seed=1000):
    fat, lng = O.make_links(dims, eps, seed)
    b = O.make_source(dims, 0, seed)
    sig = list(mass * mass + np.logspace(np.log10(smin), 0, nshift))
    refsh = [sig[0]] + [s - sig[0] for s in sig[1:]]
    tol = rel * rel * float(b @ b)
    t0 = time.perf_counter()
    st, xs, it = O.ref_solve(dims, fat, lng, b, refsh, tol, 100000)
    t1 = time.perf_counter()
    print(f"dims={dims} status={st} iterations={it} seconds={t1 - t0:.1f}", flush=True)
    res = [O.true_residual(dims, fat, lng, 0, s, b, x) for s, x in zip(sig, xs)]
    print(f"per-shift true residuals: {' '.join(f'{r:.3e}' for r in res)}; max {max(res):.3e}")


if __name__ == "__main__":
    main(**CONFIGS[sys.argv[1]])
