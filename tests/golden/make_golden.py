"""Regenerate tests/golden/golden.npz from the reference itself.

The outputs come from oracle/_ref/libkuqcd_ref.so, the UNMODIFIED reference sources compiled where they lie by
`make -C oracle ref` (oracle/ref_bridge.cpp drives DiracHISQ::Dslash, DiracHISQ::MdaggM and
kuqcd_solve_multishift).  The inputs are the seeded synthetic fields of oracle/hisq_oracle.c (make_links,
make_source); each case stores the SHA-256 of its input arrays, so a change of the generator shows up as a
fixture mismatch rather than as a silent change of what is compared.

    python tests/golden/make_golden.py        # in a checkout where the reference library can be built

Cases (all FP64 unless named):
  dslash_<lattice>_p<p>   one even-odd dslash onto parity p    (dirac_hisq.cpp:409-502)
  dslash_f32_<lattice>    the same in FP32                      (DiracHISQ<float,...>)
  full_<lattice>          non-PC dslash on a full-lattice field (KUQCD_HISQ_DIRAC, dirac_hisq.cpp:128-136, 418-424)
  mdaggm_<lattice>        D_pq D_qp                             (dirac_hisq.cpp:457-462)
  cgm_<lattice>           kuqcd_solve_multishift, 6 shifts, reference shift semantics, tol (1e-10)^2 |b|^2
  kat_test_solver         the reference's own known-answer test (test/test_solver.cpp: float 4x4x4x1, every
                          input 1.0, one shift, ODD_ODD, tol 1e-4; expected x = 0.007561)
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent / "golden.npz"
EPS, LINK_SEED = 0.3, 7
DSLASH_LATTICES = [(8, 8, 8, 8), (6, 4, 2, 8), (4, 4, 4, 1), (2, 3, 5, 4)]


def sha(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def name(dims):
    return "x".join(map(str, dims))


def main():
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libkuqcd_ref.so is missing: run `make -C oracle ref` first")
    out = {}
    for dims in DSLASH_LATTICES:
        fat, lng = O.make_links(dims, EPS, LINK_SEED)
        for p in (0, 1):
            src = O.make_source(dims, 1 - p, 11)
            out[f"dslash_{name(dims)}_p{p}"] = O.ref_dslash(dims, fat, lng, src, p)
            out[f"dslash_{name(dims)}_p{p}_sha"] = np.array(sha(fat, lng, src))
    dims = (6, 4, 2, 8)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    f32 = (fat.astype(np.float32), lng.astype(np.float32), O.make_source(dims, 1, 11).astype(np.float32))
    out[f"dslash_f32_{name(dims)}"] = O.ref_dslash(dims, *f32, 0)
    out[f"dslash_f32_{name(dims)}_sha"] = np.array(sha(*f32))
    for dims in [(4, 4, 4, 8), (6, 2, 4, 2)]:
        fat, lng = O.make_links(dims, EPS, LINK_SEED)
        src = np.concatenate([O.make_source(dims, 0, 12), O.make_source(dims, 1, 13)])
        out[f"full_{name(dims)}"] = O.ref_dslash_full(dims, fat, lng, src)
        out[f"full_{name(dims)}_sha"] = np.array(sha(fat, lng, src))
    dims = (4, 4, 4, 4)
    fat, lng = O.make_links(dims, EPS, LINK_SEED)
    src = O.make_source(dims, 0, 14)
    out[f"mdaggm_{name(dims)}"] = O.ref_mdagm(dims, fat, lng, src, 0)
    out[f"mdaggm_{name(dims)}_sha"] = np.array(sha(fat, lng, src))
    # multishift: m = 0.05, sigma 1e-4..1 absolute; reference call passes shifts[0] absolute, others relative
    dims = (4, 4, 4, 4)
    fat, lng = O.make_links(dims, EPS, 21)
    b = O.make_source(dims, 0, 5)
    ab = 0.05 ** 2 + np.logspace(-4, 0, 6)
    refsh = np.array([ab[0]] + list(ab[1:] - ab[0]))
    tol = (1e-10) ** 2 * float(b @ b)
    st, xs, it = O.ref_solve(dims, fat, lng, b, list(refsh), tol, 5000)
    assert st == 0
    out[f"cgm_{name(dims)}_x"] = np.stack(xs)
    out[f"cgm_{name(dims)}_iter"] = np.array(it)
    out[f"cgm_{name(dims)}_shifts"] = refsh
    out[f"cgm_{name(dims)}_tol"] = np.array(tol)
    out[f"cgm_{name(dims)}_sha"] = np.array(sha(fat, lng, b))
    # the reference's known-answer test
    dims = (4, 4, 4, 1)
    V = int(np.prod(dims))
    one = np.ones(V * 72, np.float32)
    bk = np.ones(V // 2 * 6, np.float32)
    st, xk, itk = O.ref_solve(dims, one, one, bk, [3.671676313381e-05], 1e-4, 6500, matpc=1)
    assert st == 0
    out["kat_test_solver_x"] = xk[0]
    out["kat_test_solver_iter"] = np.array(itk)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
