"""ORACLE / TEST INFRASTRUCTURE ONLY — ctypes access to the CPU reference implementations.

* ``port``: liboracle.so, the plain-C restatement in hisq_oracle.c (always buildable with gcc).
* ``ref``:  _ref/libkuqcd_ref.so, the unmodified reference KuQCD sources compiled with a single-rank MPI shim
  (oracle/Makefile).  Present when the reference sources were available at build time.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this module: it is what GPU results are
compared with, never part of the product path.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libkuqcd_ref.so"
_port = None
_ref = None

vp, d, i32 = C.c_void_p, C.c_double, C.c_int


def _p(a):
    return a.ctypes.data_as(vp)


def build_port() -> Path:
    if not PORT_LIB.exists() or PORT_LIB.stat().st_mtime < (HERE / "hisq_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "port"], check=True)
    return PORT_LIB


def port() -> C.CDLL:
    global _port
    if _port is None:
        build_port()
        L = C.CDLL(str(PORT_LIB))
        L.kqo_true_residual_d.restype = d
        L.kqo_hash.restype = C.c_uint64
        L.kqo_hash.argtypes = [C.c_uint64, C.c_uint64]
        L.kqo_make_links.argtypes = [C.POINTER(i32), d, C.c_uint64, vp, vp, vp]
        L.kqo_make_source.argtypes = [C.POINTER(i32), i32, C.c_uint64, vp]
        L.kqo_cgm_d.argtypes = [C.POINTER(i32), vp, vp, i32, i32, C.POINTER(d), vp, C.POINTER(vp), d, i32]
        L.kqo_cgm_f.argtypes = [C.POINTER(i32), vp, vp, i32, i32, C.POINTER(C.c_float), vp, C.POINTER(vp), d, i32]
        L.kqo_true_residual_d.argtypes = [C.POINTER(i32), vp, vp, i32, d, vp, vp]
        _port = L
    return _port


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_LIB.exists():
            raise RuntimeError(f"{REF_LIB} missing: run `make -C oracle ref` where the reference sources exist")
        L = C.CDLL(str(REF_LIB))
        L.kqref_solve_multishift.argtypes = [C.POINTER(vp), vp, i32, i32, i32, i32, i32, d, C.POINTER(d),
                                             C.POINTER(i32)]
        L.kqref_set_grid1()
        _ref = L
    return _ref


def _dims(dims):
    return (i32 * 4)(*dims)


# ---------------------------------------------------------------- port (C restatement)
def make_links(dims, eps, seed, thin=False):
    V = int(np.prod(dims))
    fat, lng = np.zeros(V * 72), np.zeros(V * 72)
    th = np.zeros(V * 72) if thin else None
    port().kqo_make_links(_dims(dims), eps, seed, _p(fat), _p(lng), _p(th) if thin else None)
    return (fat, lng, th) if thin else (fat, lng)


def make_source(dims, parity, seed):
    b = np.zeros(int(np.prod(dims)) // 2 * 6)
    port().kqo_make_source(_dims(dims), parity, seed, _p(b))
    return b


def dslash(dims, fat, lng, src, dst_parity):
    out = np.zeros_like(src)
    f = port().kqo_dslash_d if src.dtype == np.float64 else port().kqo_dslash_f
    f(_dims(dims), _p(fat), _p(lng), _p(src), _p(out), dst_parity)
    return out


def dslash_full(dims, fat, lng, src):
    """Non-PC dslash on a full-lattice field (even sites then odd sites)."""
    out = np.zeros_like(src)
    port().kqo_dslash_full_d(_dims(dims), _p(fat), _p(lng), _p(src), _p(out))
    return out


def mdagm(dims, fat, lng, src, parity):
    out, tmp = np.zeros_like(src), np.zeros_like(src)
    port().kqo_mdaggm_d(_dims(dims), _p(fat), _p(lng), _p(src), _p(out), _p(tmp), parity)
    return out


def cgm(dims, fat, lng, parity, shifts_ref, b, tol, max_iter):
    """Reference-semantics multishift CG (shifts[j>=1] relative to shifts[0]); returns (xs, iterations)."""
    n = len(shifts_ref)
    xs = [np.zeros_like(b) for _ in range(n)]
    xp = (vp * n)(*[x.ctypes.data for x in xs])
    if b.dtype == np.float64:
        sh = (d * n)(*shifts_ref)
        it = port().kqo_cgm_d(_dims(dims), _p(fat), _p(lng), parity, n, sh, _p(b), xp, tol, max_iter)
    else:
        sh = (C.c_float * n)(*shifts_ref)
        it = port().kqo_cgm_f(_dims(dims), _p(fat), _p(lng), parity, n, sh, _p(b), xp, tol, max_iter)
    return xs, it


def true_residual(dims, fat, lng, parity, sigma, b, x):
    return port().kqo_true_residual_d(_dims(dims), _p(fat), _p(lng), parity, float(sigma), _p(b), _p(x))


# ---------------------------------------------------------------- reference library
def ref_dslash(dims, fat, lng, src, dst_parity, reps=1):
    """The reference's DiracHISQ::Dslash (one set-up of fields and neighbour tables, then `reps` applications)."""
    out = np.zeros_like(src)
    f = ref().kqref_dslash_d if src.dtype == np.float64 else ref().kqref_dslash_f
    st = f((C.c_uint * 4)(*dims), _p(fat), _p(lng), _p(src), _p(out), dst_parity, reps)
    assert st == 0
    return out


def ref_mdagm(dims, fat, lng, src, parity):
    """D_pq D_qp of the reference (MdaggM, no sigma)."""
    out = np.zeros_like(src)
    st = ref().kqref_mdaggm_d((C.c_uint * 4)(*dims), _p(fat), _p(lng), _p(src), _p(out), parity, 1)
    assert st == 0
    return out


def ref_dslash_full(dims, fat, lng, src):
    out = np.zeros_like(src)
    st = ref().kqref_dslash_full_d((C.c_uint * 4)(*dims), _p(fat), _p(lng), _p(src), _p(out))
    assert st == 0
    return out


def ref_solve(dims, fat, lng, b, shifts_ref, tol, max_iter, matpc=0, prec=None, order=0, dslash_type=3):
    """kuqcd_load_gaugefield x2 + kuqcd_solve_multishift of the reference; returns (status, xs, iter)."""
    L = ref()
    prec = prec or (8 if b.dtype == np.float64 else 4)
    lat = (C.c_uint * 4)(*dims)
    L.kqref_gauge_free()
    assert L.kqref_load_gaugefield(_p(fat), lat, prec, order, 1, 2, 0) == 0
    assert L.kqref_load_gaugefield(_p(lng), lat, prec, order, 2, 2, 0) == 0
    n = len(shifts_ref)
    xs = [np.zeros_like(b) for _ in range(n)]
    xp = (vp * n)(*[x.ctypes.data for x in xs])
    it = i32()
    st = L.kqref_solve_multishift(xp, _p(b), dslash_type, matpc, prec, n, max_iter, tol, (d * n)(*shifts_ref),
                                  C.byref(it))
    L.kqref_gauge_free()
    return st, xs, it.value


def hash64(seed, counter):
    return int(port().kqo_hash(seed, counter))
