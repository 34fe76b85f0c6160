"""The C++ boundary a KuQCD caller compiles against: include/kuqcd.h with its five kuqcd:: calls (C++ linkage, the
mangled symbols of libkuqcd_b200.so) and the class-level API it brings in (Lattice, LattBase, GaugeField,
SpinorField + BLAS-1, DiracHISQ, CGM).

* The reference's own test program (test/test_solver.cpp), compiled unmodified against include/ at build time, runs
  on the GPU and passes its known-answer test.
* A C++ caller of the five calls solves BASELINE's 8^4 configuration (12 shifts, per-shift relative residual 1e-10);
  its solutions match the oracle's CGM.
* A C++ caller of the class API: Dslash (FP64, FP32, BATCH_ORDER FP32 with 16 lanes), MdaggM, the BLAS-1 functions
  and CGM::Invert against the oracle.
"""
import os
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

ROOT = Path(__file__).resolve().parents[1]
CPP = ROOT / "tests" / "cpp"
LIB = ROOT / "kuqcd_b200"


def compile_caller(name, out_dir):
    exe = Path(out_dir) / name
    cmd = ["g++", "-std=c++17", "-O2", "-I", str(ROOT / "include"), str(CPP / f"{name}.cpp"), "-L", str(LIB),
           "-lkuqcd_b200", f"-Wl,-rpath,{LIB}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def run(cmd, cwd=None):
    env = dict(os.environ, KUQCD_DEVICE="0")
    r = subprocess.run([str(c) for c in cmd], capture_output=True, text=True, cwd=cwd, env=env, timeout=600)
    return r


def shifts_8x4():
    mass, sig = 0.05, np.logspace(-4, 0, 12)
    absolute = list(mass * mass + sig)
    return absolute, [absolute[0]] + [s - absolute[0] for s in absolute[1:]]


@pytest.mark.gpu
def test_reference_test_solver_compiled_against_our_headers(cuda):
    exe = CPP / "_build" / "test_solver_ref"
    if not exe.exists():
        pytest.skip("tests/cpp/_build/test_solver_ref is built by build() where the reference sources are present")
    r = run([exe])
    assert r.returncode == 0, r.stdout + r.stderr
    passed = [ln for ln in r.stdout.splitlines() if "PASSED" in ln]
    assert len(passed) == 2, r.stdout
    assert "end test kuqcd_solve_multishift PASSED" in r.stdout and "1 tests ran, 1 tests PASSED" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("matpc", [0, 1])
def test_cpp_caller_of_the_five_calls_8x4(cuda, tmp_path, matpc):
    """BASELINE's 8^4 configuration through the mangled kuqcd:: calls from C++: eps 0.3, fat 9/8 U, long -1/24 UUU,
    m = 0.05, 12 shifts 1e-4..1, tol (1e-10)^2 |b|^2 on the reference's stopping rule."""
    exe = compile_caller("caller_kuqcd", tmp_path)
    dims = (8, 8, 8, 8)
    fat, lng = O.make_links(dims, 0.3, 1000)
    b = O.make_source(dims, matpc, 1000)
    absolute, refsh = shifts_8x4()
    tol = 1e-20 * float(b @ b)
    fat.tofile(tmp_path / "fat.bin")
    lng.tofile(tmp_path / "long.bin")
    b.tofile(tmp_path / "b.bin")
    np.array(refsh).tofile(tmp_path / "shifts.bin")
    np.array([tol]).tofile(tmp_path / "tol.bin")
    r = run([exe, tmp_path, *dims, len(refsh), 8, matpc])
    assert r.returncode == 0, r.stdout + r.stderr
    st, it = map(int, (tmp_path / "result.txt").read_text().split())
    assert st == 0
    xo, ito = O.cgm(dims, fat, lng, matpc, refsh, b, tol, 100000)
    assert abs(it - ito) <= 1, (it, ito)
    for k, s in enumerate(absolute):
        x = np.fromfile(tmp_path / f"x{k}.bin")
        assert np.abs(x - xo[k]).max() <= 1e-9 * np.abs(xo[k]).max(), k
        assert O.true_residual(dims, fat, lng, matpc, s, b, x) <= 1.5e-10, k


@pytest.mark.gpu
def test_cpp_caller_of_the_class_api(cuda, tmp_path):
    exe = compile_caller("caller_classes", tmp_path)
    dims = (32, 4, 4, 4)  # nx = 32: the width a 16-lane BATCH_ORDER float field needs
    fat, lng = O.make_links(dims, 0.3, 77)
    be, bo = O.make_source(dims, 0, 5), O.make_source(dims, 1, 6)
    absolute, refsh = shifts_8x4()
    refsh = refsh[:4]
    absolute = absolute[:4]
    tol = 1e-20 * float(be @ be)
    for name, a in [("fat", fat), ("long", lng), ("b_even", be), ("b_odd", bo)]:
        a.tofile(tmp_path / f"{name}.bin")
    np.array(refsh).tofile(tmp_path / "shifts.bin")
    np.array([tol]).tofile(tmp_path / "tol.bin")
    r = run([exe, tmp_path, *dims, len(refsh)])
    assert r.returncode == 0, r.stdout + r.stderr
    assert "caller_classes done" in r.stdout

    def rel(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())

    d_even = O.dslash(dims, fat, lng, bo, 0)
    assert rel(np.fromfile(tmp_path / "dslash_even.bin"), d_even) <= 1e-13
    assert rel(np.fromfile(tmp_path / "dslash_even_f.bin", dtype=np.float32).astype(np.float64), d_even) <= 2e-6
    assert rel(np.fromfile(tmp_path / "dslash_batch.bin", dtype=np.float32).astype(np.float64), d_even) <= 2e-6
    x = O.mdagm(dims, fat, lng, be, 0)  # D D b (the reference's MdaggM)
    assert rel(np.fromfile(tmp_path / "mdaggm_even.bin"), x) <= 1e-13

    n2, dot, nrm = map(float, (tmp_path / "blas.txt").read_text().split())
    assert n2 == pytest.approx(float(be @ be), rel=1e-13)
    assert dot == pytest.approx(float(be @ x), rel=1e-12)
    assert nrm == pytest.approx(float(np.sqrt(x @ x)), rel=1e-13)
    y = be.copy()
    y = y + 0.25 * x
    y = 2.0 * be - y
    y = y + 0.5 * x
    y = 3.0 * be + 0.5 * y
    u = 2.0 * (y - be) - be + x
    assert rel(np.fromfile(tmp_path / "axpby.bin"), u) <= 1e-14

    it = int((tmp_path / "cgm.txt").read_text())
    xo, ito = O.cgm(dims, fat, lng, 0, refsh, be, tol, 100000)
    assert abs(it - ito) <= 1
    for k, s in enumerate(absolute):
        xk = np.fromfile(tmp_path / f"x{k}.bin")
        assert rel(xk, xo[k]) <= 1e-9
        assert O.true_residual(dims, fat, lng, 0, s, be, xk) <= 1.5e-10
