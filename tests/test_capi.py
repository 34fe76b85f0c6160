"""CPU tests of the C ABI: the library loads, exports every symbol include/*.h declares, and the reference-facing
calls return the reference's status codes on every validation branch that precedes device work
(kuqcd.cpp:45-57,176-199,306-332,404-414,443-444)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import kuqcd_b200 as K
from kuqcd_b200 import lib as L

ROOT = Path(__file__).resolve().parent.parent


def declared_c_functions():
    txt = (ROOT / "include" / "kuqcd_b200.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(kq_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_declared_symbols():
    lib = K.library()
    declared = declared_c_functions()
    assert declared, "no kq_ declarations found"
    assert sorted(L.EXPORTED_SYMBOLS) == declared
    for name in declared:
        assert hasattr(lib, name), name


def test_cpp_api_symbols_are_mangled_like_the_reference():
    out = subprocess.run(["nm", "-D", "--defined-only", str(L.lib_path)], capture_output=True, text=True).stdout
    for sym in ["_ZN5kuqcd10kuqcd_initEv", "_ZN5kuqcd21kuqcd_load_gaugefieldEPvP15KuQCDGaugeParam",
                "_ZN5kuqcd22kuqcd_solve_multishiftEPPvS0_P16KuQCDInvertParam", "_ZN5kuqcd16kuqcd_gauge_freeEv",
                "_ZN5kuqcd9kuqcd_endEv"]:
        assert sym in out, sym


def test_struct_layouts_match_reference_header():
    # kuqcd_enum.h:100-121: 4 uint + 7 int-sized fields; InvertParam has tol at offset 32, shifts at 40
    assert C.sizeof(K.KuQCDGaugeParam) == 44
    assert K.KuQCDInvertParam.tol.offset == 32 and K.KuQCDInvertParam.shifts.offset == 40
    assert C.sizeof(K.KuQCDInvertParam) == 48


def gauge_param(**kw):
    p = K.KuQCDGaugeParam()
    p.lat[:] = kw.get("lat", (4, 4, 4, 4))
    p.halo_depth = 0
    p.od = K.KUQCD_TZYX_ORDER
    p.site_subset = kw.get("site_subset", K.KUQCD_ALL)
    p.gauge_order = kw.get("order", K.KUQCD_NORMAL_ORDER)
    p.prec = kw.get("prec", K.KUQCD_DOUBLE)
    p.link_type = kw.get("link_type", K.KUQCD_FAT_LINK)
    p.recon = kw.get("recon", K.KUQCD_GAUGE_RECON_NO)
    return p


@pytest.mark.parametrize("kw,expect", [
    (dict(order=5), K.KUQCD_ERR_INVALID_PARAM),
    (dict(link_type=K.KUQCD_WILSON_LINK), K.KUQCD_ERR_INVALID_PARAM),
    (dict(recon=K.KUQCD_GAUGE_RECON_12), K.KUQCD_ERR_UNSUPPORTED),
    (dict(recon=K.KUQCD_GAUGE_RECON_U14), K.KUQCD_ERR_UNSUPPORTED),
    (dict(recon=3), K.KUQCD_ERR_INVALID_PARAM),
    (dict(lat=(4, 0, 4, 4)), K.KUQCD_ERR_INVALID_PARAM),
    (dict(prec=K.KUQCD_HALF), K.KUQCD_ERR_UNSUPPORTED),
    (dict(prec=3), K.KUQCD_ERR_INVALID_PARAM),
    (dict(site_subset=7), K.KUQCD_ERR_INVALID_PARAM),
    (dict(site_subset=K.KUQCD_EVEN), K.KUQCD_ERR_INVALID_PARAM),
    (dict(lat=(5, 4, 4, 4)), K.KUQCD_ERR_INVALID_PARAM),
    (dict(order=K.KUQCD_BATCH_ORDER, prec=K.KUQCD_DOUBLE, lat=(8, 4, 4, 4)), K.KUQCD_ERR_INVALID_PARAM),
])
def test_load_gaugefield_validation(kw, expect):
    h = np.zeros(16)
    assert K.kuqcd_load_gaugefield(h, gauge_param(**kw)) == expect


def test_load_gaugefield_null_pointers():
    assert K.kuqcd_load_gaugefield(None, gauge_param()) == K.KUQCD_ERR_NULL_POINTER
    assert K.kuqcd_load_gaugefield(np.zeros(4), None) == K.KUQCD_ERR_NULL_POINTER


def invert_param(**kw):
    sh = (C.c_double * 1)(0.1)
    p = K.KuQCDInvertParam(dslash_type=kw.get("dslash", K.KUQCD_HISQPC_DIRAC), inverter_type=kw.get("inv", K.KUQCD_CGM),
                           matpc_type=kw.get("matpc", K.KUQCD_EVEN_EVEN), prec=K.KUQCD_DOUBLE,
                           num_shift=kw.get("ns", 1), max_iter=100, iter=0, tol=1e-10,
                           shifts=C.cast(sh, C.POINTER(C.c_double)))
    p._keep = sh
    return p


def test_solve_before_load_and_null_pointers():
    K.kuqcd_gauge_free()
    b = np.zeros(6)
    assert K.kuqcd_solve_multishift([b], b, invert_param()) == K.KUQCD_ERR_UNKNOWN_TYPE
    assert K.kuqcd_solve_multishift(None, b, invert_param()) == K.KUQCD_ERR_NULL_POINTER
    assert K.kuqcd_solve_multishift([b], None, invert_param()) == K.KUQCD_ERR_NULL_POINTER
    assert K.kuqcd_solve_multishift([b], b, None) == K.KUQCD_ERR_NULL_POINTER
    assert K.kuqcd_solve_multishift([b], b, invert_param(matpc=4)) == K.KUQCD_ERR_INVALID_PARAM


def test_init_grid_must_be_one_rank(monkeypatch):
    monkeypatch.setenv("KUQCD_GRID", "1,1,1,1")
    assert K.kuqcd_init() == K.KUQCD_SUCCESS
    monkeypatch.setenv("KUQCD_GRID", "2,1,1,1")
    assert K.kuqcd_init() == K.KUQCD_ERR_INVALID_PARAM
    monkeypatch.setenv("KUQCD_GRID", "1,1,1,1")
    assert K.kuqcd_init() == K.KUQCD_SUCCESS


def test_context_argument_checks():
    lib = K.library()
    h = C.c_void_p()
    assert lib.kq_context_create(None, 0, C.byref(h)) == K.KUQCD_ERR_NULL_POINTER
    assert lib.kq_context_create((C.c_uint * 4)(4, 4, 0, 4), 0, C.byref(h)) == K.KUQCD_ERR_INVALID_PARAM
    assert lib.kq_context_create((C.c_uint * 4)(3, 4, 4, 4), 0, C.byref(h)) == K.KUQCD_ERR_INVALID_PARAM
    assert lib.kq_dslash(None, 8, None, None, 0, None) == K.KUQCD_ERR_NULL_POINTER
    assert lib.kq_solve_multishift(None, None, None, None, None) == K.KUQCD_ERR_NULL_POINTER


@pytest.mark.parametrize("caller", ["caller_kuqcd", "caller_classes"])
def test_cpp_callers_compile_against_include_and_link(tmp_path, caller):
    """include/kuqcd.h and the class-level headers it brings in compile warning-free (-Wall -Wextra -Werror) in a
    C++ caller, and the caller links against libkuqcd_b200.so (the mangled kuqcd:: symbols and the C ABI)."""
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", str(ROOT / "include"),
           str(ROOT / "tests" / "cpp" / f"{caller}.cpp"), "-L", str(ROOT / "kuqcd_b200"), "-lkuqcd_b200",
           "-o", str(tmp_path / caller)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
