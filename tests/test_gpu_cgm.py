"""GPU parity of the multishift CG through the reference-facing API (kuqcd_load_gaugefield / kuqcd_solve_multishift)
against the reference library (oracle/_ref) or, where it is absent, the oracle port; FP64 true residuals checked
per shift.  Tolerances: solutions within 1e-9 relative of the reference's, true residual <= 1e-10 x 1.5 (the
reference's own stopping rule is on the recursive residual), iteration counts within 1."""
import ctypes as C

import numpy as np
import pytest

import kuqcd_b200 as K
from oracle import oracle as O


def gparam(dims, link, prec=K.KUQCD_DOUBLE, order=K.KUQCD_NORMAL_ORDER):
    p = K.KuQCDGaugeParam()
    p.lat[:] = dims
    p.halo_depth = 3
    p.od = K.KUQCD_TZYX_ORDER
    p.site_subset = K.KUQCD_ALL
    p.gauge_order = order
    p.prec = prec
    p.link_type = link
    p.recon = K.KUQCD_GAUGE_RECON_NO
    return p


def iparam(shifts, tol, max_iter, matpc=K.KUQCD_EVEN_EVEN, prec=K.KUQCD_DOUBLE):
    sh = (C.c_double * len(shifts))(*shifts)
    p = K.KuQCDInvertParam(dslash_type=K.KUQCD_HISQPC_DIRAC, inverter_type=K.KUQCD_CGM, matpc_type=matpc,
                           prec=prec, num_shift=len(shifts), max_iter=max_iter, iter=0, tol=tol,
                           shifts=C.cast(sh, C.POINTER(C.c_double)))
    p._keep = sh
    return p


def api_solve(dims, fat, lng, b, shifts, tol, max_iter, matpc=0, order=K.KUQCD_NORMAL_ORDER):
    prec = K.KUQCD_DOUBLE if b.dtype == np.float64 else K.KUQCD_SINGLE
    K.kuqcd_gauge_free()
    assert K.kuqcd_init() == 0
    assert K.kuqcd_load_gaugefield(fat, gparam(dims, K.KUQCD_FAT_LINK, prec, order)) == 0
    assert K.kuqcd_load_gaugefield(lng, gparam(dims, K.KUQCD_LONG_LINK, prec, order)) == 0
    xs = [np.zeros_like(b) for _ in shifts]
    p = iparam(shifts, tol, max_iter, matpc, prec)
    st = K.kuqcd_solve_multishift(xs, b, p)
    K.kuqcd_gauge_free()
    K.kuqcd_end()
    return st, xs, p.iter


def reference_solve(dims, fat, lng, b, shifts, tol, max_iter, matpc=0):
    if O.ref_available():
        st, xs, it = O.ref_solve(dims, fat, lng, b, shifts, tol, max_iter, matpc=matpc)
        assert st == 0
        return xs, it
    return O.cgm(dims, fat, lng, matpc, shifts, b, tol, max_iter)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_kat_through_api(cuda, dtype):
    """test/test_solver.cpp:27-130 through kuqcd_solve_multishift."""
    dims = (4, 4, 4, 1)
    V = 64
    fat, lng, b = np.ones(V * 72, dtype), np.ones(V * 72, dtype), np.ones(V // 2 * 6, dtype)
    st, xs, it = api_solve(dims, fat, lng, b, [3.671676313381e-05], 1e-4, 6500, matpc=K.KUQCD_ODD_ODD)
    assert st == 0 and it == 1
    assert np.abs(xs[0] - 0.007561).mean() < 1e-4


@pytest.mark.gpu
@pytest.mark.parametrize("matpc", [0, 1])
def test_multishift_fp64_8x4_config(cuda, matpc):
    """8^4, eps 0.3, m 0.05, 12 shifts log-spaced 1e-4..1, per-shift 1e-10 (reference-semantics shifts)."""
    dims = (8, 8, 8, 8)
    fat, lng = O.make_links(dims, 0.3, 1234)
    b = O.make_source(dims, matpc, 99)
    m, sig = 0.05, np.logspace(-4, 0, 12)
    ab = m * m + sig
    refsh = [ab[0]] + list(sig[1:] - sig[0])
    tol = (1e-10) ** 2 * float(b @ b)
    st, xg, itg = api_solve(dims, fat, lng, b, refsh, tol, 10000, matpc=matpc)
    assert st == 0
    xr, itr = reference_solve(dims, fat, lng, b, refsh, tol, 10000, matpc=matpc)
    assert abs(itg - itr) <= 1
    for k in range(12):
        assert np.abs(xg[k] - xr[k]).max() <= 1e-9 * np.abs(xr[k]).max(), k
        assert O.true_residual(dims, fat, lng, matpc, ab[k], b, xg[k]) <= 1.5e-10, k


@pytest.mark.gpu
def test_multishift_fp32_matches_reference_float(cuda):
    dims = (6, 6, 6, 6)
    fat, lng = O.make_links(dims, 0.3, 55)
    b = O.make_source(dims, 0, 3).astype(np.float32)
    refsh = [0.01, 0.05, 0.4]
    tol = 1e-10 * float(b @ b)
    st, xg, itg = api_solve(dims, fat.astype(np.float32), lng.astype(np.float32), b, refsh, tol, 3000)
    assert st == 0
    xr, itr = reference_solve(dims, fat.astype(np.float32), lng.astype(np.float32), b, refsh, tol, 3000)
    assert abs(itg - itr) <= 3
    for k in range(3):
        assert np.abs(xg[k] - xr[k]).max() <= 2e-4 * np.abs(xr[k]).max()


@pytest.mark.gpu
def test_max_iter_stops_and_reports(cuda):
    dims = (4, 4, 4, 4)
    fat, lng = O.make_links(dims, 0.3, 2)
    b = O.make_source(dims, 0, 2)
    st, xg, it = api_solve(dims, fat, lng, b, [1e-4], 1e-30, 7)
    assert st == 0 and it == 7
    xr, itr = reference_solve(dims, fat, lng, b, [1e-4], 1e-30, 7)
    assert itr == 7
    assert np.abs(xg[0] - xr[0]).max() <= 1e-11 * np.abs(xr[0]).max()


@pytest.mark.gpu
def test_batch_order_double_matches_normal_order(cuda):
    """BATCH_ORDER double records (Nbatch 8, nx = 16) give the NORMAL_ORDER answer.  (The reference's double batch
    path has no x-direction lane shuffles -- dirac_hisq.cpp:504-663 specialise float/16 only -- so it decouples
    the lanes; kuqcd_b200 uses the float path's lane mapping for both precisions.)"""
    dims = (16, 4, 4, 4)
    fat, lng = O.make_links(dims, 0.3, 8)
    b = O.make_source(dims, 0, 8)
    refsh = [0.02, 0.1]
    tol = 1e-20 * float(b @ b)
    st, xn, itn = api_solve(dims, fat, lng, b, refsh, tol, 2000)
    assert st == 0
    st2, xb, itb = api_solve(dims, *to_batch(dims, fat, lng), to_batch_spinor(dims, b, 0), refsh, tol, 2000,
                             order=K.KUQCD_BATCH_ORDER)
    assert st2 == 0 and itb == itn
    for k in range(2):
        assert np.abs(from_batch_spinor(dims, xb[k], 0) - xn[k]).max() <= 1e-12 * np.abs(xn[k]).max()


@pytest.mark.gpu
def test_batch_order_float_matches_reference(cuda):
    """BATCH_ORDER float records (Nbatch 16, nx = 32) against the reference's own float batch solve."""
    if not O.ref_available():
        pytest.skip("needs the reference library")
    dims = (32, 4, 4, 2)
    fat, lng = O.make_links(dims, 0.3, 8)
    b = O.make_source(dims, 1, 8)
    f32 = lambda a: a.astype(np.float32)
    refsh = [0.02, 0.1]
    tol = 1e-10 * float(b @ b)
    fb, lb = to_batch(dims, fat, lng, 16)
    bb = f32(to_batch_spinor(dims, b, 1, 16))
    stb, xr, itr = O.ref_solve(dims, f32(fb), f32(lb), bb, refsh, tol, 2000, order=1, matpc=1)
    st, xg, itg = api_solve(dims, f32(fb), f32(lb), bb, refsh, tol, 2000, matpc=1, order=K.KUQCD_BATCH_ORDER)
    assert stb == 0 and st == 0 and abs(itg - itr) <= 2
    for k in range(2):
        assert np.abs(xg[k] - xr[k]).max() <= 1e-4 * np.abs(xr[k]).max()


def _batch_maps(dims, nb):
    nx, ny, nz, nt = dims
    nxr, hxr, hx = nx // nb, nx // nb // 2, nx // 2
    vhr = nxr * ny * nz * nt // 2
    vh = nx * ny * nz * nt // 2
    out = []
    for par in (0, 1):
        for i in range(vhr):
            r, xcb = divmod(i, hxr)
            r, y = divmod(r, ny)
            t, z = divmod(r, nz)
            xr = 2 * xcb + ((y + z + t + par) & 1)
            for j in range(nb):
                x = xr + nxr * j
                icb = (x >> 1) + hx * (y + ny * (z + nz * t))
                rpar = (x + y + z + t) & 1
                out.append((par, i, j, icb, rpar))
    return out, vhr, vh


def to_batch(dims, fat, lng, nb=8):
    m, vhr, vh = _batch_maps(dims, nb)
    fb, lb = np.zeros_like(fat), np.zeros_like(lng)
    for par, i, j, icb, rpar in m:
        ni = j + nb * (i + par * vhr)
        s = icb + rpar * vh
        fb[72 * ni:72 * ni + 72] = fat[72 * s:72 * s + 72]
        lb[72 * ni:72 * ni + 72] = lng[72 * s:72 * s + 72]
    return fb, lb


def to_batch_spinor(dims, b, parity, nb=8):
    m, vhr, vh = _batch_maps(dims, nb)
    out = np.zeros_like(b)
    for par, i, j, icb, rpar in m:
        if par == parity:
            ni = j + nb * i
            out[6 * ni:6 * ni + 6] = b[6 * icb:6 * icb + 6]
    return out


def from_batch_spinor(dims, xb, parity, nb=8):
    m, vhr, vh = _batch_maps(dims, nb)
    out = np.zeros_like(xb)
    for par, i, j, icb, rpar in m:
        if par == parity:
            ni = j + nb * i
            out[6 * icb:6 * icb + 6] = xb[6 * ni:6 * ni + 6]
    return out


@pytest.mark.gpu
def test_device_api_solver_absolute_shifts(cuda):
    dims = (8, 4, 4, 8)
    fat, lng = O.make_links(dims, 0.3, 31)
    b = O.make_source(dims, 1, 31)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    sig = [0.003, 0.01, 0.1]
    xs, info = ctx.solve(b, sig, parity=1, tol=(1e-11) ** 2 * float(b @ b), shift_mode=1)
    assert info.status == 0
    for k, s in enumerate(sig):
        assert O.true_residual(dims, fat, lng, 1, s, b, xs[k]) < 2e-11
