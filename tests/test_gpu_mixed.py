"""GPU tests of the mixed-precision multishift solver (sloppy multishift + batched reliable-update refinement):
every shift's FP64 true relative residual, recomputed by the oracle on the CPU, meets the target."""
import ctypes as C

import numpy as np
import pytest

import kuqcd_b200 as K
from oracle import oracle as O
from tests.test_gpu_cgm import api_solve


def ctx_for(dims, eps, seed):
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    return ctx, fat, lng


@pytest.mark.gpu
@pytest.mark.parametrize("sloppy", [K.KUQCD_SINGLE, K.KUQCD_HALF])
@pytest.mark.parametrize("parity", [0, 1])
def test_mixed_8x4_config_reaches_1e10(cuda, sloppy, parity):
    dims = (8, 8, 8, 8)
    ctx, fat, lng = ctx_for(dims, 0.3, 1234)
    b = O.make_source(dims, parity, 99)
    sig = list(0.05 ** 2 + np.logspace(-4, 0, 12))
    xs, info = ctx.solve(b, sig, parity=parity, solver=K.KQ_SOLVER_MIXED, prec=sloppy, rel_residual=1e-10)
    assert info.status == 0
    # the relaxed multishift usually meets the target itself; refinement only mops up shifts it left above it
    assert info.iter > 0 and info.iter_refine >= 0
    for k, s in enumerate(sig):
        r = O.true_residual(dims, fat, lng, parity, s, b, xs[k])
        assert r <= 1.2e-10, (k, r)
        # the device's own FP64 residual agrees with the oracle's
        assert abs(info.true_residual[k] - r) <= 0.05 * r + 1e-13
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 4, 4, 6), (4, 4, 4, 1)])
def test_windowed_cgm_matches_classic(cuda, dims):
    """KQ_SOLVER_CGM_WINDOWED runs the CGM recurrences with shift updates deferred over windows of 16 iterations:
    same iteration count as the classic kernel order and the same solutions up to rounding."""
    ctx, fat, lng = ctx_for(dims, 0.3, 1234)
    b = O.make_source(dims, 0, 99)
    sig = list(0.05 ** 2 + np.logspace(-4, 0, 12))
    tol = (1e-10) ** 2 * float(b @ b)
    xc, ic = ctx.solve(b, sig, solver=K.KQ_SOLVER_CGM, prec=K.KUQCD_DOUBLE, tol=tol)
    xw, iw = ctx.solve(b, sig, solver=K.KQ_SOLVER_CGM_WINDOWED, prec=K.KUQCD_DOUBLE, tol=tol)
    assert abs(ic.iter - iw.iter) <= 1 and iw.status == 0
    for k in range(12):
        assert np.abs(xw[k] - xc[k]).max() <= 1e-9 * np.abs(xc[k]).max(), k
        assert O.true_residual(dims, fat, lng, 0, sig[k], b, xw[k]) <= 1.5e-10, k
    ctx.close()


@pytest.mark.gpu
def test_windowed_cgm_reference_shift_semantics_and_max_iter(cuda):
    dims = (4, 4, 4, 4)
    ctx, fat, lng = ctx_for(dims, 0.3, 2)
    b = O.make_source(dims, 0, 2)
    # reference semantics (shift_mode 0), stopped by max_iter in the middle of a window
    xs, info = ctx.solve(b, [1e-4, 0.5], solver=K.KQ_SOLVER_CGM_WINDOWED, tol=1e-30, max_iter=11, shift_mode=0)
    assert info.iter == 11
    xr, itr = O.cgm(dims, fat, lng, 0, [1e-4, 0.5], b, 1e-30, 11)
    assert itr == 11
    for k in range(2):
        assert np.abs(xs[k] - xr[k]).max() <= 1e-11 * np.abs(xr[k]).max()
    ctx.close()


@pytest.mark.gpu
def test_mixed_single_shift_and_tight_target(cuda):
    dims = (8, 4, 4, 8)
    ctx, fat, lng = ctx_for(dims, 0.4, 5)
    b = O.make_source(dims, 0, 5)
    xs, info = ctx.solve(b, [0.002], solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_SINGLE, rel_residual=1e-12)
    assert info.status == 0
    assert O.true_residual(dims, fat, lng, 0, 0.002, b, xs[0]) <= 1.2e-12
    ctx.close()


@pytest.mark.gpu
def test_mixed_matches_plain_solution(cuda):
    dims = (8, 8, 4, 4)
    ctx, fat, lng = ctx_for(dims, 0.3, 77)
    b = O.make_source(dims, 0, 7)
    sig = [0.01, 0.1, 1.0]
    xm, im = ctx.solve(b, sig, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF, rel_residual=1e-11)
    xp, ip = ctx.solve(b, sig, solver=K.KQ_SOLVER_CGM, prec=K.KUQCD_DOUBLE, tol=(1e-12) ** 2 * float(b @ b))
    for k in range(3):
        # both solve (sigma + D^dag D) x = b; the difference is bounded by the residuals over sigma
        bound = 2e-11 * np.linalg.norm(b) / sig[k]
        assert np.linalg.norm(xm[k] - xp[k]) <= bound
    ctx.close()


@pytest.mark.gpu
def test_mixed_through_reference_api(cuda, monkeypatch):
    """KUQCD_SOLVER=mixed switches kuqcd_solve_multishift (DOUBLE links) to the mixed solver; the reference's
    stopping rule zeta_k^2 |r|^2 < tol becomes the true residual bound |r_k| < sqrt(tol)."""
    monkeypatch.setenv("KUQCD_SOLVER", "mixed")
    dims = (8, 8, 8, 8)
    fat, lng = O.make_links(dims, 0.3, 4321)
    b = O.make_source(dims, 0, 11)
    m, sig = 0.05, np.logspace(-4, 0, 12)
    ab = m * m + sig
    refsh = [ab[0]] + list(sig[1:] - sig[0])
    tol = (1e-10) ** 2 * float(b @ b)
    st, xs, it = api_solve(dims, fat, lng, b, refsh, tol, 10000)
    assert st == 0 and it > 0
    for k in range(12):
        assert O.true_residual(dims, fat, lng, 0, ab[k], b, xs[k]) <= 1.2e-10


@pytest.mark.gpu
def test_mixed_absolute_target(cuda):
    """rel_residual < 0: the reference's absolute threshold |b - A_k x_k|^2 < tol, with |b| taken on the device
    (the path kuqcd_solve_multishift uses with KUQCD_SOLVER=mixed); it needs tol > 0, and batched systems refuse
    it."""
    import torch

    dims = (8, 8, 8, 4)
    ctx, fat, lng = ctx_for(dims, 0.3, 77)
    b = 3.0 * O.make_source(dims, 0, 5)
    sig = list(0.05 ** 2 + np.logspace(-3, 0, 4))
    tol = (2e-10) ** 2 * float(b @ b)
    xs, info = ctx.solve(b, sig, parity=0, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF, rel_residual=-1.0, tol=tol)
    assert info.status == 0
    for k, s in enumerate(sig):
        r = O.true_residual(dims, fat, lng, 0, s, b, xs[k])
        assert r <= 2.2e-10, (k, r)
    with pytest.raises(K.KuQCDError):
        ctx.solve(b, sig, parity=0, solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF, rel_residual=-1.0, tol=0.0)
    bt = K.Batch()
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    d_b = torch.zeros(vb, dtype=torch.uint8, device="cuda")
    d_x = torch.zeros(4 * vb, dtype=torch.uint8, device="cuda")
    with pytest.raises(K.KuQCDError):
        bt.add(ctx, d_b, d_x, sig, solver=K.KQ_SOLVER_MIXED, rel_residual=-1.0, tol=tol)
    bt.close()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kw", [dict(solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF),
                                dict(solver=K.KQ_SOLVER_CGM_WINDOWED), dict(solver=K.KQ_SOLVER_CGM)])
@pytest.mark.parametrize("stop", ["0.7", "3"])
def test_pinned_host_buffers_copy_during_the_solve(cuda, monkeypatch, kw, stop):
    """With page-locked host buffers each solution is copied out as soon as the solver is done with it, while the
    other shifts still iterate, and copied again if the refinement changes it afterwards (KUQCD_RELAX_STOP=3 stops
    the multishift above the target, so the mixed solver refines).  The solutions are the pageable path's, bit for
    bit; the reference-order CGM reports nothing early and copies at the end."""
    monkeypatch.setenv("KUQCD_RELAX_STOP", stop)
    dims = (8, 8, 8, 8)
    ctx, fat, lng = ctx_for(dims, 0.3, 2024)
    b = O.make_source(dims, 1, 31)
    sig = list(0.05 ** 2 + np.logspace(-4, 0, 10))
    tol = (1e-10) ** 2 * float(b @ b)
    xa, ia = ctx.solve(b, sig, parity=1, tol=tol, rel_residual=1e-10, **kw)
    xb, ib = ctx.solve(b, sig, parity=1, tol=tol, rel_residual=1e-10, pinned=True, **kw)
    assert ia.status == 0 and ib.status == 0
    assert (ia.iter, ia.iter_refine) == (ib.iter, ib.iter_refine)
    assert ia.copies_during_solve == 0
    if kw["solver"] == K.KQ_SOLVER_CGM:
        assert ib.copies_during_solve == 0
    else:
        assert ib.copies_during_solve >= len(sig) // 2, ib.copies_during_solve
    if kw["solver"] == K.KQ_SOLVER_MIXED and stop == "3":
        assert ib.iter_refine > 0
    for k, s in enumerate(sig):
        assert np.array_equal(xa[k], xb[k]), k
        assert O.true_residual(dims, fat, lng, 1, s, b, xb[k]) <= 1.5e-10, k
    ctx.close()
