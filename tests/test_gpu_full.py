"""GPU tests of the full-lattice (non-preconditioned, KUQCD_HISQ_DIRAC) operator and solve, and of the even-odd
dslash against the golden fixtures the reference library produced (tests/golden/golden.npz).

Full-lattice fields hold the even sites then the odd sites.  The non-PC dslash of the reference
(dirac_hisq.cpp:128-136, 418-424 with diracType KUQCD_HISQ_DIRAC) is, bit for bit, the even-odd dslash of each
half onto the other (tests/test_golden.py pins the oracle to it); sigma - D D is therefore block diagonal and the
full solve is checked through its FP64 true residual over both parities."""
from pathlib import Path

import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from oracle import oracle as O
from tests.conftest import dev_buffer

G = np.load(Path(__file__).resolve().parent / "golden" / "golden.npz")
EPS, LINK_SEED = 0.3, 7


def make_ctx(dims, eps=EPS, seed=LINK_SEED):
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    return ctx, fat, lng


def full_source(dims, s0, s1):
    return np.concatenate([O.make_source(dims, 0, s0), O.make_source(dims, 1, s1)])


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["8x8x8x8", "6x4x2x8", "4x4x4x1", "2x3x5x4"])
@pytest.mark.parametrize("p", [0, 1])
def test_dslash_matches_golden(cuda, name, p):
    dims = tuple(int(v) for v in name.split("x"))
    ctx, fat, lng = make_ctx(dims)
    src = O.make_source(dims, 1 - p, 11)
    a, b = dev_buffer(ctx.spinor_bytes(K.KUQCD_DOUBLE)), dev_buffer(ctx.spinor_bytes(K.KUQCD_DOUBLE))
    ctx.upload(K.KUQCD_DOUBLE, src, a)
    ctx.dslash(K.KUQCD_DOUBLE, a, b, p)
    torch.cuda.synchronize()
    ref = G[f"dslash_{name}_p{p}"]
    assert np.abs(ctx.download(K.KUQCD_DOUBLE, b) - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["4x4x4x8", "6x2x4x2"])
def test_full_dslash_matches_golden(cuda, name):
    dims = tuple(int(v) for v in name.split("x"))
    ctx, fat, lng = make_ctx(dims)
    src = full_source(dims, 12, 13)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    a, b = dev_buffer(2 * vb), dev_buffer(2 * vb)
    ctx.upload_full(K.KUQCD_DOUBLE, src, a)
    ctx.dslash_full(K.KUQCD_DOUBLE, a, b)
    torch.cuda.synchronize()
    ref = G[f"full_{name}"]
    assert np.abs(ctx.download_full(K.KUQCD_DOUBLE, b) - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (6, 4, 2, 8), (16, 8, 4, 6)])
def test_full_dslash_and_mdagm_match_oracle_all_precisions(cuda, dims):
    ctx, fat, lng = make_ctx(dims, 0.4, 3)
    src = full_source(dims, 1, 2)
    ref = O.dslash_full(dims, fat, lng, src)
    n = np.linalg.norm(ref)
    for prec, tol in [(K.KUQCD_DOUBLE, 1e-14), (K.KUQCD_SINGLE, 1e-6), (K.KUQCD_HALF, 3e-4)]:
        vb = ctx.spinor_bytes(prec)
        a, b = dev_buffer(2 * vb), dev_buffer(2 * vb)
        ctx.upload_full(prec, src, a)
        ctx.dslash_full(prec, a, b)
        torch.cuda.synchronize()
        assert np.linalg.norm(ctx.download_full(prec, b) - ref) <= tol * n, prec
    # sigma - D D on the full lattice = the even-odd operator on each half
    sigma = 0.37
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    a, b, t = dev_buffer(2 * vb), dev_buffer(2 * vb), dev_buffer(2 * vb)
    ctx.upload_full(K.KUQCD_DOUBLE, src, a)
    ctx.mdagm_full(K.KUQCD_DOUBLE, sigma, a, b, t)
    torch.cuda.synchronize()
    h = src.size // 2
    want = np.concatenate([sigma * src[:h] - O.mdagm(dims, fat, lng, src[:h], 0),
                           sigma * src[h:] - O.mdagm(dims, fat, lng, src[h:], 1)])
    got = ctx.download_full(K.KUQCD_DOUBLE, b)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [K.KQ_SOLVER_CGM, K.KQ_SOLVER_CGM_WINDOWED, K.KQ_SOLVER_MIXED])
def test_full_lattice_multishift_solve(cuda, solver):
    dims = (8, 8, 8, 8)
    ctx, fat, lng = make_ctx(dims, 0.3, 5)
    b = full_source(dims, 3, 4)
    sig = list(0.05 ** 2 + np.logspace(-4, 0, 5))
    bb = float(b @ b)
    kw = dict(parity=K.KQ_PARITY_FULL, solver=solver, max_iter=20000, shift_mode=1)
    if solver == K.KQ_SOLVER_MIXED:
        kw.update(prec=K.KUQCD_HALF, rel_residual=1e-10)
    else:
        kw.update(tol=(1e-11) ** 2 * bb)
    xs, info = ctx.solve(b, sig, **kw)
    assert info.status == 0 and info.iter > 0
    h = b.size // 2
    for k, s in enumerate(sig):
        # FP64 true residual over both parities, by the oracle
        re = O.true_residual(dims, fat, lng, 0, s, b[:h], xs[k][:h]) ** 2 * float(b[:h] @ b[:h])
        ro = O.true_residual(dims, fat, lng, 1, s, b[h:], xs[k][h:]) ** 2 * float(b[h:] @ b[h:])
        assert np.sqrt((re + ro) / bb) <= 1.05e-10, (k, s)
    # the device residual check agrees
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    db, dx = dev_buffer(2 * vb), dev_buffer(2 * vb * len(sig))
    ctx.upload_full(K.KUQCD_DOUBLE, b, db)
    for k in range(len(sig)):
        ctx.upload_full(K.KUQCD_DOUBLE, xs[k], dx[2 * k * vb:2 * (k + 1) * vb])
    res = ctx.true_residuals(K.KQ_PARITY_FULL, sig, db, dx)
    assert max(res) <= 1.05e-10


@pytest.mark.gpu
def test_full_lattice_solve_zero_half(cuda):
    """A source on one parity only: the other half of every solution is exactly zero."""
    dims = (4, 4, 4, 4)
    ctx, fat, lng = make_ctx(dims)
    b = full_source(dims, 8, 9)
    b[b.size // 2:] = 0
    xs, info = ctx.solve(b, [0.1, 0.5], parity=K.KQ_PARITY_FULL, solver=K.KQ_SOLVER_CGM_WINDOWED,
                         tol=(1e-12) ** 2 * float(b @ b))
    for s, x in zip([0.1, 0.5], xs):
        assert not np.any(x[x.size // 2:])
        assert O.true_residual(dims, fat, lng, 0, s, b[:b.size // 2], x[:x.size // 2]) < 1e-11
