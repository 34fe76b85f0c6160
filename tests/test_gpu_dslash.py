"""GPU parity of the dslash kernels against the oracle (oracle/hisq_oracle.c, itself bit-exact with the reference
DiracHISQ::Dslash, dirac_hisq.cpp:409-502).  Tolerances: FP64 <= 1e-13 relative (max norm); FP32 and HALF are
sloppy operators, checked in relative 2-norm at 1e-6 and 3e-4."""
import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from oracle import oracle as O
from tests.conftest import dev_buffer

DIMS = [(4, 4, 4, 4), (6, 6, 6, 6), (4, 6, 8, 10), (8, 8, 8, 8), (4, 4, 4, 1), (2, 3, 5, 4), (6, 4, 2, 8),
        (4, 1, 1, 2), (16, 8, 4, 6)]


def make_ctx(dims, eps=0.3, seed=7):
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    return ctx, fat, lng


def run_dslash(ctx, prec, src, parity):
    a = dev_buffer(ctx.spinor_bytes(prec))
    b = dev_buffer(ctx.spinor_bytes(prec))
    ctx.upload(prec, src, a)
    ctx.dslash(prec, a, b, parity)
    torch.cuda.synchronize()
    return ctx.download(prec, b)


@pytest.mark.gpu
@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("parity", [0, 1])
def test_dslash_fp64_matches_oracle(cuda, dims, parity):
    ctx, fat, lng = make_ctx(dims)
    src = np.random.default_rng(3).standard_normal(int(np.prod(dims)) // 2 * 6)
    ref = O.dslash(dims, fat, lng, src, parity)
    out = run_dslash(ctx, K.KUQCD_DOUBLE, src, parity)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (8, 8, 8, 8), (4, 6, 8, 10), (4, 4, 4, 1)])
def test_dslash_sloppy_precisions(cuda, dims):
    ctx, fat, lng = make_ctx(dims)
    src = np.random.default_rng(4).standard_normal(int(np.prod(dims)) // 2 * 6)
    ref = O.dslash(dims, fat, lng, src, 0)
    n = np.linalg.norm(ref)
    f32 = run_dslash(ctx, K.KUQCD_SINGLE, src, 0)
    assert np.linalg.norm(f32 - ref) <= 1e-6 * n
    f16 = run_dslash(ctx, K.KUQCD_HALF, src, 0)
    assert np.linalg.norm(f16 - ref) <= 3e-4 * n


@pytest.mark.gpu
def test_dslash_matches_reference_library_directly(cuda):
    if not O.ref_available():
        pytest.skip("reference library not shipped")
    dims = (6, 4, 4, 6)
    ctx, fat, lng = make_ctx(dims, 0.4, 17)
    src = np.random.default_rng(5).standard_normal(int(np.prod(dims)) // 2 * 6)
    for parity in (0, 1):
        ref = O.ref_dslash(dims, fat, lng, src, parity)
        out = run_dslash(ctx, K.KUQCD_DOUBLE, src, parity)
        assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
def test_mdagm_fp64(cuda):
    dims = (8, 4, 4, 8)
    ctx, fat, lng = make_ctx(dims)
    src = np.random.default_rng(6).standard_normal(int(np.prod(dims)) // 2 * 6)
    sigma = 0.37
    ref = sigma * src - O.mdagm(dims, fat, lng, src, 1)
    nb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    a, t, b = dev_buffer(nb), dev_buffer(nb), dev_buffer(nb)
    ctx.upload(K.KUQCD_DOUBLE, src, a)
    ctx.mdagm(K.KUQCD_DOUBLE, sigma, a, b, t, 1)
    out = ctx.download(K.KUQCD_DOUBLE, b)
    assert np.abs(out - ref).max() <= 1e-13 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (6, 4, 2, 8)])
def test_device_generator_matches_oracle_generator(cuda, dims):
    V = int(np.prod(dims))
    ctx = K.Context(dims)
    f = torch.zeros(V * 72, dtype=torch.float64, device="cuda")
    l = torch.zeros(V * 72, dtype=torch.float64, device="cuda")
    ctx.make_links(0.35, 1234, f, l)
    b = torch.zeros(V // 2 * 6, dtype=torch.float64, device="cuda")
    ctx.make_source(1, 77, b)
    fat, lng = O.make_links(dims, 0.35, 1234)
    assert np.abs(f.cpu().numpy() - fat).max() < 1e-13
    assert np.abs(l.cpu().numpy() - lng).max() < 1e-13
    assert np.abs(b.cpu().numpy() - O.make_source(dims, 1, 77)).max() < 1e-13


@pytest.mark.gpu
def test_precision_round_trip(cuda):
    dims = (4, 4, 4, 4)
    ctx = K.Context(dims)
    src = np.random.default_rng(8).standard_normal(128 * 6)
    for prec, tol in [(K.KUQCD_DOUBLE, 0.0), (K.KUQCD_SINGLE, 1e-7), (K.KUQCD_HALF, 4e-5)]:
        a = dev_buffer(ctx.spinor_bytes(prec))
        ctx.upload(prec, src, a)
        back = ctx.download(prec, a)
        # HALF: 16-bit fixed point relative to the per-site maximum
        site_max = np.abs(src.reshape(-1, 6)).max(axis=1, keepdims=True)
        assert np.all(np.abs(back - src).reshape(-1, 6) <= tol * site_max + 1e-300)


@pytest.mark.gpu
def test_long_links_stored_compressed_when_su3_multiples(cuda, monkeypatch):
    """Long links that are real multiples of SU(3) matrices (the generator's -1/24 U U U, like HISQ's Naik links)
    are stored as two rows + 1/s in FP64 and FP32; the operator is unchanged to rounding.  Links that are not (here
    Gaussian noise) keep full storage.  KUQCD_LONG_RECON=0 turns the compression off."""
    dims = (8, 6, 4, 4)
    src = np.random.default_rng(8).standard_normal(int(np.prod(dims)) // 2 * 6)
    ctx, fat, lng = make_ctx(dims)
    ctx.prepare(K.KUQCD_SINGLE)
    ctx.prepare(K.KUQCD_HALF)
    assert ctx.long_links_compressed(K.KUQCD_DOUBLE) == 1
    assert ctx.long_links_compressed(K.KUQCD_SINGLE) == 1
    assert ctx.long_links_compressed(K.KUQCD_HALF) == 0
    ref = O.dslash(dims, fat, lng, src, 1)
    packed = run_dslash(ctx, K.KUQCD_DOUBLE, src, 1)
    assert np.abs(packed - ref).max() <= 1e-13 * np.abs(ref).max()
    monkeypatch.setenv("KUQCD_LONG_RECON", "0")
    ctx2, _, _ = make_ctx(dims)
    assert ctx2.long_links_compressed(K.KUQCD_DOUBLE) == 0
    full = run_dslash(ctx2, K.KUQCD_DOUBLE, src, 1)
    assert np.abs(full - packed).max() <= 1e-14 * np.abs(full).max()
    monkeypatch.delenv("KUQCD_LONG_RECON")
    # not SU(3) multiples: full storage, same operator as the oracle
    noise = np.random.default_rng(3).standard_normal(lng.size)
    ctx3 = K.Context(dims)
    ctx3.load_links(K.KUQCD_FAT_LINK, fat)
    ctx3.load_links(K.KUQCD_LONG_LINK, noise)
    assert ctx3.long_links_compressed(K.KUQCD_DOUBLE) == 0
    ref3 = O.dslash(dims, fat, noise, src, 1)
    out3 = run_dslash(ctx3, K.KUQCD_DOUBLE, src, 1)
    assert np.abs(out3 - ref3).max() <= 1e-13 * np.abs(ref3).max()
