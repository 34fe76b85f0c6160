"""kq_mdagm_noalloc: the operator sigma - D_pq D_qp for callers that cannot let the library allocate device memory
while they run it (an application whose own pool holds nearly all of HBM, a latency-critical loop where cudaMalloc
may synchronise the device).  Its temporary lives in a fixed device array of the library, so the results must equal
kq_mdagm's with a caller-provided temporary, call after call.

This file sorts last so that a run stopping at the first failure has already run every other test."""
import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from oracle import oracle as O


def _field(ctx, prec):
    return torch.zeros(ctx.spinor_bytes(prec), dtype=torch.uint8, device="cuda:0")


@pytest.mark.gpu
@pytest.mark.parametrize("prec,tol", [(K.KUQCD_DOUBLE, 1e-13), (K.KUQCD_SINGLE, 1e-6), (K.KUQCD_HALF, 1e-6)])
def test_noalloc_matches_kq_mdagm_twice(cuda, prec, tol):
    dims = (8, 8, 8, 8)
    fat, lng = O.make_links(dims, 0.3, 42)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    ctx.prepare(prec)
    src = O.make_source(dims, 1, 3)
    a, ref_out, tmp = _field(ctx, prec), _field(ctx, prec), _field(ctx, prec)
    ctx.upload(prec, src, a)
    sigma = 0.123
    ctx.mdagm(prec, sigma, a, ref_out, tmp, 1)
    ref = ctx.download(prec, ref_out)
    for call in range(2):
        out = _field(ctx, prec)
        assert ctx.mdagm_noalloc(prec, sigma, a, out, 1) == K.KUQCD_SUCCESS, K.library().kq_last_error()
        torch.cuda.synchronize()
        got = ctx.download(prec, out)
        assert np.abs(got - ref).max() <= tol * np.abs(ref).max(), call
    # and against the oracle in FP64
    if prec == K.KUQCD_DOUBLE:
        want = sigma * src - O.mdagm(dims, fat, lng, src, 1)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    ctx.close()


@pytest.mark.gpu
def test_noalloc_rejects_oversized_and_unprepared(cuda):
    big = K.Context((32, 32, 32, 64))  # FP64 field of 48 MiB > 32 MiB
    d = torch.zeros(16, dtype=torch.uint8, device="cuda:0")
    assert big.mdagm_noalloc(K.KUQCD_DOUBLE, 0.1, d, d, 0) == K.KUQCD_ERR_INVALID_PARAM
    assert b"32 MiB" in K.library().kq_last_error()
    big.close()
    small = K.Context((4, 4, 4, 4))  # no links loaded: nothing resident, nothing allocated
    assert small.mdagm_noalloc(K.KUQCD_DOUBLE, 0.1, d, d, 0) == K.KUQCD_ERR_UNEXPECTED_CALL_ORDER
    small.close()
