"""Failure detection without any GPU fault: bad inputs and failed allocations come back as error statuses, and the
context stays usable afterwards; a zero source is solved exactly.  (Non-finite p.Ap is the solvers' breakdown test;
max_iter exhaustion is covered in test_gpu_cgm.py.)"""
import numpy as np
import pytest

import kuqcd_b200 as K
from oracle import oracle as O

DIMS = (8, 4, 4, 4)


def ctx_for(dims=DIMS):
    fat, lng = O.make_links(dims, 0.3, 5)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    return ctx, fat, lng


SOLVERS = [dict(solver=K.KQ_SOLVER_CGM), dict(solver=K.KQ_SOLVER_CGM_WINDOWED),
           dict(solver=K.KQ_SOLVER_MIXED, prec=K.KUQCD_HALF)]


def still_solves(ctx, fat, lng):
    b = O.make_source(DIMS, 0, 3)
    xs, info = ctx.solve(b, [0.1], parity=0, solver=K.KQ_SOLVER_CGM_WINDOWED, tol=(1e-10) ** 2 * float(b @ b))
    assert info.status == 0
    assert O.true_residual(DIMS, fat, lng, 0, 0.1, b, xs[0]) < 2e-10


@pytest.mark.gpu
@pytest.mark.parametrize("kw", SOLVERS)
def test_non_finite_source_is_an_error(cuda, kw):
    ctx, fat, lng = ctx_for()
    b = O.make_source(DIMS, 0, 4)
    b[17] = np.nan
    with pytest.raises(K.KuQCDError):
        ctx.solve(b, [0.1, 0.5], parity=0, tol=1e-20, rel_residual=1e-10, **kw)
    still_solves(ctx, fat, lng)


@pytest.mark.gpu
@pytest.mark.parametrize("kw", SOLVERS)
def test_zero_source_gives_zero_solutions(cuda, kw):
    """b = 0: every x_k = 0 exactly, no iteration (the reference would divide 0 by p.Ap = 0,
    inverter_cgm.cpp:47, and return NaN)."""
    ctx, fat, lng = ctx_for()
    b = np.zeros(O.make_source(DIMS, 0, 4).shape)
    xs, info = ctx.solve(b, [0.1, 0.7], parity=0, tol=1e-20, rel_residual=1e-10, **kw)
    assert info.status == 0 and info.iter == 0
    assert all(not np.any(x) for x in xs)
    still_solves(ctx, fat, lng)


@pytest.mark.gpu
def test_failed_allocation_reports_no_memory(cuda):
    """A network for a lattice of 2^31 sites needs ~400 GB of activations: cudaMalloc fails, the call returns
    KUQCD_ERR_NO_MEMORY, and nothing else is affected."""
    big = K.Context((256, 256, 256, 128))
    with pytest.raises(K.KuQCDError) as ei:
        K.Net(big, (1, 8, 8))
    assert ei.value.status == K.KUQCD_ERR_NO_MEMORY
    big.close()
    ctx, fat, lng = ctx_for()
    still_solves(ctx, fat, lng)


@pytest.mark.gpu
def test_net_fault_is_reported_once(cuda):
    """A tensor-core tile whose bounded wait ran out sets a device word; the next network call reports it and clears
    it, so the call after that succeeds.  The word is set from the host here: no wait is made to time out."""
    import torch

    ctx, fat, lng = ctx_for()
    net = K.Net(ctx, (1, 8, 8))
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    d_in = torch.zeros(vb, dtype=torch.uint8, device="cuda:0")
    ctx.upload(K.KUQCD_DOUBLE, O.make_source(DIMS, 0, 9), d_in)
    d_out = torch.zeros_like(d_in)
    net.apply(d_in, d_out, 0)
    assert K.library().kq_net_raise_fault_for_test(net._h) == 0
    with pytest.raises(K.KuQCDError):
        net.apply(d_in, d_out, 0)
    assert b"wait limit" in K.library().kq_last_error()
    net.apply(d_in, d_out, 0)
    net.close()
    still_solves(ctx, fat, lng)
