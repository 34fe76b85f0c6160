"""GPU tests of the t-slab domain decomposition (kq_slab.cu, kuqcd_b200/slab.py), with R ranks emulated in this
process on one GPU (LocalTransport: a rank's ghost is its neighbour's face buffer; ranks run one after another, no
kernel waits on another).  The decomposed dslash must equal the undecomposed one, and the decomposed multishift CG
(reference recurrences, reductions summed over ranks) must solve the global system."""
import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from kuqcd_b200 import slab as SL
from oracle import oracle as O

GDIMS = (8, 4, 4, 16)


def setup_slabs(R, eps=0.3, seed=7):
    fat, lng = O.make_links(GDIMS, eps, seed)
    tr = SL.LocalTransport()
    slabs = [SL.Slab(GDIMS, r, R) for r in range(R)]
    for s in slabs:
        s.load_links(SL.slab_of_links(fat, GDIMS, s.rank, R), SL.slab_of_links(lng, GDIMS, s.rank, R))
    SL.exchange_link_ghosts(slabs, tr)
    return slabs, tr, fat, lng


def upload(slabs, rec, prec=K.KUQCD_DOUBLE):
    out = []
    for s in slabs:
        f = s.field(prec)
        s.ctx.upload(prec, SL.slab_of_spinor(rec, GDIMS, s.rank, s.nranks), f)
        out.append(f)
    return out


def download(slabs, fields, prec=K.KUQCD_DOUBLE):
    torch.cuda.synchronize()
    return SL.join_spinor([s.ctx.download(prec, f) for s, f in zip(slabs, fields)])


@pytest.mark.gpu
@pytest.mark.parametrize("R", [1, 2, 4])
@pytest.mark.parametrize("parity", [0, 1])
def test_slab_dslash_equals_global(cuda, R, parity):
    slabs, tr, fat, lng = setup_slabs(R)
    src = O.make_source(GDIMS, 1 - parity, 5)
    want = O.dslash(GDIMS, fat, lng, src, parity)
    xs = upload(slabs, src)
    ys = [s.field() for s in slabs]
    SL.dslash(slabs, tr, K.KUQCD_DOUBLE, xs, ys, parity)
    got = download(slabs, ys)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()
    # the undecomposed GPU kernel, same term order: equal to rounding of the FMA contraction at most
    ctx = K.Context(GDIMS)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    a = torch.zeros(ctx.spinor_bytes(K.KUQCD_DOUBLE), dtype=torch.uint8, device="cuda")
    b = torch.zeros_like(a)
    ctx.upload(K.KUQCD_DOUBLE, src, a)
    ctx.dslash(K.KUQCD_DOUBLE, a, b, parity)
    torch.cuda.synchronize()
    glob = ctx.download(K.KUQCD_DOUBLE, b)
    assert np.abs(got - glob).max() <= 1e-15 * np.abs(glob).max()
    # FP32 slabs against the FP64 operator
    xf = upload(slabs, src, K.KUQCD_SINGLE)
    yf = [s.field(K.KUQCD_SINGLE) for s in slabs]
    SL.dslash(slabs, tr, K.KUQCD_SINGLE, xf, yf, parity)
    gotf = download(slabs, yf, K.KUQCD_SINGLE)
    assert np.linalg.norm(gotf - want) <= 1e-6 * np.linalg.norm(want)


@pytest.mark.gpu
def test_slab_sigma_minus_dslash_and_operator(cuda):
    """sigma p - D (D p) through two exchanges equals the global operator sigma - D_pq D_qp."""
    R = 2
    slabs, tr, fat, lng = setup_slabs(R, 0.4, 9)
    p = O.make_source(GDIMS, 0, 6)
    ps = upload(slabs, p)
    tmp = [s.field() for s in slabs]
    out = [s.field() for s in slabs]
    SL.dslash(slabs, tr, K.KUQCD_DOUBLE, ps, tmp, 1)
    SL.dslash(slabs, tr, K.KUQCD_DOUBLE, tmp, out, 0, pvecs=ps, sigma=0.3)
    want = 0.3 * p - O.mdagm(GDIMS, fat, lng, p, 0)
    assert np.abs(download(slabs, out) - want).max() <= 1e-13 * np.abs(want).max()


@pytest.mark.gpu
@pytest.mark.parametrize("R,poll_every", [(2, 1), (2, 5), (4, 4)])
def test_slab_multishift_cg_solves_global_system(cuda, R, poll_every):
    """The device-driven slab CGM (scalar recurrences on a device state, in-place reductions, host poll every few
    iterations) solves the global system with the reference's recurrences; steps after the stop are no-ops, so the
    iteration count does not depend on the poll interval."""
    slabs, tr, fat, lng = setup_slabs(R, 0.3, 11)
    b = O.make_source(GDIMS, 0, 8)
    m, sig = 0.05, np.logspace(-3, 0, 5)
    ab = m * m + sig
    refsh = [ab[0]] + list(sig[1:] - sig[0])
    tol = (1e-10) ** 2 * float(b @ b)
    bs = upload(slabs, b)
    xs, it = SL.cgm(slabs, tr, bs, refsh, tol, 5000, poll_every=poll_every)
    xo, ito = O.cgm(GDIMS, fat, lng, 0, refsh, b, tol, 5000)
    assert abs(it - ito) <= 1, (it, ito)  # same recurrences; reductions summed in another order
    # stream-ordered and deterministic: the same solve again gives the same count and the same bits
    xs2, it2 = SL.cgm(slabs, tr, bs, refsh, tol, 5000, poll_every=poll_every)
    assert it2 == it
    for k in range(len(ab)):
        assert torch.equal(torch.cat([xr[k] for xr in xs]), torch.cat([xr[k] for xr in xs2])), k
    for k in range(len(ab)):
        x = download(slabs, [xk[k] for xk in xs])
        assert np.abs(x - xo[k]).max() <= 1e-9 * np.abs(xo[k]).max()
        assert O.true_residual(GDIMS, fat, lng, 0, ab[k], b, x) <= 2e-10


@pytest.mark.gpu
def test_slab_rejects_bad_geometry(cuda):
    with pytest.raises(K.KuQCDError):
        SL.Slab((4, 4, 4, 12), 0, 4)  # local t extent 3: a depth-3 halo would span two ranks
    s = SL.Slab((4, 4, 4, 8), 0, 2)
    a = s.field()
    with pytest.raises(K.KuQCDError):  # ghost links not exchanged yet
        s.dslash(K.KUQCD_DOUBLE, a, a, a, s.field(), 0)


@pytest.mark.gpu
@pytest.mark.parametrize("R", [1, 2, 4])
def test_slab_dslash_parts_and_half(cuda, R):
    """The interior launch (run while the faces are in flight) plus the boundary launch equal the whole-slab launch
    bit for bit, in every precision; HALF slabs (ghost links quantised with the receiving slab's link scales) match
    the FP64 operator to HALF accuracy."""
    slabs, tr, fat, lng = setup_slabs(R, 0.35, 13)
    src = O.make_source(GDIMS, 1, 14)
    want = O.dslash(GDIMS, fat, lng, src, 0)
    for prec, tol in [(K.KUQCD_DOUBLE, 1e-13), (K.KUQCD_SINGLE, 1e-6), (K.KUQCD_HALF, 5e-4)]:
        xs = upload(slabs, src, prec)
        ys = [s.field(prec) for s in slabs]
        zs = [s.field(prec) for s in slabs]
        SL.dslash(slabs, tr, prec, xs, ys, 0, overlap=True)
        SL.dslash(slabs, tr, prec, xs, zs, 0, overlap=False)
        got, whole = download(slabs, ys, prec), download(slabs, zs, prec)
        assert np.array_equal(got, whole), prec
        assert np.linalg.norm(got - want) <= tol * np.linalg.norm(want), prec


@pytest.mark.gpu
def test_slab_cgm_zero_source_and_iteration_cap(cuda):
    """b = 0 stops before the first iteration with x = 0; max_iter caps the device-side count exactly."""
    slabs, tr, fat, lng = setup_slabs(2, 0.3, 12)
    zero = upload(slabs, np.zeros(GDIMS[0] * GDIMS[1] * GDIMS[2] * GDIMS[3] // 2 * 6))
    xs, it = SL.cgm(slabs, tr, zero, [0.01, 0.1], 1e-20, 50)
    assert it == 0
    assert not np.any(download(slabs, [xk[0] for xk in xs]))
    b = O.make_source(GDIMS, 0, 9)
    xs, it = SL.cgm(slabs, tr, upload(slabs, b), [0.0025, 0.1], 1e-40, 7, poll_every=3)
    assert it == 7


@pytest.mark.gpu
@pytest.mark.parametrize("R,sloppy", [(2, K.KUQCD_SINGLE), (2, K.KUQCD_HALF), (4, K.KUQCD_HALF)])
def test_slab_mixed_cg_reaches_fp64_target(cuda, R, sloppy):
    """The relaxed-precision multishift over slabs (FP64 -> FP32 -> HALF operator as |r| falls) plus the FP64 check /
    refinement: every shift's true residual, recomputed by the oracle on the gathered solution, is at the target, and
    the sloppy operators did run."""
    slabs, tr, fat, lng = setup_slabs(R, 0.3, 15)
    b = O.make_source(GDIMS, 0, 16)
    m, sig = 0.05, np.logspace(-3, 0, 5)
    ab = m * m + sig
    refsh = [ab[0]] + list(sig[1:] - sig[0])
    xs, info = SL.cgm_mixed(slabs, tr, upload(slabs, b), refsh, 1e-10, 5000, sloppy=sloppy)
    assert len(info["true_residuals"]) == len(ab) and max(info["true_residuals"]) <= 1e-10, info
    by = info["iterations_by_precision"]
    assert by.get("double", 0) > 0 and by.get("single", 0) > 0, by
    if sloppy == K.KUQCD_HALF:
        assert by.get("half", 0) > 0, by
    for k in range(len(ab)):
        x = download(slabs, [xk[k] for xk in xs])
        assert O.true_residual(GDIMS, fat, lng, 0, ab[k], b, x) <= 1.2e-10, k


@pytest.mark.gpu
def test_library_calls_follow_torch_stream(cuda):
    """torch's default stream (handle 0) reaches the library as cudaStreamLegacy, never as NULL (which would mean the
    context's own non-blocking stream, unordered with torch's work); a side stream reaches it as itself."""
    from kuqcd_b200 import lib

    assert lib._torch_stream(0).value == lib.CUDA_STREAM_LEGACY
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        assert lib._torch_stream(0).value == side.cuda_stream
    # a buffer zero-filled by torch and then uploaded by the library holds the upload
    slabs, tr, fat, lng = setup_slabs(1, 0.3, 17)
    src = O.make_source(GDIMS, 1, 18)
    for _ in range(3):
        f = slabs[0].field()
        slabs[0].ctx.upload(K.KUQCD_DOUBLE, SL.slab_of_spinor(src, GDIMS, 0, 1), f)
        assert np.array_equal(download(slabs, [f]), src)
