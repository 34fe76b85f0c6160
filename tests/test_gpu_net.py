"""GPU tests of the learned preconditioner: forward and backward kernels against the numpy oracle
(oracle/ptc_oracle.py, itself checked against finite differences), training on solver-generated pairs, and the FCG
polish with and without the trained network."""
import numpy as np
import pytest
import torch

import kuqcd_b200 as K
from kuqcd_b200 import learned as LN
from oracle import oracle as O
from oracle import ptc_oracle as P

CH = (1, 8, 8)  # N: 1 -> 8 -> 8 channels; M = N^dag N runs four layers


def ctx_for(dims, eps, seed, mass_links=None):
    fat, lng = O.make_links(dims, eps, seed)
    ctx = K.Context(dims)
    ctx.load_links(K.KUQCD_FAT_LINK, fat)
    ctx.load_links(K.KUQCD_LONG_LINK, lng)
    return ctx, fat, lng


def field(ctx):
    return torch.zeros(ctx.spinor_bytes(K.KUQCD_DOUBLE), dtype=torch.uint8, device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("parity", [0, 1])
def test_net_forward_matches_oracle(cuda, parity):
    dims = (8, 4, 4, 4)
    ctx, fat, lng = ctx_for(dims, 0.4, 3)
    net = K.Net(ctx, CH)
    w = (0.3 * np.random.default_rng(0).standard_normal(net.nw)).astype(np.float32)
    net.weights = w
    r = O.make_source(dims, parity, 9)
    a, z = field(ctx), field(ctx)
    ctx.upload(K.KUQCD_DOUBLE, r, a)
    net.apply(a, z, parity)
    got = ctx.download(K.KUQCD_DOUBLE, z)
    lat = P.Lattice(dims, fat)
    Ws = P.weights_from_flat(w.astype(np.float64), CH)
    want = P.apply(lat, Ws, r, parity)
    # against exact arithmetic: BF16 operands in four layers, a few parts in a thousand
    assert np.linalg.norm(got - want) <= 3e-2 * np.linalg.norm(want)
    # against the oracle that rounds the tensor-core operands as the kernels do: what is left are the few BF16
    # roundings that an FP32 transported value and its FP64 counterpart take to different neighbours (up to 1.4e-4
    # on this small lattice, measured on the oracle with FP32 transports) and FP32 accumulation; a wrong gather index
    # in a single path would leave a relative error near 1/9, the BF16 operands themselves 1.6e-3
    want16 = P.apply(lat, Ws, r, parity, bf=True)
    assert np.linalg.norm(got - want16) <= 5e-4 * np.linalg.norm(want16)


@pytest.mark.gpu
@pytest.mark.parametrize("whole_tile", ["0", "1"])
def test_net_forward_kernels_agree_on_a_ragged_lattice(cuda, monkeypatch, whole_tile):
    """The K-chunked forward kernel of the 8-channel layers and the whole-tile kernel both match the BF16-rounding
    oracle, on a lattice whose last tile is partly past the end (Vh = 1350 sites, 11 tiles of 128)."""
    monkeypatch.setenv("KUQCD_PTC_WHOLE_TILE", whole_tile)
    import subprocess
    import sys
    code = f"""
import numpy as np, torch, kuqcd_b200 as K
from oracle import oracle as O
from oracle import ptc_oracle as P
dims = (10, 6, 5, 9)
fat, lng = O.make_links(dims, 0.35, 12)
ctx = K.Context(dims)
ctx.load_links(K.KUQCD_FAT_LINK, fat)
ctx.load_links(K.KUQCD_LONG_LINK, lng)
net = K.Net(ctx, (1, 8, 8))
w = (0.3 * np.random.default_rng(3).standard_normal(net.nw)).astype(np.float32)
net.weights = w
r = O.make_source(dims, 1, 4)
a = torch.zeros(ctx.spinor_bytes(K.KUQCD_DOUBLE), dtype=torch.uint8, device='cuda')
z = torch.zeros_like(a)
ctx.upload(K.KUQCD_DOUBLE, r, a)
net.apply(a, z, 1)
got = ctx.download(K.KUQCD_DOUBLE, z)
want = P.apply(P.Lattice(dims, fat), P.weights_from_flat(w.astype(np.float64), (1, 8, 8)), r, 1, bf=True)
print(float(np.linalg.norm(got - want) / np.linalg.norm(want)))
"""
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr[-3000:]
    assert float(out.stdout.strip().splitlines()[-1]) <= 2e-4


@pytest.mark.gpu
def test_net_apply_is_symmetric_positive(cuda):
    """M = N^dag N: <u, M v> = <M u, v> up to BF16 rounding, and <v, M v> > 0."""
    dims = (8, 4, 4, 4)
    ctx, fat, lng = ctx_for(dims, 0.4, 5)
    net = K.Net(ctx, CH)
    net.weights = (0.3 * np.random.default_rng(2).standard_normal(net.nw)).astype(np.float32)
    u, v = O.make_source(dims, 0, 21), O.make_source(dims, 0, 22)
    du, dv, mu, mv = field(ctx), field(ctx), field(ctx), field(ctx)
    ctx.upload(K.KUQCD_DOUBLE, u, du)
    ctx.upload(K.KUQCD_DOUBLE, v, dv)
    net.apply(du, mu, 0)
    net.apply(dv, mv, 0)
    Mu, Mv = ctx.download(K.KUQCD_DOUBLE, mu), ctx.download(K.KUQCD_DOUBLE, mv)
    assert abs(u @ Mv - Mu @ v) <= 2e-2 * np.linalg.norm(Mu) * np.linalg.norm(v)
    assert v @ Mv > 0 and u @ Mu > 0


@pytest.mark.gpu
def test_net_gradient_matches_oracle(cuda):
    dims = (8, 4, 4, 4)
    ctx, fat, lng = ctx_for(dims, 0.4, 4)
    net = K.Net(ctx, CH)
    w = (0.3 * np.random.default_rng(1).standard_normal(net.nw)).astype(np.float32)
    net.weights = w
    r = O.make_source(dims, 0, 5)
    e = O.make_source(dims, 0, 6)
    dr, de = field(ctx), field(ctx)
    ctx.upload(K.KUQCD_DOUBLE, r, dr)
    ctx.upload(K.KUQCD_DOUBLE, e, de)
    net.zero_grad()
    loss = net.train_pair(dr, de, 0, float(e @ e))
    g = net.grad().astype(np.float64)
    lat = P.Lattice(dims, fat)
    Ws = P.weights_from_flat(w.astype(np.float64), CH)
    Lw, grads = P.loss_and_grad(lat, Ws, r, e, 0)
    gw = P.flat_from_weights(grads)
    assert abs(loss - Lw) <= 3e-2 * Lw
    assert np.linalg.norm(g - gw) <= 5e-2 * np.linalg.norm(gw)
    # against the oracle that rounds the tensor-core operands as the kernels do, per layer (the chain rule through
    # the adjoint layers)
    L16, grads16 = P.loss_and_grad(lat, Ws, r, e, 0, bf=True)
    g16 = P.flat_from_weights(grads16)
    assert abs(loss - L16) <= 1e-4 * L16
    off = 0
    for ci, co in zip(CH[:-1], CH[1:]):
        n = 2 * ci * co * 9
        assert np.linalg.norm(g[off:off + n] - g16[off:off + n]) <= 2e-4 * np.linalg.norm(g16[off:off + n])
        off += n


@pytest.mark.gpu
def test_fcg_polish_plain_cg_converges(cuda):
    dims = (8, 4, 4, 8)
    ctx, fat, lng = ctx_for(dims, 0.3, 8)
    b = O.make_source(dims, 0, 8)
    db = field(ctx)
    ctx.upload(K.KUQCD_DOUBLE, b, db)
    sig = [0.01, 0.2]
    dx = torch.zeros(2 * ctx.spinor_bytes(K.KUQCD_DOUBLE), dtype=torch.uint8, device="cuda")
    info = K.fcg_polish(ctx, None, db, dx, sig, rel_residual=1e-10)
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    for k, s in enumerate(sig):
        x = ctx.download(K.KUQCD_DOUBLE, dx[k * vb:(k + 1) * vb])
        assert O.true_residual(dims, fat, lng, 0, s, b, x) <= 1.05e-10
        assert info.true_residual[k] <= 1e-10


@pytest.mark.gpu
def test_trained_network_reduces_polish_iterations(cuda):
    """Train on solver-generated pairs from 3 gauge fields, evaluate on a held-out field: the FCG polish with the
    network (on the three smallest shifts) needs fewer iterations than the unpreconditioned polish from the same
    loose multishift solution, and every shift still reaches the FP64 true-residual target."""
    dims = (8, 8, 8, 8)
    eps, mass = 0.45, 0.05
    sig0 = mass * mass + 1e-4
    train_ctx = [ctx_for(dims, eps, 100 + s)[0] for s in range(3)]
    data = [(c, LN.make_pairs(c, sig0, 3, 10 * i)) for i, c in enumerate(train_ctx)]
    net = K.Net(train_ctx[0], CH)
    c0 = np.mean([np.sqrt(e2 / float((r.view(torch.float64) ** 2).sum())) for c, ps in data for r, e, e2 in ps])
    net.weights = LN.init_weights(CH, c0, noise=0.01)
    before = LN.eval_loss(net, data)
    LN.train(net, data, steps=150, lr=5e-3, batch=3)
    after = LN.eval_loss(net, data)
    assert after < 0.8 * before
    # held-out field
    ctx, fat, lng = ctx_for(dims, eps, 999)
    b = O.make_source(dims, 0, 77)
    db = field(ctx)
    ctx.upload(K.KUQCD_DOUBLE, b, db)
    sig = list(mass * mass + np.logspace(-4, 0, 6))
    vb = ctx.spinor_bytes(K.KUQCD_DOUBLE)
    dx1 = torch.zeros(6 * vb, dtype=torch.uint8, device="cuda")
    dx2 = torch.zeros(6 * vb, dtype=torch.uint8, device="cuda")
    _, plain = LN.solve_with_polish(ctx, None, db, dx1, sig)
    _, learned = LN.solve_with_polish(ctx, net, db, dx2, sig, net_max_shift=0.01)
    assert plain.status == 0 and learned.status == 0
    for k, s in enumerate(sig):
        x = ctx.download(K.KUQCD_DOUBLE, dx2[k * vb:(k + 1) * vb])
        assert O.true_residual(dims, fat, lng, 0, s, b, x) <= 1.05e-10
    assert learned.iter > 0
    assert learned.iter_refine < plain.iter_refine, (learned.iter_refine, plain.iter_refine)
