"""CPU tests of the numpy restatement of the learned preconditioner (oracle/ptc_oracle.py): gauge covariance,
adjointness of the backward layer, symmetry and positivity of the Gram operator, and gradients against finite
differences."""
import numpy as np

from oracle import oracle as O
from oracle import ptc_oracle as P

DIMS = (4, 4, 2, 2)
CH = [1, 8, 8]


def setup(seed=0):
    fat, lng = O.make_links(DIMS, 0.4, 7)
    lat = P.Lattice(DIMS, fat)
    rng = np.random.default_rng(seed)
    nw = sum(2 * a * b * 9 for a, b in zip(CH[:-1], CH[1:]))
    Ws = P.weights_from_flat(0.3 * rng.standard_normal(nw), CH)
    return lat, Ws, rng


def test_layer_adjoint_is_adjoint():
    lat, Ws, rng = setup()
    W = Ws[1]
    v = rng.standard_normal((8, 2, lat.vh, 3)) + 1j * rng.standard_normal((8, 2, lat.vh, 3))
    g = rng.standard_normal((8, 2, lat.vh, 3)) + 1j * rng.standard_normal((8, 2, lat.vh, 3))
    lhs = np.vdot(g, P.layer(lat, W, v))
    rhs = np.vdot(P.layer_adjoint(lat, W, g), v)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_gram_operator_is_symmetric_positive():
    """M = P^T N^dag N P: <u, M v> = <M u, v> and <v, M v> > 0 in the real inner product of the solver's fields."""
    lat, Ws, rng = setup()
    for par in (0, 1):
        u = O.make_source(DIMS, par, 11)
        v = O.make_source(DIMS, par, 12)
        Mu, Mv = P.apply(lat, Ws, u, par), P.apply(lat, Ws, v, par)
        assert abs(u @ Mv - Mu @ v) < 1e-12 * np.linalg.norm(Mu) * np.linalg.norm(v)
        assert v @ Mv > 0


def test_gauge_covariance():
    """M(Omega r) = Omega M(r) for a gauge transformation Omega(x) applied to links and fields."""
    lat, Ws, rng = setup()
    vh = lat.vh
    # random SU(3)-like unitary per site (QR of a Gaussian matrix)
    A = rng.standard_normal((2, vh, 3, 3)) + 1j * rng.standard_normal((2, vh, 3, 3))
    Om, _ = np.linalg.qr(A)
    lat2 = P.Lattice(DIMS, O.make_links(DIMS, 0.4, 7)[0])
    for par in (0, 1):
        q = 1 - par
        for mu in range(4):
            # U_mu(x) -> Om(x) U_mu(x) Om(x+mu)^dag
            lat2.U[par, :, mu] = Om[par] @ lat.U[par, :, mu] @ np.conj(np.swapaxes(Om[q][lat.fwd[par, mu]], -1, -2))
    r = O.make_source(DIMS, 0, 3)
    z = P.apply(lat, Ws, r, 0)
    rc = (r[0::2] + 1j * r[1::2]).reshape(vh, 3)
    rt = np.einsum("iab,ib->ia", Om[0], rc).reshape(-1)
    rr = np.empty(2 * rt.size)
    rr[0::2], rr[1::2] = rt.real, rt.imag
    z2 = P.apply(lat2, Ws, rr, 0)
    zc = (z[0::2] + 1j * z[1::2]).reshape(vh, 3)
    zt = np.einsum("iab,ib->ia", Om[0], zc).reshape(-1)
    z2c = z2[0::2] + 1j * z2[1::2]
    assert np.abs(z2c - zt).max() < 1e-12 * np.abs(zt).max()


def test_gradients_match_finite_differences():
    lat, Ws, rng = setup(1)
    r = O.make_source(DIMS, 1, 5)
    e = O.make_source(DIMS, 1, 6)
    L, grads = P.loss_and_grad(lat, Ws, r, e, 1)
    flat = P.flat_from_weights(Ws)
    gflat = P.flat_from_weights(grads)
    h = 1e-6
    for k in rng.choice(flat.size, 24, replace=False):
        fp, fm = flat.copy(), flat.copy()
        fp[k] += h
        fm[k] -= h
        Lp = P.loss_and_grad(lat, P.weights_from_flat(fp, CH), r, e, 1)[0]
        Lm = P.loss_and_grad(lat, P.weights_from_flat(fm, CH), r, e, 1)[0]
        fd = (Lp - Lm) / (2 * h)
        assert abs(fd - gflat[k]) <= 1e-6 * max(1.0, abs(fd)), (k, fd, gflat[k])


def test_bf16_mode_rounds_the_tensor_core_operands():
    """bf16 rounds to nearest with ties to even (through FP32, as the GPU converts), and the BF16-operand network
    differs from the exact one by a few parts in a thousand -- the gap the exact-oracle tolerances allow for."""
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9, -3.14159, 0.0])
    assert list(P.bf16(x)) == [1.0, 1.0, 1.0 + 2 ** -6, 1.0, -3.140625, 0.0]
    lat, Ws, rng = setup(3)
    u = O.make_source(DIMS, 0, 13)
    exact, rounded = P.apply(lat, Ws, u, 0), P.apply(lat, Ws, u, 0, bf=True)
    rel = np.linalg.norm(rounded - exact) / np.linalg.norm(exact)
    assert 1e-5 < rel < 3e-2
