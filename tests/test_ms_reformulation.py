"""CPU check of the recurrences the GPU multishift solver runs (kuqcd_b200/csrc/kq_msrelax.cu, kq_ms_device.cuh),
restated here in numpy on the oracle's dslash, against the reference-order CGM (oracle/hisq_oracle.c, itself pinned to
the reference library):

* <p, A p> = sigma0 |p|^2 + |D_qp p|^2 for A = sigma0 - D_pq D_qp, because D_pq = -D_qp^dag (the backward hops apply
  the adjoints of the same links), so the beta step can follow the first dslash and s is never stored;
* |p|^2 carried by the recurrence |p'|^2 = |r'|^2 + a0^2 |p|^2 (r' is orthogonal to p);
* shift vectors updated once per window of 16 iterations from a ring of residuals, with the window coefficients
  accumulated by the scalar steps.

Iteration counts within one of the reference order and the same solutions up to rounding."""
import numpy as np
import pytest

from oracle import oracle as O

W = 16  # window of the GPU solver (kWin)


def windowed_multishift(dims, fat, lng, parity, sh, b, tol, max_iter):
    """sh: reference semantics (sh[0] absolute, sh[j] relative to sh[0]).  Returns (xs, iterations)."""
    ns = len(sh)
    D = lambda v, out_parity: O.dslash(dims, fat, lng, v, out_parity)  # noqa: E731
    a = np.zeros(ns)
    B, Z, Zm1 = np.ones(ns), np.ones(ns), np.ones(ns)
    c, e = np.ones(ns), np.zeros(ns)
    d, f = np.zeros((ns, W)), np.zeros((ns, W))
    Bm1, rr, pp = 1.0, float(b @ b), float(b @ b)
    mt, wpos, wmax, it = ns, 0, ns, 0
    p0 = b.copy()
    ring = [np.zeros_like(b) for _ in range(W)]
    ring[0] = b.copy()
    x = [np.zeros_like(b) for _ in range(ns)]
    pw = [b.copy() for _ in range(ns)]

    def flush(n, kmax):
        for k in range(kmax):
            rs = sum(d[k, l] * ring[(l + 1) % W] for l in range(n))
            fs = sum(f[k, l] * ring[(l + 1) % W] for l in range(n))
            x[k] = x[k] + e[k] * pw[k] + fs
            pw[k] = c[k] * pw[k] + rs

    while mt > 0 and it < max_iter:
        # K1: tmp = D_qp p0, |tmp|^2, beta step with <p0, A p0> = sigma0 |p0|^2 + |tmp|^2
        tmp = D(p0, 1 - parity)
        pAp = sh[0] * pp + float(tmp @ tmp)
        B0 = -rr / pAp
        jw = wpos
        if jw == 0:
            c[:], e[:], d[:], f[:] = 1.0, 0.0, 0.0, 0.0
            wmax = mt
        for j in range(1, mt):
            rr1 = Bm1 * Zm1[j] / (B0 * a[0] * (Zm1[j] - Z[j]) + Zm1[j] * Bm1 * (1.0 - sh[j] * B0))
            Zm1[j], Z[j], B[j] = Z[j], Z[j] * rr1, B0 * rr1
        B[0], Bm1 = B0, B0
        for k in range(mt):
            e[k] -= B[k] * c[k]
            f[k, :jw] -= B[k] * d[k, :jw]
        nu = mt
        # K2: r <- r + B0 (sigma0 p0 - D_pq tmp) into the ring, |r|^2, alpha step
        r = ring[it % W] + B0 * (sh[0] * p0 - D(tmp, parity))
        ring[(it + 1) % W] = r
        lam2 = float(r @ r)
        a0 = lam2 / rr
        a[0] = a0
        for j in range(1, nu):
            a[j] = a0 * Z[j] * B[j] / (Zm1[j] * B0)
        for k in range(nu):
            c[k] *= a[k]
            d[k, :jw] *= a[k]
            d[k, jw] = Z[k]
        while mt > 0 and Z[mt - 1] ** 2 * lam2 < tol:
            mt -= 1
        rr, pp = lam2, lam2 + a0 * a0 * pp
        it += 1
        wpos = jw + 1
        # K3: p0 <- r + a0 p0
        p0 = r + a0 * p0
        if wpos == W or mt == 0 or it >= max_iter:
            flush(wpos, wmax)
            wpos = 0
    return x, it


def test_dslash_is_anti_hermitian_between_parities():
    """<y, D_pq x> = -<D_qp y, x>: what makes <p, A p> = sigma |p|^2 + |D_qp p|^2."""
    dims = (4, 4, 4, 6)
    fat, lng = O.make_links(dims, 0.35, 8)
    xq = O.make_source(dims, 1, 3)  # field on the odd sites
    yp = O.make_source(dims, 0, 4)  # field on the even sites
    lhs = float(yp @ O.dslash(dims, fat, lng, xq, 0))
    rhs = -float(O.dslash(dims, fat, lng, yp, 1) @ xq)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    p = O.make_source(dims, 0, 9)
    sigma = 0.07
    pAp = float(p @ (sigma * p - O.dslash(dims, fat, lng, O.dslash(dims, fat, lng, p, 1), 0)))
    tq = O.dslash(dims, fat, lng, p, 1)
    assert abs(pAp - (sigma * float(p @ p) + float(tq @ tq))) <= 1e-12 * pAp


@pytest.mark.parametrize("dims,parity,nshift", [((8, 8, 8, 8), 0, 12), ((6, 4, 4, 6), 1, 12), ((4, 4, 4, 8), 0, 16)])
def test_gpu_recurrences_match_reference_order(dims, parity, nshift):
    """Iteration counts agree to one.  (On a lattice as small as 4^4, where the solve takes about a third as many
    iterations as the system has unknowns, rounding alone moves the stop by a few iterations: the windowed form
    with either step-length formula stops at 282 there against the reference order's 287, solutions equal to
    6e-12.)"""
    fat, lng = O.make_links(dims, 0.3, 40 + nshift)
    b = O.make_source(dims, parity, 7)
    m, sig = 0.05, np.logspace(-4, 0, nshift)
    ab = m * m + sig
    sh = [ab[0]] + list(sig[1:] - sig[0])
    tol = (1e-10) ** 2 * float(b @ b)
    xr, itr = O.cgm(dims, fat, lng, parity, sh, b, tol, 5000)
    xw, itw = windowed_multishift(dims, fat, lng, parity, sh, b, tol, 5000)
    assert abs(itw - itr) <= 1, (itw, itr)
    for k in range(nshift):
        assert np.abs(xw[k] - xr[k]).max() <= 1e-9 * np.abs(xr[k]).max(), k
        assert O.true_residual(dims, fat, lng, parity, ab[k], b, xw[k]) < 2e-10, k
