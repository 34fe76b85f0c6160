"""ORACLE / TEST INFRASTRUCTURE ONLY — numpy float64 restatement of the parallel-transport convolution network of
the learned preconditioner (kuqcd_b200/csrc/kq_ptc.cu, kq_net.cu), with its gradients.  Used by tests as the
checker of the GPU forward and backward kernels (and checked itself against finite differences).

Fields are arrays of shape (C, 2, Vh, 3) complex: channel, parity, checkerboard index, colour.  Links: the fat
links of the host record scaled by 1/2 (the device copy the CUDA kernels read).  Layer:

    y_o(x) = sum_c sum_p W[o, c, p] (T_p v_c)(x),  p = 0: identity, 1+2mu: F_mu(x) v(x+mu),
                                                   2+2mu: F_mu(x-mu)^dag v(x-mu)

and the preconditioner is the Gram operator M = P^T N^dag N P of the chain N = L_{K-1} ... L_0 (P: embedding of
one parity into a one-channel full-lattice field).

With bf16=True every function rounds what the GPU rounds: the transported inputs T_p v (computed in FP32, then
rounded to BF16 for the tensor cores), the weights (BF16 operands) and, in the weight gradient, the output gradient
(BF16 operand of the gradient GEMM); sums stay exact (float64), as the tensor cores accumulate in FP32.  That
oracle agrees with the GPU to FP32 accumulation error, so tests can hold the kernels to ~1e-4 instead of the
few-parts-in-a-thousand gap between BF16 and exact arithmetic.
"""
from __future__ import annotations

import numpy as np


def bf16(a):
    """Round to the nearest BF16 (ties to even), through FP32 as the GPU does (float64 -> FP32 -> BF16); complex
    arrays are rounded per real and imaginary part."""
    if np.iscomplexobj(a):
        return bf16(a.real) + 1j * bf16(a.imag)
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


class Lattice:
    def __init__(self, dims, fat_record):
        self.dims = tuple(dims)
        nx, ny, nz, nt = dims
        self.vh = nx * ny * nz * nt // 2
        hx = nx // 2
        i = np.arange(self.vh)
        xcb = i % hx
        r = i // hx
        y = r % ny
        r //= ny
        z = r % nz
        t = r // nz
        self.fwd = np.zeros((2, 4, self.vh), dtype=np.int64)
        self.bwd = np.zeros((2, 4, self.vh), dtype=np.int64)
        for par in (0, 1):
            x = 2 * xcb + ((y + z + t + par) & 1)
            c = [x, y, z, t]
            n = [nx, ny, nz, nt]
            for mu in range(4):
                for hop, tab in ((1, self.fwd), (-1, self.bwd)):
                    d = list(c)
                    d[mu] = (c[mu] + hop) % n[mu]
                    tab[par, mu] = (d[0] >> 1) + hx * (d[1] + ny * (d[2] + nz * d[3]))
        F = fat_record.reshape(2, self.vh, 4, 9, 2)
        self.U = 0.5 * (F[..., 0] + 1j * F[..., 1]).reshape(2, self.vh, 4, 3, 3)  # [par, i, mu, row, col]

    def transports(self, v):
        """v: (2, Vh, 3) -> list of 9 transported fields (identity, fwd mu, bwd mu ...)."""
        out = [v]
        for mu in range(4):
            f = np.empty_like(v)
            b = np.empty_like(v)
            for par in (0, 1):
                q = 1 - par
                vn = v[q][self.fwd[par, mu]]
                f[par] = np.einsum("iab,ib->ia", self.U[par, :, mu], vn)
                nb = self.bwd[par, mu]
                ub = self.U[q][nb, mu]
                b[par] = np.einsum("iba,ib->ia", ub.conj(), v[q][nb])
            out += [f, b]
        return out


def _round(x, on):
    return bf16(x) if on else x


def layer(lat, W, v, bf=False):
    """W: (Cout, Cin, 9) complex; v: (Cin, 2, Vh, 3)."""
    W = _round(W, bf)
    y = np.zeros((W.shape[0],) + v.shape[1:], dtype=complex)
    for c in range(W.shape[1]):
        ts = lat.transports(v[c])
        for p in range(9):
            y += W[:, c, p][:, None, None, None] * _round(ts[p], bf)[None]
    return y


def layer_adjoint(lat, W, g, bf=False):
    """Adjoint of `layer`: T_fwd^dag = T_bwd and vice versa, weights conjugate-transposed."""
    swap = [0, 2, 1, 4, 3, 6, 5, 8, 7]
    W = _round(W, bf)
    out = np.zeros((W.shape[1],) + g.shape[1:], dtype=complex)
    for o in range(W.shape[0]):
        ts = lat.transports(g[o])
        for p in range(9):
            out += np.conj(W[o, :, p])[:, None, None, None] * _round(ts[swap[p]], bf)[None]
    return out


def embed(r, parity, vh):
    v = np.zeros((1, 2, vh, 3), dtype=complex)
    v[0, parity] = (r[0::2] + 1j * r[1::2]).reshape(vh, 3)
    return v


def extract(y, parity):
    z = y[0, parity].reshape(-1)
    out = np.empty(2 * z.size)
    out[0::2], out[1::2] = z.real, z.imag
    return out


def weights_from_flat(flat, channels):
    Ws, off = [], 0
    for ci, co in zip(channels[:-1], channels[1:]):
        n = co * ci * 9
        w = flat[off:off + 2 * n]
        Ws.append((w[0::2] + 1j * w[1::2]).reshape(co, ci, 9))
        off += 2 * n
    return Ws


def flat_from_weights(Ws):
    return np.concatenate([np.stack([W.real.ravel(), W.imag.ravel()], 1).ravel() for W in Ws])


def _chains(lat, Ws, r, parity, bf=False):
    """Forward chain a_0 = embed(r), a_{l+1} = L_l a_l and adjoint chain c_K = a_K, c_l = L_l^dag c_{l+1}."""
    acts = [embed(r, parity, lat.vh)]
    for W in Ws:
        acts.append(layer(lat, W, acts[-1], bf))
    cs = [None] * len(Ws) + [acts[-1]]
    for li in range(len(Ws) - 1, -1, -1):
        cs[li] = layer_adjoint(lat, Ws[li], cs[li + 1], bf)
    return acts, cs


def apply(lat, Ws, r, parity, bf=False):
    """M(r) = extract(N^dag N embed(r)), N = L_{K-1} ... L_0 (the Gram form kq_net.cu evaluates)."""
    return extract(_chains(lat, Ws, r, parity, bf)[1][0], parity)


def _wgrad(lat, v, g, ncout, swap=False, bf=False):
    """sum over sites and colours of g_o * conj(T_p v_c): the complex gradient of a layer's weights W[o, c, p]
    (swap: path labels of the adjoint layer)."""
    order = [0, 2, 1, 4, 3, 6, 5, 8, 7] if swap else list(range(9))
    g = _round(g, bf)
    dW = np.zeros((ncout, v.shape[0], 9), dtype=complex)
    for c in range(v.shape[0]):
        ts = lat.transports(v[c])
        for p in range(9):
            dW[:, c, p] = (g * np.conj(_round(ts[order[p]], bf))[None]).sum(axis=(1, 2, 3))
    return dW


def loss_and_grad(lat, Ws, r, e, parity, bf=False):
    """L = |M(r) - e|^2 / |e|^2 and dL/dW (complex, re part = dL/dW_re, im part = dL/dW_im) per layer; each layer
    collects one term through L_l and one through L_l^dag (whose weights are conj(W)^T, hence the conj)."""
    acts, cs = _chains(lat, Ws, r, parity, bf)
    y = extract(cs[0], parity)
    e2 = float(e @ e)
    L = float(((y - e) ** 2).sum()) / e2
    d = 2 * (y - e) / e2
    g = np.zeros_like(cs[0])
    g[0, parity] = (d[0::2] + 1j * d[1::2]).reshape(lat.vh, 3)
    K = len(Ws)
    grads = [np.zeros_like(W) for W in Ws]
    for li in range(K):  # adjoint chain: g = dL/dc_li
        W = Ws[li]
        dWa = _wgrad(lat, cs[li + 1], g, W.shape[1], swap=True, bf=bf)  # [i, o, p] of the adjoint layer
        grads[li] += np.conj(dWa.transpose(1, 0, 2))
        g = layer(lat, W, g, bf)
    for li in range(K - 1, -1, -1):  # forward chain: g = dL/da_{li+1}
        W = Ws[li]
        grads[li] += _wgrad(lat, acts[li], g, W.shape[0], bf=bf)
        if li > 0:
            g = layer_adjoint(lat, W, g, bf)
    return L, grads
