// Scalar steps of the windowed multishift CG (device side), shared by the single-system solver (kq_msrelax.cu)
// and the batched multi-system solver (kq_batch.cu).  They restate the recurrences of inverter_cgm.cpp:45-77 and
// accumulate the window coefficients of the deferred shift updates.
#pragma once
#include "kq_msrelax.h"

namespace kq {

// ---------------------------------------------------------------------------------------------------- scalar steps
// Both steps are run by the 32 lanes of one warp (of the last block to finish the reduction).  Every lane reads the
// shared scalars before any lane writes (__syncwarp); then lane l computes the per-shift scalars of shifts l and
// l + 32, and after a __syncwarp the window coefficients are updated one (shift, position) item per lane.  Each
// value has one writer per phase, so the result is that of the reference's sequential loops, while the loads of
// different shifts overlap instead of forming a chain of dependent global-memory round trips (this runs in the
// tail of a kernel, after every other block has finished).  The item loop keeps few values live, so the step does
// not raise the register count of the dslash kernel that hosts it.

// beta step (inverter_cgm.cpp:48-57, 61-63): B_0 = -|r|^2 / <p, A p>, the shifted B_k and zeta_k, and
// x_k -= B_k p_k in the window representation of p_k
__device__ __forceinline__ void ms_step_beta(MsState *st, double pAp)
{
    const int lane = threadIdx.x & 31;
    const double rNorm2 = st->rNorm2, Bm1 = st->Bm1, a0 = st->a[0];
    const int mt = st->maxTerm, ns = st->ns, jw = st->wpos;  // ring positions 0..jw-1 are in use
    const double B0 = -rNorm2 / pAp;
    const bool bad = !(pAp != 0.0) || !isfinite(B0);
    __syncwarp();
    if (bad) {
        if (lane == 0) {
            st->pAp = pAp;
            st->status = KQ_STATUS_BREAKDOWN;
            st->active = 0;
            st->halt = 1;
        }
        return;
    }
#pragma unroll 1
    for (int k = lane; k < mt; k += 32) {
        double Bk = B0;
        if (k > 0) {
            const double zm1 = st->Zm1[k], z = st->Z[k], sh = st->shift[k];
            const double rr1 = Bm1 * zm1 / (B0 * a0 * (zm1 - z) + zm1 * Bm1 * (1.0 - sh * B0));
            st->Zm1[k] = z;
            st->Z[k] = z * rr1;
            Bk = B0 * rr1;
        }
        st->B[k] = Bk;
    }
    __syncwarp();
    if (jw == 0) {
        // first iteration of a window: identity representation p = p_old (c = 1), x = x_old, then x -= B p
#pragma unroll 1
        for (int k = lane; k < ns; k += 32) {
            st->c[k] = 1.0;
            st->e[k] = k < mt ? -st->B[k] : 0.0;
        }
#pragma unroll 1
        for (int t = lane; t < ns * kWin; t += 32) {
            const int k = t / kWin, l = t - k * kWin;
            st->d[k][l] = 0.0;
            st->f[k][l] = 0.0;
        }
    } else {
        // e_k -= B_k c_k (item l = jw) and f_kl -= B_k d_kl (items l < jw)
        const int per = jw + 1;
#pragma unroll 1
        for (int t = lane; t < mt * per; t += 32) {
            const int k = t / per, l = t - k * per;
            const double Bk = st->B[k];
            if (l == jw) st->e[k] -= Bk * st->c[k];
            else st->f[k][l] -= Bk * st->d[k][l];
        }
    }
    if (lane == 0) {
        st->pAp = pAp;
        st->Bm1 = B0;
        st->nupd = mt;
        if (jw == 0) st->wmax = mt;
    }
}

// alpha step (inverter_cgm.cpp:58-60, 64-77): a_0 = |r_new|^2 / |r|^2, the shifted a_k, p_k = Z_k r_new + a_k p_k
// in the window representation, and the converged shifts dropped from the top (zeta_k^2 |r|^2 < tol)
__device__ __forceinline__ void ms_step_alpha(MsState *st, double lambda2)
{
    const int lane = threadIdx.x & 31;
    const double rNorm2 = st->rNorm2, B0 = st->B[0], tol = st->tol;
    const int nu = st->nupd, jw = st->wpos, mt0 = st->maxTerm, halt0 = st->halt;
    const double a0 = lambda2 / rNorm2;
    __syncwarp();
    // a_k, and the new maxTerm: one above the highest shift still above tolerance (the reference's do-while)
    int mt = 0;
#pragma unroll
    for (int base = 0; base < kMaxShift; base += 32) {
        const int k = base + lane;
        bool keep = false;
        if (k < nu) st->a[k] = k == 0 ? a0 : a0 * st->Z[k] * st->B[k] / (st->Zm1[k] * B0);
        if (k < mt0) {
            const double z = st->Z[k];
            keep = !(z * z * lambda2 < tol);
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (m) mt = base + 32 - __clz((int)m);
    }
    __syncwarp();
    // c_k *= a_k (item l = jw, which also records Z_k as the weight of the new residual), d_kl *= a_k (l < jw)
    const int per = jw + 1;
#pragma unroll 1
    for (int t = lane; t < nu * per; t += 32) {
        const int k = t / per, l = t - k * per;
        const double ak = st->a[k];
        if (l == jw) {
            st->c[k] *= ak;
            st->d[k][jw] = st->Z[k];
        } else {
            st->d[k][l] *= ak;
        }
    }
    if (lane == 0) {
        st->lambda2 = lambda2;
        st->a[0] = a0;
        st->rNorm2 = lambda2;
        // |p_new|^2 = |r_new|^2 + a0^2 |p|^2, since the step makes r_new orthogonal to p
        st->pp = lambda2 + a0 * a0 * st->pp;
        st->maxTerm = mt;
        st->iter += 1;
        st->wpos = jw + 1;
        const bool finite = isfinite(lambda2);
        if (!finite) {
            st->status = KQ_STATUS_BREAKDOWN;
            st->halt = 1;
        }
        st->active = (mt > 0 && st->iter < st->max_iter && !halt0 && finite) ? 1 : 0;
        if (!st->active && st->running) atomicSub(st->running, 1);
        // relaxed operator precision for the next iteration, from the base residual (the batched solver's)
        const double rel2 = lambda2 / st->bnorm2;
        st->next_mode =
            (st->rho16_2 > 0.0 && rel2 < st->rho16_2) ? 2 : (st->rho32_2 > 0.0 && rel2 < st->rho32_2) ? 1 : 0;
    }
}

// Windowed shift update of one site, one colour component at a time (keeps W ring values in registers, not 6 W):
//   p_k <- c_k p_k + sum_l d_kl r_l ,  x_k <- x_k + e_k p_k + sum_l f_kl r_l   for k < kmax.
// Window position l (0-based) holds r^(i0+l+1) in ring slot (l+1) % W; positions >= n are unused (zero weight).
// FP64 spinor fields are three double2 planes of pv sites (kq_prec.cuh).  KU shifts at a time: their p and x are
// loaded before any of them is stored (the stores could alias later loads for the compiler), so KU x 2 loads per
// thread are in flight instead of 2.
__device__ __forceinline__ void window_update_one(const double2 p, const double2 x, const double2 *rl, double c,
                                                  double e, const double *d, const double *f, double2 &pn,
                                                  double2 &xn)
{
    pn = make_double2(c * p.x, c * p.y);
    xn = make_double2(x.x + e * p.x, x.y + e * p.y);
#pragma unroll
    for (int l = 0; l < kWin; ++l) {
        pn.x += d[l] * rl[l].x;
        pn.y += d[l] * rl[l].y;
        xn.x += f[l] * rl[l].x;
        xn.y += f[l] * rl[l].y;
    }
}

template <int KU = 1>
__device__ __forceinline__ void window_update_site(const char *ring, size_t vb, int pv, int i, int n, int kmax,
                                                   const double *sc, const double *se, const double (*sd)[kWin],
                                                   const double (*sf)[kWin], char *pw0, char *x0)
{
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
        const size_t off = (size_t)c * pv + i;
        double2 rl[kWin];
#pragma unroll
        for (int l = 0; l < kWin; ++l)
            rl[l] = l < n ? __ldg(reinterpret_cast<const double2 *>(ring + (size_t)((l + 1) % kWin) * vb) + off)
                          : make_double2(0.0, 0.0);
        int k = 0;
#pragma unroll 1
        for (; k + KU <= kmax; k += KU) {
            double2 p[KU], x[KU];
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                p[u] = reinterpret_cast<const double2 *>(pw0 + (k + u) * vb)[off];
                x[u] = reinterpret_cast<const double2 *>(x0 + (k + u) * vb)[off];
            }
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                double2 pn, xn;
                window_update_one(p[u], x[u], rl, sc[k + u], se[k + u], sd[k + u], sf[k + u], pn, xn);
                reinterpret_cast<double2 *>(pw0 + (k + u) * vb)[off] = pn;
                reinterpret_cast<double2 *>(x0 + (k + u) * vb)[off] = xn;
            }
        }
#pragma unroll 1
        for (; k < kmax; ++k) {
            double2 *pp = reinterpret_cast<double2 *>(pw0 + k * vb) + off;
            double2 *xp = reinterpret_cast<double2 *>(x0 + k * vb) + off;
            double2 pn, xn;
            window_update_one(*pp, *xp, rl, sc[k], se[k], sd[k], sf[k], pn, xn);
            *pp = pn;
            *xp = xn;
        }
    }
}

}  // namespace kq
