// Scalar steps of the windowed multishift CG (device side), shared by the single-system solver (kq_msrelax.cu)
// and the batched multi-system solver (kq_batch.cu).  They restate the recurrences of inverter_cgm.cpp:45-77 and
// accumulate the window coefficients of the deferred shift updates.
#pragma once
#include "kq_msrelax.h"

namespace kq {

// ---------------------------------------------------------------------------------------------------- scalar steps
__device__ __forceinline__ void ms_step_beta(MsState *st, double pAp)
{
    st->pAp = pAp;
    const double B0 = -st->rNorm2 / pAp;
    if (!(pAp != 0.0) || !isfinite(B0)) {
        st->status = KQ_STATUS_BREAKDOWN;
        st->active = 0;
        st->halt = 1;
        return;
    }
    const int mt = st->maxTerm;
    if (st->wpos == 0) {  // first iteration of a window: identity representation p = p_old, x = x_old
        for (int k = 0; k < st->ns; ++k) {
            st->c[k] = 1.0;
            st->e[k] = 0.0;
            for (int l = 0; l < kWin; ++l) st->d[k][l] = st->f[k][l] = 0.0;
        }
        st->wmax = mt;
    }
    st->B[0] = B0;
    const double Bm1 = st->Bm1, a0 = st->a[0];
    for (int j = 1; j < mt; ++j) {
        const double rr1 = Bm1 * st->Zm1[j] /
                           (B0 * a0 * (st->Zm1[j] - st->Z[j]) + st->Zm1[j] * Bm1 * (1.0 - st->shift[j] * B0));
        st->Zm1[j] = st->Z[j];
        st->Z[j] = st->Z[j] * rr1;
        st->B[j] = B0 * rr1;
    }
    st->Bm1 = B0;
    // x_k -= B_k p_k with p_k in its current window representation
    const int jw = st->wpos;  // ring positions 0..jw-1 are in use
    for (int k = 0; k < mt; ++k) {
        const double Bk = st->B[k];
        st->e[k] -= Bk * st->c[k];
        for (int l = 0; l < jw; ++l) st->f[k][l] -= Bk * st->d[k][l];
    }
    st->nupd = mt;
}

__device__ __forceinline__ void ms_step_alpha(MsState *st, double lambda2)
{
    st->lambda2 = lambda2;
    st->a[0] = lambda2 / st->rNorm2;
    st->rNorm2 = lambda2;
    const int nu = st->nupd;
    for (int j = 1; j < nu; ++j) st->a[j] = st->a[0] * st->Z[j] * st->B[j] / (st->Zm1[j] * st->B[0]);
    // p_k = Z_k r^(new) + a_k p_k
    const int jw = st->wpos;
    for (int k = 0; k < nu; ++k) {
        const double ak = st->a[k];
        st->c[k] *= ak;
        for (int l = 0; l < jw; ++l) st->d[k][l] *= ak;
        st->d[k][jw] = st->Z[k];
    }
    int mt = st->maxTerm;
    double lambda;
    do {
        lambda = st->Z[mt - 1] * st->Z[mt - 1] * lambda2;
        if (lambda < st->tol) mt--;
    } while (mt > 0 && lambda < st->tol);
    st->maxTerm = mt;
    st->iter += 1;
    st->wpos = jw + 1;
    if (!isfinite(lambda2)) {
        st->status = KQ_STATUS_BREAKDOWN;
        st->halt = 1;
    }
    st->active = (mt > 0 && st->iter < st->max_iter && !st->halt) ? 1 : 0;
    if (!st->active && st->running) atomicSub(st->running, 1);
    // relaxed operator precision for the next iteration, from the base residual
    const double rel2 = lambda2 / st->bnorm2;
    st->mode = (st->rho16_2 > 0.0 && rel2 < st->rho16_2) ? 2 : (st->rho32_2 > 0.0 && rel2 < st->rho32_2) ? 1 : 0;
}

// Windowed shift update of one site, one colour component at a time (keeps 8 ring values in registers, not 48):
//   p_k <- c_k p_k + sum_l d_kl r_l ,  x_k <- x_k + e_k p_k + sum_l f_kl r_l   for k < kmax.
// Window position l (0-based) holds r^(i0+l+1) in ring slot (l+1) % W; positions >= n are unused (zero weight).
// FP64 spinor fields are three double2 planes of pv sites (kq_prec.cuh).
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
        for (int k = 0; k < kmax; ++k) {
            double2 *pp = reinterpret_cast<double2 *>(pw0 + k * vb) + off;
            double2 *xp = reinterpret_cast<double2 *>(x0 + k * vb) + off;
            const double2 p = *pp, x = *xp;
            double2 pn = make_double2(sc[k] * p.x, sc[k] * p.y);
            double2 xn = make_double2(x.x + se[k] * p.x, x.y + se[k] * p.y);
#pragma unroll
            for (int l = 0; l < kWin; ++l) {
                pn.x += sd[k][l] * rl[l].x;
                pn.y += sd[k][l] * rl[l].y;
                xn.x += sf[k][l] * rl[l].x;
                xn.y += sf[k][l] * rl[l].y;
            }
            *pp = pn;
            *xp = xn;
        }
    }
}

}  // namespace kq
