// Mixed-precision multishift solver (KQ_SOLVER_MIXED): every shift reaches an FP64 true relative residual target.
//
// Phase 1  relaxed-precision multishift CG (kq_msrelax.cu: the CGM recurrences of inverter_cgm.cpp:17-87 with FP64
//          vectors, the operator switched to FP32 and then HALF links as the residual falls below the points where
//          their accumulated error still fits under the target), stopped at a fraction of the target.
// Phase 2  an FP64 check of every shift's true residual; shifts above the target (rare: the operator-error
//          model missed) are refined together by a multi-RHS CG with reliable updates:
//          FP32 / HALF-link iterations in lockstep over the still-active systems, each dslash loading every link
//          once for R systems; when a system's iterated residual has fallen by `delta` since its last true residual
//          (or below the target), its FP32 correction is folded into the FP64 solution and its residual is
//          recomputed in FP64 (b - (sigma_k - D_pq D_qp) x_k).  A system stops when that FP64 residual meets the
//          target.  All bookkeeping (active / flagged lists, alpha, beta) lives on the device; the host replays a
//          CUDA graph of `chunk` iterations and polls one word.
//
// Per iteration: K1 tmp_k = D p_k;  K2 ap_k = sigma_k p_k - D tmp_k, <p_k, ap_k>;  K3 xs_k += a p_k, r_k -= a ap_k,
// |r_k|^2 and the reliable-update decision;  K4-K6 the FP64 update of flagged systems;  K7 p_k = r_k + b p_k and
// the compaction of the active list.
#include <cmath>
#include <cstdlib>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_msrelax.h"

namespace kq {

cudaError_t launch_dslash2(const Geom &g, const GaugeDev &gd, int lp, int sp, const void *src, void *dst,
                           int dst_parity, const int *gate, cudaStream_t s, int block);

struct MrState {
    int nact, nflag, iter, max_iter;  // polled by the host (first 16 bytes)
    int first, status, nupdates, ns;
    unsigned ticket[4];
    double target2, delta2, bnorm2, pad;
    int act[kMaxShift], flag[kMaxShift], conv[kMaxShift], sys_iter[kMaxShift];
    double sigma[kMaxShift], rr[kMaxShift], maxrr[kMaxShift], alpha[kMaxShift], beta[kMaxShift];
    double res[kMaxShift];    // true relative residual at the last FP64 update
    double res0[kMaxShift];   // true relative residual entering phase 2
};

struct MrBuffers {
    const void *b;      // FP64
    void *x64;          // FP64 solutions, vb64 apart
    void *r, *p, *xs, *ap, *tmp;  // FP32 sloppy vectors, vb32 apart
    void *tmp64;        // FP64, vb64 apart (other parity)
    size_t vb32, vb64;
    double *partials;   // ns * site_blocks
    MrState *st;
};

constexpr int kBS = 256;

template <int R>
__device__ __forceinline__ void group_systems(const int *list, int n, int grp, int sys[R])
{
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int idx = grp * R + r;
        sys[r] = idx < n ? list[idx] : -1;
    }
}

// true in every thread of the last block of the grid to finish (after all others published their partials)
__device__ __forceinline__ bool last_block(unsigned *ticket)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ double sum_partials(const double *p, int n, double *sm)
{
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += ((volatile const double *)p)[b];
    return block_sum(s, sm);
}

// ---------------------------------------------------------------------------------------------------- kernels
// K1: tmp_k = D p_k (output parity q) for the active systems
template <int LP, int R>
__global__ void __launch_bounds__(kBS) mr_dslash_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const char *p0,
                                                        char *tmp0, size_t vb, int q, const MrState *st)
{
    int sys[R];
    group_systems<R>(st->act, st->nact, blockIdx.x, sys);
    if (sys[0] < 0) return;
    const int i = blockIdx.y * kBS + threadIdx.x;
    if (i >= g.vh) return;
    float acc[R][6];
    dslash_site_mrhs<LP, 1, R>(g, pv, fat, lng, p0, vb, sys, q, i, acc);
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (sys[r] >= 0) st_spinor<1>(tmp0 + sys[r] * vb, pv, i, acc[r]);
}

// K2: ap_k = sigma_k p_k - D tmp_k ; pAp_k -> alpha_k = rr_k / pAp_k
template <int LP, int R>
__global__ void __launch_bounds__(kBS) mr_dslash2_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const char *tmp0,
                                                         const char *p0, char *ap0, size_t vb, int parity, MrState *st,
                                                         double *partials)
{
    __shared__ double sm[32];
    int sys[R];
    const int n = st->nact;
    group_systems<R>(st->act, n, blockIdx.x, sys);
    const int i = blockIdx.y * kBS + threadIdx.x;
    double dot[R];
#pragma unroll
    for (int r = 0; r < R; ++r) dot[r] = 0.0;
    if (sys[0] >= 0 && i < g.vh) {
        float acc[R][6];
        dslash_site_mrhs<LP, 1, R>(g, pv, fat, lng, tmp0, vb, sys, parity, i, acc);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                float pv6[6];
                ld_spinor<1>(p0 + sys[r] * vb, pv, i, pv6);
                const float sg = (float)st->sigma[sys[r]];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    acc[r][k] = sg * pv6[k] - acc[r][k];
                    dot[r] += (double)pv6[k] * (double)acc[r][k];
                }
                st_spinor<1>(ap0 + sys[r] * vb, pv, i, acc[r]);
            }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double s = block_sum(dot[r], sm);
        if (threadIdx.x == 0 && sys[r] >= 0) partials[sys[r] * gridDim.y + blockIdx.y] = s;
    }
    if (!last_block(&st->ticket[0])) return;
    for (int a = 0; a < n; ++a) {
        const int k = st->act[a];
        const double pAp = sum_partials(partials + k * gridDim.y, gridDim.y, sm);
        if (threadIdx.x == 0) st->alpha[k] = st->rr[k] / pAp;
    }
    if (threadIdx.x == 0) st->ticket[0] = 0;
}

// K3: xs_k += alpha_k p_k ; r_k -= alpha_k ap_k ; |r_k|^2 -> reliable-update decision or beta_k
template <int R>
__global__ void __launch_bounds__(kBS) mr_update_kernel(int vh, int pv, const char *p0, const char *ap0, char *r0,
                                                        char *xs0, size_t vb, MrState *st, double *partials)
{
    __shared__ double sm[32];
    int sys[R];
    const int n = st->nact;
    group_systems<R>(st->act, n, blockIdx.x, sys);
    const int i = blockIdx.y * kBS + threadIdx.x;
    double nn[R];
#pragma unroll
    for (int r = 0; r < R; ++r) nn[r] = 0.0;
    if (i < vh) {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                const int k = sys[r];
                const float a = (float)st->alpha[k];
                float pv6[6], av[6], rv[6], xv[6];
                ld_spinor<1>(p0 + k * vb, pv, i, pv6);
                ld_spinor<1>(ap0 + k * vb, pv, i, av);
                ld_spinor<1>(r0 + k * vb, pv, i, rv);
                ld_spinor<1>(xs0 + k * vb, pv, i, xv);
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    xv[e] += a * pv6[e];
                    rv[e] -= a * av[e];
                    nn[r] += (double)rv[e] * (double)rv[e];
                }
                st_spinor<1>(xs0 + k * vb, pv, i, xv);
                st_spinor<1>(r0 + k * vb, pv, i, rv);
            }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double s = block_sum(nn[r], sm);
        if (threadIdx.x == 0 && sys[r] >= 0) partials[sys[r] * gridDim.y + blockIdx.y] = s;
    }
    if (!last_block(&st->ticket[1])) return;
    __shared__ int nflag;
    if (threadIdx.x == 0) nflag = 0;
    __syncthreads();
    for (int a = 0; a < n; ++a) {
        const int k = st->act[a];
        const double rr = sum_partials(partials + k * gridDim.y, gridDim.y, sm);
        if (threadIdx.x == 0) {
            st->sys_iter[k] += 1;
            if (rr < st->target2 || rr < st->delta2 * st->maxrr[k] || !isfinite(rr)) {
                st->flag[nflag++] = k;   // fold into FP64 and recompute the true residual
            } else {
                st->beta[k] = rr / st->rr[k];
                st->rr[k] = rr;
            }
        }
    }
    if (threadIdx.x == 0) {
        st->nflag = nflag;
        st->ticket[1] = 0;
    }
}

// K4: x64_k += xs_k ; xs_k = 0  (flagged systems)
template <int R>
__global__ void __launch_bounds__(kBS) mr_accum_kernel(int vh, int pv, char *xs0, size_t vb, char *x640,
                                                       size_t vb64, const MrState *st)
{
    int sys[R];
    group_systems<R>(st->flag, st->nflag, blockIdx.x, sys);
    if (sys[0] < 0) return;
    const int i = blockIdx.y * kBS + threadIdx.x;
    if (i >= vh) return;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (sys[r] >= 0) {
            const int k = sys[r];
            float xv[6];
            double xd[6];
            ld_spinor<1>(xs0 + k * vb, pv, i, xv);
            ld_spinor<0>(x640 + k * vb64, pv, i, xd);
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                xd[e] += (double)xv[e];
                xv[e] = 0.f;
            }
            st_spinor<0>(x640 + k * vb64, pv, i, xd);
            st_spinor<1>(xs0 + k * vb, pv, i, xv);
        }
}

// K5: tmp64_k = D x64_k (FP64, flagged systems, output parity q)
template <int R>
__global__ void __launch_bounds__(kBS) mr_dslash64_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const char *x640,
                                                          char *t640, size_t vb64, int q, const MrState *st)
{
    int sys[R];
    group_systems<R>(st->flag, st->nflag, blockIdx.x, sys);
    if (sys[0] < 0) return;
    const int i = blockIdx.y * kBS + threadIdx.x;
    if (i >= g.vh) return;
    double acc[R][6];
    dslash_site_mrhs<0, 0, R>(g, pv, fat, lng, x640, vb64, sys, q, i, acc);
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (sys[r] >= 0) st_spinor<0>(t640 + sys[r] * vb64, pv, i, acc[r]);
}

// K6: r_k = b - (sigma_k x64_k - D tmp64_k) in FP64, stored FP32 ; |r_k|^2 -> convergence or beta_k (flagged)
template <int R>
__global__ void __launch_bounds__(kBS) mr_resid_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const char *t640,
                                                       const char *x640, size_t vb64, const void *b, char *r0,
                                                       size_t vb, int parity, MrState *st, double *partials)
{
    __shared__ double sm[32];
    const int n = st->nflag;
    if (n == 0) return;
    int sys[R];
    group_systems<R>(st->flag, n, blockIdx.x, sys);
    const int i = blockIdx.y * kBS + threadIdx.x;
    double nn[R];
#pragma unroll
    for (int r = 0; r < R; ++r) nn[r] = 0.0;
    if (sys[0] >= 0 && i < g.vh) {
        double acc[R][6], bv[6];
        dslash_site_mrhs<0, 0, R>(g, pv, fat, lng, t640, vb64, sys, parity, i, acc);
        ld_spinor<0>(b, pv, i, bv);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                const int k = sys[r];
                double xv[6];
                float rv[6];
                ld_spinor<0>(x640 + k * vb64, pv, i, xv);
                const double sg = st->sigma[k];
#pragma unroll
                for (int e = 0; e < 6; ++e) {
                    const double res = bv[e] - (sg * xv[e] - acc[r][e]);
                    nn[r] += res * res;
                    rv[e] = (float)res;
                }
                st_spinor<1>(r0 + k * vb, pv, i, rv);
            }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const double s = block_sum(nn[r], sm);
        if (threadIdx.x == 0 && sys[r] >= 0) partials[sys[r] * gridDim.y + blockIdx.y] = s;
    }
    if (!last_block(&st->ticket[2])) return;
    for (int a = 0; a < n; ++a) {
        const int k = st->flag[a];
        const double rr = sum_partials(partials + k * gridDim.y, gridDim.y, sm);
        if (threadIdx.x == 0) {
            const double rel = sqrt(rr / st->bnorm2);
            st->res[k] = rel;
            if (st->first) st->res0[k] = rel;
            if (!isfinite(rr)) {
                st->status = KQ_STATUS_BREAKDOWN;
                st->conv[k] = 1;
            } else if (rr < st->target2) {
                st->conv[k] = 1;
            } else {
                st->beta[k] = st->first ? 0.0 : rr / st->rr[k];
                st->rr[k] = rr;
                st->maxrr[k] = rr;
            }
            st->nupdates += 1;
        }
    }
    if (threadIdx.x == 0) st->ticket[2] = 0;
}

// K7: p_k = r_k + beta_k p_k for active, unconverged systems ; compaction of the active list
template <int R>
__global__ void __launch_bounds__(kBS) mr_p_kernel(int vh, int pv, const char *r0, char *p0, size_t vb, MrState *st)
{
    int sys[R];
    const int n = st->nact;
    group_systems<R>(st->act, n, blockIdx.x, sys);
    const int i = blockIdx.y * kBS + threadIdx.x;
    if (i < vh) {
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0 && !st->conv[sys[r]]) {
                const int k = sys[r];
                const float bt = (float)st->beta[k];
                float rv[6], pv6[6];
                ld_spinor<1>(r0 + k * vb, pv, i, rv);
                ld_spinor<1>(p0 + k * vb, pv, i, pv6);
#pragma unroll
                for (int e = 0; e < 6; ++e) pv6[e] = rv[e] + bt * pv6[e];
                st_spinor<1>(p0 + k * vb, pv, i, pv6);
            }
    }
    if (!last_block(&st->ticket[3])) return;
    if (threadIdx.x == 0) {
        int m = 0;
        for (int a = 0; a < n; ++a)
            if (!st->conv[st->act[a]]) st->act[m++] = st->act[a];
        if (!st->first) st->iter += 1;
        st->first = 0;
        st->nflag = 0;
        if (st->iter >= st->max_iter && m > 0) {
            st->status = KQ_STATUS_MAXITER;
            m = 0;
        }
        st->nact = m;
        st->ticket[3] = 0;
    }
}

// |v|^2 of an FP64 field (fixed-order partials, summed on the host)
__global__ void __launch_bounds__(kBS) norm2_partials_kernel(int vh, int pv, const void *v, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * kBS + threadIdx.x;
    double s = 0.0;
    if (i < vh) {
        double a[6];
        ld_spinor<0>(v, pv, i, a);
#pragma unroll
        for (int e = 0; e < 6; ++e) s += a[e] * a[e];
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------------------------------- driver
constexpr int kR = 4;    // systems per thread in the sloppy multi-RHS kernels
constexpr int kR64 = 2;  // systems per thread in the FP64 reliable-update kernels

template <int LP>
static void enqueue_reliable(const Geom &g, const GaugeDev &gd, const MrBuffers &w, int parity, int ns, cudaStream_t s)
{
    const int pv = pad_sites(g.vh), sb = (g.vh + kBS - 1) / kBS;
    const dim3 g64((ns + kR64 - 1) / kR64, sb), gs((ns + kR - 1) / kR, sb);
    mr_accum_kernel<kR><<<gs, kBS, 0, s>>>(g.vh, pv, (char *)w.xs, w.vb32, (char *)w.x64, w.vb64, w.st);
    mr_dslash64_kernel<kR64><<<g64, kBS, 0, s>>>(g, pv, gd.fat[0], gd.lng[0], (const char *)w.x64, (char *)w.tmp64,
                                                 w.vb64, 1 - parity, w.st);
    mr_resid_kernel<kR64><<<g64, kBS, 0, s>>>(g, pv, gd.fat[0], gd.lng[0], (const char *)w.tmp64,
                                              (const char *)w.x64, w.vb64, w.b, (char *)w.r, w.vb32, parity, w.st,
                                              w.partials);
    mr_p_kernel<kR><<<gs, kBS, 0, s>>>(g.vh, pv, (const char *)w.r, (char *)w.p, w.vb32, w.st);
}

template <int LP>
static void enqueue_mr_iteration(const Geom &g, const GaugeDev &gd, const MrBuffers &w, int parity, int ns,
                                 cudaStream_t s)
{
    const int pv = pad_sites(g.vh), sb = (g.vh + kBS - 1) / kBS;
    const dim3 gs((ns + kR - 1) / kR, sb);
    mr_dslash_kernel<LP, kR><<<gs, kBS, 0, s>>>(g, pv, gd.fat[LP], gd.lng[LP], (const char *)w.p, (char *)w.tmp,
                                                w.vb32, 1 - parity, w.st);
    mr_dslash2_kernel<LP, kR><<<gs, kBS, 0, s>>>(g, pv, gd.fat[LP], gd.lng[LP], (const char *)w.tmp,
                                                 (const char *)w.p, (char *)w.ap, w.vb32, parity, w.st, w.partials);
    mr_update_kernel<kR><<<gs, kBS, 0, s>>>(g.vh, pv, (const char *)w.p, (const char *)w.ap, (char *)w.r,
                                            (char *)w.xs, w.vb32, w.st, w.partials);
    enqueue_reliable<LP>(g, gd, w, parity, ns, s);
}

static double env_double(const char *name, double dflt)
{
    const char *v = getenv(name);
    return v ? atof(v) : dflt;
}

// run_phase1 = false: d_x already holds a multishift solution (the batched solver's); only the FP64 check and the
// refinement of shifts above the target run.
cudaError_t mixed_solve(::kq_context *ctx, const kq_solve_param *param, const double *sig, const void *d_b,
                        void *d_x, kq_solve_info *info, bool run_phase1)
{
    const Geom &g = ctx->g;
    cudaStream_t s = ctx->stream;
    const int ns = param->num_shift;
    const int lp = prec_from_api(param->prec);  // sloppy link precision
    if (lp != P32 && lp != P16) {
        set_last_error("mixed solver: sloppy precision must be SINGLE or HALF");
        return cudaErrorInvalidValue;
    }
    // rel_residual < 0: the absolute target |b - A_k x_k|^2 < tol (the reference's stopping threshold), turned into
    // a relative one once |b| is known
    double target = param->rel_residual > 0 ? param->rel_residual : 1e-10;
    // Effective error of the sloppy operators relative to |r| at the switch.  The HALF operator's residual gap grows
    // to ~1e-3 x the residual norm at which it starts (measured on the oracle).  For FP32 the schedule was swept on
    // B200 (32^4 and 48^3 x 96, 12 and 16 shifts, target 1e-10): 1e-5 -> 3e-7 cuts the solve time by 10-11 % with
    // 4 refinement iterations and the per-shift FP64 true residual still at target; below 1e-7 the sloppy phase
    // ends further above target and the refinement grows (28 iterations at 3e-8 on 48^3 x 96).
    const double eps32 = env_double("KUQCD_RELAX_EPS32", 3e-7);
    const double eps16 = env_double("KUQCD_RELAX_EPS16", 1e-3);
    const double relax_frac = env_double("KUQCD_RELAX_FRAC", 0.3);  // share of the target each precision may use
    const double stop_frac = env_double("KUQCD_RELAX_STOP", 0.7);   // recursive-residual stop, x target
    const double delta = env_double("KUQCD_MIXED_DELTA", 0.1);     // reliable-update trigger of the refinement
    const int need[3] = {P64, P32, lp};  // the relaxed schedule runs FP64, then FP32, then (HALF) links
    for (int p : need)
        if (!ctx->gd.have[p]) {
            if (kq_prepare_links(ctx, p == P64 ? KUQCD_DOUBLE : p == P32 ? KUQCD_SINGLE : KUQCD_HALF) != KUQCD_SUCCESS)
                return cudaErrorInvalidValue;
        }
    const size_t vb32 = spinor_bytes(g, P32), vb64 = spinor_bytes(g, P64);
    const int sb = (g.vh + kBS - 1) / kBS;
    // ---- workspace
    auto layout = [&](Carve &c, MsBuffers &cw, MrBuffers &mw) {
        ms_layout(c, g, ns, d_b, d_x, cw);
        mw.partials = static_cast<double *>(c.take(sizeof(double) * (size_t)sb * ns));
        mw.b = d_b;
        mw.x64 = d_x;
        mw.vb32 = vb32;
        mw.vb64 = vb64;
        // phase-2 vectors reuse nothing of phase 1 except the partials buffer
        mw.r = c.take(vb32 * ns);
        mw.p = c.take(vb32 * ns);
        mw.xs = c.take(vb32 * ns);
        mw.ap = c.take(vb32 * ns);
        mw.tmp = c.take(vb32 * ns);
        mw.tmp64 = c.take(vb64 * ns);
        mw.st = static_cast<MrState *>(c.take(sizeof(MrState)));
    };
    MsBuffers cw;
    MrBuffers mw;
    Carve probe(nullptr);
    layout(probe, cw, mw);
    KQ_CUDA_TRY(ensure_work(ctx, probe.off));
    Carve c(ctx->work);
    layout(c, cw, mw);
    long long launches = 0;

    // ---- |b|^2
    {
        const int pv = pad_sites(g.vh);
        norm2_partials_kernel<<<sb, kBS, 0, s>>>(g.vh, pv, d_b, mw.partials);
        std::vector<double> h(sb);
        KQ_CUDA_TRY(cudaMemcpyAsync(h.data(), mw.partials, sizeof(double) * sb, cudaMemcpyDeviceToHost, s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        launches += 1;
        double bb = 0;
        for (double v : h) bb += v;
        if (!std::isfinite(bb)) {
            set_last_error("mixed solver: the source is not finite");
            return cudaErrorInvalidValue;
        }
        if (bb == 0.0) {  // b = 0: every x_k = 0, exactly
            KQ_CUDA_TRY(cudaMemsetAsync(d_x, 0, vb64 * ns, s));
            KQ_CUDA_TRY(cudaStreamSynchronize(s));
            info->iter = 0;
            info->kernel_launches = launches;
            for (int k = 0; k < ns; ++k) info->true_residual[k] = 0.0;
            return cudaSuccess;
        }
        if (param->rel_residual < 0) {
            if (!(param->tol > 0)) {
                set_last_error("mixed solver: an absolute target (rel_residual < 0) needs tol > 0");
                return cudaErrorInvalidValue;
            }
            target = std::sqrt(param->tol / bb);
        }
        MrState hs;
        memset(&hs, 0, sizeof(hs));
        hs.bnorm2 = bb;
        hs.target2 = target * target * bb;
        hs.delta2 = delta * delta;
        hs.ns = ns;
        hs.max_iter = param->max_iter > 0 ? param->max_iter : 100000;
        hs.nact = ns;
        hs.nflag = ns;
        hs.first = 1;
        for (int k = 0; k < ns; ++k) {
            hs.act[k] = k;
            hs.flag[k] = k;
            hs.sigma[k] = sig[k];
            hs.rr[k] = 1.0;
        }
        KQ_CUDA_TRY(cudaMemcpyAsync(mw.st, &hs, sizeof(hs), cudaMemcpyHostToDevice, s));
        // phase 1: relaxed-precision multishift, stopped (reference rule) at a fraction of the target so that the
        // operator's accumulated error still fits under it
        double rs[kMaxShift];
        rs[0] = sig[0];
        for (int k = 1; k < ns; ++k) rs[k] = sig[k] - sig[0];
        const double rho32 = relax_frac * target / eps32;
        const double rho16 = lp == P16 ? relax_frac * target / eps16 : 0.0;
        if (run_phase1) {
            NvtxRange nvtx("mixed: relaxed-precision multishift");
            MsResult r1;
            KQ_CUDA_TRY(ms_solve(ctx, cw, param->parity, ns, rs, stop_frac * stop_frac * target * target * bb,
                                 param->max_iter > 0 ? param->max_iter : 100000, rho32, rho16, &r1));
            info->iter = r1.iter;
            launches += r1.launches;
        }
    }

    // ---- phase 2
    NvtxRange nvtx2("mixed: FP64 check and refinement");
    KQ_CUDA_TRY(cudaMemsetAsync(mw.xs, 0, vb32 * ns, s));
    KQ_CUDA_TRY(cudaMemsetAsync(mw.p, 0, vb32 * ns, s));
    // opening reliable update of every system: r_k = b - A_k x_k in FP64, p_k = r_k
    if (lp == P32) enqueue_reliable<1>(g, ctx->gd, mw, param->parity, ns, s);
    else enqueue_reliable<2>(g, ctx->gd, mw, param->parity, ns, s);
    KQ_CUDA_TRY(cudaGetLastError());
    launches += 4;

    const int chunk = 4;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    KQ_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int it = 0; it < chunk; ++it) {
        if (lp == P32) enqueue_mr_iteration<1>(g, ctx->gd, mw, param->parity, ns, s);
        else enqueue_mr_iteration<2>(g, ctx->gd, mw, param->parity, ns, s);
    }
    cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        set_last_error(std::string("mixed solver: graph capture failed: ") + cudaGetErrorString(ee));
        return ee;
    }
    ee = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    KQ_CUDA_TRY(ee);
    // the pinned poll page receives the first four ints of MrState: nact, nflag, iter, max_iter
    int *poll = reinterpret_cast<int *>(ctx->poll);
    cudaError_t err = cudaSuccess;
    int replays = 0;
    const int hs_max_iter = param->max_iter > 0 ? param->max_iter : 100000;
    for (;;) {
        KQ_CUDA_TRY(cudaMemcpyAsync(poll, mw.st, 4 * sizeof(int), cudaMemcpyDeviceToHost, s));
        err = cudaStreamSynchronize(s);
        if (err != cudaSuccess || poll[0] == 0) break;  // no active system left
        err = cudaGraphLaunch(exec, s);
        if (err != cudaSuccess) break;
        launches += 7LL * chunk;
        if (++replays > hs_max_iter / chunk + 8) break;  // the refinement stops by then while its state is consistent
    }
    cudaGraphExecDestroy(exec);
    KQ_CUDA_TRY(err);
    MrState hs;
    KQ_CUDA_TRY(cudaMemcpyAsync(&hs, mw.st, sizeof(hs), cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    info->iter_refine = hs.iter;
    info->status = hs.status;
    info->kernel_launches = launches;
    double worst0 = 0;
    for (int k = 0; k < ns; ++k) {
        info->true_residual[k] = hs.res[k];
        worst0 = std::max(worst0, hs.res0[k]);
    }
    info->sloppy_residual = worst0;
    // the refinement changed the solutions of the systems it iterated on
    if (ctx->solution_ready)
        for (int k = 0; k < ns; ++k)
            if (hs.sys_iter[k] > 0) ctx->solution_ready(ctx, k, ctx->solution_ready_user);
    return cudaSuccess;
}

}  // namespace kq
