// Multishift CG with windowed shift updates and a relaxed-precision operator.
//
// Recurrences and stopping rule are those of CGM::Invert (inverter_cgm.cpp:17-87).  Two changes of schedule:
//
// 1. Windowed shift updates.  The classic iteration reads and writes every shift's x_k and p_k every iteration
//    (Ymax + Axpby, inverter_cgm.cpp:61-69: 4 vectors per shift).  Here the base direction p_0 is updated every
//    iteration (the operator needs it), the residuals r^(i) go to a ring of W slots, and every W iterations one
//    kernel applies  p_k <- c_k p_k + sum_l d_kl r^(l),  x_k <- x_k + e_k p_k + sum_l f_kl r^(l)  for all shifts,
//    with coefficients accumulated by the scalar code from the same B_k, Z_k, a_k.  Per iteration the shift traffic
//    drops from 4N vectors to (4N + W)/W.
//
// 2. Relaxed operator precision (inexact Krylov).  The operator may be computed less accurately as the residual
//    shrinks: a matvec error eps*|A||p| made when |r| = rho |b| perturbs the final residual by about eps_eff * rho.
//    For multishift CG every shifted residual gap is a sum of the same matvec errors weighted by zeta_k <= 1, so it
//    is bounded by the base gap.  The host therefore switches the operator from FP64 to FP32 links (FP32 temporary)
//    at |r| < rho32 |b| and to HALF links (16-bit temporary) at |r| < rho16 |b|; all vectors and scalars stay FP64.
//    With rho = 0 the solver is the plain FP64 multishift CG with windowed updates.
//
// 3. Three kernels per iteration.  The operator is A = sigma0 - D_pq D_qp with D_pq = -D_qp^dag (the backward hops
//    apply the adjoints of the same stored links), so <p, A p> = sigma0 |p|^2 + |D_qp p|^2: the beta step can run
//    at the end of the first dslash, and the second dslash applies r <- r + B0 s directly, never storing s
//    (inverter_cgm.cpp:45-50 forms s, then <p, s>, then r).  In FP64 the two forms of <p, A p> agree to rounding;
//    with a 16-bit temporary the step length uses |D p|^2 before the temporary is rounded (relative 3e-5), while
//    the residual update uses the operator actually applied, so the recurrence stays exact.
//
// Kernels per iteration: K1 tmp = D p0, |tmp|^2 (beta step + x coefficients);  K2 r <- r + B0 (sigma0 p0 - D tmp)
// into the ring, |r|^2 (alpha step + p coefficients + shift dropping + |p0|^2 = |r|^2 + a0^2 |p0|^2, r being
// orthogonal to the old p0);  K3 p0 <- r + a0 p0.
// One CUDA graph per operator precision, kChunk iterations each followed by K4, the windowed shift update, which
// applies the window once it is full (W = 2 kChunk iterations) or the solve has stopped, and otherwise returns at
// once.  The window sets the shift-update traffic, the chunk the granularity of the precision switches.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_ms_device.cuh"
#include "kq_msrelax.h"

namespace kq {

constexpr int kBSm = 256;

// ---------------------------------------------------------------------------------------------------- kernels
__global__ void __launch_bounds__(kBSm) ms_init_kernel(int vh, int pv, const void *__restrict__ b, char *x0,
                                                       char *pw0, size_t vb, void *p0, char *ring, int ns,
                                                       MsState *st, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * kBSm + threadIdx.x;
    double nn = 0.0;
    if (i < vh) {
        double v[6], z[6] = {0, 0, 0, 0, 0, 0};
        ld_spinor<0>(b, pv, i, v);
        st_spinor<0>(p0, pv, i, v);
        st_spinor<0>(ring, pv, i, v);  // r^(0) in slot 0
        for (int l = 1; l < kWin; ++l) st_spinor<0>(ring + l * vb, pv, i, z);
        for (int k = 0; k < ns; ++k) {
            st_spinor<0>(pw0 + k * vb, pv, i, v);
            st_spinor<0>(x0 + k * vb, pv, i, z);
        }
#pragma unroll
        for (int e = 0; e < 6; ++e) nn += v[e] * v[e];
    }
    double tot;
    if (grid_sum_last(nn, partials, &st->ticket[0], sm, &tot)) {
        st->rNorm2 = tot;
        st->bnorm2 = tot;
        st->pp = tot;  // p0 = b
        st->Bm1 = 1.0;
        for (int k = 0; k < st->ns; ++k) {
            st->a[k] = 0.0;
            st->B[k] = 1.0;
            st->Z[k] = 1.0;
            st->Zm1[k] = 1.0;
        }
        st->maxTerm = st->ns;
        st->wmax = st->ns;
        st->iter = 0;
        st->wpos = 0;
        st->nupd = 0;
        st->halt = 0;
        // b = 0: x = 0 is the solution; a non-finite source is a breakdown
        const bool finite = isfinite(tot);
        st->status = finite ? 0 : KQ_STATUS_BREAKDOWN;
        st->active = (finite && tot > 0.0) ? 1 : 0;
    }
}

// K1: tmp = D p0 (p0 FP64; links LP; tmp stored in SO); |tmp|^2, then the beta step with
// <p0, A p0> = sigma0 |p0|^2 + |tmp|^2 (|p0|^2 from the alpha step's recurrence)
template <int LP, int SO>
__global__ void __launch_bounds__(kBSm) ms_dslash1_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const void *__restrict__ p0, void *__restrict__ tmp, int q,
                                                          MsState *st, double *partials)
{
    if (st->active == 0) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * kBSm + threadIdx.x;
    double tt = 0.0;
    if (i < g.vh) {
        typedef typename Acc2<LP, LP>::T T;
        T acc[6];
        dslash_site_t<LP, 0, T>(g, pv, fat, lng, p0, q, i, acc);
        st_spinor_as<SO>(tmp, pv, i, acc);
#pragma unroll
        for (int k = 0; k < 6; ++k) tt += (double)acc[k] * (double)acc[k];
    }
    double tot;
    if (grid_sum_last_warp(tt, partials, &st->ticket[1], sm, &tot)) ms_step_beta(st, st->shift[0] * st->pp + tot);
}

// K2: s = sigma0 p0 - D tmp (tmp stored in SI, links LP; s stays in registers); r^(i+1) = r^(i) + B0 s into the
// ring; |r|^2, then the alpha step
template <int LP, int SI>
__global__ void __launch_bounds__(kBSm) ms_dslash2_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const void *__restrict__ tmp, const void *__restrict__ p0,
                                                          char *ring, size_t vb, int p, MsState *st,
                                                          double *partials)
{
    if (st->active == 0) return;
    __shared__ double sm[32];
    const int it = st->iter;  // iterations completed before this one
    const char *rin = ring + (size_t)(it % kWin) * vb;
    char *rout = ring + (size_t)((it + 1) % kWin) * vb;
    const int i = blockIdx.x * kBSm + threadIdx.x;
    double nn = 0.0;
    if (i < g.vh) {
        typedef typename Acc2<LP, LP>::T T;
        T acc[6];
        dslash_site_t<LP, SI, T>(g, pv, fat, lng, tmp, p, i, acc);
        double pv6[6], rv[6];
        ld_spinor<0>(p0, pv, i, pv6);
        ld_spinor<0>(rin, pv, i, rv);
        const double sig = st->shift[0], b0 = st->B[0];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            rv[k] += b0 * (sig * pv6[k] - (double)acc[k]);
            nn += rv[k] * rv[k];
        }
        st_spinor<0>(rout, pv, i, rv);
    }
    double tot;
    if (grid_sum_last_warp(nn, partials, &st->ticket[2], sm, &tot)) ms_step_alpha(st, tot);
}

// K3: p0 = r^(i) + a0 p0
__global__ void __launch_bounds__(kBSm) ms_p0_kernel(int vh, int pv, const char *ring, size_t vb, void *p0,
                                                     const MsState *st)
{
    if (st->active == 0) return;
    const int i = blockIdx.x * kBSm + threadIdx.x;
    if (i >= vh) return;
    const char *r = ring + (size_t)(st->iter % kWin) * vb;
    double rv[6], pv6[6];
    ld_spinor<0>(r, pv, i, rv);
    ld_spinor<0>(p0, pv, i, pv6);
    const double a0 = st->a[0];
#pragma unroll
    for (int k = 0; k < 6; ++k) pv6[k] = rv[k] + a0 * pv6[k];
    st_spinor<0>(p0, pv, i, pv6);
}

// K4: windowed shift update p_k <- c_k p_k + sum_l d_kl r_l ; x_k <- x_k + e_k p_k + sum_l f_kl r_l
template <int KU>
__global__ void __launch_bounds__(kBSm, 2) ms_window_kernel(int vh, int pv, const char *ring, size_t vb, char *pw0,
                                                         char *x0, MsState *st)
{
    __shared__ double sc[kMaxShift], se[kMaxShift], sd[kMaxShift][kWin], sf[kMaxShift][kWin];
    __shared__ int nw, km, act;
    if (threadIdx.x == 0) {
        nw = st->wpos;
        km = st->wmax;
        act = st->active;
    }
    __syncthreads();
    const int n = nw, kmax = km;
    // every block reads the same wpos / active (the reset below comes after all blocks have arrived)
    if (n == 0 || (n < kWin && act)) return;  // window not full and the solve still iterating
    for (int t = threadIdx.x; t < kmax; t += kBSm) {
        sc[t] = st->c[t];
        se[t] = st->e[t];
        for (int l = 0; l < kWin; ++l) {
            sd[t][l] = st->d[t][l];
            sf[t][l] = st->f[t][l];
        }
    }
    __syncthreads();
    const int i = blockIdx.x * kBSm + threadIdx.x;
    if (i < vh) window_update_site<KU>(ring, vb, pv, i, n, kmax, sc, se, sd, sf, pw0, x0);
    // last block resets the window
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&st->ticket[0], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        st->wpos = 0;
        st->ticket[0] = 0;
    }
}

// shifts updated per step of the window kernel's loop (KUQCD_WINDOW_UNROLL = 1 | 2 | 4)
static int window_unroll()
{
    static const int k = [] {
        const char *e = getenv("KUQCD_WINDOW_UNROLL");
        const int v = e ? atoi(e) : 4;
        return v == 1 || v == 2 ? v : 4;
    }();
    return k;
}

// ---------------------------------------------------------------------------------------------------- driver
template <int LP, int SO>
static void enqueue_ms_chunk(const Geom &g, const GaugeDev &gd, const MsBuffers &w, int parity, cudaStream_t s)
{
    const int pv = pad_sites(g.vh), nb = (g.vh + kBSm - 1) / kBSm;
    for (int it = 0; it < kChunk; ++it) {
        ms_dslash1_kernel<LP, SO><<<nb, kBSm, 0, s>>>(g, pv, gd.fat[LP], gd.lng[LP], w.p0, w.tmp, 1 - parity, w.st,
                                                      w.partials);
        ms_dslash2_kernel<LP, SO><<<nb, kBSm, 0, s>>>(g, pv, gd.fat[LP], gd.lng[LP], w.tmp, w.p0, (char *)w.ring,
                                                      w.vb, parity, w.st, w.partials);
        ms_p0_kernel<<<nb, kBSm, 0, s>>>(g.vh, pv, (const char *)w.ring, w.vb, w.p0, w.st);
    }
    switch (window_unroll()) {
        case 1: ms_window_kernel<1><<<nb, kBSm, 0, s>>>(g.vh, pv, (const char *)w.ring, w.vb, (char *)w.pw, (char *)w.x, w.st); break;
        case 2: ms_window_kernel<2><<<nb, kBSm, 0, s>>>(g.vh, pv, (const char *)w.ring, w.vb, (char *)w.pw, (char *)w.x, w.st); break;
        default: ms_window_kernel<4><<<nb, kBSm, 0, s>>>(g.vh, pv, (const char *)w.ring, w.vb, (char *)w.pw, (char *)w.x, w.st); break;
    }
}

size_t ms_workspace_bytes(const Geom &g, int ns)
{
    MsBuffers w;
    Carve c(nullptr);
    ms_layout(c, g, ns, nullptr, nullptr, w);
    return c.off;
}

void ms_layout(Carve &c, const Geom &g, int ns, const void *d_b, void *d_x, MsBuffers &w)
{
    const size_t vb = spinor_bytes(g, P64);
    const int nb = (g.vh + kBSm - 1) / kBSm;
    w.vb = vb;
    w.b = d_b;
    w.x = d_x;
    w.p0 = c.take(vb);
    w.tmp = c.take(vb);  // big enough for any temporary precision
    w.ring = c.take(vb * kWin);
    w.pw = c.take(vb * ns);
    w.partials = static_cast<double *>(c.take(sizeof(double) * nb));
    w.st = static_cast<MsState *>(c.take(sizeof(MsState)));
}

cudaError_t ms_solve(::kq_context *ctx, const MsBuffers &w, int parity, int ns, const double *shifts_ref, double tol,
                     int max_iter, double rho32, double rho16, MsResult *res)
{
    const Geom &g = ctx->g;
    cudaStream_t s = ctx->stream;
    if (ns < 1 || ns > kMaxShift) {
        set_last_error("multishift: num_shift out of range (1..64)");
        return cudaErrorInvalidValue;
    }
    const bool use32 = rho32 > 0.0, use16 = rho16 > 0.0;
    if (!ctx->gd.have[P64] || (use32 && !ctx->gd.have[P32]) || (use16 && !ctx->gd.have[P16])) {
        set_last_error("multishift: links not resident in a precision the schedule needs");
        return cudaErrorInvalidValue;
    }
    MsState h;
    memset(&h, 0, sizeof(h));
    h.ns = ns;
    h.max_iter = max_iter;
    h.tol = tol;
    for (int k = 0; k < ns; ++k) h.shift[k] = shifts_ref[k];
    KQ_CUDA_TRY(cudaMemcpyAsync(w.st, &h, sizeof(MsState), cudaMemcpyHostToDevice, s));
    const int pv = pad_sites(g.vh), nb = (g.vh + kBSm - 1) / kBSm;
    ms_init_kernel<<<nb, kBSm, 0, s>>>(g.vh, pv, w.b, (char *)w.x, (char *)w.pw, w.vb, w.p0, (char *)w.ring, ns, w.st,
                                       w.partials);
    KQ_CUDA_TRY(cudaGetLastError());
    long long launches = 1;

    // one graph per operator precision, each W iterations + the window update
    cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
    for (int m = 0; m < 3; ++m) {
        if ((m == 1 && !use32) || (m == 2 && !use16)) continue;
        cudaGraph_t graph = nullptr;
        KQ_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (m == 0) enqueue_ms_chunk<0, 0>(g, ctx->gd, w, parity, s);
        else if (m == 1) enqueue_ms_chunk<1, 1>(g, ctx->gd, w, parity, s);
        else enqueue_ms_chunk<2, 2>(g, ctx->gd, w, parity, s);
        cudaError_t ee = cudaStreamEndCapture(s, &graph);
        if (ee == cudaSuccess) ee = cudaGraphInstantiate(&exec[m], graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (ee != cudaSuccess) {
            for (auto &x : exec)
                if (x) cudaGraphExecDestroy(x);
            set_last_error(std::string("multishift: graph build failed: ") + cudaGetErrorString(ee));
            return ee;
        }
    }
    MsPoll *poll = reinterpret_cast<MsPoll *>(ctx->poll);
    cudaError_t err = cudaSuccess;
    int chunks[3] = {0, 0, 0};
    // Shifts k >= final_from have been reported final.  A shift dropped from the iteration (k >= maxTerm) receives
    // its last update in the next window flush; once the window is flushed (wpos = 0), x_k no longer changes.
    int final_from = ns;
    auto report = [&](int mt) {
        if (ctx->solution_ready)
            for (int k = final_from - 1; k >= mt; --k) ctx->solution_ready(ctx, k, ctx->solution_ready_user);
        final_from = std::min(final_from, mt);
    };
    for (;;) {
        err = cudaMemcpyAsync(poll, w.st, sizeof(MsPoll), cudaMemcpyDeviceToHost, s);
        if (err == cudaSuccess) err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) break;
        if (!poll->active) {
            if (poll->wpos == 0) report(0);  // stopped, last window flushed: every x_k is final
            break;
        }
        const int mt = poll->maxTerm, flushed = poll->wpos == 0;
        const double rel2 = poll->rNorm2 / poll->bnorm2;
        int m = 0;
        if (use16 && rel2 < rho16 * rho16) m = 2;
        else if (use32 && rel2 < rho32 * rho32) m = 1;
        err = cudaGraphLaunch(exec[m], s);
        if (err != cudaSuccess) break;
        if (flushed) report(mt);  // the work it enqueues runs behind this chunk
        chunks[m] += 1;
        launches += 3 * kChunk + 1;
        if (chunks[0] + chunks[1] + chunks[2] > max_iter / kChunk + 2) break;
    }
    for (auto &x : exec)
        if (x) cudaGraphExecDestroy(x);
    KQ_CUDA_TRY(err);
    KQ_CUDA_TRY(cudaMemcpyAsync(&h, w.st, sizeof(MsState), cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    res->iter = h.iter;
    res->status = h.status ? h.status : (h.iter >= max_iter && h.maxTerm > 0 ? KQ_STATUS_MAXITER : 0);
    res->launches = launches;
    for (int m = 0; m < 3; ++m) res->chunks[m] = chunks[m];
    return cudaSuccess;
}

}  // namespace kq
