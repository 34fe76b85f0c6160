// Multishift CG (CGM) on the device with the reference's recurrences and stopping rule
// (inverter_cgm.cpp:17-87):
//   x_0 solves (shifts[0] - D_pq D_qp) x = b,  x_j (j >= 1) solves (shifts[0] + shifts[j] - D_pq D_qp) x = b;
//   shift k stops when Z_k^2 |r|^2 < tol, dropped from the end of the list; iteration ends when no shift is left or
//   iter reaches max_iter.
//
// One iteration is four kernels, all device-resident (no host round trip):
//   K1  tmp = D_qp p0                                             (dslash, gated on state->active)
//   K2  s = shifts[0] p0 - D_pq tmp;  pAp = Re<p0, s>             (fused dslash + Axmy + RealDot, dirac_hisq.cpp:
//       last block: B0 = -|r|^2/pAp and the zeta/beta recurrences     457-462, inverter_cgm.cpp:45-56)
//   K3  r += B0 s;  |r|^2                                          (Axpy + Norm2, inverter_cgm.cpp:50,58)
//       last block: a_j, shift dropping, iteration count          (inverter_cgm.cpp:59-77)
//   K4  for every shift still updated: x_i -= B_i p_i; p_i = Z_i r + a_i p_i   (Ymax + Axpby, :61-69, one pass)
// Scalars live in FP64 in a device state block; reductions are deterministic (fixed-order block partials summed by
// the last block).  The host only polls the state every `chunk` iterations.
#include <vector>

#include "kq_dslash_core.cuh"
#include "kq_solver.h"

namespace kq {

cudaError_t launch_dslash_gated(const Geom &g, const GaugeDev &gd, int lp, int sp, const void *src, void *dst,
                                int dst_parity, const int *gate, cudaStream_t s);

// ------------------------------------------------------------------------------------------------ scalar steps
// Run by the 32 lanes of one warp (of the last block of the reduction), lane l owning shifts l and l + 32: shared
// scalars are read by every lane before any lane writes, per-shift values only by their owner, so the result is
// that of the reference's sequential loops (inverter_cgm.cpp:48-57, 58-60, 64-77) with the loads overlapped.
__device__ void cgm_step_beta(CgmState *st, double pAp)
{
    const int lane = threadIdx.x & 31;
    const double rNorm2 = st->rNorm2, Bm1 = st->Bm1, a0 = st->a[0];
    const int mt = st->maxTerm;
    const double B0 = -rNorm2 / pAp;
    const bool bad = !(pAp != 0.0) || !isfinite(B0);  // breakdown: zero or non-finite p.Ap
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
    for (int j = 1 + lane; j < mt; j += 32) {
        const double zm1 = st->Zm1[j], z = st->Z[j], sh = st->shift[j];
        const double rr1 = Bm1 * zm1 / (B0 * a0 * (zm1 - z) + zm1 * Bm1 * (1.0 - sh * B0));
        st->Zm1[j] = z;
        st->Z[j] = z * rr1;
        st->B[j] = B0 * rr1;
    }
    __syncwarp();
    if (lane == 0) {
        st->pAp = pAp;
        st->B[0] = B0;
        st->Bm1 = B0;
    }
}

__device__ void cgm_step_alpha(CgmState *st, double lambda2)
{
    const int lane = threadIdx.x & 31;
    const double rNorm2 = st->rNorm2, B0 = st->B[0], tol = st->tol;
    const int mt0 = st->maxTerm, halt0 = st->halt;
    const double a0 = lambda2 / rNorm2;
    __syncwarp();
    int mt = 0;
#pragma unroll
    for (int base = 0; base < kMaxShift; base += 32) {
        const int k = base + lane;
        bool keep = false;
        if (k < mt0) {
            const double z = st->Z[k];
            if (k > 0) st->a[k] = a0 * z * st->B[k] / (st->Zm1[k] * B0);
            keep = !(z * z * lambda2 < tol);  // converged shifts drop from the top
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (m) mt = base + 32 - __clz((int)m);
    }
    __syncwarp();
    if (lane == 0) {
        st->lambda2 = lambda2;
        st->a[0] = a0;
        st->rNorm2 = lambda2;
        st->nupd = mt0;
        st->maxTerm = mt;
        st->iter += 1;
        const bool finite = isfinite(lambda2);
        if (!finite) {
            st->status = KQ_STATUS_BREAKDOWN;
            st->halt = 1;
        }
        st->active = (mt > 0 && st->iter < st->max_iter && !halt0 && finite) ? 1 : 0;
    }
}

// ------------------------------------------------------------------------------------------------ kernels
template <int P>
__global__ void __launch_bounds__(256) cgm_init_kernel(int vh, int pv, const void *__restrict__ b, void *r, void *p,
                                                       size_t pstride, void *x, size_t xstride, int ns, CgmState *st,
                                                       double *partials)
{
    using T = typename Acc<P>::T;
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < vh) {
        T v[6], z[6] = {0, 0, 0, 0, 0, 0};
        ld_spinor<P>(b, pv, i, v);
        st_spinor<P>(r, pv, i, v);
        for (int k = 0; k < ns; ++k) {
            st_spinor<P>(static_cast<char *>(p) + k * pstride, pv, i, v);
            st_spinor<P>(static_cast<char *>(x) + k * xstride, pv, i, z);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) nn += (double)v[k] * (double)v[k];
    }
    double tot;
    if (grid_sum_last(nn, partials, &st->ticket, sm, &tot)) {
        st->rNorm2 = tot;
        st->Bm1 = 1.0;
        for (int k = 0; k < st->ns; ++k) {
            st->a[k] = 0.0;
            st->B[k] = 1.0;
            st->Z[k] = 1.0;
            st->Zm1[k] = 1.0;
        }
        st->maxTerm = st->ns;
        st->iter = 0;
        st->nupd = 0;
        st->halt = 0;
        // b = 0: x = 0 is the solution (no iteration; the reference would divide 0 by p.Ap = 0);
        // a non-finite source is a breakdown
        const bool finite = isfinite(tot);
        st->status = finite ? 0 : KQ_STATUS_BREAKDOWN;
        st->active = (finite && tot > 0.0) ? 1 : 0;
    }
}

// s = shifts[0] * p0 - D tmp ; pAp = Re<p0, s>   (links LP, vectors P)
template <int LP, int P>
__global__ void __launch_bounds__(256) cgm_dslash2_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const void *__restrict__ tmp, const void *__restrict__ p0,
                                                          void *__restrict__ s, int p, CgmState *st, double *partials)
{
    using T = typename Acc<P>::T;
    if (st->active == 0) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double dot = 0.0;
    if (i < g.vh) {
        T acc[6], pv6[6];
        dslash_site2<LP, P>(g, pv, fat, lng, tmp, p, i, acc);
        ld_spinor<P>(p0, pv, i, pv6);
        const T sig = (T)st->shift[0];
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] = sig * pv6[k] - acc[k];
        st_spinor<P>(s, pv, i, acc);
        // re-read what was stored so the reduction sees the stored precision
#pragma unroll
        for (int k = 0; k < 6; ++k) dot += (double)pv6[k] * (double)acc[k];
    }
    double tot;
    if (grid_sum_last_warp(dot, partials, &st->ticket, sm, &tot)) cgm_step_beta(st, tot);
}

// r += B0 s ; |r|^2
template <int P>
__global__ void __launch_bounds__(256) cgm_r_kernel(int vh, int pv, void *__restrict__ r, const void *__restrict__ s,
                                                    CgmState *st, double *partials)
{
    using T = typename Acc<P>::T;
    if (st->active == 0) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < vh) {
        T rv[6], sv[6];
        ld_spinor<P>(r, pv, i, rv);
        ld_spinor<P>(s, pv, i, sv);
        const T b0 = (T)st->B[0];
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            rv[k] += b0 * sv[k];
            nn += (double)rv[k] * (double)rv[k];
        }
        st_spinor<P>(r, pv, i, rv);
    }
    double tot;
    if (grid_sum_last_warp(nn, partials, &st->ticket, sm, &tot)) cgm_step_alpha(st, tot);
}

// x_k -= B_k p_k ; p_k = Z_k r + a_k p_k   for k < nupd
template <int P, int XP>
__global__ void __launch_bounds__(256) cgm_xp_kernel(int vh, int pv, const void *__restrict__ r, void *p,
                                                     size_t pstride, void *x, size_t xstride, CgmState *st)
{
    using T = typename Acc<P>::T;
    using TX = typename Acc<XP>::T;
    const int n = st->nupd;
    if (n == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < vh) {
        T rv[6];
        ld_spinor<P>(r, pv, i, rv);
        for (int k = 0; k < n; ++k) {
            void *pk = static_cast<char *>(p) + k * pstride;
            void *xk = static_cast<char *>(x) + k * xstride;
            T pv6[6];
            TX xv[6];
            ld_spinor<P>(pk, pv, i, pv6);
            ld_spinor<XP>(xk, pv, i, xv);
            const T Bk = (T)st->B[k], Zk = (T)st->Z[k], ak = (T)st->a[k];
#pragma unroll
            for (int e = 0; e < 6; ++e) {
                xv[e] -= (TX)(Bk * pv6[e]);
                pv6[e] = Zk * rv[e] + ak * pv6[e];
            }
            st_spinor<XP>(xk, pv, i, xv);
            st_spinor<P>(pk, pv, i, pv6);
        }
    }
    // last block clears nupd so that gated-off iterations do no updates
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&st->ticket_upd, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        st->nupd = 0;
        st->ticket_upd = 0;
    }
}

// ------------------------------------------------------------------------------------------------ driver
template <int LP, int P>
static cudaError_t enqueue_iteration(const Geom &g, const GaugeDev &gd, const CgmBuffers &w, int parity,
                                     CgmState *st, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int bs = 256, nb = (g.vh + bs - 1) / bs;
    KQ_CUDA_TRY(launch_dslash_gated(g, gd, LP, P, w.p, w.tmp, 1 - parity, &st->active, s));
    cgm_dslash2_kernel<LP, P><<<nb, bs, 0, s>>>(g, pv, gd.fat[LP], gd.lng[LP], w.tmp, w.p, w.s, parity, st,
                                                w.partials);
    cgm_r_kernel<P><<<nb, bs, 0, s>>>(g.vh, pv, w.r, w.s, st, w.partials);
    cgm_xp_kernel<P, P><<<nb, bs, 0, s>>>(g.vh, pv, w.r, w.p, w.vec_bytes, w.x, w.vec_bytes, st);
    return cudaGetLastError();
}

cudaError_t cgm_solve(const Geom &g, const GaugeDev &gd, int lp, int prec, const CgmBuffers &w, int parity, int ns,
                      const double *shifts, double tol, int max_iter, int chunk, CgmResult *res, cudaStream_t s)
{
    if (!((lp == prec) || (lp == P16 && prec == P32)) || !gd.have[lp]) {
        set_last_error("cgm: unsupported link/vector precision pair or links not resident");
        return cudaErrorInvalidValue;
    }
    if (ns < 1 || ns > kMaxShift) {
        set_last_error("cgm: num_shift out of range (1..64)");
        return cudaErrorInvalidValue;
    }
    if (prec != P64 && prec != P32) {
        set_last_error("cgm: plain multishift CG runs in FP64 or FP32");
        return cudaErrorInvalidValue;
    }
    CgmState h;
    memset(&h, 0, sizeof(h));
    h.ns = ns;
    h.max_iter = max_iter;
    h.tol = tol;
    for (int k = 0; k < ns; ++k) h.shift[k] = shifts[k];
    KQ_CUDA_TRY(cudaMemcpyAsync(w.state, &h, sizeof(CgmState), cudaMemcpyHostToDevice, s));
    const int pv = pad_sites(g.vh);
    const int bs = 256, nb = (g.vh + bs - 1) / bs;
    if (prec == P64)
        cgm_init_kernel<0><<<nb, bs, 0, s>>>(g.vh, pv, w.b, w.r, w.p, w.vec_bytes, w.x, w.vec_bytes, ns, w.state,
                                             w.partials);
    else
        cgm_init_kernel<1><<<nb, bs, 0, s>>>(g.vh, pv, w.b, w.r, w.p, w.vec_bytes, w.x, w.vec_bytes, ns, w.state,
                                             w.partials);
    KQ_CUDA_TRY(cudaGetLastError());
    if (chunk < 1) chunk = 8;

    // one chunk of iterations captured once as a CUDA graph, replayed until the state says stop
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cs = s;
    KQ_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaSuccess;
    for (int c = 0; c < chunk && ce == cudaSuccess; ++c)
        ce = prec == P64  ? enqueue_iteration<0, 0>(g, gd, w, parity, w.state, cs)
             : lp == P32 ? enqueue_iteration<1, 1>(g, gd, w, parity, w.state, cs)
                         : enqueue_iteration<2, 1>(g, gd, w, parity, w.state, cs);
    cudaError_t ee = cudaStreamEndCapture(cs, &graph);
    if (ce != cudaSuccess || ee != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        set_last_error(std::string("cgm: graph capture failed: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        return ce != cudaSuccess ? ce : ee;
    }
    ee = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    KQ_CUDA_TRY(ee);

    CgmPoll *poll = w.poll;  // pinned host mirror
    int launched = 0;
    cudaError_t err = cudaSuccess;
    for (;;) {
        err = cudaGraphLaunch(exec, s);
        if (err != cudaSuccess) break;
        launched += chunk;
        err = cudaMemcpyAsync(poll, &w.state->iter, sizeof(CgmPoll), cudaMemcpyDeviceToHost, s);
        if (err != cudaSuccess) break;
        err = cudaStreamSynchronize(s);
        if (err != cudaSuccess) break;
        if (!poll->active) break;
        if (launched > max_iter + chunk) break;  // cannot happen while the state is consistent
    }
    cudaGraphExecDestroy(exec);
    KQ_CUDA_TRY(err);
    KQ_CUDA_TRY(cudaMemcpyAsync(&h, w.state, sizeof(CgmState), cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    res->launches = 1 + 4LL * launched;
    res->iter = h.iter;
    res->status = h.status;
    res->rnorm2 = h.rNorm2;
    for (int k = 0; k < ns; ++k) res->zeta[k] = h.Z[k];
    return cudaSuccess;
}

}  // namespace kq
