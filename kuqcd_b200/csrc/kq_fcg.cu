// Per-shift flexible CG polish (FCG with one A-orthogonalisation, Notay's truncated FCG(1)) preconditioned by the
// learned network: after a loose multishift pass, every shift's FP64 solution is driven to the true-residual
// target with the FP64 operator (sigma_k + D^dag D).  Without a network, or when the preconditioned iteration
// breaks down, stagnates or exhausts its budget, the same loop continues unpreconditioned (plain CG from the
// current x), and every shift ends with an FP64 true-residual check.  No reference counterpart.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"

struct kq_net;
int net_apply_launches(const kq_net *n);

namespace kq {

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s);
cudaError_t ptc_check_fault(cudaStream_t s);

// Device state of one shift's polish.  The scalar steps run in the last block of each reducing kernel, so the
// host only looks at the state once per chunk of iterations.
struct FcgState {
    double bb, target2, rr, rr_check, pw, alpha, beta;
    int it, max_iter, active, leave, use_net, total, net_it;
    unsigned ticket;
};

constexpr int kFcgBS = 256;
constexpr int kStall = 200;  // the network phase must halve |r|^2 every kStall iterations

// fixed-order grid reduction of up to two doubles per block: true in thread 0 of the last block to arrive, with the
// totals in out[0..n)
template <int N>
__device__ __forceinline__ bool fcg_grid_sum(const double (&v)[N], double *partials, unsigned *ticket, double *sm,
                                             double (&out)[N])
{
    __shared__ bool last;
    double b[N];
#pragma unroll
    for (int j = 0; j < N; ++j) b[j] = block_sum(v[j], sm);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < N; ++j) partials[j * gridDim.x + blockIdx.x] = b[j];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
#pragma unroll
    for (int j = 0; j < N; ++j) {
        double s = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) s += ((volatile double *)partials)[j * gridDim.x + k];
        out[j] = block_sum(s, sm);
    }
    if (threadIdx.x == 0) *ticket = 0u;
    return threadIdx.x == 0;
}

// |b|^2 and the state of a new shift
__global__ void __launch_bounds__(kFcgBS) fcg_init_kernel(int vh, int pv, const void *b, FcgState *st,
                                                          double *partials, double target, int max_iter, int use_net)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    double v[1] = {0.0};
    if (i < vh) {
        double bv[6];
        ld_spinor<0>(b, pv, i, bv);
#pragma unroll
        for (int e = 0; e < 6; ++e) v[0] += bv[e] * bv[e];
    }
    double tot[1];
    if (fcg_grid_sum<1>(v, partials, &st->ticket, sm, tot)) {
        st->bb = tot[0];
        st->target2 = target * target * tot[0];
        st->max_iter = max_iter;
        st->use_net = use_net;
        st->it = st->total = st->net_it = 0;
        st->leave = 0;
        st->active = 0;
    }
}

// r = b - s and |r|^2; (re)starts a phase: active while |r| is above target and the budget lasts
__global__ void __launch_bounds__(kFcgBS) fcg_residual_kernel(int vh, int pv, const void *b, const void *s, void *r,
                                                              FcgState *st, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    double v[1] = {0.0};
    if (i < vh) {
        double bv[6], sv[6];
        ld_spinor<0>(b, pv, i, bv);
        ld_spinor<0>(s, pv, i, sv);
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            bv[e] -= sv[e];
            v[0] += bv[e] * bv[e];
        }
        st_spinor<0>(r, pv, i, bv);
    }
    double tot[1];
    if (fcg_grid_sum<1>(v, partials, &st->ticket, sm, tot)) {
        st->rr = tot[0];
        st->rr_check = tot[0];
        st->leave = 0;
        st->active = (tot[0] > st->target2 && st->it < st->max_iter) ? 1 : 0;
    }
}

// <p, w> and <p, r> -> alpha; a non-positive or non-finite p.Ap is a breakdown (the network phase hands over to
// plain CG)
__global__ void __launch_bounds__(kFcgBS) fcg_alpha_kernel(int vh, int pv, const void *p, const void *w,
                                                           const void *r, FcgState *st, double *partials)
{
    if (!st->active) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    double v[2] = {0.0, 0.0};
    if (i < vh) {
        double pv6[6], wv[6], rv[6];
        ld_spinor<0>(p, pv, i, pv6);
        ld_spinor<0>(w, pv, i, wv);
        ld_spinor<0>(r, pv, i, rv);
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            v[0] += pv6[e] * wv[e];
            v[1] += pv6[e] * rv[e];
        }
    }
    double tot[2];
    if (fcg_grid_sum<2>(v, partials, &st->ticket, sm, tot)) {
        const double alpha = tot[1] / tot[0];
        st->pw = tot[0];
        st->alpha = alpha;
        if (!(tot[0] > 0) || !isfinite(alpha)) {
            st->active = 0;
            st->leave = st->use_net;
            st->alpha = 0.0;
        }
    }
}

// x += alpha p ; r -= alpha w ; |r|^2 -> convergence, stagnation and budget tests
__global__ void __launch_bounds__(kFcgBS) fcg_update_kernel(int vh, int pv, void *x, void *r, const void *p,
                                                            const void *w, FcgState *st, double *partials)
{
    if (!st->active) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    const double alpha = st->alpha;
    double v[1] = {0.0};
    if (i < vh) {
        double xv[6], rv[6], pv6[6], wv[6];
        ld_spinor<0>(x, pv, i, xv);
        ld_spinor<0>(r, pv, i, rv);
        ld_spinor<0>(p, pv, i, pv6);
        ld_spinor<0>(w, pv, i, wv);
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            xv[e] += alpha * pv6[e];
            rv[e] -= alpha * wv[e];
            v[0] += rv[e] * rv[e];
        }
        st_spinor<0>(x, pv, i, xv);
        st_spinor<0>(r, pv, i, rv);
    }
    double tot[1];
    if (fcg_grid_sum<1>(v, partials, &st->ticket, sm, tot)) {
        const double rr = tot[0];
        st->rr = rr;
        st->it += 1;
        st->total += 1;
        if (st->use_net) st->net_it += 1;
        if (rr <= st->target2) {
            st->active = 0;
        } else if (st->use_net && st->it % kStall == 0) {
            if (!(rr < 0.5 * st->rr_check)) {
                st->active = 0;
                st->leave = 1;
            } else {
                st->rr_check = rr;
            }
        }
        if (st->active && st->it >= st->max_iter) {
            st->active = 0;
            st->leave = st->use_net;
        }
    }
}

// <z, w> -> beta = -<z, w> / <p, w> (one A-orthogonalisation against the previous direction)
__global__ void __launch_bounds__(kFcgBS) fcg_beta_kernel(int vh, int pv, const void *z, const void *w, FcgState *st,
                                                          double *partials)
{
    if (!st->active) return;
    __shared__ double sm[32];
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    double v[1] = {0.0};
    if (i < vh) {
        double zv[6], wv[6];
        ld_spinor<0>(z, pv, i, zv);
        ld_spinor<0>(w, pv, i, wv);
#pragma unroll
        for (int e = 0; e < 6; ++e) v[0] += zv[e] * wv[e];
    }
    double tot[1];
    if (fcg_grid_sum<1>(v, partials, &st->ticket, sm, tot)) st->beta = -tot[0] / st->pw;
}

// p = z + beta p (restart = 1: p = z)
__global__ void __launch_bounds__(kFcgBS) fcg_xpay_kernel(int vh, int pv, const void *z, void *p, const FcgState *st,
                                                          int restart)
{
    if (!st->active) return;
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    if (i >= vh) return;
    const double beta = restart ? 0.0 : st->beta;
    double zv[6], pv6[6];
    ld_spinor<0>(z, pv, i, zv);
    ld_spinor<0>(p, pv, i, pv6);
#pragma unroll
    for (int e = 0; e < 6; ++e) pv6[e] = zv[e] + beta * pv6[e];
    st_spinor<0>(p, pv, i, pv6);
}

// z = r (the unpreconditioned phase)
__global__ void __launch_bounds__(kFcgBS) fcg_copy_kernel(int vh, int pv, const void *r, void *z, const FcgState *st)
{
    if (!st->active) return;
    const int i = blockIdx.x * kFcgBS + threadIdx.x;
    if (i >= vh) return;
    double v[6];
    ld_spinor<0>(r, pv, i, v);
    st_spinor<0>(z, pv, i, v);
}

}  // namespace kq

using namespace kq;

struct kq_net;
cudaError_t net_apply_async(kq_net *n, const void *d_in, void *d_out, int parity);

#define KQ_API extern "C" __attribute__((visibility("default")))

// Polish every shift of d_x (num_shift FP64 fields, initial guesses) to |b - A_k x_k| < rel_residual |b|.
// net may be NULL (plain CG).  info->iter_refine: total polish iterations; info->true_residual[k]: final residuals;
// info->iter: iterations that used the network.  The loop runs on the device: every reduction ends in its kernel's
// last block, which also takes the scalar step (alpha, beta, the convergence, stagnation and budget tests); the
// host enqueues kChunkIt iterations at a time and reads the state once per chunk.
KQ_API KuQCDStatus kq_fcg_polish(kq_context *ctx, kq_net *net, const kq_solve_param *param, const void *d_b,
                                 void *d_x, kq_solve_info *info)
{
    kq::NvtxRange nvtx_range_("kq_fcg_polish");
    if (!ctx || !param || !param->shifts || !d_b || !d_x) return KUQCD_ERR_NULL_POINTER;
    if (param->num_shift < 1 || param->num_shift > kMaxShift || (param->parity != 0 && param->parity != 1))
        return KUQCD_ERR_INVALID_PARAM;
    if (!ctx->gd.have[P64]) {
        KuQCDStatus st = kq_prepare_links(ctx, KUQCD_DOUBLE);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const size_t vb = spinor_bytes(g, P64);
    const int nb = (g.vh + kFcgBS - 1) / kFcgBS, pv = pad_sites(g.vh);
    Carve probe(nullptr);
    for (int k = 0; k < 6; ++k) probe.take(vb);
    probe.take(sizeof(double) * 2 * nb);
    probe.take(sizeof(FcgState));
    cudaError_t e = ensure_work(ctx, probe.off);
    if (e != cudaSuccess) return status_of(e);
    Carve c(ctx->work);
    void *r = c.take(vb), *z = c.take(vb), *p = c.take(vb), *w = c.take(vb), *tmp = c.take(vb), *s = c.take(vb);
    double *partials = static_cast<double *>(c.take(sizeof(double) * 2 * nb));
    FcgState *dst = static_cast<FcgState *>(c.take(sizeof(FcgState)));
    FcgState *hst = nullptr;
    e = cudaMallocHost(&hst, sizeof(FcgState));
    if (e != cudaSuccess) return status_of(e);
    const double target = param->rel_residual > 0 ? param->rel_residual : 1e-10;
    const int max_iter = param->max_iter > 0 ? param->max_iter : 20000;
    const int parity = param->parity;
    cudaStream_t st = ctx->stream;
    kq_solve_info local;
    if (!info) info = &local;
    memset(info, 0, sizeof(*info));
    info->num_shift = param->num_shift;
    long long launches = 0;
    constexpr int kChunkIt = 4;
    for (int k = 0; k < param->num_shift && e == cudaSuccess; ++k) {
        const double sig = (param->shift_mode == 0 && k > 0) ? param->shifts[0] + param->shifts[k] : param->shifts[k];
        void *x = static_cast<char *>(d_x) + k * vb;
        auto matvec = [&](const void *in, void *out) {
            if (e == cudaSuccess) e = launch_mdagm(g, ctx->gd, P64, sig, in, tmp, out, parity, st);
            launches += 2;
        };
        auto precond = [&](bool use_net) {  // z = M r
            if (e != cudaSuccess) return;
            if (use_net) {
                e = net_apply_async(net, r, z, parity);
                launches += net_apply_launches(net);
            } else {
                fcg_copy_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, r, z, dst);
                launches += 1;
            }
        };
        auto read_state = [&]() {
            if (e == cudaSuccess) e = cudaMemcpyAsync(hst, dst, sizeof(FcgState), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess && net) e = ptc_check_fault(st);
        };
        bool use_net = net != nullptr;
        // the state starts from zero: its ticket counts the blocks of every reduction
        if (e == cudaSuccess) e = cudaMemsetAsync(dst, 0, sizeof(FcgState), st);
        fcg_init_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, d_b, dst, partials, target, max_iter, use_net ? 1 : 0);
        launches += 1;
        // every chunk advances an active state by kChunkIt iterations and each phase has max_iter of them, so more
        // chunks than this mean the device state stopped advancing: an internal error, not a long solve
        const long long chunk_cap = 2LL * (max_iter / kChunkIt + 2) + 8;
        long long chunks = 0;
        for (;;) {  // phases: with the network, then (after a breakdown, stagnation or its budget) plain CG
            // r = b - A x, then the restart p = M r, w = A p
            matvec(x, s);
            fcg_residual_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, d_b, s, r, dst, partials);
            precond(use_net);
            fcg_xpay_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, z, p, dst, 1);
            matvec(p, w);
            launches += 2;
            for (;;) {
                for (int j = 0; j < kChunkIt && e == cudaSuccess; ++j) {
                    fcg_alpha_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, p, w, r, dst, partials);
                    fcg_update_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, x, r, p, w, dst, partials);
                    precond(use_net);
                    fcg_beta_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, z, w, dst, partials);
                    fcg_xpay_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, z, p, dst, 0);
                    matvec(p, w);
                    launches += 4;
                }
                if (e == cudaSuccess) e = cudaGetLastError();
                read_state();
                if (e != cudaSuccess || !hst->active) break;
                if (++chunks > chunk_cap) {
                    e = cudaErrorUnknown;
                    set_last_error("kq_fcg_polish: the polish state stopped advancing");
                    break;
                }
            }
            if (e == cudaSuccess && use_net && hst->leave) {
                // hand over to plain CG from the current x with a budget of its own
                use_net = false;
                FcgState h = *hst;
                h.use_net = 0;
                h.leave = 0;
                h.it = 0;
                e = cudaMemcpyAsync(dst, &h, sizeof(FcgState), cudaMemcpyHostToDevice, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                continue;
            }
            break;
        }
        // final FP64 true residual
        matvec(x, s);
        fcg_residual_kernel<<<nb, kFcgBS, 0, st>>>(g.vh, pv, d_b, s, r, dst, partials);
        launches += 1;
        read_state();
        if (e != cudaSuccess) break;
        info->iter_refine += hst->total;
        info->iter += hst->net_it;
        info->true_residual[k] = hst->bb > 0 ? std::sqrt(hst->rr / hst->bb) : 0.0;
        if (hst->rr > hst->target2) info->status = KQ_STATUS_MAXITER;
    }
    cudaFreeHost(hst);
    info->kernel_launches = launches;
    if (e != cudaSuccess) {
        if (e != cudaErrorUnknown) set_last_error(std::string("kq_fcg_polish: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    return KUQCD_SUCCESS;
}
