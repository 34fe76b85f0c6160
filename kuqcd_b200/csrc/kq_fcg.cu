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
extern "C" KuQCDStatus kq_net_apply(kq_net *n, const void *d_in, void *d_out, int parity);
int net_apply_launches(const kq_net *n);

namespace kq {

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s);

// partials of up to three dot products <a_j, b_j> of FP64 fields
__global__ void __launch_bounds__(256) fcg_dots_kernel(int vh, int pv, int nd, const void *a0, const void *b0,
                                                       const void *a1, const void *b1, const void *a2,
                                                       const void *b2, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * 256 + threadIdx.x;
    const void *A[3] = {a0, a1, a2}, *B[3] = {b0, b1, b2};
    for (int j = 0; j < nd; ++j) {
        double s = 0.0;
        if (i < vh) {
            double x[6], y[6];
            ld_spinor<0>(A[j], pv, i, x);
            ld_spinor<0>(B[j], pv, i, y);
#pragma unroll
            for (int e = 0; e < 6; ++e) s += x[e] * y[e];
        }
        s = block_sum(s, sm);
        if (threadIdx.x == 0) partials[j * gridDim.x + blockIdx.x] = s;
        __syncthreads();
    }
}

// x += alpha p ; r -= alpha w
__global__ void fcg_update_kernel(int vh, int pv, void *x, void *r, const void *p, const void *w, double alpha)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= vh) return;
    double xv[6], rv[6], pv6[6], wv[6];
    ld_spinor<0>(x, pv, i, xv);
    ld_spinor<0>(r, pv, i, rv);
    ld_spinor<0>(p, pv, i, pv6);
    ld_spinor<0>(w, pv, i, wv);
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        xv[e] += alpha * pv6[e];
        rv[e] -= alpha * wv[e];
    }
    st_spinor<0>(x, pv, i, xv);
    st_spinor<0>(r, pv, i, rv);
}

// p = z + beta p   (beta = 0: p = z)
__global__ void fcg_xpay_kernel(int vh, int pv, const void *z, void *p, double beta)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= vh) return;
    double zv[6], pv6[6];
    ld_spinor<0>(z, pv, i, zv);
    ld_spinor<0>(p, pv, i, pv6);
#pragma unroll
    for (int e = 0; e < 6; ++e) pv6[e] = zv[e] + beta * pv6[e];
    st_spinor<0>(p, pv, i, pv6);
}

// r = b - s
__global__ void fcg_sub_kernel(int vh, int pv, const void *b, const void *s, void *r)
{
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= vh) return;
    double bv[6], sv[6];
    ld_spinor<0>(b, pv, i, bv);
    ld_spinor<0>(s, pv, i, sv);
#pragma unroll
    for (int e = 0; e < 6; ++e) bv[e] -= sv[e];
    st_spinor<0>(r, pv, i, bv);
}

}  // namespace kq

using namespace kq;

namespace {

struct Fcg {
    kq_context *ctx;
    int nb, pv;
    double *partials;
    std::vector<double> h;
    cudaError_t err = cudaSuccess;

    void dots(int nd, const void *a0, const void *b0, const void *a1, const void *b1, const void *a2,
              const void *b2, double *out)
    {
        if (err != cudaSuccess) return;
        fcg_dots_kernel<<<nb, 256, 0, ctx->stream>>>(ctx->g.vh, pv, nd, a0, b0, a1, b1, a2, b2, partials);
        err = cudaMemcpyAsync(h.data(), partials, sizeof(double) * nb * nd, cudaMemcpyDeviceToHost, ctx->stream);
        if (err == cudaSuccess) err = cudaStreamSynchronize(ctx->stream);
        for (int j = 0; j < nd; ++j) {
            double s = 0;
            for (int b = 0; b < nb; ++b) s += h[j * nb + b];
            out[j] = s;
        }
    }
};

}  // namespace

#define KQ_API extern "C" __attribute__((visibility("default")))

// Polish every shift of d_x (num_shift FP64 fields, initial guesses) to |b - A_k x_k| < rel_residual |b|.
// net may be NULL (plain CG).  info->iter_refine: total polish iterations; info->true_residual[k]: final residuals;
// info->iter: iterations that used the network.
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
    Fcg F;
    F.ctx = ctx;
    F.nb = (g.vh + 255) / 256;
    F.pv = pad_sites(g.vh);
    F.h.resize(3 * F.nb);
    Carve probe(nullptr);
    for (int k = 0; k < 6; ++k) probe.take(vb);
    probe.take(sizeof(double) * 3 * F.nb);
    cudaError_t e = ensure_work(ctx, probe.off);
    if (e != cudaSuccess) return status_of(e);
    Carve c(ctx->work);
    void *r = c.take(vb), *z = c.take(vb), *p = c.take(vb), *w = c.take(vb), *tmp = c.take(vb), *s = c.take(vb);
    F.partials = static_cast<double *>(c.take(sizeof(double) * 3 * F.nb));
    const double target = param->rel_residual > 0 ? param->rel_residual : 1e-10;
    const int max_iter = param->max_iter > 0 ? param->max_iter : 20000;
    const int parity = param->parity;
    cudaStream_t st = ctx->stream;
    const int nb = F.nb, pv = F.pv;
    double bb;
    F.dots(1, d_b, d_b, nullptr, nullptr, nullptr, nullptr, &bb);
    kq_solve_info local;
    if (!info) info = &local;
    memset(info, 0, sizeof(*info));
    info->num_shift = param->num_shift;
    long long launches = 0;
    for (int k = 0; k < param->num_shift && F.err == cudaSuccess; ++k) {
        const double sig = (param->shift_mode == 0 && k > 0) ? param->shifts[0] + param->shifts[k] : param->shifts[k];
        void *x = static_cast<char *>(d_x) + k * vb;
        auto matvec = [&](const void *in, void *out) {
            if (F.err == cudaSuccess) F.err = launch_mdagm(g, ctx->gd, P64, sig, in, tmp, out, parity, st);
            launches += 2;
        };
        auto precond = [&](const void *in, void *out, bool use_net) {
            if (F.err != cudaSuccess) return;
            if (use_net) {
                if (kq_net_apply(net, in, out, parity) != KUQCD_SUCCESS) F.err = cudaErrorUnknown;
                launches += net_apply_launches(net);
            } else {
                F.err = cudaMemcpyAsync(out, in, vb, cudaMemcpyDeviceToDevice, st);
            }
        };
        // r = b - A x
        matvec(x, s);
        fcg_sub_kernel<<<nb, 256, 0, st>>>(g.vh, pv, d_b, s, r);
        double rr;
        F.dots(1, r, r, nullptr, nullptr, nullptr, nullptr, &rr);
        // The network phase ends on convergence, on a breakdown (p^T A p <= 0), on stagnation (|r|^2 not halved over
        // kStall iterations) or when its budget is spent; the unpreconditioned phase then starts from the current x
        // with a budget of its own.  Every iteration of both phases counts in iter_refine.
        constexpr int kStall = 200;
        bool use_net = net != nullptr;
        int it = 0;  // iterations of the current phase
        while (F.err == cudaSuccess && rr > target * target * bb && it < max_iter) {
            // (re)start: p = M r, w = A p
            precond(r, z, use_net);
            fcg_xpay_kernel<<<nb, 256, 0, st>>>(g.vh, pv, z, p, 0.0);
            matvec(p, w);
            bool leave_net = false;
            double rr_check = rr;
            while (F.err == cudaSuccess && it < max_iter) {
                double d2[2];
                F.dots(2, p, w, p, r, nullptr, nullptr, d2);  // pw, pr
                const double pw = d2[0], alpha = d2[1] / pw;
                if (!(pw > 0) || !std::isfinite(alpha)) {
                    leave_net = use_net;
                    break;
                }
                fcg_update_kernel<<<nb, 256, 0, st>>>(g.vh, pv, x, r, p, w, alpha);
                ++it;
                info->iter_refine += 1;
                if (use_net) info->iter += 1;
                F.dots(1, r, r, nullptr, nullptr, nullptr, nullptr, &rr);
                if (rr <= target * target * bb) break;
                if (use_net && it % kStall == 0) {
                    if (!(rr < 0.5 * rr_check)) {
                        leave_net = true;
                        break;
                    }
                    rr_check = rr;
                }
                precond(r, z, use_net);
                double zw;
                F.dots(1, z, w, nullptr, nullptr, nullptr, nullptr, &zw);
                fcg_xpay_kernel<<<nb, 256, 0, st>>>(g.vh, pv, z, p, -zw / pw);
                matvec(p, w);
                launches += 5;
            }
            if (use_net && (leave_net || (rr > target * target * bb && it >= max_iter))) {
                use_net = false;
                it = 0;
                if (F.err == cudaSuccess) {  // the breakdown may have left no update: recompute r = b - A x
                    matvec(x, s);
                    fcg_sub_kernel<<<nb, 256, 0, st>>>(g.vh, pv, d_b, s, r);
                    F.dots(1, r, r, nullptr, nullptr, nullptr, nullptr, &rr);
                }
                continue;
            }
            break;
        }
        // final FP64 true residual
        matvec(x, s);
        fcg_sub_kernel<<<nb, 256, 0, st>>>(g.vh, pv, d_b, s, r);
        F.dots(1, r, r, nullptr, nullptr, nullptr, nullptr, &rr);
        info->true_residual[k] = std::sqrt(rr / bb);
        if (rr > target * target * bb) info->status = KQ_STATUS_MAXITER;
    }
    info->kernel_launches = launches;
    if (F.err != cudaSuccess) {
        set_last_error(std::string("kq_fcg_polish: ") + cudaGetErrorString(F.err));
        return status_of(F.err);
    }
    return KUQCD_SUCCESS;
}
