// The learned preconditioner as an object: a stack of parallel-transport convolution layers (kq_ptc.cu) with its
// weights, activations, gradients and Adam state on the device, and the C ABI to train and apply it.
//
// Weights: per layer complex W[o][i][p] (o < C_out, i < C_in, p < 9), stored as interleaved (re, im) floats, layers
// concatenated.  The layers form a linear map N = L_{K-1} ... L_0 from one channel to C_K channels; the
// preconditioner is its Gram operator
//     M(r) = extract( L_0^dag ... L_{K-1}^dag L_{K-1} ... L_0 embed(r) )
// read back on r's parity, symmetric positive semi-definite by construction (up to BF16 rounding), as a CG-type
// outer iteration wants.  Training pairs (r, e): loss |M(r) - e|^2 / |e|^2; every layer's weights get two gradient
// contributions, one through L_l and one through L_l^dag (kq_ptc.cu computes both with the same GEMM kernels).
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_ptc.h"

using namespace kq;

namespace kq {

// Bt[n][k] (BF16) of the real GEMM for one layer.  Forward: k = (p*C_in + i)*2 + kr, n = o*2 + nr.  Adjoint: the
// layer maps C_out -> C_in channels with W'[i][o][p] = conj(W[o][i][p]).
__global__ void net_build_bt_kernel(const float *__restrict__ W, int cin, int cout, int adjoint,
                                    __nv_bfloat16 *__restrict__ Bt, int kp, int np)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= kp * np) return;
    const int n = e / kp, k = e - n * kp;
    const int ci = adjoint ? cout : cin;  // input channels of the GEMM
    const int co = adjoint ? cin : cout;  // output channels of the GEMM
    float v = 0.f;
    if (k < ci * 18 && n < co * 2) {
        const int p = k / (2 * ci), a = (k >> 1) - p * ci, kr = k & 1;  // a: GEMM input channel
        const int b = n >> 1, nr = n & 1;                   // b: GEMM output channel
        // forward: W[o=b][i=a][p];  adjoint: W'[i=b][o=a][p] = conj(W[o=a][i=b][p])
        const int o = adjoint ? a : b, i = adjoint ? b : a;
        const float wr = W[2 * ((o * cin + i) * 9 + p)];
        float wi = W[2 * ((o * cin + i) * 9 + p) + 1];
        if (adjoint) wi = -wi;
        v = (kr == 0) ? (nr == 0 ? wr : wi) : (nr == 0 ? -wi : wr);
    }
    Bt[e] = __float2bfloat16_rn(v);
}

// grad[o][i][p] += dL/dW from the GEMM gradient dB[k][n] of the layer (cin -> cout).  Forward layer: k =
// (p*cin+i)*2+kr, n = o*2+nr.  Adjoint layer (the GEMM runs cout -> cin with W' = conj(W)): k = (p*cout+o)*2+kr,
// n = i*2+nr, and dL/dW = conj(dL/dW').  np: the GEMM's padded column count.
__global__ void net_accum_grad_kernel(const float *__restrict__ dB, int cin, int cout, int np, int adjoint,
                                      float *__restrict__ grad)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= cout * cin * 9) return;
    const int o = e / (cin * 9), rem = e - o * cin * 9, i = rem / 9, p = rem - i * 9;
    const int k0 = (p * (adjoint ? cout : cin) + (adjoint ? o : i)) * 2, n0 = (adjoint ? i : o) * 2;
    const float d00 = dB[k0 * np + n0], d01 = dB[k0 * np + n0 + 1];
    const float d10 = dB[(k0 + 1) * np + n0], d11 = dB[(k0 + 1) * np + n0 + 1];
    grad[2 * e] += d00 + d11;                                // d/dW_re
    grad[2 * e + 1] += adjoint ? d10 - d01 : d01 - d10;      // d/dW_im
}

}  // namespace kq

struct kq_net {
    kq_context *ctx = nullptr;
    int dims[4] = {0, 0, 0, 0};  // lattice of the contexts the network may use
    int device = 0;
    int nl = 0;
    std::vector<int> ch;     // nl + 1 channel counts
    std::vector<size_t> woff;  // float offsets of each layer's weights
    size_t nw = 0;           // floats
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
    std::vector<void *> bt, bta;  // per-layer forward / adjoint BF16 matrices
    std::vector<float2 *> act;    // nl + 1 activations of the forward chain: a_0 = embed(r), a_{l+1} = L_l a_l
    std::vector<float2 *> cact;   // adjoint chain c_l = L_l^dag c_{l+1}, l < nl (c_nl = a_nl)
    float2 *gbuf[2] = {nullptr, nullptr};
    float *partial = nullptr, *dB = nullptr;
    double *lpart = nullptr;
    size_t act_stride = 0;  // floats2 per channel (2 parities x 3 colours x pv)
    int step = 0;
    bool bt_dirty = true;
};

#define KQ_API extern "C" __attribute__((visibility("default")))

static void net_free(kq_net *n)
{
    auto F = [](void *p) {
        if (p) cudaFree(p);
    };
    F(n->w), F(n->g), F(n->m), F(n->v), F(n->partial), F(n->dB), F(n->lpart);
    for (void *p : n->bt) F(p);
    for (void *p : n->bta) F(p);
    for (float2 *p : n->act) F(p);
    for (float2 *p : n->cact) F(p);
    F(n->gbuf[0]), F(n->gbuf[1]);
}

KQ_API void kq_net_destroy(kq_net *n)
{
    if (!n) return;
    // the context the network last used may already be gone: synchronise the device instead of its stream
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    net_free(n);
    delete n;
}

KQ_API KuQCDStatus kq_net_create(kq_context *ctx, int nlayers, const int *channels, kq_net **out)
{
    if (!ctx || !channels || !out) return KUQCD_ERR_NULL_POINTER;
    if (nlayers < 1 || nlayers > 16 || channels[0] != 1) {
        set_last_error("kq_net_create: 1..16 layers and one input channel");
        return KUQCD_ERR_INVALID_PARAM;
    }
    for (int l = 0; l <= nlayers; ++l)
        if (channels[l] != 1 && channels[l] != 8) {
            set_last_error("kq_net_create: hidden layers have 8 channels");
            return KUQCD_ERR_UNSUPPORTED;
        }
    kq_net *n = new (std::nothrow) kq_net();
    if (!n) return KUQCD_ERR_NO_MEMORY;
    n->ctx = ctx;
    for (int d = 0; d < 4; ++d) n->dims[d] = ctx->g.n[d];
    n->device = ctx->device;
    n->nl = nlayers;
    n->ch.assign(channels, channels + nlayers + 1);
    for (int l = 0; l < nlayers; ++l) {
        n->woff.push_back(n->nw);
        n->nw += 2 * (size_t)n->ch[l] * n->ch[l + 1] * 9;
    }
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const size_t pv = pad_sites(g.vh);
    n->act_stride = 6 * pv;
    cudaError_t e = cudaSuccess;
    auto A = [&](void **p, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) e = cudaMemset(*p, 0, bytes);
    };
    A((void **)&n->w, n->nw * 4);
    A((void **)&n->g, n->nw * 4);
    A((void **)&n->m, n->nw * 4);
    A((void **)&n->v, n->nw * 4);
    n->act.assign(nlayers + 1, nullptr);
    for (int l = 0; l <= nlayers; ++l) A((void **)&n->act[l], n->act_stride * n->ch[l] * sizeof(float2));
    n->cact.assign(nlayers, nullptr);
    for (int l = 0; l < nlayers; ++l) A((void **)&n->cact[l], n->act_stride * n->ch[l] * sizeof(float2));
    A((void **)&n->gbuf[0], n->act_stride * 8 * sizeof(float2));
    A((void **)&n->gbuf[1], n->act_stride * 8 * sizeof(float2));
    n->bt.assign(nlayers, nullptr);
    n->bta.assign(nlayers, nullptr);
    size_t maxkn = 0;
    for (int l = 0; l < nlayers; ++l) {
        const int ci = n->ch[l], co = n->ch[l + 1];
        A(&n->bt[l], (size_t)ptc_kpad(ci) * ptc_npad(co) * 2);
        A(&n->bta[l], (size_t)ptc_kpad(co) * ptc_npad(ci) * 2);
        maxkn = std::max(maxkn, (size_t)ptc_kpad(ci) * ptc_npad(co));
        maxkn = std::max(maxkn, (size_t)ptc_kpad(co) * ptc_npad(ci));
    }
    A((void **)&n->partial, (size_t)ptc_tiles(g) * maxkn * 4);
    A((void **)&n->dB, maxkn * 4);
    A((void **)&n->lpart, sizeof(double) * ((g.vh + 255) / 256 + 1));
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_net_create: ") + cudaGetErrorString(e));
        net_free(n);
        delete n;
        return status_of(e);
    }
    *out = n;
    return KUQCD_SUCCESS;
}

KQ_API size_t kq_net_num_weights(const kq_net *n) { return n ? n->nw : 0; }

KQ_API KuQCDStatus kq_net_set_weights(kq_net *n, const float *w, size_t count)
{
    if (!n || !w) return KUQCD_ERR_NULL_POINTER;
    if (count != n->nw) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(n->ctx->device);
    cudaError_t e = cudaMemcpy(n->w, w, count * 4, cudaMemcpyHostToDevice);
    n->bt_dirty = true;
    return status_of(e);
}

KQ_API KuQCDStatus kq_net_get_weights(const kq_net *n, float *w, size_t count)
{
    if (!n || !w) return KUQCD_ERR_NULL_POINTER;
    if (count != n->nw) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(n->ctx->device);
    cudaStreamSynchronize(n->ctx->stream);
    return status_of(cudaMemcpy(w, n->w, count * 4, cudaMemcpyDeviceToHost));
}

KQ_API KuQCDStatus kq_net_get_grad(const kq_net *n, float *gr, size_t count)
{
    if (!n || !gr) return KUQCD_ERR_NULL_POINTER;
    if (count != n->nw) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(n->ctx->device);
    cudaStreamSynchronize(n->ctx->stream);
    return status_of(cudaMemcpy(gr, n->g, count * 4, cudaMemcpyDeviceToHost));
}

KQ_API KuQCDStatus kq_net_zero_grad(kq_net *n)
{
    if (!n) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(n->ctx->device);
    return status_of(cudaMemsetAsync(n->g, 0, n->nw * 4, n->ctx->stream));
}

// use the links of another context (same lattice) from now on; the previous context may already be destroyed
KQ_API KuQCDStatus kq_net_set_context(kq_net *n, kq_context *ctx)
{
    if (!n || !ctx) return KUQCD_ERR_NULL_POINTER;
    for (int d = 0; d < 4; ++d)
        if (ctx->g.n[d] != n->dims[d] || ctx->device != n->device) {
            set_last_error("kq_net_set_context: different lattice or device");
            return KUQCD_ERR_INVALID_PARAM;
        }
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    n->ctx = ctx;
    return KUQCD_SUCCESS;
}

namespace {

cudaError_t ensure_bt(kq_net *n)
{
    if (!n->bt_dirty) return cudaSuccess;
    cudaStream_t s = n->ctx->stream;
    for (int l = 0; l < n->nl; ++l) {
        const int ci = n->ch[l], co = n->ch[l + 1];
        const int kp = ptc_kpad(ci), np = ptc_npad(co), kpa = ptc_kpad(co), npa = ptc_npad(ci);
        net_build_bt_kernel<<<(kp * np + 255) / 256, 256, 0, s>>>(n->w + n->woff[l], ci, co, 0,
                                                                   (__nv_bfloat16 *)n->bt[l], kp, np);
        net_build_bt_kernel<<<(kpa * npa + 255) / 256, 256, 0, s>>>(n->w + n->woff[l], ci, co, 1,
                                                                     (__nv_bfloat16 *)n->bta[l], kpa, npa);
    }
    n->bt_dirty = false;
    return cudaGetLastError();
}

// a_0 = embed(d_in), a_{l+1} = L_l a_l, c_nl = a_nl, c_l = L_l^dag c_{l+1}; the result is c_0 (cact[0])
cudaError_t forward(kq_net *n, const void *d_in, int parity, double in_scale)
{
    kq_context *ctx = n->ctx;
    const LinkSet &fat = ctx->gd.fat[P32];
    KQ_CUDA_TRY(ensure_bt(n));
    KQ_CUDA_TRY(ptc_embed(ctx->g, d_in, parity, n->act[0], in_scale, ctx->stream));
    for (int l = 0; l < n->nl; ++l)
        KQ_CUDA_TRY(ptc_forward(ctx->g, fat, n->ch[l], n->ch[l + 1], n->act[l], n->act[l + 1], n->bt[l], false,
                                ctx->stream));
    for (int l = n->nl - 1; l >= 0; --l) {
        const float2 *in = (l == n->nl - 1) ? n->act[n->nl] : n->cact[l + 1];
        KQ_CUDA_TRY(ptc_forward(ctx->g, fat, n->ch[l + 1], n->ch[l], in, n->cact[l], n->bta[l], true, ctx->stream));
    }
    return cudaSuccess;
}

KuQCDStatus prepare(kq_net *n)
{
    if (!n->ctx->gd.have[P32]) return kq_prepare_links(n->ctx, KUQCD_SINGLE);
    return KUQCD_SUCCESS;
}

}  // namespace

// ptc_check_fault reports a tile whose bounded wait ran out as cudaErrorLaunchTimeout
static const char *net_error_text(cudaError_t e)
{
    return e == cudaErrorLaunchTimeout ? "a tensor-core tile did not complete within the wait limit"
                                       : cudaGetErrorString(e);
}

// kernels one kq_net_apply launches once its BF16 matrices are built: embed, 2 x nl layers, extract
int net_apply_launches(const kq_net *n) { return n ? 2 + 2 * n->nl : 0; }

// d_out = M(d_in) enqueued on the context's stream without waiting for it: the caller checks the tensor-core
// fault word later (ptc_check_fault), once for many applications (the FCG polish, once per chunk of iterations)
cudaError_t net_apply_async(kq_net *n, const void *d_in, void *d_out, int parity)
{
    if (prepare(n) != KUQCD_SUCCESS) return cudaErrorInvalidValue;
    KQ_CUDA_TRY(forward(n, d_in, parity, 1.0));
    return ptc_extract(n->ctx->g, n->cact[0], parity, d_out, 1.0, n->ctx->stream);
}

// d_out = M(d_in) on `parity` (FP64 fields of the context's layout)
KQ_API KuQCDStatus kq_net_apply(kq_net *n, const void *d_in, void *d_out, int parity)
{
    kq::NvtxRange nvtx_range_("kq_net_apply");
    if (!n || !d_in || !d_out) return KUQCD_ERR_NULL_POINTER;
    if (parity != 0 && parity != 1) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(n->ctx->device);
    KuQCDStatus st = prepare(n);
    if (st != KUQCD_SUCCESS) return st;
    cudaError_t e = forward(n, d_in, parity, 1.0);
    if (e == cudaSuccess) e = ptc_extract(n->ctx->g, n->cact[0], parity, d_out, 1.0, n->ctx->stream);
    if (e == cudaSuccess) e = ptc_check_fault(n->ctx->stream);
    if (e != cudaSuccess) set_last_error(std::string("kq_net_apply: ") + net_error_text(e));
    return status_of(e);
}

// forward + loss + backward for one pair (r, e); gradients are added to the accumulator.  loss: |M(r)-e|^2/|e|^2
KQ_API KuQCDStatus kq_net_train_pair(kq_net *n, const void *d_r, const void *d_e, int parity, double e_norm2,
                                     double *loss)
{
    kq::NvtxRange nvtx_range_("kq_net_train_pair");
    if (!n || !d_r || !d_e) return KUQCD_ERR_NULL_POINTER;
    if ((parity != 0 && parity != 1) || !(e_norm2 > 0)) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(n->ctx->device);
    KuQCDStatus st = prepare(n);
    if (st != KUQCD_SUCCESS) return st;
    kq_context *ctx = n->ctx;
    const LinkSet &fat = ctx->gd.fat[P32];
    cudaStream_t s = ctx->stream;
    cudaError_t e = forward(n, d_r, parity, 1.0);
    double l = 0;
    int cur = 0;
    if (e == cudaSuccess) e = ptc_loss(ctx->g, n->cact[0], d_e, parity, 1.0 / e_norm2, n->gbuf[cur], n->lpart, &l, s);
    auto accum = [&](int layer, bool adjoint) {
        if (e != cudaSuccess) return;
        const int ci = n->ch[layer], co = n->ch[layer + 1];
        net_accum_grad_kernel<<<(co * ci * 9 + 255) / 256, 256, 0, s>>>(
            n->dB, ci, co, ptc_npad(adjoint ? ci : co), adjoint ? 1 : 0, n->g + n->woff[layer]);
        e = cudaGetLastError();
    };
    // adjoint chain, output side first: gbuf[cur] holds dL/dc_l; c_l = L_l^dag c_{l+1} gives the adjoint-layer
    // weight gradient and dL/dc_{l+1} = L_l dL/dc_l
    for (int layer = 0; layer < n->nl && e == cudaSuccess; ++layer) {
        const int ci = n->ch[layer], co = n->ch[layer + 1];
        const float2 *in = (layer == n->nl - 1) ? n->act[n->nl] : n->cact[layer + 1];
        e = ptc_wgrad(ctx->g, fat, co, ci, in, n->gbuf[cur], n->partial, n->dB, true, s);
        accum(layer, true);
        if (e == cudaSuccess) e = ptc_forward(ctx->g, fat, ci, co, n->gbuf[cur], n->gbuf[1 - cur], n->bt[layer], false, s);
        cur = 1 - cur;
    }
    // forward chain: gbuf[cur] holds dL/da_{l+1}; dL/da_l = L_l^dag dL/da_{l+1}
    for (int layer = n->nl - 1; layer >= 0 && e == cudaSuccess; --layer) {
        const int ci = n->ch[layer], co = n->ch[layer + 1];
        e = ptc_wgrad(ctx->g, fat, ci, co, n->act[layer], n->gbuf[cur], n->partial, n->dB, false, s);
        accum(layer, false);
        if (layer > 0 && e == cudaSuccess) {
            e = ptc_forward(ctx->g, fat, co, ci, n->gbuf[cur], n->gbuf[1 - cur], n->bta[layer], true, s);
            cur = 1 - cur;
        }
    }
    if (e == cudaSuccess) e = ptc_check_fault(s);
    if (loss) *loss = l;
    if (e != cudaSuccess) set_last_error(std::string("kq_net_train_pair: ") + net_error_text(e));
    return status_of(e);
}

// sets the device fault word the network's tensor-core tiles raise on a timed-out wait, from the host
KQ_API KuQCDStatus kq_net_raise_fault_for_test(kq_net *n)
{
    if (!n) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(n->ctx->device);
    return status_of(ptc_raise_fault_for_test());
}

// Adam step with the accumulated gradient scaled by grad_scale (e.g. 1/batch); clears the accumulator
KQ_API KuQCDStatus kq_net_adam(kq_net *n, float lr, float grad_scale)
{
    if (!n) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(n->ctx->device);
    cudaStream_t s = n->ctx->stream;
    n->step += 1;
    // the kernel scales the gradient, steps and clears the accumulator
    cudaError_t e = ptc_adam(n->w, n->g, n->m, n->v, (int)n->nw, lr, grad_scale, n->step, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    n->bt_dirty = true;
    return status_of(e);
}
