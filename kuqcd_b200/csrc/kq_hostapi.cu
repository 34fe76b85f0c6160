// Host-record entry points behind the class-level API (include/dirac_hisq.h, spinor_field.h, inverter_cgm.h, ...).
//
// The reference's class API works on fields whose values live in host memory (LatticeField::data,
// lattice_field.h:23-39): DiracHISQ::Dslash / MdaggM (dirac_hisq.cpp:409-462) and the BLAS-1 free functions
// (spinor_field.cpp:130-252) read and write `data` directly.  The header-only shells keep that contract -- `data`
// stays host memory a caller may touch between calls -- and run every operation on the GPU through these calls: the
// operands are copied in, the kernels run, the result is copied back before the call returns.
//
// Records are the NORMAL_ORDER layouts of kuqcd.cpp:103-169 (spinor h[reim + 2*(c + 3*i_cb)] over one parity, or
// even sites then odd sites for a full-lattice field).  Staging buffers come from the stream-ordered pool
// (cudaMallocAsync) and are returned to it at the end of each call.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "kq_context.h"
#include "kq_internal.h"

#define KQ_API extern "C" __attribute__((visibility("default")))

namespace kq {
cudaError_t launch_dslash_full(const Geom &g, const GaugeDev &gd, int prec, const void *src, const void *pvec,
                               void *dst, double sigma, cudaStream_t s);
cudaError_t launch_mdagm_full(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                              void *dst, cudaStream_t s);
cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s);
}  // namespace kq

using namespace kq;

namespace {

// ------------------------------------------------------------------------------------------ BLAS-1 on records
// y = a x + b y over n reals, in T as the reference's loops (spinor_field.cpp:130-200)
template <typename T>
__global__ void vec_axpby_kernel(size_t n, double a, const T *__restrict__ x, double b, T *__restrict__ y)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const T ta = (T)a, tb = (T)b;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) y[i] = ta * x[i] + tb * y[i];
}

constexpr int kDotThreads = 256;

// per-block FP64 partial sums of x_i y_i in a fixed order (grid-stride per thread, then a tree over the block)
template <typename T>
__global__ void vec_dot_kernel(size_t n, const T *__restrict__ x, const T *__restrict__ y, double *partial)
{
    __shared__ double red[kDotThreads];
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc += (double)x[i] * (double)y[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kDotThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// sum of the block partials, in block order, by one thread
__global__ void vec_sum_kernel(const double *partial, int nblocks, double *out)
{
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[b];
    *out = s;
}

int blocks_for(size_t n, int device)
{
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    const size_t want = (n + kDotThreads - 1) / kDotThreads;
    return (int)std::max<size_t>(1, std::min<size_t>(want, (size_t)nsm * 8));
}

// one stream per device for the record BLAS (created on first use, kept until exit)
cudaStream_t vec_stream(int device)
{
    static std::mutex mu;
    static std::vector<cudaStream_t> streams;
    std::lock_guard<std::mutex> lk(mu);
    if ((int)streams.size() <= device) streams.resize(device + 1, nullptr);
    if (!streams[device]) cudaStreamCreateWithFlags(&streams[device], cudaStreamNonBlocking);
    return streams[device];
}

struct Pool {  // stream-ordered staging allocations, released at scope exit
    cudaStream_t s;
    std::vector<void *> ptrs;
    explicit Pool(cudaStream_t st) : s(st) {}
    cudaError_t get(void **p, size_t bytes)
    {
        *p = nullptr;
        const cudaError_t e = cudaMallocAsync(p, bytes, s);
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
    ~Pool()
    {
        for (void *p : ptrs) cudaFreeAsync(p, s);
    }
};

bool record_prec_ok(int host_prec) { return host_prec == KUQCD_DOUBLE || host_prec == KUQCD_SINGLE; }

}  // namespace

KQ_API KuQCDStatus kq_host_alloc(size_t bytes, void **out)
{
    if (!out) return KUQCD_ERR_NULL_POINTER;
    *out = nullptr;
    if (bytes == 0) bytes = 64;
    if (cudaMallocHost(out, bytes) != cudaSuccess) {
        cudaGetLastError();
        // page-locking failed (limits, no device): plain 64-byte aligned host memory, as the reference allocates
        *out = aligned_alloc(64, (bytes + 63) & ~size_t(63));
        if (!*out) return KUQCD_ERR_NO_MEMORY;
    }
    return KUQCD_SUCCESS;
}

KQ_API void kq_host_free(void *p)
{
    if (!p) return;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost) {
        cudaFreeHost(p);
        return;
    }
    cudaGetLastError();
    free(p);
}

KQ_API KuQCDStatus kq_vec_axpby(int device, int host_prec, size_t n, double a, const void *h_x, double b, void *h_y)
{
    if (!h_x || !h_y) return KUQCD_ERR_NULL_POINTER;
    if (!record_prec_ok(host_prec)) return KUQCD_ERR_INVALID_PARAM;
    if (n == 0) return KUQCD_SUCCESS;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return status_of(e);
    const size_t w = host_prec == KUQCD_DOUBLE ? 8 : 4;
    cudaStream_t s = vec_stream(device);
    {
        Pool pool(s);
        void *dx = nullptr, *dy = nullptr;
        e = pool.get(&dx, n * w);
        if (e == cudaSuccess) e = pool.get(&dy, n * w);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dx, h_x, n * w, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(dy, h_y, n * w, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            const int nb = blocks_for(n, device);
            if (w == 8)
                vec_axpby_kernel<double><<<nb, 256, 0, s>>>(n, a, (const double *)dx, b, (double *)dy);
            else
                vec_axpby_kernel<float><<<nb, 256, 0, s>>>(n, a, (const float *)dx, b, (float *)dy);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(h_y, dy, n * w, cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) set_last_error(std::string("kq_vec_axpby: ") + cudaGetErrorString(e));
    return status_of(e);
}

KQ_API KuQCDStatus kq_vec_dot(int device, int host_prec, size_t n, const void *h_x, const void *h_y, double *out)
{
    if (!h_x || !h_y || !out) return KUQCD_ERR_NULL_POINTER;
    if (!record_prec_ok(host_prec)) return KUQCD_ERR_INVALID_PARAM;
    *out = 0.0;
    if (n == 0) return KUQCD_SUCCESS;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return status_of(e);
    const size_t w = host_prec == KUQCD_DOUBLE ? 8 : 4;
    cudaStream_t s = vec_stream(device);
    double result = 0.0;
    {
        Pool pool(s);
        void *dx = nullptr, *dy = nullptr, *dp = nullptr;
        const int nb = blocks_for(n, device);
        const bool same = h_x == h_y;
        e = pool.get(&dx, n * w);
        if (e == cudaSuccess && !same) e = pool.get(&dy, n * w);
        if (e == cudaSuccess) e = pool.get(&dp, (nb + 1) * sizeof(double));
        if (same) dy = dx;
        if (e == cudaSuccess) e = cudaMemcpyAsync(dx, h_x, n * w, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess && !same) e = cudaMemcpyAsync(dy, h_y, n * w, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) {
            double *part = (double *)dp;
            if (w == 8)
                vec_dot_kernel<double><<<nb, kDotThreads, 0, s>>>(n, (const double *)dx, (const double *)dy, part);
            else
                vec_dot_kernel<float><<<nb, kDotThreads, 0, s>>>(n, (const float *)dx, (const float *)dy, part);
            vec_sum_kernel<<<1, 1, 0, s>>>(part, nb, part + nb);
            e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaMemcpyAsync(&result, part + nb, sizeof(double), cudaMemcpyDeviceToHost, s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_vec_dot: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    *out = result;
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_apply_host(kq_context *ctx, int op, int prec, double sigma, const void *h_src, void *h_dst,
                                 int parity, int host_prec)
{
    if (!ctx || !h_src || !h_dst) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    const bool full = parity == KQ_PARITY_FULL;
    if (p < 0 || !record_prec_ok(host_prec) || (op != KQ_OP_DSLASH && op != KQ_OP_DD && op != KQ_OP_SIGMA_MINUS_DD) ||
        (parity != 0 && parity != 1 && !full)) {
        set_last_error("kq_apply_host: invalid operator, precision or parity");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->fat_loaded || !ctx->long_loaded) {
        set_last_error("kq_apply_host: load the fat and long links first");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    if (!ctx->gd.have[p]) {
        const KuQCDStatus st = kq_prepare_links(ctx, prec);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    cudaStream_t s = ctx->stream;
    const Geom &g = ctx->g;
    const size_t half = spinor_bytes(g, p);
    const size_t nb = full ? 2 * half : half;
    const size_t rec_half = (size_t)g.vh * 6 * (host_prec == KUQCD_DOUBLE ? 8 : 4);
    cudaError_t e = cudaSuccess;
    KuQCDStatus st = KUQCD_SUCCESS;
    {
        Pool pool(s);
        void *a = nullptr, *b = nullptr, *t = nullptr;
        e = pool.get(&a, nb);
        if (e == cudaSuccess) e = pool.get(&b, nb);
        if (e == cudaSuccess && op != KQ_OP_DSLASH) e = pool.get(&t, nb);
        if (e != cudaSuccess) {
            set_last_error(std::string("kq_apply_host: ") + cudaGetErrorString(e));
            return status_of(e);
        }
        // records in (one parity, or both halves of a full-lattice record)
        const int nparts = full ? 2 : 1;
        for (int h = 0; h < nparts && st == KUQCD_SUCCESS; ++h)
            st = kq_spinor_upload(ctx, prec, static_cast<const char *>(h_src) + h * rec_half, host_prec,
                                  static_cast<char *>(a) + h * half, s);
        if (st != KUQCD_SUCCESS) return st;
        if (full) {
            if (op == KQ_OP_DSLASH) e = launch_dslash_full(g, ctx->gd, p, a, nullptr, b, 0.0, s);
            else if (op == KQ_OP_DD) {
                e = launch_dslash_full(g, ctx->gd, p, a, nullptr, t, 0.0, s);
                if (e == cudaSuccess) e = launch_dslash_full(g, ctx->gd, p, t, nullptr, b, 0.0, s);
            } else
                e = launch_mdagm_full(g, ctx->gd, p, sigma, a, t, b, s);
        } else {
            if (op == KQ_OP_DSLASH) e = launch_dslash(g, ctx->gd, p, a, b, parity, s);
            else if (op == KQ_OP_DD) {
                e = launch_dslash(g, ctx->gd, p, a, t, 1 - parity, s);
                if (e == cudaSuccess) e = launch_dslash(g, ctx->gd, p, t, b, parity, s);
            } else
                e = launch_mdagm(g, ctx->gd, p, sigma, a, t, b, parity, s);
        }
        if (e != cudaSuccess) {
            set_last_error(std::string("kq_apply_host: ") + cudaGetErrorString(e));
            return status_of(e);
        }
        for (int h = 0; h < nparts && st == KUQCD_SUCCESS; ++h)
            st = kq_spinor_download(ctx, prec, static_cast<const char *>(b) + h * half,
                                    static_cast<char *>(h_dst) + h * rec_half, host_prec, s);
    }
    if (st == KUQCD_SUCCESS) {
        e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_last_error(std::string("kq_apply_host: ") + cudaGetErrorString(e));
            return status_of(e);
        }
    }
    return st;
}
