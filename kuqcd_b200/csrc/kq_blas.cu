// FP64 true residuals |b - (sigma - D_pq D_qp) x| / |b| on the device (the check the reference never makes,
// inverter_cgm.cpp:71-77 only tracks the recursive residual).
#include <vector>

#include "kq_dslash_core.cuh"

namespace kq {

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s);
cudaError_t launch_mdagm_full(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                              void *dst, cudaStream_t s);

__global__ void __launch_bounds__(256) resid_partials_kernel(int vh, int pv, const void *__restrict__ b,
                                                             const void *__restrict__ s, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double rr = 0.0, bb = 0.0;
    if (i < vh) {
        double bv[6], sv[6];
        ld_spinor<0>(b, pv, i, bv);
        ld_spinor<0>(s, pv, i, sv);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const double d = bv[k] - sv[k];
            rr += d * d;
            bb += bv[k] * bv[k];
        }
    }
    rr = block_sum(rr, sm);
    __syncthreads();
    bb = block_sum(bb, sm);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = rr;
        partials[2 * blockIdx.x + 1] = bb;
    }
}

cudaError_t true_residuals(const Geom &g, const GaugeDev &gd, int parity, int ns, const double *sigma,
                           const void *d_b, const void *d_x, size_t xstride, void *d_tmp, void *d_s, double *partials,
                           double *out, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int nb = (g.vh + 255) / 256;
    std::vector<double> h(2 * (size_t)nb);
    for (int k = 0; k < ns; ++k) {
        const void *xk = static_cast<const char *>(d_x) + k * xstride;
        KQ_CUDA_TRY(launch_mdagm(g, gd, P64, sigma[k], xk, d_tmp, d_s, parity, s));
        resid_partials_kernel<<<nb, 256, 0, s>>>(g.vh, pv, d_b, d_s, partials);
        KQ_CUDA_TRY(cudaGetLastError());
        KQ_CUDA_TRY(cudaMemcpyAsync(h.data(), partials, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        double rr = 0, bb = 0;
        for (int b = 0; b < nb; ++b) {
            rr += h[2 * b];
            bb += h[2 * b + 1];
        }
        out[k] = bb > 0 ? sqrt(rr / bb) : 0.0;
    }
    return cudaSuccess;
}

// Full-lattice fields (parity 0 then parity 1, spinor_bytes apart): |b - (sigma - D D) x| / |b| over both parities.
// d_tmp, d_s: one full-lattice field each; partials: 4 * nb doubles.
cudaError_t true_residuals_full(const Geom &g, const GaugeDev &gd, int ns, const double *sigma, const void *d_b,
                                const void *d_x, size_t xstride, void *d_tmp, void *d_s, double *partials,
                                double *out, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int nb = (g.vh + 255) / 256;
    const size_t half = spinor_bytes(g, P64);
    std::vector<double> h(4 * (size_t)nb);
    for (int k = 0; k < ns; ++k) {
        const void *xk = static_cast<const char *>(d_x) + k * xstride;
        KQ_CUDA_TRY(launch_mdagm_full(g, gd, P64, sigma[k], xk, d_tmp, d_s, s));
        for (int p = 0; p < 2; ++p)
            resid_partials_kernel<<<nb, 256, 0, s>>>(g.vh, pv, static_cast<const char *>(d_b) + p * half,
                                                     static_cast<const char *>(d_s) + p * half, partials + 2 * p * nb);
        KQ_CUDA_TRY(cudaGetLastError());
        KQ_CUDA_TRY(cudaMemcpyAsync(h.data(), partials, sizeof(double) * 4 * nb, cudaMemcpyDeviceToHost, s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        double rr = 0, bb = 0;
        for (int b = 0; b < 2 * nb; ++b) {
            rr += h[2 * b];
            bb += h[2 * b + 1];
        }
        out[k] = bb > 0 ? sqrt(rr / bb) : 0.0;
    }
    return cudaSuccess;
}

// |v|^2 of one FP64 parity field (partials: 2 * nb doubles)
cudaError_t norm2_p64(const Geom &g, const void *v, double *partials, double *out, cudaStream_t s)
{
    const int nb = (g.vh + 255) / 256;
    resid_partials_kernel<<<nb, 256, 0, s>>>(g.vh, pad_sites(g.vh), v, v, partials);  // |v - v|^2, |v|^2
    KQ_CUDA_TRY(cudaGetLastError());
    std::vector<double> h(2 * (size_t)nb);
    KQ_CUDA_TRY(cudaMemcpyAsync(h.data(), partials, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    double bb = 0;
    for (int b = 0; b < nb; ++b) bb += h[2 * b + 1];
    *out = bb;
    return cudaSuccess;
}

}  // namespace kq
