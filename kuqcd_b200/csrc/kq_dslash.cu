// Stand-alone HISQ even-odd dslash kernels: dst = D src, and s = sigma*p - D src (the second half of
// sigma - D_pq D_qp, MdaggM + Axmy of inverter_cgm.cpp:45-46).  One thread per output site; links are
// streamed from HBM once, neighbour spinors come through L1/L2.
#include "kq_dslash_core.cuh"

namespace kq {

template <int P>
__global__ void __launch_bounds__(256) dslash_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const void *__restrict__ src,
                                                     void *__restrict__ dst, int p, const int *__restrict__ gate)
{
    if (gate && *gate == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    typename Acc<P>::T acc[6];
    dslash_site<P>(g, pv, fat, lng, src, p, i, acc);
    st_spinor<P>(dst, pv, i, acc);
}

// s = sigma * pvec - D src   (pvec, s on parity p)
template <int P>
__global__ void __launch_bounds__(256) dslash_xmy_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                         const void *__restrict__ src, const void *__restrict__ pvec,
                                                         void *__restrict__ s, int p, double sigma)
{
    using T = typename Acc<P>::T;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    T acc[6], pv6[6];
    dslash_site<P>(g, pv, fat, lng, src, p, i, acc);
    ld_spinor<P>(pvec, pv, i, pv6);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = (T)sigma * pv6[k] - acc[k];
    st_spinor<P>(s, pv, i, acc);
}

cudaError_t launch_dslash(const Geom &g, const GaugeDev &gd, int prec, const void *src, void *dst, int dst_parity,
                          cudaStream_t s, int block)
{
    if (!gd.have[prec]) {
        set_last_error("dslash: links not resident in the requested precision");
        return cudaErrorInvalidValue;
    }
    const int bs = block > 0 ? block : 256;
    const int nb = (g.vh + bs - 1) / bs;
    const int pv = pad_sites(g.vh);
    switch (prec) {
        case P64: dslash_kernel<0><<<nb, bs, 0, s>>>(g, pv, gd.fat[0], gd.lng[0], src, dst, dst_parity, nullptr); break;
        case P32: dslash_kernel<1><<<nb, bs, 0, s>>>(g, pv, gd.fat[1], gd.lng[1], src, dst, dst_parity, nullptr); break;
        default: dslash_kernel<2><<<nb, bs, 0, s>>>(g, pv, gd.fat[2], gd.lng[2], src, dst, dst_parity, nullptr); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_dslash_gated(const Geom &g, const GaugeDev &gd, int prec, const void *src, void *dst,
                                int dst_parity, const int *gate, cudaStream_t s)
{
    const int bs = 256;
    const int nb = (g.vh + bs - 1) / bs;
    const int pv = pad_sites(g.vh);
    switch (prec) {
        case P64: dslash_kernel<0><<<nb, bs, 0, s>>>(g, pv, gd.fat[0], gd.lng[0], src, dst, dst_parity, gate); break;
        case P32: dslash_kernel<1><<<nb, bs, 0, s>>>(g, pv, gd.fat[1], gd.lng[1], src, dst, dst_parity, gate); break;
        default: dslash_kernel<2><<<nb, bs, 0, s>>>(g, pv, gd.fat[2], gd.lng[2], src, dst, dst_parity, gate); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s)
{
    if (!gd.have[prec]) {
        set_last_error("mdagm: links not resident in the requested precision");
        return cudaErrorInvalidValue;
    }
    cudaError_t e = launch_dslash(g, gd, prec, src, tmp, 1 - parity, s, 0);
    if (e != cudaSuccess) return e;
    const int bs = 256;
    const int nb = (g.vh + bs - 1) / bs;
    const int pv = pad_sites(g.vh);
    switch (prec) {
        case P64: dslash_xmy_kernel<0><<<nb, bs, 0, s>>>(g, pv, gd.fat[0], gd.lng[0], tmp, src, dst, parity, sigma); break;
        case P32: dslash_xmy_kernel<1><<<nb, bs, 0, s>>>(g, pv, gd.fat[1], gd.lng[1], tmp, src, dst, parity, sigma); break;
        default: dslash_xmy_kernel<2><<<nb, bs, 0, s>>>(g, pv, gd.fat[2], gd.lng[2], tmp, src, dst, parity, sigma); break;
    }
    return cudaGetLastError();
}

}  // namespace kq
