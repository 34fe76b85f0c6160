// Stand-alone HISQ even-odd dslash kernels: dst = D src, and s = sigma*p - D src (the second half of
// sigma - D_pq D_qp, MdaggM + Axmy of inverter_cgm.cpp:45-46).  One thread per output site; links are
// streamed from HBM once, neighbour spinors come through L1/L2.  Link and spinor precisions are independent
// template parameters (FP64/FP64, FP32/FP32, HALF/HALF, HALF links with FP32 spinors).
#include <cstdlib>
#include <cstring>

#include "kq_dslash_core.cuh"
#include "kq_dslash_half2.cuh"

namespace kq {

template <int LP, int SP>
__global__ void __launch_bounds__(256) dslash_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, const void *__restrict__ src,
                                                     void *__restrict__ dst, int p, const int *__restrict__ gate)
{
    if (gate && *gate == 0) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    typename Acc2<LP, SP>::T acc[6];
    dslash_site2<LP, SP>(g, pv, fat, lng, src, p, i, acc);
    st_spinor<SP>(dst, pv, i, acc);
}

// s = sigma * pvec - D src   (pvec, s on parity p)
template <int LP, int SP>
__global__ void __launch_bounds__(256) dslash_xmy_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                         const void *__restrict__ src, const void *__restrict__ pvec,
                                                         void *__restrict__ s, int p, double sigma)
{
    using T = typename Acc2<LP, SP>::T;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    T acc[6], pv6[6];
    dslash_site2<LP, SP>(g, pv, fat, lng, src, p, i, acc);
    ld_spinor<SP>(pvec, pv, i, pv6);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = (T)sigma * pv6[k] - acc[k];
    st_spinor<SP>(s, pv, i, acc);
}

// Full-lattice (non-preconditioned, KUQCD_HISQ_DIRAC) operator: a full field is the parity-0 field followed by the
// parity-1 field, `half` bytes apart.  blockIdx.y = output parity p; the input is the other half.  dst = D src on
// both parities in one launch (dirac_hisq.cpp:128-136, 418-424 with offseti = offsetg = 0), or, with pvec,
// dst = sigma * pvec - D src (the second half of sigma - D D).
template <int LP, int SP>
__global__ void __launch_bounds__(256) dslash_full_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const char *__restrict__ src, const char *__restrict__ pvec,
                                                          char *__restrict__ dst, size_t half, double sigma)
{
    using T = typename Acc2<LP, SP>::T;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.vh) return;
    const int p = blockIdx.y;
    T acc[6];
    dslash_site2<LP, SP>(g, pv, fat, lng, src + (1 - p) * half, p, i, acc);
    if (pvec) {
        T pv6[6];
        ld_spinor<SP>(pvec + p * half, pv, i, pv6);
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] = (T)sigma * pv6[k] - acc[k];
    }
    st_spinor<SP>(dst + p * half, pv, i, acc);
}

// HALF kernel: 0 one site per thread, 4 .. 7 two sites per thread in packed FP32 with 4 .. 7 resident 128-thread
// CTAs per SM (KUQCD_HALF_DSLASH = site | pair4 | pair5 | pair6 | pair7).  Default pair7: the kernel is latency-
// bound, and 28 warps per SM at 72 registers (40 B of spills) beat 20 at 96 (48^3x96: 536 against 577 us).
static int half_kernel()
{
    static const int k = [] {
        const char *e = getenv("KUQCD_HALF_DSLASH");
        if (!e) return 7;
        if (e[0] == 's') return 0;
        if (strncmp(e, "pair", 4) == 0 && e[4] >= '4' && e[4] <= '7' && e[5] == 0) return e[4] - '0';
        return 7;
    }();
    return k;
}

static bool pair_ok(int lp, int sp)
{
    return (lp == sp) || (lp == P16 && sp == P32);
}

#define KQ_DISPATCH_PAIR(LPv, SPv, CALL)                                   \
    if (LPv == P64 && SPv == P64) { constexpr int LP = 0, SP = 0; CALL; } \
    else if (LPv == P32 && SPv == P32) { constexpr int LP = 1, SP = 1; CALL; } \
    else if (LPv == P16 && SPv == P16) { constexpr int LP = 2, SP = 2; CALL; } \
    else { constexpr int LP = 2, SP = 1; CALL; }

cudaError_t launch_dslash2(const Geom &g, const GaugeDev &gd, int lp, int sp, const void *src, void *dst,
                           int dst_parity, const int *gate, cudaStream_t s, int block)
{
    if (!gd.have[lp] || !pair_ok(lp, sp)) {
        set_last_error("dslash: links not resident in the requested precision, or unsupported precision pair");
        return cudaErrorInvalidValue;
    }
    const int pv = pad_sites(g.vh);
    if (lp == P16 && sp == P16 && !gate && half_kernel() != 0) {
        // HALF: two sites per thread in packed FP32 (kq_dslash_half2.cuh)
        constexpr int kBS2 = 128;
        const int nb2 = (g.vh + 2 * kBS2 - 1) / (2 * kBS2);
        switch (half_kernel()) {
            case 4: dslash_half2_kernel<kBS2, 4><<<nb2, kBS2, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], src, dst, dst_parity); break;
            case 6: dslash_half2_kernel<kBS2, 6><<<nb2, kBS2, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], src, dst, dst_parity); break;
            case 7: dslash_half2_kernel<kBS2, 7><<<nb2, kBS2, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], src, dst, dst_parity); break;
            default: dslash_half2_kernel<kBS2, 5><<<nb2, kBS2, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], src, dst, dst_parity); break;
        }
        return cudaGetLastError();
    }
    const int bs = block > 0 ? block : 256;
    const int nb = (g.vh + bs - 1) / bs;
    KQ_DISPATCH_PAIR(lp, sp, (dslash_kernel<LP, SP><<<nb, bs, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], src, dst,
                                                                       dst_parity, gate)));
    return cudaGetLastError();
}

cudaError_t launch_dslash(const Geom &g, const GaugeDev &gd, int prec, const void *src, void *dst, int dst_parity,
                          cudaStream_t s, int block)
{
    return launch_dslash2(g, gd, prec, prec, src, dst, dst_parity, nullptr, s, block);
}

cudaError_t launch_dslash_gated(const Geom &g, const GaugeDev &gd, int lp, int sp, const void *src, void *dst,
                                int dst_parity, const int *gate, cudaStream_t s)
{
    return launch_dslash2(g, gd, lp, sp, src, dst, dst_parity, gate, s, 0);
}

cudaError_t launch_mdagm2(const Geom &g, const GaugeDev &gd, int lp, int sp, double sigma, const void *src,
                          void *tmp, void *dst, int parity, cudaStream_t s)
{
    cudaError_t e = launch_dslash2(g, gd, lp, sp, src, tmp, 1 - parity, nullptr, s, 0);
    if (e != cudaSuccess) return e;
    const int bs = 256;
    const int nb = (g.vh + bs - 1) / bs;
    const int pv = pad_sites(g.vh);
    KQ_DISPATCH_PAIR(lp, sp, (dslash_xmy_kernel<LP, SP><<<nb, bs, 0, s>>>(g, pv, gd.fat[lp], gd.lng[lp], tmp, src,
                                                                           dst, parity, sigma)));
    return cudaGetLastError();
}

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s)
{
    return launch_mdagm2(g, gd, prec, prec, sigma, src, tmp, dst, parity, s);
}

// full-lattice fields (2 x spinor_bytes): dst = D src, or dst = sigma * pvec - D src when pvec != nullptr
cudaError_t launch_dslash_full(const Geom &g, const GaugeDev &gd, int prec, const void *src, const void *pvec,
                               void *dst, double sigma, cudaStream_t s)
{
    if (!gd.have[prec]) {
        set_last_error("dslash: links not resident in the requested precision");
        return cudaErrorInvalidValue;
    }
    const dim3 grid((g.vh + 255) / 256, 2);
    const int pv = pad_sites(g.vh);
    const size_t half = spinor_bytes(g, prec);
    auto S = static_cast<const char *>(src);
    auto Pv = static_cast<const char *>(pvec);
    auto D = static_cast<char *>(dst);
    KQ_DISPATCH_PAIR(prec, prec, (dslash_full_kernel<LP, SP><<<grid, 256, 0, s>>>(g, pv, gd.fat[prec], gd.lng[prec],
                                                                                  S, Pv, D, half, sigma)));
    return cudaGetLastError();
}

// dst = sigma src - D D src on full-lattice fields; tmp: one full-lattice field
cudaError_t launch_mdagm_full(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                              void *dst, cudaStream_t s)
{
    cudaError_t e = launch_dslash_full(g, gd, prec, src, nullptr, tmp, 0.0, s);
    if (e != cudaSuccess) return e;
    return launch_dslash_full(g, gd, prec, tmp, src, dst, sigma, s);
}

}  // namespace kq
