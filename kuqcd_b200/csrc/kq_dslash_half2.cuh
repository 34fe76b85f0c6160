// HALF dslash, two output sites per thread with packed FP32 arithmetic (sm_100's f32x2 FMA / add / mul).
//
// The HALF kernel moves only 608 B per site, and decoding its int16 links and spinors plus the 36 FMAs of every
// 3x3 complex mat-vec give it as many instructions as the FP64 kernel with a third of the bytes: its instruction
// issue competes with its memory time.  Here every thread computes the sites i and i + BS of its block: the two
// sites' values sit side by side in 64-bit register pairs and one f32x2 instruction does the work of two FP32 ones
// (mat-vec FMAs, the int16 bias subtraction, the spinor norm products).  The arithmetic per site is that of the
// one-site kernel (dslash_site2<2,2>: the same int16 decode, the per-field link scales folded out, FP32 sums); the
// backward hops enter with their spinor negated in the decode, so one accumulator serves all sixteen terms.
#pragma once
#include "kq_dslash_core.cuh"

namespace kq {
namespace h2 {

typedef unsigned long long f2;  // two floats: low half = site 0, high half = site 1

__device__ __forceinline__ f2 pack(float lo, float hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ f2 pack_bits(unsigned lo, unsigned hi)
{
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "r"(lo), "r"(hi));
    return r;
}
__device__ __forceinline__ void unpack(f2 v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c)
{
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b)
{
    f2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b)
{
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b)
{
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}

// int16 -> float for a pair of words (the exact bias trick of kq_prec.cuh, i16_to_f): the biased values of the two
// sites go into one register pair and a single f32x2 add removes the bias from both
constexpr float kBias = 8421376.0f;  // 2^23 + 32768
__device__ __forceinline__ f2 q_lo(int w0, int w1)
{
    const unsigned a = 0x4B000000u | (((unsigned)w0 & 0xffffu) ^ 0x8000u);
    const unsigned b = 0x4B000000u | (((unsigned)w1 & 0xffffu) ^ 0x8000u);
    return sub2(pack_bits(a, b), pack(kBias, kBias));
}
__device__ __forceinline__ f2 q_hi(int w0, int w1)
{
    const unsigned a = 0x4B000000u | (((unsigned)w0 >> 16) ^ 0x8000u);
    const unsigned b = 0x4B000000u | (((unsigned)w1 >> 16) ^ 0x8000u);
    return sub2(pack_bits(a, b), pack(kBias, kBias));
}

// raw int16 link of site i0 (lanes lo) and i1 (lanes hi) of one direction: u[2 (col + 3 row) + reim]
__device__ __forceinline__ void ld_link_pair(const void *par_base, int pv, int dir, int i0, int i1, f2 u[18])
{
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 36 * pv;
    const int4 *b4 = reinterpret_cast<const int4 *>(d);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int4 w0 = ld_stream(b4 + (size_t)k * pv + i0), w1 = ld_stream(b4 + (size_t)k * pv + i1);
        u[8 * k + 0] = q_lo(w0.x, w1.x); u[8 * k + 1] = q_hi(w0.x, w1.x);
        u[8 * k + 2] = q_lo(w0.y, w1.y); u[8 * k + 3] = q_hi(w0.y, w1.y);
        u[8 * k + 4] = q_lo(w0.z, w1.z); u[8 * k + 5] = q_hi(w0.z, w1.z);
        u[8 * k + 6] = q_lo(w0.w, w1.w); u[8 * k + 7] = q_hi(w0.w, w1.w);
    }
    const int *b1 = reinterpret_cast<const int *>(d + (size_t)32 * pv);
    const int w0 = ld_stream(b1 + i0), w1 = ld_stream(b1 + i1);
    u[16] = q_lo(w0, w1);
    u[17] = q_hi(w0, w1);
}

// HALF spinors of sites n0, n1: v = q * norm / 32767 times `extra` (the long-link scale ratio; negative for the
// backward hops, whose terms are subtracted); w: the three components that enter the mat-vec with the other sign
// (-imaginary parts for U v, -real parts for U^dag v)
template <bool ADJ>
__device__ __forceinline__ void ld_spinor_pair(const void *base, int n0, int n1, f2 extra, f2 v[6], f2 w[3])
{
    const int4 a = __ldg(static_cast<const int4 *>(base) + n0), b = __ldg(static_cast<const int4 *>(base) + n1);
    const f2 s = mul2(pack(__int_as_float(a.w), __int_as_float(b.w)), extra);
    v[0] = mul2(q_lo(a.x, b.x), s); v[1] = mul2(q_hi(a.x, b.x), s);
    v[2] = mul2(q_lo(a.y, b.y), s); v[3] = mul2(q_hi(a.y, b.y), s);
    v[4] = mul2(q_lo(a.z, b.z), s); v[5] = mul2(q_hi(a.z, b.z), s);
    const f2 m1 = pack(-1.f, -1.f);
#pragma unroll
    for (int c = 0; c < 3; ++c) w[c] = mul2(v[2 * c + (ADJ ? 0 : 1)], m1);
}

// acc += U v   (re += ur vr - ui vi, im += ur vi + ui vr); w = -vi
__device__ __forceinline__ void mv_add2(const f2 u[18], const f2 v[6], const f2 w[3], f2 acc[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const f2 ur = u[2 * (c + 3 * r)], ui = u[2 * (c + 3 * r) + 1];
            acc[2 * r] = fma2(ur, v[2 * c], acc[2 * r]);
            acc[2 * r] = fma2(ui, w[c], acc[2 * r]);
            acc[2 * r + 1] = fma2(ur, v[2 * c + 1], acc[2 * r + 1]);
            acc[2 * r + 1] = fma2(ui, v[2 * c], acc[2 * r + 1]);
        }
}

// acc += U^dag v   ((U^dag v)_r = sum_c conj(U_cr) v_c: re += ur vr + ui vi, im += ur vi - ui vr); w = -vr.
// The backward hops come with v already negated, so this adds -U^dag v_true into the one accumulator.
__device__ __forceinline__ void mdv_add2(const f2 u[18], const f2 v[6], const f2 w[3], f2 acc[6])
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const f2 ur = u[2 * (r + 3 * c)], ui = u[2 * (r + 3 * c) + 1];
            acc[2 * r] = fma2(ur, v[2 * c], acc[2 * r]);
            acc[2 * r] = fma2(ui, v[2 * c + 1], acc[2 * r]);
            acc[2 * r + 1] = fma2(ur, v[2 * c + 1], acc[2 * r + 1]);
            acc[2 * r + 1] = fma2(ui, w[c], acc[2 * r + 1]);
        }
}

}  // namespace h2

// dst = D src on HALF fields, sites i0 = block * 2 BS + t and i1 = i0 + BS (i1 past the end: computed on i0's
// neighbours and not stored)
template <int BS, int MINB>
__global__ void __launch_bounds__(BS, MINB) dslash_half2_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const void *__restrict__ src, void *__restrict__ dst, int p)
{
    using namespace h2;
    const int i0 = blockIdx.x * 2 * BS + threadIdx.x;
    if (i0 >= g.vh) return;
    const int i1r = i0 + BS;
    const bool two = i1r < g.vh;
    const int i1 = two ? i1r : i0;
    const SiteCoord c0 = site_coord(g, i0, p), c1 = site_coord(g, i1, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    // spinor values come as q * norm / 32767; the long-link terms carry scale_long / scale_fat in the spinor
    // (the link values stay raw int16 and the fat scale is applied once at the end)
    const float inv = 1.0f / 32767.0f, rl = lng.scale / fat.scale;
    const f2 e_fat = pack(inv, inv), e_lng = pack(inv * rl, inv * rl);
    const f2 n_fat = pack(-inv, -inv), n_lng = pack(-inv * rl, -inv * rl);  // backward hops: subtracted
    f2 acc[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = pack(0.f, 0.f);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        f2 u[18], v[6], w[3];
        ld_link_pair(fat_p, pv, dir, i0, i1, u);
        ld_spinor_pair<false>(src, nbr_index(g, c0, i0, dir, 1), nbr_index(g, c1, i1, dir, 1), e_fat, v, w);
        mv_add2(u, v, w, acc);
        ld_link_pair(lng_p, pv, dir, i0, i1, u);
        ld_spinor_pair<false>(src, nbr_index(g, c0, i0, dir, 3), nbr_index(g, c1, i1, dir, 3), e_lng, v, w);
        mv_add2(u, v, w, acc);
        const int b10 = nbr_index(g, c0, i0, dir, -1), b11 = nbr_index(g, c1, i1, dir, -1);
        ld_link_pair(fat_q, pv, dir, b10, b11, u);
        ld_spinor_pair<true>(src, b10, b11, n_fat, v, w);
        mdv_add2(u, v, w, acc);
        const int b30 = nbr_index(g, c0, i0, dir, -3), b31 = nbr_index(g, c1, i1, dir, -3);
        ld_link_pair(lng_q, pv, dir, b30, b31, u);
        ld_spinor_pair<true>(src, b30, b31, n_lng, v, w);
        mdv_add2(u, v, w, acc);
    }
    const float sf = fat.scale * inv;
    const f2 s2 = pack(sf, sf);
    float o0[6], o1[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) unpack(mul2(acc[k], s2), o0[k], o1[k]);
    st_spinor<2>(dst, pv, i0, o0);
    if (two) st_spinor<2>(dst, pv, i1, o1);
}

}  // namespace kq
