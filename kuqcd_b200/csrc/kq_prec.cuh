// Per-precision storage access for device spinor and link fields (layouts in kq_internal.h).
// All field planes are strided by `pv`, the padded per-parity site count (a multiple of 64), so every plane
// starts on a 1 KiB boundary and every vector load is naturally aligned.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace kq {

constexpr int kPad = 64;
__host__ __device__ inline int pad_sites(int vh) { return (vh + kPad - 1) / kPad * kPad; }

// ------------------------------------------------------------------------------------------------ load helpers
// Links are read once per dslash: stream them (evict-first) so the L2 keeps the re-read spinor neighbours.
__device__ __forceinline__ double2 ld_stream(const double2 *p) { return __ldcs(p); }
__device__ __forceinline__ float4 ld_stream(const float4 *p) { return __ldcs(p); }
__device__ __forceinline__ float2 ld_stream(const float2 *p) { return __ldcs(p); }
__device__ __forceinline__ int4 ld_stream(const int4 *p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }

// int16 fixed point: q = rint(v * 32767 / scale)
// int16 -> float without the int-to-float conversion unit: flipping the sign bit of q gives q + 32768 in
// [0, 65535]; placed in the mantissa of 2^23 it is the float 2^23 + q + 32768, and subtracting 2^23 + 32768 leaves q
// exactly (both operands are integers below 2^24).  One logic op and one float add per value, both full rate; the
// results equal (float)(short) bit for bit.
__device__ __forceinline__ float i16_to_f(unsigned biased16)
{
    return __uint_as_float(0x4B000000u | biased16) - 8421376.0f;  // 8421376 = 2^23 + 32768
}
__device__ __forceinline__ float lo16(int w) { return i16_to_f(((unsigned)w & 0xffffu) ^ 0x8000u); }
__device__ __forceinline__ float hi16(int w) { return i16_to_f(((unsigned)w >> 16) ^ 0x8000u); }
__device__ __forceinline__ int pack16(float a, float b)
{
    const int qa = __float2int_rn(a), qb = __float2int_rn(b);
    return (qa & 0xffff) | (qb << 16);
}

// ------------------------------------------------------------------------------------------------ spinors
// Accumulation type: double for FP64, float for FP32 and HALF.
template <int P> struct Acc { using T = float; };
template <> struct Acc<0> { using T = double; };

template <int P> __device__ __forceinline__ void ld_spinor(const void *base, int pv, int i, typename Acc<P>::T v[6]);
template <int P> __device__ __forceinline__ void st_spinor(void *base, int pv, int i, const typename Acc<P>::T v[6]);

template <> __device__ __forceinline__ void ld_spinor<0>(const void *base, int pv, int i, double v[6])
{
    const double2 *b = static_cast<const double2 *>(base);
    const double2 a = __ldg(b + i), c = __ldg(b + pv + i), d = __ldg(b + 2 * pv + i);
    v[0] = a.x; v[1] = a.y; v[2] = c.x; v[3] = c.y; v[4] = d.x; v[5] = d.y;
}
template <> __device__ __forceinline__ void st_spinor<0>(void *base, int pv, int i, const double v[6])
{
    double2 *b = static_cast<double2 *>(base);
    b[i] = make_double2(v[0], v[1]);
    b[pv + i] = make_double2(v[2], v[3]);
    b[2 * pv + i] = make_double2(v[4], v[5]);
}

template <> __device__ __forceinline__ void ld_spinor<1>(const void *base, int pv, int i, float v[6])
{
    const float4 a = __ldg(static_cast<const float4 *>(base) + i);
    const float2 c = __ldg(reinterpret_cast<const float2 *>(static_cast<const float4 *>(base) + pv) + i);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = c.x; v[5] = c.y;
}
template <> __device__ __forceinline__ void st_spinor<1>(void *base, int pv, int i, const float v[6])
{
    static_cast<float4 *>(base)[i] = make_float4(v[0], v[1], v[2], v[3]);
    reinterpret_cast<float2 *>(static_cast<float4 *>(base) + pv)[i] = make_float2(v[4], v[5]);
}

// HALF spinor: int4 {c0.re|c0.im, c1.re|c1.im, c2.re|c2.im, float norm}, value = q * norm / 32767
template <> __device__ __forceinline__ void ld_spinor<2>(const void *base, int pv, int i, float v[6])
{
    (void)pv;
    const int4 w = __ldg(static_cast<const int4 *>(base) + i);
    const float s = __int_as_float(w.w) * (1.0f / 32767.0f);
    v[0] = lo16(w.x) * s; v[1] = hi16(w.x) * s;
    v[2] = lo16(w.y) * s; v[3] = hi16(w.y) * s;
    v[4] = lo16(w.z) * s; v[5] = hi16(w.z) * s;
}
template <> __device__ __forceinline__ void st_spinor<2>(void *base, int pv, int i, const float v[6])
{
    (void)pv;
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) m = fmaxf(m, fabsf(v[k]));
    const float inv = m > 0.f ? 32767.0f / m : 0.f;
    int4 w;
    w.x = pack16(v[0] * inv, v[1] * inv);
    w.y = pack16(v[2] * inv, v[3] * inv);
    w.z = pack16(v[4] * inv, v[5] * inv);
    w.w = __float_as_int(m);
    static_cast<int4 *>(base)[i] = w;
}

// load / store a spinor of storage precision P into / from registers of any floating type T
template <int P, typename T>
__device__ __forceinline__ void ld_spinor_as(const void *base, int pv, int i, T v[6])
{
    typename Acc<P>::T w[6];
    ld_spinor<P>(base, pv, i, w);
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = (T)w[k];
}
template <int P, typename T>
__device__ __forceinline__ void st_spinor_as(void *base, int pv, int i, const T v[6])
{
    typename Acc<P>::T w[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = (typename Acc<P>::T)v[k];
    st_spinor<P>(base, pv, i, w);
}

// ------------------------------------------------------------------------------------------------ links
// One 3x3 complex matrix, row-major u[2*(col + 3*row)] (re, im).
// FP64: 9 double2 planes per direction.     dir stride = 9 * pv double2
// FP32: 4 float4 planes + 1 float2 plane.   dir stride = 72 * pv bytes
// HALF: 2 int4 planes + 1 int plane.        dir stride = 36 * pv bytes
template <int P> struct LinkBytes;
template <> struct LinkBytes<0> { static constexpr int v = 144; };
template <> struct LinkBytes<1> { static constexpr int v = 72; };
template <> struct LinkBytes<2> { static constexpr int v = 36; };

template <int P>
__device__ __forceinline__ void ld_link(const void *par_base, int pv, int dir, int i, float scale,
                                        typename Acc<P>::T u[18]);

template <> __device__ __forceinline__ void ld_link<0>(const void *par_base, int pv, int dir, int i, float scale,
                                                       double u[18])
{
    (void)scale;
    const double2 *b = static_cast<const double2 *>(par_base) + (size_t)dir * 9 * pv + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double2 w = ld_stream(b + (size_t)k * pv);
        u[2 * k] = w.x;
        u[2 * k + 1] = w.y;
    }
}

template <> __device__ __forceinline__ void ld_link<1>(const void *par_base, int pv, int dir, int i, float scale,
                                                       float u[18])
{
    (void)scale;
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 72 * pv;
    const float4 *b4 = reinterpret_cast<const float4 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float4 w = ld_stream(b4 + (size_t)k * pv);
        u[4 * k] = w.x; u[4 * k + 1] = w.y; u[4 * k + 2] = w.z; u[4 * k + 3] = w.w;
    }
    const float2 w = ld_stream(reinterpret_cast<const float2 *>(d + (size_t)64 * pv) + i);
    u[16] = w.x;
    u[17] = w.y;
}

template <> __device__ __forceinline__ void ld_link<2>(const void *par_base, int pv, int dir, int i, float scale,
                                                       float u[18])
{
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 36 * pv;
    const int4 *b4 = reinterpret_cast<const int4 *>(d) + i;
    const float s = scale * (1.0f / 32767.0f);
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int4 w = ld_stream(b4 + (size_t)k * pv);
        u[8 * k + 0] = lo16(w.x) * s; u[8 * k + 1] = hi16(w.x) * s;
        u[8 * k + 2] = lo16(w.y) * s; u[8 * k + 3] = hi16(w.y) * s;
        u[8 * k + 4] = lo16(w.z) * s; u[8 * k + 5] = hi16(w.z) * s;
        u[8 * k + 6] = lo16(w.w) * s; u[8 * k + 7] = hi16(w.w) * s;
    }
    const int w = ld_stream(reinterpret_cast<const int *>(d + (size_t)32 * pv) + i);
    u[16] = lo16(w) * s;
    u[17] = hi16(w) * s;
}

// HALF link as raw int16 values (the per-field scale is applied by the caller, once per site)
__device__ __forceinline__ void ld_link_q16(const void *par_base, int pv, int dir, int i, float u[18])
{
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 36 * pv;
    const int4 *b4 = reinterpret_cast<const int4 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int4 w = ld_stream(b4 + (size_t)k * pv);
        u[8 * k + 0] = lo16(w.x); u[8 * k + 1] = hi16(w.x);
        u[8 * k + 2] = lo16(w.y); u[8 * k + 3] = hi16(w.y);
        u[8 * k + 4] = lo16(w.z); u[8 * k + 5] = hi16(w.z);
        u[8 * k + 6] = lo16(w.w); u[8 * k + 7] = hi16(w.w);
    }
    const int w = ld_stream(reinterpret_cast<const int *>(d + (size_t)32 * pv) + i);
    u[16] = lo16(w);
    u[17] = hi16(w);
}

// store one link (used by the layout-conversion kernels)
template <int P>
__device__ __forceinline__ void st_link(void *par_base, int pv, int dir, int i, float scale, const double u[18]);

template <> __device__ __forceinline__ void st_link<0>(void *par_base, int pv, int dir, int i, float scale,
                                                       const double u[18])
{
    (void)scale;
    double2 *b = static_cast<double2 *>(par_base) + (size_t)dir * 9 * pv + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) b[(size_t)k * pv] = make_double2(u[2 * k], u[2 * k + 1]);
}
template <> __device__ __forceinline__ void st_link<1>(void *par_base, int pv, int dir, int i, float scale,
                                                       const double u[18])
{
    (void)scale;
    char *d = static_cast<char *>(par_base) + (size_t)dir * 72 * pv;
    float4 *b4 = reinterpret_cast<float4 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        b4[(size_t)k * pv] = make_float4((float)u[4 * k], (float)u[4 * k + 1], (float)u[4 * k + 2], (float)u[4 * k + 3]);
    reinterpret_cast<float2 *>(d + (size_t)64 * pv)[i] = make_float2((float)u[16], (float)u[17]);
}
template <> __device__ __forceinline__ void st_link<2>(void *par_base, int pv, int dir, int i, float scale,
                                                       const double u[18])
{
    char *d = static_cast<char *>(par_base) + (size_t)dir * 36 * pv;
    int4 *b4 = reinterpret_cast<int4 *>(d) + i;
    const double inv = scale > 0.f ? 32767.0 / (double)scale : 0.0;
    float q[18];
#pragma unroll
    for (int k = 0; k < 18; ++k) q[k] = (float)(u[k] * inv);
#pragma unroll
    for (int k = 0; k < 2; ++k)
        b4[(size_t)k * pv] = make_int4(pack16(q[8 * k], q[8 * k + 1]), pack16(q[8 * k + 2], q[8 * k + 3]),
                                       pack16(q[8 * k + 4], q[8 * k + 5]), pack16(q[8 * k + 6], q[8 * k + 7]));
    reinterpret_cast<int *>(d + (size_t)32 * pv)[i] = pack16(q[16], q[17]);
}

// ------------------------------------------------------------------------------------------------ compressed links
// L = s W with W in SU(3) (s real): rows 0 and 1 of L and 1/s are stored; row 2 = conj(row0 x row1) / s.
// FP64: 6 double2 planes + 1 double plane per direction (104 B per link); FP32: 3 float4 + 1 float (52 B).
template <typename T>
__device__ __forceinline__ void rebuild_row2(T u[18], T inv_s)
{
    // (a x b)_c = a_{c+1} b_{c+2} - a_{c+2} b_{c+1}; row 2 = conj(a x b) * inv_s with a = row 0, b = row 1
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        const T ar1 = u[2 * c1], ai1 = u[2 * c1 + 1], ar2 = u[2 * c2], ai2 = u[2 * c2 + 1];
        const T br1 = u[6 + 2 * c1], bi1 = u[6 + 2 * c1 + 1], br2 = u[6 + 2 * c2], bi2 = u[6 + 2 * c2 + 1];
        const T re = (ar1 * br2 - ai1 * bi2) - (ar2 * br1 - ai2 * bi1);
        const T im = (ar1 * bi2 + ai1 * br2) - (ar2 * bi1 + ai2 * br1);
        u[12 + 2 * c] = re * inv_s;
        u[12 + 2 * c + 1] = -im * inv_s;
    }
}

template <int P>
__device__ __forceinline__ void ld_link_recon(const void *par_base, int pv, int dir, int i,
                                              typename Acc<P>::T u[18]);

template <> __device__ __forceinline__ void ld_link_recon<0>(const void *par_base, int pv, int dir, int i, double u[18])
{
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 104 * pv;
    const double2 *b = reinterpret_cast<const double2 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const double2 w = ld_stream(b + (size_t)k * pv);
        u[2 * k] = w.x;
        u[2 * k + 1] = w.y;
    }
    rebuild_row2(u, __ldcs(reinterpret_cast<const double *>(d + (size_t)96 * pv) + i));
}

template <> __device__ __forceinline__ void ld_link_recon<1>(const void *par_base, int pv, int dir, int i, float u[18])
{
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * 52 * pv;
    const float4 *b4 = reinterpret_cast<const float4 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 w = ld_stream(b4 + (size_t)k * pv);
        u[4 * k] = w.x; u[4 * k + 1] = w.y; u[4 * k + 2] = w.z; u[4 * k + 3] = w.w;
    }
    rebuild_row2(u, __ldcs(reinterpret_cast<const float *>(d + (size_t)48 * pv) + i));
}

template <> __device__ __forceinline__ void ld_link_recon<2>(const void *, int, int, int, float u[18])
{
#pragma unroll
    for (int k = 0; k < 18; ++k) u[k] = 0.f;  // HALF links are never stored compressed
}

// any storage of a LinkSet: full (recon = 0) or compressed
template <int P>
__device__ __forceinline__ void ld_link_any(const void *par_base, int pv, int dir, int i, float scale, int recon,
                                            typename Acc<P>::T u[18])
{
    if (P != 2 && recon) ld_link_recon<P>(par_base, pv, dir, i, u);
    else ld_link<P>(par_base, pv, dir, i, scale, u);
}

// store rows 0, 1 and inv_s of one link in the compressed layout
template <int P>
__device__ __forceinline__ void st_link_recon(void *par_base, int pv, int dir, int i, const double u[18], double inv_s);

template <> __device__ __forceinline__ void st_link_recon<0>(void *par_base, int pv, int dir, int i, const double u[18],
                                                             double inv_s)
{
    char *d = static_cast<char *>(par_base) + (size_t)dir * 104 * pv;
    double2 *b = reinterpret_cast<double2 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 6; ++k) b[(size_t)k * pv] = make_double2(u[2 * k], u[2 * k + 1]);
    reinterpret_cast<double *>(d + (size_t)96 * pv)[i] = inv_s;
}

template <> __device__ __forceinline__ void st_link_recon<1>(void *par_base, int pv, int dir, int i, const double u[18],
                                                             double inv_s)
{
    char *d = static_cast<char *>(par_base) + (size_t)dir * 52 * pv;
    float4 *b4 = reinterpret_cast<float4 *>(d) + i;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        b4[(size_t)k * pv] = make_float4((float)u[4 * k], (float)u[4 * k + 1], (float)u[4 * k + 2], (float)u[4 * k + 3]);
    reinterpret_cast<float *>(d + (size_t)48 * pv)[i] = (float)inv_s;
}

}  // namespace kq
