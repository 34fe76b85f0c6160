// The HISQ even-odd hopping term for one output site, shared by every kernel that applies it.
//
//   (D v)(x) = sum_mu [ F_mu(x) v(x+mu) + L_mu(x) v(x+3mu) - F_mu(x-mu)^dag v(x-mu) - L_mu(x-3mu)^dag v(x-3mu) ]
//
// with the reference's factors 1/2 and c3 = -1/48 already folded into the device links (dirac_hisq.cpp:464-502,
// dirac_hisq.cpp:40).  Output sites have parity p; neighbours are read from the parity-(1-p) field at their
// checkerboard index, with periodic wrap in every direction (Position::Normalize, space_time.cpp:187-197); the
// backward links live at the neighbour site on the other parity (dirac_hisq.cpp:492,499).
#pragma once
#include "kq_internal.h"
#include "kq_prec.cuh"

namespace kq {

// Periodic coordinate for hops of at most 3 (any extent >= 1, so nt = 1 wraps onto itself as in the reference).
__device__ __forceinline__ int wrap3(int v, int n)
{
    if (n > 3) return v < 0 ? v + n : (v >= n ? v - n : v);
    v %= n;
    return v < 0 ? v + n : v;
}

template <typename T>
__device__ __forceinline__ void mv_add(const T u[18], const T v[6], T acc[6])
{
    // acc += U v, U row-major
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        T re = acc[2 * r], im = acc[2 * r + 1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T ur = u[2 * (c + 3 * r)], ui = u[2 * (c + 3 * r) + 1];
            re += ur * v[2 * c] - ui * v[2 * c + 1];
            im += ur * v[2 * c + 1] + ui * v[2 * c];
        }
        acc[2 * r] = re;
        acc[2 * r + 1] = im;
    }
}

template <typename T>
__device__ __forceinline__ void mdv_sub(const T u[18], const T v[6], T acc[6])
{
    // acc -= U^dag v : (U^dag v)_r = sum_c conj(U_cr) v_c
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        T re = acc[2 * r], im = acc[2 * r + 1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T ur = u[2 * (r + 3 * c)], ui = u[2 * (r + 3 * c) + 1];
            re -= ur * v[2 * c] + ui * v[2 * c + 1];
            im -= ur * v[2 * c + 1] - ui * v[2 * c];
        }
        acc[2 * r] = re;
        acc[2 * r + 1] = im;
    }
}

// Checkerboard coordinates of output site i on parity p.
struct SiteCoord {
    int x, y, z, t, xcb;
};

__device__ __forceinline__ SiteCoord site_coord(const Geom &g, int i, int p)
{
    SiteCoord c;
    int r = i / g.hx;
    c.xcb = i - r * g.hx;
    const int r2 = r / g.n[1];
    c.y = r - r2 * g.n[1];
    c.t = r2 / g.n[2];
    c.z = r2 - c.t * g.n[2];
    c.x = 2 * c.xcb + ((c.y + c.z + c.t + p) & 1);
    return c;
}

// Neighbour checkerboard index for a hop of `hop` in direction dir.
__device__ __forceinline__ int nbr_index(const Geom &g, const SiteCoord &c, int i, int dir, int hop)
{
    switch (dir) {
        case 0: return i - c.xcb + (wrap3(c.x + hop, g.n[0]) >> 1);
        case 1: return i + (wrap3(c.y + hop, g.n[1]) - c.y) * g.sy;
        case 2: return i + (wrap3(c.z + hop, g.n[2]) - c.z) * g.sz;
        default: return i + (wrap3(c.t + hop, g.n[3]) - c.t) * g.st;
    }
}

// One link as type T.  HALF links (LP = 2) come back as raw int16 values: a site's fat-link terms are accumulated
// in units of the fat field's scale, the long-link terms have their spinor multiplied by scale_long / scale_fat
// (6 products instead of 18 on the link), and the sum is scaled once at the end (fold_scale_*).
template <int LP, typename T>
__device__ __forceinline__ void ld_link_fold(const void *base, int pv, int dir, int i, const LinkSet &L, T u[18])
{
    if constexpr (LP == 2) {
        float q[18];
        ld_link_q16(base, pv, dir, i, q);
#pragma unroll
        for (int k = 0; k < 18; ++k) u[k] = (T)q[k];
    } else {
        typename Acc<LP>::T w[18];
        ld_link_any<LP>(base, pv, dir, i, L.scale, L.recon, w);
#pragma unroll
        for (int k = 0; k < 18; ++k) u[k] = (T)w[k];
    }
}

template <int LP, typename T>
__device__ __forceinline__ T fold_scale_long(const LinkSet &fat, const LinkSet &lng)
{
    return LP == 2 ? (T)(lng.scale / fat.scale) : T(1);
}

template <int LP, typename T>
__device__ __forceinline__ void fold_scale_site(const LinkSet &fat, T acc[6])
{
    if constexpr (LP == 2) {
        const T s = (T)(fat.scale * (1.0f / 32767.0f));
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] *= s;
    }
}

template <int LP, typename T>
__device__ __forceinline__ void fold_long_spinor(T rl, T v[6])
{
    if constexpr (LP == 2) {
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] *= rl;
    }
}

// Accumulation type of a (link precision, spinor precision) pair: double only when both are FP64.
template <int LP, int SP> struct Acc2 { using T = float; };
template <> struct Acc2<0, 0> { using T = double; };

// acc = (D src)(i) for output parity p.  src is the parity-(1-p) field.  Links in precision LP, spinors in SP.
template <int LP, int SP>
__device__ __forceinline__ void dslash_site2(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                             const void *src, int p, int i, typename Acc2<LP, SP>::T acc[6])
{
    using T = typename Acc2<LP, SP>::T;
    static_assert(sizeof(typename Acc<LP>::T) == sizeof(T) && sizeof(typename Acc<SP>::T) == sizeof(T),
                  "FP64 links go with FP64 spinors");
    const SiteCoord c = site_coord(g, i, p);
    // select parity planes without indexing the parameter arrays dynamically (keeps them out of local memory)
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const T rl = fold_scale_long<LP, T>(fat, lng);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        const int nf1 = nbr_index(g, c, i, dir, 1);
        const int nf3 = nbr_index(g, c, i, dir, 3);
        const int nb1 = nbr_index(g, c, i, dir, -1);
        const int nb3 = nbr_index(g, c, i, dir, -3);
        T u[18], v[6];
        ld_link_fold<LP>(fat_p, pv, dir, i, fat, u);
        ld_spinor<SP>(src, pv, nf1, v);
        mv_add(u, v, acc);
        ld_link_fold<LP>(lng_p, pv, dir, i, lng, u);
        ld_spinor<SP>(src, pv, nf3, v);
        fold_long_spinor<LP>(rl, v);
        mv_add(u, v, acc);
        ld_link_fold<LP>(fat_q, pv, dir, nb1, fat, u);
        ld_spinor<SP>(src, pv, nb1, v);
        mdv_sub(u, v, acc);
        ld_link_fold<LP>(lng_q, pv, dir, nb3, lng, u);
        ld_spinor<SP>(src, pv, nb3, v);
        fold_long_spinor<LP>(rl, v);
        mdv_sub(u, v, acc);
    }
    fold_scale_site<LP>(fat, acc);
}

template <int P>
__device__ __forceinline__ void dslash_site(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                            const void *src, int p, int i, typename Acc<P>::T acc[6])
{
    dslash_site2<P, P>(g, pv, fat, lng, src, p, i, acc);
}

// General form: links in LP, input spinors stored in SP, arithmetic in T (double only for FP64 links).
// Used where a sloppy operator reads an FP64 vector (the inexact-matvec phases of the multishift solver).
template <int LP, int SP, typename T>
__device__ __forceinline__ void dslash_site_t(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                              const void *src, int p, int i, T acc[6])
{
    const SiteCoord c = site_coord(g, i, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const T rl = fold_scale_long<LP, T>(fat, lng);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        const int nf1 = nbr_index(g, c, i, dir, 1);
        const int nf3 = nbr_index(g, c, i, dir, 3);
        const int nb1 = nbr_index(g, c, i, dir, -1);
        const int nb3 = nbr_index(g, c, i, dir, -3);
        T u[18], v[6];
        ld_link_fold<LP>(fat_p, pv, dir, i, fat, u);
        ld_spinor_as<SP>(src, pv, nf1, v);
        mv_add(u, v, acc);
        ld_link_fold<LP>(lng_p, pv, dir, i, lng, u);
        ld_spinor_as<SP>(src, pv, nf3, v);
        fold_long_spinor<LP>(rl, v);
        mv_add(u, v, acc);
        ld_link_fold<LP>(fat_q, pv, dir, nb1, fat, u);
        ld_spinor_as<SP>(src, pv, nb1, v);
        mdv_sub(u, v, acc);
        ld_link_fold<LP>(lng_q, pv, dir, nb3, lng, u);
        ld_spinor_as<SP>(src, pv, nb3, v);
        fold_long_spinor<LP>(rl, v);
        mdv_sub(u, v, acc);
    }
    fold_scale_site<LP>(fat, acc);
}

// Multi-RHS form: the links of site i are loaded once and applied to R right-hand sides whose fields are
// src0 + sys[r] * stride (sys[r] < 0: slot unused).  acc[r] receives (D src_r)(i).
template <int LP, int SP, int R>
__device__ __forceinline__ void dslash_site_mrhs(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                                 const char *src0, size_t stride, const int sys[R], int p, int i,
                                                 typename Acc2<LP, SP>::T acc[R][6])
{
    using T = typename Acc2<LP, SP>::T;
    const SiteCoord c = site_coord(g, i, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const T rl = fold_scale_long<LP, T>(fat, lng);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[r][k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        const int nf1 = nbr_index(g, c, i, dir, 1);
        const int nf3 = nbr_index(g, c, i, dir, 3);
        const int nb1 = nbr_index(g, c, i, dir, -1);
        const int nb3 = nbr_index(g, c, i, dir, -3);
        T u[18], v[6];
        ld_link_fold<LP>(fat_p, pv, dir, i, fat, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                ld_spinor<SP>(src0 + sys[r] * stride, pv, nf1, v);
                mv_add(u, v, acc[r]);
            }
        ld_link_fold<LP>(lng_p, pv, dir, i, lng, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                ld_spinor<SP>(src0 + sys[r] * stride, pv, nf3, v);
                fold_long_spinor<LP>(rl, v);
                mv_add(u, v, acc[r]);
            }
        ld_link_fold<LP>(fat_q, pv, dir, nb1, fat, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                ld_spinor<SP>(src0 + sys[r] * stride, pv, nb1, v);
                mdv_sub(u, v, acc[r]);
            }
        ld_link_fold<LP>(lng_q, pv, dir, nb3, lng, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (sys[r] >= 0) {
                ld_spinor<SP>(src0 + sys[r] * stride, pv, nb3, v);
                fold_long_spinor<LP>(rl, v);
                mdv_sub(u, v, acc[r]);
            }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) fold_scale_site<LP>(fat, acc[r]);
}

// Multi-RHS form with the input fields in any storage precision SP and arithmetic in T (the batched solver's
// grouped systems: R systems on one gauge field, fields at src0 + r * stride).  The links of site i are loaded
// once per call and applied to every right-hand side r with use & (1 << r).
template <int LP, int SP, typename T, int R>
__device__ __forceinline__ void dslash_site_mrhs_t(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                                   const char *src0, size_t stride, unsigned use, int p, int i,
                                                   T acc[R][6])
{
    const SiteCoord c = site_coord(g, i, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const T rl = fold_scale_long<LP, T>(fat, lng);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[r][k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        const int nf1 = nbr_index(g, c, i, dir, 1);
        const int nf3 = nbr_index(g, c, i, dir, 3);
        const int nb1 = nbr_index(g, c, i, dir, -1);
        const int nb3 = nbr_index(g, c, i, dir, -3);
        T u[18], v[6];
        ld_link_fold<LP>(fat_p, pv, dir, i, fat, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                ld_spinor_as<SP>(src0 + r * stride, pv, nf1, v);
                mv_add(u, v, acc[r]);
            }
        ld_link_fold<LP>(lng_p, pv, dir, i, lng, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                ld_spinor_as<SP>(src0 + r * stride, pv, nf3, v);
                fold_long_spinor<LP>(rl, v);
                mv_add(u, v, acc[r]);
            }
        ld_link_fold<LP>(fat_q, pv, dir, nb1, fat, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                ld_spinor_as<SP>(src0 + r * stride, pv, nb1, v);
                mdv_sub(u, v, acc[r]);
            }
        ld_link_fold<LP>(lng_q, pv, dir, nb3, lng, u);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                ld_spinor_as<SP>(src0 + r * stride, pv, nb3, v);
                fold_long_spinor<LP>(rl, v);
                mdv_sub(u, v, acc[r]);
            }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) fold_scale_site<LP>(fat, acc[r]);
}

// ------------------------------------------------------------------------------------------------ reductions
// Deterministic block sum of a double (fixed shuffle tree, then warp 0 over the per-warp sums).
__device__ __forceinline__ double block_sum(double v, double *smem32)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) smem32[w] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? smem32[threadIdx.x] : 0.0;
    if (w == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;  // valid in thread 0
}

// Publish this block's partial sum; returns true in the 32 threads of warp 0 of the last block to arrive, each
// holding in *total the fixed-order sum of all partials.  Every block calls this unconditionally.
__device__ __forceinline__ bool grid_sum_last_warp(double v, double *partials, unsigned *ticket, double *smem32,
                                                   double *total)
{
    __shared__ bool am_last;
    v = block_sum(v, smem32);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = v;
        __threadfence();
        const unsigned t = atomicAdd(ticket, 1u);
        am_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) s += *((volatile double *)partials + b);
    s = block_sum(s, smem32);
    if (threadIdx.x >= 32) return false;
    *total = __shfl_sync(0xffffffffu, s, 0);
    if (threadIdx.x == 0) *ticket = 0u;
    return true;
}

// As grid_sum_last_warp, but true in exactly one thread (thread 0 of the last block).
__device__ __forceinline__ bool grid_sum_last(double v, double *partials, unsigned *ticket, double *smem32,
                                              double *total)
{
    return grid_sum_last_warp(v, partials, ticket, smem32, total) && threadIdx.x == 0;
}

}  // namespace kq
