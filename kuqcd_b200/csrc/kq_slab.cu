// Domain decomposition along t: one context per rank holds the slab t0 = rank * nt_local .. t0 + nt_local - 1 of
// the global lattice; the dslash's t hops that leave the slab read ghost slices received from the neighbouring
// ranks.  This is the multi-rank path of the reference's dslash (halo pack / exchange / unpack,
// dirac_hisq.cpp:236-407, and the Communicator of communication.cpp:73-138), restated for GPUs: the faces are
// packed by a kernel into the sender's own buffer, the caller moves them (NCCL send/recv over NVLink, or any
// transport), and the dslash reads the received buffers in place -- there is no unpack step.
//
// Geometry.  The local extent nt_local is even and >= 4, so local and global site parities agree and a depth-3
// halo comes from one neighbour.  Every t slice of one parity holds S = nx*ny*nz/2 sites, contiguous in the
// checkerboard index (i = j + S*t, j the index inside the slice), so a face of 3 slices is 3*S consecutive sites
// of every plane.  Ghost fields use the device spinor layout with pitch pad(3*S): slot s of the lower ghost is
// global t0 - 3 + s, slot s of the upper ghost is t0 + nt_local + s.
//
// Links.  Forward hops use the link at the output site (local).  Backward t hops from t < 3 need the t-direction
// fat link of slice -1 and long links of slices -3..-1, owned by the rank below: that rank packs its top 3 slices
// of t links (kq_slab_pack_link_face), the caller delivers them once after loading, and kq_slab_set_link_ghosts
// stores them (FP64, with an FP32 copy made on first use).
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_msrelax.h"

namespace kq {

struct SlabArgs {
    const void *glo, *ghi;  // ghost spinors (other parity), pitch pvg
    int pvg;
    const void *gfat_q, *glng_q;  // ghost t links of the other parity (one direction, 3 slices), pitch pvg
    const void *pvec;             // optional: dst = sigma * pvec - D src
    double sigma;
};

// D src at output site i (parity p) of the slab; same term order as dslash_site2, so results match the
// undecomposed operator bit for bit.
template <int P>
__device__ __forceinline__ void slab_site(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                          const void *src, const SlabArgs &a, int p, int i,
                                          typename Acc2<P, P>::T acc[6])
{
    using T = typename Acc2<P, P>::T;
    const SiteCoord c = site_coord(g, i, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const int S = g.st, lt = g.n[3];
    const int j = i - c.t * S;  // index inside the t slice
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] = T(0);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
        T u[18], v[6];
        if (dir < 3) {
            const int nf1 = nbr_index(g, c, i, dir, 1);
            const int nf3 = nbr_index(g, c, i, dir, 3);
            const int nb1 = nbr_index(g, c, i, dir, -1);
            const int nb3 = nbr_index(g, c, i, dir, -3);
            ld_link<P>(fat_p, pv, dir, i, fat.scale, u);
            ld_spinor<P>(src, pv, nf1, v);
            mv_add(u, v, acc);
            ld_link_any<P>(lng_p, pv, dir, i, lng.scale, lng.recon, u);
            ld_spinor<P>(src, pv, nf3, v);
            mv_add(u, v, acc);
            ld_link<P>(fat_q, pv, dir, nb1, fat.scale, u);
            ld_spinor<P>(src, pv, nb1, v);
            mdv_sub(u, v, acc);
            ld_link_any<P>(lng_q, pv, dir, nb3, lng.scale, lng.recon, u);
            ld_spinor<P>(src, pv, nb3, v);
            mdv_sub(u, v, acc);
        } else {
            // forward hops: upper ghost slot t + h - lt when the hop leaves the slab
#pragma unroll
            for (int h = 1; h <= 3; h += 2) {
                const int tt = c.t + h;
                if (h == 1) ld_link<P>(fat_p, pv, 3, i, fat.scale, u);
                else ld_link_any<P>(lng_p, pv, 3, i, lng.scale, lng.recon, u);
                if (tt < lt) ld_spinor<P>(src, pv, i + h * S, v);
                else ld_spinor<P>(a.ghi, a.pvg, (tt - lt) * S + j, v);
                mv_add(u, v, acc);
            }
            // backward hops: lower ghost slot t - h + 3 (spinor and link) when the hop leaves the slab
#pragma unroll
            for (int h = 1; h <= 3; h += 2) {
                const int tt = c.t - h;
                if (tt >= 0) {
                    if (h == 1) ld_link<P>(fat_q, pv, 3, i - h * S, fat.scale, u);
                    else ld_link_any<P>(lng_q, pv, 3, i - h * S, lng.scale, lng.recon, u);
                    ld_spinor<P>(src, pv, i - h * S, v);
                } else {
                    // ghost links share the local fields' HALF scales (unused in FP64 / FP32)
                    ld_link<P>(h == 1 ? a.gfat_q : a.glng_q, a.pvg, 0, (tt + 3) * S + j,
                               h == 1 ? fat.scale : lng.scale, u);
                    ld_spinor<P>(a.glo, a.pvg, (tt + 3) * S + j, v);
                }
                mdv_sub(u, v, acc);
            }
        }
    }
}

// Which output sites a launch covers.  Interior sites (3 <= t < nt_local - 3) read no ghost, so their dslash can
// run while the faces are in flight; the boundary sites (the 3 slices at each end) wait for the ghosts.
enum { kSlabAll = 0, kSlabInterior = 1, kSlabBoundary = 2 };

__host__ __device__ inline int slab_part_sites(const Geom &g, int part)
{
    const int S = g.st, lt = g.n[3];
    if (part == kSlabInterior) return lt > 6 ? (lt - 6) * S : 0;
    if (part == kSlabBoundary) return lt > 6 ? 6 * S : g.vh;
    return g.vh;
}

// site of entry k of a part
__device__ __forceinline__ int slab_part_site(const Geom &g, int part, int k)
{
    const int S = g.st, lt = g.n[3];
    if (part == kSlabInterior) return 3 * S + k;
    if (part == kSlabBoundary && lt > 6) return k < 3 * S ? k : k + (lt - 6) * S;
    return k;
}

template <int P>
__global__ void __launch_bounds__(256) slab_dslash_kernel(Geom g, int pv, LinkSet fat, LinkSet lng,
                                                          const void *__restrict__ src, SlabArgs a,
                                                          void *__restrict__ dst, int p, int part)
{
    using T = typename Acc2<P, P>::T;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= slab_part_sites(g, part)) return;
    const int i = slab_part_site(g, part, k);
    T acc[6];
    slab_site<P>(g, pv, fat, lng, src, a, p, i, acc);
    if (a.pvec) {
        T pv6[6];
        ld_spinor<P>(a.pvec, pv, i, pv6);
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] = (T)a.sigma * pv6[k] - acc[k];
    }
    st_spinor<P>(dst, pv, i, acc);
}

// faces of a spinor: lo = slices 0..2, hi = slices lt-3..lt-1 (pitch pvg)
template <int P>
__global__ void slab_pack_kernel(Geom g, int pv, const void *__restrict__ src, int pvg, void *__restrict__ lo,
                                 void *__restrict__ hi)
{
    const int S = g.st, n = 3 * S;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    typename Acc<P>::T v[6];
    ld_spinor<P>(src, pv, k, v);
    st_spinor<P>(lo, pvg, k, v);
    ld_spinor<P>(src, pv, (g.n[3] - 3) * S + k, v);
    st_spinor<P>(hi, pvg, k, v);
}

// top 3 slices of the t-direction FP64 links (fat and long, both parities) -> face [fat p0|fat p1|lng p0|lng p1]
__global__ void slab_link_pack_kernel(Geom g, int pv, LinkSet fat, LinkSet lng, int pvg, size_t part_bytes,
                                      char *__restrict__ face)
{
    const int S = g.st, n = 3 * S;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = (g.n[3] - 3) * S + k;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const LinkSet &L = q < 2 ? fat : lng;
        double u[18];
        ld_link_any<0>(q & 1 ? L.par[1] : L.par[0], pv, 3, i, 1.f, L.recon, u);
        st_link<0>(face + q * part_bytes, pvg, 0, k, 1.f, u);
    }
}

// FP64 ghost links -> FP32 copy, or a HALF copy with the per-field scales of the local HALF links (fat for the
// two fat parts, long for the two long parts) and the same device factors
template <int P>
__global__ void slab_link_conv_kernel(int n, int pvg, size_t part64, const char *__restrict__ g64, size_t partp,
                                      char *__restrict__ gp, float scale_fat, float scale_lng)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double u[18];
        ld_link<0>(g64 + q * part64, pvg, 0, k, 1.f, u);
        if (P == 2) {
            // the local field's scale need not cover a neighbour's largest entry: saturate instead of wrapping
            const double lim = (double)(q < 2 ? scale_fat : scale_lng);
#pragma unroll
            for (int e = 0; e < 18; ++e) u[e] = fmin(fmax(u[e], -lim), lim);
        }
        st_link<P>(gp + q * partp, pvg, 0, k, q < 2 ? scale_fat : scale_lng, u);
    }
}

// <x, y> of FP64 fields summed into *out on the device: block partials, then one block over them in a fixed order
__global__ void field_sum_kernel(const double *__restrict__ partials, int n, double *__restrict__ out)
{
    __shared__ double sm[32];
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += partials[b];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

// y = a x + b y on FP64 fields (pitch pv), and the block partials of <x, y>
__global__ void field_axpby_kernel(int vh, int pv, double a, const void *__restrict__ x, double b, void *y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vh) return;
    double xv[6], yv[6];
    ld_spinor<0>(x, pv, i, xv);
    ld_spinor<0>(y, pv, i, yv);
#pragma unroll
    for (int k = 0; k < 6; ++k) yv[k] = a * xv[k] + b * yv[k];
    st_spinor<0>(y, pv, i, yv);
}

__global__ void __launch_bounds__(256) field_dot_kernel(int vh, int pv, const void *__restrict__ x,
                                                        const void *__restrict__ y, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * 256 + threadIdx.x;
    double s = 0.0;
    if (i < vh) {
        double xv[6], yv[6];
        ld_spinor<0>(x, pv, i, xv);
        ld_spinor<0>(y, pv, i, yv);
#pragma unroll
        for (int k = 0; k < 6; ++k) s += xv[k] * yv[k];
    }
    s = block_sum(s, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

static int face_sites(const Geom &g) { return 3 * g.st; }
static int face_pitch(const Geom &g) { return pad_sites(face_sites(g)); }

static size_t ghost_link_part(const Geom &g, int prec)  // one type, one parity, one direction, 3 slices
{
    return (size_t)(prec == P64 ? 144 : prec == P32 ? 72 : 36) * face_pitch(g);
}

}  // namespace kq

using namespace kq;

#define KQ_API extern "C" __attribute__((visibility("default")))

static KuQCDStatus slab_check(const kq_context *ctx, const char *where)
{
    if (!ctx) return KUQCD_ERR_NULL_POINTER;
    if (ctx->slab_nranks < 1) {
        set_last_error(std::string(where) + ": the context is not a slab (kq_slab_set)");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_slab_set(kq_context *ctx, int rank, int nranks)
{
    if (!ctx) return KUQCD_ERR_NULL_POINTER;
    const int lt = ctx->g.n[3];
    if (nranks < 1 || rank < 0 || rank >= nranks || lt < 4 || (lt & 1)) {
        set_last_error("kq_slab_set: 0 <= rank < nranks, and the local t extent must be even and >= 4");
        return KUQCD_ERR_INVALID_PARAM;
    }
    ctx->slab_rank = rank;
    ctx->slab_nranks = nranks;
    ctx->have_ghost[0] = ctx->have_ghost[1] = ctx->have_ghost[2] = false;
    return KUQCD_SUCCESS;
}

KQ_API size_t kq_slab_face_bytes(const kq_context *ctx, int prec)
{
    const int p = ctx ? prec_from_api(prec) : -1;
    if (p < 0) return 0;
    const size_t per_site = p == P64 ? 48 : p == P32 ? 24 : 16;
    return per_site * face_pitch(ctx->g);
}

KQ_API KuQCDStatus kq_slab_pack_faces(kq_context *ctx, int prec, const void *d_src, void *d_face_lo, void *d_face_hi,
                                      void *stream)
{
    KuQCDStatus st = slab_check(ctx, "kq_slab_pack_faces");
    if (st != KUQCD_SUCCESS) return st;
    if (!d_src || !d_face_lo || !d_face_hi) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const int n = face_sites(g), pv = pad_sites(g.vh), pvg = face_pitch(g);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    const int nb = (n + 255) / 256;
    if (p == P64) slab_pack_kernel<0><<<nb, 256, 0, s>>>(g, pv, d_src, pvg, d_face_lo, d_face_hi);
    else if (p == P32) slab_pack_kernel<1><<<nb, 256, 0, s>>>(g, pv, d_src, pvg, d_face_lo, d_face_hi);
    else slab_pack_kernel<2><<<nb, 256, 0, s>>>(g, pv, d_src, pvg, d_face_lo, d_face_hi);
    return status_of(cudaGetLastError());
}

KQ_API size_t kq_slab_link_face_bytes(const kq_context *ctx)
{
    return ctx ? 4 * ghost_link_part(ctx->g, P64) : 0;
}

KQ_API KuQCDStatus kq_slab_pack_link_face(kq_context *ctx, void *d_face)
{
    KuQCDStatus st = slab_check(ctx, "kq_slab_pack_link_face");
    if (st != KUQCD_SUCCESS) return st;
    if (!d_face) return KUQCD_ERR_NULL_POINTER;
    if (!ctx->gd.have[P64]) {
        st = kq_prepare_links(ctx, KUQCD_DOUBLE);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const int n = face_sites(g);
    slab_link_pack_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(g, pad_sites(g.vh), ctx->gd.fat[P64],
                                                                     ctx->gd.lng[P64], face_pitch(g),
                                                                     ghost_link_part(g, P64),
                                                                     static_cast<char *>(d_face));
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return status_of(e);
}

KQ_API KuQCDStatus kq_slab_set_link_ghosts(kq_context *ctx, const void *d_face)
{
    KuQCDStatus st = slab_check(ctx, "kq_slab_set_link_ghosts");
    if (st != KUQCD_SUCCESS) return st;
    if (!d_face) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    const size_t bytes = 4 * ghost_link_part(ctx->g, P64);
    cudaError_t e = cudaSuccess;
    if (!ctx->ghost_links[0]) e = cudaMalloc(&ctx->ghost_links[0], bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->ghost_links[0], d_face, bytes, cudaMemcpyDeviceToDevice, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    ctx->have_ghost[0] = e == cudaSuccess;
    ctx->have_ghost[1] = ctx->have_ghost[2] = false;
    return status_of(e);
}

// ghost links in a sloppy precision, derived once from the FP64 ghosts (HALF with the local HALF links' scales)
static cudaError_t ensure_ghost(kq_context *ctx, int p)
{
    if (p == P64 || ctx->have_ghost[p]) return cudaSuccess;
    const Geom &g = ctx->g;
    if (!ctx->ghost_links[p]) KQ_CUDA_TRY(cudaMalloc(&ctx->ghost_links[p], 4 * ghost_link_part(g, p)));
    const int n = face_sites(g), nb = (n + 255) / 256;
    const char *g64 = static_cast<const char *>(ctx->ghost_links[0]);
    char *gp = static_cast<char *>(ctx->ghost_links[p]);
    if (p == P32)
        slab_link_conv_kernel<1><<<nb, 256, 0, ctx->stream>>>(n, face_pitch(g), ghost_link_part(g, P64), g64,
                                                              ghost_link_part(g, P32), gp, 1.f, 1.f);
    else
        slab_link_conv_kernel<2><<<nb, 256, 0, ctx->stream>>>(n, face_pitch(g), ghost_link_part(g, P64), g64,
                                                              ghost_link_part(g, P16), gp, ctx->gd.fat[P16].scale,
                                                              ctx->gd.lng[P16].scale);
    KQ_CUDA_TRY(cudaGetLastError());
    ctx->have_ghost[p] = true;
    return cudaSuccess;
}

KQ_API KuQCDStatus kq_slab_dslash_part(kq_context *ctx, int prec, const void *d_src, const void *d_ghost_lo,
                                       const void *d_ghost_hi, void *d_dst, int dst_parity, const void *d_pvec,
                                       double sigma, int part, void *stream)
{
    KuQCDStatus st = slab_check(ctx, "kq_slab_dslash");
    if (st != KUQCD_SUCCESS) return st;
    if (part != kSlabAll && part != kSlabInterior && part != kSlabBoundary) return KUQCD_ERR_INVALID_PARAM;
    // the interior reads no ghost: its launch may run before the ghosts exist
    if (!d_src || !d_dst || (part != kSlabInterior && (!d_ghost_lo || !d_ghost_hi))) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0 || (dst_parity != 0 && dst_parity != 1)) {
        set_last_error("kq_slab_dslash: DOUBLE, SINGLE or HALF, parity 0 or 1");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->have_ghost[0]) {
        set_last_error("kq_slab_dslash: ghost links not set (kq_slab_set_link_ghosts)");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    if (!ctx->gd.have[p]) {
        st = kq_prepare_links(ctx, prec);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    cudaError_t e = ensure_ghost(ctx, p);
    if (e != cudaSuccess) return status_of(e);
    const Geom &g = ctx->g;
    const size_t gpart = ghost_link_part(g, p);
    const char *gl = static_cast<const char *>(ctx->ghost_links[p]);
    const int q = 1 - dst_parity;
    SlabArgs a;
    a.glo = d_ghost_lo;
    a.ghi = d_ghost_hi;
    a.pvg = face_pitch(g);
    a.gfat_q = gl + (0 + q) * gpart;
    a.glng_q = gl + (2 + q) * gpart;
    a.pvec = d_pvec;
    a.sigma = sigma;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    if (stream && stream != (void *)ctx->stream) {
        // the sloppy ghost links were derived on the context's stream
        cudaEvent_t ev;
        e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) return status_of(e);
        cudaEventRecord(ev, ctx->stream);
        cudaStreamWaitEvent(s, ev, 0);
        cudaEventDestroy(ev);
    }
    const int n = slab_part_sites(g, part);
    if (n == 0) return KUQCD_SUCCESS;
    const int nb = (n + 255) / 256, pv = pad_sites(g.vh);
    const LinkSet &F = ctx->gd.fat[p], &Lk = ctx->gd.lng[p];
    if (p == P64) slab_dslash_kernel<0><<<nb, 256, 0, s>>>(g, pv, F, Lk, d_src, a, d_dst, dst_parity, part);
    else if (p == P32) slab_dslash_kernel<1><<<nb, 256, 0, s>>>(g, pv, F, Lk, d_src, a, d_dst, dst_parity, part);
    else slab_dslash_kernel<2><<<nb, 256, 0, s>>>(g, pv, F, Lk, d_src, a, d_dst, dst_parity, part);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_slab_dslash(kq_context *ctx, int prec, const void *d_src, const void *d_ghost_lo,
                                  const void *d_ghost_hi, void *d_dst, int dst_parity, const void *d_pvec,
                                  double sigma, void *stream)
{
    return kq_slab_dslash_part(ctx, prec, d_src, d_ghost_lo, d_ghost_hi, d_dst, dst_parity, d_pvec, sigma, kSlabAll,
                               stream);
}

KQ_API KuQCDStatus kq_field_dot_device(kq_context *ctx, const void *d_x, const void *d_y, double *d_out,
                                       void *stream)
{
    if (!ctx || !d_x || !d_y || !d_out) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const int nb = (g.vh + 255) / 256;
    Carve probe(nullptr);
    probe.take(sizeof(double) * nb);
    cudaError_t e = ensure_work(ctx, probe.off);
    if (e != cudaSuccess) return status_of(e);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    double *partials = static_cast<double *>(ctx->work);
    field_dot_kernel<<<nb, 256, 0, s>>>(g.vh, pad_sites(g.vh), d_x, d_y, partials);
    field_sum_kernel<<<1, 256, 0, s>>>(partials, nb, d_out);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_field_axpby(kq_context *ctx, double a, const void *d_x, double b, void *d_y, void *stream)
{
    if (!ctx || !d_x || !d_y) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    const Geom &g = ctx->g;
    field_axpby_kernel<<<(g.vh + 255) / 256, 256, 0, s>>>(g.vh, pad_sites(g.vh), a, d_x, b, d_y);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_field_dot(kq_context *ctx, const void *d_x, const void *d_y, double *out)
{
    if (!ctx || !d_x || !d_y || !out) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const int nb = (g.vh + 255) / 256;
    Carve probe(nullptr);
    probe.take(sizeof(double) * nb);
    cudaError_t e = ensure_work(ctx, probe.off);
    if (e != cudaSuccess) return status_of(e);
    double *partials = static_cast<double *>(ctx->work);
    field_dot_kernel<<<nb, 256, 0, ctx->stream>>>(g.vh, pad_sites(g.vh), d_x, d_y, partials);
    std::vector<double> h(nb);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), partials, sizeof(double) * nb, cudaMemcpyDeviceToHost, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    double sum = 0;
    for (double v : h) sum += v;
    *out = sum;
    return status_of(e);
}

// ------------------------------------------------------------------------------------ device-driven multishift CG
// The CGM recurrences of inverter_cgm.cpp:17-87 on a device state, so that a solve over slabs never waits on the
// host: the local sums go to state->sums (sums[0] = <p, A p>, sums[1] = |r|^2), the caller all-reduces them in place
// on the device in stream order, and every step reads its scalars from the state.  Once the solve has stopped
// (state->done) every step is a no-op, so a caller may enqueue several iterations between two polls.
static_assert(offsetof(kq_slab_cgm_state, iter) == 40 && sizeof(kq_slab_cgm_state) == 2624,
              "kq_slab_cgm_state layout (read by hosts through kq_slab_cgm_poll)");

struct CgmInit {
    int ns, max_iter;
    double tol;
    double sh[kMaxShift];
};

__global__ void slab_cgm_init_kernel(kq_slab_cgm_state *st, CgmInit in)
{
    const int j = threadIdx.x;
    if (j == 0) {
        st->sums[0] = st->sums[1] = 0.0;
        st->rr = 0.0;
        st->Bm1 = 1.0;
        st->tol = in.tol;
        st->iter = 0;
        st->max_iter = in.max_iter;
        st->num_shift = in.ns;
        st->max_term = in.ns;
        st->done = 0;
        st->reserved = 0;
    }
    for (int k = j; k < kMaxShift; k += blockDim.x) {
        st->sh[k] = k < in.ns ? in.sh[k] : 0.0;
        st->a[k] = 0.0;
        st->B[k] = st->Z[k] = st->Zm1[k] = 1.0;
    }
}

// one block of kMaxShift threads; thread j updates shift j (the vectorised loop over shifts of inverter_cgm.cpp:49-60)
__global__ void slab_cgm_step_kernel(kq_slab_cgm_state *st, int step)
{
    if (st->done) return;  // uniform over the block
    const int j = threadIdx.x;
    if (step == KQ_CGM_START) {
        // |b|^2 = 0: x = 0 solves every shift; a non-finite source stops at once
        if (j == 0) {
            st->rr = st->sums[1];
            if (!(st->rr > 0.0) || !isfinite(st->rr)) st->done = 1;
        }
    } else if (step == KQ_CGM_ALPHA) {
        // B_0 = -|r|^2 / <p, A p>; the shifted B_j, Z_j with the previous a_0 and B_0 (inverter_cgm.cpp:47-57).
        // Every product and sum rounded on its own (no FMA contraction), as a host evaluates the same expressions.
        const double B0 = -st->rr / st->sums[0], a0 = st->a[0], Bm1 = st->Bm1;
        if (j >= 1 && j < st->max_term) {
            const double z = st->Z[j], zm1 = st->Zm1[j];
            const double den = __dadd_rn(__dmul_rn(__dmul_rn(B0, a0), __dsub_rn(zm1, z)),
                                         __dmul_rn(__dmul_rn(zm1, Bm1), __dsub_rn(1.0, __dmul_rn(st->sh[j], B0))));
            const double rr1 = __dmul_rn(Bm1, zm1) / den;
            st->Zm1[j] = z;
            st->Z[j] = __dmul_rn(z, rr1);
            st->B[j] = __dmul_rn(B0, rr1);
        }
        __syncthreads();
        if (j == 0) {
            st->B[0] = B0;
            st->Bm1 = B0;
        }
    } else if (step == KQ_CGM_BETA) {
        // a_0 = |r_new|^2 / |r|^2 and the shifted a_j (inverter_cgm.cpp:58-66)
        const double lam2 = st->sums[1], a0 = lam2 / st->rr, B0 = st->B[0];
        if (j >= 1 && j < st->max_term)
            st->a[j] = __dmul_rn(__dmul_rn(a0, st->Z[j]), st->B[j]) / __dmul_rn(st->Zm1[j], B0);
        __syncthreads();
        if (j == 0) {
            st->a[0] = a0;
            st->rr = lam2;
        }
    } else if (j == 0) {  // KQ_CGM_FINISH: drop converged shifts from the end (inverter_cgm.cpp:70-80)
        int mt = st->max_term;
        while (mt > 0 && __dmul_rn(__dmul_rn(st->Z[mt - 1], st->Z[mt - 1]), st->rr) < st->tol) --mt;
        st->max_term = mt;
        st->iter += 1;
        st->done = (mt == 0 || st->iter >= st->max_iter) ? 1 : 0;
    }
}

// r += B_0 s and the block partials of |r|^2
__global__ void slab_cgm_residual_kernel(int vh, int pv, const kq_slab_cgm_state *st, const void *__restrict__ s_,
                                         void *r_, double *partials)
{
    __shared__ double sm[32];
    if (st->done) return;  // uniform over the grid
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double nn = 0.0;
    if (i < vh) {
        const double b0 = st->B[0];
        double sv[6], rv[6];
        ld_spinor<0>(s_, pv, i, sv);
        ld_spinor<0>(r_, pv, i, rv);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            rv[k] += b0 * sv[k];
            nn += rv[k] * rv[k];
        }
        st_spinor<0>(r_, pv, i, rv);
    }
    nn = block_sum(nn, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = nn;
}

__global__ void slab_cgm_sum_kernel(const kq_slab_cgm_state *st, const double *__restrict__ partials, int n,
                                    double *out)
{
    __shared__ double sm[32];
    if (st->done) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += partials[b];
    s = block_sum(s, sm);
    if (threadIdx.x == 0) *out = s;
}

// x_j -= B_j p_j ; p_j = Z_j r + a_j p_j for the shifts still iterating, coefficients from the state
__global__ void slab_cgm_update_kernel(int vh, int pv, const kq_slab_cgm_state *st, const void *__restrict__ r,
                                       char *p, char *x, size_t stride)
{
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vh) return;
    const int n = st->max_term;
    double rv[6];
    ld_spinor<0>(r, pv, i, rv);
    for (int j = 0; j < n; ++j) {
        const double B = st->B[j], Z = st->Z[j], a = st->a[j];
        double pv6[6], xv[6];
        ld_spinor<0>(p + j * stride, pv, i, pv6);
        ld_spinor<0>(x + j * stride, pv, i, xv);
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            xv[k] -= B * pv6[k];
            pv6[k] = Z * rv[k] + a * pv6[k];
        }
        st_spinor<0>(x + j * stride, pv, i, xv);
        st_spinor<0>(p + j * stride, pv, i, pv6);
    }
}

KQ_API size_t kq_slab_cgm_state_bytes(void) { return sizeof(kq_slab_cgm_state); }

KQ_API KuQCDStatus kq_slab_cgm_init(kq_context *ctx, kq_slab_cgm_state *d_state, int num_shift,
                                    const double *shifts_ref, double tol, int max_iter, void *stream)
{
    if (!ctx || !d_state || !shifts_ref) return KUQCD_ERR_NULL_POINTER;
    if (num_shift < 1 || num_shift > kMaxShift || max_iter < 1) return KUQCD_ERR_INVALID_PARAM;
    if ((reinterpret_cast<uintptr_t>(d_state) & 7) != 0) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    CgmInit in;
    in.ns = num_shift;
    in.max_iter = max_iter;
    in.tol = tol;
    for (int j = 0; j < kMaxShift; ++j) in.sh[j] = j < num_shift ? shifts_ref[j] : 0.0;
    slab_cgm_init_kernel<<<1, kMaxShift, 0, s>>>(d_state, in);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_slab_cgm_step(kq_context *ctx, kq_slab_cgm_state *d_state, int step, void *stream)
{
    if (!ctx || !d_state) return KUQCD_ERR_NULL_POINTER;
    if (step < KQ_CGM_START || step > KQ_CGM_FINISH) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    slab_cgm_step_kernel<<<1, kMaxShift, 0, s>>>(d_state, step);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_slab_cgm_residual(kq_context *ctx, kq_slab_cgm_state *d_state, const void *d_s, void *d_r,
                                        void *stream)
{
    if (!ctx || !d_state || !d_s || !d_r) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const int nb = (g.vh + 255) / 256;
    Carve probe(nullptr);
    probe.take(sizeof(double) * nb);
    cudaError_t e = ensure_work(ctx, probe.off);
    if (e != cudaSuccess) return status_of(e);
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    double *partials = static_cast<double *>(ctx->work);
    slab_cgm_residual_kernel<<<nb, 256, 0, s>>>(g.vh, pad_sites(g.vh), d_state, d_s, d_r, partials);
    slab_cgm_sum_kernel<<<1, 256, 0, s>>>(d_state, partials, nb, &d_state->sums[1]);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_slab_cgm_update(kq_context *ctx, const kq_slab_cgm_state *d_state, const void *d_r, void *d_p,
                                      void *d_x, size_t stride, void *stream)
{
    if (!ctx || !d_state || !d_r || !d_p || !d_x) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    slab_cgm_update_kernel<<<(g.vh + 255) / 256, 256, 0, s>>>(g.vh, pad_sites(g.vh), d_state, d_r,
                                                              static_cast<char *>(d_p), static_cast<char *>(d_x),
                                                              stride);
    return status_of(cudaGetLastError());
}

KQ_API KuQCDStatus kq_slab_cgm_poll(kq_context *ctx, const kq_slab_cgm_state *d_state, int *iter, int *done,
                                    double *rr, void *stream)
{
    if (!ctx || !d_state || !iter || !done) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    kq_slab_cgm_state h;  // the scalar head: sums, rr, Bm1, tol and the counters
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    cudaError_t e = cudaMemcpyAsync(&h, d_state, offsetof(kq_slab_cgm_state, sh), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_slab_cgm_poll: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    *iter = h.iter;
    *done = h.done;
    if (rr) *rr = h.rr;
    return KUQCD_SUCCESS;
}
