// C ABI of libkuqcd_b200.so: contexts, link loading, dslash, solver entry points and the C-linkage twins of the
// reference's five exported calls (kuqcd.cpp:288-487).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "kq_context.h"
#include "kq_internal.h"
#include "kq_msrelax.h"
#include "kq_prec.cuh"
#include "kq_solver.h"

namespace kq {

static thread_local std::string g_last_error;
void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

cudaError_t launch_mdagm(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                         void *dst, int parity, cudaStream_t s);
cudaError_t true_residuals(const Geom &g, const GaugeDev &gd, int parity, int ns, const double *sigma,
                           const void *d_b, const void *d_x, size_t xstride, void *d_tmp, void *d_s, double *partials,
                           double *out, cudaStream_t s);
cudaError_t true_residuals_full(const Geom &g, const GaugeDev &gd, int ns, const double *sigma, const void *d_b,
                                const void *d_x, size_t xstride, void *d_tmp, void *d_s, double *partials,
                                double *out, cudaStream_t s);
cudaError_t launch_dslash_full(const Geom &g, const GaugeDev &gd, int prec, const void *src, const void *pvec,
                               void *dst, double sigma, cudaStream_t s);
cudaError_t launch_mdagm_full(const Geom &g, const GaugeDev &gd, int prec, double sigma, const void *src, void *tmp,
                              void *dst, cudaStream_t s);
cudaError_t norm2_p64(const Geom &g, const void *v, double *partials, double *out, cudaStream_t s);

}  // namespace kq

using namespace kq;

// ------------------------------------------------------------------------------------------------ context
namespace kq {

cudaError_t ensure_work(::kq_context *ctx, size_t bytes)
{
    if (ctx->work_bytes >= bytes) return cudaSuccess;
    if (ctx->work) {
        KQ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->work);
        ctx->work = nullptr;
        ctx->work_bytes = 0;
    }
    KQ_CUDA_TRY(cudaMalloc(&ctx->work, bytes));
    ctx->work_bytes = bytes;
    return cudaSuccess;
}

static cudaError_t alloc_links(::kq_context *ctx, int prec)
{
    if (ctx->gd.block[prec]) return cudaSuccess;
    const size_t lb = links_bytes(ctx->g, prec);
    void *blk = nullptr;
    KQ_CUDA_TRY(cudaMalloc(&blk, 4 * lb));
    ctx->gd.block[prec] = blk;
    char *b = static_cast<char *>(blk);
    ctx->gd.fat[prec].par[0] = b;
    ctx->gd.fat[prec].par[1] = b + lb;
    ctx->gd.lng[prec].par[0] = b + 2 * lb;
    ctx->gd.lng[prec].par[1] = b + 3 * lb;
    ctx->gd.fat[prec].scale = ctx->gd.lng[prec].scale = 1.f;
    return cudaSuccess;
}

static void free_links(::kq_context *ctx, int prec)
{
    if (ctx->gd.block[prec]) cudaFree(ctx->gd.block[prec]);
    ctx->gd.block[prec] = nullptr;
    ctx->gd.have[prec] = false;
}

KuQCDStatus status_of(cudaError_t e)
{
    if (e == cudaSuccess) return KUQCD_SUCCESS;
    // the error is being reported to the caller now: clear the runtime's per-thread last error, so that a failed
    // allocation does not resurface in the next launch check of an unrelated call
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation) return KUQCD_ERR_NO_MEMORY;
    if (e == cudaErrorInvalidValue) return KUQCD_ERR_INVALID_PARAM;
    return KUQCD_ERR_UNKNOWN_ERROR;
}

}  // namespace kq

#define KQ_API extern "C" __attribute__((visibility("default")))

static cudaStream_t pick_stream(kq_context *ctx, void *stream)
{
    return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

KQ_API const char *kq_last_error(void) { return kq::last_error(); }

KQ_API KuQCDStatus kq_context_create(const unsigned lat[4], int device, kq_context **out)
{
    if (!lat || !out) {
        set_last_error("kq_context_create: null pointer");
        return KUQCD_ERR_NULL_POINTER;
    }
    for (int i = 0; i < 4; ++i)
        if (lat[i] == 0) {
            set_last_error("kq_context_create: lattice extent is 0");
            return KUQCD_ERR_INVALID_PARAM;
        }
    if (lat[0] & 1u) {
        set_last_error("kq_context_create: x extent must be even for even-odd preconditioning");
        return KUQCD_ERR_INVALID_PARAM;
    }
    const double V = (double)lat[0] * lat[1] * lat[2] * lat[3];
    if (V / 2 > 2.0e9) {
        set_last_error("kq_context_create: more than 2^31 sites per parity");
        return KUQCD_ERR_INVALID_PARAM;
    }
    kq_context *c = new (std::nothrow) kq_context();
    if (!c) return KUQCD_ERR_NO_MEMORY;
    c->device = device;
    memcpy(c->lat, lat, sizeof(c->lat));
    c->g = make_geom(lat);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_scratch, 256);
    if (e == cudaSuccess) e = cudaMallocHost(&c->poll, 4096);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_context_create: ") + cudaGetErrorString(e));
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->d_scratch) cudaFree(c->d_scratch);
        delete c;
        return status_of(e);
    }
    *out = c;
    return KUQCD_SUCCESS;
}

KQ_API void kq_context_destroy(kq_context *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (int p = 0; p < 3; ++p) free_links(ctx, p);
    for (void *gl : ctx->ghost_links)
        if (gl) cudaFree(gl);
    if (ctx->work) cudaFree(ctx->work);
    if (ctx->io) cudaFree(ctx->io);
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    if (ctx->poll) cudaFreeHost(ctx->poll);
    if (ctx->copy_stream) {
        cudaStreamSynchronize(ctx->copy_stream);
        cudaStreamDestroy(ctx->copy_stream);
    }
    if (ctx->copy_ready) cudaEventDestroy(ctx->copy_ready);
    if (ctx->copy_done) cudaEventDestroy(ctx->copy_done);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

// Long links that are real multiples of SU(3) matrices (HISQ's Naik links: products of reunitarised links) are kept
// as two rows + 1/s (104 B instead of 144 B per FP64 link, 52 B instead of 72 B in FP32): 13 % less traffic for
// every FP64 and FP32 dslash.  KUQCD_LONG_RECON=0 keeps full storage.
static cudaError_t compress_long(kq_context *ctx, int prec)
{
    const char *env = getenv("KUQCD_LONG_RECON");
    if (env && env[0] == '0') return cudaSuccess;
    if (prec != P64 && prec != P32) return cudaSuccess;
    bool done = false;
    return links_compress(ctx->g, ctx->gd.lng[prec], prec, prec == P64 ? 1e-12 : 2e-6, ctx->d_scratch, ctx->stream,
                          &done);
}

KQ_API KuQCDStatus kq_long_links_compressed(const kq_context *ctx, int prec, int *out)
{
    if (!ctx || !out) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0) return KUQCD_ERR_INVALID_PARAM;
    *out = ctx->gd.have[p] ? ctx->gd.lng[p].recon : -1;
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_load_links(kq_context *ctx, int link_type, const void *host, int host_prec)
{
    if (!ctx || !host) {
        set_last_error("kq_load_links: null pointer");
        return KUQCD_ERR_NULL_POINTER;
    }
    if (link_type != KUQCD_FAT_LINK && link_type != KUQCD_LONG_LINK) {
        set_last_error("kq_load_links: link_type is invalid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    const int rp = prec_from_api(host_prec);
    if (rp != P64 && rp != P32) {
        set_last_error("kq_load_links: host precision must be DOUBLE or SINGLE");
        return host_prec == KUQCD_HALF ? KUQCD_ERR_UNSUPPORTED : KUQCD_ERR_INVALID_PARAM;
    }
    cudaSetDevice(ctx->device);
    if (ctx->master < 0) ctx->master = rp;
    const int mp = ctx->master;
    cudaError_t e = alloc_links(ctx, mp);
    if (e != cudaSuccess) return status_of(e);
    const size_t V = 2 * (size_t)ctx->g.vh;
    const size_t rec_bytes = V * 72 * (rp == P64 ? 8 : 4);
    void *stage = nullptr;
    e = cudaMalloc(&stage, rec_bytes);
    if (e != cudaSuccess) {
        set_last_error("kq_load_links: cannot stage the host record on the device");
        return status_of(e);
    }
    e = cudaMemcpyAsync(stage, host, rec_bytes, cudaMemcpyHostToDevice, ctx->stream);
    // fold the reference kernel's factors into the device links: 1/2 for fat, c3 = -1/48 for long
    const double factor = link_type == KUQCD_FAT_LINK ? 0.5 : -1.0 / 48.0;
    LinkSet &dst = link_type == KUQCD_FAT_LINK ? ctx->gd.fat[mp] : ctx->gd.lng[mp];
    if (e == cudaSuccess) e = links_from_host_record(ctx->g, stage, rp, factor, dst, mp, ctx->d_scratch, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    cudaFree(stage);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_load_links: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    if (link_type == KUQCD_FAT_LINK) ctx->fat_loaded = true;
    else ctx->long_loaded = true;
    ctx->have_ghost[0] = ctx->have_ghost[1] = ctx->have_ghost[2] = false;  // a slab's ghost links belong to the
                                                                           // previous links
    if (link_type == KUQCD_LONG_LINK) {
        e = compress_long(ctx, mp);
        if (e != cudaSuccess) {
            set_last_error(std::string("kq_load_links: ") + cudaGetErrorString(e));
            return status_of(e);
        }
    }
    ctx->gd.have[mp] = ctx->fat_loaded && ctx->long_loaded;
    // derived copies are stale now
    for (int p = 0; p < 3; ++p)
        if (p != mp) free_links(ctx, p);
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_prepare_links(kq_context *ctx, int prec)
{
    if (!ctx) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0) {
        set_last_error("kq_prepare_links: invalid precision");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->fat_loaded || !ctx->long_loaded) {
        set_last_error("kq_prepare_links: load the fat and long links first");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    if (ctx->gd.have[p]) return KUQCD_SUCCESS;
    cudaSetDevice(ctx->device);
    cudaError_t e = alloc_links(ctx, p);
    if (e == cudaSuccess)
        e = links_convert(ctx->g, ctx->gd.fat[ctx->master], ctx->master, ctx->gd.fat[p], p, ctx->d_scratch, ctx->stream);
    if (e == cudaSuccess)
        e = links_convert(ctx->g, ctx->gd.lng[ctx->master], ctx->master, ctx->gd.lng[p], p, ctx->d_scratch, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e == cudaSuccess) e = compress_long(ctx, p);
    if (e != cudaSuccess) {
        free_links(ctx, p);
        set_last_error(std::string("kq_prepare_links: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    ctx->gd.have[p] = true;
    return KUQCD_SUCCESS;
}

KQ_API size_t kq_spinor_bytes(const kq_context *ctx, int prec)
{
    const int p = prec_from_api(prec);
    if (!ctx || p < 0) return 0;
    return spinor_bytes(ctx->g, p);
}

KQ_API KuQCDStatus kq_spinor_upload(kq_context *ctx, int prec, const void *host, int host_prec, void *d_field,
                                    void *stream)
{
    if (!ctx || !host || !d_field) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec), rp = prec_from_api(host_prec);
    if (p < 0 || (rp != P64 && rp != P32)) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    cudaStream_t s = pick_stream(ctx, stream);
    const size_t rb = (size_t)ctx->g.vh * 6 * (rp == P64 ? 8 : 4);
    void *stage = nullptr;
    cudaError_t e = cudaMallocAsync(&stage, rb, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(stage, host, rb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = spinor_from_record(ctx->g, stage, rp, d_field, p, s);
    if (stage) cudaFreeAsync(stage, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) set_last_error(std::string("kq_spinor_upload: ") + cudaGetErrorString(e));
    return status_of(e);
}

KQ_API KuQCDStatus kq_spinor_download(kq_context *ctx, int prec, const void *d_field, void *host, int host_prec,
                                      void *stream)
{
    if (!ctx || !host || !d_field) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec), rp = prec_from_api(host_prec);
    if (p < 0 || (rp != P64 && rp != P32)) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    cudaStream_t s = pick_stream(ctx, stream);
    const size_t rb = (size_t)ctx->g.vh * 6 * (rp == P64 ? 8 : 4);
    void *stage = nullptr;
    cudaError_t e = cudaMallocAsync(&stage, rb, s);
    if (e == cudaSuccess) e = spinor_to_record(ctx->g, d_field, p, stage, rp, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, stage, rb, cudaMemcpyDeviceToHost, s);
    if (stage) cudaFreeAsync(stage, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) set_last_error(std::string("kq_spinor_download: ") + cudaGetErrorString(e));
    return status_of(e);
}

KQ_API KuQCDStatus kq_spinor_convert(kq_context *ctx, const void *d_src, int src_prec, void *d_dst, int dst_prec,
                                     void *stream)
{
    if (!ctx || !d_src || !d_dst) return KUQCD_ERR_NULL_POINTER;
    const int a = prec_from_api(src_prec), b = prec_from_api(dst_prec);
    if (a < 0 || b < 0) return KUQCD_ERR_INVALID_PARAM;
    cudaSetDevice(ctx->device);
    return status_of(spinor_convert(ctx->g, d_src, a, d_dst, b, pick_stream(ctx, stream)));
}

KQ_API KuQCDStatus kq_dslash(kq_context *ctx, int prec, const void *d_src, void *d_dst, int dst_parity, void *stream)
{
    if (!ctx || !d_src || !d_dst) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0 || (dst_parity != 0 && dst_parity != 1)) return KUQCD_ERR_INVALID_PARAM;
    if (!ctx->gd.have[p]) {
        KuQCDStatus st = kq_prepare_links(ctx, prec);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    return status_of(launch_dslash(ctx->g, ctx->gd, p, d_src, d_dst, dst_parity, pick_stream(ctx, stream), 0));
}

KQ_API KuQCDStatus kq_mdagm(kq_context *ctx, int prec, double sigma, const void *d_src, void *d_dst, void *d_tmp,
                            int parity, void *stream)
{
    if (!ctx || !d_src || !d_dst || !d_tmp) return KUQCD_ERR_NULL_POINTER;
    const int p = prec_from_api(prec);
    if (p < 0 || (parity != 0 && parity != 1)) return KUQCD_ERR_INVALID_PARAM;
    if (!ctx->gd.have[p]) {
        KuQCDStatus st = kq_prepare_links(ctx, prec);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    return status_of(launch_mdagm(ctx->g, ctx->gd, p, sigma, d_src, d_tmp, d_dst, parity, pick_stream(ctx, stream)));
}

static KuQCDStatus full_prep(kq_context *ctx, int prec, int *p)
{
    *p = prec_from_api(prec);
    if (*p < 0) return KUQCD_ERR_INVALID_PARAM;
    if (!ctx->gd.have[*p]) {
        KuQCDStatus st = kq_prepare_links(ctx, prec);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_dslash_full(kq_context *ctx, int prec, const void *d_src, void *d_dst, void *stream)
{
    if (!ctx || !d_src || !d_dst) return KUQCD_ERR_NULL_POINTER;
    int p;
    KuQCDStatus st = full_prep(ctx, prec, &p);
    if (st != KUQCD_SUCCESS) return st;
    return status_of(launch_dslash_full(ctx->g, ctx->gd, p, d_src, nullptr, d_dst, 0.0, pick_stream(ctx, stream)));
}

KQ_API KuQCDStatus kq_mdagm_full(kq_context *ctx, int prec, double sigma, const void *d_src, void *d_dst, void *d_tmp,
                                 void *stream)
{
    if (!ctx || !d_src || !d_dst || !d_tmp) return KUQCD_ERR_NULL_POINTER;
    int p;
    KuQCDStatus st = full_prep(ctx, prec, &p);
    if (st != KUQCD_SUCCESS) return st;
    return status_of(launch_mdagm_full(ctx->g, ctx->gd, p, sigma, d_src, d_tmp, d_dst, pick_stream(ctx, stream)));
}

KQ_API KuQCDStatus kq_make_links_record(kq_context *ctx, double eps, uint64_t seed, double *d_fat, double *d_long)
{
    if (!ctx || !d_fat || !d_long) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    cudaError_t e = make_links_record(ctx->g, eps, seed, d_fat, d_long, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return status_of(e);
}

KQ_API KuQCDStatus kq_make_source_record(kq_context *ctx, int parity, uint64_t seed, double *d_b)
{
    if (!ctx || !d_b) return KUQCD_ERR_NULL_POINTER;
    cudaSetDevice(ctx->device);
    cudaError_t e = make_source_record(ctx->g, parity, seed, d_b, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    return status_of(e);
}

// ------------------------------------------------------------------------------------------------ solver
static void absolute_shifts(const kq_solve_param *p, double *out)
{
    for (int k = 0; k < p->num_shift; ++k)
        out[k] = (p->shift_mode == 0 && k > 0) ? p->shifts[0] + p->shifts[k] : p->shifts[k];
}

static KuQCDStatus check_solve_param(const kq_context *ctx, const kq_solve_param *p)
{
    if (!ctx || !p || !p->shifts) {
        set_last_error("solve: null pointer");
        return KUQCD_ERR_NULL_POINTER;
    }
    if (p->num_shift <= 0 || p->num_shift > kMaxShift) {
        set_last_error("solve: num_shift must be in 1..64");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (p->parity != 0 && p->parity != 1 && p->parity != KQ_PARITY_FULL) {
        set_last_error("solve: parity must be 0, 1 or KQ_PARITY_FULL");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->fat_loaded || !ctx->long_loaded) {
        set_last_error("solve: load the fat and long links first");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_true_residuals(kq_context *ctx, int parity, int num_shift, const double *sigma,
                                     const void *d_b, const void *d_x, double *out)
{
    if (!ctx || !sigma || !d_b || !d_x || !out) return KUQCD_ERR_NULL_POINTER;
    const bool full = parity == KQ_PARITY_FULL;
    if (num_shift < 1 || num_shift > kMaxShift || (parity != 0 && parity != 1 && !full))
        return KUQCD_ERR_INVALID_PARAM;
    if (!ctx->gd.have[P64]) {
        KuQCDStatus st = kq_prepare_links(ctx, KUQCD_DOUBLE);
        if (st != KUQCD_SUCCESS) return st;
    }
    cudaSetDevice(ctx->device);
    const size_t vb = spinor_bytes(ctx->g, P64) * (full ? 2 : 1);
    const int nb = (ctx->g.vh + 255) / 256;
    Carve c(nullptr);
    c.take(vb);
    c.take(vb);
    c.take(sizeof(double) * 4 * nb);
    cudaError_t e = ensure_work(ctx, c.off);
    if (e != cudaSuccess) return status_of(e);
    Carve w(ctx->work);
    void *tmp = w.take(vb), *s = w.take(vb);
    double *partials = static_cast<double *>(w.take(sizeof(double) * 4 * nb));
    if (full)
        e = true_residuals_full(ctx->g, ctx->gd, num_shift, sigma, d_b, d_x, vb, tmp, s, partials, out, ctx->stream);
    else
        e = true_residuals(ctx->g, ctx->gd, parity, num_shift, sigma, d_b, d_x, vb, tmp, s, partials, out,
                           ctx->stream);
    return status_of(e);
}

static KuQCDStatus solve_full(kq_context *ctx, const kq_solve_param *p, const void *d_b, void *d_x,
                              kq_solve_info *info);

KQ_API KuQCDStatus kq_solve_multishift_device(kq_context *ctx, const kq_solve_param *p, const void *d_b, void *d_x,
                                              kq_solve_info *info)
{
    kq::NvtxRange nvtx_range_("kq_solve_multishift_device");
    KuQCDStatus st = check_solve_param(ctx, p);
    if (st != KUQCD_SUCCESS) return st;
    if (!d_b || !d_x) return KUQCD_ERR_NULL_POINTER;
    if (p->parity == KQ_PARITY_FULL) return solve_full(ctx, p, d_b, d_x, info);
    cudaSetDevice(ctx->device);
    double sig[kMaxShift];
    absolute_shifts(p, sig);
    kq_solve_info local;
    if (!info) info = &local;
    memset(info, 0, sizeof(*info));
    info->num_shift = p->num_shift;

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    cudaError_t e = cudaSuccess;
    if (p->solver == KQ_SOLVER_MIXED) {
        e = mixed_solve(ctx, p, sig, d_b, d_x, info, true);
    } else if (p->solver == KQ_SOLVER_CGM_WINDOWED) {
        MsBuffers w;
        Carve probe(nullptr);
        ms_layout(probe, ctx->g, p->num_shift, d_b, d_x, w);
        e = ensure_work(ctx, probe.off);
        if (e == cudaSuccess) {
            Carve c(ctx->work);
            ms_layout(c, ctx->g, p->num_shift, d_b, d_x, w);
            double rs[kMaxShift];
            rs[0] = sig[0];
            for (int k = 1; k < p->num_shift; ++k) rs[k] = sig[k] - sig[0];
            MsResult r;
            e = ms_solve(ctx, w, p->parity, p->num_shift, rs, p->tol, p->max_iter, 0.0, 0.0, &r);
            if (e == cudaSuccess) {
                info->iter = r.iter;
                info->status = r.status;
                info->kernel_launches = r.launches;
            }
        }
    } else {
        const int prec = prec_from_api(p->prec);
        if (prec != P64 && prec != P32) {
            set_last_error("solve: KQ_SOLVER_CGM runs in DOUBLE or SINGLE");
            return KUQCD_ERR_INVALID_PARAM;
        }
        if (!ctx->gd.have[prec]) {
            st = kq_prepare_links(ctx, p->prec);
            if (st != KUQCD_SUCCESS) return st;
        }
        const Geom &g = ctx->g;
        const size_t vb = spinor_bytes(g, prec), vb64 = spinor_bytes(g, P64);
        const int nb = (g.vh + 255) / 256;
        const int ns = p->num_shift;
        auto layout = [&](Carve &c, CgmBuffers &w) {
            w.vec_bytes = vb;
            w.r = c.take(vb);
            w.s = c.take(vb);
            w.tmp = c.take(vb);
            w.p = c.take(vb * ns);
            w.partials = static_cast<double *>(c.take(sizeof(double) * nb));
            w.state = static_cast<CgmState *>(c.take(sizeof(CgmState)));
            if (prec != P64) {
                w.b = c.take(vb);
                w.x = c.take(vb * ns);
            } else {
                w.b = d_b;
                w.x = d_x;
            }
        };
        CgmBuffers w;
        Carve probe(nullptr);
        layout(probe, w);
        e = ensure_work(ctx, probe.off);
        if (e != cudaSuccess) return status_of(e);
        Carve c(ctx->work);
        layout(c, w);
        w.poll = ctx->poll;
        if (prec != P64) e = spinor_convert(g, d_b, P64, const_cast<void *>(w.b), prec, ctx->stream);
        // reference shift semantics inside the recurrence: shifts[0] absolute, shifts[j] relative
        double rs[kMaxShift];
        rs[0] = sig[0];
        for (int k = 1; k < ns; ++k) rs[k] = sig[k] - sig[0];
        CgmResult r;
        if (e == cudaSuccess) e = cgm_solve(g, ctx->gd, prec, prec, w, p->parity, ns, rs, p->tol, p->max_iter, 8, &r, ctx->stream);
        if (e == cudaSuccess && prec != P64)
            for (int k = 0; k < ns && e == cudaSuccess; ++k)
                e = spinor_convert(g, static_cast<char *>(w.x) + k * vb, prec, static_cast<char *>(d_x) + k * vb64,
                                   P64, ctx->stream);
        if (e == cudaSuccess) {
            info->iter = r.iter;
            info->kernel_launches = r.launches + (prec != P64 ? 1 + ns : 0);
            info->status = r.status ? r.status : (r.iter >= p->max_iter ? KQ_STATUS_MAXITER : 0);
        }
    }
    cudaEventRecord(e1, ctx->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    info->seconds = ms * 1e-3;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e != cudaSuccess) {
        if (std::string(last_error()).empty()) set_last_error(cudaGetErrorString(e));
        return status_of(e);
    }
    return info->status == KQ_STATUS_BREAKDOWN ? KUQCD_ERR_UNKNOWN_ERROR : KUQCD_SUCCESS;
}

// Full-lattice solve: sigma - D D has no even-odd coupling, so x = (x_e, x_o) with each half the solution of its
// own parity system.  The reference's rule on the full residual, zeta^2 (|r_e|^2 + |r_o|^2) < tol, holds when each
// half meets tol / 2; a relative target eps |b| holds when each half meets eps |b| / sqrt(2).  Each half is solved
// into a contiguous scratch (the parity solvers take shift-contiguous fields) and copied into the strided halves.
static KuQCDStatus solve_full(kq_context *ctx, const kq_solve_param *p, const void *d_b, void *d_x,
                              kq_solve_info *info)
{
    cudaSetDevice(ctx->device);
    const Geom &g = ctx->g;
    const size_t vb = spinor_bytes(g, P64);
    const int ns = p->num_shift;
    kq_solve_info local;
    if (!info) info = &local;
    memset(info, 0, sizeof(*info));
    info->num_shift = ns;
    const int nb = (g.vh + 255) / 256;
    void *scratch = nullptr;
    cudaError_t e = cudaMallocAsync(&scratch, vb * ns + sizeof(double) * 2 * nb, ctx->stream);
    if (e != cudaSuccess) return status_of(e);
    double *partials = reinterpret_cast<double *>(static_cast<char *>(scratch) + vb * ns);
    double bb[2] = {0, 0};
    for (int par = 0; par < 2 && e == cudaSuccess; ++par)
        e = norm2_p64(g, static_cast<const char *>(d_b) + par * vb, partials, &bb[par], ctx->stream);
    const double bt = bb[0] + bb[1];
    double rr[kMaxShift] = {0};
    KuQCDStatus st = status_of(e);
    for (int par = 0; par < 2 && st == KUQCD_SUCCESS; ++par) {
        char *xh = static_cast<char *>(d_x) + par * vb;
        if (!(bb[par] > 0)) {  // zero source half: zero solution half
            e = cudaMemset2DAsync(xh, 2 * vb, 0, vb, ns, ctx->stream);
            st = status_of(e);
            continue;
        }
        kq_solve_param q = *p;
        q.parity = par;
        q.tol = p->tol / 2;
        q.rel_residual = p->rel_residual * std::sqrt(bt / (2 * bb[par]));
        kq_solve_info hi;
        st = kq_solve_multishift_device(ctx, &q, static_cast<const char *>(d_b) + par * vb, scratch, &hi);
        if (st != KUQCD_SUCCESS && st != KUQCD_ERR_UNKNOWN_ERROR) break;
        e = cudaMemcpy2DAsync(xh, 2 * vb, scratch, vb, vb, ns, cudaMemcpyDeviceToDevice, ctx->stream);
        if (e != cudaSuccess) st = status_of(e);
        info->iter = std::max(info->iter, hi.iter);
        info->iter_refine += hi.iter_refine;
        info->status = std::max(info->status, hi.status);
        info->seconds += hi.seconds;
        info->kernel_launches += hi.kernel_launches + 1;
        info->sloppy_residual = std::max(info->sloppy_residual, hi.sloppy_residual);
        for (int k = 0; k < ns; ++k) rr[k] += hi.true_residual[k] * hi.true_residual[k] * bb[par];
    }
    for (int k = 0; k < ns; ++k) info->true_residual[k] = bt > 0 ? std::sqrt(rr[k] / bt) : 0.0;
    cudaFreeAsync(scratch, ctx->stream);
    cudaError_t e2 = cudaStreamSynchronize(ctx->stream);
    if (st == KUQCD_SUCCESS && e2 != cudaSuccess) st = status_of(e2);
    if (st == KUQCD_SUCCESS && info->status == KQ_STATUS_BREAKDOWN) st = KUQCD_ERR_UNKNOWN_ERROR;
    return st;
}

// Solutions into pinned host buffers leave while the solve goes on: the solver reports each solution once it is
// final (kq_context::solution_ready), and it is converted to the host record on the solver's stream and copied on
// a second stream, so only the copies of the last shifts to converge remain after the solve.  A solution that a
// later phase changes is reported again and copied again.  Pageable buffers are copied after the solve: a copy into
// pageable memory holds the calling thread, which would delay the solver's next launches.
struct SolutionCopy {
    char *d_x;
    size_t vb;  // device solutions, vb apart
    char *sg;
    size_t hrec;  // host-record staging, one slot per solution
    int hp;
    void *const *host_x;
    std::vector<char> sent;
    cudaError_t err;
};

static void copy_solution(kq_context *ctx, int k, void *user)
{
    auto *c = static_cast<SolutionCopy *>(user);
    if (c->err != cudaSuccess) return;
    cudaError_t e = cudaSuccess;
    // a staging slot is rewritten only after the copy that read it has completed
    if (c->sent[k]) e = cudaStreamWaitEvent(ctx->stream, ctx->copy_done, 0);
    if (e == cudaSuccess)
        e = spinor_to_record(ctx->g, c->d_x + k * c->vb, P64, c->sg + k * c->hrec, c->hp, ctx->stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->copy_ready, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_ready, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(c->host_x[k], c->sg + k * c->hrec, c->hrec, cudaMemcpyDeviceToHost, ctx->copy_stream);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->copy_done, ctx->copy_stream);
    c->sent[k] = 1;
    c->err = e;
}

static bool host_pinned(const void *ptr)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static cudaError_t ensure_copy_stream(kq_context *ctx)
{
    cudaError_t e = cudaSuccess;
    if (!ctx->copy_stream) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess && !ctx->copy_ready) e = cudaEventCreateWithFlags(&ctx->copy_ready, cudaEventDisableTiming);
    if (e == cudaSuccess && !ctx->copy_done) e = cudaEventCreateWithFlags(&ctx->copy_done, cudaEventDisableTiming);
    return e;
}

KQ_API KuQCDStatus kq_solve_multishift(kq_context *ctx, const kq_solve_param *p, const void *host_b,
                                       void *const *host_x, kq_solve_info *info)
{
    KuQCDStatus st = check_solve_param(ctx, p);
    if (st != KUQCD_SUCCESS) return st;
    if (!host_b || !host_x) return KUQCD_ERR_NULL_POINTER;
    for (int k = 0; k < p->num_shift; ++k)
        if (!host_x[k]) return KUQCD_ERR_NULL_POINTER;
    const int hp = prec_from_api(p->host_prec);
    if (hp != P64 && hp != P32) {
        set_last_error("solve: host precision must be DOUBLE or SINGLE");
        return KUQCD_ERR_INVALID_PARAM;
    }
    cudaSetDevice(ctx->device);
    const int halves = p->parity == KQ_PARITY_FULL ? 2 : 1;
    const size_t vb = spinor_bytes(ctx->g, P64) * halves;  // one (full-lattice or parity) field
    const size_t hvb = spinor_bytes(ctx->g, P64);            // one parity
    const size_t hrec = (size_t)ctx->g.vh * 6 * (hp == P64 ? 8 : 4);  // one parity host record
    // one context-owned buffer (kept between calls): b, the solutions, and the host-record staging of all fields
    const int nrec = p->num_shift * halves;
    const size_t fields = (size_t)vb * (1 + p->num_shift), need = fields + hrec * (size_t)nrec;
    if (ctx->io_bytes < need) {
        cudaStreamSynchronize(ctx->stream);
        if (ctx->io) cudaFree(ctx->io);
        ctx->io = nullptr;
        ctx->io_bytes = 0;
        cudaError_t ea = cudaMalloc(&ctx->io, need);
        if (ea != cudaSuccess) {
            set_last_error(std::string("kq_solve_multishift: ") + cudaGetErrorString(ea));
            return status_of(ea);
        }
        ctx->io_bytes = need;
    }
    char *base = static_cast<char *>(ctx->io);
    void *d_b = base, *d_x = base + vb;
    char *sg = base + fields;
    cudaError_t e = cudaSuccess;
    for (int h = 0; h < halves && e == cudaSuccess; ++h) {
        e = cudaMemcpyAsync(sg + h * hrec, static_cast<const char *>(host_b) + h * hrec, hrec, cudaMemcpyHostToDevice,
                            ctx->stream);
        if (e == cudaSuccess) e = spinor_from_record(ctx->g, sg + h * hrec, hp, static_cast<char *>(d_b) + h * hvb, P64,
                                                     ctx->stream);
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_solve_multishift: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    bool overlap = halves == 1;
    for (int k = 0; k < p->num_shift && overlap; ++k) overlap = host_pinned(host_x[k]);
    if (overlap && ensure_copy_stream(ctx) != cudaSuccess) {
        cudaGetLastError();
        overlap = false;
    }
    SolutionCopy cp{static_cast<char *>(d_x), vb, sg, hrec, hp, host_x, std::vector<char>(p->num_shift, 0),
                    cudaSuccess};
    if (overlap) {
        ctx->solution_ready = copy_solution;
        ctx->solution_ready_user = &cp;
    }
    st = kq_solve_multishift_device(ctx, p, d_b, d_x, info);
    ctx->solution_ready = nullptr;
    ctx->solution_ready_user = nullptr;
    if (info) info->copies_during_solve = (int)std::count(cp.sent.begin(), cp.sent.end(), 1);
    if (overlap && (st == KUQCD_SUCCESS || st == KUQCD_ERR_UNKNOWN_ERROR)) {
        // the solutions not reported during the solve
        for (int k = 0; k < p->num_shift; ++k)
            if (!cp.sent[k]) copy_solution(ctx, k, &cp);
        cudaError_t e2 = cp.err;
        if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(ctx->copy_stream);
        if (e2 != cudaSuccess) {
            set_last_error(std::string("kq_solve_multishift: ") + cudaGetErrorString(e2));
            st = status_of(e2);
        }
    } else if (st == KUQCD_SUCCESS || st == KUQCD_ERR_UNKNOWN_ERROR) {
        // every solution into host-record layout, then one copy per field and one sync
        cudaError_t e2 = cudaSuccess;
        for (int k = 0; k < p->num_shift && e2 == cudaSuccess; ++k)
            for (int h = 0; h < halves && e2 == cudaSuccess; ++h)
                e2 = spinor_to_record(ctx->g, static_cast<char *>(d_x) + k * vb + h * hvb, P64,
                                      sg + (size_t)(k * halves + h) * hrec, hp, ctx->stream);
        for (int k = 0; k < p->num_shift && e2 == cudaSuccess; ++k)
            for (int h = 0; h < halves && e2 == cudaSuccess; ++h)
                e2 = cudaMemcpyAsync(static_cast<char *>(host_x[k]) + h * hrec, sg + (size_t)(k * halves + h) * hrec,
                                     hrec, cudaMemcpyDeviceToHost, ctx->stream);
        if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(ctx->stream);
        if (e2 != cudaSuccess) {
            set_last_error(std::string("kq_solve_multishift: ") + cudaGetErrorString(e2));
            st = status_of(e2);
        }
    }
    // no copy into the caller's buffers may still be running when this returns
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamSynchronize(ctx->stream);
    return st;
}
