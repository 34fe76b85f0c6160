// kq_mdagm_noalloc: sigma*src - D_pq D_qp src without any device allocation.
//
// Who needs it: callers that cannot have the library allocate device memory while they run the operator.  Some
// applications reserve nearly all of HBM for their own memory pool at start-up, so a cudaMalloc here would fail or
// fragment their pool; others apply the operator inside a latency-critical loop, where cudaMalloc / cudaFree can
// synchronise the whole device.  kq_mdagm asks the caller for the parity-(1-p) temporary; this variant takes it from
// a fixed device array that every GPU loading the library holds from module load until process exit.
//
// Limits and sharing:
//   * the temporary needs kq_spinor_bytes(ctx, prec) bytes; anything above kStaticScratchBytes (32 MiB) is rejected
//     with KUQCD_ERR_INVALID_PARAM (FP64 up to 699,050 sites per parity, e.g. a 32^4 lattice);
//   * every call on a device uses the same array and leaves its last contents there; the first dslash overwrites
//     every site it later reads, so nothing has to start at zero -- but calls that overlap on the GPU (two streams,
//     two host threads) race on the array and must be serialised by the caller;
//   * the links must already be resident in `prec` (kq_load_links / kq_prepare_links): this call never converts or
//     allocates them;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress with that device
//     current) and caches it for the life of the process; make that first call before any stream capture.  A
//     cudaDeviceReset in the same process invalidates the cached address: do not call this entry point on a
//     device after resetting it.
#include <mutex>

#include "kq_context.h"
#include "kq_internal.h"

namespace kq {
cudaError_t launch_mdagm2(const Geom &g, const GaugeDev &gd, int lp, int sp, double sigma, const void *src,
                          void *tmp, void *dst, int parity, cudaStream_t s);
}

using namespace kq;

namespace {

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr int kMaxDevices = 64;

// The scratch itself.  In host code this name is only a stand-in for the symbol: its device address comes from
// cudaGetSymbolAddress below, never from taking the address here.
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of the scratch on the current device; looked up once per device.
cudaError_t scratch_address(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = p;
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) KuQCDStatus kq_mdagm_noalloc(kq_context *ctx, int prec,
                                                                                double sigma, const void *d_src,
                                                                                void *d_dst, int parity,
                                                                                void *stream)
{
    if (!ctx || !d_src || !d_dst) {
        set_last_error("kq_mdagm_noalloc: null pointer");
        return KUQCD_ERR_NULL_POINTER;
    }
    const int p = prec_from_api(prec);
    if (p < 0 || (parity != 0 && parity != 1)) {
        set_last_error("kq_mdagm_noalloc: invalid precision or parity");
        return KUQCD_ERR_INVALID_PARAM;
    }
    const size_t need = spinor_bytes(ctx->g, p);
    if (need > kStaticScratchBytes) {
        set_last_error("kq_mdagm_noalloc: lattice too large for the 32 MiB static scratch (needs " +
                       std::to_string(need) + " bytes); use kq_mdagm with a caller-provided temporary");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->gd.have[p]) {
        set_last_error("kq_mdagm_noalloc: links are not resident in this precision; call kq_prepare_links first");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    void *tmp = nullptr;
    if (e == cudaSuccess) e = scratch_address(ctx->device, &tmp);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_mdagm_noalloc: scratch lookup failed: ") + cudaGetErrorString(e));
        return KUQCD_ERR_UNKNOWN_ERROR;
    }
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
    e = launch_mdagm2(ctx->g, ctx->gd, p, p, sigma, d_src, tmp, d_dst, parity, s);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_mdagm_noalloc: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    return KUQCD_SUCCESS;
}
