// Internal declarations shared by the kuqcd_b200 CUDA translation units.
//
// Device data layout (one GPU, one lattice nx*ny*nz*nt, V sites, Vh = V/2 per parity):
//   checkerboard index  i = (x >> 1) + hx*(y + ny*(z + nz*t)),  hx = nx/2, x = 2*(i % hx) + ((y+z+t+parity) & 1)
//   (the reference's CB index, latt_base.cpp:170-212 / index_utils.cpp:91-100).
//
//   Spinor field of one parity (structure of arrays, one plane per "vector word", index = site):
//     FP64: 3 planes of double2  (colour c: re, im)                                         48 B/site
//     FP32: plane0 float4 (c0.re c0.im c1.re c1.im), plane1 float2 (c2.re c2.im)            24 B/site
//     HALF: 1 plane of int4 = 6 x int16 fixed point (value/norm * 32767) + float norm         16 B/site
//   Link field (fat or long) of one parity, 4 directions:
//     FP64: [dir][9 complex][site] double2                                                 144 B/link
//     FP32: [dir][4 x float4 + 1 x float2][site]  (18 floats, row-major)                    72 B/link
//     HALF: [dir][2 x int4 + 1 x int (2 x int16)][site], value = q * scale / 32767          36 B/link
//   Device links carry the reference kernel's constants: fat_dev = 1/2 * F, long_dev = c3 * L with
//   c3 = -1/48 (dirac_hisq.cpp:40,464-502), so the dslash is a plain sum of U v and U^dag v products.
//   Long links that are a real multiple of an SU(3) matrix, L = s W (HISQ's Naik links are products of
//   reunitarised links), are stored compressed: rows 0 and 1 and 1/s, row 2 = conj(row0 x row1) / s:
//     FP64: [dir][6 x double2 + 1 x double][site]                                          104 B/link
//     FP32: [dir][3 x float4 + 1 x float][site]                                              52 B/link
#pragma once
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <string>

#include <nvtx3/nvToolsExt.h>

#include "kuqcd_b200.h"

namespace kq {

// NVTX range for the host side of a phase (header-only NVTX 3: a no-op unless a profiler is attached), so that
// traces and ncu's --nvtx filters can pick out solver phases, batched solves and network steps
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

enum Prec { P64 = 0, P32 = 1, P16 = 2 };

inline int prec_from_api(int api_prec)
{
    // KuQCDPrecision values (kuqcd_enum.h:40-45): HALF = 2, SINGLE = 4, DOUBLE = 8
    return api_prec == 8 ? P64 : api_prec == 4 ? P32 : api_prec == 2 ? P16 : -1;
}

struct Geom {
    int n[4];      // nx ny nz nt
    int hx;        // nx / 2
    int vh;        // sites per parity
    int sy, sz, st;  // checkerboard strides of y, z, t: hx, hx*ny, hx*ny*nz
};

Geom make_geom(const unsigned lat[4]);

// sizes (bytes) of one parity field in the device layout
size_t spinor_bytes(const Geom &g, int prec);
size_t links_bytes(const Geom &g, int prec);  // one parity, 4 directions

// ---------------------------------------------------------------------------------------------------------------
// device views
struct SpinorView {
    void *p;  // base of the parity field
    int prec;
};

struct LinkSet {          // one link type (fat or long) in one precision, both parities
    void *par[2];         // device pointer per parity
    float scale;          // HALF only: value = q * scale / 32767
    int recon;            // FP64 / FP32 only: 1 = two rows + 1/s per link, the third row rebuilt (kq_prec.cuh);
                          // 0 in a value-initialised context, set by every link writer
};

struct GaugeDev {
    bool have[3] = {false, false, false};
    LinkSet fat[3], lng[3];   // per precision
    void *block[3] = {nullptr, nullptr, nullptr};  // one allocation per precision holding both link types
};

// ---------------------------------------------------------------------------------------------------------------
// kernels / launchers (stream = cudaStream_t)
// dst(parity p) = D src(parity 1-p)
cudaError_t launch_dslash(const Geom &g, const GaugeDev &gd, int prec, const void *src, void *dst, int dst_parity,
                          cudaStream_t s, int block = 0);

// Fused second half of (sigma - D D): s = sigma * p - D_pq tmp; and the deterministic partial sums of Re<p,s>
// (FP64) over blocks; the last block to finish calls `finish` (see kq_cgm.cu) through the state pointer.
struct CgmState;
cudaError_t launch_dslash_axmy_dot(const Geom &g, const GaugeDev &gd, int prec, const void *tmp, const void *p,
                                   void *s_out, int parity, CgmState *st, cudaStream_t s);

// layout conversion (host records staged on the device, kuqcd.cpp:103-169 layouts)
// `scratch` is one device word used for the HALF scale reduction.
cudaError_t links_from_host_record(const Geom &g, const void *d_rec, int rec_prec, double factor, LinkSet &out,
                                   int out_prec, unsigned *scratch, cudaStream_t s);
cudaError_t links_convert(const Geom &g, const LinkSet &in, int in_prec, LinkSet &out, int out_prec,
                          unsigned *scratch, cudaStream_t s);
float links_absmax(const Geom &g, const LinkSet &in, int in_prec, unsigned *scratch, cudaStream_t s);
// store an FP64 / FP32 link set compressed (two rows + 1/s) in place if every link is a real multiple of an SU(3)
// matrix to relative accuracy tol; *done reports whether it did
cudaError_t links_compress(const Geom &g, LinkSet &lk, int prec, double tol, unsigned *scratch, cudaStream_t s,
                           bool *done);
cudaError_t spinor_from_record(const Geom &g, const void *d_rec, int rec_prec, void *dst, int prec, cudaStream_t s);
cudaError_t spinor_to_record(const Geom &g, const void *src, int prec, void *d_rec, int rec_prec, cudaStream_t s);
cudaError_t spinor_convert(const Geom &g, const void *src, int src_prec, void *dst, int dst_prec, cudaStream_t s);

// generators of the synthetic benchmark fields, on the device
cudaError_t make_links_record(const Geom &g, double eps, uint64_t seed, double *d_fat_rec, double *d_long_rec,
                              cudaStream_t s);
cudaError_t make_source_record(const Geom &g, int parity, uint64_t seed, double *d_rec, cudaStream_t s);

// error helpers
void set_last_error(const std::string &msg);
const char *last_error();

#define KQ_CUDA_TRY(expr)                                                                    \
    do {                                                                                      \
        cudaError_t kq_e_ = (expr);                                                           \
        if (kq_e_ != cudaSuccess) {                                                           \
            ::kq::set_last_error(std::string(#expr) + ": " + cudaGetErrorString(kq_e_));      \
            return kq_e_;                                                                     \
        }                                                                                     \
    } while (0)

}  // namespace kq
