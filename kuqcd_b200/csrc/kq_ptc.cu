// Gauge-covariant parallel-transport convolution (PTC) network: the learned preconditioner of the FCG polish.
// (No reference counterpart: the reference has no preconditioner, inverter_cgm.cpp:17-87.)
//
// Field of C channels on the full lattice (both parities), activation layout: plane ((c*2 + parity)*3 + colour) of
// float2 (re, im) per checkerboard site, planes pv sites apart.  One layer, C_in -> C_out channels:
//
//   y_o(x) = sum_i sum_p W[o][i][p] (T_p v_i)(x)
//   T_0 = 1,  T_{1+2mu} v (x) = F_mu(x) v(x+mu),  T_{2+2mu} v (x) = F_mu(x-mu)^dag v(x-mu)
//
// with the FP32 device fat links F (they carry the dslash's factor 1/2) and complex weights W.  Per tile of 128
// sites of one parity the transported inputs are gathered in FP32 and rounded to BF16 into shared memory; the
// channel mixing is then a real GEMM per colour, [128 x K] x [K x N] with K = 9 paths x C_in x (re, im) in the
// order k = (p * C_in + i) * 2 + reim and N = C_out * 2 (padded to 16).  Forward layers run it on the
// fifth-generation tensor cores: one thread issues tcgen05.mma (BF16 operands in shared memory in the canonical
// K-major layout, FP32 accumulators in tensor memory, M = 128, N = 16, K = 16 per instruction) for the three
// colours, and the epilogue reads the accumulators back with tcgen05.ld, one site row per thread.  The adjoint layer
// (for input gradients) is the same kernel with weights W'[i][o][p'] = conj(W[o][i][p]) and forward/backward hops
// swapped.  The weight gradient dL/dB = T^T G is also a tcgen05 GEMM, reading the same gathered tile MN-major
// (M = k, K = sites) with the accumulator kept in tensor memory across a persistent CTA's tiles; the per-CTA
// partials are summed in a fixed order.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_ptc.h"
#include "kq_umma.cuh"

namespace kq {

constexpr int kTile = 128;  // sites per CTA
constexpr int kThr = 128;   // threads per CTA (4 warps)
constexpr int kPaths = 9;

__host__ __device__ constexpr int kpad_of(int cin) { return ((cin * kPaths * 2 + 15) / 16) * 16; }
__host__ __device__ constexpr int npad_of(int cout) { return ((cout * 2 + 7) / 8) * 8; }

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}


__device__ __forceinline__ float2 ld_act(const float2 *act, int pv, int c, int par, int a, int i)
{
    return __ldg(act + (size_t)((c * 2 + par) * 3 + a) * pv + i);
}

// Gather the transported inputs of site i (parity par) path by path: emit(p, vals) with vals[a][2 c + reim] the
// colour-a component of (T_p v_c)(x), i.e. GEMM columns k = p * 2 CIN + 2 c + reim.
template <int CIN, typename Emit>
__device__ __forceinline__ void gather_paths(const Geom &g, int pv, const LinkSet &fat, const float2 *act, int par,
                                             int i, bool swap_paths, Emit emit)
{
    const SiteCoord cd = site_coord(g, i, par);
    const int q = 1 - par;
    const void *fat_p = par ? fat.par[1] : fat.par[0];
    const void *fat_q = par ? fat.par[0] : fat.par[1];
    float vals[3][2 * CIN];
    // identity path
#pragma unroll
    for (int c = 0; c < CIN; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float2 v = ld_act(act, pv, c, par, a, i);
            vals[a][2 * c] = v.x;
            vals[a][2 * c + 1] = v.y;
        }
    emit(0, vals);
#pragma unroll 1
    for (int dir = 0; dir < 4; ++dir) {
#pragma unroll
        for (int fb = 0; fb < 2; ++fb) {
            // fb = 0: forward hop F(x) v(x+mu); fb = 1: backward hop F(x-mu)^dag v(x-mu)
            const int nb = nbr_index(g, cd, i, dir, fb == 0 ? 1 : -1);
            float u[18];
            ld_link<1>(fb == 0 ? fat_p : fat_q, pv, dir, fb == 0 ? i : nb, 1.f, u);
            // adjoint layers run the hops with swapped path labels
            const int p = 1 + 2 * dir + (swap_paths ? 1 - fb : fb);
#pragma unroll
            for (int c = 0; c < CIN; ++c) {
                float v[6], o[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float2 w = ld_act(act, pv, c, q, a, nb);
                    v[2 * a] = w.x;
                    v[2 * a + 1] = w.y;
                }
                if (fb == 0) mv_add(u, v, o);
                else {
                    mdv_sub(u, v, o);
#pragma unroll
                    for (int k = 0; k < 6; ++k) o[k] = -o[k];
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    vals[a][2 * c] = o[2 * a];
                    vals[a][2 * c + 1] = o[2 * a + 1];
                }
            }
            emit(p, vals);
        }
    }
}

// ---------------------------------------------------------------------------------------------------- forward
// Gathered inputs of one 128-site tile into shared memory as BF16, one [128 sites x KP] matrix per colour in the
// canonical core-matrix layout (8 sites x 16 bytes of k per core matrix; k-chunks 128 bytes apart, 8-site groups
// (KP/8)*128 bytes apart).  The forward GEMM reads it K-major (M = sites), the weight-gradient GEMM MN-major
// (M = k, K = sites).  Thread t owns site base + t; sites past the end of the lattice are zero rows.
template <int CIN>
__device__ __forceinline__ void gather_tile(const Geom &g, int pv, const LinkSet &fat, const float2 *in, int par,
                                            int base, int t, bool swap_paths, unsigned char *As)
{
    constexpr int KP = kpad_of(CIN), KV = CIN * kPaths * 2;
    constexpr uint32_t A_BYTES = kTile * KP * 2;
    const int i = base + t;
    if (i < g.vh) {
        gather_paths<CIN>(g, pv, fat, in, par, i, swap_paths, [&](int p, const float (&vals)[3][2 * CIN]) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                unsigned char *row = As + a * A_BYTES;
                if constexpr (CIN == 8) {
                    // 16 columns = two core-matrix rows of 16 bytes
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        uint4 w;
                        w.x = pack_bf16(vals[a][8 * h + 0], vals[a][8 * h + 1]);
                        w.y = pack_bf16(vals[a][8 * h + 2], vals[a][8 * h + 3]);
                        w.z = pack_bf16(vals[a][8 * h + 4], vals[a][8 * h + 5]);
                        w.w = pack_bf16(vals[a][8 * h + 6], vals[a][8 * h + 7]);
                        *reinterpret_cast<uint4 *>(row + umma::kmajor_offset(t, p * 16 + 8 * h, KP)) = w;
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 2 * CIN; j += 2)
                        *reinterpret_cast<uint32_t *>(row + umma::kmajor_offset(t, p * 2 * CIN + j, KP)) =
                            pack_bf16(vals[a][j], vals[a][j + 1]);
                }
            }
        });
#pragma unroll
        for (int a = 0; a < 3; ++a)
            for (int k = KV; k < KP; k += 2)
                *reinterpret_cast<uint32_t *>(As + a * A_BYTES + umma::kmajor_offset(t, k, KP)) = 0u;
    } else {
#pragma unroll
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < KP; k += 8)
                *reinterpret_cast<uint4 *>(As + a * A_BYTES + umma::kmajor_offset(t, k, KP)) = make_uint4(0, 0, 0, 0);
    }
}

// out (C_out channels, both parities) = layer(in); Bt: [NP][KP] BF16 weights (device), built by the host.
// fault: set when the tensor cores did not signal completion within the wait limit (the tile is then not written).
constexpr int kNT = 16;                      // N of the tensor-core tile (C_out * 2 padded)
constexpr uint32_t kTmemCols = 64;           // 3 colours x 16 FP32 accumulator columns, rounded up
constexpr uint32_t kWaitLimit = 1u << 24;    // mbarrier polls before a tile gives up

template <int CIN, int COUT>
__global__ void __launch_bounds__(kThr) ptc_forward_kernel(Geom g, int pv, LinkSet fat, const float2 *__restrict__ in,
                                                           float2 *__restrict__ out, const __nv_bfloat16 *__restrict__ Bt,
                                                           int swap_paths, int *fault)
{
    constexpr int KP = kpad_of(CIN), NP = npad_of(COUT);
    constexpr uint32_t A_BYTES = kTile * KP * 2;   // one colour's [128 x KP] operand
    constexpr uint32_t SBO = (KP / 8) * 128;       // bytes between 8-row groups
    static_assert(NP <= kNT && KP % 16 == 0, "tile shape");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *As = smem_raw;                  // [3][A_BYTES]
    unsigned char *Bs = As + 3 * A_BYTES;          // [kNT x KP]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + kNT * KP * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    // tiles in parity-interleaved order (block 2j: tile j of parity 0, block 2j + 1: tile j of parity 1): the two
    // uses of every link (forward hop at its site, backward hop at the neighbour) and of every activation (own
    // site, eight neighbours) then fall close together in time and the second one hits L2
    const int par = blockIdx.x & 1;
    const int base = (blockIdx.x >> 1) * kTile;
    const int t = threadIdx.x, warp = t >> 5;
    if (warp == 0) umma::tmem_alloc(tslot, kTmemCols);
    if (t == 0) {
        umma::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int e = t; e < kNT * KP; e += kThr) {
        const int n = e / KP, k = e - n * KP;
        *reinterpret_cast<__nv_bfloat16 *>(Bs + umma::kmajor_offset(n, k, KP)) =
            n < NP ? Bt[n * KP + k] : __float2bfloat16_rn(0.f);
    }
    gather_tile<CIN>(g, pv, fat, in, par, base, t, swap_paths != 0, As);
    umma::fence_smem_to_async();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = *tslot;
    if (t == 0) {
        constexpr uint32_t idesc = umma::idesc_bf16_f32(kTile, kNT);
        const uint32_t a0 = umma::smem_u32(As), b0 = umma::smem_u32(Bs);
#pragma unroll 1
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int ks = 0; ks < KP / 16; ++ks)
                umma::mma_bf16(tbase + a * kNT, umma::smem_desc(a0 + a * A_BYTES + ks * 256, SBO),
                               umma::smem_desc(b0 + ks * 256, SBO), idesc, ks > 0 ? 1u : 0u);
        umma::mma_commit(mbar);
    }
    bool ok = umma::mbar_wait(mbar, 0, kWaitLimit);
    ok = __syncthreads_and(ok);
    if (!ok) {
        if (t == 0) atomicExch(fault, 1);
        umma::mbar_wait(mbar, 0, kWaitLimit);  // give the MMAs in flight a last chance before freeing their memory
    }
    umma::fence_after_sync();
    if (ok) {
        const int site = base + t;  // tensor-memory lane t = row t of the tile
#pragma unroll 1
        for (int a = 0; a < 3; ++a) {
            float d[16];
            umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + a * kNT, d);
            if (site < g.vh) {
#pragma unroll
                for (int o = 0; o < COUT; ++o)
                    out[(size_t)((o * 2 + par) * 3 + a) * pv + site] = make_float2(d[2 * o], d[2 * o + 1]);
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tbase, kTmemCols);
}

// Forward layer with 8 input channels, K-chunked by path: K = 9 paths x 16 columns, and each path's 16 columns of
// the gathered tile are one K = 16 step of the MMA.  The CTA gathers path j into one of two chunk buffers while the
// tensor cores multiply chunk j - 1 from the other, so shared memory holds 2 x 3 x [128 x 16] BF16 (24 KB) instead
// of the whole [128 x 144] tile per colour (108 KB): five or more CTAs fit on an SM and hide each other's gather
// latency.  Chunk j's MMAs commit to mbarrier (j & 1); before chunk j + 2 overwrites that buffer every thread waits
// for the commit's phase (j >> 1) & 1 (bounded, as in the whole-tile kernel).
constexpr uint32_t kChunkColBytes = kTile * 16 * 2;  // one colour's [128 x 16] BF16 chunk
template <int COUT, int MINB>
__global__ void __launch_bounds__(kThr, MINB) ptc_forward8_kernel(Geom g, int pv, LinkSet fat, const float2 *__restrict__ in,
                                                            float2 *__restrict__ out, const __nv_bfloat16 *__restrict__ Bt,
                                                            int swap_paths, int *fault)
{
    constexpr int CIN = 8, KP = kpad_of(CIN), NP = npad_of(COUT);
    constexpr uint32_t CH_BYTES = 3 * kChunkColBytes;  // one chunk: 3 colours
    constexpr uint32_t SBO_A = (16 / 8) * 128, SBO_B = (KP / 8) * 128;
    static_assert(KP == kPaths * 16 && NP <= kNT, "one path per K step");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *Ach = smem_raw;                  // [2][3][kChunkColBytes]
    unsigned char *Bs = Ach + 2 * CH_BYTES;         // [kNT x KP]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Bs + kNT * KP * 2);  // [2]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 2);
    const int par = blockIdx.x & 1;  // parity-interleaved tile order (see ptc_forward_kernel)
    const int base = (blockIdx.x >> 1) * kTile;
    const int t = threadIdx.x, warp = t >> 5;
    if (warp == 0) umma::tmem_alloc(tslot, kTmemCols);
    if (t == 0) {
        umma::mbar_init(&mbar[0], 1);
        umma::mbar_init(&mbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int e = t; e < kNT * KP; e += kThr) {
        const int n = e / KP, k = e - n * KP;
        *reinterpret_cast<__nv_bfloat16 *>(Bs + umma::kmajor_offset(n, k, KP)) =
            n < NP ? Bt[n * KP + k] : __float2bfloat16_rn(0.f);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = *tslot;
    const int i = base + t;
    const bool valid = i < g.vh;
    const SiteCoord cd = site_coord(g, valid ? i : 0, par);
    const int q = 1 - par;
    const void *fat_p = par ? fat.par[1] : fat.par[0];
    const void *fat_q = par ? fat.par[0] : fat.par[1];
    constexpr uint32_t idesc = umma::idesc_bf16_f32(kTile, kNT);
    const uint32_t a0 = umma::smem_u32(Ach), b0 = umma::smem_u32(Bs);
    bool ok = true;
#pragma unroll 1
    for (int j = 0; j < kPaths && ok; ++j) {
        const int buf = j & 1;
        if (j >= 2) {  // the MMAs of chunk j - 2 must be done reading this buffer
            ok = __syncthreads_and(umma::mbar_wait(&mbar[buf], ((j - 2) >> 1) & 1, kWaitLimit));
            if (!ok) break;
            umma::fence_after_sync();
        }
        // path j: identity, then for each direction the forward and the backward hop
        int p = 0;
        float vals[3][2 * CIN];
        if (j == 0) {
#pragma unroll
            for (int c = 0; c < CIN; ++c)
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float2 v = valid ? ld_act(in, pv, c, par, a, i) : make_float2(0.f, 0.f);
                    vals[a][2 * c] = v.x;
                    vals[a][2 * c + 1] = v.y;
                }
        } else {
            const int dir = (j - 1) >> 1, fb = (j - 1) & 1;
            p = 1 + 2 * dir + (swap_paths ? 1 - fb : fb);
            if (valid) {
                const int nb = nbr_index(g, cd, i, dir, fb == 0 ? 1 : -1);
                float u[18];
                ld_link<1>(fb == 0 ? fat_p : fat_q, pv, dir, fb == 0 ? i : nb, 1.f, u);
#pragma unroll
                for (int c = 0; c < CIN; ++c) {
                    float v[6], o[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const float2 w = ld_act(in, pv, c, q, a, nb);
                        v[2 * a] = w.x;
                        v[2 * a + 1] = w.y;
                    }
                    if (fb == 0) mv_add(u, v, o);
                    else {
                        mdv_sub(u, v, o);
#pragma unroll
                        for (int k = 0; k < 6; ++k) o[k] = -o[k];
                    }
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        vals[a][2 * c] = o[2 * a];
                        vals[a][2 * c + 1] = o[2 * a + 1];
                    }
                }
            } else {
#pragma unroll
                for (int a = 0; a < 3; ++a)
#pragma unroll
                    for (int k = 0; k < 2 * CIN; ++k) vals[a][k] = 0.f;
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            unsigned char *col = Ach + buf * CH_BYTES + a * kChunkColBytes;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint4 w;
                w.x = pack_bf16(vals[a][8 * h + 0], vals[a][8 * h + 1]);
                w.y = pack_bf16(vals[a][8 * h + 2], vals[a][8 * h + 3]);
                w.z = pack_bf16(vals[a][8 * h + 4], vals[a][8 * h + 5]);
                w.w = pack_bf16(vals[a][8 * h + 6], vals[a][8 * h + 7]);
                *reinterpret_cast<uint4 *>(col + umma::kmajor_offset(t, 8 * h, 16)) = w;
            }
        }
        umma::fence_smem_to_async();
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
        if (t == 0) {
#pragma unroll
            for (int a = 0; a < 3; ++a)
                umma::mma_bf16(tbase + a * kNT, umma::smem_desc(a0 + buf * CH_BYTES + a * kChunkColBytes, SBO_A),
                               umma::smem_desc(b0 + p * 256, SBO_B), idesc, j > 0 ? 1u : 0u);
            umma::mma_commit(&mbar[buf]);
        }
    }
    // the last two chunks (7 on buffer 1, 8 on buffer 0) complete their barriers' phases 1 and 0
    if (ok) ok = __syncthreads_and(umma::mbar_wait(&mbar[1], 1, kWaitLimit) && umma::mbar_wait(&mbar[0], 0, kWaitLimit));
    if (!ok) {
        if (t == 0) atomicExch(fault, 1);
        // give the MMAs in flight a last chance before freeing their memory
        umma::mbar_wait(&mbar[0], 0, kWaitLimit);
        umma::mbar_wait(&mbar[1], 1, kWaitLimit);
    }
    umma::fence_after_sync();
    if (ok) {
#pragma unroll 1
        for (int a = 0; a < 3; ++a) {
            float d[16];
            umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + a * kNT, d);
            if (valid) {
#pragma unroll
                for (int o = 0; o < COUT; ++o)
                    out[(size_t)((o * 2 + par) * 3 + a) * pv + i] = make_float2(d[2 * o], d[2 * o + 1]);
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tbase, kTmemCols);
}

// ---------------------------------------------------------------------------------------------------- weight grad
// partial[cta][k][n] = sum over the tiles this CTA visits (tile = blockIdx.x + j * gridDim.x) and over their rows
// (sites x colours) of T[row][k] * G[row][n]  (swap_paths: T gathered as by the adjoint layer).
// Persistent: the accumulator D (M = k, N = 16) stays in tensor memory across all of the CTA's tiles.  A is the
// gathered tile read MN-major (M = k, K = sites); B = G, [site][n] in 8 x 16-byte core matrices, also MN-major.
// With KP = 144 two M tiles cover k < 256; the rows of D past KP read neighbouring data and are never stored.
template <int CIN, int COUT>
__global__ void __launch_bounds__(kThr) ptc_wgrad_kernel(Geom g, int pv, LinkSet fat, const float2 *__restrict__ in,
                                                         const float2 *__restrict__ gout, float *__restrict__ partial,
                                                         int swap_paths, int *fault)
{
    constexpr int KP = kpad_of(CIN), NP = npad_of(COUT), MT = (KP + 127) / 128;
    constexpr uint32_t A_BYTES = kTile * KP * 2, G_BYTES = kTile * kNT * 2;
    constexpr uint32_t A_GROUP = (KP / 8) * 128, G_GROUP = (kNT / 8) * 128;  // bytes between 8-site groups
    static_assert(NP <= kNT && MT <= 2, "tile shape");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char *As = smem_raw;             // [3][A_BYTES]
    unsigned char *Gs = As + 3 * A_BYTES;     // [3][G_BYTES]
    uint64_t *mbar = reinterpret_cast<uint64_t *>(Gs + 3 * G_BYTES);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    const int ntiles = 2 * ((g.vh + kTile - 1) / kTile);
    const int t = threadIdx.x, warp = t >> 5;
    if (warp == 0) umma::tmem_alloc(tslot, 32);
    if (t == 0) {
        umma::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tbase = *tslot;
    bool ok = true;
    int round = 0;
    for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x, ++round) {
        if (round > 0) {  // the previous tile's MMAs must be done reading shared memory
            ok = __syncthreads_and(umma::mbar_wait(mbar, (round - 1) & 1, kWaitLimit));
            if (!ok) break;
            umma::fence_after_sync();
        }
        const int par = tile & 1;  // parity-interleaved tile order, as in the forward kernels
        const int base = (tile >> 1) * kTile;
        gather_tile<CIN>(g, pv, fat, in, par, base, t, swap_paths != 0, As);
        const int i = base + t;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float gv[kNT];
#pragma unroll
            for (int o = 0; o < kNT / 2; ++o) {
                float2 w = make_float2(0.f, 0.f);
                if (o < COUT && i < g.vh) w = ld_act(gout, pv, o, par, a, i);
                gv[2 * o] = w.x;
                gv[2 * o + 1] = w.y;
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                uint4 w;
                w.x = pack_bf16(gv[8 * h + 0], gv[8 * h + 1]);
                w.y = pack_bf16(gv[8 * h + 2], gv[8 * h + 3]);
                w.z = pack_bf16(gv[8 * h + 4], gv[8 * h + 5]);
                w.w = pack_bf16(gv[8 * h + 6], gv[8 * h + 7]);
                *reinterpret_cast<uint4 *>(Gs + a * G_BYTES + (t >> 3) * G_GROUP + h * 128 + (t & 7) * 16) = w;
            }
        }
        umma::fence_smem_to_async();
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
        if (t == 0) {
            constexpr uint32_t idesc = umma::idesc_bf16_f32(128, kNT, true, true);
            const uint32_t a0 = umma::smem_u32(As), b0 = umma::smem_u32(Gs);
#pragma unroll 1
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int ks = 0; ks < kTile / 16; ++ks)
#pragma unroll
                    for (int mt = 0; mt < MT; ++mt)
                        umma::mma_bf16(tbase + mt * kNT,
                                       umma::smem_desc2(a0 + a * A_BYTES + 2 * ks * A_GROUP + mt * 16 * 128, A_GROUP, 128),
                                       umma::smem_desc2(b0 + a * G_BYTES + 2 * ks * G_GROUP, G_GROUP, 128), idesc,
                                       (round > 0 || a > 0 || ks > 0) ? 1u : 0u);
            umma::mma_commit(mbar);
        }
    }
    if (ok && round > 0) ok = __syncthreads_and(umma::mbar_wait(mbar, (round - 1) & 1, kWaitLimit));
    if (!ok) {
        if (t == 0) atomicExch(fault, 1);
        umma::mbar_wait(mbar, (round - 1) & 1, kWaitLimit);  // a last chance for MMAs in flight
    }
    umma::fence_after_sync();
    float *out = partial + (size_t)blockIdx.x * KP * NP;
    if (ok) {
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
            float d[16];
            umma::tmem_ld16(tbase + ((uint32_t)(warp * 32) << 16) + mt * kNT, d);  // lane = row k of this M tile
            const int k = mt * 128 + warp * 32 + (t & 31);
            if (k < KP) {
#pragma unroll
                for (int n = 0; n < NP; ++n) out[(size_t)k * NP + n] = round > 0 ? d[n] : 0.f;
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tbase, 32);
}

// fixed-order sum of the per-tile partials: dB[e] = sum_tile partial[tile][e]
__global__ void ptc_reduce_kernel(const float *__restrict__ partial, int ntiles, int nelem, float *__restrict__ dB)
{
    __shared__ double sm[32];
    for (int e = blockIdx.x; e < nelem; e += gridDim.x) {
        double s = 0.0;
        for (int b = threadIdx.x; b < ntiles; b += blockDim.x) s += partial[(size_t)b * nelem + e];
        s = block_sum(s, sm);
        if (threadIdx.x == 0) dB[e] = (float)s;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------- glue kernels
// embed an FP64 parity field into channel 0 of a full-lattice activation (other parity zero)
__global__ void ptc_embed_kernel(int vh, int pv, const void *__restrict__ src, int parity, float2 *__restrict__ act,
                                 double scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vh) return;
    double v[6];
    ld_spinor<0>(src, pv, i, v);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        act[(size_t)(parity * 3 + a) * pv + i] = make_float2((float)(scale * v[2 * a]), (float)(scale * v[2 * a + 1]));
        act[(size_t)((1 - parity) * 3 + a) * pv + i] = make_float2(0.f, 0.f);
    }
}

// channel 0, parity `parity` of an activation -> FP64 parity field (times scale)
__global__ void ptc_extract_kernel(int vh, int pv, const float2 *__restrict__ act, int parity, void *__restrict__ dst,
                                   double scale)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= vh) return;
    double v[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float2 w = act[(size_t)(parity * 3 + a) * pv + i];
        v[2 * a] = scale * w.x;
        v[2 * a + 1] = scale * w.y;
    }
    st_spinor<0>(dst, pv, i, v);
}

// loss and output gradient of one pair: L = |y - e|^2 / |e|^2 on the parity sites; G = 2 (y - e) / |e|^2 there,
// zero on the other parity.  y = channel 0 of the last activation; e an FP64 parity field.
__global__ void ptc_loss_kernel(int vh, int pv, const float2 *__restrict__ y, const void *__restrict__ e, int parity,
                                double inv_e2, float2 *__restrict__ gout, double *partials)
{
    __shared__ double sm[32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0;
    if (i < vh) {
        double ev[6];
        ld_spinor<0>(e, pv, i, ev);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float2 w = y[(size_t)(parity * 3 + a) * pv + i];
            const double dr = w.x - ev[2 * a], di = w.y - ev[2 * a + 1];
            l += dr * dr + di * di;
            gout[(size_t)(parity * 3 + a) * pv + i] = make_float2((float)(2 * dr * inv_e2), (float)(2 * di * inv_e2));
            gout[(size_t)((1 - parity) * 3 + a) * pv + i] = make_float2(0.f, 0.f);
        }
    }
    l = block_sum(l * inv_e2, sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = l;
}

// Adam on grad * grad_scale (the accumulated gradient of a batch times 1/batch); the accumulator is cleared here, so
// the next batch starts from zero without a separate memset
__global__ void ptc_adam_kernel(float *w, float *grad, float *m, float *v, int n, float lr, float grad_scale, float b1,
                                float b2, float eps, int step)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const float gk = grad[k] * grad_scale;
    grad[k] = 0.0f;
    m[k] = b1 * m[k] + (1 - b1) * gk;
    v[k] = b2 * v[k] + (1 - b2) * gk * gk;
    const float mh = m[k] / (1 - powf(b1, (float)step)), vh = v[k] / (1 - powf(b2, (float)step));
    w[k] -= lr * mh / (sqrtf(vh) + eps);
}

// ---------------------------------------------------------------------------------------------------- host side
template <int CIN, int COUT>
static size_t fwd_smem() { return (size_t)(3 * kTile + kNT) * kpad_of(CIN) * 2 + 16; }
// operands + barrier words, plus one colour's worth of slack: the MMAs of the second M tile read up to a site
// group past the last colour's A block, and the slack keeps every operand read inside the allocation whatever the
// stride order of the descriptor
template <int CIN, int COUT>
static size_t wgrad_smem() { return (size_t)3 * kTile * (kpad_of(CIN) + kNT) * 2 + 16 + (size_t)kTile * kpad_of(CIN) * 2; }

// device word the forward kernels set when a tile's tensor-core work did not complete in time
__device__ int g_ptc_fault;

static int *fault_flag()
{
    static int *ptr[64] = {nullptr};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return nullptr;
    if (!ptr[dev] && cudaGetSymbolAddress(reinterpret_cast<void **>(&ptr[dev]), g_ptc_fault) != cudaSuccess)
        ptr[dev] = nullptr;
    return ptr[dev];
}

cudaError_t ptc_check_fault(cudaStream_t s)
{
    int *f = fault_flag();
    if (!f) return cudaErrorInvalidDevicePointer;
    int h = 0;
    KQ_CUDA_TRY(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, s));
    KQ_CUDA_TRY(cudaStreamSynchronize(s));
    if (h) {
        // the word reports this call's failure once; cleared so that the next call starts clean
        KQ_CUDA_TRY(cudaMemsetAsync(f, 0, sizeof(int), s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        set_last_error("ptc: tensor-core tile did not complete within the wait limit");
        return cudaErrorLaunchTimeout;
    }
    return cudaSuccess;
}

cudaError_t ptc_raise_fault_for_test()
{
    int *f = fault_flag();
    if (!f) return cudaErrorInvalidDevicePointer;
    const int one = 1;
    return cudaMemcpy(f, &one, sizeof(int), cudaMemcpyHostToDevice);
}

// Resident CTAs per SM the 8-channel kernel is compiled for (KUQCD_PTC_CTAS = 4 .. 7; 64 TMEM columns and 29 KB of
// shared memory each, so 7 fit the SM's 512 columns and 228 KB).  The gather is latency-bound: six CTAs at 80
// registers (8 B spilled) apply M in 1.50 ms at 32^4 against 1.79 ms for four at 128.
static int ptc_ctas()
{
    static const int k = [] {
        const char *e = getenv("KUQCD_PTC_CTAS");
        const int v = e ? atoi(e) : 6;
        return v >= 4 && v <= 7 ? v : 6;
    }();
    return k;
}

template <int COUT, int MINB>
static cudaError_t run_forward8_b(const Geom &g, const LinkSet &fat, const float2 *in, float2 *out,
                                  const __nv_bfloat16 *Bt, bool swap, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int tiles = 2 * ((g.vh + kTile - 1) / kTile);
    const size_t sm = (size_t)2 * 3 * kChunkColBytes + (size_t)kNT * kpad_of(8) * 2 + 32;
    KQ_CUDA_TRY(cudaFuncSetAttribute(ptc_forward8_kernel<COUT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
    int *fault = fault_flag();
    if (!fault) return cudaErrorInvalidDevicePointer;
    ptc_forward8_kernel<COUT, MINB><<<tiles, kThr, sm, s>>>(g, pv, fat, in, out, Bt, swap ? 1 : 0, fault);
    return cudaGetLastError();
}

template <int COUT>
static cudaError_t run_forward8(const Geom &g, const LinkSet &fat, const float2 *in, float2 *out,
                                const __nv_bfloat16 *Bt, bool swap, cudaStream_t s)
{
    switch (ptc_ctas()) {
        case 4: return run_forward8_b<COUT, 4>(g, fat, in, out, Bt, swap, s);
        case 5: return run_forward8_b<COUT, 5>(g, fat, in, out, Bt, swap, s);
        case 7: return run_forward8_b<COUT, 7>(g, fat, in, out, Bt, swap, s);
        default: return run_forward8_b<COUT, 6>(g, fat, in, out, Bt, swap, s);
    }
}

template <int CIN, int COUT>
static cudaError_t run_forward(const Geom &g, const LinkSet &fat, const float2 *in, float2 *out,
                               const __nv_bfloat16 *Bt, bool swap, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int tiles = 2 * ((g.vh + kTile - 1) / kTile);
    const size_t sm = fwd_smem<CIN, COUT>();
    KQ_CUDA_TRY(cudaFuncSetAttribute(ptc_forward_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
    int *fault = fault_flag();
    if (!fault) return cudaErrorInvalidDevicePointer;
    ptc_forward_kernel<CIN, COUT><<<tiles, kThr, sm, s>>>(g, pv, fat, in, out, Bt, swap ? 1 : 0, fault);
    return cudaGetLastError();
}

template <int CIN, int COUT>
static cudaError_t run_wgrad(const Geom &g, const LinkSet &fat, const float2 *in, const float2 *gout, float *partial,
                             float *dB, bool swap, cudaStream_t s)
{
    const int pv = pad_sites(g.vh);
    const int tiles = 2 * ((g.vh + kTile - 1) / kTile);
    const size_t sm = wgrad_smem<CIN, COUT>();
    KQ_CUDA_TRY(cudaFuncSetAttribute(ptc_wgrad_kernel<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sm));
    int *fault = fault_flag();
    if (!fault) return cudaErrorInvalidDevicePointer;
    // persistent: one CTA per SM (the operand tiles fill most of shared memory), each accumulating its tiles
    int dev = 0, nsm = 148;
    KQ_CUDA_TRY(cudaGetDevice(&dev));
    KQ_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int ctas = std::max(1, std::min(tiles, nsm));
    ptc_wgrad_kernel<CIN, COUT><<<ctas, kThr, sm, s>>>(g, pv, fat, in, gout, partial, swap ? 1 : 0, fault);
    const int nelem = kpad_of(CIN) * npad_of(COUT);
    ptc_reduce_kernel<<<std::min(nelem, 1024), 256, 0, s>>>(partial, ctas, nelem, dB);
    return cudaGetLastError();
}

cudaError_t ptc_forward(const Geom &g, const LinkSet &fat, int cin, int cout, const float2 *in, float2 *out,
                        const void *Bt, bool swap, cudaStream_t s)
{
    const __nv_bfloat16 *B = static_cast<const __nv_bfloat16 *>(Bt);
    if (cin == 1 && cout == 8) return run_forward<1, 8>(g, fat, in, out, B, swap, s);
    // 8 input channels: the K-chunked kernel (KUQCD_PTC_WHOLE_TILE=1 keeps the whole-tile one)
    static const bool whole = getenv("KUQCD_PTC_WHOLE_TILE") && getenv("KUQCD_PTC_WHOLE_TILE")[0] == '1';
    if (cin == 8 && cout == 8) return whole ? run_forward<8, 8>(g, fat, in, out, B, swap, s)
                                            : run_forward8<8>(g, fat, in, out, B, swap, s);
    if (cin == 8 && cout == 1) return whole ? run_forward<8, 1>(g, fat, in, out, B, swap, s)
                                            : run_forward8<1>(g, fat, in, out, B, swap, s);
    if (cin == 1 && cout == 1) return run_forward<1, 1>(g, fat, in, out, B, swap, s);
    set_last_error("ptc: channel counts must be 1 or 8");
    return cudaErrorInvalidValue;
}

cudaError_t ptc_wgrad(const Geom &g, const LinkSet &fat, int cin, int cout, const float2 *in, const float2 *gout,
                      float *partial, float *dB, bool swap, cudaStream_t s)
{
    if (cin == 1 && cout == 8) return run_wgrad<1, 8>(g, fat, in, gout, partial, dB, swap, s);
    if (cin == 8 && cout == 8) return run_wgrad<8, 8>(g, fat, in, gout, partial, dB, swap, s);
    if (cin == 8 && cout == 1) return run_wgrad<8, 1>(g, fat, in, gout, partial, dB, swap, s);
    if (cin == 1 && cout == 1) return run_wgrad<1, 1>(g, fat, in, gout, partial, dB, swap, s);
    set_last_error("ptc: channel counts must be 1 or 8");
    return cudaErrorInvalidValue;
}

int ptc_kpad(int cin) { return kpad_of(cin); }
int ptc_npad(int cout) { return npad_of(cout); }
int ptc_tiles(const Geom &g) { return 2 * ((g.vh + kTile - 1) / kTile); }

cudaError_t ptc_embed(const Geom &g, const void *src, int parity, float2 *act, double scale, cudaStream_t s)
{
    ptc_embed_kernel<<<(g.vh + 255) / 256, 256, 0, s>>>(g.vh, pad_sites(g.vh), src, parity, act, scale);
    return cudaGetLastError();
}

cudaError_t ptc_extract(const Geom &g, const float2 *act, int parity, void *dst, double scale, cudaStream_t s)
{
    ptc_extract_kernel<<<(g.vh + 255) / 256, 256, 0, s>>>(g.vh, pad_sites(g.vh), act, parity, dst, scale);
    return cudaGetLastError();
}

cudaError_t ptc_loss(const Geom &g, const float2 *y, const void *e, int parity, double inv_e2, float2 *gout,
                     double *partials, double *loss_host, cudaStream_t s)
{
    const int nb = (g.vh + 255) / 256;
    ptc_loss_kernel<<<nb, 256, 0, s>>>(g.vh, pad_sites(g.vh), y, e, parity, inv_e2, gout, partials);
    KQ_CUDA_TRY(cudaGetLastError());
    if (loss_host) {
        std::vector<double> h(nb);
        KQ_CUDA_TRY(cudaMemcpyAsync(h.data(), partials, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
        KQ_CUDA_TRY(cudaStreamSynchronize(s));
        double l = 0;
        for (double v : h) l += v;
        *loss_host = l;
    }
    return cudaSuccess;
}

cudaError_t ptc_adam(float *w, float *grad, float *m, float *v, int n, float lr, float grad_scale, int step,
                     cudaStream_t s)
{
    ptc_adam_kernel<<<(n + 255) / 256, 256, 0, s>>>(w, grad, m, v, n, lr, grad_scale, 0.9f, 0.999f, 1e-8f, step);
    return cudaGetLastError();
}

}  // namespace kq
