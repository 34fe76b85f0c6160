// Batched multi-system multishift solver: many independent systems (own lattice, own links, own shifts, own source)
// advanced together, every kernel of an iteration one persistent launch over a work list of (system, site tile)
// items, W iterations captured in one CUDA graph.
//
// Why: one system of a small lattice (16^4: 32,768 sites per parity = 128 tiles) cannot fill 148 SMs, and a solve
// of many small systems one after another is dominated by launch latency and tail effects.  Interleaving all
// systems' tiles in each launch fills the GPU and amortises every launch over all systems.
//
// Each system runs the windowed multishift CG of kq_msrelax.cu (the CGM recurrences of inverter_cgm.cpp:17-87,
// deferred shift updates, operator precision relaxed FP64 -> FP32 -> HALF as its own residual falls -- decided on
// the device per system, kq_ms_device.cuh).  Reductions are per system: every tile publishes a partial sum and
// the CTA that completes a system's last tile (per-system atomic ticket) runs that system's scalar step.
// After the batched phase every system gets the FP64 true-residual check (and, if needed, the refinement) of the
// single-system mixed solver.
//
// Tuning: tile size (threads per CTA) and resident CTAs per SM of the persistent grid are chosen by timing one
// window of the actual batch (kq_tune.cu), cached on disk.  Systems large enough to fill the GPU alone go through
// the single-system solver instead, concurrently with the batched small ones (kq_batch_solve).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <mutex>
#include <thread>
#include <vector>

#include "kq_context.h"
#include "kq_dslash_core.cuh"
#include "kq_dslash_half2.cuh"
#include "kq_ms_device.cuh"
#include "kq_msrelax.h"
#include "kq_tune.h"

namespace kq {

struct SysDesc {
    Geom g;
    int pv, parity, ntiles, pad;
    LinkSet fat[3], lng[3];
    const void *b;
    void *x, *p0, *tmp, *ring, *pw;
    void *p0s;  // p0 in the operator precision of the FP32 / HALF phases (written by the p update), group-consecutive
    size_t vb, vbs;
    double *partials;  // one per tile
    MsState *st;
};

// Systems that share one gauge field (the same context) and parity form a group of up to R members; the dslash
// kernels work on (group, tile) items and load every link once for all members of the group that run in the
// kernel's operator precision (the multi-RHS form of the dslash).  A group's p0 and tmp fields are consecutive,
// vb bytes apart, so member r's field is the group base + r * vb.
constexpr int kMaxR = 8;
struct GroupDesc {
    int n;             // members
    int mem[kMaxR];    // system index of member r
};

// The descriptors live in constant memory: every CTA works on one system (or group) at a time, so the
// (warp-uniform) indexed constant loads are cheap and the fields need not be held in registers across the dslash
// (with the descriptors in global memory the FP64 kernels needed ~40 more registers and lost occupancy).  One
// batch solves at a time per process (kq_batch_solve holds a lock); at most kMaxBatch systems.
constexpr int kMaxBatch = 128;
__constant__ SysDesc c_sys[kMaxBatch];
__constant__ GroupDesc c_grp[kMaxBatch];

// ---------------------------------------------------------------------------------------------------- helpers
__device__ __forceinline__ bool tile_ticket_last(unsigned *ticket, int ntiles)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)(ntiles - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ double tile_partials_sum(const double *p, int n, double *sm)
{
    double s = 0.0;
    for (int b = threadIdx.x; b < n; b += blockDim.x) s += ((volatile const double *)p)[b];
    return block_sum(s, sm);
}

// site of step s of this thread in tile `tile` (a tile is spt x BS consecutive sites)
template <int BS>
__device__ __forceinline__ int tile_site(int tile, int spt, int s)
{
    return (tile * spt + s) * BS + threadIdx.x;
}

// members of group G whose system iterates with operator precision M in this launch (uniform over the CTA: the
// states only change in the scalar steps, which run after every tile of the system has passed)
template <int R, int M>
__device__ __forceinline__ unsigned group_mask(const GroupDesc &G)
{
    unsigned use = 0;
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (r < G.n) {
            const MsState *st = c_sys[G.mem[r]].st;
            if (st->active && st->mode == M) use |= 1u << r;
        }
    return use;
}

// ------------------------------------------------------------------ grouped dslash of one site, FP32 arithmetic
// With several members the FP32 / HALF grouped kernels are instruction-bound: the link is loaded once, but every
// member needs its own mat-vecs.  Members 2q and 2q + 1 therefore share f32x2 registers (low half member 2q), every
// link element is duplicated into both halves once per link (negated for the backward hops, so that one accumulator
// takes all sixteen terms), and each packed FMA serves two members: 36 f32x2 FMAs per pair and link instead of 72.
// Same terms in the same order as dslash_site_mrhs_t; a member outside `use` enters as zeros.
template <int SP>
__device__ __forceinline__ void ld_member_pair(const char *src0, size_t stride, int r0, unsigned use, int pv, int n,
                                               h2::f2 v[6])
{
    float a[6], b[6];
    if (use & (1u << r0)) ld_spinor_as<SP>(src0 + (size_t)r0 * stride, pv, n, a);
    else
#pragma unroll
        for (int k = 0; k < 6; ++k) a[k] = 0.f;
    if (use & (2u << r0)) ld_spinor_as<SP>(src0 + (size_t)(r0 + 1) * stride, pv, n, b);
    else
#pragma unroll
        for (int k = 0; k < 6; ++k) b[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 6; ++k) v[k] = h2::pack(a[k], b[k]);
}

template <int LP, int SP, int RP>
__device__ __forceinline__ void dslash_site_mrhs_pair(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                                      const char *src0, size_t stride, unsigned use, int p, int i,
                                                      float acc[RP][6])
{
    using namespace h2;
    static_assert(RP % 2 == 0, "members come in pairs");
    constexpr int NP = RP / 2;
    const SiteCoord c = site_coord(g, i, p);
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const float rl = fold_scale_long<LP, float>(fat, lng);
    const f2 rl2 = pack(rl, rl), m1 = pack(-1.f, -1.f);
    f2 a2[NP][6];
#pragma unroll
    for (int q = 0; q < NP; ++q)
#pragma unroll
        for (int k = 0; k < 6; ++k) a2[q][k] = pack(0.f, 0.f);
#pragma unroll
    for (int dir = 0; dir < 4; ++dir) {
#pragma unroll
        for (int h = 0; h < 4; ++h) {  // fat forward, long forward, fat backward, long backward
            const bool bwd = h >= 2, isl = (h & 1) != 0;
            const int n = nbr_index(g, c, i, dir, h == 0 ? 1 : h == 1 ? 3 : h == 2 ? -1 : -3);
            const LinkSet &L = isl ? lng : fat;
            float u[18];
            ld_link_fold<LP>(h == 0 ? fat_p : h == 1 ? lng_p : h == 2 ? fat_q : lng_q, pv, dir, bwd ? n : i, L, u);
            f2 uu[18];
#pragma unroll
            for (int k = 0; k < 18; ++k) uu[k] = bwd ? pack(-u[k], -u[k]) : pack(u[k], u[k]);
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                if (!(use & (3u << (2 * q)))) continue;
                f2 v[6], w[3];
                ld_member_pair<SP>(src0, stride, 2 * q, use, pv, n, v);
                if (LP == 2 && isl)
#pragma unroll
                    for (int k = 0; k < 6; ++k) v[k] = mul2(v[k], rl2);
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) w[cc] = mul2(v[2 * cc + (bwd ? 0 : 1)], m1);
                if (bwd) mdv_add2(uu, v, w, a2[q]);  // + (-U)^dag v
                else mv_add2(uu, v, w, a2[q]);
            }
        }
    }
    const float sf = LP == 2 ? fat.scale * (1.0f / 32767.0f) : 1.0f;
#pragma unroll
    for (int q = 0; q < NP; ++q)
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float lo, hi;
            unpack(a2[q][k], lo, hi);
            acc[2 * q][k] = LP == 2 ? lo * sf : lo;
            acc[2 * q + 1][k] = LP == 2 ? hi * sf : hi;
        }
}

// the grouped dslash of one site: FP32 arithmetic with an even member count in the packed member-pair form
template <int M, int SP, typename T, int RP>
__device__ __forceinline__ void grouped_site(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                             const char *src0, size_t stride, unsigned use, int p, int i,
                                             T acc[RP][6])
{
    if constexpr (M != 0 && RP % 2 == 0) dslash_site_mrhs_pair<M, SP, RP>(g, pv, fat, lng, src0, stride, use, p, i, acc);
    else dslash_site_mrhs_t<M, SP, T, RP>(g, pv, fat, lng, src0, stride, use, p, i, acc);
}

// Members per pass over a tile: every pass loads the links once for its members.  FP64 accumulators take twice the
// registers, so FP64 passes take at most P64 members (1, 2 or 4, a tuned value): with 4 the FP64 kernel needs ~190
// registers and one 256-thread CTA per SM, with 1 it keeps the single-system kernel's occupancy and reuses nothing.
template <int M, int R, int P64> struct Pass { static constexpr int v = M == 0 ? (R < P64 ? R : P64) : R; };

// ---------------------------------------------------------------------------------------------------- kernels
template <int BS>
__global__ void __launch_bounds__(BS) bk_init_kernel(const int2 *__restrict__ items, int nitems, int spt)
{
    __shared__ double sm[32];
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const SysDesc &d = c_sys[w.x];
        MsState *st = d.st;
        double nn = 0.0;
        for (int sidx = 0; sidx < spt; ++sidx) {
            const int i = tile_site<BS>(w.y, spt, sidx);
            if (i >= d.g.vh) break;
            double v[6], z[6] = {0, 0, 0, 0, 0, 0};
            ld_spinor<0>(d.b, d.pv, i, v);
            st_spinor<0>(d.p0, d.pv, i, v);
            char *ring = static_cast<char *>(d.ring);
            st_spinor<0>(ring, d.pv, i, v);
            for (int l = 1; l < kWin; ++l) st_spinor<0>(ring + l * d.vb, d.pv, i, z);
            for (int k = 0; k < st->ns; ++k) {
                st_spinor<0>(static_cast<char *>(d.pw) + k * d.vb, d.pv, i, v);
                st_spinor<0>(static_cast<char *>(d.x) + k * d.vb, d.pv, i, z);
            }
#pragma unroll
            for (int e = 0; e < 6; ++e) nn += v[e] * v[e];
        }
        nn = block_sum(nn, sm);
        if (threadIdx.x == 0) d.partials[w.y] = nn;
        if (tile_ticket_last(&st->ticket[0], d.ntiles)) {
            const double tot = tile_partials_sum(d.partials, d.ntiles, sm);
            if (threadIdx.x == 0) {
                st->rNorm2 = tot;
                st->bnorm2 = tot;
                // a negative tol is a relative stopping point: tol = (rel |b|)^2
                if (st->tol < 0.0) st->tol = st->tol * st->tol * tot;
                st->Bm1 = 1.0;
                for (int k = 0; k < st->ns; ++k) {
                    st->a[k] = 0.0;
                    st->B[k] = 1.0;
                    st->Z[k] = 1.0;
                    st->Zm1[k] = 1.0;
                }
                st->maxTerm = st->ns;
                st->wmax = st->ns;
                st->iter = st->wpos = st->nupd = st->halt = 0;
                st->mode = st->next_mode = 0;
                st->pp = tot;  // p0 = b
                // b = 0: x = 0 is the solution; a non-finite source is a breakdown
                const bool finite = isfinite(tot);
                st->status = finite ? 0 : KQ_STATUS_BREAKDOWN;
                st->active = (finite && tot > 0.0) ? 1 : 0;
                if (!st->active && st->running) atomicSub(st->running, 1);
                st->ticket[0] = 0;
            }
        }
        __syncthreads();
    }
}

// Launch bounds of the dslash kernels: one group member (R = 1) keeps the single-system shapes (FP32: three
// 256-thread CTAs per SM; FP64 and HALF up to 128 registers, at the 85-register cap the long-link row rebuild and
// the HALF decode spill); several members need room for their accumulators (FP64: one 256-thread CTA per SM).  The
// FP32 / HALF kernels of 2 or 4 members (dslash_site_mrhs_pair) are latency-bound and take three
// 256-thread CTAs per SM at 80 registers (at most 32 B spilled); 8 members keep two (they would spill ~1 KB).
template <int BS, int M, int RP> struct Bounds {
    static constexpr int v = RP == 1 ? (M == 1 ? 768 : 512) / BS : (M == 0 ? 256 : RP <= 4 ? 768 : 512) / BS;
};

// K1: tmp_r = D p0_r and |tmp_r|^2 -> beta step with <p0, A p0> = sigma0 |p0|^2 + |tmp|^2 (|p0|^2 from the alpha
// step's recurrence), for the members of each group whose operator precision is M (one launch per precision, so
// that each launch is specialised; members in the other precisions are skipped).  In the FP32 / HALF phases p0 is
// read from its copy in precision M.
template <int BS, int M, int R, int P64>
__global__ void __launch_bounds__(BS, Bounds<BS, M, Pass<M, R, P64>::v>::v) bk_dslash1_kernel(
    const int2 *__restrict__ items, int nitems, int spt)
{
    typedef typename Acc2<M, M>::T T;
    constexpr int RP = Pass<M, R, P64>::v;
    __shared__ double sm[32];
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const GroupDesc &G = c_grp[w.x];
        const unsigned use = group_mask<R, M>(G);
        if (!use) continue;
        const SysDesc &d0 = c_sys[G.mem[0]];
        double tt[R];
#pragma unroll
        for (int r = 0; r < R; ++r) tt[r] = 0.0;
        for (int sidx = 0; sidx < spt; ++sidx) {
            const int i = tile_site<BS>(w.y, spt, sidx);
            if (i >= d0.g.vh) break;
#pragma unroll
            for (int base = 0; base < R; base += RP) {
                const unsigned u = (use >> base) & ((1u << RP) - 1u);
                if (!u) continue;
                T acc[RP][6];
                // the FP32 / HALF phases gather p0 from its copy in their own precision (a third or half of the
                // FP64 bytes through L1/L2 for each of the RP members)
                const char *src = static_cast<const char *>(M == 0 ? d0.p0 : d0.p0s);
                const size_t vbx = M == 0 ? d0.vb : d0.vbs;
                grouped_site<M, M, T, RP>(d0.g, d0.pv, d0.fat[M], d0.lng[M], src + base * vbx, vbx, u,
                                                1 - d0.parity, i, acc);
#pragma unroll
                for (int r = 0; r < RP; ++r)
                    if (u & (1u << r)) {
                        st_spinor_as<M>(static_cast<char *>(d0.tmp) + (base + r) * d0.vb, d0.pv, i, acc[r]);
#pragma unroll
                        for (int k = 0; k < 6; ++k) tt[base + r] += (double)acc[r][k] * (double)acc[r][k];
                    }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                const SysDesc &d = c_sys[G.mem[r]];
                MsState *st = d.st;
                const double bt = block_sum(tt[r], sm);
                if (threadIdx.x == 0) d.partials[w.y] = bt;
                if (tile_ticket_last(&st->ticket[1], d.ntiles)) {
                    const double tot = tile_partials_sum(d.partials, d.ntiles, sm);
                    if (threadIdx.x < 32) {
                        ms_step_beta(st, st->shift[0] * st->pp + __shfl_sync(0xffffffffu, tot, 0));
                        if (threadIdx.x == 0) st->ticket[1] = 0;
                    }
                }
                __syncthreads();
            }
    }
}

// K2: r_r^(i+1) = r_r^(i) + B0 (sigma0 p0_r - D tmp_r) into each member's ring (s stays in registers), |r_r|^2 ->
// alpha step, for the members in precision M.  The alpha step picks the next iteration's precision in next_mode,
// applied in K3, so the K2 launches of the other precisions in this iteration do not pick the system up again.
template <int BS, int M, int R, int P64>
__global__ void __launch_bounds__(BS, Bounds<BS, M, Pass<M, R, P64>::v>::v) bk_dslash2_kernel(
    const int2 *__restrict__ items, int nitems, int spt)
{
    typedef typename Acc2<M, M>::T T;
    constexpr int RP = Pass<M, R, P64>::v;
    __shared__ double sm[32];
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const GroupDesc &G = c_grp[w.x];
        const unsigned use = group_mask<R, M>(G);
        if (!use) continue;
        const SysDesc &d0 = c_sys[G.mem[0]];
        double nn[R];
#pragma unroll
        for (int r = 0; r < R; ++r) nn[r] = 0.0;
        for (int sidx = 0; sidx < spt; ++sidx) {
            const int i = tile_site<BS>(w.y, spt, sidx);
            if (i >= d0.g.vh) break;
#pragma unroll
            for (int base = 0; base < R; base += RP) {
                const unsigned u = (use >> base) & ((1u << RP) - 1u);
                if (!u) continue;
                T acc[RP][6];
                grouped_site<M, M, T, RP>(d0.g, d0.pv, d0.fat[M], d0.lng[M],
                                                static_cast<const char *>(d0.tmp) + base * d0.vb, d0.vb, u,
                                                d0.parity, i, acc);
#pragma unroll
                for (int r = 0; r < RP; ++r)
                    if (u & (1u << r)) {
                        const SysDesc &d = c_sys[G.mem[base + r]];
                        const MsState *st = d.st;
                        const int itc = st->iter;
                        const char *rin = static_cast<const char *>(d.ring) + (size_t)(itc % kWin) * d.vb;
                        char *rout = static_cast<char *>(d.ring) + (size_t)((itc + 1) % kWin) * d.vb;
                        double pv6[6], rv[6];
                        ld_spinor<0>(d.p0, d.pv, i, pv6);
                        ld_spinor<0>(rin, d.pv, i, rv);
                        const double sig = st->shift[0], b0 = st->B[0];
#pragma unroll
                        for (int k = 0; k < 6; ++k) {
                            rv[k] += b0 * (sig * pv6[k] - (double)acc[r][k]);
                            nn[base + r] += rv[k] * rv[k];
                        }
                        st_spinor<0>(rout, d.pv, i, rv);
                    }
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (use & (1u << r)) {
                const SysDesc &d = c_sys[G.mem[r]];
                MsState *st = d.st;
                const double bn = block_sum(nn[r], sm);
                if (threadIdx.x == 0) d.partials[w.y] = bn;
                if (tile_ticket_last(&st->ticket[2], d.ntiles)) {
                    const double tot = tile_partials_sum(d.partials, d.ntiles, sm);
                    if (threadIdx.x < 32) {
                        ms_step_alpha(st, __shfl_sync(0xffffffffu, tot, 0));
                        if (threadIdx.x == 0) st->ticket[2] = 0;
                    }
                }
                __syncthreads();
            }
    }
}

// ---------------------------------------------------------------------------- staged multi-RHS dslash (FP64)
// The grouped kernels above hold every member's accumulators in one thread: with four FP64 members that is ~190
// registers and one 256-thread CTA per SM, too few warps to cover the neighbour gathers.  The staged form spreads
// the members over the warps instead: a CTA works on S = BS / R sites at a time (a round) and warp group r
// (S / 32 warps) applies D to member r, so every thread keeps the single-system register footprint.  The four
// links of one direction (fat and long, forward and backward) of the S sites are copied from global memory into
// shared memory once -- warp group r copies every R-th 16-byte plane of them, with cp.async, so the copies hold no
// registers -- and every member's threads decode their site's links from there.  Stages (round, direction) run in
// a pipeline over two buffers: the next stage's copies are in flight while the current one is applied, one barrier
// per stage.

// A link in its storage form: n16 planes of 16 bytes, then a tail plane of tb bytes (FP64: 9 + 0, compressed
// 6 + 8 (1/s); FP32: 4 + 8, compressed 3 + 4; HALF: 2 + 4); each plane pv sites long, one block per direction.
template <int LP> __device__ __forceinline__ int form_n16(int recon)
{
    return LP == 0 ? (recon ? 6 : 9) : LP == 1 ? (recon ? 3 : 4) : 2;
}
template <int LP> __device__ __forceinline__ int form_tail(int recon)
{
    return LP == 0 ? (recon ? 8 : 0) : LP == 1 ? (recon ? 4 : 8) : 4;
}
template <int LP> __device__ __forceinline__ int form_bytes(int recon) { return 16 * form_n16<LP>(recon) + form_tail<LP>(recon); }
template <int LP> struct LinkMaxBytes { static constexpr int v = LP == 0 ? 144 : LP == 1 ? 72 : 36; };
// shared memory of one staged kernel: two stage buffers of four links per site
template <int LP> constexpr size_t staged_smem(int S) { return (size_t)2 * 4 * LinkMaxBytes<LP>::v * S; }

__device__ __forceinline__ void cp_async(void *sdst, const void *gsrc, int bytes)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(sdst);
    if (bytes == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
    else if (bytes == 8) asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// this thread's share of the link of site li (direction dir) into a stage buffer: planes r, r + R, ...; the tail if
// n16 % R == r.  Sources and destinations are 16-byte aligned (pv is a multiple of 64, S of 32).
template <int LP, int R>
__device__ __forceinline__ void stage_link(char *sb, int S, int s, const void *par_base, int pv, int dir, int li,
                                           int recon, int r)
{
    const int n16 = form_n16<LP>(recon), tb = form_tail<LP>(recon);
    const char *d = static_cast<const char *>(par_base) + (size_t)dir * (16 * n16 + tb) * pv;
    for (int k = r; k < n16; k += R) cp_async(sb + (k * S + s) * 16, d + ((size_t)k * pv + li) * 16, 16);
    if (tb && n16 % R == r) cp_async(sb + n16 * 16 * S + s * tb, d + (size_t)n16 * 16 * pv + (size_t)li * tb, tb);
}

// the link of staged site s (same arithmetic as ld_link_fold: HALF values come back as raw int16)
template <int LP, typename T>
__device__ __forceinline__ void sm_link(const char *buf, int S, int s, int recon, T u[18])
{
    if constexpr (LP == 0) {
        const int n = recon ? 6 : 9;
#pragma unroll
        for (int k = 0; k < 9; ++k)
            if (k < n) {
                const double2 w = reinterpret_cast<const double2 *>(buf + k * 16 * S)[s];
                u[2 * k] = w.x;
                u[2 * k + 1] = w.y;
            }
        if (recon) rebuild_row2(u, reinterpret_cast<const double *>(buf + 96 * S)[s]);
    } else if constexpr (LP == 1) {
        float w[18];
        const int n = recon ? 3 : 4;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) {
                const float4 a = reinterpret_cast<const float4 *>(buf + k * 16 * S)[s];
                w[4 * k] = a.x; w[4 * k + 1] = a.y; w[4 * k + 2] = a.z; w[4 * k + 3] = a.w;
            }
        if (recon) {
            rebuild_row2(w, reinterpret_cast<const float *>(buf + 48 * S)[s]);
        } else {
            const float2 a = reinterpret_cast<const float2 *>(buf + 64 * S)[s];
            w[16] = a.x;
            w[17] = a.y;
        }
#pragma unroll
        for (int k = 0; k < 18; ++k) u[k] = (T)w[k];
    } else {
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int4 a = reinterpret_cast<const int4 *>(buf + k * 16 * S)[s];
            u[8 * k + 0] = lo16(a.x); u[8 * k + 1] = hi16(a.x);
            u[8 * k + 2] = lo16(a.y); u[8 * k + 3] = hi16(a.y);
            u[8 * k + 4] = lo16(a.z); u[8 * k + 5] = hi16(a.z);
            u[8 * k + 6] = lo16(a.w); u[8 * k + 7] = hi16(a.w);
        }
        const int a = reinterpret_cast<const int *>(buf + 32 * S)[s];
        u[16] = lo16(a);
        u[17] = hi16(a);
    }
}

// One staged pass over a (group, tile) item: for every round j (sites tile0 + j S + s) acc = (D src_r)(i) on output
// parity p, then epi(i, acc) if this thread's member is applied and the site exists.  Every thread of the CTA calls
// this.  Stage (j, d) holds direction d's links [fat at i | long at i | fat at i - mu | long at i - 3 mu] in
// buffer d & 1.  The terms are those of dslash_site_t in the same order.
template <int LP, int SP, typename T, int R, int S, typename Epi>
__device__ __forceinline__ void staged_pass(const Geom &g, int pv, const LinkSet &fat, const LinkSet &lng,
                                            const void *src, int p, int tile0, int rounds, int r, int s, bool mine,
                                            char *buf0, char *buf1, Epi epi)
{
    const void *fat_p = p ? fat.par[1] : fat.par[0], *fat_q = p ? fat.par[0] : fat.par[1];
    const void *lng_p = p ? lng.par[1] : lng.par[0], *lng_q = p ? lng.par[0] : lng.par[1];
    const T rl = fold_scale_long<LP, T>(fat, lng);
    const int fb = form_bytes<LP>(fat.recon) * S, lb = form_bytes<LP>(lng.recon) * S;
    const int off[4] = {0, fb, fb + lb, 2 * fb + lb};  // link k of a stage buffer
    auto site_of = [&](int j) {
        const int i = tile0 + j * S + s;
        return i < g.vh ? i : g.vh - 1;
    };
    auto issue = [&](char *sb, int dir, int i, const SiteCoord &c) {
        stage_link<LP, R>(sb + off[0], S, s, fat_p, pv, dir, i, fat.recon, r);
        stage_link<LP, R>(sb + off[1], S, s, lng_p, pv, dir, i, lng.recon, r);
        stage_link<LP, R>(sb + off[2], S, s, fat_q, pv, dir, nbr_index(g, c, i, dir, -1), fat.recon, r);
        stage_link<LP, R>(sb + off[3], S, s, lng_q, pv, dir, nbr_index(g, c, i, dir, -3), lng.recon, r);
    };
    int in = site_of(0);
    SiteCoord cn = site_coord(g, in, p);
    issue(buf0, 0, in, cn);
    cp_async_commit();
#pragma unroll 1
    for (int j = 0; j < rounds; ++j) {
        const int i = in;
        const SiteCoord c = cn;
        const bool work = mine && tile0 + j * S + s < g.vh;
        T acc[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) acc[k] = T(0);
#pragma unroll
        for (int dir = 0; dir < 4; ++dir) {
            char *cur = (dir & 1) ? buf1 : buf0, *nxt = (dir & 1) ? buf0 : buf1;
            // stage (j, dir) has landed for every thread, and every thread is done with the buffer the next
            // stage goes to (it held stage (j, dir - 1))
            cp_async_wait_all();
            __syncthreads();
            if (dir < 3) {
                issue(nxt, dir + 1, i, c);
            } else if (j + 1 < rounds) {
                in = site_of(j + 1);
                cn = site_coord(g, in, p);
                issue(nxt, 0, in, cn);
            }
            cp_async_commit();
            if (work) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    T u[18], v[6];
                    ld_spinor_as<SP>(src, pv, nbr_index(g, c, i, dir, k == 0 ? 1 : k == 1 ? 3 : k == 2 ? -1 : -3), v);
                    sm_link<LP, T>(cur + off[k], S, s, (k & 1) ? lng.recon : fat.recon, u);
                    if (k & 1) fold_long_spinor<LP>(rl, v);
                    if (k < 2) mv_add(u, v, acc);
                    else mdv_sub(u, v, acc);
                }
            }
        }
        if (work) {
            fold_scale_site<LP>(fat, acc);
            epi(i, acc);
        }
    }
}

// per-member partial sums of a tile: warp sums, then member r's S / 32 warps in order; thread 0 writes member r's
// partial and the member's last tile runs the scalar step (`step`)
template <int BS, int R, typename Step>
__device__ __forceinline__ void staged_member_steps(const GroupDesc &G, unsigned use, int tile, double v,
                                                    int ticket, double *wsum, double *sm, Step step)
{
    constexpr int WPM = BS / R / 32;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r)
        if (use & (1u << r)) {
            const SysDesc &d = c_sys[G.mem[r]];
            MsState *st = d.st;
            if (threadIdx.x == 0) {
                double a = 0.0;
                for (int q = 0; q < WPM; ++q) a += wsum[r * WPM + q];
                d.partials[tile] = a;
            }
            if (tile_ticket_last(&st->ticket[ticket], d.ntiles)) {
                const double tot = tile_partials_sum(d.partials, d.ntiles, sm);
                if (threadIdx.x < 32) {
                    step(st, __shfl_sync(0xffffffffu, tot, 0));
                    if (threadIdx.x == 0) st->ticket[ticket] = 0;
                }
            }
            __syncthreads();
        }
}

// rounds of a tile of spt BS sites on a lattice of vh sites per parity
template <int BS, int S>
__device__ __forceinline__ int staged_rounds(int tile0, int spt, int vh)
{
    const int left = vh - tile0;
    const int n = (left + S - 1) / S;
    return n < spt * (BS / S) ? n : spt * (BS / S);
}

// K1 (as bk_dslash1_kernel) with the members spread over the warps and the links staged in shared memory
template <int BS, int M, int R>
__global__ void __launch_bounds__(BS, Bounds<BS, M, 1>::v) bk_dslash1_staged_kernel(
    const int2 *__restrict__ items, int nitems, int spt)
{
    typedef typename Acc2<M, M>::T T;
    constexpr int S = BS / R;
    static_assert(S % 32 == 0, "a member's sites fill whole warps");
    extern __shared__ __align__(16) char dyn[];
    char *buf0 = dyn, *buf1 = dyn + staged_smem<M>(S) / 2;
    __shared__ double wsum[BS / 32], sm[32];
    const int r = threadIdx.x / S, s = threadIdx.x % S;
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const GroupDesc &G = c_grp[w.x];
        const unsigned use = group_mask<R, M>(G);
        if (!use) continue;
        const SysDesc &d0 = c_sys[G.mem[0]];
        const char *src = static_cast<const char *>(d0.p0) + r * d0.vb;
        char *dst = static_cast<char *>(d0.tmp) + r * d0.vb;
        const int tile0 = w.y * spt * BS;
        double tt = 0.0;
        staged_pass<M, 0, T, R, S>(d0.g, d0.pv, d0.fat[M], d0.lng[M], src, 1 - d0.parity, tile0,
                                   staged_rounds<BS, S>(tile0, spt, d0.g.vh), r, s, (use >> r) & 1u, buf0, buf1,
                                   [&](int i, const T acc[6]) {
                                       st_spinor_as<M>(dst, d0.pv, i, acc);
#pragma unroll
                                       for (int k = 0; k < 6; ++k) tt += (double)acc[k] * (double)acc[k];
                                   });
        staged_member_steps<BS, R>(G, use, w.y, tt, 1, wsum, sm, [](MsState *st, double tot) {
            ms_step_beta(st, st->shift[0] * st->pp + tot);
        });
    }
}

// K2 (as bk_dslash2_kernel), staged
template <int BS, int M, int R>
__global__ void __launch_bounds__(BS, Bounds<BS, M, 1>::v) bk_dslash2_staged_kernel(
    const int2 *__restrict__ items, int nitems, int spt)
{
    typedef typename Acc2<M, M>::T T;
    constexpr int S = BS / R;
    static_assert(S % 32 == 0, "a member's sites fill whole warps");
    extern __shared__ __align__(16) char dyn[];
    char *buf0 = dyn, *buf1 = dyn + staged_smem<M>(S) / 2;
    __shared__ double wsum[BS / 32], sm[32];
    const int r = threadIdx.x / S, s = threadIdx.x % S;
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const GroupDesc &G = c_grp[w.x];
        const unsigned use = group_mask<R, M>(G);
        if (!use) continue;
        const SysDesc &d0 = c_sys[G.mem[0]];
        const bool mine = (use >> r) & 1u;
        const SysDesc &d = c_sys[G.mem[mine ? r : 0]];
        const char *src = static_cast<const char *>(d0.tmp) + r * d0.vb;
        const int tile0 = w.y * spt * BS;
        double nn = 0.0;
        staged_pass<M, M, T, R, S>(d0.g, d0.pv, d0.fat[M], d0.lng[M], src, d0.parity, tile0,
                                   staged_rounds<BS, S>(tile0, spt, d0.g.vh), r, s, mine, buf0, buf1,
                                   [&](int i, const T acc[6]) {
                                       const MsState *st = d.st;
                                       const int itc = st->iter;
                                       const char *rin = static_cast<const char *>(d.ring) +
                                                         (size_t)(itc % kWin) * d.vb;
                                       char *rout = static_cast<char *>(d.ring) + (size_t)((itc + 1) % kWin) * d.vb;
                                       double pv6[6], rv[6];
                                       ld_spinor<0>(d.p0, d.pv, i, pv6);
                                       ld_spinor<0>(rin, d.pv, i, rv);
                                       const double sig = st->shift[0], b0 = st->B[0];
#pragma unroll
                                       for (int k = 0; k < 6; ++k) {
                                           rv[k] += b0 * (sig * pv6[k] - (double)acc[k]);
                                           nn += rv[k] * rv[k];
                                       }
                                       st_spinor<0>(rout, d.pv, i, rv);
                                   });
        staged_member_steps<BS, R>(G, use, w.y, nn, 2, wsum, sm,
                                   [](MsState *st, double tot) { ms_step_alpha(st, tot); });
    }
}

// K3: p0 = r^(i) + a0 p0 (and its copy in the next iteration's precision when that is FP32 or HALF); the next
// iteration's precision takes effect.  A system that stopped in K2 no longer needs p0.
template <int BS>
__global__ void __launch_bounds__(BS) bk_p0_kernel(const int2 *__restrict__ items, int nitems, int spt)
{
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const SysDesc &d = c_sys[w.x];
        MsState *st = d.st;
        if (!st->active) continue;
        const char *r = static_cast<const char *>(d.ring) + (size_t)(st->iter % kWin) * d.vb;
        const double a0 = st->a[0];
        const int nm = st->next_mode;  // the next iteration's operator precision (set by the alpha step)
        for (int sidx = 0; sidx < spt; ++sidx) {
            const int i = tile_site<BS>(w.y, spt, sidx);
            if (i >= d.g.vh) break;
            double rv[6], pv6[6];
            ld_spinor<0>(r, d.pv, i, rv);
            ld_spinor<0>(d.p0, d.pv, i, pv6);
#pragma unroll
            for (int k = 0; k < 6; ++k) pv6[k] = rv[k] + a0 * pv6[k];
            st_spinor<0>(d.p0, d.pv, i, pv6);
            // the copy the next K1 gathers from in the FP32 / HALF phases
            if (nm == 1) st_spinor_as<1>(d.p0s, d.pv, i, pv6);
            else if (nm == 2) st_spinor_as<2>(d.p0s, d.pv, i, pv6);
        }
        if (tile_ticket_last(&st->ticket[3], d.ntiles) && threadIdx.x == 0) {
            st->mode = st->next_mode;
            st->ticket[3] = 0;
        }
        __syncthreads();
    }
}

// K4: windowed shift update of every system that iterated in this window
template <int BS>
__global__ void __launch_bounds__(BS) bk_window_kernel(const int2 *__restrict__ items, int nitems, int spt)
{
    __shared__ double sc[kMaxShift], se[kMaxShift], sd[kMaxShift][kWin], sf[kMaxShift][kWin];
#pragma unroll 1
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int2 w = items[it];
        const SysDesc &d = c_sys[w.x];
        MsState *st = d.st;
        const int n = st->wpos, kmax = st->wmax;
        // uniform per system: apply a full window, or a partial one once the system has stopped
        if (n == 0 || (n < kWin && st->active)) continue;
        __syncthreads();
        for (int t = threadIdx.x; t < kmax; t += BS) {
            sc[t] = st->c[t];
            se[t] = st->e[t];
            for (int l = 0; l < kWin; ++l) {
                sd[t][l] = st->d[t][l];
                sf[t][l] = st->f[t][l];
            }
        }
        __syncthreads();
        for (int sidx = 0; sidx < spt; ++sidx) {
            const int i = tile_site<BS>(w.y, spt, sidx);
            if (i >= d.g.vh) break;
            window_update_site(static_cast<const char *>(d.ring), d.vb, d.pv, i, n, kmax, sc, se, sd, sf,
                               static_cast<char *>(d.pw), static_cast<char *>(d.x));
        }
        if (tile_ticket_last(&st->ticket[0], d.ntiles)) {
            if (threadIdx.x == 0) {
                st->wpos = 0;
                st->ticket[0] = 0;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------------- host
// items: per-system (system, tile) items for init / p0 / window, per-group (group, tile) items for the dslash steps
struct BatchItems {
    const int2 *sys;
    int nsys;
    const int2 *grp;
    int ngrp;
};

template <int BS>
static void enqueue_batch_init(const BatchItems &it, int grid, int spt, cudaStream_t s)
{
    bk_init_kernel<BS><<<grid, BS, 0, s>>>(it.sys, it.nsys, spt);
}

// the staged FP64 kernels need whole warps per member: R in 2..BS / 32
constexpr bool staged_ok(int bs, int r) { return r > 1 && (bs / r) % 32 == 0; }

// the staged kernels' dynamic shared memory (two stage buffers: up to 144 KB for 128 sites per round)
template <int BS, int R>
static cudaError_t staged_attr()
{
    if constexpr (staged_ok(BS, R)) {
        const int sm = (int)staged_smem<0>(BS / R);
        KQ_CUDA_TRY(cudaFuncSetAttribute(bk_dslash1_staged_kernel<BS, 0, R>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        KQ_CUDA_TRY(cudaFuncSetAttribute(bk_dslash2_staged_kernel<BS, 0, R>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    }
    return cudaSuccess;
}

static cudaError_t staged_attrs()
{
    KQ_CUDA_TRY((staged_attr<128, 2>()));
    KQ_CUDA_TRY((staged_attr<128, 4>()));
    KQ_CUDA_TRY((staged_attr<256, 2>()));
    KQ_CUDA_TRY((staged_attr<256, 4>()));
    KQ_CUDA_TRY((staged_attr<256, 8>()));
    return cudaSuccess;
}

template <int BS, int R, int P64>
static void enqueue_batch_chunk_r(const BatchItems &it, int grid, int spt, cudaStream_t s)
{
    for (int k = 0; k < kChunk; ++k) {
        // (P64 only shapes the FP64 kernels, 0 = staged; the sloppy ones are instantiated once)
        if constexpr (P64 == 0)
            bk_dslash1_staged_kernel<BS, 0, R><<<grid, BS, staged_smem<0>(BS / R), s>>>(it.grp, it.ngrp, spt);
        else bk_dslash1_kernel<BS, 0, R, P64><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        bk_dslash1_kernel<BS, 1, R, 1><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        bk_dslash1_kernel<BS, 2, R, 1><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        if constexpr (P64 == 0)
            bk_dslash2_staged_kernel<BS, 0, R><<<grid, BS, staged_smem<0>(BS / R), s>>>(it.grp, it.ngrp, spt);
        else bk_dslash2_kernel<BS, 0, R, P64><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        bk_dslash2_kernel<BS, 1, R, 1><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        bk_dslash2_kernel<BS, 2, R, 1><<<grid, BS, 0, s>>>(it.grp, it.ngrp, spt);
        bk_p0_kernel<BS><<<grid, BS, 0, s>>>(it.sys, it.nsys, spt);
    }
    bk_window_kernel<BS><<<grid, BS, 0, s>>>(it.sys, it.nsys, spt);
}

template <int BS, int R>
static void enqueue_batch_chunk_p(const BatchItems &it, int grid, int spt, int p64, cudaStream_t s)
{
    if constexpr (staged_ok(BS, R))
        if (p64 == 0) {
            enqueue_batch_chunk_r<BS, R, 0>(it, grid, spt, s);
            return;
        }
    if (R == 1 || p64 == 1) enqueue_batch_chunk_r<BS, R, 1>(it, grid, spt, s);
    else if (R == 2 || p64 == 2) enqueue_batch_chunk_r<BS, R, 2>(it, grid, spt, s);
    else enqueue_batch_chunk_r<BS, R, 4>(it, grid, spt, s);
}

template <int BS>
static void enqueue_batch_chunk(const BatchItems &it, int grid, int rhs, int spt, int p64, cudaStream_t s)
{
    switch (rhs) {
        case 8: enqueue_batch_chunk_p<BS, 8>(it, grid, spt, p64, s); break;
        case 4: enqueue_batch_chunk_p<BS, 4>(it, grid, spt, p64, s); break;
        case 2: enqueue_batch_chunk_p<BS, 2>(it, grid, spt, p64, s); break;
        default: enqueue_batch_chunk_r<BS, 1, 1>(it, grid, spt, s); break;
    }
}

}  // namespace kq

using namespace kq;

struct BatchSystem {
    kq_context *ctx;
    kq_solve_param param;
    std::vector<double> shifts;
    const void *d_b;
    void *d_x;
    kq_solve_info info;
};

struct kq_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<BatchSystem> sys;
    void *work = nullptr;
    size_t work_bytes = 0;
    int *d_running = nullptr;
    int *h_running = nullptr;  // pinned
    int2 *d_items = nullptr;   // per-system items, then per-group items
    size_t items_cap = 0;
};

#define KQ_API extern "C" __attribute__((visibility("default")))

KQ_API KuQCDStatus kq_batch_create(int device, kq_batch **out)
{
    if (!out) return KUQCD_ERR_NULL_POINTER;
    kq_batch *b = new (std::nothrow) kq_batch();
    if (!b) return KUQCD_ERR_NO_MEMORY;
    b->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_running, sizeof(int) * 4);
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_running, sizeof(int) * 4);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_batch_create: ") + cudaGetErrorString(e));
        delete b;
        return status_of(e);
    }
    *out = b;
    return KUQCD_SUCCESS;
}

KQ_API void kq_batch_destroy(kq_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->work) cudaFree(b->work);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_running) cudaFree(b->d_running);
    if (b->h_running) cudaFreeHost(b->h_running);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

KQ_API KuQCDStatus kq_batch_add(kq_batch *b, kq_context *ctx, const kq_solve_param *param, const void *d_b,
                                void *d_x)
{
    if (!b || !ctx || !param || !param->shifts || !d_b || !d_x) {
        set_last_error("kq_batch_add: null pointer");
        return KUQCD_ERR_NULL_POINTER;
    }
    if (param->num_shift < 1 || param->num_shift > kMaxShift || (param->parity != 0 && param->parity != 1)) {
        set_last_error("kq_batch_add: num_shift must be 1..64 and parity 0 or 1");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->solver != KQ_SOLVER_MIXED && param->solver != KQ_SOLVER_CGM_WINDOWED) {
        set_last_error("kq_batch_add: batched systems use KQ_SOLVER_MIXED or KQ_SOLVER_CGM_WINDOWED");
        return KUQCD_ERR_UNSUPPORTED;
    }
    if (param->solver == KQ_SOLVER_MIXED && param->rel_residual < 0) {
        set_last_error("kq_batch_add: batched systems take a relative target (rel_residual > 0)");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (ctx->device != b->device) {
        set_last_error("kq_batch_add: context on another device");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (!ctx->fat_loaded || !ctx->long_loaded || ctx->master != P64) {
        set_last_error("kq_batch_add: load FP64 fat and long links into the context first");
        return KUQCD_ERR_UNEXPECTED_CALL_ORDER;
    }
    BatchSystem s;
    s.ctx = ctx;
    s.param = *param;
    s.shifts.assign(param->shifts, param->shifts + param->num_shift);
    s.param.shifts = nullptr;
    s.d_b = d_b;
    s.d_x = d_x;
    memset(&s.info, 0, sizeof(s.info));
    if ((int)b->sys.size() >= kMaxBatch) {
        set_last_error("kq_batch_add: at most 128 systems per batch");
        return KUQCD_ERR_UNSUPPORTED;
    }
    b->sys.push_back(s);
    return KUQCD_SUCCESS;
}

KQ_API int kq_batch_size(const kq_batch *b) { return b ? (int)b->sys.size() : 0; }

KQ_API KuQCDStatus kq_batch_system_info(const kq_batch *b, int i, kq_solve_info *out)
{
    if (!b || !out) return KUQCD_ERR_NULL_POINTER;
    if (i < 0 || i >= (int)b->sys.size()) return KUQCD_ERR_INVALID_PARAM;
    *out = b->sys[i].info;
    return KUQCD_SUCCESS;
}

namespace {

struct BatchPlan {
    std::vector<SysDesc> desc;
    std::vector<GroupDesc> groups;
    std::vector<int2> sys_items, grp_items;
    std::vector<MsState> init;
};

// Systems on the same context (gauge field) and parity, in batch order, in groups of at most rhs members.
std::vector<GroupDesc> form_groups(const std::vector<BatchSystem> &sys, int rhs)
{
    std::vector<GroupDesc> groups;
    std::vector<int> open;  // index of the group each system's (context, parity) currently fills, -1 if none
    for (size_t si = 0; si < sys.size(); ++si) {
        int gi = -1;
        for (size_t g = 0; g < groups.size(); ++g) {
            const BatchSystem &m = sys[groups[g].mem[0]];
            if (m.ctx == sys[si].ctx && m.param.parity == sys[si].param.parity && groups[g].n < rhs) gi = (int)g;
        }
        if (gi < 0) {
            GroupDesc G;
            memset(&G, 0, sizeof(G));
            groups.push_back(G);
            gi = (int)groups.size() - 1;
        }
        groups[gi].mem[groups[gi].n++] = (int)si;
    }
    return groups;
}

// largest number of systems sharing one context and parity (the most right-hand sides a link load can serve)
int max_shared(const std::vector<BatchSystem> &sys)
{
    int best = 0;
    for (const GroupDesc &G : form_groups(sys, kMaxR)) best = std::max(best, G.n);
    return best;
}

// Lay out every system's buffers in the batch workspace and build descriptors, groups, work items and initial
// states.  A tile is spt x bs consecutive sites.
cudaError_t batch_plan(kq_batch *b, int bs, int rhs, int spt, BatchPlan &plan, bool carve_only, size_t *bytes)
{
    Carve c(carve_only ? nullptr : b->work);
    plan.desc.assign(b->sys.size(), SysDesc{});
    plan.init.assign(b->sys.size(), MsState{});
    plan.sys_items.clear();
    plan.grp_items.clear();
    plan.groups = form_groups(b->sys, rhs);
    const int tile = bs * spt;
    for (size_t gi = 0; gi < plan.groups.size(); ++gi) {
        const GroupDesc &G = plan.groups[gi];
        const Geom &g = b->sys[G.mem[0]].ctx->g;
        const size_t vb = spinor_bytes(g, P64), vbs = spinor_bytes(g, P32);
        const int ntiles = (g.vh + tile - 1) / tile;
        // the group's p0, sloppy p0 and tmp fields are consecutive (the multi-RHS dslash addresses member r at
        // base + r vb); the sloppy copy holds FP32 or HALF, in FP32-sized slots
        char *p0 = static_cast<char *>(c.take(vb * G.n));
        char *p0s = static_cast<char *>(c.take(vbs * G.n));
        char *tmp = static_cast<char *>(c.take(vb * G.n));
        for (int t = 0; t < ntiles; ++t) plan.grp_items.push_back(make_int2((int)gi, t));
        for (int r = 0; r < G.n; ++r) {
            const int si = G.mem[r];
            BatchSystem &S = b->sys[si];
            kq_context *ctx = S.ctx;
            const int ns = S.param.num_shift;
            SysDesc &d = plan.desc[si];
            memset(&d, 0, sizeof(d));
            d.g = g;
            d.pv = pad_sites(g.vh);
            d.parity = S.param.parity;
            d.ntiles = ntiles;
            for (int p = 0; p < 3; ++p) {
                d.fat[p] = ctx->gd.fat[p];
                d.lng[p] = ctx->gd.lng[p];
            }
            d.vb = vb;
            d.vbs = vbs;
            d.p0s = p0s ? p0s + r * vbs : nullptr;
            d.b = S.d_b;
            d.x = S.d_x;
            d.p0 = p0 ? p0 + r * vb : nullptr;
            d.tmp = tmp ? tmp + r * vb : nullptr;
            d.ring = c.take(vb * kWin);
            d.pw = c.take(vb * ns);
            d.partials = static_cast<double *>(c.take(sizeof(double) * ntiles));
            d.st = static_cast<MsState *>(c.take(sizeof(MsState)));
            MsState &h = plan.init[si];
            memset(&h, 0, sizeof(h));
            h.ns = ns;
            h.max_iter = S.param.max_iter > 0 ? S.param.max_iter : 100000;
            std::vector<double> sig(ns);
            for (int k = 0; k < ns; ++k)
                sig[k] = (S.param.shift_mode == 0 && k > 0) ? S.shifts[0] + S.shifts[k] : S.shifts[k];
            h.shift[0] = sig[0];
            for (int k = 1; k < ns; ++k) h.shift[k] = sig[k] - sig[0];
            if (S.param.solver == KQ_SOLVER_MIXED) {
                // the single-system mixed solver's schedule (kq_mixed.cu): stop at 0.7 x target, FP32 from
                // 0.3 target / 3e-7, HALF from 0.3 target / 1e-3
                const double tgt = S.param.rel_residual > 0 ? S.param.rel_residual : 1e-10;
                const char *sf = getenv("KUQCD_RELAX_STOP");
                const double stop = sf ? atof(sf) : 0.7;
                h.tol = -stop * tgt;  // relative: the init kernel turns it into (0.7 tgt |b|)^2
                const double r32 = 0.3 * tgt / 3e-7, r16 = 0.3 * tgt / 1e-3;
                h.rho32_2 = r32 * r32;
                h.rho16_2 = prec_from_api(S.param.prec) == P16 ? r16 * r16 : 0.0;
            } else {
                h.tol = S.param.tol;
            }
            h.running = b->d_running;
        }
    }
    for (size_t si = 0; si < b->sys.size(); ++si)
        for (int t = 0; t < plan.desc[si].ntiles; ++t) plan.sys_items.push_back(make_int2((int)si, t));
    *bytes = c.off;
    return cudaSuccess;
}

}  // namespace

static std::mutex g_batch_mu;  // the descriptor tables in constant memory are shared by all batches

// The batched iterations over every system in b->sys, then each system's FP64 check / refinement.
static KuQCDStatus solve_batched(kq_batch *b, kq_batch_info *out)
{
    cudaSetDevice(b->device);
    cudaStream_t s = b->stream;
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, b->device);
    const int shared = max_shared(b->sys);
    if (const cudaError_t e = staged_attrs(); e != cudaSuccess) {
        set_last_error(std::string("kq_batch_solve: ") + cudaGetErrorString(e));
        return status_of(e);
    }

    // launch shape: tuned once per batch signature (sizes, shared gauge fields, shifts, schedule), cached on disk
    std::string key = "batch7";
    for (auto &S : b->sys) {
        int owner = 0;  // first system on the same context: systems sharing links share this number
        while (b->sys[owner].ctx != S.ctx) ++owner;
        key += "_" + std::to_string(S.ctx->g.n[0]) + "x" + std::to_string(S.ctx->g.n[1]) + "x" +
               std::to_string(S.ctx->g.n[2]) + "x" + std::to_string(S.ctx->g.n[3]) + "c" + std::to_string(owner) +
               "s" + std::to_string(S.param.num_shift) + "m" + std::to_string(S.param.solver) + "p" +
               std::to_string(S.param.prec);
    }
    BatchTune tune;
    bool have_tune = tune_lookup(key, &tune);
    // KUQCD_BATCH_SHAPE="threads,ctas_per_sm,rhs,sites_per_thread[,fp64_rhs_per_pass]" fixes the shape (no tuning)
    if (const char *shape = getenv("KUQCD_BATCH_SHAPE")) {
        BatchTune t{256, 4, 1, 1, 1};
        const int n = sscanf(shape, "%d,%d,%d,%d,%d", &t.bs, &t.ctas_per_sm, &t.rhs, &t.spt, &t.p64);
        if (n == 4) t.p64 = t.rhs < 4 ? t.rhs : 4;
        if (n >= 4 && (t.bs == 128 || t.bs == 256) && t.ctas_per_sm >= 1 && t.ctas_per_sm <= 32 &&
            (t.rhs == 1 || t.rhs == 2 || t.rhs == 4 || t.rhs == 8) && (t.spt == 1 || t.spt == 2) &&
            (t.p64 == 1 || t.p64 == 2 || t.p64 == 4 || (t.p64 == 0 && staged_ok(t.bs, t.rhs)))) {
            tune = t;
            have_tune = true;
        }
    }
    if (!have_tune) {
        tune.bs = 256;
        tune.ctas_per_sm = 4;
        tune.rhs = 1;
        tune.spt = 1;
        tune.p64 = 1;
    }

    auto run = [&](const BatchTune &t, int max_chunks, float *ms_out, long long *launches, int *chunks_out,
                   int *ngroups) -> cudaError_t {
        BatchPlan plan;
        size_t bytes = 0;
        batch_plan(b, t.bs, t.rhs, t.spt, plan, true, &bytes);
        if (b->work_bytes < bytes) {
            if (b->work) cudaFree(b->work);
            b->work = nullptr;
            b->work_bytes = 0;
            KQ_CUDA_TRY(cudaMalloc(&b->work, bytes));
            b->work_bytes = bytes;
        }
        batch_plan(b, t.bs, t.rhs, t.spt, plan, false, &bytes);
        const size_t nsys = plan.desc.size(), nsi = plan.sys_items.size(), ngi = plan.grp_items.size();
        if (b->items_cap < nsi + ngi) {
            if (b->d_items) cudaFree(b->d_items);
            b->d_items = nullptr;
            KQ_CUDA_TRY(cudaMalloc(&b->d_items, sizeof(int2) * (nsi + ngi)));
            b->items_cap = nsi + ngi;
        }
        KQ_CUDA_TRY(cudaMemcpyToSymbolAsync(c_sys, plan.desc.data(), sizeof(SysDesc) * nsys, 0,
                                            cudaMemcpyHostToDevice, s));
        KQ_CUDA_TRY(cudaMemcpyToSymbolAsync(c_grp, plan.groups.data(), sizeof(GroupDesc) * plan.groups.size(), 0,
                                            cudaMemcpyHostToDevice, s));
        KQ_CUDA_TRY(cudaMemcpyAsync(b->d_items, plan.sys_items.data(), sizeof(int2) * nsi, cudaMemcpyHostToDevice,
                                    s));
        KQ_CUDA_TRY(cudaMemcpyAsync(b->d_items + nsi, plan.grp_items.data(), sizeof(int2) * ngi,
                                    cudaMemcpyHostToDevice, s));
        for (size_t i = 0; i < nsys; ++i)
            KQ_CUDA_TRY(cudaMemcpyAsync(plan.desc[i].st, &plan.init[i], sizeof(MsState), cudaMemcpyHostToDevice, s));
        const int nsys_i = (int)nsys;
        KQ_CUDA_TRY(cudaMemcpyAsync(b->d_running, &nsys_i, sizeof(int), cudaMemcpyHostToDevice, s));
        const BatchItems items{b->d_items, (int)nsi, b->d_items + nsi, (int)ngi};
        const int grid = std::max(1, std::min((int)nsi, dev_sms * t.ctas_per_sm));
        *ngroups = (int)plan.groups.size();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        if (t.bs == 128) enqueue_batch_init<128>(items, grid, t.spt, s);
        else enqueue_batch_init<256>(items, grid, t.spt, s);
        KQ_CUDA_TRY(cudaGetLastError());
        *launches = 1;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        KQ_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        if (t.bs == 128) enqueue_batch_chunk<128>(items, grid, t.rhs, t.spt, t.p64, s);
        else enqueue_batch_chunk<256>(items, grid, t.rhs, t.spt, t.p64, s);
        cudaError_t ee = cudaStreamEndCapture(s, &graph);
        if (ee == cudaSuccess) ee = cudaGraphInstantiate(&exec, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        KQ_CUDA_TRY(ee);
        int chunks = 0;
        int chunk_cap = 8;
        for (const MsState &h : plan.init) chunk_cap = std::max(chunk_cap, h.max_iter / kChunk + 8);
        cudaError_t err = cudaSuccess;
        cudaEventRecord(e0, s);  // device time of the iterations (after the init kernel and graph set-up)
        for (;;) {
            err = cudaMemcpyAsync(b->h_running, b->d_running, sizeof(int), cudaMemcpyDeviceToHost, s);
            if (err == cudaSuccess) err = cudaStreamSynchronize(s);
            if (err != cudaSuccess || *b->h_running <= 0) break;
            if (max_chunks > 0 && chunks >= max_chunks) break;
            err = cudaGraphLaunch(exec, s);
            if (err != cudaSuccess) break;
            ++chunks;
            *launches += 7 * kChunk + 1;  // two dslash steps x three precisions + p0 per iteration, + window
            if (chunks > chunk_cap) break;  // every system has stopped by then while the states are consistent
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(ms_out, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaGraphExecDestroy(exec);
        *chunks_out = chunks;
        return err;
    };

    if (!have_tune) {
        // Time the real batch per candidate shape (the solve restarts afterwards), one dimension at a time: tile x
        // CTAs per SM on two windows, with every shared gauge field serving as many right-hand sides as it can;
        // per group width, the FP64 pass mode on two windows (the solve's first windows run on FP64 links); the
        // group widths against each other on complete solves (the width also sets the sloppy kernels' register
        // use, which the first windows do not see); CTAs per SM again for that width, on complete solves; then the
        // sites per thread.
        auto timed = [&](const BatchTune &t, int chunks, float *ms) -> cudaError_t {
            long long l = 0;
            int ch = 0, ng = 0;
            *ms = 1e30f;
            float m = 0;
            const cudaError_t e = run(t, chunks, &m, &l, &ch, &ng);
            if (e == cudaSuccess && ch > 0) *ms = m;
            return e;
        };
        float best = 1e30f;
        int rmax = 1;
        while (rmax < std::min(shared, kMaxR)) rmax *= 2;
        BatchTune t{256, 4, rmax, 1, std::min(rmax, 4)};
        const int bss[2] = {128, 256}, cpss[4] = {2, 4, 8, 16};
        for (int bs : bss)
            for (int cps : cpss) {
                if (bs == 256 && cps > 8) continue;
                BatchTune c = t;
                c.bs = bs;
                c.ctas_per_sm = cps;
                float ms;
                const cudaError_t e = timed(c, 2, &ms);
                if (e != cudaSuccess) return status_of(e);
                if (ms < best) {
                    best = ms;
                    tune = c;
                }
            }
        if (rmax > 1) {
            const BatchTune base = tune;
            best = 1e30f;
            for (int r = 1; r <= rmax; r *= 2) {
                // FP64 pass modes of this width: members per pass 1, 2, 4 (up to r) and the staged kernels
                int modes[4], nm = 0;
                for (int p = 1; p <= std::min(r, 4); p *= 2) modes[nm++] = p;
                if (staged_ok(base.bs, r)) modes[nm++] = 0;
                BatchTune wbest = base;
                float wms = 1e30f;
                for (int q = 0; q < nm; ++q) {
                    BatchTune c = base;
                    c.rhs = r;
                    c.p64 = modes[q];
                    float ms;
                    const cudaError_t e = nm > 1 ? timed(c, 2, &ms) : cudaSuccess;
                    if (e != cudaSuccess) return status_of(e);
                    if (nm == 1 || ms < wms) {
                        wms = ms;
                        wbest = c;
                    }
                }
                float ms;
                const cudaError_t e = timed(wbest, 0, &ms);
                if (e != cudaSuccess) return status_of(e);
                if (ms < best) {
                    best = ms;
                    tune = wbest;
                }
            }
        }
        if (rmax > 1) {
            // CTAs per SM of the persistent grid again, for the chosen width (its kernels' residency differs from
            // the widest group's, on which the first sweep ran), on complete solves
            const BatchTune w = tune;
            for (int cps : {4, 8, 16}) {
                if (cps == w.ctas_per_sm || (w.bs == 256 && cps > 8)) continue;
                BatchTune c = w;
                c.ctas_per_sm = cps;
                float ms;
                const cudaError_t e = timed(c, 0, &ms);
                if (e != cudaSuccess) return status_of(e);
                if (ms < best) {
                    best = ms;
                    tune = c;
                }
            }
        }
        {
            BatchTune c = tune;
            c.spt = 2;
            float ms1, ms2;
            cudaError_t e = timed(tune, 2, &ms1);
            if (e == cudaSuccess) e = timed(c, 2, &ms2);
            if (e != cudaSuccess) return status_of(e);
            if (ms2 < ms1) tune = c;
        }
        tune_store(key, tune);
    }
    float ms = 0;
    long long launches = 0;
    int chunks = 0, ngroups = 0;
    cudaError_t e = run(tune, 0, &ms, &launches, &chunks, &ngroups);
    if (e != cudaSuccess) {
        set_last_error(std::string("kq_batch_solve: ") + cudaGetErrorString(e));
        return status_of(e);
    }
    // per-system results, then the FP64 check / refinement of the mixed systems
    const auto t_check = std::chrono::steady_clock::now();
    int refine_total = 0;
    BatchPlan plan;
    size_t bytes = 0;
    batch_plan(b, tune.bs, tune.rhs, tune.spt, plan, false, &bytes);
    int refined = 0;
    double worst = 0.0;
    int maxit = 0;
    for (size_t i = 0; i < b->sys.size(); ++i) {
        BatchSystem &S = b->sys[i];
        MsState h;
        const cudaError_t ec = cudaMemcpy(&h, plan.desc[i].st, sizeof(MsState), cudaMemcpyDeviceToHost);
        if (ec != cudaSuccess) {
            set_last_error(std::string("kq_batch_solve: ") + cudaGetErrorString(ec));
            return status_of(ec);
        }
        memset(&S.info, 0, sizeof(S.info));
        S.info.iter = h.iter;
        S.info.status = h.status;
        S.info.num_shift = S.param.num_shift;
        maxit = std::max(maxit, h.iter);
    }
    // FP64 check and refinement of the mixed systems: the systems of one context one after another (they share its
    // stream and workspace), different contexts concurrently on their own streams, one host thread each
    std::vector<std::vector<int>> by_ctx;
    for (size_t i = 0; i < b->sys.size(); ++i) {
        if (b->sys[i].param.solver != KQ_SOLVER_MIXED) continue;
        bool placed = false;
        for (auto &v : by_ctx)
            if (b->sys[v[0]].ctx == b->sys[i].ctx) {
                v.push_back((int)i);
                placed = true;
                break;
            }
        if (!placed) by_ctx.push_back({(int)i});
    }
    std::vector<cudaError_t> errs(by_ctx.size(), cudaSuccess);
    std::vector<std::string> msgs(by_ctx.size());
    auto check_ctx = [&](size_t c) {
        for (int i : by_ctx[c]) {
            BatchSystem &S = b->sys[i];
            std::vector<double> sig(S.param.num_shift);
            for (int k = 0; k < S.param.num_shift; ++k)
                sig[k] = (S.param.shift_mode == 0 && k > 0) ? S.shifts[0] + S.shifts[k] : S.shifts[k];
            kq_solve_param p = S.param;
            p.shifts = S.shifts.data();
            kq_solve_info ri;
            memset(&ri, 0, sizeof(ri));
            cudaSetDevice(S.ctx->device);
            const cudaError_t e2 = mixed_solve(S.ctx, &p, sig.data(), S.d_b, S.d_x, &ri, false);
            if (e2 != cudaSuccess) {
                errs[c] = e2;
                msgs[c] = last_error();
                return;
            }
            S.info.iter_refine = ri.iter_refine;
            S.info.kernel_launches = ri.kernel_launches;
            for (int k = 0; k < S.param.num_shift; ++k) S.info.true_residual[k] = ri.true_residual[k];
            if (ri.status) S.info.status = ri.status;
        }
    };
    {
        std::vector<std::thread> pool;
        for (size_t c = 1; c < by_ctx.size(); ++c) pool.emplace_back(check_ctx, c);
        if (!by_ctx.empty()) check_ctx(0);
        for (auto &t : pool) t.join();
    }
    for (size_t c = 0; c < by_ctx.size(); ++c)
        if (errs[c] != cudaSuccess) {
            set_last_error(msgs[c]);
            return status_of(errs[c]);
        }
    for (auto &v : by_ctx)
        for (int i : v) {
            const BatchSystem &S = b->sys[i];
            refine_total += S.info.iter_refine;
            if (S.info.iter_refine > 0) ++refined;
            for (int k = 0; k < S.param.num_shift; ++k) worst = std::max(worst, S.info.true_residual[k]);
        }
    cudaSetDevice(b->device);
    if (out) {
        memset(out, 0, sizeof(*out));
        out->num_systems = (int)b->sys.size();
        out->iterations = maxit;
        out->batched_seconds = ms * 1e-3;
        out->kernel_launches = launches;
        out->tile = tune.bs;
        out->ctas_per_sm = tune.ctas_per_sm;
        out->max_true_residual = worst;
        out->refined_systems = refined;
        out->tuned_now = have_tune ? 0 : 1;
        out->rhs_per_cta = tune.rhs;
        out->sites_per_thread = tune.spt;
        out->fp64_rhs_per_pass = tune.p64;
        out->groups = ngroups;
        out->check_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_check).count();
        out->refine_iterations = refine_total;
    }
    return KUQCD_SUCCESS;
}

// Systems of at least this many sites per parity fill the GPU on their own, and the single-system solver (kernels
// specialised for one lattice, no per-item mode checks) runs them faster than the batched kernels (measured on
// B200: 24^3 x 48 and 32^4 systems 10-16 % faster one after another); smaller systems are batched.  A large system
// that shares its gauge field with another system of the batch stays batched: there the grouped dslash loads each
// link once for all of them.  Override with KUQCD_BATCH_LARGE_SITES.
static int large_sites()
{
    const char *e = getenv("KUQCD_BATCH_LARGE_SITES");
    return e ? atoi(e) : 131072;
}

// host threads solving the large systems at once (KUQCD_BATCH_LARGE_THREADS, 1 .. 8)
static int large_threads()
{
    const char *e = getenv("KUQCD_BATCH_LARGE_THREADS");
    const int v = e ? atoi(e) : 2;
    return v >= 1 && v <= 8 ? v : 2;
}

KQ_API KuQCDStatus kq_batch_solve(kq_batch *b, kq_batch_info *out)
{
    kq::NvtxRange nvtx_range_("kq_batch_solve");
    if (!b) return KUQCD_ERR_NULL_POINTER;
    std::lock_guard<std::mutex> lk(g_batch_mu);
    if (b->sys.empty()) {
        set_last_error("kq_batch_solve: empty batch");
        return KUQCD_ERR_INVALID_PARAM;
    }
    cudaSetDevice(b->device);
    // links the schedules need
    for (auto &S : b->sys) {
        const bool mixed = S.param.solver == KQ_SOLVER_MIXED;
        const int precs[3] = {KUQCD_DOUBLE, KUQCD_SINGLE, KUQCD_HALF};
        const int need = mixed ? (prec_from_api(S.param.prec) == P16 ? 3 : 2) : 1;
        for (int p = 0; p < need; ++p) {
            KuQCDStatus st = kq_prepare_links(S.ctx, precs[p]);
            if (st != KUQCD_SUCCESS) return st;
        }
    }
    const int big = large_sites();
    std::vector<int> large, small;
    for (size_t i = 0; i < b->sys.size(); ++i) {
        int sharing = 0;
        for (const BatchSystem &o : b->sys) sharing += (o.ctx == b->sys[i].ctx) ? 1 : 0;
        (b->sys[i].ctx->g.vh >= big && sharing == 1 ? large : small).push_back((int)i);
    }
    if (large.empty()) return solve_batched(b, out);

    // the small systems, batched, in a helper thread on the batch's stream; meanwhile the large ones one after
    // another on their own contexts' streams (the two kinds of work overlap on the GPU)
    std::vector<BatchSystem> all;
    all.swap(b->sys);
    for (int i : small) b->sys.push_back(all[i]);
    kq_batch_info bi;
    memset(&bi, 0, sizeof(bi));
    KuQCDStatus st_small = KUQCD_SUCCESS;
    std::string err_small;
    std::thread th;
    if (!b->sys.empty())
        th = std::thread([&]() {
            st_small = solve_batched(b, &bi);
            if (st_small != KUQCD_SUCCESS) err_small = last_error();
        });
    // The large systems, each on its own context's stream, on large_threads() host threads at once: one solve's
    // latency-bound steps (reductions, scalar steps, the refinement's small grids) overlap another's kernels.
    KuQCDStatus st_large = KUQCD_SUCCESS;
    std::string err_large;
    double worst = 0.0;
    int maxit = 0, refined = 0;
    long long launches = 0;
    std::atomic<size_t> next_large{0};
    std::mutex large_mu;
    auto large_worker = [&]() {
        cudaSetDevice(b->device);
        for (size_t q; (q = next_large.fetch_add(1)) < large.size();) {
            BatchSystem &S = all[large[q]];
            kq_solve_param p = S.param;
            p.shifts = S.shifts.data();
            const KuQCDStatus st = kq_solve_multishift_device(S.ctx, &p, S.d_b, S.d_x, &S.info);
            std::lock_guard<std::mutex> lk(large_mu);
            if (st != KUQCD_SUCCESS && st_large == KUQCD_SUCCESS) {
                st_large = st;
                err_large = last_error();
            }
            maxit = std::max(maxit, S.info.iter);
            launches += S.info.kernel_launches;
            if (S.info.iter_refine > 0) ++refined;
            if (S.param.solver == KQ_SOLVER_MIXED)
                for (int k = 0; k < S.param.num_shift; ++k) worst = std::max(worst, S.info.true_residual[k]);
        }
    };
    std::vector<std::thread> large_threads_v;
    const int nlw = (int)std::min<size_t>((size_t)large_threads(), large.size());
    for (int t = 1; t < nlw; ++t) large_threads_v.emplace_back(large_worker);
    large_worker();
    for (auto &t : large_threads_v) t.join();
    if (th.joinable()) th.join();
    for (size_t j = 0; j < small.size(); ++j) all[small[j]].info = b->sys[j].info;
    b->sys.swap(all);
    cudaSetDevice(b->device);
    if (out) {
        memset(out, 0, sizeof(*out));
        out->num_systems = (int)b->sys.size();
        out->iterations = std::max(maxit, bi.iterations);
        out->batched_seconds = bi.batched_seconds;
        out->kernel_launches = launches + bi.kernel_launches;
        out->tile = bi.tile;
        out->ctas_per_sm = bi.ctas_per_sm;
        out->max_true_residual = std::max(worst, bi.max_true_residual);
        out->refined_systems = refined + bi.refined_systems;
        out->tuned_now = bi.tuned_now;
        out->rhs_per_cta = bi.rhs_per_cta;
        out->sites_per_thread = bi.sites_per_thread;
        out->fp64_rhs_per_pass = bi.fp64_rhs_per_pass;
        out->groups = bi.groups + (int)large.size();
        out->check_seconds = bi.check_seconds;
        out->refine_iterations = bi.refine_iterations;
    }
    if (st_small != KUQCD_SUCCESS) {
        set_last_error(err_small);
        return st_small;
    }
    if (st_large != KUQCD_SUCCESS) set_last_error(err_large);
    return st_large;
}
