// The kq_context object behind the C ABI handle, and the workspace helpers the solvers share.
#pragma once
#include "kq_internal.h"
#include "kq_solver.h"

struct kq_context {
    int device = 0;
    unsigned lat[4] = {0, 0, 0, 0};
    kq::Geom g{};
    cudaStream_t stream = nullptr;
    kq::GaugeDev gd;
    int master = -1;  // precision of the loaded links (P64 or P32)
    bool fat_loaded = false, long_loaded = false;
    unsigned *d_scratch = nullptr;
    // solver workspace (grown on demand, never shrunk)
    void *work = nullptr;
    size_t work_bytes = 0;
    // device fields and host-record staging of kq_solve_multishift (host buffers in and out), grown on demand
    void *io = nullptr;
    size_t io_bytes = 0;
    kq::CgmPoll *poll = nullptr;  // pinned host page for state polling
    // t-slab of a domain-decomposed lattice (kq_slab.cu): this context holds local t = 0 .. nt-1 of global
    // t0 = slab_rank * nt; ghost links are the t-direction fat and long links of the 3 slices below t0, per
    // precision (P64, P32, P16): [fat par0 | fat par1 | long par0 | long par1], each one direction of 3 slices
    int slab_rank = -1, slab_nranks = 0;
    void *ghost_links[3] = {nullptr, nullptr, nullptr};  // per precision: P64 (received), P32, P16 (derived)
    bool have_ghost[3] = {false, false, false};
    // Solution notification of a parity solve (set by kq_solve_multishift for the duration of one call): the
    // solvers call solution_ready(ctx, k, user) on the host thread once solution k of their d_x holds the value it
    // will be returned with, and again if a later phase changes it.  Work it enqueues on `stream` runs after
    // everything the solver enqueued so far.
    void (*solution_ready)(kq_context *ctx, int k, void *user) = nullptr;
    void *solution_ready_user = nullptr;
    // copies of solutions to the host that overlap the rest of the solve (created on first use)
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ready = nullptr, copy_done = nullptr;
};

namespace kq {

// 256-byte aligned bump allocator over a workspace; with a null base it only measures.
struct Carve {
    char *base;
    size_t off = 0;
    explicit Carve(void *b) : base(static_cast<char *>(b)) {}
    void *take(size_t n)
    {
        off = (off + 255) & ~size_t(255);
        void *p = base ? base + off : nullptr;
        off += n;
        return p;
    }
};

cudaError_t ensure_work(::kq_context *ctx, size_t bytes);
KuQCDStatus status_of(cudaError_t e);

// KQ_SOLVER_MIXED on one context (kq_mixed.cu); shifts_abs are absolute.  With run_phase1 = false, d_x already
// holds a multishift solution and only the FP64 check / refinement runs.
cudaError_t mixed_solve(::kq_context *ctx, const kq_solve_param *param, const double *shifts_abs, const void *d_b,
                        void *d_x, kq_solve_info *info, bool run_phase1);

}  // namespace kq
