// Solver state and buffers shared between the solver kernels and their host drivers.
#pragma once
#include "kq_internal.h"

namespace kq {

constexpr int kMaxShift = 64;

enum { KQ_STATUS_OK = 0, KQ_STATUS_BREAKDOWN = 1, KQ_STATUS_MAXITER = 2, KQ_STATUS_TIMEOUT = 3 };

// Device-resident CGM state (FP64 scalars).  The first four ints are polled by the host (CgmPoll).
struct CgmState {
    int iter;      // iterations done
    int maxTerm;   // shifts still iterated (reference `maxTerm`)
    int nupd;      // shifts the x/p update kernel must update in the current iteration
    int active;    // 1 while the loop condition of inverter_cgm.cpp:78 holds
    int ns, max_iter, status, halt;
    unsigned ticket, ticket_upd, pad0, pad1;
    double tol;
    double rNorm2, Bm1, pAp, lambda2;
    double shift[kMaxShift];
    double a[kMaxShift], B[kMaxShift], Z[kMaxShift], Zm1[kMaxShift];
};

struct CgmPoll {
    int iter, maxTerm, nupd, active;
};

struct CgmBuffers {
    const void *b;      // source, parity p (solver precision)
    void *r, *s;        // parity p
    void *tmp;          // parity 1-p
    void *p;            // ns direction vectors, vec_bytes apart
    void *x;            // ns solutions, vec_bytes apart
    size_t vec_bytes;
    double *partials;   // one double per block
    CgmState *state;
    CgmPoll *poll;      // pinned host memory
};

struct CgmResult {
    int iter;
    int status;
    double rnorm2;
    double zeta[kMaxShift];
    long long launches;  // kernels enqueued (graph nodes included)
};

// Multishift CG with the reference's recurrences: vectors in `prec` (FP64 or FP32), links in `lp` (= prec, or
// HALF links with FP32 vectors), scalars and reductions in FP64.
cudaError_t cgm_solve(const Geom &g, const GaugeDev &gd, int lp, int prec, const CgmBuffers &w, int parity, int ns,
                      const double *shifts, double tol, int max_iter, int chunk, CgmResult *res, cudaStream_t s);

}  // namespace kq
