// Windowed, relaxed-precision multishift CG (kq_msrelax.cu).
#pragma once
#include "kq_context.h"

namespace kq {

constexpr int kWin = 16;   // iterations per shift-update window (ring of residuals)
constexpr int kChunk = 8;  // iterations per CUDA graph: the host picks the operator precision between chunks

struct MsState {
    int iter, maxTerm, active, wpos;  // polled
    double rNorm2, bnorm2;            // polled
    int ns, max_iter, status, halt;
    int nupd, wmax, pad0, pad1;
    unsigned ticket[4];
    double tol;
    double Bm1, pAp, lambda2;
    double pp;  // |p0|^2, kept by the recurrence |p'|^2 = |r'|^2 + a0^2 |p|^2; <p0, A p0> = sigma0 |p0|^2 + |D p0|^2
    double shift[kMaxShift];  // reference semantics: shift[0] absolute, shift[j] = sigma_j - sigma_0
    double a[kMaxShift], B[kMaxShift], Z[kMaxShift], Zm1[kMaxShift];
    double c[kMaxShift], e[kMaxShift];           // p_k, x_k coefficients of p_k at the window start
    double d[kMaxShift][kWin], f[kMaxShift][kWin];  // coefficients of the ring residuals
    int mode, next_mode;  // batched solver: operator precision of this / the next iteration (0 FP64, 1 FP32, 2 HALF)
    double rho32_2, rho16_2;  // squared relative-residual switch points (0: never)
    int *running;             // batched solver: systems still iterating (decremented when this one stops)
};

struct MsPoll {
    int iter, maxTerm, active, wpos;
    double rNorm2, bnorm2;
};

struct MsBuffers {
    const void *b;  // FP64 source
    void *x;        // ns FP64 solutions, vb apart
    void *p0, *tmp, *ring, *pw;
    size_t vb;
    double *partials;
    MsState *st;
};

struct MsResult {
    int iter, status;
    long long launches;
    int chunks[3];  // chunks of kChunk iterations run with FP64 / FP32 / HALF operators
};

void ms_layout(Carve &c, const Geom &g, int ns, const void *d_b, void *d_x, MsBuffers &w);
size_t ms_workspace_bytes(const Geom &g, int ns);

// rho32 / rho16: switch the operator to FP32 / HALF links once |r| < rho |b| (0 disables that precision).
// tol follows the reference rule zeta_k^2 |r|^2 < tol; shifts_ref are in reference semantics.
cudaError_t ms_solve(::kq_context *ctx, const MsBuffers &w, int parity, int ns, const double *shifts_ref, double tol,
                     int max_iter, double rho32, double rho16, MsResult *res);

}  // namespace kq
