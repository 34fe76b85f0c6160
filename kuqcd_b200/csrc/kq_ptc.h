// Parallel-transport convolution layers (kq_ptc.cu) used by the learned preconditioner (kq_net.cu).
#pragma once
#include "kq_internal.h"

namespace kq {

// One layer, cin -> cout channels (1 or 8), on full-lattice activations (layout in kq_ptc.cu).  Bt: [npad][kpad]
// BF16 GEMM matrix built from the complex weights, column k = (p * cin + i) * 2 + reim for path p, input channel i.  swap = true gathers the hops with swapped path labels (the
// adjoint layer, with conjugate-transposed weights).
cudaError_t ptc_forward(const Geom &g, const LinkSet &fat, int cin, int cout, const float2 *in, float2 *out,
                        const void *Bt, bool swap, cudaStream_t s);
// dB[kpad][npad] = sum over all rows of T^T G  (T: the gathered inputs of `in` -- with swapped path labels for an
// adjoint layer -- and G: the output gradient)
cudaError_t ptc_wgrad(const Geom &g, const LinkSet &fat, int cin, int cout, const float2 *in, const float2 *gout,
                      float *partial, float *dB, bool swap, cudaStream_t s);
// cudaErrorLaunchTimeout when a forward tile's tensor-core work did not complete within its wait limit (the
// kernels then leave that tile unwritten); synchronises the stream
cudaError_t ptc_check_fault(cudaStream_t s);
// sets the fault word of the current device from the host, as a timed-out tile would (tests of the error path)
cudaError_t ptc_raise_fault_for_test();
int ptc_kpad(int cin);
int ptc_npad(int cout);
int ptc_tiles(const Geom &g);

cudaError_t ptc_embed(const Geom &g, const void *src, int parity, float2 *act, double scale, cudaStream_t s);
cudaError_t ptc_extract(const Geom &g, const float2 *act, int parity, void *dst, double scale, cudaStream_t s);
cudaError_t ptc_loss(const Geom &g, const float2 *y, const void *e, int parity, double inv_e2, float2 *gout,
                     double *partials, double *loss_host, cudaStream_t s);
// Adam step on grad * grad_scale; clears grad
cudaError_t ptc_adam(float *w, float *grad, float *m, float *v, int n, float lr, float grad_scale, int step,
                     cudaStream_t s);

}  // namespace kq
