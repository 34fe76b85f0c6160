// Mixed-precision multishift solver (placeholder until the sloppy/refinement kernels land).
#include "kq_internal.h"
#include "kq_solver.h"

namespace kq {
cudaError_t mixed_solve(::kq_context *ctx, const kq_solve_param *param, const double *shifts_abs, const void *d_b,
                        void *d_x, kq_solve_info *info)
{
    (void)ctx; (void)param; (void)shifts_abs; (void)d_b; (void)d_x; (void)info;
    set_last_error("mixed solver not available in this build");
    return cudaErrorNotSupported;
}
}  // namespace kq
