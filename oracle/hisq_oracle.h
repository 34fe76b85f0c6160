/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — a plain-C restatement of the KuQCD HISQ even-odd dslash and multishift CG,
 * used by tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py as the checker.  The kuqcd_b200
 * product never links, loads or calls it.
 *
 * Parity pinned: against the reference library built from its own sources (oracle/_ref/libkuqcd_ref.so, see
 * oracle/Makefile) and against the reference's known-answer test (test/test_solver.cpp:27-130).
 *
 * Host layouts (NORMAL_ORDER, one rank; kuqcd.cpp:103-169, latt_base.cpp:170-212, index_utils.cpp:91-100):
 *   checkerboard index  i_cb = (x >> 1) + (nx/2) * (y + ny * (z + nz * t)),  x = 2*xcb + ((y+z+t+parity) & 1)
 *   gauge  g[reim + 2*(l + 9*(dir + 4*i))], i in [0, V): even sites (i = i_cb) then odd (i = Vh + i_cb);
 *          l = col + 3*row (row-major SU(3), kuqcd_math.cpp:20-35)
 *   spinor s[reim + 2*(c + 3*i_cb)] over one parity.
 */
#ifndef KQ_HISQ_ORACLE_H
#define KQ_HISQ_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* one even-odd dslash: dst(parity p) = D src(parity 1-p)      (dirac_hisq.cpp:409-502) */
void kqo_dslash_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst,
                  int dst_parity);
void kqo_dslash_f(const int dims[4], const float *fat, const float *lng, const float *src, float *dst,
                  int dst_parity);
/* full lattice (KUQCD_HISQ_DIRAC, dirac_hisq.cpp:128-136, 418-424): src/dst hold even sites then odd sites
 * (V*6 values); every output site gets D applied to the other parity half */
void kqo_dslash_full_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst);
/* dst = D_pq D_qp src  (MdaggM, dirac_hisq.cpp:457-462); tmp has Vh*6 entries */
void kqo_mdaggm_d(const int dims[4], const double *fat, const double *lng, const double *src, double *dst,
                  double *tmp, int parity);

/* CGM::Invert (inverter_cgm.cpp:17-87) with the reference's shift semantics: x_0 solves (shifts[0] - DD) x = b,
 * x_j (j >= 1) solves (shifts[0] + shifts[j] - DD) x = b; stops shift k when Z_k^2 |r|^2 < tol.
 * x: num_shift arrays of Vh*6.  Returns the iteration count. */
int kqo_cgm_d(const int dims[4], const double *fat, const double *lng, int parity, int num_shift,
              const double *shifts, const double *b, double **x, double tol, int max_iter);
int kqo_cgm_f(const int dims[4], const float *fat, const float *lng, int parity, int num_shift,
              const float *shifts, const float *b, float **x, double tol, int max_iter);

/* |b - (sigma - D D) x| / |b| in FP64 (sigma absolute) */
double kqo_true_residual_d(const int dims[4], const double *fat, const double *lng, int parity, double sigma,
                           const double *b, const double *x);

/* Synthetic benchmark fields: thin U_mu(x) = exp(i eps H), H traceless Hermitian from seeded Gaussians;
 * staggered phases eta folded in; fat = 9/8 eta U; long = -1/24 eta U(x) U(x+mu) U(x+2mu).  Writes the host
 * gauge layout above.  thin may be NULL. */
void kqo_make_links(const int dims[4], double eps, uint64_t seed, double *fat, double *lng, double *thin);
/* Gaussian complex colour vectors on one parity (Vh*6 doubles) */
void kqo_make_source(const int dims[4], int parity, uint64_t seed, double *b);
/* the generator's building blocks, exposed for unit tests */
uint64_t kqo_hash(uint64_t seed, uint64_t counter);
void kqo_su3_exp_iH(const double *H, double eps, double *U); /* H, U: 9 complex, interleaved re/im */

#ifdef __cplusplus
}
#endif
#endif
