/*
 * kuqcd_b200 — C ABI of the B200 (sm_100a) HISQ dslash + multishift CG library (libkuqcd_b200.so).
 *
 * Plain pointers and sizes only.  Precision arguments use KuQCDPrecision values (DOUBLE = 8, SINGLE = 4,
 * HALF = 2).  `stream` arguments are cudaStream_t values passed as void*; NULL selects the context's own stream.
 * Every call returns a KuQCDStatus (0 = success); kq_last_error() gives the message of the last failure on the
 * calling thread.
 *
 * Host record layouts are the reference's NORMAL_ORDER layouts (kuqcd.cpp:103-169):
 *   gauge  h[reim + 2*(l + 9*(dir + 4*s))], s in [0,V): even sites first, then odd; l = col + 3*row
 *   spinor h[reim + 2*(c + 3*i_cb)] over one parity, i_cb = (x>>1) + (nx/2)*(y + ny*(z + nz*t))
 * BATCH_ORDER gauge records (kuqcd.cpp:112-124) are accepted by the kuqcd API twins below.
 */
#ifndef KUQCD_B200_H
#define KUQCD_B200_H

#include <stddef.h>
#include <stdint.h>

#include "kuqcd_enum.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ================================================================ reference-facing entry points
 * C-linkage twins of the five exported calls of include/kuqcd.h:29-34 (the C++ kuqcd:: versions in kuqcd.h
 * forward to these).  Same arguments, same status codes, same call order and ownership rules. */

/* replaces kuqcd::kuqcd_init (kuqcd.cpp:288-301) */
KuQCDStatus kq_kuqcd_init(void);
/* replaces kuqcd::kuqcd_load_gaugefield (kuqcd.cpp:303-402) */
KuQCDStatus kq_kuqcd_load_gaugefield(void *h_gauge, KuQCDGaugeParam *param);
/* replaces kuqcd::kuqcd_solve_multishift (kuqcd.cpp:404-445) */
KuQCDStatus kq_kuqcd_solve_multishift(void **hp_x, void *hp_b, KuQCDInvertParam *param);
/* replaces kuqcd::kuqcd_gauge_free (kuqcd.cpp:447-476) */
void kq_kuqcd_gauge_free(void);
/* replaces kuqcd::kuqcd_end (kuqcd.cpp:477-487) */
void kq_kuqcd_end(void);

/* ================================================================ device-level API
 * A context owns one lattice on one GPU: the device-resident links (FP64 master plus FP32 / HALF copies made on
 * demand), a stream and the solver workspaces.  It replaces the reference's LattBase + GaugeField pair
 * (latt_base.h:19-50, gauge_field.h:19-45) for one rank. */
typedef struct kq_context kq_context;

/* lat = {nx, ny, nz, nt}; nx must be even (checkerboarding, latt_base.cpp:114-116). */
KuQCDStatus kq_context_create(const unsigned lat[4], int device, kq_context **out);
void kq_context_destroy(kq_context *ctx);

/* Copy one link field (KUQCD_FAT_LINK or KUQCD_LONG_LINK) from a NORMAL_ORDER host record of precision
 * host_prec to the device.  Replaces kuqcd_gaugefield_set_values (kuqcd.cpp:103-127). */
KuQCDStatus kq_load_links(kq_context *ctx, int link_type, const void *host, int host_prec);
/* Make both link fields resident in precision prec (SINGLE or HALF copies derived from the loaded master). */
KuQCDStatus kq_prepare_links(kq_context *ctx, int prec);

/* 1 when the long links of precision prec are stored compressed (two rows + 1/s; they are real multiples of SU(3)
 * matrices, as HISQ's Naik links are), 0 for full storage, -1 when not resident.  Set KUQCD_LONG_RECON=0 to keep
 * full storage.  (The reference's reconstruct options are stubs, su3.cpp:250-254; this one needs no caller input.) */
KuQCDStatus kq_long_links_compressed(const kq_context *ctx, int prec, int *out);
/* Bytes of one parity spinor field in the device layout of precision prec. */
size_t kq_spinor_bytes(const kq_context *ctx, int prec);
/* Host record (precision host_prec) <-> device field (precision prec).  Replaces kuqcd_spinorfield_set/get_values
 * (kuqcd.cpp:129-169). */
KuQCDStatus kq_spinor_upload(kq_context *ctx, int prec, const void *host, int host_prec, void *d_field, void *stream);
KuQCDStatus kq_spinor_download(kq_context *ctx, int prec, const void *d_field, void *host, int host_prec,
                               void *stream);
/* Precision conversion between two device fields of the same parity. */
KuQCDStatus kq_spinor_convert(kq_context *ctx, const void *d_src, int src_prec, void *d_dst, int dst_prec,
                              void *stream);

/* d_dst (parity dst_parity) = D d_src (other parity).  Replaces DiracHISQ::Dslash (dirac_hisq.cpp:409-455). */
KuQCDStatus kq_dslash(kq_context *ctx, int prec, const void *d_src, void *d_dst, int dst_parity, void *stream);
/* d_dst = sigma*d_src - D_pq D_qp d_src on parity `parity`; d_tmp holds one field of the other parity.
 * Replaces DiracHISQ::MdaggM (dirac_hisq.cpp:457-462) followed by Axmy (spinor_field.cpp:130-144). */
KuQCDStatus kq_mdagm(kq_context *ctx, int prec, double sigma, const void *d_src, void *d_dst, void *d_tmp,
                     int parity, void *stream);
/* kq_mdagm without a caller temporary and without any device allocation (no counterpart in the reference).
 * For callers that cannot let the library allocate while they apply the operator: applications whose own memory
 * pool reserves nearly all of HBM, and latency-critical loops where cudaMalloc / cudaFree may synchronise the
 * device.  The temporary comes from a 32 MiB array that each GPU loading the library holds until exit; larger
 * fields are rejected with KUQCD_ERR_INVALID_PARAM.  All calls share that array: calls overlapping on the GPU race.
 * Links must already be resident in prec.  The first call on a device looks up the array's address; make it before
 * any stream capture, and do not use this entry point on a device after a cudaDeviceReset in the same process. */
KuQCDStatus kq_mdagm_noalloc(kq_context *ctx, int prec, double sigma, const void *d_src, void *d_dst, int parity,
                             void *stream);

/* Full-lattice (non-preconditioned, KUQCD_HISQ_DIRAC) fields: the parity-0 field followed by the parity-1 field,
 * each kq_spinor_bytes(ctx, prec) long (host records: even sites then odd sites, V*6 values).
 * d_dst = D d_src on both parities in one launch.  Replaces DiracHISQ::Dslash with diracType KUQCD_HISQ_DIRAC on
 * KUQCD_ALL fields (dirac_hisq.cpp:128-136 neighbour offsets, 418-424 site/link offsets). */
KuQCDStatus kq_dslash_full(kq_context *ctx, int prec, const void *d_src, void *d_dst, void *stream);
/* d_dst = sigma*d_src - D D d_src on full-lattice fields; d_tmp: one full-lattice field.  Replaces
 * DiracHISQ::MdaggM (dirac_hisq.cpp:457-462) with KUQCD_HISQ_DIRAC followed by Axmy (spinor_field.cpp:130-144). */
KuQCDStatus kq_mdagm_full(kq_context *ctx, int prec, double sigma, const void *d_src, void *d_dst, void *d_tmp,
                          void *stream);

/* ---------------------------------------------------------------- host-record operators
 * The class-level API of the reference (DiracHISQ::Dslash / MdaggM, dirac_hisq.cpp:409-462; the BLAS-1 free
 * functions of spinor_field.h:40-62) keeps field values in host memory (LatticeField::data, lattice_field.h:23-39).
 * These calls back the header-only classes of include/dirac_hisq.h, spinor_field.h, ...: each copies its operands
 * to the GPU, runs the kernels there and copies the result back before it returns.  Records are NORMAL_ORDER host
 * records (layout above; full-lattice records hold the even sites, then the odd sites). */
/* page-locked host memory for field storage (plain 64-byte aligned memory if page-locking fails) */
KuQCDStatus kq_host_alloc(size_t bytes, void **out);
void kq_host_free(void *p);
enum { KQ_OP_DSLASH = 0, KQ_OP_DD = 1, KQ_OP_SIGMA_MINUS_DD = 2 };
/* h_dst (parity `parity`, or KQ_PARITY_FULL) = op(h_src):
 *   KQ_OP_DSLASH          D h_src, h_src on the other parity (DiracHISQ::Dslash, dirac_hisq.cpp:409-455)
 *   KQ_OP_DD              D D h_src, h_src on the same parity (DiracHISQ::MdaggM, dirac_hisq.cpp:457-462)
 *   KQ_OP_SIGMA_MINUS_DD  sigma h_src - D D h_src (MdaggM followed by Axmy, inverter_cgm.cpp:45-46)
 * prec: precision of the operator (links prepared on first use); host_prec: DOUBLE or SINGLE records. */
KuQCDStatus kq_apply_host(kq_context *ctx, int op, int prec, double sigma, const void *h_src, void *h_dst,
                          int parity, int host_prec);
/* h_y = a h_x + b h_y over n reals of host_prec, computed in host_prec.  Covers Axmy, Axpy, Ymax, Axpby and the
 * field operators of spinor_field.cpp:62-200. */
KuQCDStatus kq_vec_axpby(int device, int host_prec, size_t n, double a, const void *h_x, double b, void *h_y);
/* *out = sum_i h_x[i] h_y[i] over n reals, accumulated in FP64 in a fixed order (RealDot / Norm2,
 * spinor_field.cpp:200-252; h_x == h_y gives Norm2) */
KuQCDStatus kq_vec_dot(int device, int host_prec, size_t n, const void *h_x, const void *h_y, double *out);

/* ---------------------------------------------------------------- domain decomposition along t
 * The multi-rank path of the reference's dslash (halo pack / exchange, dirac_hisq.cpp:236-407; Communicator,
 * communication.cpp:73-138) for one GPU per rank.  Each rank's context holds its slab of the global lattice
 * (local extents nx, ny, nz, nt_local; global t0 = rank * nt_local; nt_local even and >= 4).  The library packs
 * faces into caller buffers; the caller moves them (NCCL send/recv, or any transport) and passes the received
 * buffers to the dslash, which reads them in place:
 *   ghost_lo of rank r = face_hi of rank r-1 (its top 3 t slices), ghost_hi of rank r = face_lo of rank r+1.
 * Ghost links (t-direction links of the 3 slices below t0) are exchanged the same way once after loading:
 * kq_slab_pack_link_face on rank r-1, kq_slab_set_link_ghosts on rank r. */
KuQCDStatus kq_slab_set(kq_context *ctx, int rank, int nranks);
size_t kq_slab_face_bytes(const kq_context *ctx, int prec);          /* one face: 3 t slices of one parity */
KuQCDStatus kq_slab_pack_faces(kq_context *ctx, int prec, const void *d_src, void *d_face_lo, void *d_face_hi,
                               void *stream);
size_t kq_slab_link_face_bytes(const kq_context *ctx);               /* FP64 t links, 3 slices, both types */
KuQCDStatus kq_slab_pack_link_face(kq_context *ctx, void *d_face);  /* top 3 slices, for rank + 1 */
KuQCDStatus kq_slab_set_link_ghosts(kq_context *ctx, const void *d_face); /* received from rank - 1 */
/* d_dst (parity dst_parity) = D d_src on the slab, or sigma * d_pvec - D d_src when d_pvec != NULL; DOUBLE,
 * SINGLE or HALF.  Replaces DiracHISQ::Dslash with np > 1 (StartComm / interior / EndComm, dirac_hisq.cpp:409-455). */
KuQCDStatus kq_slab_dslash(kq_context *ctx, int prec, const void *d_src, const void *d_ghost_lo,
                           const void *d_ghost_hi, void *d_dst, int dst_parity, const void *d_pvec, double sigma,
                           void *stream);
/* The dslash of one part of the slab's output sites: part 0 all, 1 the interior (3 <= t < nt_local - 3; reads no
 * ghost, the ghost pointers may be NULL, so it can run while the faces are in flight), 2 the boundary (the 3 slices at
 * each end, after the ghosts have arrived).  The interior and boundary launches together equal part 0.  DOUBLE,
 * SINGLE or HALF (HALF ghost links take the scales of the context's HALF links). */
KuQCDStatus kq_slab_dslash_part(kq_context *ctx, int prec, const void *d_src, const void *d_ghost_lo,
                                const void *d_ghost_hi, void *d_dst, int dst_parity, const void *d_pvec, double sigma,
                                int part, void *stream);
/* BLAS-1 on FP64 fields of the context (spinor_field.cpp:130-252): y = a x + b y; local Re<x, y> (the caller
 * sums it over ranks, as the reference's MPI_Allreduce does, spinor_field.cpp:207-215) */
KuQCDStatus kq_field_axpby(kq_context *ctx, double a, const void *d_x, double b, void *d_y, void *stream);
KuQCDStatus kq_field_dot(kq_context *ctx, const void *d_x, const void *d_y, double *out);
/* the local Re<x, y> into the device double *d_out, in stream order without a host round trip (an all-reduce over
 * ranks can then run on the device buffer) */
KuQCDStatus kq_field_dot_device(kq_context *ctx, const void *d_x, const void *d_y, double *d_out, void *stream);
/* Device-driven multishift CG over slabs: the recurrences of CGM::Invert (inverter_cgm.cpp:17-87) on a state in
 * device memory, so that no step waits on the host.  Per iteration, in stream order on every rank:
 *   s = shifts_ref[0] p_0 - D D p_0 (two kq_slab_dslash with the halo exchange);
 *   kq_field_dot_device(p_0, s, &state->sums[0]); the caller all-reduces sums[0] in place over ranks;
 *   kq_slab_cgm_step(KQ_CGM_ALPHA); kq_slab_cgm_residual(s, r)   (r += B_0 s, local |r|^2 -> sums[1]);
 *   the caller all-reduces sums[1]; kq_slab_cgm_step(KQ_CGM_BETA); kq_slab_cgm_update(r, p, x);
 *   kq_slab_cgm_step(KQ_CGM_FINISH)   (drops converged shifts, counts the iteration, sets done).
 * Before the first iteration: r = p_j = b, kq_field_dot_device(r, r, &sums[1]), all-reduce, KQ_CGM_START.  Once
 * done is set every step is a no-op, so several iterations may be enqueued between two kq_slab_cgm_poll calls; the
 * iteration count is the reference's.  shifts_ref have the reference's meaning (shift 0 absolute, shift j relative
 * to it); shift j stops when Z_j^2 |r|^2 < tol.  d_state: kq_slab_cgm_state_bytes() of device memory, 8-byte
 * aligned. */
typedef struct {
    double sums[2]; /* [0] <p_0, A p_0>, [1] |r|^2: local sums from the library, all-reduced in place by the caller */
    double rr, Bm1, tol;
    int iter, max_iter, num_shift, max_term, done, reserved;
    double sh[64], a[64], B[64], Z[64], Zm1[64];
} kq_slab_cgm_state;
enum { KQ_CGM_START = 0, KQ_CGM_ALPHA = 1, KQ_CGM_BETA = 2, KQ_CGM_FINISH = 3 };
size_t kq_slab_cgm_state_bytes(void);
KuQCDStatus kq_slab_cgm_init(kq_context *ctx, kq_slab_cgm_state *d_state, int num_shift, const double *shifts_ref,
                             double tol, int max_iter, void *stream);
KuQCDStatus kq_slab_cgm_step(kq_context *ctx, kq_slab_cgm_state *d_state, int step, void *stream);
KuQCDStatus kq_slab_cgm_residual(kq_context *ctx, kq_slab_cgm_state *d_state, const void *d_s, void *d_r,
                                 void *stream);
KuQCDStatus kq_slab_cgm_update(kq_context *ctx, const kq_slab_cgm_state *d_state, const void *d_r, void *d_p,
                               void *d_x, size_t stride, void *stream);
/* iterations so far, whether the solve has stopped and (rr != NULL) the current |r|^2 (waits for the stream) */
KuQCDStatus kq_slab_cgm_poll(kq_context *ctx, const kq_slab_cgm_state *d_state, int *iter, int *done, double *rr,
                             void *stream);

/* ---------------------------------------------------------------- solver */
enum {
    KQ_SOLVER_CGM = 0,        /* multishift CG with the reference's recurrences (CGM::Invert), FP64 or FP32 */
    KQ_SOLVER_MIXED = 1,      /* relaxed-precision multishift (FP64 -> FP32 -> HALF operator as |r| falls) with an
                                 FP64 true-residual check and batched reliable-update refinement of any shift left
                                 above rel_residual; prec = SINGLE or HALF is the cheapest operator it may use */
    KQ_SOLVER_CGM_WINDOWED = 2 /* the CGM recurrences in FP64 with windowed shift updates (same iterates as
                                  KQ_SOLVER_CGM up to rounding, 4N -> (4N+8)/8 vector sweeps per iteration) */
};

enum { KQ_PARITY_FULL = 2 };

typedef struct {
    int parity;               /* 0: source and solutions on even sites (EVEN_EVEN), 1: odd (ODD_ODD),
                                 KQ_PARITY_FULL: full-lattice fields (KUQCD_HISQ_DIRAC); sigma - D D is block
                                 diagonal there, so each parity is solved on its own, to tol / 2 (the reference
                                 rule over both parities) or to the share of rel_residual |b| that keeps the
                                 full-lattice residual within target */
    int num_shift;            /* 1..64 */
    const double *shifts;     /* see shift_mode */
    int shift_mode;           /* 0: reference semantics, x_j solves (shifts[0] + shifts[j] - DD) for j >= 1
                                 1: absolute, x_j solves (shifts[j] - DD) x = b */
    int solver;               /* KQ_SOLVER_* */
    int prec;                 /* KQ_SOLVER_CGM: DOUBLE or SINGLE; KQ_SOLVER_MIXED: sloppy SINGLE or HALF */
    int host_prec;            /* precision of the host b / x records */
    int max_iter;
    double tol;               /* KQ_SOLVER_CGM: reference stopping rule zeta_k^2 |r|^2 < tol */
    double rel_residual;      /* KQ_SOLVER_MIXED: per-shift true relative residual target; < 0: absolute target
                                 |b - A_k x_k|^2 < tol instead (single-system solves) */
} kq_solve_param;

typedef struct {
    int iter;                 /* multishift iterations */
    int iter_refine;          /* refinement iterations summed over shifts (KQ_SOLVER_MIXED) */
    int status;               /* 0 ok, 1 breakdown, 2 max_iter reached */
    int num_shift;
    double true_residual[64]; /* |b - (sigma_k - DD) x_k| / |b| in FP64, when computed */
    double seconds;           /* device time of the solve */
    long long kernel_launches;/* kernels the solve enqueued (graph nodes included) */
    double sloppy_residual;   /* KQ_SOLVER_MIXED: largest true relative residual after the sloppy multishift */
    int copies_during_solve;  /* kq_solve_multishift: solutions whose copy to the host began before the solve ended */
} kq_solve_info;

/* Host b (Vh*6 values of host_prec; V*6 for KQ_PARITY_FULL) -> host x[k].  Copies in, solves on the device,
 * copies out.  With page-locked x buffers (cudaHostAlloc / cudaHostRegister) and a parity solve, each solution is
 * copied out as soon as the solver has finished with it (a shift that converges early), on a second stream, while
 * the solve continues; a solution that the refinement changes afterwards is copied again.  The call returns after
 * every copy has completed. */
KuQCDStatus kq_solve_multishift(kq_context *ctx, const kq_solve_param *param, const void *host_b,
                                void *const *host_x, kq_solve_info *info);
/* Same with device fields in FP64 (d_b: one field; d_x: num_shift fields, kq_spinor_bytes(ctx, 8) apart; twice
 * that for KQ_PARITY_FULL). */
KuQCDStatus kq_solve_multishift_device(kq_context *ctx, const kq_solve_param *param, const void *d_b, void *d_x,
                                       kq_solve_info *info);
/* FP64 true relative residuals |b - (sigma_k - DD) x_k| / |b| of device FP64 fields (absolute sigmas; parity
 * KQ_PARITY_FULL: full-lattice fields, norms over both parities). */
KuQCDStatus kq_true_residuals(kq_context *ctx, int parity, int num_shift, const double *sigma, const void *d_b,
                              const void *d_x, double *out);

/* ---------------------------------------------------------------- batched systems
 * Many independent systems (each its own context: lattice, links; its own shifts and source) solved together: each
 * kernel of an iteration is one persistent launch over all systems' site tiles, captured in CUDA graphs.  Systems
 * added with the same context (several sources or masses on one gauge field) and parity are grouped: the dslash
 * loads each link once for every member of the group (multi-RHS).  Launch shape -- threads per CTA, CTAs per SM,
 * right-hand sides per CTA, sites per thread -- autotuned on the batch and cached on disk (KUQCD_TUNE_CACHE).  No reference counterpart: the reference solves one
 * system per kuqcd_solve_multishift call (kuqcd.cpp:404-445), so this replaces a loop of such calls. */
typedef struct kq_batch kq_batch;
typedef struct {
    int num_systems;
    int iterations;           /* largest iteration count over the systems */
    double batched_seconds;   /* device time of the batched iterations */
    long long kernel_launches;
    int tile;                 /* sites per tile = threads per CTA */
    int ctas_per_sm;          /* persistent grid: CTAs per SM */
    double max_true_residual; /* over the KQ_SOLVER_MIXED systems' shifts (FP64, after any refinement) */
    int refined_systems;      /* systems the FP64 check sent to refinement */
    int tuned_now;            /* 1 when this call measured the launch shape */
    int rhs_per_cta;          /* systems on one gauge field whose dslash shares each link load (1, 2, 4 or 8) */
    int sites_per_thread;     /* sites each thread handles per work item */
    int fp64_rhs_per_pass;    /* right-hand sides the FP64 dslash serves per link load (1, 2 or 4); 0: all of a
                                 group, spread over the warps with the links staged in shared memory */
    int groups;               /* groups of systems sharing link loads (+ systems solved on their own) */
    double check_seconds;     /* wall time of the batched systems' FP64 checks and refinements */
    int refine_iterations;    /* refinement iterations summed over the batched systems */
} kq_batch_info;

KuQCDStatus kq_batch_create(int device, kq_batch **out);
void kq_batch_destroy(kq_batch *b);
/* d_b: FP64 device field of ctx; d_x: num_shift FP64 fields, kq_spinor_bytes(ctx, DOUBLE) apart.  solver:
 * KQ_SOLVER_MIXED or KQ_SOLVER_CGM_WINDOWED.  ctx must hold FP64 links and outlive the batch. */
KuQCDStatus kq_batch_add(kq_batch *b, kq_context *ctx, const kq_solve_param *param, const void *d_b, void *d_x);
int kq_batch_size(const kq_batch *b);
KuQCDStatus kq_batch_solve(kq_batch *b, kq_batch_info *info);
KuQCDStatus kq_batch_system_info(const kq_batch *b, int i, kq_solve_info *out);

/* ---------------------------------------------------------------- learned preconditioner
 * A gauge-covariant parallel-transport convolution network (layers of y_o = sum_i,p W[o][i][p] T_p v_i with the
 * context's fat links as parallel transporters; BF16 tensor-core channel mixing, FP32 accumulation) trained on
 * solver-generated residual/error pairs, used by a per-shift flexible-CG polish.  The preconditioner is the Gram
 * operator M = N^dag N of the layer chain N (symmetric positive semi-definite by construction).  No reference
 * counterpart (the reference's CGM is unpreconditioned, inverter_cgm.cpp:17-87). */
typedef struct kq_net kq_net;
/* channels[0..nlayers] of N: 1, then 1 or 8 each (M runs the 2 * nlayers layers of N and N^dag) */
KuQCDStatus kq_net_create(kq_context *ctx, int nlayers, const int *channels, kq_net **out);
void kq_net_destroy(kq_net *net);
size_t kq_net_num_weights(const kq_net *net); /* floats: complex weights as (re, im) pairs, layers concatenated */
KuQCDStatus kq_net_set_weights(kq_net *net, const float *w, size_t count);
KuQCDStatus kq_net_get_weights(const kq_net *net, float *w, size_t count);
KuQCDStatus kq_net_get_grad(const kq_net *net, float *grad, size_t count);
KuQCDStatus kq_net_zero_grad(kq_net *net);
/* switch to the links of another context of the same lattice */
KuQCDStatus kq_net_set_context(kq_net *net, kq_context *ctx);
/* d_out = M(d_in), FP64 fields of parity `parity` */
KuQCDStatus kq_net_apply(kq_net *net, const void *d_in, void *d_out, int parity);
/* one training pair: forward, loss |M(r) - e|^2 / e_norm2, backward; the weight gradient is accumulated */
KuQCDStatus kq_net_train_pair(kq_net *net, const void *d_r, const void *d_e, int parity, double e_norm2,
                              double *loss);
/* Adam step on the accumulated gradient times grad_scale; clears the accumulator */
KuQCDStatus kq_net_adam(kq_net *net, float lr, float grad_scale);
/* Test hook (no reference counterpart): sets the device word that a tensor-core tile sets when its bounded wait runs
 * out, so that the next kq_net_apply / kq_net_train_pair reports KUQCD_ERR_UNKNOWN_ERROR once and the call after it
 * succeeds.  Exercises the error path without making any GPU wait time out. */
KuQCDStatus kq_net_raise_fault_for_test(kq_net *net);
/* Polish every shift of d_x (initial guesses, num_shift FP64 fields) to the FP64 true relative residual
 * param->rel_residual with FCG preconditioned by net (NULL: plain CG, also the fallback on breakdown, stagnation
 * or an exhausted budget).  info->iter_refine: all polish iterations; info->iter: those that applied the net. */
KuQCDStatus kq_fcg_polish(kq_context *ctx, kq_net *net, const kq_solve_param *param, const void *d_b, void *d_x,
                          kq_solve_info *info);

/* ---------------------------------------------------------------- synthetic fields
 * thin U = exp(i eps H), H traceless Hermitian from seeded Gaussians; staggered phases folded in;
 * fat = 9/8 U, long = -1/24 U(x) U(x+mu) U(x+2mu); written as FP64 NORMAL_ORDER host records into DEVICE
 * buffers of V*72 doubles each.  Source: Gaussian colour vectors on one parity (Vh*6 doubles). */
KuQCDStatus kq_make_links_record(kq_context *ctx, double eps, uint64_t seed, double *d_fat, double *d_long);
KuQCDStatus kq_make_source_record(kq_context *ctx, int parity, uint64_t seed, double *d_b);

const char *kq_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
