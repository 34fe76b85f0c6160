/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * extern "C" entry points into the UNMODIFIED reference KuQCD sources, compiled together with them into
 * oracle/_ref/libkuqcd_ref.so by oracle/Makefile.  Tests, golden-fixture generation and the CPU-baseline leg of
 * bench.py call these through ctypes to get the reference's own answers; the kuqcd_b200 product never links
 * or loads this library.
 *
 * What each entry point drives in the reference:
 *   kqref_set_grid1        -> the effect of kuqcd_init() (kuqcd.cpp:288-301) with a 1x1x1x1 grid, without
 *                             reading stdin (command_line.cpp:31-84 reads the grid from stdin).
 *   kqref_load_gaugefield  -> kuqcd::kuqcd_load_gaugefield (kuqcd.cpp:303-402)
 *   kqref_solve_multishift -> kuqcd::kuqcd_solve_multishift (kuqcd.cpp:404-445) -> CGM::Invert
 *                             (inverter_cgm.cpp:17-87)
 *   kqref_gauge_free / kqref_end -> kuqcd.cpp:447-487
 *   kqref_dslash_{d,f}     -> one DiracHISQ<T,1,NO,NO>::Dslash (dirac_hisq.cpp:409-455) on even-odd fields,
 *                             host arrays in the NORMAL_ORDER layout of kuqcd.cpp:103-169.
 *   kqref_mdaggm_d         -> DiracHISQ::MdaggM (dirac_hisq.cpp:457-462).
 *   kqref_dslash_full_d    -> DiracHISQ<double,1,NO,NO>::Dslash with diracType KUQCD_HISQ_DIRAC on KUQCD_ALL
 *                             fields (the non-preconditioned operator, dirac_hisq.cpp:128-136, 418-424); host
 *                             arrays hold even sites then odd sites.
 */
#include <cstring>
#include <new>
#include "kuqcd.h"

namespace kuqcd {
extern std::array<unsigned short, 4> g_grid_dim;
}

using namespace kuqcd;

namespace {

template <typename T>
void scatter_gauge(GaugeField<T, 1, KUQCD_GAUGE_RECON_NO> &g, const T *h)
{
    // host record: h[reim + 2*(l + 9*(dir + 4*i))], i = even-odd site index (kuqcd.cpp:103-127, Nbatch = 1)
    const size_t vol = g.latBase.lenBulk;
    for (size_t i = 0; i < vol; ++i) {
        const size_t f = g.latBase.myIdx.idx[i];
        for (int dir = 0; dir < 4; ++dir)
            for (int l = 0; l < 9; ++l) {
                g.data[dir + 4 * f].m[l].z[0] = h[0 + 2 * (l + 9 * (dir + 4 * i))];
                g.data[dir + 4 * f].m[l].z[1] = h[1 + 2 * (l + 9 * (dir + 4 * i))];
            }
    }
}

template <typename T>
void scatter_spinor(SpinorField<T, 1, 1> &s, const T *h)
{
    const size_t vol = s.latBase.lenBulk;
    for (size_t i = 0; i < vol; ++i) {
        const size_t f = s.latBase.myIdx.idx[i];
        for (int c = 0; c < 3; ++c) {
            s.data[f].c[c].z[0] = h[0 + 2 * (c + 3 * i)];
            s.data[f].c[c].z[1] = h[1 + 2 * (c + 3 * i)];
        }
    }
}

template <typename T>
void gather_spinor(const SpinorField<T, 1, 1> &s, T *h)
{
    const size_t vol = s.latBase.lenBulk;
    for (size_t i = 0; i < vol; ++i) {
        const size_t f = s.latBase.myIdx.idx[i];
        for (int c = 0; c < 3; ++c) {
            h[0 + 2 * (c + 3 * i)] = s.data[f].c[c].z[0];
            h[1 + 2 * (c + 3 * i)] = s.data[f].c[c].z[1];
        }
    }
}

/* One even-odd dslash (or M^dag M when mdaggm != 0) on freshly built reference objects.
 * dst_parity: 0 = even output sites, 1 = odd.  src lives on the other parity. */
template <typename T>
int run_dslash(const unsigned *lat, const T *fat, const T *lng, const T *src, T *dst, int dst_parity, int mdaggm,
               int reps)
{
    std::array<unsigned short, 4> grid{1, 1, 1, 1};
    const KuQCDPrecision prec = sizeof(T) == 8 ? KUQCD_DOUBLE : KUQCD_SINGLE;
    Lattice sup(lat[0], lat[1], lat[2], lat[3]);
    LattBase all(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, prec, KUQCD_ALL);
    LattBase even(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, prec, KUQCD_EVEN);
    LattBase odd(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, prec, KUQCD_ODD);
    CommBase comm(all);
    GaugeField<T, 1, KUQCD_GAUGE_RECON_NO> gf(all, comm), gl(all, comm);
    scatter_gauge(gf, fat);
    scatter_gauge(gl, lng);
    LattBase &lp = dst_parity == 0 ? even : odd;
    LattBase &lq = dst_parity == 0 ? odd : even;
    if (mdaggm) {
        // MdaggM maps parity p -> p through a temporary on the other parity (dirac_hisq.cpp:457-462)
        SpinorField<T, 1, 1> in(lp), out(lp), tmp(lq);
        scatter_spinor(in, src);
        DiracHISQ<T, 1, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> d(KUQCD_HISQPC_DIRAC, gf, gl, 0, &tmp);
        for (int r = 0; r < reps; ++r) d.MdaggM(in, out, true);
        gather_spinor(out, dst);
    } else {
        SpinorField<T, 1, 1> in(lq), out(lp);
        scatter_spinor(in, src);
        DiracHISQ<T, 1, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> d(KUQCD_HISQPC_DIRAC, gf, gl, 0, nullptr);
        for (int r = 0; r < reps; ++r) d.Dslash(in, out, false);
        gather_spinor(out, dst);
    }
    return 0;
}

/* One non-PC dslash on full-lattice reference objects (KUQCD_ALL spinors, KUQCD_HISQ_DIRAC). */
int run_dslash_full(const unsigned *lat, const double *fat, const double *lng, const double *src, double *dst)
{
    std::array<unsigned short, 4> grid{1, 1, 1, 1};
    Lattice sup(lat[0], lat[1], lat[2], lat[3]);
    LattBase all(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_DOUBLE, KUQCD_ALL);
    CommBase comm(all);
    GaugeField<double, 1, KUQCD_GAUGE_RECON_NO> gf(all, comm), gl(all, comm);
    scatter_gauge(gf, fat);
    scatter_gauge(gl, lng);
    SpinorField<double, 1, 1> in(all), out(all);
    scatter_spinor(in, src);
    DiracHISQ<double, 1, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> d(KUQCD_HISQ_DIRAC, gf, gl, 0, nullptr);
    d.Dslash(in, out, false);
    gather_spinor(out, dst);
    return 0;
}

} // namespace

extern "C" {

__attribute__((visibility("default"))) int kqref_dslash_full_d(const unsigned *lat, const double *fat,
                                                               const double *lng, const double *src, double *dst)
{
    try {
        return run_dslash_full(lat, fat, lng, src, dst);
    } catch (...) {
        return -1;
    }
}

__attribute__((visibility("default"))) void kqref_set_grid1()
{
    g_grid_dim = {1, 1, 1, 1};
}

__attribute__((visibility("default"))) int kqref_load_gaugefield(void *h, const unsigned *lat, int prec, int order,
                                                                 int link_type, int site_subset, int halo_depth)
{
    KuQCDGaugeParam p;
    std::memset(&p, 0, sizeof(p));
    for (int i = 0; i < 4; ++i) p.lat[i] = lat[i];
    p.halo_depth = halo_depth;
    p.od = KUQCD_TZYX_ORDER;
    p.site_subset = (KuQCDSiteSubset)site_subset;
    p.gauge_order = (KuQCDGaugeOrder)order;
    p.prec = (KuQCDPrecision)prec;
    p.link_type = (KuQCDLinkType)link_type;
    p.recon = KUQCD_GAUGE_RECON_NO;
    return (int)kuqcd_load_gaugefield(h, &p);
}

__attribute__((visibility("default"))) int kqref_solve_multishift(void **x, void *b, int dslash_type, int matpc,
                                                                  int prec, int num_shift, int max_iter, double tol,
                                                                  double *shifts, int *iter_out)
{
    KuQCDInvertParam p;
    std::memset(&p, 0, sizeof(p));
    p.dslash_type = (KuQCDDslashType)dslash_type;
    p.inverter_type = KUQCD_CGM;
    p.matpc_type = (KuQCDMatPCType)matpc;
    p.prec = (KuQCDPrecision)prec;
    p.num_shift = num_shift;
    p.max_iter = max_iter;
    p.tol = tol;
    p.shifts = shifts;
    KuQCDStatus st = kuqcd_solve_multishift(x, b, &p);
    if (iter_out) *iter_out = p.iter;
    return (int)st;
}

__attribute__((visibility("default"))) void kqref_gauge_free()
{
    kuqcd_gauge_free();
}

__attribute__((visibility("default"))) void kqref_end()
{
    kuqcd_end();
}

__attribute__((visibility("default"))) int kqref_dslash_d(const unsigned *lat, const double *fat, const double *lng,
                                                          const double *src, double *dst, int dst_parity, int reps)
{
    try {
        return run_dslash<double>(lat, fat, lng, src, dst, dst_parity, 0, reps);
    } catch (std::bad_alloc &) {
        return -4;
    }
}

__attribute__((visibility("default"))) int kqref_dslash_f(const unsigned *lat, const float *fat, const float *lng,
                                                          const float *src, float *dst, int dst_parity, int reps)
{
    try {
        return run_dslash<float>(lat, fat, lng, src, dst, dst_parity, 0, reps);
    } catch (std::bad_alloc &) {
        return -4;
    }
}

__attribute__((visibility("default"))) int kqref_mdaggm_d(const unsigned *lat, const double *fat, const double *lng,
                                                          const double *src, double *dst, int parity, int reps)
{
    try {
        return run_dslash<double>(lat, fat, lng, src, dst, parity, 1, reps);
    } catch (std::bad_alloc &) {
        return -4;
    }
}

} // extern "C"
