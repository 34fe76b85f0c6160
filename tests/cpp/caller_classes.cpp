// A caller of KuQCD's class-level API (the types kuqcd.h brings in: Lattice, LattBase, CommBase, GaugeField,
// SpinorField and its BLAS-1 functions, DiracHISQ, CGM), written as the reference's own glue uses them
// (kuqcd.cpp:41-286): fields filled through data[] and latBase.myIdx, the operator built from the two link fields,
// the inverter from the operator.
//
//   caller_classes <dir> nx ny nz nt num_shift
//
// reads <dir>/fat.bin, <dir>/long.bin (V*72 doubles, NORMAL_ORDER records), <dir>/b_even.bin, <dir>/b_odd.bin
// (V/2*6 doubles), <dir>/shifts.bin (num_shift doubles, reference semantics), <dir>/tol.bin; writes
//   dslash_even.bin   D b_odd onto even sites (FP64)          dslash_even_f.bin  the same in FP32
//   mdaggm_even.bin   D D b_even (FP64)                       blas.txt           BLAS-1 results (see below)
//   axpby.bin         the field after the BLAS sequence        x<k>.bin, cgm.txt  CGM::Invert solutions, iterations
//   dslash_batch.bin  D b_odd in FP32 through BATCH_ORDER (16-lane) fields, written back in NORMAL order
//                     (only when nx = 32, the width BATCH_ORDER float needs)
// Test infrastructure: the GPU tests compare these with the oracle.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "kuqcd.h"

using namespace kuqcd;

static std::vector<double> read_all(const std::string &path, size_t n)
{
    std::vector<double> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(double), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(2);
    }
    fclose(f);
    return v;
}

template <typename T>
static void write_all(const std::string &path, const std::vector<T> &v)
{
    FILE *f = fopen(path.c_str(), "wb");
    fwrite(v.data(), sizeof(T), v.size(), f);
    fclose(f);
}

// NORMAL_ORDER record <-> fields, through myIdx (kuqcd.cpp:103-169 with Nbatch = 1)
template <typename T>
static void set_gauge(GaugeField<T, 1, KUQCD_GAUGE_RECON_NO> &g, const std::vector<double> &rec)
{
    for (size_t i = 0; i < g.latBase.lenBulk; ++i) {
        const size_t f = g.latBase.myIdx.idx[i];
        for (int dir = 0; dir < 4; ++dir)
            for (int l = 0; l < 9; ++l) {
                g.data[dir + 4 * f].m[l].z[0] = (T)rec[72 * i + 18 * dir + 2 * l];
                g.data[dir + 4 * f].m[l].z[1] = (T)rec[72 * i + 18 * dir + 2 * l + 1];
            }
    }
}
template <typename T>
static void set_spinor(SpinorField<T, 1, 1> &s, const std::vector<double> &rec)
{
    for (size_t i = 0; i < s.latBase.lenBulk; ++i) {
        const size_t f = s.latBase.myIdx.idx[i];
        for (int c = 0; c < 3; ++c) {
            s.data[f].c[c].z[0] = (T)rec[6 * i + 2 * c];
            s.data[f].c[c].z[1] = (T)rec[6 * i + 2 * c + 1];
        }
    }
}
template <typename T>
static std::vector<T> get_spinor(const SpinorField<T, 1, 1> &s)
{
    std::vector<T> rec(6 * s.latBase.lenBulk);
    for (size_t i = 0; i < s.latBase.lenBulk; ++i) {
        const size_t f = s.latBase.myIdx.idx[i];
        for (int c = 0; c < 3; ++c) {
            rec[6 * i + 2 * c] = s.data[f].c[c].z[0];
            rec[6 * i + 2 * c + 1] = s.data[f].c[c].z[1];
        }
    }
    return rec;
}

// BATCH_ORDER (Nb lanes along x): real site of lane j of reduced checkerboard site i of parity par, written from
// the layout rule itself -- reduced x_r = 2 x_cb + ((y + z + t + par) & 1), real x = x_r + (nx / Nb) j
static size_t batch_real_cb(const LattBase &lb, size_t i, int par, int j, const unsigned lat[4])
{
    const Lattice &red = lb.latSubBulkCB;
    const size_t xcb = i % red.nx, y = (i / red.nx) % red.ny, z = (i / red.nx / red.ny) % red.nz,
                 t = i / red.nx / red.ny / red.nz;
    const size_t xr = 2 * xcb + ((y + z + t + par) & 1);
    const size_t x = xr + (lat[0] / lb.Nbatch) * j;
    return (x >> 1) + (lat[0] / 2) * (y + lat[1] * (z + lat[2] * t));
}

static void batch_dslash(const std::string &dir, const unsigned lat[4], const std::vector<double> &fat,
                         const std::vector<double> &lng, const std::vector<double> &b_odd)
{
    constexpr int NB = 16;
    const std::array<unsigned short, 4> grid{1, 1, 1, 1};
    const Lattice sup(lat[0], lat[1], lat[2], lat[3]);
    LattBase all(sup, grid, 0, KUQCD_BATCH_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_ALL);
    LattBase even(sup, grid, 0, KUQCD_BATCH_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_EVEN);
    LattBase odd(sup, grid, 0, KUQCD_BATCH_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_ODD);
    CommBase comm(all);
    GaugeField<float, NB, KUQCD_GAUGE_RECON_NO> gf(all, comm), gl(all, comm);
    const size_t vh = sup.V / 2, vhr = all.latSubBulkCB.V;
    for (size_t i = 0; i < all.lenBulk; ++i) {
        const int par = i < vhr ? 0 : 1;
        const size_t f = all.myIdx.idx[i];
        for (int j = 0; j < NB; ++j) {
            const size_t s = batch_real_cb(all, par ? i - vhr : i, par, j, lat) + (par ? vh : 0);
            for (int d = 0; d < 4; ++d)
                for (int l = 0; l < 9; ++l) {
                    gf.data[d + 4 * f].m[l].z[j] = (float)fat[72 * s + 18 * d + 2 * l];
                    gf.data[d + 4 * f].m[l].z[NB + j] = (float)fat[72 * s + 18 * d + 2 * l + 1];
                    gl.data[d + 4 * f].m[l].z[j] = (float)lng[72 * s + 18 * d + 2 * l];
                    gl.data[d + 4 * f].m[l].z[NB + j] = (float)lng[72 * s + 18 * d + 2 * l + 1];
                }
        }
    }
    SpinorField<float, NB, 1> in(odd), out(even);
    for (size_t i = 0; i < odd.lenBulk; ++i)
        for (int j = 0; j < NB; ++j) {
            const size_t s = batch_real_cb(odd, i, 1, j, lat);
            for (int c = 0; c < 3; ++c) {
                in.data[odd.myIdx.idx[i]].c[c].z[j] = (float)b_odd[6 * s + 2 * c];
                in.data[odd.myIdx.idx[i]].c[c].z[NB + j] = (float)b_odd[6 * s + 2 * c + 1];
            }
        }
    DiracHISQ<float, NB, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> d(KUQCD_HISQPC_DIRAC, gf, gl, 0.0);
    d.Dslash(in, out, false);
    std::vector<float> rec(6 * vh);
    for (size_t i = 0; i < even.lenBulk; ++i)
        for (int j = 0; j < NB; ++j) {
            const size_t s = batch_real_cb(even, i, 0, j, lat);
            for (int c = 0; c < 3; ++c) {
                rec[6 * s + 2 * c] = out.data[even.myIdx.idx[i]].c[c].z[j];
                rec[6 * s + 2 * c + 1] = out.data[even.myIdx.idx[i]].c[c].z[NB + j];
            }
        }
    write_all(dir + "/dslash_batch.bin", rec);
}

int main(int argc, char **argv)
{
    if (argc != 7) {
        fprintf(stderr, "usage: %s dir nx ny nz nt num_shift\n", argv[0]);
        return 1;
    }
    const std::string dir = argv[1];
    const unsigned lat[4] = {(unsigned)atoi(argv[2]), (unsigned)atoi(argv[3]), (unsigned)atoi(argv[4]),
                             (unsigned)atoi(argv[5])};
    const int ns = atoi(argv[6]);
    const size_t V = (size_t)lat[0] * lat[1] * lat[2] * lat[3];
    const std::vector<double> fat = read_all(dir + "/fat.bin", V * 72), lng = read_all(dir + "/long.bin", V * 72);
    const std::vector<double> be = read_all(dir + "/b_even.bin", V / 2 * 6), bo = read_all(dir + "/b_odd.bin", V / 2 * 6);
    std::vector<double> shifts = read_all(dir + "/shifts.bin", ns);
    const double tol = read_all(dir + "/tol.bin", 1)[0];

    const std::array<unsigned short, 4> grid{1, 1, 1, 1};
    const Lattice sup(lat[0], lat[1], lat[2], lat[3]);
    // FP64, NORMAL_ORDER: the reference's glue builds exactly these objects (kuqcd.cpp:218-286)
    {
        LattBase all(sup, grid, 3, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_DOUBLE, KUQCD_ALL);
        LattBase even(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_DOUBLE, KUQCD_EVEN);
        LattBase odd(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_DOUBLE, KUQCD_ODD);
        CommBase comm(all);
        GaugeField<double, 1, KUQCD_GAUGE_RECON_NO> gf(all, comm), gl(all, comm);
        set_gauge(gf, fat);
        set_gauge(gl, lng);
        SpinorField<double, 1, 1> src_e(even), src_o(odd), out_e(even), tmp_o(odd);
        set_spinor(src_e, be);
        set_spinor(src_o, bo);
        DiracHISQ<double, 1, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> dirac(KUQCD_HISQPC_DIRAC, gf, gl, 0.0,
                                                                             &tmp_o);
        dirac.Dslash(src_o, out_e, false);
        write_all(dir + "/dslash_even.bin", get_spinor(out_e));
        dirac.MdaggM(src_e, out_e, false);
        write_all(dir + "/mdaggm_even.bin", get_spinor(out_e));

        // BLAS-1 sequence on y = copy of b_even, x = D D b_even (now in out_e)
        SpinorField<double, 1, 1> y(src_e);
        const double n2 = Norm2(y), dot = RealDot(y, out_e), nrm = Norm(out_e);
        Axpy(y, out_e, 0.25);      // y = b + 0.25 x
        Axmy(y, src_e, 2.0);       // y = 2 b - y
        Ymax(y, out_e, -0.5);      // y = y + 0.5 x
        Axpby(y, src_e, 3.0, 0.5); // y = 3 b + 0.5 y
        SpinorField<double, 1, 1> w = y - src_e;      // w = y - b
        SpinorField<double, 1, 1> v = w * 2.0;        // v = 2 w
        v -= src_e;                                    // v = 2 w - b
        SpinorField<double, 1, 1> u = v + out_e;      // u = 2 w - b + x
        write_all(dir + "/axpby.bin", get_spinor(u));
        FILE *f = fopen((dir + "/blas.txt").c_str(), "w");
        fprintf(f, "%.17g %.17g %.17g\n", n2, dot, nrm);
        fclose(f);

        // CGM::Invert on even sites with the reference's shift semantics (kuqcd.cpp:254-273)
        CGM<double, SpinorField<double, 1, 1>> cgm(KUQCD_CGM, &dirac);
        std::vector<SpinorField<double, 1, 1> *> sol;
        for (int k = 0; k < ns; ++k) sol.push_back(new SpinorField<double, 1, 1>(even));
        const int it = cgm.Invert(ns, shifts.data(), src_e, sol.data(), tol, 100000);
        for (int k = 0; k < ns; ++k) {
            write_all(dir + "/x" + std::to_string(k) + ".bin", get_spinor(*sol[k]));
            delete sol[k];
        }
        f = fopen((dir + "/cgm.txt").c_str(), "w");
        fprintf(f, "%d\n", it);
        fclose(f);
    }
    // FP32, NORMAL_ORDER
    {
        LattBase all(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_ALL);
        LattBase even(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_EVEN);
        LattBase odd(sup, grid, 0, KUQCD_NORMAL_ORDER, KUQCD_TZYX_ORDER, KUQCD_SINGLE, KUQCD_ODD);
        CommBase comm(all);
        GaugeField<float, 1, KUQCD_GAUGE_RECON_NO> gf(all, comm), gl(all, comm);
        set_gauge(gf, fat);
        set_gauge(gl, lng);
        SpinorField<float, 1, 1> in(odd), out(even);
        set_spinor(in, bo);
        DiracHISQ<float, 1, KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_NO> dirac(KUQCD_HISQPC_DIRAC, gf, gl, 0.0);
        dirac.Dslash(in, out);
        write_all(dir + "/dslash_even_f.bin", get_spinor(out));
    }
    if (lat[0] == 32) batch_dslash(dir, lat, fat, lng, bo);
    rootLogger.Info("caller_classes done");
    return 0;
}
