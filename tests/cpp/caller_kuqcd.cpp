// A KuQCD application as the reference's users write one (test/test_solver.cpp, docs call order): the five
// kuqcd:: calls of include/kuqcd.h, C++ linkage, on host arrays in the NORMAL_ORDER layouts.
//
//   caller_kuqcd <dir> nx ny nz nt num_shift prec(4|8) matpc(0|1)
//
// reads <dir>/fat.bin, <dir>/long.bin (V*72 reals of prec), <dir>/b.bin (V/2*6 reals), <dir>/shifts.bin
// (num_shift doubles, the reference's shift semantics) and <dir>/tol.bin (one double); writes <dir>/x<k>.bin and
// <dir>/result.txt ("status iterations").  Test infrastructure: the GPU tests compare its output with the oracle.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "kuqcd.h"

template <typename T>
static std::vector<T> read_all(const std::string &path, size_t n)
{
    std::vector<T> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(2);
    }
    fclose(f);
    return v;
}

template <typename T>
static int run(const std::string &dir, const unsigned lat[4], int ns, int matpc)
{
    const size_t V = (size_t)lat[0] * lat[1] * lat[2] * lat[3];
    std::vector<T> fat = read_all<T>(dir + "/fat.bin", V * 72), lng = read_all<T>(dir + "/long.bin", V * 72);
    std::vector<T> b = read_all<T>(dir + "/b.bin", V / 2 * 6);
    std::vector<double> shifts = read_all<double>(dir + "/shifts.bin", ns);
    const double tol = read_all<double>(dir + "/tol.bin", 1)[0];

    if (kuqcd::kuqcd_init() != KUQCD_SUCCESS) return 3;
    KuQCDGaugeParam gp;
    for (int d = 0; d < 4; ++d) gp.lat[d] = lat[d];
    gp.halo_depth = 3;
    gp.od = KUQCD_TZYX_ORDER;
    gp.site_subset = KUQCD_ALL;
    gp.gauge_order = KUQCD_NORMAL_ORDER;
    gp.prec = sizeof(T) == 8 ? KUQCD_DOUBLE : KUQCD_SINGLE;
    gp.recon = KUQCD_GAUGE_RECON_NO;
    gp.link_type = KUQCD_FAT_LINK;
    KuQCDStatus st = kuqcd::kuqcd_load_gaugefield(fat.data(), &gp);
    gp.link_type = KUQCD_LONG_LINK;
    if (st == KUQCD_SUCCESS) st = kuqcd::kuqcd_load_gaugefield(lng.data(), &gp);
    if (st != KUQCD_SUCCESS) return 4;

    KuQCDInvertParam ip;
    ip.dslash_type = KUQCD_HISQPC_DIRAC;
    ip.inverter_type = KUQCD_CGM;
    ip.matpc_type = matpc ? KUQCD_ODD_ODD : KUQCD_EVEN_EVEN;
    ip.prec = gp.prec;
    ip.num_shift = ns;
    ip.max_iter = 100000;
    ip.iter = 0;
    ip.tol = tol;
    ip.shifts = shifts.data();
    std::vector<std::vector<T>> x(ns, std::vector<T>(V / 2 * 6));
    std::vector<void *> xp(ns);
    for (int k = 0; k < ns; ++k) xp[k] = x[k].data();
    st = kuqcd::kuqcd_solve_multishift(xp.data(), b.data(), &ip);
    for (int k = 0; k < ns; ++k) {
        FILE *f = fopen((dir + "/x" + std::to_string(k) + ".bin").c_str(), "wb");
        fwrite(x[k].data(), sizeof(T), x[k].size(), f);
        fclose(f);
    }
    FILE *f = fopen((dir + "/result.txt").c_str(), "w");
    fprintf(f, "%d %d\n", (int)st, ip.iter);
    fclose(f);
    kuqcd::kuqcd_gauge_free();
    kuqcd::kuqcd_end();
    return st == KUQCD_SUCCESS ? 0 : 5;
}

int main(int argc, char **argv)
{
    if (argc != 9) {
        fprintf(stderr, "usage: %s dir nx ny nz nt num_shift prec matpc\n", argv[0]);
        return 1;
    }
    const unsigned lat[4] = {(unsigned)atoi(argv[2]), (unsigned)atoi(argv[3]), (unsigned)atoi(argv[4]),
                             (unsigned)atoi(argv[5])};
    const int ns = atoi(argv[6]), prec = atoi(argv[7]), matpc = atoi(argv[8]);
    return prec == 8 ? run<double>(argv[1], lat, ns, matpc) : run<float>(argv[1], lat, ns, matpc);
}
