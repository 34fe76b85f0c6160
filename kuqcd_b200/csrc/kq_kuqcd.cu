// The reference's five exported calls (kuqcd.h:29-34, kuqcd.cpp:288-487) on top of the device API:
// same validation order and status codes, same precision dispatch (P6: the loaded link pair decides; batch-float,
// batch-double, float, double in that order, kuqcd.cpp:415-435), same host layouts and ownership (links copied at
// load, b read and num_shift solutions written at solve, param->iter set).
//
// Deliberate differences, each one turning undefined behaviour of the reference into an error:
//   * x extent odd, or a gauge field loaded with site_subset != KUQCD_ALL  -> KUQCD_ERR_INVALID_PARAM
//     (the reference prints a warning and later reads out of bounds)
//   * a second load with other lattice extents into the same precision slot -> KUQCD_ERR_INVALID_PARAM
//   * non-finite p.Ap or |r|^2 (breakdown) -> KUQCD_ERR_UNKNOWN_ERROR (the reference returns NaN solutions)
//   * the process grid is 1x1x1x1 (one GPU per process); kuqcd_init reads the grid from stdin only when
//     KUQCD_GRID_STDIN=1 (command_line.cpp:31-84 always reads stdin), else from KUQCD_GRID ("1,1,1,1").
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "kq_internal.h"
#include "kq_solver.h"
#define KUQCD_NO_CLASS_API  // the five calls only; the class-level API is header-only for callers
#include "kuqcd.h"

#define KQ_API extern "C" __attribute__((visibility("default")))

namespace {

std::mutex g_mu;
int g_grid[4] = {1, 1, 1, 1};
bool g_grid_set = false;

// precision slots in the reference's dispatch order: batch-float, batch-double, float, double
enum { SLOT_F16 = 0, SLOT_D8 = 1, SLOT_F1 = 2, SLOT_D1 = 3, NSLOT = 4 };
struct Slot {
    kq_context *ctx = nullptr;
    bool fat = false, lng = false;
    unsigned lat[4] = {0, 0, 0, 0};
};
Slot g_slot[NSLOT];
bool g_parity_latbase = false;  // the reference creates the parity lattices on the first gauge load

void log_error(const char *msg)
{
    fprintf(stderr, "[KuQCD ERROR] %s\n", msg);
    kq::set_last_error(msg);
}

int slot_of(KuQCDGaugeOrder order, KuQCDPrecision prec)
{
    if (order == KUQCD_BATCH_ORDER) return prec == KUQCD_SINGLE ? SLOT_F16 : SLOT_D8;
    return prec == KUQCD_SINGLE ? SLOT_F1 : SLOT_D1;
}

int nbatch_of(int slot) { return slot == SLOT_F16 ? 16 : slot == SLOT_D8 ? 8 : 1; }

// BATCH_ORDER host record -> NORMAL_ORDER record (kuqcd.cpp:103-127 with Nbatch lanes; latt_base.cpp:77-93):
// the batch lattice has nx/Nbatch reduced x sites, lane j of reduced site xr is the real site x = xr + (nx/Nbatch)*j,
// and the record entry of (lane j, reduced even-odd site i) is at ni = j + Nbatch*i.
template <typename T>
void batch_to_normal_gauge(const unsigned lat[4], int nb, const T *in, T *out)
{
    const long nx = lat[0], ny = lat[1], nz = lat[2], nt = lat[3];
    const long nxr = nx / nb, hxr = nxr / 2, hx = nx / 2;
    const long vhr = nxr * ny * nz * nt / 2, vh = nx * ny * nz * nt / 2;
    for (int par = 0; par < 2; ++par)
        for (long i = 0; i < vhr; ++i) {
            long r = i / hxr;
            const long xcb = i - r * hxr;
            const long y = r % ny;
            r /= ny;
            const long z = r % nz, t = r / nz;
            const long xr = 2 * xcb + ((y + z + t + par) & 1);
            const long ir = i + par * vhr;
            for (int j = 0; j < nb; ++j) {
                const long x = xr + nxr * j;
                const int rpar = (int)((x + y + z + t) & 1);
                const long icb = (x >> 1) + hx * (y + ny * (z + nz * t));
                const long s = icb + (rpar ? vh : 0);
                const long ni = j + (long)nb * ir;
                memcpy(out + 72 * s, in + 72 * ni, 72 * sizeof(T));
            }
        }
}

}  // namespace

KQ_API KuQCDStatus kq_kuqcd_init(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    int grid[4] = {1, 1, 1, 1};
    const char *rd = getenv("KUQCD_GRID_STDIN");
    if (rd && rd[0] == '1') {
        // same key=value format as command_line.cpp:31-84
        std::map<std::string, int *> vars = {{"gridx", &grid[0]}, {"gridy", &grid[1]}, {"gridz", &grid[2]},
                                             {"gridt", &grid[3]}};
        std::string line;
        while (std::getline(std::cin, line)) {
            const size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            auto trim = [](std::string s) {
                const size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
                return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
            };
            auto it = vars.find(trim(line.substr(0, eq)));
            if (it == vars.end()) continue;
            try {
                *it->second = std::stoi(trim(line.substr(eq + 1)));
            } catch (...) {
            }
        }
    } else if (const char *gs = getenv("KUQCD_GRID")) {
        sscanf(gs, "%d,%d,%d,%d", &grid[0], &grid[1], &grid[2], &grid[3]);
    }
    memcpy(g_grid, grid, sizeof(grid));
    g_grid_set = true;
    // one process drives one GPU: np == 1 (kuqcd.cpp:294-298 compares the grid with np)
    if (grid[0] * grid[1] * grid[2] * grid[3] != 1) {
        log_error("g_grid_dim is not equal np");
        return KUQCD_ERR_INVALID_PARAM;
    }
    return KUQCD_SUCCESS;
}

KQ_API KuQCDStatus kq_kuqcd_load_gaugefield(void *h_gauge, KuQCDGaugeParam *param)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (h_gauge == nullptr || param == nullptr) {
        log_error("h_gauge or param is nullptr");
        return KUQCD_ERR_NULL_POINTER;
    }
    if (param->gauge_order != KUQCD_BATCH_ORDER && param->gauge_order != KUQCD_NORMAL_ORDER) {
        log_error("gauge_order is invalid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->link_type != KUQCD_FAT_LINK && param->link_type != KUQCD_LONG_LINK) {
        log_error("link_type is invalid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->recon != KUQCD_GAUGE_RECON_NO) {
        if (param->recon == KUQCD_GAUGE_RECON_U14 || param->recon == KUQCD_GAUGE_RECON_12 ||
            param->recon == KUQCD_GAUGE_RECON_8) {
            log_error("recon is not support");
            return KUQCD_ERR_UNSUPPORTED;
        }
        log_error("recon is invalid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->lat[0] == 0 || param->lat[1] == 0 || param->lat[2] == 0 || param->lat[3] == 0) {
        log_error("param->lat is 0");
        return KUQCD_ERR_INVALID_PARAM;
    }
    // set_latbase checks (kuqcd.cpp:41-57)
    if (param->prec != KUQCD_SINGLE && param->prec != KUQCD_DOUBLE) {
        if (param->prec == KUQCD_HALF) {
            log_error("prec is not support");
            return KUQCD_ERR_UNSUPPORTED;
        }
        log_error("prec is not valid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->site_subset < KUQCD_EVEN || param->site_subset >= KUQCD_INVALID_PARITY) {
        log_error("site_subset is not valid");
        return KUQCD_ERR_INVALID_PARAM;
    }
    if (param->site_subset != KUQCD_ALL) {
        log_error("gauge fields must cover all sites (site_subset KUQCD_ALL)");
        return KUQCD_ERR_INVALID_PARAM;
    }
    const int slot = slot_of(param->gauge_order, param->prec);
    const int nb = nbatch_of(slot);
    // NORMAL_ORDER: x even (latt_base.cpp:114-116).  BATCH_ORDER: the reference's lane shuffles
    // (dirac_hisq.cpp:504-663) assume two reduced x sites, i.e. nx == 2*Nbatch.
    if (nb == 1 ? (param->lat[0] % 2u) != 0 : param->lat[0] != 2u * nb) {
        log_error(nb > 1 ? "batch order needs nx == 2*Nbatch" : "x direction lattice should be even");
        return KUQCD_ERR_INVALID_PARAM;
    }
    Slot &S = g_slot[slot];
    if (S.ctx && memcmp(S.lat, param->lat, sizeof(S.lat)) != 0) {
        log_error("lattice extents differ from the links already loaded in this precision");
        return KUQCD_ERR_INVALID_PARAM;
    }
    try {
        if (!S.ctx) {
            KuQCDStatus st = kq_context_create(param->lat, 0, &S.ctx);
            if (st != KUQCD_SUCCESS) {
                log_error(kq_last_error());
                return st;
            }
            memcpy(S.lat, param->lat, sizeof(S.lat));
        }
        const size_t V = (size_t)param->lat[0] * param->lat[1] * param->lat[2] * param->lat[3];
        const void *rec = h_gauge;
        std::vector<char> reordered;
        if (nb > 1) {
            const size_t esz = param->prec == KUQCD_DOUBLE ? 8 : 4;
            reordered.resize(V * 72 * esz);
            if (esz == 8)
                batch_to_normal_gauge<double>(param->lat, nb, static_cast<const double *>(h_gauge),
                                              reinterpret_cast<double *>(reordered.data()));
            else
                batch_to_normal_gauge<float>(param->lat, nb, static_cast<const float *>(h_gauge),
                                             reinterpret_cast<float *>(reordered.data()));
            rec = reordered.data();
        }
        KuQCDStatus st = kq_load_links(S.ctx, param->link_type, rec, param->prec);
        if (st != KUQCD_SUCCESS) {
            log_error(kq_last_error());
            return st;
        }
        if (param->link_type == KUQCD_FAT_LINK) S.fat = true;
        else S.lng = true;
        g_parity_latbase = true;
    } catch (std::bad_alloc &) {
        return KUQCD_ERR_NO_MEMORY;
    } catch (...) {
        return KUQCD_ERR_UNKNOWN_ERROR;
    }
    return KUQCD_SUCCESS;
}

// BATCH_ORDER spinor record <-> NORMAL_ORDER (kuqcd.cpp:129-169 with Nbatch lanes)
template <typename T>
static void spinor_batch_map(const unsigned lat[4], int nb, int par, const T *in, T *out, bool to_normal)
{
    const long nx = lat[0], ny = lat[1], nz = lat[2], nt = lat[3];
    const long nxr = nx / nb, hxr = nxr / 2, hx = nx / 2;
    const long vhr = nxr * ny * nz * nt / 2;
    for (long i = 0; i < vhr; ++i) {
        long r = i / hxr;
        const long xcb = i - r * hxr;
        const long y = r % ny;
        r /= ny;
        const long z = r % nz, t = r / nz;
        const long xr = 2 * xcb + ((y + z + t + par) & 1);
        for (int j = 0; j < nb; ++j) {
            const long x = xr + nxr * j;
            const long icb = (x >> 1) + hx * (y + ny * (z + nz * t));
            const long ni = j + (long)nb * i;
            if (to_normal) memcpy(out + 6 * icb, in + 6 * ni, 6 * sizeof(T));
            else memcpy(out + 6 * ni, in + 6 * icb, 6 * sizeof(T));
        }
    }
}

KQ_API KuQCDStatus kq_kuqcd_solve_multishift(void **hp_x, void *hp_b, KuQCDInvertParam *param)
{
    std::lock_guard<std::mutex> lk(g_mu);
    try {
        if (hp_x == nullptr || hp_b == nullptr || param == nullptr) {
            log_error("hp_x or hp_b or param is nullptr");
            return KUQCD_ERR_NULL_POINTER;
        }
        if (param->matpc_type != KUQCD_EVEN_EVEN && param->matpc_type != KUQCD_ODD_ODD) {
            log_error("matpc_type is error!");
            return KUQCD_ERR_INVALID_PARAM;
        }
        int slot = -1;
        for (int s = 0; s < NSLOT; ++s)
            if (g_slot[s].ctx && g_slot[s].fat && g_slot[s].lng) {
                slot = s;
                break;
            }
        if (slot < 0) {
            log_error("no init gauge_smeared and gauge_naik");
            return KUQCD_ERR_UNKNOWN_TYPE;
        }
        // kuqcd_inverter validation (kuqcd.cpp:176-199)
        if (param->inverter_type != KUQCD_CGM) {
            log_error("Inverter is not support");
            return KUQCD_ERR_UNSUPPORTED;
        }
        if (param->dslash_type == KUQCD_WILSON_DIRAC || param->dslash_type == KUQCD_WILSONPC_DIRAC) {
            log_error("dirac type should be hisq or hisq pc!");
            return KUQCD_ERR_UNSUPPORTED;
        }
        if (param->dslash_type != KUQCD_HISQ_DIRAC && param->dslash_type != KUQCD_HISQPC_DIRAC) {
            log_error("dirac type is error!");
            return KUQCD_ERR_INVALID_PARAM;
        }
        if (param->num_shift <= 0) {
            log_error("num_shift < 0!");
            return KUQCD_ERR_INVALID_PARAM;
        }
        if (param->num_shift > kq::kMaxShift) {
            log_error("num_shift > 64 is not supported");
            return KUQCD_ERR_UNSUPPORTED;
        }
        if (param->shifts == nullptr) {
            log_error("shifts is nullptr");
            return KUQCD_ERR_NULL_POINTER;
        }
        for (int k = 0; k < param->num_shift; ++k)
            if (hp_x[k] == nullptr) {
                log_error("hp_x[k] is nullptr");
                return KUQCD_ERR_NULL_POINTER;
            }
        Slot &S = g_slot[slot];
        const bool dbl = slot == SLOT_D8 || slot == SLOT_D1;
        const int nb = nbatch_of(slot);
        const int parity = param->matpc_type == KUQCD_EVEN_EVEN ? 0 : 1;
        kq_solve_param sp;
        memset(&sp, 0, sizeof(sp));
        sp.parity = parity;
        sp.num_shift = param->num_shift;
        sp.shifts = param->shifts;
        sp.shift_mode = 0;
        sp.solver = KQ_SOLVER_CGM;
        sp.prec = dbl ? KUQCD_DOUBLE : KUQCD_SINGLE;
        sp.host_prec = dbl ? KUQCD_DOUBLE : KUQCD_SINGLE;
        sp.max_iter = param->max_iter;
        sp.tol = param->tol;
        // optional sloppy solver for FP64 links: KUQCD_SOLVER=mixed, target |r_k| < sqrt(tol) (the reference's
        // stopping rule zeta_k^2 |r|^2 < tol bounds the squared residual norm of shift k)
        const char *solver = getenv("KUQCD_SOLVER");
        const bool mixed_half = dbl && solver && strcmp(solver, "mixed-half") == 0;
        const bool mixed = mixed_half || (dbl && solver && strcmp(solver, "mixed") == 0);
        const size_t vh = (size_t)S.lat[0] * S.lat[1] * S.lat[2] * S.lat[3] / 2;
        const size_t esz = dbl ? 8 : 4;
        const void *b = hp_b;
        std::vector<char> bre;
        std::vector<std::vector<char>> xre;
        std::vector<void *> xs(param->num_shift);
        if (nb > 1) {
            bre.resize(vh * 6 * esz);
            if (dbl) spinor_batch_map<double>(S.lat, nb, parity, (const double *)hp_b, (double *)bre.data(), true);
            else spinor_batch_map<float>(S.lat, nb, parity, (const float *)hp_b, (float *)bre.data(), true);
            b = bre.data();
            xre.resize(param->num_shift);
            for (int k = 0; k < param->num_shift; ++k) {
                xre[k].resize(vh * 6 * esz);
                xs[k] = xre[k].data();
            }
        } else {
            for (int k = 0; k < param->num_shift; ++k) xs[k] = hp_x[k];
        }
        if (mixed) {
            sp.solver = KQ_SOLVER_MIXED;
            sp.prec = mixed_half ? KUQCD_HALF : KUQCD_SINGLE;
            sp.rel_residual = -1.0;  // absolute: |b - A_k x_k|^2 < tol, |b| taken on the device
        }
        kq_solve_info info;
        KuQCDStatus st = kq_solve_multishift(S.ctx, &sp, b, xs.data(), &info);
        param->iter = info.iter;
        if (st == KUQCD_SUCCESS) {
            if (info.status == kq::KQ_STATUS_MAXITER) printf("CGM: Warning max iteration reached %d\n", info.iter);
            else printf("CGM: # iterations %d\n", info.iter);
        } else {
            log_error(kq_last_error());
        }
        if (nb > 1)
            for (int k = 0; k < param->num_shift; ++k) {
                if (dbl) spinor_batch_map<double>(S.lat, nb, parity, (const double *)xs[k], (double *)hp_x[k], false);
                else spinor_batch_map<float>(S.lat, nb, parity, (const float *)xs[k], (float *)hp_x[k], false);
            }
        return st;
    } catch (std::bad_alloc &) {
        return KUQCD_ERR_NO_MEMORY;
    } catch (...) {
        return KUQCD_ERR_UNKNOWN_ERROR;
    }
}

KQ_API void kq_kuqcd_gauge_free(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    for (int s = 0; s < NSLOT; ++s) {
        if (g_slot[s].ctx) kq_context_destroy(g_slot[s].ctx);
        g_slot[s] = Slot();
    }
    g_parity_latbase = false;
}

KQ_API void kq_kuqcd_end(void)
{
    // solver workspaces belong to the contexts released by kq_kuqcd_gauge_free; nothing else is held
    std::lock_guard<std::mutex> lk(g_mu);
}

// ------------------------------------------------------------------------------------------------ C++ API
namespace kuqcd {
KuQCDStatus kuqcd_init() { return kq_kuqcd_init(); }
KuQCDStatus kuqcd_load_gaugefield(void *h_gauge, KuQCDGaugeParam *param)
{
    return kq_kuqcd_load_gaugefield(h_gauge, param);
}
KuQCDStatus kuqcd_solve_multishift(void **_hp_x, void *_hp_b, KuQCDInvertParam *param)
{
    return kq_kuqcd_solve_multishift(_hp_x, _hp_b, param);
}
void kuqcd_gauge_free() { kq_kuqcd_gauge_free(); }
void kuqcd_end() { kq_kuqcd_end(); }
}  // namespace kuqcd
