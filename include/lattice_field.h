/*
 * Field storage of the class-level API (the reference's lattice_field.h:19-39, lattice_field.cpp:22-49): a field
 * owns locSize * lenFull reals of its precision in host memory (`data`), addressed through latBase.myIdx.
 *
 * The GPU sees a field as a NORMAL_ORDER host record (kuqcd.cpp:103-169): spinor h[reim + 2*(c + 3*i_cb)] over
 * one parity (a full-lattice spinor: even sites, then odd sites), gauge h[reim + 2*(l + 9*(dir + 4*s))].  With
 * Nbatch = 1, one rank and full link storage, `data` already is that record and is handed to the GPU as it is; a
 * BATCH_ORDER field (Nbatch SIMD lanes along x, latt_base.cpp:77-93) is re-indexed into a record first -- lane j of
 * reduced site x_r is the real site x_r + (nx / Nbatch) j.
 */
#ifndef LATTICE_FIELD_H
#define LATTICE_FIELD_H

#include <stdexcept>
#include <string>
#include <vector>

#include "kuqcd_memory.h"
#include "latt_base.h"
#include "space_time.h"
#include "spinor.h"
#include "su3.h"

namespace kuqcd {

template <typename FieldT>
class LatticeField : public KMemory {
public:
    LattBase &latBase;
    FieldT *data = nullptr;
    int locSize;
    size_t length;

    LatticeField() = delete;
    LatticeField(const LatticeField &lf) : KMemory(lf), latBase(lf.latBase), locSize(lf.locSize), length(lf.length)
    {
        data = static_cast<FieldT *>(this->rawPtr);
    }
    LatticeField(LattBase &latBase_, const int locSize_)
        : KMemory((size_t)locSize_ * latBase_.lenFull * (size_t)latBase_.prec),
          latBase(latBase_),
          locSize(locSize_),
          length(latBase_.lenFull)
    {
        data = static_cast<FieldT *>(this->rawPtr);
        this->Clear();
    }
    LatticeField &operator=(const LatticeField &lf)
    {
        if (locSize != lf.locSize || length != lf.length || this->size != lf.size)
            Rank0Fprintf(stderr, "lattice field length does not match!\n");
        Copy(lf);
        return *this;
    }
    virtual ~LatticeField() { data = nullptr; }
};

namespace detail {

inline KuQCDStatus check(KuQCDStatus st, const char *where)
{
    if (st != KUQCD_SUCCESS) {
        const char *msg = kq_last_error();
        throw std::runtime_error(std::string(where) + ": status " + std::to_string((int)st) +
                                 (msg && *msg ? std::string(" (") + msg + ")" : std::string()));
    }
    return st;
}

template <typename T>
constexpr int prec_of() { return sizeof(T) == 8 ? KUQCD_DOUBLE : KUQCD_SINGLE; }

/* one rank, no halo: every bulk site is stored at its own index */
inline bool identity_layout(const LattBase &lb)
{
    for (int d = 0; d < 4; ++d)
        if (lb.gridDim[d] != 1) return false;
    return lb.lenFull == lb.lenBulk;
}

/* real checkerboard index (within its parity) of lane j of reduced checkerboard site ir of parity par */
inline size_t lane_site(const LattBase &lb, size_t ir, int par, int j)
{
    const Lattice &red = lb.latSupBulkCB;  // reduced checkerboard lattice (nx / Nbatch / 2 wide)
    const Position cb = GetPosition((unsigned)ir, red);
    const long nxr = 2 * (long)red.nx;
    const long xr = 2 * (long)cb.x + ((cb.y + cb.z + cb.t + par) & 1);
    const long x = xr + nxr * j;
    const long hx = nxr * (long)lb.Nbatch / 2;
    return (size_t)((x >> 1) + hx * (cb.y + (long)red.ny * (cb.z + (long)red.nz * cb.t)));
}

/* parity of the spinor field's sites: 0, 1, or 2 for a full-lattice field */
inline int field_parity(const LattBase &lb) { return lb.site_subset == KUQCD_ALL ? 2 : (int)lb.site_subset; }

/* A spinor field as a NORMAL_ORDER record: the field's own memory when it already has that layout, else a copy
 * (load()) that store() writes back. */
template <typename T, int Nbatch>
class SpinorRecord {
public:
    SpinorRecord(const LattBase &lb, ColorSpinor<T, Nbatch> *data, int Ns) : lb_(lb), data_(data), ns_(Ns)
    {
        if (Ns != 1) throw std::invalid_argument("the HISQ operator acts on one-component (Ns = 1) spinor fields");
        direct_ = Nbatch == 1 && identity_layout(lb);
        const size_t vh = lb.RealLattice().V / 2;
        reals_ = (field_parity(lb) == 2 ? 2 * vh : vh) * 6;
        if (!direct_) buf_.assign(reals_, T(0));
    }
    T *ptr() { return direct_ ? reinterpret_cast<T *>(data_) : buf_.data(); }
    void load()
    {
        if (direct_) return;
        visit([&](size_t f, int j, size_t rec) {
            for (int c = 0; c < 3; ++c) {
                buf_[rec + 2 * c] = data_[f].c[c].z[j];
                buf_[rec + 2 * c + 1] = data_[f].c[c].z[Nbatch + j];
            }
        });
    }
    void store()
    {
        if (direct_) return;
        visit([&](size_t f, int j, size_t rec) {
            for (int c = 0; c < 3; ++c) {
                data_[f].c[c].z[j] = buf_[rec + 2 * c];
                data_[f].c[c].z[Nbatch + j] = buf_[rec + 2 * c + 1];
            }
        });
    }

private:
    // fn(storage index, lane, record offset) over every bulk site and lane
    template <typename F>
    void visit(F fn)
    {
        const int par = field_parity(lb_);
        const size_t vhr = lb_.latSupBulkCB.V, vh = lb_.RealLattice().V / 2;
        for (size_t i = 0; i < lb_.lenBulk; ++i) {
            const size_t f = (size_t)lb_.myIdx.idx[i];
            const int p = par == 2 ? (i < vhr ? 0 : 1) : par;
            const size_t ir = par == 2 && i >= vhr ? i - vhr : i;
            for (int j = 0; j < Nbatch; ++j) {
                const size_t s = lane_site(lb_, ir, p, j) + (par == 2 && p == 1 ? vh : 0);
                fn(f, j, 6 * s);
            }
        }
    }
    const LattBase &lb_;
    ColorSpinor<T, Nbatch> *data_;
    int ns_;
    bool direct_ = false;
    size_t reals_ = 0;
    std::vector<T> buf_;
};

}  // namespace detail

}  // namespace kuqcd

#endif
