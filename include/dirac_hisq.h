/*
 * The HISQ staggered operator of the class-level API (the reference's dirac_hisq.h:24-77, dirac_hisq.cpp:30-462),
 * computed on the GPU.
 *
 *   Dslash(src, dst): dst = D src, with D the even-odd dslash of 1-hop fat and 3-hop Naik links (staggered phases
 *                     folded into the links): parity fields give the preconditioned operator (dst on the other
 *                     parity), KUQCD_ALL fields the full-lattice one (KUQCD_HISQ_DIRAC).
 *   MdaggM(src, dst): dst = D D src (dirac_hisq.cpp:457-462; -D^dag D, since D_qp = -D_pq^dag).
 *
 * Construction copies both link fields to the GPU (a kq_context of libkuqcd_b200 holds them; the Naik factor
 * c3000 = -(1 + naikEps)/48 and the 1/2 of the 1-hop term are folded in there, dirac_hisq.cpp:40, 464-502).  Each
 * call copies its spinor fields to the GPU and the result back, so `data` of every field always holds its current
 * values; a caller after throughput keeps its fields on the GPU with the device API (kq_dslash, kq_mdagm,
 * kq_solve_multishift_device) instead.  The mass is stored and, as in the reference, not applied (P3 of the
 * reference's semantics: callers fold m^2 into the shifts).  Only full link storage (KUQCD_GAUGE_RECON_NO) runs;
 * the reference's reconstruction is a stub (su3.cpp:250-254), and other recon values throw.
 */
#ifndef DIRAC_HISQ_H
#define DIRAC_HISQ_H

#include <array>
#include <stdexcept>
#include <vector>

#include "communication.h"
#include "dirac.h"
#include "gauge_field.h"
#include "spinor_field.h"

namespace kuqcd {

namespace detail {
/* what an inverter needs of an operator to solve on the GPU */
class DeviceOperator {
public:
    virtual ~DeviceOperator() = default;
    virtual kq_context *DeviceContext() const = 0;
};
}  // namespace detail

template <typename T, int Nbatch, KuQCDReconstructType ReconS, KuQCDReconstructType ReconN>
class DiracHISQ : public Dirac<SpinorField<T, Nbatch, 1>>, public detail::DeviceOperator {
public:
    typedef ColorSpinor<T, Nbatch> SpinorT;
    typedef SpinorField<T, Nbatch, 1> VecT;
    typedef SU3<T, Nbatch, ReconS> GaugeST;
    typedef SU3<T, Nbatch, ReconN> GaugeNT;
    typedef GaugeField<T, Nbatch, ReconS> LinkST;
    typedef GaugeField<T, Nbatch, ReconN> LinkNT;

    const LinkST &gaugeSmeared;
    const LinkNT &gaugeNaik;
    VecT *tmp = nullptr;
    LattBase &latBase;
    double mass = 0;
    T mass2 = 0, c3000 = -1.0 / 48.0;
    int myRank = 0;
    int np = 1;
    std::array<unsigned short, 4> &gridDim;

    DiracHISQ(KuQCDDslashType diracType, const LinkST &gaugeSmeared_, const LinkNT &gaugeNaik_, const double mass_,
              VecT *tmp_ = nullptr, T naikEps = 0)
        : Dirac<VecT>(diracType),
          gaugeSmeared(gaugeSmeared_),
          gaugeNaik(gaugeNaik_),
          tmp(tmp_),
          latBase(gaugeSmeared_.latBase),
          mass(mass_),
          mass2((T)(mass_ * mass_)),
          c3000((T)(-(1.0 + naikEps) / 48.0)),
          myRank(GetRank()),
          np(GetNp()),
          gridDim(gaugeSmeared_.latBase.gridDim),
          naik_scale_(1.0 + (double)naikEps)
    {
        if (diracType != KUQCD_HISQ_DIRAC && diracType != KUQCD_HISQPC_DIRAC)
            throw std::invalid_argument("DiracHISQ: dirac type should be hisq or hisq pc");
        if (ReconS != KUQCD_GAUGE_RECON_NO || ReconN != KUQCD_GAUGE_RECON_NO)
            throw std::invalid_argument("DiracHISQ: only KUQCD_GAUGE_RECON_NO link storage is supported");
        for (int d = 0; d < 4; ++d)
            if (gridDim[d] != 1) throw std::invalid_argument("DiracHISQ: one rank per GPU (grid 1x1x1x1)");
        const Lattice lat = latBase.RealLattice();
        const unsigned dims[4] = {lat.nx, lat.ny, lat.nz, lat.nt};
        detail::check(kq_context_create(dims, DefaultDevice(), &ctx_), "DiracHISQ: kq_context_create");
        try {
            UpdateLinks();
        } catch (...) {
            kq_context_destroy(ctx_);
            ctx_ = nullptr;
            throw;
        }
    }
    DiracHISQ(const DiracHISQ &) = delete;
    DiracHISQ &operator=(const DiracHISQ &) = delete;
    ~DiracHISQ() override
    {
        if (ctx_) kq_context_destroy(ctx_);
    }

    /* copies the current values of both link fields to the GPU (done by the constructor) */
    void UpdateLinks()
    {
        if constexpr (ReconS == KUQCD_GAUGE_RECON_NO && ReconN == KUQCD_GAUGE_RECON_NO) {
            std::vector<T> fbuf, lbuf;
            const T *fat = gaugeSmeared.Record(fbuf);
            const T *lng = gaugeNaik.Record(lbuf);
            if (naik_scale_ != 1.0) {
                // c3000 = -(1 + naikEps)/48: scale a copy of the long links on the GPU by (1 + naikEps)
                if (lng != lbuf.data()) lbuf.assign(lng, lng + latBase.RealLattice().V * 72);
                detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), lbuf.size(), naik_scale_ - 1.0,
                                           lbuf.data(), 1.0, lbuf.data()),
                              "DiracHISQ: naikEps");
                lng = lbuf.data();
            }
            detail::check(kq_load_links(ctx_, KUQCD_FAT_LINK, fat, detail::prec_of<T>()), "DiracHISQ: fat links");
            detail::check(kq_load_links(ctx_, KUQCD_LONG_LINK, lng, detail::prec_of<T>()), "DiracHISQ: long links");
        }
    }

    void Dslash(const VecT &src, VecT &dst, bool update = false) override
    {
        (void)update;  // halo update flag of the multi-rank path: one rank has no halo
        const int ps = detail::field_parity(src.latBase), pd = detail::field_parity(dst.latBase);
        if ((ps == 2) != (pd == 2) || (ps != 2 && ps == pd))
            throw std::invalid_argument("DiracHISQ::Dslash: dst must be the other parity of src (or both full)");
        Apply(KQ_OP_DSLASH, src, dst, pd);
    }

    void MdaggM(const VecT &src, VecT &dst, bool update = false) override
    {
        (void)update;
        const int ps = detail::field_parity(src.latBase), pd = detail::field_parity(dst.latBase);
        if (ps != pd) throw std::invalid_argument("DiracHISQ::MdaggM: src and dst must have the same parity");
        Apply(KQ_OP_DD, src, dst, pd);
    }

    kq_context *DeviceContext() const override { return ctx_; }

private:
    void Apply(int op, const VecT &src, VecT &dst, int parity)
    {
        if ((parity == 2) != (this->diracType == KUQCD_HISQ_DIRAC))
            throw std::invalid_argument(
                "DiracHISQ: KUQCD_HISQ_DIRAC acts on KUQCD_ALL fields, KUQCD_HISQPC_DIRAC on parity fields");
        detail::SpinorRecord<T, Nbatch> in(src.latBase, const_cast<SpinorT *>(src.data), 1);
        detail::SpinorRecord<T, Nbatch> out(dst.latBase, dst.data, 1);
        in.load();
        detail::check(kq_apply_host(ctx_, op, detail::prec_of<T>(), 0.0, in.ptr(), out.ptr(),
                                    parity == 2 ? KQ_PARITY_FULL : parity, detail::prec_of<T>()),
                      op == KQ_OP_DSLASH ? "DiracHISQ::Dslash" : "DiracHISQ::MdaggM");
        out.store();
    }

    kq_context *ctx_ = nullptr;
    double naik_scale_ = 1.0;
};

}  // namespace kuqcd

#endif
