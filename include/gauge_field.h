/*
 * Link fields of the class-level API (the reference's gauge_field.h:19-45, gauge_field.cpp:22-112): four links per
 * site in host memory, data[dir + 4 * myIdx[i]], built on a KUQCD_ALL lattice.  A DiracHISQ copies the fat and long
 * fields to the GPU when it is constructed (kq_load_links), as kuqcd_load_gaugefield copies the caller's arrays
 * (kuqcd.cpp:346-390); call DiracHISQ::UpdateLinks after changing `data` to copy them again.  With one rank there
 * is no gauge halo: Update() has nothing to exchange.
 */
#ifndef GAUGE_FIELD_H
#define GAUGE_FIELD_H

#include "communication.h"
#include "lattice_field.h"

namespace kuqcd {

template <typename T, int Nbatch, KuQCDReconstructType Recon>
class GaugeField : public LatticeField<SU3<T, Nbatch, Recon>> {
public:
    typedef SU3<T, Nbatch, Recon> GaugeT;

    GaugeT *even;
    GaugeT *odd;  // as the reference sets it: data + latSubFullCB.V (gauge_field.cpp:24)
    CommBase &comm;

    GaugeField() = delete;
    GaugeField(const GaugeField &g) : LatticeField<GaugeT>(g), comm(g.comm) { SetHalves(); }
    GaugeField(LattBase &latBase, CommBase &comm_) : LatticeField<GaugeT>(latBase, 4 * Nbatch * Recon), comm(comm_)
    {
        SetHalves();
    }

    SU3<T, Nbatch, KUQCD_GAUGE_RECON_NO> GetLinkCopy(size_t i, int dir) const
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "only full link storage is supported");
        return this->data[dir + 4 * i];
    }
    SU3<T, Nbatch, KUQCD_GAUGE_RECON_NO> GetLinkDaggCopy(size_t i, int dir) const
    {
        SU3<T, Nbatch, KUQCD_GAUGE_RECON_NO> u = GetLinkCopy(i, dir);
        u.Dagger();
        return u;
    }
    /* gauge halo exchange (gauge_field.cpp:114-245): nothing to exchange on one rank */
    void Update(KuQCDHalo = KUQCD_COMMALL) {}
    void StartComm(KuQCDHalo) {}
    void EndComm(KuQCDHalo) {}

    /* The links as a NORMAL_ORDER FP record h[reim + 2*(l + 9*(dir + 4*s))] over the V real sites (even sites
     * first): `data` itself for Nbatch = 1 on one rank, else a re-indexed copy in `buf`. */
    const T *Record(std::vector<T> &buf) const
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "only full link storage is supported");
        const LattBase &lb = this->latBase;
        if (lb.site_subset != KUQCD_ALL) throw std::invalid_argument("link fields live on a KUQCD_ALL lattice");
        if (Nbatch == 1 && detail::identity_layout(lb)) return reinterpret_cast<const T *>(this->data);
        const size_t vh = lb.RealLattice().V / 2, vhr = lb.latSupBulkCB.V;
        buf.assign(vh * 2 * 72, T(0));
        for (size_t i = 0; i < lb.lenBulk; ++i) {
            const size_t f = (size_t)lb.myIdx.idx[i];
            const int par = i < vhr ? 0 : 1;
            const size_t ir = par ? i - vhr : i;
            for (int j = 0; j < Nbatch; ++j) {
                const size_t s = detail::lane_site(lb, ir, par, j) + (par ? vh : 0);
                for (int dir = 0; dir < 4; ++dir)
                    for (int l = 0; l < 9; ++l) {
                        buf[72 * s + 18 * dir + 2 * l] = this->data[dir + 4 * f].m[l].z[j];
                        buf[72 * s + 18 * dir + 2 * l + 1] = this->data[dir + 4 * f].m[l].z[Nbatch + j];
                    }
            }
        }
        return buf.data();
    }

private:
    void SetHalves()
    {
        even = this->data;
        odd = this->data + this->latBase.latSubFullCB.V;
    }
};

}  // namespace kuqcd

#endif
