/*
 * Lattice geometry of one field (the reference's latt_base.h:19-50, latt_base.cpp:48-212): the super / sub,
 * flat / checkerboard lattices, the batch width of BATCH_ORDER, and myIdx, the storage index of every bulk site.
 * Callers address LatticeField::data through myIdx, so its construction follows the reference: for a parity field
 * myIdx[i] is the checkerboard index of bulk site i on the halo-padded lattice; for a full (KUQCD_ALL) field the
 * even sites come first, then the odd ones.  With one rank (the only grid kuqcd_b200 runs) there is no halo and
 * myIdx is the identity.
 */
#ifndef LATT_BASE_H
#define LATT_BASE_H

#include <array>

#include "index_utils.h"
#include "kuqcd_memory.h"
#include "space_time.h"

namespace kuqcd {

class LattBase {
public:
    Lattice latSupBulkFL;  // super bulk flat lattice
    Lattice latSupBulkCB;  // super bulk checkerboard lattice
    Lattice latSubFullFL;  // sub full flat lattice
    Lattice latSubFullCB;  // sub full checkerboard lattice
    Lattice latSubBulkFL;  // sub bulk flat lattice
    Lattice latSubBulkCB;  // sub bulk checkerboard lattice
    Lattice *latFull = nullptr;
    Lattice *latBulk = nullptr;
    size_t lenFull = 0;
    size_t lenBulk = 0;
    std::array<unsigned short, 4> gridDim{1, 1, 1, 1};
    unsigned short haloDepth = 0;
    unsigned int Nbatch = 1;
    int myRank = 0;
    int np = 1;
    KuQCDPrecision prec = KUQCD_DOUBLE;
    KuQCDGaugeOrder gauge_order = KUQCD_NORMAL_ORDER;
    KuQCDRankOrder rankOrder = KUQCD_TZYX_ORDER;
    KuQCDSiteSubset site_subset = KUQCD_ALL;
    Index myIdx;

    LattBase() = default;
    LattBase(const LattBase &o) { *this = o; }
    LattBase(const Lattice &lat, const std::array<unsigned short, 4> &gridDim_, unsigned short depth,
             KuQCDGaugeOrder order_, KuQCDRankOrder rankOrder_, KuQCDPrecision prec_,
             KuQCDSiteSubset parity_ = KUQCD_ALL)
        : gridDim(gridDim_), haloDepth(depth), myRank(GetRank()), np(GetNp()), prec(prec_), gauge_order(order_),
          rankOrder(rankOrder_), site_subset(parity_)
    {
        const bool pc = site_subset == KUQCD_EVEN || site_subset == KUQCD_ODD;
        if (gridDim[0] * gridDim[1] * gridDim[2] * gridDim[3] != np)
            Rank0Fprintf(stderr, "%d != %d * %d * %d * %d!\n", np, gridDim[0], gridDim[1], gridDim[2], gridDim[3]);
        if (gauge_order == KUQCD_BATCH_ORDER) {
            // SIMD lanes along x: 16 floats or 8 doubles per complex word (latt_base.cpp:77-93)
            Nbatch = prec == KUQCD_SINGLE ? 16 : 8;
            if (gridDim[0] > 1)
                Rank0Fprintf(stderr, "if using batch gauge_order the x direction should not communicate!\n");
            if (lat[0] % Nbatch != 0)
                Rank0Fprintf(stderr, "x direction lattice %d cannot divided by %u!\n", lat[0], Nbatch);
        } else {
            Nbatch = 1;
        }
        unsigned short n[4], nFull[4];
        for (int d = 0; d < 4; ++d) {
            if (lat[d] % gridDim[d] != 0)
                Rank0Fprintf(stderr, "dir %d lattice %d cannot be splitted into %d part!\n", d, lat[d], gridDim[d]);
            n[d] = (unsigned short)(lat[d] / gridDim[d] / (d == 0 ? Nbatch : 1));
            nFull[d] = (unsigned short)(gridDim[d] > 1 ? n[d] + 2 * depth : n[d]);
        }
        if (pc && (n[0] & 1)) Rank0Fprintf(stderr, "x direction lattice %d should be even!\n", n[0]);
        latSupBulkFL = Lattice((unsigned short)(lat.nx / Nbatch), lat.ny, lat.nz, lat.nt);
        latSupBulkCB = Lattice((unsigned short)(lat.nx / Nbatch / 2), lat.ny, lat.nz, lat.nt);
        latSubFullFL = Lattice(nFull[0], nFull[1], nFull[2], nFull[3]);
        latSubFullCB = Lattice((unsigned short)(nFull[0] / 2), nFull[1], nFull[2], nFull[3]);
        latSubBulkFL = Lattice(n[0], n[1], n[2], n[3]);
        latSubBulkCB = Lattice((unsigned short)(n[0] / 2), n[1], n[2], n[3]);
        SetPointers();
        InitIdx();
    }

    LattBase &operator=(const LattBase &o)
    {
        if (this == &o) return *this;
        latSupBulkFL = o.latSupBulkFL;
        latSupBulkCB = o.latSupBulkCB;
        latSubFullFL = o.latSubFullFL;
        latSubFullCB = o.latSubFullCB;
        latSubBulkFL = o.latSubBulkFL;
        latSubBulkCB = o.latSubBulkCB;
        gridDim = o.gridDim;
        haloDepth = o.haloDepth;
        Nbatch = o.Nbatch;
        myRank = o.myRank;
        np = o.np;
        prec = o.prec;
        gauge_order = o.gauge_order;
        rankOrder = o.rankOrder;
        site_subset = o.site_subset;
        myIdx = o.myIdx;
        SetPointers();
        return *this;
    }

    void InitIdx()
    {
        myIdx.Init(lenBulk);
        const size_t vcb = latSubBulkCB.V;
        for (size_t i = 0; i < vcb; ++i) {
            const Position cb = GetPosition((unsigned)i, latSubBulkCB);
            if (site_subset == KUQCD_ALL) {
                for (int par = 0; par < 2; ++par) {
                    const Position full =
                        GetFullPosFromBulkPos(GetPosFromCBPos(cb, (KuQCDSiteSubset)par), haloDepth, gridDim);
                    myIdx.idx[i + par * vcb] = (long)(full.Index(latSubFullFL) / 2 + par * (latSubFullFL.V / 2));
                }
            } else {
                myIdx.idx[i] = (long)GetFullPosFromBulkPos(cb, haloDepth, gridDim).Index(latSubFullCB);
            }
        }
    }

    /* the real (unbatched) global extents */
    Lattice RealLattice() const
    {
        return Lattice((unsigned short)(latSupBulkFL.nx * Nbatch), latSupBulkFL.ny, latSupBulkFL.nz, latSupBulkFL.nt);
    }

private:
    void SetPointers()
    {
        const bool pc = site_subset == KUQCD_EVEN || site_subset == KUQCD_ODD;
        latFull = pc ? &latSubFullCB : &latSubFullFL;
        latBulk = pc ? &latSubBulkCB : &latSubBulkFL;
        lenFull = latFull->V;
        lenBulk = latBulk->V;
    }
};

}  // namespace kuqcd

#endif
