/*
 * Site-index helpers of the class-level API (the reference's index_utils.h:19-84, index_utils.cpp:17-122): the
 * position <-> index maps of the four-level lattice (super / sub lattice, flat / checkerboard).  They define the
 * host layouts callers fill (x fastest; checkerboard x = 2*x_cb + ((y + z + t + parity) & 1)), so they follow the
 * reference's conventions exactly.
 */
#ifndef INDEX_UTILS_H
#define INDEX_UTILS_H

#include "space_time.h"

namespace kuqcd {

/* position of flat index i on lat, x fastest */
inline Position GetPosition(const unsigned int i, const Lattice &lat)
{
    unsigned r = i;
    const unsigned x = r % lat.nx;
    r /= lat.nx;
    const unsigned y = r % lat.ny;
    r /= lat.ny;
    const unsigned z = r % lat.nz;
    const unsigned t = r / lat.nz;
    return Position((short)x, (short)y, (short)z, (short)t);
}

/* position of flat index i on lat, t fastest */
inline Position GetAntiPosition(const unsigned int i, const Lattice &lat)
{
    unsigned r = i;
    const unsigned t = r % lat.nt;
    r /= lat.nt;
    const unsigned z = r % lat.nz;
    r /= lat.nz;
    const unsigned y = r % lat.ny;
    const unsigned x = r / lat.ny;
    return Position((short)x, (short)y, (short)z, (short)t);
}

inline unsigned int GetIndex(const Position &pos, const Lattice &lat) { return pos.Index(lat); }

/* super-lattice position of a sub-lattice position on rank myRank (ranks x fastest over gridDim) */
inline Position GetSupPosFromSubPos(const Position &pos, const Lattice &subLat,
                                    const std::array<unsigned short, 4> &gridDim, const int myRank)
{
    int r = myRank;
    Position p;
    for (int d = 0; d < 4; ++d) {
        const int g = r % gridDim[d];
        r /= gridDim[d];
        p[d] = (short)(pos[d] + g * subLat[d]);
    }
    return p;
}

inline Position GetSubPosFromSupPos(const Position &pos, const Lattice &subLat)
{
    Position p;
    for (int d = 0; d < 4; ++d) p[d] = (short)(pos[d] % subLat[d]);
    return p;
}

/* flat position of a checkerboard position of the given parity */
inline Position GetPosFromCBPos(const Position &pos, const KuQCDSiteSubset site_subset)
{
    return Position((short)(2 * pos.x + ((pos.y + pos.z + pos.t + (int)site_subset) & 1)), pos.y, pos.z, pos.t);
}

inline Position GetCBPos(const Position &pos) { return Position((short)(pos.x >> 1), pos.y, pos.z, pos.t); }

/* full (halo-padded) position of a bulk position: directions split over ranks carry haloDepth sites each side */
inline Position GetFullPosFromBulkPos(const Position &pos, int haloDepth, const std::array<unsigned short, 4> &gridDim)
{
    Position p(pos);
    for (int d = 0; d < 4; ++d)
        if (gridDim[d] > 1) p[d] = (short)(p[d] + haloDepth);
    return p;
}

inline unsigned int GetCBIdx(const unsigned int i) { return i >> 1; }

/* flat index of checkerboard index i of the given parity on the checkerboard lattice latCB */
inline unsigned int GetSupIdx(const unsigned int i, const KuQCDSiteSubset site_subset, const Lattice &latCB)
{
    const Position cb = GetPosition(i, latCB);
    const Lattice fl((unsigned short)(2 * latCB.nx), latCB.ny, latCB.nz, latCB.nt);
    return GetPosFromCBPos(cb, site_subset).Index(fl);
}

}  // namespace kuqcd

#endif
