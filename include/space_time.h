/*
 * Lattice extents and site positions of the class-level API (the reference's space_time.h:19-80,
 * space_time.cpp): the same members, constructors and index conventions (x fastest, then y, z, t).
 */
#ifndef SPACE_TIME_H
#define SPACE_TIME_H

#include <array>
#include <iostream>

#include "kuqcd_enum.h"
#include "kuqcd_utils.h"

namespace kuqcd {

class Lattice {
public:
    unsigned short nx = 0;
    unsigned short ny = 0;
    unsigned short nz = 0;
    unsigned short nt = 0;
    size_t V = 0;  // nx*ny*nz*nt

    Lattice() = default;
    Lattice(const Lattice &lat) = default;
    Lattice(const unsigned short x, const unsigned short y, const unsigned short z, const unsigned short t)
        : nx(x), ny(y), nz(z), nt(t), V((size_t)x * y * z * t)
    {
    }
    Lattice &operator=(const Lattice &lat) = default;
    unsigned short &operator[](int dir) { return dir == 0 ? nx : dir == 1 ? ny : dir == 2 ? nz : nt; }
    const unsigned short &operator[](int dir) const { return dir == 0 ? nx : dir == 1 ? ny : dir == 2 ? nz : nt; }
    size_t ComputeVolume()
    {
        V = (size_t)nx * ny * nz * nt;
        return V;
    }
    void Print() const { printf("lattice %u %u %u %u (V = %zu)\n", nx, ny, nz, nt, V); }
};

inline std::ostream &operator<<(std::ostream &os, const Lattice &l)
{
    return os << l.nx << " " << l.ny << " " << l.nz << " " << l.nt;
}

class Position {
public:
    short x = 0;
    short y = 0;
    short z = 0;
    short t = 0;

    Position() = default;
    Position(const Position &pos) = default;
    Position(const short x_, const short y_, const short z_, const short t_) : x(x_), y(y_), z(z_), t(t_) {}
    Position &operator=(const Position &pos) = default;
    short &operator[](int dir) { return dir == 0 ? x : dir == 1 ? y : dir == 2 ? z : t; }
    const short &operator[](int dir) const { return dir == 0 ? x : dir == 1 ? y : dir == 2 ? z : t; }
    bool operator==(const Position &p) const { return x == p.x && y == p.y && z == p.z && t == p.t; }
    bool operator!=(const Position &p) const { return !(*this == p); }
    Position operator+(const Position &p) const { return Position(x + p.x, y + p.y, z + p.z, t + p.t); }
    Position operator-(const Position &p) const { return Position(x - p.x, y - p.y, z - p.z, t - p.t); }
    Position &operator+=(const Position &p) { return *this = *this + p; }
    Position &operator-=(const Position &p) { return *this = *this - p; }
    /* periodic wrap of one coordinate into [0, lat[dir]) */
    void Normalize(int dir, const Lattice &lat)
    {
        const int n = lat[dir];
        int v = (*this)[dir] % n;
        if (v < 0) v += n;
        (*this)[dir] = (short)v;
    }
    KuQCDSiteSubset Parity() const { return ((x + y + z + t) & 1) ? KUQCD_ODD : KUQCD_EVEN; }
    /* x fastest */
    unsigned int Index(const Lattice &lat) const
    {
        return (unsigned)x + lat.nx * ((unsigned)y + lat.ny * ((unsigned)z + lat.nz * (unsigned)t));
    }
    /* t fastest */
    unsigned int IndexAnti(const Lattice &lat) const
    {
        return (unsigned)t + lat.nt * ((unsigned)z + lat.nz * ((unsigned)y + lat.ny * (unsigned)x));
    }
    void Print() const { printf("%d %d %d %d\n", x, y, z, t); }
};

inline std::ostream &operator<<(std::ostream &os, const Position &p)
{
    return os << p.x << " " << p.y << " " << p.z << " " << p.t;
}

}  // namespace kuqcd

#endif
