/*
 * Small utilities of the class-level API (the reference's kuqcd_utils.h:40-59, 103-121): rank helpers, the
 * Rank0Printf macros and the uint4 state type.  kuqcd_b200 drives one GPU per process with a 1x1x1x1 process grid
 * (kuqcd_init rejects any other grid), so the rank is 0 and the process count 1; no MPI is needed.
 */
#ifndef KUQCD_UTILS_H
#define KUQCD_UTILS_H

#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>

namespace kuqcd {

inline int GetRank() { return 0; }
inline int GetNp() { return 1; }

#define Rank0Printf     \
    if (GetRank() == 0) \
    printf
#define Rank0Fprintf    \
    if (GetRank() == 0) \
    fprintf

struct uint4 {
    unsigned int x, y, z, w;
    uint4() = default;
    uint4(unsigned int x_, unsigned int y_, unsigned int z_, unsigned int w_) : x(x_), y(y_), z(z_), w(w_) {}
};

inline void Divmod(int nominator, int denominator, int &quotient, int &remainder)
{
    quotient = nominator / denominator;
    remainder = nominator - quotient * denominator;
}

inline void Divmod(size_t nominator, size_t denominator, size_t &quotient, size_t &remainder)
{
    quotient = nominator / denominator;
    remainder = nominator - quotient * denominator;
}

inline bool IsOdd(int cand) { return (cand & 0x1) != 0; }

/* GPU the class-level objects of this process use: KUQCD_DEVICE, default 0 */
inline int DefaultDevice()
{
    const char *s = std::getenv("KUQCD_DEVICE");
    return s ? std::atoi(s) : 0;
}

}  // namespace kuqcd

#endif
