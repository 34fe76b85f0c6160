/*
 * Communication layer of the class-level API (the reference's communication.h:19-141).  One GPU per process with a
 * 1x1x1x1 grid: every neighbour rank is this rank, halos are periodic wrap-around inside the kernels, and the scalar
 * helpers are the identity.  CommBase keeps the reference's constructor, so GaugeField(LattBase&, CommBase&)
 * callers compile unchanged.  (Several GPUs: the t-slab decomposition of the device API, kq_slab_*.)
 */
#ifndef COMMUNICATION_H
#define COMMUNICATION_H

#include <array>
#include <cstdint>

#include "latt_base.h"

namespace kuqcd {

inline void Root2All(int &) {}
inline void Root2All(int64_t &) {}
inline void Root2All(size_t &) {}
inline void Root2All(bool &) {}
inline void Root2All(float &) {}
inline void Root2All(double &) {}
inline int Reduce(int in) { return in; }
inline uint32_t Reduce(uint32_t in) { return in; }
inline float Reduce(float in) { return in; }
inline double Reduce(double in) { return in; }

/* neighbour ranks of the gauge-field halo geometry; all this rank */
class CommBase {
public:
    LattBase &latBase;
    std::array<std::array<int, 2>, 4> rankHyperPlane{};
    std::array<size_t, 4> lenHyperPlane{};
    std::array<std::array<int, 4>, 6> rankPlane{};
    std::array<size_t, 6> lenPlane{};
    std::array<std::array<int, 8>, 4> rankStripe{};
    std::array<size_t, 4> lenStripe{};
    std::array<int, 16> rankCorner{};
    size_t lenCorner = 0;

    CommBase() = delete;
    CommBase(const CommBase &o) = default;
    explicit CommBase(LattBase &lb) : latBase(lb) {}
    CommBase &operator=(const CommBase &) = delete;
};

}  // namespace kuqcd

#endif
