/*
 * 3x3 link matrix of the class-level API (the reference's su3.h:19-71): Recon/2 batched complex entries, row-major
 * (m[col + 3*row], kuqcd_math.cpp:20-35).  It is the element of GaugeField::data, so its layout is kept exactly.
 * Only full storage (KUQCD_GAUGE_RECON_NO) reaches the GPU: the reference's reconstruction is a stub
 * (su3.cpp:250-254) and its API rejects the other recon values.
 */
#ifndef SU3_H
#define SU3_H

#include "kuqcd_complex.h"
#include "kuqcd_enum.h"
#include "spinor.h"

namespace kuqcd {

template <typename T, int Nbatch, KuQCDReconstructType Recon>
class SU3 {
public:
    Complex<T, Nbatch> m[Recon >> 1];

    SU3() = default;
    SU3(const SU3 &other) = default;
    SU3 &operator=(const SU3 &other) = default;

    SU3 &operator+=(const SU3 &o)
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l] += o.m[l];
        return *this;
    }
    SU3 &operator-=(const SU3 &o)
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l] -= o.m[l];
        return *this;
    }
    /* matrix product (full storage) */
    SU3 &operator*=(const SU3 &o)
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "matrix product needs full storage");
        SU3 r;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                Complex<T, Nbatch> s;
                for (int k = 0; k < 3; ++k) s += m[k + 3 * i] * o.m[j + 3 * k];
                r.m[j + 3 * i] = s;
            }
        return *this = r;
    }
    SU3 &operator*=(const Complex<T, Nbatch> &s)
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l] *= s;
        return *this;
    }
    SU3 &operator*=(T s)
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l] *= s;
        return *this;
    }
    SU3 &operator/=(T s)
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l] /= s;
        return *this;
    }
    SU3 operator-() const
    {
        SU3 r(*this);
        for (int l = 0; l < (Recon >> 1); ++l) r.m[l] = -r.m[l];
        return r;
    }
    void Conj()
    {
        for (int l = 0; l < (Recon >> 1); ++l) m[l].Conj();
    }
    void Trans()
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "transpose needs full storage");
        for (int i = 0; i < 3; ++i)
            for (int j = i + 1; j < 3; ++j) {
                const Complex<T, Nbatch> t = m[j + 3 * i];
                m[j + 3 * i] = m[i + 3 * j];
                m[i + 3 * j] = t;
            }
    }
    void Dagger()
    {
        Trans();
        Conj();
    }
    Complex<T, Nbatch> Trace() const
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "trace needs full storage");
        return m[0] + m[4] + m[8];
    }
    T RealTrace() const { return RealSum(Trace()); }
    void Identity()
    {
        static_assert(Recon == KUQCD_GAUGE_RECON_NO, "identity needs full storage");
        for (int l = 0; l < 9; ++l) m[l] = Complex<T, Nbatch>((l % 4 == 0) ? T(1) : T(0));
    }
    void Print() const
    {
        for (int l = 0; l < (Recon >> 1); ++l) std::cout << m[l] << ((l % 3 == 2) ? "\n" : " ");
    }
};

template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator+(SU3<T, Nbatch, Recon> lhs, const SU3<T, Nbatch, Recon> &rhs)
{
    return lhs += rhs;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator-(SU3<T, Nbatch, Recon> lhs, const SU3<T, Nbatch, Recon> &rhs)
{
    return lhs -= rhs;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator*(T s, SU3<T, Nbatch, Recon> rhs)
{
    return rhs *= s;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator*(SU3<T, Nbatch, Recon> lhs, T s)
{
    return lhs *= s;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator*(const Complex<T, Nbatch> &s, SU3<T, Nbatch, Recon> rhs)
{
    return rhs *= s;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator*(SU3<T, Nbatch, Recon> lhs, const Complex<T, Nbatch> &s)
{
    return lhs *= s;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
SU3<T, Nbatch, Recon> operator/(SU3<T, Nbatch, Recon> lhs, T s)
{
    return lhs /= s;
}
template <typename T, int Nbatch, KuQCDReconstructType Recon>
std::ostream &operator<<(std::ostream &os, const SU3<T, Nbatch, Recon> &u)
{
    for (int l = 0; l < (Recon >> 1); ++l) os << u.m[l] << ((l % 3 == 2) ? "\n" : " ");
    return os;
}

}  // namespace kuqcd

#endif
