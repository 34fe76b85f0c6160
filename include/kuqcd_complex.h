/*
 * Batched complex number of the class-level API (the reference's kuqcd_complex.h:19-108): z holds the Nbatch real
 * parts, then the Nbatch imaginary parts.  This is the element layout of the host fields (a ColorSpinor is three of
 * them, an SU3 nine), so it is kept exactly.  Arithmetic here is per-site host convenience; field-wide arithmetic runs
 * on the GPU (spinor_field.h).
 */
#ifndef KUQCD_COMPLEX_H
#define KUQCD_COMPLEX_H

#include <cmath>
#include <iostream>

#include "kuqcd_utils.h"

namespace kuqcd {

template <typename T, int Nbatch>
class Complex {
public:
    T z[Nbatch << 1] = {0};

    Complex() = default;
    explicit Complex(T real, T imag = 0)
    {
        for (int j = 0; j < Nbatch; ++j) {
            z[j] = real;
            z[Nbatch + j] = imag;
        }
    }
    explicit Complex(const T values[2 * Nbatch])
    {
        for (int j = 0; j < 2 * Nbatch; ++j) z[j] = values[j];
    }
    Complex(const T realParts[Nbatch], const T imagParts[Nbatch])
    {
        for (int j = 0; j < Nbatch; ++j) {
            z[j] = realParts[j];
            z[Nbatch + j] = imagParts[j];
        }
    }
    Complex(const Complex &other) = default;
    Complex &operator=(const Complex &other) = default;
    Complex &operator=(T real)
    {
        for (int j = 0; j < Nbatch; ++j) {
            z[j] = real;
            z[Nbatch + j] = 0;
        }
        return *this;
    }

    constexpr T Real(int i = 0) const noexcept { return z[i]; }
    constexpr T &Real(int i = 0) noexcept { return z[i]; }
    constexpr T Imag(int i = 0) const noexcept { return z[Nbatch + i]; }
    constexpr T &Imag(int i = 0) noexcept { return z[Nbatch + i]; }
    T &DataSafe(int i) { return z[i < 0 ? 0 : (i >= 2 * Nbatch ? 2 * Nbatch - 1 : i)]; }
    const T &DataSafe(int i) const { return z[i < 0 ? 0 : (i >= 2 * Nbatch ? 2 * Nbatch - 1 : i)]; }

    void Conj()
    {
        for (int j = 0; j < Nbatch; ++j) z[Nbatch + j] = -z[Nbatch + j];
    }
    Complex<T, 1> GetBatch(int i = 0) const { return Complex<T, 1>(z[i], z[Nbatch + i]); }

    Complex &operator+=(const Complex &o)
    {
        for (int j = 0; j < 2 * Nbatch; ++j) z[j] += o.z[j];
        return *this;
    }
    Complex &operator-=(const Complex &o)
    {
        for (int j = 0; j < 2 * Nbatch; ++j) z[j] -= o.z[j];
        return *this;
    }
    Complex &operator*=(const Complex &o)
    {
        for (int j = 0; j < Nbatch; ++j) {
            const T re = z[j] * o.z[j] - z[Nbatch + j] * o.z[Nbatch + j];
            const T im = z[j] * o.z[Nbatch + j] + z[Nbatch + j] * o.z[j];
            z[j] = re;
            z[Nbatch + j] = im;
        }
        return *this;
    }
    Complex &operator/=(const Complex &o)
    {
        for (int j = 0; j < Nbatch; ++j) {
            const T d = o.z[j] * o.z[j] + o.z[Nbatch + j] * o.z[Nbatch + j];
            const T re = (z[j] * o.z[j] + z[Nbatch + j] * o.z[Nbatch + j]) / d;
            const T im = (z[Nbatch + j] * o.z[j] - z[j] * o.z[Nbatch + j]) / d;
            z[j] = re;
            z[Nbatch + j] = im;
        }
        return *this;
    }
    Complex &operator*=(T s)
    {
        for (int j = 0; j < 2 * Nbatch; ++j) z[j] *= s;
        return *this;
    }
    Complex &operator/=(T s)
    {
        for (int j = 0; j < 2 * Nbatch; ++j) z[j] /= s;
        return *this;
    }
    Complex operator-() const
    {
        Complex r(*this);
        for (int j = 0; j < 2 * Nbatch; ++j) r.z[j] = -r.z[j];
        return r;
    }
};

template <typename T, int Nbatch>
Complex<T, Nbatch> Conj(const Complex<T, Nbatch> &a)
{
    Complex<T, Nbatch> r(a);
    r.Conj();
    return r;
}
template <typename T, int Nbatch>
T Norm2(const Complex<T, Nbatch> &a, int i)
{
    return a.z[i] * a.z[i] + a.z[Nbatch + i] * a.z[Nbatch + i];
}
template <typename T, int Nbatch>
T Abs(const Complex<T, Nbatch> &a, int i)
{
    return std::sqrt(Norm2(a, i));
}
template <typename T, int Nbatch>
T Arg(const Complex<T, Nbatch> &a, int i)
{
    return std::atan2(a.z[Nbatch + i], a.z[i]);
}
template <typename T, int Nbatch>
T Norm2(const Complex<T, Nbatch> &a)
{
    T s = 0;
    for (int j = 0; j < Nbatch; ++j) s += Norm2(a, j);
    return s;
}
template <typename T, int Nbatch>
T Abs(const Complex<T, Nbatch> &a)
{
    T s = 0;
    for (int j = 0; j < Nbatch; ++j) s += Abs(a, j);
    return s;
}
template <typename T, int Nbatch>
T RealSum(const Complex<T, Nbatch> &a)
{
    T s = 0;
    for (int j = 0; j < Nbatch; ++j) s += a.z[j];
    return s;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator+(Complex<T, Nbatch> lhs, const Complex<T, Nbatch> &rhs)
{
    return lhs += rhs;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator-(Complex<T, Nbatch> lhs, const Complex<T, Nbatch> &rhs)
{
    return lhs -= rhs;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator*(Complex<T, Nbatch> lhs, const Complex<T, Nbatch> &rhs)
{
    return lhs *= rhs;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator/(Complex<T, Nbatch> lhs, const Complex<T, Nbatch> &rhs)
{
    return lhs /= rhs;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator*(T s, Complex<T, Nbatch> rhs)
{
    return rhs *= s;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator*(Complex<T, Nbatch> lhs, T s)
{
    return lhs *= s;
}
template <typename T, int Nbatch>
Complex<T, Nbatch> operator/(Complex<T, Nbatch> lhs, T s)
{
    return lhs /= s;
}
template <typename T, int Nbatch>
bool operator==(const Complex<T, Nbatch> &lhs, const Complex<T, Nbatch> &rhs)
{
    for (int j = 0; j < 2 * Nbatch; ++j)
        if (lhs.z[j] != rhs.z[j]) return false;
    return true;
}
template <typename T, int Nbatch>
bool operator!=(const Complex<T, Nbatch> &lhs, const Complex<T, Nbatch> &rhs)
{
    return !(lhs == rhs);
}
template <typename T, int Nbatch>
std::ostream &operator<<(std::ostream &os, const Complex<T, Nbatch> &a)
{
    for (int j = 0; j < Nbatch; ++j) os << "(" << a.z[j] << "," << a.z[Nbatch + j] << ")" << (j + 1 < Nbatch ? " " : "");
    return os;
}

}  // namespace kuqcd

#endif
