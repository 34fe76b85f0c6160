/*
 * Colour vector of the class-level API (the reference's spinor.h:19-67): three batched complex components.  It is
 * the element of SpinorField::data, so its layout (c[3] of Complex<T, Nbatch>) is kept exactly.
 */
#ifndef SPINOR_H
#define SPINOR_H

#include "kuqcd_complex.h"

namespace kuqcd {

template <typename T, int Nbatch>
class ColorSpinor {
public:
    Complex<T, Nbatch> c[3];

    ColorSpinor() = default;
    ColorSpinor(const ColorSpinor &other) = default;
    explicit ColorSpinor(const Complex<T, Nbatch> &other) { c[0] = c[1] = c[2] = other; }
    ColorSpinor(const Complex<T, Nbatch> &r, const Complex<T, Nbatch> &g, const Complex<T, Nbatch> &b)
    {
        c[0] = r;
        c[1] = g;
        c[2] = b;
    }
    explicit ColorSpinor(const Complex<T, Nbatch> comps[3])
    {
        for (int i = 0; i < 3; ++i) c[i] = comps[i];
    }
    ColorSpinor(T real, T imag = 0) { c[0] = c[1] = c[2] = Complex<T, Nbatch>(real, imag); }

    Complex<T, Nbatch> &ColorComponent(int i) { return c[i < 0 ? 0 : (i > 2 ? 2 : i)]; }
    const Complex<T, Nbatch> &ColorComponent(int i) const { return c[i < 0 ? 0 : (i > 2 ? 2 : i)]; }

    ColorSpinor &operator=(const ColorSpinor &other) = default;
    ColorSpinor &operator+=(const ColorSpinor &o)
    {
        for (int i = 0; i < 3; ++i) c[i] += o.c[i];
        return *this;
    }
    ColorSpinor &operator-=(const ColorSpinor &o)
    {
        for (int i = 0; i < 3; ++i) c[i] -= o.c[i];
        return *this;
    }
    ColorSpinor &operator*=(const ColorSpinor &o)
    {
        for (int i = 0; i < 3; ++i) c[i] *= o.c[i];
        return *this;
    }
    ColorSpinor &operator*=(T s)
    {
        for (int i = 0; i < 3; ++i) c[i] *= s;
        return *this;
    }
    ColorSpinor &operator/=(T s)
    {
        for (int i = 0; i < 3; ++i) c[i] /= s;
        return *this;
    }
    ColorSpinor operator-() const
    {
        ColorSpinor r(*this);
        for (int i = 0; i < 3; ++i) r.c[i] = -r.c[i];
        return r;
    }
    void Conj()
    {
        for (int i = 0; i < 3; ++i) c[i].Conj();
    }
    ColorSpinor<T, 1> GetBatch(int i = 0) const
    {
        return ColorSpinor<T, 1>(c[0].GetBatch(i), c[1].GetBatch(i), c[2].GetBatch(i));
    }
    void Clear()
    {
        for (int i = 0; i < 3; ++i) c[i] = Complex<T, Nbatch>();
    }
    void PrintBatch(int i) const
    {
        const ColorSpinor<T, 1> b = GetBatch(i);
        std::cout << b.c[0] << " " << b.c[1] << " " << b.c[2] << "\n";
    }
};

template <typename T, int Nbatch>
T Norm2(const ColorSpinor<T, Nbatch> &a)
{
    return Norm2(a.c[0]) + Norm2(a.c[1]) + Norm2(a.c[2]);
}
template <typename T, int Nbatch>
T Norm(const ColorSpinor<T, Nbatch> &a)
{
    return std::sqrt(Norm2(a));
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> Conj(const ColorSpinor<T, Nbatch> &a)
{
    ColorSpinor<T, Nbatch> r(a);
    r.Conj();
    return r;
}
/* sum over colours of conj(bra) * ket */
template <typename T, int Nbatch>
Complex<T, Nbatch> Dot(const ColorSpinor<T, Nbatch> &bra, const ColorSpinor<T, Nbatch> &ket)
{
    Complex<T, Nbatch> s;
    for (int i = 0; i < 3; ++i) s += Conj(bra.c[i]) * ket.c[i];
    return s;
}
template <typename T, int Nbatch>
T RealDot(const ColorSpinor<T, Nbatch> &bra, const ColorSpinor<T, Nbatch> &ket)
{
    T s = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 2 * Nbatch; ++j) s += bra.c[i].z[j] * ket.c[i].z[j];
    return s;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator+(ColorSpinor<T, Nbatch> lhs, const ColorSpinor<T, Nbatch> &rhs)
{
    return lhs += rhs;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator-(ColorSpinor<T, Nbatch> lhs, const ColorSpinor<T, Nbatch> &rhs)
{
    return lhs -= rhs;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator*(ColorSpinor<T, Nbatch> lhs, const ColorSpinor<T, Nbatch> &rhs)
{
    return lhs *= rhs;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator*(T s, ColorSpinor<T, Nbatch> rhs)
{
    return rhs *= s;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator*(ColorSpinor<T, Nbatch> lhs, T s)
{
    return lhs *= s;
}
template <typename T, int Nbatch>
ColorSpinor<T, Nbatch> operator/(ColorSpinor<T, Nbatch> lhs, T s)
{
    return lhs /= s;
}
template <typename T, int Nbatch>
bool operator==(const ColorSpinor<T, Nbatch> &a, const ColorSpinor<T, Nbatch> &b)
{
    return a.c[0] == b.c[0] && a.c[1] == b.c[1] && a.c[2] == b.c[2];
}
template <typename T, int Nbatch>
bool operator!=(const ColorSpinor<T, Nbatch> &a, const ColorSpinor<T, Nbatch> &b)
{
    return !(a == b);
}
template <typename T, int Nbatch>
std::ostream &operator<<(std::ostream &os, const ColorSpinor<T, Nbatch> &cs)
{
    return os << cs.c[0] << " " << cs.c[1] << " " << cs.c[2];
}

}  // namespace kuqcd

#endif
