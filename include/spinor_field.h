/*
 * Colour-vector fields and their BLAS-1 of the class-level API (the reference's spinor_field.h:19-62,
 * spinor_field.cpp:17-252).  Same constructors, members and free functions; every field-wide operation runs on the
 * GPU (kq_vec_axpby / kq_vec_dot of libkuqcd_b200): the first lenBulk * Ns sites of `data` (the sites the
 * reference's loops visit) are copied to the device, combined there and the result copied back before the call
 * returns, so `data` always holds the current values.  Reductions accumulate in FP64 in a fixed order on the device
 * (the reference reduces in T with OpenMP); they are returned in T.
 */
#ifndef SPINOR_FIELD_H
#define SPINOR_FIELD_H

#include <cmath>

#include "lattice_field.h"

namespace kuqcd {

template <typename T, int Nbatch, int Ns>
class SpinorField : public LatticeField<ColorSpinor<T, Nbatch>> {
public:
    typedef ColorSpinor<T, Nbatch> SpinorT;

    SpinorField() = delete;
    SpinorField(const SpinorField &spinor) : LatticeField<SpinorT>(spinor) {}
    explicit SpinorField(LattBase &latBase) : LatticeField<SpinorT>(latBase, Ns * Nbatch * 6) {}
    SpinorField &operator=(const SpinorField &o)
    {
        LatticeField<SpinorT>::operator=(o);
        return *this;
    }

    SpinorT GetSpinorCopy(size_t i, int ns) const { return this->data[ns + Ns * i]; }
    SpinorT &GetSpinorRef(size_t i, int ns) { return this->data[ns + Ns * i]; }
    inline int GetNbatch() { return Nbatch; }

    /* reals the BLAS-1 functions combine: the first lenBulk sites, as the reference's loops */
    size_t BulkReals() const { return this->latBase.lenBulk * (size_t)Ns * 6 * Nbatch; }
    T *Reals() { return reinterpret_cast<T *>(this->data); }
    const T *Reals() const { return reinterpret_cast<const T *>(this->data); }

    SpinorField operator*(T scalar)
    {
        SpinorField res(*this);
        detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), BulkReals(), (double)scalar, Reals(), 0.0,
                                   res.Reals()),
                      "SpinorField::operator*");
        return res;
    }
    SpinorField &operator-=(const SpinorField &v)
    {
        detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), BulkReals(), -1.0, v.Reals(), 1.0, Reals()),
                      "SpinorField::operator-=");
        return *this;
    }
    SpinorField operator+(const SpinorField &v)
    {
        SpinorField res(*this);
        detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), BulkReals(), 1.0, v.Reals(), 1.0,
                                   res.Reals()),
                      "SpinorField::operator+");
        return res;
    }
};

/* vec1 - vec2 */
template <typename T, int Nbatch, int Ns>
SpinorField<T, Nbatch, Ns> operator-(const SpinorField<T, Nbatch, Ns> &vec1, const SpinorField<T, Nbatch, Ns> &vec2)
{
    SpinorField<T, Nbatch, Ns> res(vec1);
    detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), res.BulkReals(), -1.0, vec2.Reals(), 1.0,
                               res.Reals()),
                  "operator-");
    return res;
}

/* sum over bulk sites of |v|^2 (spinor_field.cpp:228-252) */
template <typename T, int Nbatch, int Ns>
T Norm2(const SpinorField<T, Nbatch, Ns> &vec)
{
    double r = 0.0;
    detail::check(kq_vec_dot(DefaultDevice(), detail::prec_of<T>(), vec.BulkReals(), vec.Reals(), vec.Reals(), &r),
                  "Norm2");
    return (T)r;
}

template <typename T, int Nbatch, int Ns>
T Norm(const SpinorField<T, Nbatch, Ns> &vec)
{
    return std::sqrt(Norm2(vec));
}

/* y = a x - y (spinor_field.cpp:130-144) */
template <typename T, int Nbatch, int Ns>
void Axmy(SpinorField<T, Nbatch, Ns> &y, const SpinorField<T, Nbatch, Ns> &x, T a)
{
    detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), y.BulkReals(), (double)a, x.Reals(), -1.0,
                               y.Reals()),
                  "Axmy");
}

/* y = y + a x */
template <typename T, int Nbatch, int Ns>
void Axpy(SpinorField<T, Nbatch, Ns> &y, const SpinorField<T, Nbatch, Ns> &x, T a)
{
    detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), y.BulkReals(), (double)a, x.Reals(), 1.0,
                               y.Reals()),
                  "Axpy");
}

/* y = y - a x */
template <typename T, int Nbatch, int Ns>
void Ymax(SpinorField<T, Nbatch, Ns> &y, const SpinorField<T, Nbatch, Ns> &x, T a)
{
    detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), y.BulkReals(), -(double)a, x.Reals(), 1.0,
                               y.Reals()),
                  "Ymax");
}

/* y = a x + b y */
template <typename T, int Nbatch, int Ns>
void Axpby(SpinorField<T, Nbatch, Ns> &y, const SpinorField<T, Nbatch, Ns> &x, T a, T b)
{
    detail::check(kq_vec_axpby(DefaultDevice(), detail::prec_of<T>(), y.BulkReals(), (double)a, x.Reals(), (double)b,
                               y.Reals()),
                  "Axpby");
}

/* sum over bulk sites of Re(conj(bra) ket), i.e. the real dot product of the reals (spinor_field.cpp:200-226) */
template <typename T, int Nbatch, int Ns>
T RealDot(const SpinorField<T, Nbatch, Ns> &bra, const SpinorField<T, Nbatch, Ns> &ket)
{
    double r = 0.0;
    detail::check(kq_vec_dot(DefaultDevice(), detail::prec_of<T>(), bra.BulkReals(), bra.Reals(), ket.Reals(), &r),
                  "RealDot");
    return (T)r;
}

}  // namespace kuqcd

#endif
