/*
 * Inverter interface of the class-level API (the reference's inverter.h:19-34).
 */
#ifndef INVERTER_H
#define INVERTER_H

#include "dirac.h"
#include "kuqcd_enum.h"
#include "spinor.h"
#include "spinor_field.h"

namespace kuqcd {

template <typename T, typename VecT>
class Inverter {
public:
    KuQCDInverterType inverterType;
    Dirac<VecT> *dirac = nullptr;
    Inverter(KuQCDInverterType it, Dirac<VecT> *dirac_) : inverterType(it), dirac(dirac_) {}
    virtual ~Inverter() {}
    virtual int Invert(int noShifts, T shifts[], const VecT &src, VecT *sol[], const double tol, int maxIters) = 0;
};

}  // namespace kuqcd

#endif
