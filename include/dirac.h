/*
 * Operator interface of the class-level API (the reference's dirac.h:19-28): what an inverter sees of an operator.
 */
#ifndef DIRAC_H
#define DIRAC_H

#include "kuqcd_enum.h"

namespace kuqcd {

template <typename VecT>
class Dirac {
public:
    KuQCDDslashType diracType = KUQCD_INVALID_DIRAC;
    explicit Dirac(KuQCDDslashType dt) : diracType(dt) {}
    virtual ~Dirac() {}
    virtual void Dslash(const VecT &src, VecT &dst, bool update) = 0;
    virtual void MdaggM(const VecT &src, VecT &dst, bool update) = 0;
};

}  // namespace kuqcd

#endif
