/*
 * Multishift CG of the class-level API (the reference's inverter_cgm.h:19-28, inverter_cgm.cpp:17-87), solved on
 * the GPU by libkuqcd_b200 (kq_solve_multishift, KQ_SOLVER_CGM) with the reference's recurrences, shift semantics
 * and stopping rule:
 *   sol[0] solves (shifts[0] - D D) x = src; sol[j >= 1] solves (shifts[0] + shifts[j] - D D) x = src;
 *   shift k stops when zeta_k^2 |r|^2 < tol; the return value is the iteration count.
 * The operator must be a DiracHISQ of this library (its links are already on the GPU).  src and the solutions are
 * host fields: src is copied in, the solutions are copied out as they converge.  Scalars and reductions run in
 * FP64 on the GPU in either precision (the reference's float path reduces in float).  A breakdown (non-finite p.Ap)
 * throws std::runtime_error; reaching maxIters prints the reference's warning and returns maxIters.
 */
#ifndef CGM_H
#define CGM_H

#include <cstdio>
#include <stdexcept>
#include <vector>

#include "dirac_hisq.h"
#include "inverter.h"

namespace kuqcd {

template <typename T, typename VecT>
class CGM : public Inverter<T, VecT> {
public:
    CGM(KuQCDInverterType it, Dirac<VecT> *dirac_) : Inverter<T, VecT>(it, dirac_) {}
    ~CGM() override {}

    int Invert(int noShifts, T shifts[], const VecT &src, VecT *sol[], const double tol, int maxIters) override
    {
        auto *op = dynamic_cast<detail::DeviceOperator *>(this->dirac);
        if (!op || !op->DeviceContext())
            throw std::invalid_argument("CGM::Invert: the operator must be a kuqcd_b200 DiracHISQ");
        if (noShifts <= 0 || noShifts > 64) throw std::invalid_argument("CGM::Invert: 1..64 shifts");
        typedef typename std::remove_reference<decltype(*src.data)>::type SpinorT;
        constexpr int Nb = sizeof(SpinorT) / (6 * sizeof(T));
        const int parity = detail::field_parity(src.latBase);
        std::vector<double> sh(shifts, shifts + noShifts);
        detail::SpinorRecord<T, Nb> b(src.latBase, const_cast<SpinorT *>(src.data), 1);
        b.load();
        std::vector<detail::SpinorRecord<T, Nb>> xs;
        std::vector<void *> xp;
        xs.reserve(noShifts);
        for (int k = 0; k < noShifts; ++k) {
            if (detail::field_parity(sol[k]->latBase) != parity)
                throw std::invalid_argument("CGM::Invert: solutions must live on the source's sites");
            xs.emplace_back(sol[k]->latBase, sol[k]->data, 1);
            xp.push_back(xs.back().ptr());
        }
        kq_solve_param p{};
        p.parity = parity == 2 ? KQ_PARITY_FULL : parity;
        p.num_shift = noShifts;
        p.shifts = sh.data();
        p.shift_mode = 0;
        p.solver = KQ_SOLVER_CGM;
        p.prec = detail::prec_of<T>();
        p.host_prec = detail::prec_of<T>();
        p.max_iter = maxIters;
        p.tol = tol;
        p.rel_residual = 0.0;
        kq_solve_info info{};
        detail::check(kq_solve_multishift(op->DeviceContext(), &p, b.ptr(), xp.data(), &info), "CGM::Invert");
        for (auto &x : xs) x.store();
        if (info.status == 1) throw std::runtime_error("CGM::Invert: breakdown (non-finite p.Ap)");
        if (info.status == 2) printf("CGM: Warning max iteration reached %d\n", info.iter);
        return info.iter;
    }
};

}  // namespace kuqcd

#endif
