/*
 * KuQCD public API, drop-in for the reference's include/kuqcd.h:14-34: the same five calls in namespace kuqcd,
 * C++ linkage, default visibility, implemented by libkuqcd_b200.so on the GPU (they forward to the C-linkage twins
 * declared in kuqcd_b200.h).  Like the reference's header it also brings in the class-level API -- Lattice,
 * LattBase, GaugeField, SpinorField and the BLAS-1 functions, DiracHISQ, CGM, the loggers -- as header-only
 * classes over the same library (dirac_hisq.h, inverter_cgm.h, ...).  No MPI is needed: one GPU per process.
 *
 * Call order (reference docs, kuqcd.cpp): kuqcd_init -> kuqcd_load_gaugefield(fat) -> kuqcd_load_gaugefield(long)
 * -> kuqcd_solve_multishift (repeatable) -> kuqcd_gauge_free -> kuqcd_end.
 */
#ifndef KUQCD_H
#define KUQCD_H

#include "kuqcd_b200.h"
#include "kuqcd_enum.h"

#ifdef __cplusplus
#include <cstdio>

#ifndef KUQCD_NO_CLASS_API
#include "command_line.h"
#include "dirac_hisq.h"
#include "index_utils.h"
#include "inverter_cgm.h"
#include "logger.h"
#endif

#define kuqcd_export __attribute__((visibility("default")))

namespace kuqcd {

kuqcd_export KuQCDStatus kuqcd_init();
kuqcd_export KuQCDStatus kuqcd_load_gaugefield(void *h_gauge, KuQCDGaugeParam *param);
kuqcd_export KuQCDStatus kuqcd_solve_multishift(void **_hp_x, void *_hp_b, KuQCDInvertParam *param);

kuqcd_export void kuqcd_gauge_free();
kuqcd_export void kuqcd_end();

}  // namespace kuqcd
#endif

#endif
