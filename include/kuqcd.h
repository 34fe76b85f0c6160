/*
 * KuQCD public API, drop-in for the reference's include/kuqcd.h:26-34: the same five calls in namespace kuqcd,
 * C++ linkage, default visibility.  They are implemented by libkuqcd_b200.so on the GPU and forward to the
 * C-linkage twins declared in kuqcd_b200.h.
 *
 * Call order (reference docs, kuqcd.cpp): kuqcd_init -> kuqcd_load_gaugefield(fat) -> kuqcd_load_gaugefield(long)
 * -> kuqcd_solve_multishift (repeatable) -> kuqcd_gauge_free -> kuqcd_end.
 */
#ifndef KUQCD_H
#define KUQCD_H

#include "kuqcd_enum.h"
#include "kuqcd_b200.h"

#define kuqcd_export __attribute__((visibility("default")))

#ifdef __cplusplus
namespace kuqcd {

kuqcd_export KuQCDStatus kuqcd_init();
kuqcd_export KuQCDStatus kuqcd_load_gaugefield(void *h_gauge, KuQCDGaugeParam *param);
kuqcd_export KuQCDStatus kuqcd_solve_multishift(void **_hp_x, void *_hp_b, KuQCDInvertParam *param);

kuqcd_export void kuqcd_gauge_free();
kuqcd_export void kuqcd_end();

}  // namespace kuqcd
#endif

#endif
