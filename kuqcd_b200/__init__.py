"""kuqcd_b200 — B200-native HISQ staggered even-odd dslash and multishift CG behind KuQCD's API.

The product is ``libkuqcd_b200.so`` (CUDA, sm_100a) built from ``csrc/`` by :mod:`kuqcd_b200.build`.
This package is the Python host mirror of its C ABI (``include/kuqcd_b200.h``): ctypes bindings of the
reference-facing calls ``kuqcd_init / kuqcd_load_gaugefield / kuqcd_solve_multishift / kuqcd_gauge_free /
kuqcd_end`` (reference ``include/kuqcd.h:29-34``) and of the device-level context API.

There is no CPU fallback: importing works without a GPU, but every compute call goes to the CUDA library and
raises if it is missing.
"""
from .lib import (  # noqa: F401
    KUQCD_SUCCESS, KUQCD_ERR_INVALID_PARAM, KUQCD_ERR_UNSUPPORTED, KUQCD_ERR_NULL_POINTER, KUQCD_ERR_NO_MEMORY,
    KUQCD_ERR_UNKNOWN_TYPE, KUQCD_ERR_UNEXPECTED_CALL_ORDER, KUQCD_ERR_NO_RESOURCE, KUQCD_ERR_UNKNOWN_ERROR,
    KUQCD_EVEN, KUQCD_ODD, KUQCD_ALL, KUQCD_HALF, KUQCD_SINGLE, KUQCD_DOUBLE, KUQCD_NORMAL_ORDER,
    KUQCD_BATCH_ORDER, KUQCD_EVEN_EVEN, KUQCD_ODD_ODD, KUQCD_FAT_LINK, KUQCD_LONG_LINK, KUQCD_WILSON_LINK,
    KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_12, KUQCD_GAUGE_RECON_U14, KUQCD_GAUGE_RECON_8,
    KUQCD_WILSON_DIRAC, KUQCD_WILSONPC_DIRAC, KUQCD_HISQ_DIRAC, KUQCD_HISQPC_DIRAC, KUQCD_CG, KUQCD_CGM,
    KUQCD_XYZT_ORDER, KUQCD_TZYX_ORDER, KQ_SOLVER_CGM, KQ_SOLVER_MIXED, KQ_SOLVER_CGM_WINDOWED, KQ_PARITY_FULL,
    KuQCDGaugeParam, KuQCDInvertParam, SolveParam, SolveInfo, EXPORTED_SYMBOLS,
    library, lib_path, kuqcd_init, kuqcd_load_gaugefield, kuqcd_solve_multishift, kuqcd_gauge_free, kuqcd_end,
    Context, KuQCDError, Batch, BatchInfo, Net, fcg_polish,
)
