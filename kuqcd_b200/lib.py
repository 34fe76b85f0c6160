"""ctypes bindings of libkuqcd_b200.so (declarations in include/kuqcd_b200.h and include/kuqcd.h).

Host-side mirror of the reference API (kuqcd.h:29-34, kuqcd_enum.h:15-121): same enum values, same parameter
structs, same status codes and call order.  Arrays are numpy arrays in the reference's NORMAL_ORDER host layouts
(kuqcd.cpp:103-169).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

# ---------------------------------------------------------------- enums (kuqcd_enum.h:15-98 of the reference)
KUQCD_SUCCESS = 0
KUQCD_ERR_INVALID_PARAM = -1
KUQCD_ERR_UNSUPPORTED = -2
KUQCD_ERR_NULL_POINTER = -3
KUQCD_ERR_NO_MEMORY = -4
KUQCD_ERR_UNKNOWN_TYPE = -5
KUQCD_ERR_UNEXPECTED_CALL_ORDER = -6
KUQCD_ERR_NO_RESOURCE = -7
KUQCD_ERR_UNKNOWN_ERROR = -8
KUQCD_EVEN, KUQCD_ODD, KUQCD_ALL = 0, 1, 2
KUQCD_HALF, KUQCD_SINGLE, KUQCD_DOUBLE = 2, 4, 8
KUQCD_XYZT_ORDER, KUQCD_TZYX_ORDER = 0, 1
KUQCD_NORMAL_ORDER, KUQCD_BATCH_ORDER = 0, 1
KUQCD_EVEN_EVEN, KUQCD_ODD_ODD = 0, 1
KUQCD_WILSON_LINK, KUQCD_FAT_LINK, KUQCD_LONG_LINK = 0, 1, 2
KUQCD_GAUGE_RECON_NO, KUQCD_GAUGE_RECON_U14, KUQCD_GAUGE_RECON_12, KUQCD_GAUGE_RECON_8 = 18, 14, 12, 8
KUQCD_WILSON_DIRAC, KUQCD_WILSONPC_DIRAC, KUQCD_HISQ_DIRAC, KUQCD_HISQPC_DIRAC = 0, 1, 2, 3
KUQCD_CG, KUQCD_CGM = 0, 1
KQ_SOLVER_CGM, KQ_SOLVER_MIXED, KQ_SOLVER_CGM_WINDOWED = 0, 1, 2
KQ_PARITY_FULL = 2  # full-lattice (KUQCD_HISQ_DIRAC) fields: parity 0 then parity 1
KQ_CGM_START, KQ_CGM_ALPHA, KQ_CGM_BETA, KQ_CGM_FINISH = 0, 1, 2, 3  # kq_slab_cgm_step


class KuQCDGaugeParam(C.Structure):
    _fields_ = [("lat", C.c_uint * 4), ("halo_depth", C.c_int), ("od", C.c_int), ("site_subset", C.c_int),
                ("gauge_order", C.c_int), ("prec", C.c_int), ("link_type", C.c_int), ("recon", C.c_int)]


class KuQCDInvertParam(C.Structure):
    _fields_ = [("dslash_type", C.c_int), ("inverter_type", C.c_int), ("matpc_type", C.c_int), ("prec", C.c_int),
                ("num_shift", C.c_int), ("max_iter", C.c_int), ("iter", C.c_int), ("tol", C.c_double),
                ("shifts", C.POINTER(C.c_double))]


class SolveParam(C.Structure):
    _fields_ = [("parity", C.c_int), ("num_shift", C.c_int), ("shifts", C.POINTER(C.c_double)),
                ("shift_mode", C.c_int), ("solver", C.c_int), ("prec", C.c_int), ("host_prec", C.c_int),
                ("max_iter", C.c_int), ("tol", C.c_double), ("rel_residual", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("iter", C.c_int), ("iter_refine", C.c_int), ("status", C.c_int), ("num_shift", C.c_int),
                ("true_residual", C.c_double * 64), ("seconds", C.c_double), ("kernel_launches", C.c_longlong),
                ("sloppy_residual", C.c_double), ("copies_during_solve", C.c_int)]


# every symbol include/*.h declares for the C ABI (checked by the CPU test suite)
EXPORTED_SYMBOLS = [
    "kq_kuqcd_init", "kq_kuqcd_load_gaugefield", "kq_kuqcd_solve_multishift", "kq_kuqcd_gauge_free",
    "kq_kuqcd_end", "kq_context_create", "kq_context_destroy", "kq_load_links", "kq_prepare_links",
    "kq_spinor_bytes", "kq_spinor_upload", "kq_spinor_download", "kq_spinor_convert", "kq_dslash", "kq_mdagm",
    "kq_mdagm_noalloc", "kq_dslash_full", "kq_mdagm_full", "kq_long_links_compressed", "kq_slab_set",
    "kq_slab_face_bytes", "kq_slab_pack_faces", "kq_slab_link_face_bytes", "kq_slab_pack_link_face", "kq_slab_set_link_ghosts",
    "kq_slab_dslash", "kq_slab_dslash_part", "kq_field_axpby", "kq_field_dot", "kq_field_dot_device",
    "kq_slab_cgm_state_bytes", "kq_slab_cgm_init", "kq_slab_cgm_step",
    "kq_slab_cgm_residual", "kq_slab_cgm_update", "kq_slab_cgm_poll", "kq_host_alloc", "kq_host_free", "kq_apply_host",
    "kq_vec_axpby", "kq_vec_dot",
    "kq_solve_multishift", "kq_solve_multishift_device", "kq_true_residuals", "kq_make_links_record",
    "kq_make_source_record", "kq_last_error", "kq_batch_create", "kq_batch_destroy", "kq_batch_add",
    "kq_batch_size", "kq_batch_solve", "kq_batch_system_info", "kq_net_create", "kq_net_destroy",
    "kq_net_num_weights", "kq_net_set_weights", "kq_net_get_weights", "kq_net_get_grad", "kq_net_zero_grad",
    "kq_net_set_context", "kq_net_apply", "kq_net_train_pair", "kq_net_adam", "kq_net_raise_fault_for_test",
    "kq_fcg_polish",
]


class BatchInfo(C.Structure):
    _fields_ = [("num_systems", C.c_int), ("iterations", C.c_int), ("batched_seconds", C.c_double),
                ("kernel_launches", C.c_longlong), ("tile", C.c_int), ("ctas_per_sm", C.c_int),
                ("max_true_residual", C.c_double), ("refined_systems", C.c_int), ("tuned_now", C.c_int),
                ("rhs_per_cta", C.c_int), ("sites_per_thread", C.c_int), ("fp64_rhs_per_pass", C.c_int),
                ("groups", C.c_int),
                ("check_seconds", C.c_double), ("refine_iterations", C.c_int)]

_PKG = Path(__file__).resolve().parent
lib_path = Path(os.environ.get("KUQCD_B200_LIB", _PKG / "libkuqcd_b200.so"))
_lib = None


class KuQCDError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = library().kq_last_error().decode(errors="replace")
        super().__init__(f"{where} failed with status {status}: {msg}")
        self.status = status


def library() -> C.CDLL:
    """Load libkuqcd_b200.so (raises if it has not been built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not lib_path.exists():
        raise RuntimeError(f"{lib_path} is missing: build it with `python -m kuqcd_b200.build`")
    L = C.CDLL(str(lib_path))
    vp, i, u, d, sz = C.c_void_p, C.c_int, C.c_uint, C.c_double, C.c_size_t
    sig = {
        "kq_kuqcd_init": (i, []),
        "kq_kuqcd_load_gaugefield": (i, [vp, C.POINTER(KuQCDGaugeParam)]),
        "kq_kuqcd_solve_multishift": (i, [C.POINTER(vp), vp, C.POINTER(KuQCDInvertParam)]),
        "kq_kuqcd_gauge_free": (None, []),
        "kq_kuqcd_end": (None, []),
        "kq_context_create": (i, [C.POINTER(u), i, C.POINTER(vp)]),
        "kq_context_destroy": (None, [vp]),
        "kq_load_links": (i, [vp, i, vp, i]),
        "kq_prepare_links": (i, [vp, i]),
        "kq_spinor_bytes": (sz, [vp, i]),
        "kq_spinor_upload": (i, [vp, i, vp, i, vp, vp]),
        "kq_spinor_download": (i, [vp, i, vp, vp, i, vp]),
        "kq_spinor_convert": (i, [vp, vp, i, vp, i, vp]),
        "kq_dslash": (i, [vp, i, vp, vp, i, vp]),
        "kq_mdagm": (i, [vp, i, d, vp, vp, vp, i, vp]),
        "kq_mdagm_noalloc": (i, [vp, i, d, vp, vp, i, vp]),
        "kq_dslash_full": (i, [vp, i, vp, vp, vp]),
        "kq_mdagm_full": (i, [vp, i, d, vp, vp, vp, vp]),
        "kq_long_links_compressed": (i, [vp, i, C.POINTER(i)]),
        "kq_slab_set": (i, [vp, i, i]),
        "kq_slab_face_bytes": (sz, [vp, i]),
        "kq_slab_pack_faces": (i, [vp, i, vp, vp, vp, vp]),
        "kq_slab_link_face_bytes": (sz, [vp]),
        "kq_slab_pack_link_face": (i, [vp, vp]),
        "kq_slab_set_link_ghosts": (i, [vp, vp]),
        "kq_slab_dslash": (i, [vp, i, vp, vp, vp, vp, i, vp, d, vp]),
        "kq_field_axpby": (i, [vp, d, vp, d, vp, vp]),
        "kq_field_dot": (i, [vp, vp, vp, C.POINTER(d)]),
        "kq_slab_dslash_part": (i, [vp, i, vp, vp, vp, vp, i, vp, d, i, vp]),
        "kq_field_dot_device": (i, [vp, vp, vp, vp, vp]),
        "kq_slab_cgm_state_bytes": (sz, []),
        "kq_slab_cgm_init": (i, [vp, vp, i, C.POINTER(d), d, i, vp]),
        "kq_slab_cgm_step": (i, [vp, vp, i, vp]),
        "kq_slab_cgm_residual": (i, [vp, vp, vp, vp, vp]),
        "kq_slab_cgm_update": (i, [vp, vp, vp, vp, vp, sz, vp]),
        "kq_slab_cgm_poll": (i, [vp, vp, C.POINTER(i), C.POINTER(i), C.POINTER(d), vp]),
        "kq_solve_multishift": (i, [vp, C.POINTER(SolveParam), vp, C.POINTER(vp), C.POINTER(SolveInfo)]),
        "kq_solve_multishift_device": (i, [vp, C.POINTER(SolveParam), vp, vp, C.POINTER(SolveInfo)]),
        "kq_true_residuals": (i, [vp, i, i, C.POINTER(d), vp, vp, C.POINTER(d)]),
        "kq_make_links_record": (i, [vp, d, C.c_uint64, vp, vp]),
        "kq_make_source_record": (i, [vp, i, C.c_uint64, vp]),
        "kq_last_error": (C.c_char_p, []),
        "kq_batch_create": (i, [i, C.POINTER(vp)]),
        "kq_batch_destroy": (None, [vp]),
        "kq_batch_add": (i, [vp, vp, C.POINTER(SolveParam), vp, vp]),
        "kq_batch_size": (i, [vp]),
        "kq_batch_solve": (i, [vp, C.POINTER(BatchInfo)]),
        "kq_batch_system_info": (i, [vp, i, C.POINTER(SolveInfo)]),
        "kq_net_create": (i, [vp, i, C.POINTER(i), C.POINTER(vp)]),
        "kq_net_destroy": (None, [vp]),
        "kq_net_num_weights": (sz, [vp]),
        "kq_net_set_weights": (i, [vp, C.POINTER(C.c_float), sz]),
        "kq_net_get_weights": (i, [vp, C.POINTER(C.c_float), sz]),
        "kq_net_get_grad": (i, [vp, C.POINTER(C.c_float), sz]),
        "kq_net_zero_grad": (i, [vp]),
        "kq_net_set_context": (i, [vp, vp]),
        "kq_net_apply": (i, [vp, vp, vp, i]),
        "kq_net_train_pair": (i, [vp, vp, vp, i, d, C.POINTER(d)]),
        "kq_net_adam": (i, [vp, C.c_float, C.c_float]),
        "kq_net_raise_fault_for_test": (i, [vp]),
        "kq_fcg_polish": (i, [vp, vp, C.POINTER(SolveParam), vp, vp, C.POINTER(SolveInfo)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _ptr(a) -> C.c_void_p:
    if a is None:
        return None
    if isinstance(a, int):
        return C.c_void_p(a)
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _np_prec(a: np.ndarray) -> int:
    if a.dtype == np.float64:
        return KUQCD_DOUBLE
    if a.dtype == np.float32:
        return KUQCD_SINGLE
    raise TypeError(f"host records are float64 or float32, not {a.dtype}")


# ---------------------------------------------------------------- reference-facing calls (kuqcd.h:29-34)
def kuqcd_init() -> int:
    return library().kq_kuqcd_init()


def kuqcd_load_gaugefield(h_gauge, param: KuQCDGaugeParam) -> int:
    return library().kq_kuqcd_load_gaugefield(_ptr(h_gauge), C.byref(param) if param is not None else None)


def kuqcd_solve_multishift(hp_x, hp_b, param: KuQCDInvertParam) -> int:
    xs = None
    if hp_x is not None:
        xs = (C.c_void_p * len(hp_x))(*[_ptr(x).value if x is not None else None for x in hp_x])
    return library().kq_kuqcd_solve_multishift(xs, _ptr(hp_b), C.byref(param) if param is not None else None)


def kuqcd_gauge_free() -> None:
    library().kq_kuqcd_gauge_free()


def kuqcd_end() -> None:
    library().kq_kuqcd_end()


# ---------------------------------------------------------------- device-level API
# Device buffers usually come from torch, whose kernels (a torch.zeros fill, a copy) run on torch's current stream,
# while a context's own stream is non-blocking.  So the calls below run on torch's current stream unless given one,
# and the calls that only use the library's own streams first wait for torch's pending work on the device.  Every
# call returns with its results complete, or enqueued on torch's stream.
CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream, by a handle that is not NULL


def _torch_stream(device: int):
    """torch's current stream on `device` as a library stream argument.  torch's default stream has the handle 0,
    which the library would read as 'the context's own stream', so it is passed as cudaStreamLegacy."""
    import torch

    h = torch.cuda.current_stream(device).cuda_stream
    return C.c_void_p(h if h else CUDA_STREAM_LEGACY)


def _torch_wait(device: int):
    import torch

    torch.cuda.current_stream(device).synchronize()


class Context:
    """One lattice on one GPU (kq_context): device links, stream, solver workspace."""

    def __init__(self, lat, device: int = 0):
        self.lat = tuple(int(v) for v in lat)
        self.V = int(np.prod(self.lat))
        self.Vh = self.V // 2
        L = library()
        h = C.c_void_p()
        st = L.kq_context_create((C.c_uint * 4)(*self.lat), device, C.byref(h))
        if st != 0:
            raise KuQCDError(st, "kq_context_create")
        self._h = h
        self.device = device

    def _s(self, stream):
        return stream if stream is not None else _torch_stream(self.device)

    def close(self):
        if getattr(self, "_h", None):
            library().kq_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, st, where):
        if st != 0:
            raise KuQCDError(st, where)

    def load_links(self, link_type: int, host: np.ndarray):
        host = np.ascontiguousarray(host)
        assert host.size == self.V * 72, "gauge record has V*4*18 reals"
        self._chk(library().kq_load_links(self._h, link_type, _ptr(host), _np_prec(host)), "kq_load_links")

    def prepare(self, prec: int):
        self._chk(library().kq_prepare_links(self._h, prec), "kq_prepare_links")

    def spinor_bytes(self, prec: int) -> int:
        return int(library().kq_spinor_bytes(self._h, prec))

    def upload(self, prec: int, host: np.ndarray, dev, stream=None):
        host = np.ascontiguousarray(host)
        self._chk(library().kq_spinor_upload(self._h, prec, _ptr(host), _np_prec(host), _ptr(dev), self._s(stream)),
                  "kq_spinor_upload")

    def download(self, prec: int, dev, host_dtype=np.float64, stream=None) -> np.ndarray:
        out = np.empty(self.Vh * 6, dtype=host_dtype)
        self._chk(library().kq_spinor_download(self._h, prec, _ptr(dev), _ptr(out), _np_prec(out), self._s(stream)),
                  "kq_spinor_download")
        return out

    def convert(self, src, src_prec: int, dst, dst_prec: int, stream=None):
        self._chk(library().kq_spinor_convert(self._h, _ptr(src), src_prec, _ptr(dst), dst_prec, self._s(stream)),
                  "kq_spinor_convert")

    def dslash(self, prec: int, src, dst, dst_parity: int, stream=None):
        self._chk(library().kq_dslash(self._h, prec, _ptr(src), _ptr(dst), dst_parity, self._s(stream)), "kq_dslash")

    def mdagm(self, prec: int, sigma: float, src, dst, tmp, parity: int, stream=None):
        self._chk(library().kq_mdagm(self._h, prec, sigma, _ptr(src), _ptr(dst), _ptr(tmp), parity, self._s(stream)),
                  "kq_mdagm")

    def mdagm_noalloc(self, prec: int, sigma: float, src, dst, parity: int, stream=None) -> int:
        """kq_mdagm_noalloc: returns the status (callers test the rejection paths)."""
        return library().kq_mdagm_noalloc(self._h, prec, sigma, _ptr(src), _ptr(dst), parity, self._s(stream))

    def long_links_compressed(self, prec: int) -> int:
        """1: long links of prec stored as two rows + 1/s; 0: full storage; -1: not resident."""
        v = C.c_int()
        self._chk(library().kq_long_links_compressed(self._h, prec, C.byref(v)), "kq_long_links_compressed")
        return v.value

    def upload_full(self, prec: int, host: np.ndarray, dev, stream=None):
        """Full-lattice host record (even sites then odd sites, V*6 values) -> full-lattice device field."""
        h = np.ascontiguousarray(host)
        n = h.size // 2
        vb = self.spinor_bytes(prec)
        self.upload(prec, h[:n], dev[:vb], stream)
        self.upload(prec, h[n:], dev[vb:2 * vb], stream)

    def download_full(self, prec: int, dev, host_dtype=np.float64, stream=None) -> np.ndarray:
        vb = self.spinor_bytes(prec)
        return np.concatenate([self.download(prec, dev[:vb], host_dtype, stream),
                               self.download(prec, dev[vb:2 * vb], host_dtype, stream)])

    def dslash_full(self, prec: int, src, dst, stream=None):
        """kq_dslash_full: D on full-lattice fields (both parities, one launch)."""
        self._chk(library().kq_dslash_full(self._h, prec, _ptr(src), _ptr(dst), self._s(stream)), "kq_dslash_full")

    def mdagm_full(self, prec: int, sigma: float, src, dst, tmp, stream=None):
        self._chk(library().kq_mdagm_full(self._h, prec, sigma, _ptr(src), _ptr(dst), _ptr(tmp), self._s(stream)),
                  "kq_mdagm_full")

    @staticmethod
    def _param(shifts, parity, solver, prec, host_prec, max_iter, tol, rel_residual, shift_mode):
        sh = (C.c_double * len(shifts))(*[float(s) for s in shifts])
        p = SolveParam(parity=parity, num_shift=len(shifts), shifts=C.cast(sh, C.POINTER(C.c_double)),
                       shift_mode=shift_mode, solver=solver, prec=prec, host_prec=host_prec, max_iter=max_iter,
                       tol=tol, rel_residual=rel_residual)
        return p, sh

    def solve(self, b: np.ndarray, shifts, parity=0, solver=KQ_SOLVER_CGM, prec=KUQCD_DOUBLE, max_iter=10000,
              tol=0.0, rel_residual=1e-10, shift_mode=1, pinned=False):
        """Host b -> list of host x (dtype of b).  shift_mode 1: absolute shifts, 0: reference semantics.
        pinned: pass page-locked host buffers (the library then copies each solution out while the solve goes on)."""
        b = np.ascontiguousarray(b)
        if pinned:
            import torch
            tb = torch.from_numpy(b).pin_memory()
            tx = [torch.zeros(b.shape, dtype=tb.dtype).pin_memory() for _ in shifts]
            bp, xptrs = C.c_void_p(tb.data_ptr()), [t.data_ptr() for t in tx]
        else:
            xs = [np.zeros_like(b) for _ in shifts]
            bp, xptrs = _ptr(b), [x.ctypes.data for x in xs]
        p, keep = self._param(shifts, parity, solver, prec, _np_prec(b), max_iter, tol, rel_residual, shift_mode)
        info = SolveInfo()
        xp = (C.c_void_p * len(xptrs))(*xptrs)
        st = library().kq_solve_multishift(self._h, C.byref(p), bp, xp, C.byref(info))
        self._chk(st, "kq_solve_multishift")
        if pinned:
            xs = [t.numpy().copy() for t in tx]
        return xs, info

    def solve_device(self, d_b, d_x, shifts, parity=0, solver=KQ_SOLVER_CGM, prec=KUQCD_DOUBLE, max_iter=10000,
                     tol=0.0, rel_residual=1e-10, shift_mode=1):
        p, keep = self._param(shifts, parity, solver, prec, KUQCD_DOUBLE, max_iter, tol, rel_residual, shift_mode)
        info = SolveInfo()
        _torch_wait(self.device)
        self._chk(library().kq_solve_multishift_device(self._h, C.byref(p), _ptr(d_b), _ptr(d_x), C.byref(info)),
                  "kq_solve_multishift_device")
        return info

    def true_residuals(self, parity, sigmas, d_b, d_x):
        sg = (C.c_double * len(sigmas))(*[float(s) for s in sigmas])
        out = (C.c_double * len(sigmas))()
        _torch_wait(self.device)
        self._chk(library().kq_true_residuals(self._h, parity, len(sigmas), sg, _ptr(d_b), _ptr(d_x), out),
                  "kq_true_residuals")
        return list(out)

    def make_links(self, eps: float, seed: int, d_fat, d_long):
        _torch_wait(self.device)
        self._chk(library().kq_make_links_record(self._h, eps, seed, _ptr(d_fat), _ptr(d_long)),
                  "kq_make_links_record")

    def make_source(self, parity: int, seed: int, d_b):
        _torch_wait(self.device)
        self._chk(library().kq_make_source_record(self._h, parity, seed, _ptr(d_b)), "kq_make_source_record")


class Batch:
    """kq_batch: independent systems (each a Context with its own lattice and links) solved together."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = library().kq_batch_create(device, C.byref(h))
        if st != 0:
            raise KuQCDError(st, "kq_batch_create")
        self._h = h
        self._device = device
        self._keep = []

    def add(self, ctx: Context, d_b, d_x, shifts, parity=0, solver=KQ_SOLVER_MIXED, prec=KUQCD_HALF,
            rel_residual=1e-10, tol=0.0, max_iter=100000, shift_mode=1):
        p, sh = Context._param(shifts, parity, solver, prec, KUQCD_DOUBLE, max_iter, tol, rel_residual, shift_mode)
        self._keep.append((ctx, d_b, d_x, sh))
        st = library().kq_batch_add(self._h, ctx._h, C.byref(p), _ptr(d_b), _ptr(d_x))
        if st != 0:
            raise KuQCDError(st, "kq_batch_add")

    def solve(self) -> BatchInfo:
        info = BatchInfo()
        _torch_wait(self._device)
        st = library().kq_batch_solve(self._h, C.byref(info))
        if st != 0:
            raise KuQCDError(st, "kq_batch_solve")
        return info

    def system_info(self, i: int) -> SolveInfo:
        info = SolveInfo()
        st = library().kq_batch_system_info(self._h, i, C.byref(info))
        if st != 0:
            raise KuQCDError(st, "kq_batch_system_info")
        return info

    def close(self):
        if getattr(self, "_h", None):
            library().kq_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Net:
    """kq_net: the gauge-covariant parallel-transport convolution preconditioner of a context's lattice."""

    def __init__(self, ctx: Context, channels=(1, 8, 8)):
        h = C.c_void_p()
        ch = (C.c_int * len(channels))(*channels)
        st = library().kq_net_create(ctx._h, len(channels) - 1, ch, C.byref(h))
        if st != 0:
            raise KuQCDError(st, "kq_net_create")
        self._h = h
        self.ctx = ctx
        self.channels = tuple(channels)
        self.nw = int(library().kq_net_num_weights(h))

    def _chk(self, st, where):
        if st != 0:
            raise KuQCDError(st, where)

    @property
    def weights(self) -> np.ndarray:
        w = np.empty(self.nw, dtype=np.float32)
        self._chk(library().kq_net_get_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), self.nw), "get_w")
        return w

    @weights.setter
    def weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._chk(library().kq_net_set_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), w.size), "set_w")

    def grad(self) -> np.ndarray:
        g = np.empty(self.nw, dtype=np.float32)
        self._chk(library().kq_net_get_grad(self._h, g.ctypes.data_as(C.POINTER(C.c_float)), self.nw), "get_grad")
        return g

    def zero_grad(self):
        self._chk(library().kq_net_zero_grad(self._h), "zero_grad")

    def use_context(self, ctx: Context):
        self._chk(library().kq_net_set_context(self._h, ctx._h), "kq_net_set_context")
        self.ctx = ctx

    def apply(self, d_in, d_out, parity: int):
        _torch_wait(self.ctx.device)
        self._chk(library().kq_net_apply(self._h, _ptr(d_in), _ptr(d_out), parity), "kq_net_apply")

    def train_pair(self, d_r, d_e, parity: int, e_norm2: float) -> float:
        loss = C.c_double()
        _torch_wait(self.ctx.device)
        self._chk(library().kq_net_train_pair(self._h, _ptr(d_r), _ptr(d_e), parity, e_norm2, C.byref(loss)),
                  "kq_net_train_pair")
        return loss.value

    def adam(self, lr: float, grad_scale: float = 1.0):
        self._chk(library().kq_net_adam(self._h, lr, grad_scale), "kq_net_adam")

    def close(self):
        if getattr(self, "_h", None):
            library().kq_net_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fcg_polish(ctx: Context, net, d_b, d_x, shifts, parity=0, rel_residual=1e-10, max_iter=20000) -> SolveInfo:
    """kq_fcg_polish: drive every shift of d_x (initial guesses) to the FP64 true-residual target; net=None: CG."""
    p, keep = Context._param(shifts, parity, KQ_SOLVER_MIXED, KUQCD_DOUBLE, KUQCD_DOUBLE, max_iter, 0.0,
                             rel_residual, 1)
    info = SolveInfo()
    _torch_wait(ctx.device)
    st = library().kq_fcg_polish(ctx._h, net._h if net is not None else None, C.byref(p), _ptr(d_b), _ptr(d_x),
                                 C.byref(info))
    if st != 0:
        raise KuQCDError(st, "kq_fcg_polish")
    return info
