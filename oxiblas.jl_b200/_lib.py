"""ctypes binding of liboxiblas_b200.so (the C ABI declared in include/oxiblas_b200.h).

The shared library is the product: if it is missing or cannot be loaded the
import fails loudly -- there is no CPU or eager fallback anywhere in this
package.  Status codes are mapped to the exceptions the reference raises
(src/lapack/factorizations.jl, src/api/linalg_api.jl).
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboxiblas_b200.so")

OXI_OK, OXI_EINVAL, OXI_ESINGULAR, OXI_ENONFINITE, OXI_EOVERFLOW = 0, 1, 2, 3, 4
OXI_ECUDA, OXI_ETIMEOUT, OXI_ENOMEM, OXI_ENOTCONVERGED = 5, 6, 7, 8
OXI_ESCRATCH = 9
OXI_ENOTPOSDEF = 10
OPT_BLOCKSIZE, OPT_GEMM, OPT_TRSM_LEAF, OPT_LOOKAHEAD = 1, 2, 3, 4
OPT_MIXED_BLOCKSIZE, OPT_STOP_NORMWISE, OPT_GMRES_RESTART = 5, 6, 7
OPT_GRAPHS, OPT_TOURNAMENT = 8, 9
OPT_WAIT_LIMIT_US, OPT_TEST_MISSING_PRODUCER = 10, 11


class SingularException(Exception):
    """LinearAlgebra.SingularException(info): zero pivot at 1-based column info."""

    def __init__(self, info: int):
        super().__init__(f"SingularException({info})")
        self.info = int(info)


class DimensionMismatch(ValueError):
    pass


class ArgumentError(ValueError):
    pass


class ExtensionMissing(ImportError):
    pass


_i64 = ctypes.c_int64
_vp = ctypes.c_void_p
_lib = None
_lock = threading.Lock()

_SIGS = {
    "oxi_create": ([ctypes.POINTER(_vp)], ctypes.c_int),
    "oxi_destroy": ([_vp], ctypes.c_int),
    "oxi_set_stream": ([_vp, _vp], ctypes.c_int),
    "oxi_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "oxi_last_error": ([_vp], ctypes.c_char_p),
    "oxi_set_option": ([_vp, ctypes.c_int, _i64], ctypes.c_int),
    "oxi_get_option": ([_vp, ctypes.c_int, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_dgetrf": ([_vp, _i64, _i64, _vp, _i64, _vp, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_sgetrf": ([_vp, _i64, _i64, _vp, _i64, _vp, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_dgetrs": ([_vp, ctypes.c_char, _i64, _i64, _vp, _i64, _vp, _vp, _i64], ctypes.c_int),
    "oxi_sgetrs": ([_vp, ctypes.c_char, _i64, _i64, _vp, _i64, _vp, _vp, _i64], ctypes.c_int),
    "oxi_dgetrs_noalloc": ([_vp, ctypes.c_char, _i64, _i64, _vp, _i64, _vp, _vp, _i64], ctypes.c_int),
    "oxi_dlu_adjoint": ([_vp, _i64, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64],
                        ctypes.c_int),
    "oxi_dlu_adjoint_batched_uneven": ([_vp, _i64] + [_vp] * 14, ctypes.c_int),
    "oxi_dgetrf_batched_uneven": ([_vp, _i64, _vp, _vp, _vp, _vp, _vp], ctypes.c_int),
    "oxi_dgesv_batched_uneven": ([_vp, ctypes.c_int, _i64, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                  _vp, _vp, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "oxi_batched_autotune": ([_vp, ctypes.c_int, _i64, _vp, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)],
                             ctypes.c_int),
    "oxi_batched_get_tuning": ([_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)],
                               ctypes.c_int),
    "oxi_batched_set_tuning": ([_vp, ctypes.c_int, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "oxi_dgemm_update": ([_vp, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64], ctypes.c_int),
    "oxi_sgemm_update_lowp": ([_vp, ctypes.c_int, _i64, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64],
                              ctypes.c_int),
    "oxi_profile_enable": ([_vp, ctypes.c_int], ctypes.c_int),
    "oxi_profile_timeline": ([_vp, _i64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_profile_read": ([_vp, ctypes.c_int, ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_double),
                          ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "oxi_launch_count": ([_vp, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_launch_count_reset": ([_vp], ctypes.c_int),
    "oxi_dexpert_solve": ([_vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64, ctypes.c_int, ctypes.c_double,
                           ctypes.c_int, _vp, _vp, _vp, _i64, _vp, _vp], ctypes.c_int),
    "oxi_drefine_solve": ([_vp, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _i64, ctypes.c_int,
                           ctypes.c_double, _vp], ctypes.c_int),
    "oxi_dinverse_norm_estimate": ([_vp, _i64, _vp, _i64, _vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)],
                                   ctypes.c_int),
    "oxi_dgetri": ([_vp, _i64, _vp, _i64, _vp, _vp, _i64], ctypes.c_int),
    "oxi_dpotrf": ([_vp, _i64, _vp, _i64, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_dpotrs": ([_vp, _i64, _i64, _vp, _i64, _vp, _i64], ctypes.c_int),
    "oxi_transpose": ([_vp, ctypes.c_int, _i64, _i64, _vp, _i64, _vp, _i64], ctypes.c_int),
    "oxi_zgetrf": ([_vp, _i64, _i64, _vp, _i64, _vp, ctypes.POINTER(_i64)], ctypes.c_int),
    "oxi_zgetrs": ([_vp, ctypes.c_char, _i64, _i64, _vp, _i64, _vp, _vp, _i64], ctypes.c_int),
    "oxi_dequilibrate": ([_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i64], ctypes.c_int),
    "oxi_dgesv_mixed": ([_vp, ctypes.c_int, ctypes.c_int, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64,
                         ctypes.c_int, ctypes.c_double, _vp], ctypes.c_int),
    "oxi_dposv_mixed": ([_vp, ctypes.c_int, ctypes.c_int, _i64, _i64, _vp, _i64, _vp, _i64, _vp, _i64,
                         ctypes.c_int, ctypes.c_double, _vp], ctypes.c_int),
}


def exported_symbols():
    """Names of the C ABI entry points this binding declares."""
    return list(_SIGS)


def load():
    """Load the shared library (once).  Raises ExtensionMissing when absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ExtensionMissing(
                f"{LIB_PATH} is not built; run `python oxiblas.jl_b200/build_lib.py` "
                "(or __graft_entry__.build()) -- there is no fallback implementation")
        L = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.argtypes = args
            f.restype = res
        _lib = L
        return L


class Handle:
    """One oxi_handle_t per (thread, device); bound to torch's current stream
    at each call, so work is ordered with the caller's torch operations."""

    _tls = threading.local()

    def __init__(self):
        L = load()
        h = _vp()
        st = L.oxi_create(ctypes.byref(h))
        if st != OXI_OK:
            raise RuntimeError(f"oxi_create failed: {L.oxi_status_string(st).decode()}")
        self.ptr = h
        self.lib = L

    @classmethod
    def get(cls, device=None):
        import torch
        dev = torch.cuda.current_device() if device is None else int(device)
        cache = getattr(cls._tls, "handles", None)
        if cache is None:
            cache = cls._tls.handles = {}
        h = cache.get(dev)
        if h is None:
            with torch.cuda.device(dev):
                h = cache[dev] = Handle()
        stream = torch.cuda.current_stream(dev).cuda_stream
        h.lib.oxi_set_stream(h.ptr, _vp(stream))
        return h

    def set_option(self, opt: int, value: int):
        self.check(self.lib.oxi_set_option(self.ptr, opt, int(value)))

    def get_option(self, opt: int) -> int:
        v = _i64(0)
        self.check(self.lib.oxi_get_option(self.ptr, opt, ctypes.byref(v)))
        return int(v.value)

    KERNEL_CLASSES = ("leaf", "rowmoves", "trsm_leaf", "gemm_ref", "gemm_dmma", "gemm_tc", "convert",
                      "trsv", "residual", "other")

    def profile(self, on: bool):
        self.check(self.lib.oxi_profile_enable(self.ptr, 1 if on else 0))

    def profile_read(self):
        """{class: (timed launches, total ms, flops, bytes)} for the enabled window."""
        out = {}
        for k, name in enumerate(self.KERNEL_CLASSES):
            c, ms, fl, by = _i64(0), ctypes.c_double(0), ctypes.c_double(0), ctypes.c_double(0)
            self.check(self.lib.oxi_profile_read(self.ptr, k, ctypes.byref(c), ctypes.byref(ms),
                                                 ctypes.byref(fl), ctypes.byref(by)))
            if c.value:
                out[name] = (int(c.value), ms.value, fl.value, by.value)
        return out

    def profile_timeline(self, max_records: int = 1 << 16):
        """[(class, stream index, start ms, end ms)] of the profiled launches."""
        buf = (ctypes.c_double * (4 * max_records))()
        cnt = _i64(0)
        self.check(self.lib.oxi_profile_timeline(self.ptr, max_records, buf, ctypes.byref(cnt)))
        n = min(int(cnt.value), max_records)
        return [(self.KERNEL_CLASSES[int(buf[4 * i])], int(buf[4 * i + 1]), buf[4 * i + 2], buf[4 * i + 3])
                for i in range(n)]

    def launches(self) -> int:
        v = _i64(0)
        self.check(self.lib.oxi_launch_count(self.ptr, ctypes.byref(v)))
        return int(v.value)

    def reset_launches(self):
        self.check(self.lib.oxi_launch_count_reset(self.ptr))

    def check(self, status: int, info: int = 0):
        if status == OXI_OK:
            return
        L = self.lib
        msg = L.oxi_status_string(status).decode()
        if status == OXI_ESINGULAR:
            raise SingularException(info)
        if status == OXI_EINVAL:
            raise ArgumentError(msg)
        if status in (OXI_ENONFINITE,):
            raise ArgumentError("finite mixed input required")
        if status == OXI_EOVERFLOW:
            raise OverflowError(msg)
        if status == OXI_ETIMEOUT:
            raise TimeoutError(msg)
        if status == OXI_ENOMEM:
            raise MemoryError(msg)
        err = L.oxi_last_error(self.ptr).decode()
        raise RuntimeError(f"{msg}: {err}")
