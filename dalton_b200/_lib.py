"""ctypes binding of libdgfock.so (the C ABI declared in include/dgfock.h).

The library is the product's only compute path: if it is missing or cannot be
loaded this module raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdgfock.so")

dgf_int = ctypes.c_int64
_ip = ctypes.POINTER(dgf_int)
_dp = ctypes.POINTER(ctypes.c_double)

DGF_OK, DGF_ERR_ARG, DGF_ERR_NOMEM, DGF_ERR_CUDA, DGF_ERR_UNSUPPORTED, DGF_ERR_TIMEOUT, DGF_ERR_NODEVICE = range(7)

# Every symbol include/dgfock.h declares.
EXPORTS = ["dgf_default_options", "dgf_create", "dgf_destroy", "dgf_fock", "dgf_fock_device", "dgf_grad2e",
           "dgf_grad2e_device", "dgf_grad2e_bilinear_device", "dgf_oneint", "dgf_grad1e", "dgf_set_profiling", "dgf_get_profile",
           "dgf_measure_fma_peak", "dgf_autotune", "dgf_info", "dgf_strerror", "dgf_last_error",
           "dgf_batch_create", "dgf_batch_destroy", "dgf_batch_layout", "dgf_fock_batch",
           "dgf_fock_device_noalloc", "dgf_count_ao_quartets", "dgf_copy_tuning", "dgf_set_class_kernel",
           "dgf_store_integrals", "dgf_fock_stored", "dgf_store_release"]


class DgfBasis(ctypes.Structure):
    _fields_ = [("nblock", dgf_int), ("natom", dgf_int), ("nbf", dgf_int), ("spherical", dgf_int),
                ("block_l", _ip), ("block_atom", _ip), ("block_nprim", _ip), ("block_ncontr", _ip),
                ("block_ao_offset", _ip), ("block_prim_offset", _ip), ("block_coef_offset", _ip),
                ("prim_exp", _dp), ("coef", _dp), ("atom_xyz", _dp), ("atom_charge", _dp)]


class DgfOptions(ctypes.Structure):
    _fields_ = [("thrs", ctypes.c_double), ("ifthrs", dgf_int), ("hfxfac", ctypes.c_double),
                ("mixed_cutoff", ctypes.c_double), ("shard_index", dgf_int), ("shard_count", dgf_int),
                ("icedif", dgf_int), ("hfxmu", ctypes.c_double), ("hfxatt", ctypes.c_double)]


class DgfStats(ctypes.Structure):
    _fields_ = [("quartets_total", ctypes.c_int64), ("quartets_fp64", ctypes.c_int64),
                ("quartets_fp32", ctypes.c_int64), ("quartets_skipped", ctypes.c_int64),
                ("prim_quartets", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("ms_device", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DgfClassTime(ctypes.Structure):
    _fields_ = [("la", ctypes.c_int32), ("lb", ctypes.c_int32), ("lc", ctypes.c_int32), ("ld", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("kernel", ctypes.c_int32), ("quartets", ctypes.c_int64),
                ("evaluated", ctypes.c_int64), ("prim_quartets", ctypes.c_int64), ("ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class DgfError(RuntimeError):
    def __init__(self, status, where, detail=""):
        super().__init__(f"{where}: status {status} ({strerror(status)}) {detail}".strip())
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Load libdgfock.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libdgfock.so not built ({LIB_PATH}); run `python -m dalton_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    lib.dgf_default_options.argtypes = [ctypes.POINTER(DgfOptions)]
    lib.dgf_default_options.restype = None
    lib.dgf_create.argtypes = [ctypes.POINTER(DgfBasis), ctypes.c_int, ctypes.POINTER(vp)]
    lib.dgf_destroy.argtypes = [vp]
    lib.dgf_destroy.restype = None
    lib.dgf_fock.argtypes = [vp, dgf_int, _ip, _dp, _dp, ctypes.POINTER(DgfOptions), ctypes.POINTER(DgfStats)]
    lib.dgf_fock_device.argtypes = [vp, dgf_int, _ip, vp, vp, ctypes.POINTER(DgfOptions), vp,
                                    ctypes.POINTER(DgfStats)]
    lib.dgf_grad2e.argtypes = [vp, _dp, ctypes.c_double, ctypes.c_double, _dp]
    lib.dgf_grad2e_device.argtypes = [vp, vp, ctypes.c_double, ctypes.c_double, vp, vp]
    lib.dgf_grad2e_bilinear_device.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_double, vp, vp]
    lib.dgf_oneint.argtypes = [vp, _dp, _dp, _dp]
    lib.dgf_grad1e.argtypes = [vp, _dp, _dp, _dp]
    lib.dgf_info.argtypes = [vp, _ip, _ip, _ip]
    lib.dgf_count_ao_quartets.argtypes = [vp, ctypes.c_double, _ip]
    lib.dgf_copy_tuning.argtypes = [vp, vp]
    lib.dgf_set_class_kernel.argtypes = [vp] + [ctypes.c_int] * 6
    lib.dgf_store_integrals.argtypes = [vp, ctypes.c_double, ctypes.c_int64, vp, ctypes.POINTER(ctypes.c_int64)]
    lib.dgf_fock_stored.argtypes = [vp, dgf_int, _ip, vp, vp, ctypes.POINTER(DgfOptions), vp, ctypes.POINTER(DgfStats)]
    lib.dgf_store_release.argtypes = [vp]
    lib.dgf_set_profiling.argtypes = [vp, ctypes.c_int]
    lib.dgf_get_profile.argtypes = [vp, ctypes.POINTER(DgfClassTime), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.dgf_measure_fma_peak.argtypes = [ctypes.c_int, _dp, _dp]
    lib.dgf_autotune.argtypes = [vp, vp, ctypes.POINTER(DgfOptions), vp, ctypes.c_char_p, ctypes.c_size_t]
    lib.dgf_strerror.argtypes = [ctypes.c_int]
    lib.dgf_strerror.restype = ctypes.c_char_p
    lib.dgf_last_error.argtypes = []
    lib.dgf_last_error.restype = ctypes.c_char_p
    lib.dgf_batch_create.argtypes = [ctypes.POINTER(vp), dgf_int, ctypes.POINTER(vp)]
    lib.dgf_batch_destroy.argtypes = [vp]
    lib.dgf_batch_destroy.restype = None
    lib.dgf_batch_layout.argtypes = [vp, _ip]
    lib.dgf_fock_batch.argtypes = [vp, vp, vp, ctypes.POINTER(DgfOptions), ctypes.c_int, vp,
                                   ctypes.POINTER(DgfStats)]
    _lib = lib
    return lib


def strerror(status: int) -> str:
    try:
        return load().dgf_strerror(int(status)).decode()
    except Exception:  # noqa: BLE001 - message helper must not raise
        return "unknown"


def last_error() -> str:
    return load().dgf_last_error().decode()


def check(status: int, where: str):
    if status != DGF_OK:
        raise DgfError(status, where, last_error())


def default_options(**kw) -> DgfOptions:
    o = DgfOptions()
    load().dgf_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if v is not None:
            setattr(o, k, v)
    return o


def measure_fma_peak(device: int = 0):
    """(FP64, FP32) FMA throughput in TFLOP/s measured on `device`."""
    a, b = ctypes.c_double(), ctypes.c_double()
    check(load().dgf_measure_fma_peak(int(device), ctypes.byref(a), ctypes.byref(b)), "dgf_measure_fma_peak")
    return a.value, b.value
