"""ctypes binding of libfunicular_b200.so, the C ABI declared in
include/funicular_b200.h.

This is the Python counterpart of the `ccall` shim a Julia package extension
would hold: every function here is one C entry point, status codes become the
exceptions the reference raises (ArgumentError for bad arguments and refused
factorizations, DimensionMismatch for shapes), and nothing computes on the
host. There is no fallback: if the shared library is missing the import
fails, naming the build command.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY_PATH = os.path.join(_HERE, "libfunicular_b200.so")

FB_OK, FB_EINVAL, FB_EDIM, FB_ENOMEM, FB_ENOTSPD, FB_ECUDA, FB_ENOTSUP = range(7)
FB_C128, FB_C64, FB_F64, FB_F32 = range(4)


class ArgumentError(ValueError):
    """Raised where the reference raises ArgumentError."""


class DimensionMismatch(ValueError):
    """Raised where the reference raises DimensionMismatch."""


class NotPositiveDefinite(ArgumentError):
    """The Gram matrix stayed indefinite after the shift (src/panelblas.jl:153)."""


class DeviceError(RuntimeError):
    """The CUDA runtime reported an error."""


class OutOfDeviceMemory(ArgumentError):
    """An allocation or a workspace did not fit."""


_EXCEPTIONS = {
    FB_EINVAL: ArgumentError,
    FB_EDIM: DimensionMismatch,
    FB_ENOMEM: OutOfDeviceMemory,
    FB_ENOTSPD: NotPositiveDefinite,
    FB_ECUDA: DeviceError,
    FB_ENOTSUP: ArgumentError,
}


class Z128(ctypes.Structure):
    _fields_ = [("re", ctypes.c_double), ("im", ctypes.c_double)]


def z128(x) -> Z128:
    x = complex(x)
    return Z128(x.real, x.imag)


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int
_sz = ctypes.c_size_t
_pint = ctypes.POINTER(ctypes.c_int)
_pdbl = ctypes.POINTER(ctypes.c_double)
_psz = ctypes.POINTER(ctypes.c_size_t)
_pvp = ctypes.POINTER(ctypes.c_void_p)

# name -> argument types (every function returns int unless listed in _RESTYPES)
SIGNATURES = {
    "fb_abi_version": [],
    "fb_last_error": [],
    "fb_kernel_launches": [],
    "fb_device_count": [_pint],
    "fb_set_device": [_int],
    "fb_alloc_device": [_pvp, _sz],
    "fb_free_device": [_vp],
    "fb_alloc_host_slab": [_pvp, _sz],
    "fb_free_host_slab": [_vp],
    "fb_pin_host": [_vp, _sz],
    "fb_unpin_host": [_vp],
    "fb_queue_create": [_pvp],
    "fb_queue_destroy": [_vp],
    "fb_event_record": [_vp, _pvp],
    "fb_event_destroy": [_vp],
    "fb_queue_wait_event": [_vp, _vp],
    "fb_queue_sync": [_vp],
    "fb_event_sync": [_vp],
    "fb_event_query": [_vp, _pint],
    "fb_sync_all": [],
    "fb_copy2d": [_vp, _sz, _vp, _sz, _sz, _sz, _vp],
    "fb_convert_copy": [_vp, _int, _i64, _vp, _int, _i64, _i64, _i64, _vp],
    "fb_zgram_workspace_size": [_i64, _int, _int, _int, _psz],
    "fb_zgram": [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _int, _int, Z128, Z128, _vp, _sz, _vp],
    "fb_zgram_static": [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _int, _int, Z128, Z128, _vp],
    "fb_ztrsm_workspace_size": [_int, _psz],
    "fb_ztrsm_right_upper": [_vp, _i64, _i64, _int, _vp, _i64, _vp, _sz, _vp],
    "fb_zgemm_right": [_vp, _i64, _vp, _i64, _i64, _int, _vp, _i64, _int, _vp],
    "fb_zpotrf_workspace_size": [_int, _psz],
    "fb_zpotrf_shifted": [_vp, _i64, _vp, _i64, _int, _i64, _vp, _i64, _vp, _i64, _pint, _pdbl, _vp, _sz, _vp],
    "fb_zcholqr2_workspace_size": [_i64, _int, _psz],
    "fb_zcholqr2": [_vp, _i64, _i64, _int, _vp, _i64, _pint, _pint, _vp, _sz, _vp],
    "fb_zcholqr2_query": [_vp, _pint, _pint, _pdbl],
    "fb_zcholqr2_staged_blocks": [_i64, _int, _pint],
    "fb_zcholqr2_staged_workspace_size": [_i64, _int, _int, _psz],
    "fb_zcholqr2_staged": [_vp, _int, _vp, _vp, _int, _vp, _i64, _i64, _int, _vp, _i64, ctypes.c_double, _pint,
                           _pint, _vp, _sz, _vp],
    "fb_zcholqr2_tc": [_vp, _i64, _i64, _int, _vp, _i64, _pint, _pint, _vp, _sz, _vp],
    "fb_zgram_tc_workspace_size": [_i64, _int, _psz],
    "fb_zgram_tc": [_vp, _i64, _vp, _i64, _i64, _int, Z128, Z128, _vp, _sz, _vp],
    "fb_zlaplace7_apply": [_vp, _i64, _vp, _i64, _int, _int, _int, _int, Z128, _vp],
    "fb_graph_capture_begin": [_vp],
    "fb_graph_capture_end": [_vp, _pvp],
    "fb_graph_launch": [_vp, _vp],
    "fb_graph_destroy": [_vp],
    "fb_zcholqr2_batched_workspace_size": [_vp, _vp, _int, _psz],
    "fb_zcholqr2_batched": [_vp, _vp, _vp, _vp, _vp, _vp, _int, _int, _vp, _sz, _vp],
    "fb_zcholqr2_batched_query": [_vp, _int, _vp, _vp],
    "fb_zcholqr2_batched_persistent_workspace_size": [_vp, _vp, _int, _psz],
    "fb_zcholqr2_batched_persistent": [_vp, _vp, _vp, _vp, _vp, _vp, _int, _vp, _sz, _vp],
    "fb_ghost_fill": [_vp, _int, _i64, _i64, _i64, _i64, _i64, ctypes.c_uint64, _int, _vp],
    "fb_zcholqr2_adjoint_workspace_size": [_i64, _int, _psz],
    "fb_zcholqr2_adjoint": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _int, _vp, _sz, _vp],
    "fb_zproject_adjoint_workspace_size": [_int, _psz],
    "fb_zproject_adjoint": [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _i64, _int, _int, _vp, _sz, _vp],
    "fb_zhband_apply": [_vp, _i64, _vp, _i64, _vp, _i64, _i64, _int, _int, _vp],
    "fb_tune_set_gram_chunks": [_i64, _int, _int],
    "fb_tune_get_gram_chunks": [_i64, _int, _pint],
    "fb_tune_clear": [],
    "fb_tune_set_batch_lanes": [_int],
    "fb_tune_get_batch_lanes": [_pint],
    "fb_zcholqr3_shifted": [_vp, _i64, _i64, _int, _vp, _i64, ctypes.c_double, _pint, _pint, _vp, _sz, _vp],
    "fb_zpotrf_forced_shift": [_vp, _i64, _vp, _i64, _int, _i64, _vp, _i64, _vp, _i64, ctypes.c_double, _pdbl,
                               _vp, _sz, _vp],
}
_RESTYPES = {"fb_last_error": ctypes.c_char_p, "fb_abi_version": ctypes.c_int,
             "fb_kernel_launches": ctypes.c_uint64}

_lock = threading.Lock()
_lib = None


def load() -> ctypes.CDLL:
    """The loaded library, with argument types set. Raises ImportError if it
    has not been built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIBRARY_PATH):
            raise ImportError(
                f"{LIBRARY_PATH} is missing: build it with `make -C {os.path.join(_HERE, 'csrc')}` "
                "(or __graft_entry__.build()). There is no CPU fallback.")
        lib = ctypes.CDLL(LIBRARY_PATH, mode=ctypes.RTLD_GLOBAL)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = lib
        return lib


def last_error() -> str:
    return load().fb_last_error().decode(errors="replace")


def check(status: int, what: str = "") -> None:
    """Turns a non-zero status into the matching exception."""
    if status == FB_OK:
        return
    exc = _EXCEPTIONS.get(status, DeviceError)
    msg = last_error()
    raise exc(f"{what}: {msg}" if what else msg)


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def kernel_launches() -> int:
    """Kernels the library has launched in this process."""
    return int(load().fb_kernel_launches())


def staged_blocks(N: int, k: int) -> int:
    """Row blocks fb_zcholqr2_staged moves an N x k matrix in."""
    n = ctypes.c_int(0)
    call("fb_zcholqr2_staged_blocks", ctypes.c_int64(N), k, ctypes.byref(n))
    return n.value


def device_count() -> int:
    n = ctypes.c_int(0)
    call("fb_device_count", ctypes.byref(n))
    return n.value
