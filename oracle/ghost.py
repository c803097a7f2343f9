"""Test infrastructure only: ctypes access to the C restatement of the
GhostPanels entries (ghost_oracle.c), built by this directory's Makefile.
The tests compare the device fill against it bit for bit. Nothing in the
product imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libghost_oracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        lib = ctypes.CDLL(_LIB_PATH)
        lib.ghost_oracle_fill.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                          ctypes.c_int64, ctypes.c_int64, ctypes.c_uint64, ctypes.c_int, ctypes.c_int]
        lib.ghost_oracle_fill.restype = None
        lib.ghost_oracle_philox.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ghost_oracle_philox.restype = None
        lib.ghost_oracle_ln.argtypes = [ctypes.c_double]
        lib.ghost_oracle_ln.restype = ctypes.c_double
        lib.ghost_oracle_cos_sin_2pi.argtypes = [ctypes.c_double, ctypes.c_void_p]
        lib.ghost_oracle_cos_sin_2pi.restype = None
        _lib = lib
    return _lib


def philox4x32_10(ctr, key):
    out = (ctypes.c_uint32 * 4)()
    load().ghost_oracle_philox(out, (ctypes.c_uint32 * 4)(*ctr), (ctypes.c_uint32 * 2)(*key))
    return tuple(int(v) for v in out)


def ln(x: float) -> float:
    return load().ghost_oracle_ln(x)


def cos_sin_2pi(u: float):
    out = (ctypes.c_double * 2)()
    load().ghost_oracle_cos_sin_2pi(u, out)
    return out[0], out[1]


def ghost_block(dtype, rows: int, cols: int, row0: int, col0: int, seed: int, value_dtype=None) -> np.ndarray:
    """The rows x cols block at (row0, col0) of the ghost matrix with `seed`,
    its values rounded to value_dtype (default: dtype), returned in dtype."""
    dtype = np.dtype(dtype)
    value_dtype = dtype if value_dtype is None else np.dtype(value_dtype)
    is_complex = dtype.kind == "c"
    narrow = value_dtype.itemsize < (16 if is_complex else 8)
    buf = np.empty((rows, cols), dtype=np.complex128 if is_complex else np.float64, order="F")
    if rows and cols:
        load().ghost_oracle_fill(buf.ctypes.data, rows, rows, cols, row0, col0, int(seed) & 0xFFFFFFFFFFFFFFFF,
                                 int(is_complex), int(narrow))
    return buf.astype(dtype)
