"""funicular_b200: the B200 device backend of Funicular's panel linear
algebra, driven from Python the way Funicular.jl drives a backend.

`device_api` and `kernels` are the backend proper: the device API of
src/device_api.jl and the kernel overrides of src/kernels.jl, each a thin call
into libfunicular_b200.so (C ABI in include/funicular_b200.h). The remaining
modules restate the host layers that call a backend (plan, panels, executor,
panel BLAS, ghosts) so that the backend runs under the same call sequences as
in Funicular.jl.
"""
from ._lib import (ArgumentError, DeviceError, DimensionMismatch, NotPositiveDefinite,
                   OutOfDeviceMemory, LIBRARY_PATH)
from . import _lib
from .device_api import B200Backend, DeviceMatrix, HostSlab, b200_backend
from . import kernels

__all__ = ["ArgumentError", "DimensionMismatch", "NotPositiveDefinite", "DeviceError",
           "OutOfDeviceMemory", "B200Backend", "DeviceMatrix", "HostSlab", "b200_backend",
           "kernels", "LIBRARY_PATH"]
