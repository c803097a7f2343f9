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
from .plan import (GiB, ResidencyPlan, choose_panel_width, row_block_height, device_bytes_allocated,
                   host_bytes_reserved, host_bytes_in_use, host_bytes_free)
from .panels import PanelMatrix, free
from .executor import (sweep, foreachpanel, readpanels, writepanels, updatepanels, PanelSteps, RowSteps,
                       rowtraversal)
from .panelblas import (gram, panelmul, cholqr2, cholqr3, project, rightmul, DenseOperator, ColumnOperator,
                        DeviceOperator, Laplacian7, HermitianBand, cholesky_upper)
from .ghosts import GhostPanels, isghost
from . import autodiff
from .autodiff import rrule
from . import autotune

__all__ = ["ArgumentError", "DimensionMismatch", "NotPositiveDefinite", "DeviceError",
           "OutOfDeviceMemory", "B200Backend", "DeviceMatrix", "HostSlab", "b200_backend",
           "kernels", "LIBRARY_PATH", "GiB", "ResidencyPlan", "choose_panel_width", "row_block_height",
           "device_bytes_allocated", "host_bytes_reserved", "host_bytes_in_use", "host_bytes_free",
           "PanelMatrix", "free", "sweep", "foreachpanel", "readpanels", "writepanels", "updatepanels",
           "PanelSteps", "RowSteps", "rowtraversal", "gram", "panelmul", "cholqr2", "cholqr3", "project", "rightmul",
           "DenseOperator", "ColumnOperator", "DeviceOperator", "Laplacian7", "HermitianBand", "cholesky_upper", "GhostPanels", "isghost",
           "autodiff", "rrule", "autotune"]
