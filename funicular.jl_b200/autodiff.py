"""Reverse-mode rules for the device-resident panel algebra: the counterpart
of the ChainRulesCore.rrule methods the north-star backend adds to Funicular
(the reference has none; Project.toml:6-9 has no ChainRulesCore).

`rrule(f, args...)` follows ChainRulesCore's contract: it returns the
primal result and a pullback that maps the output cotangent to the input
cotangents, or None when there is no rule. The rules take device matrices
(the resident fast path; a PanelMatrix is uploaded first by the caller), do
not mutate their inputs, and hold what their pullbacks need:

- rrule(cholqr2, Y) -> ((Q, R), pullback); pullback(Qbar, Rbar) -> Ybar.
  The pullback keeps the ORIGINAL Y and R, not Q: Q is recomputed as Y R^-1
  inside the adjoint kernel's products (fb_zcholqr2_adjoint). Y must not be
  changed between the two calls.
- rrule(project, Q, G) -> (S, pullback); pullback(Sbar) -> (Qbar, None), the
  operator getting no tangent. The pullback keeps G Q from the forward pass
  and applies G^H to Q only when G is not Hermitian.

Cotangents are device matrices or None (a zero tangent). Each pullback takes
`into=`: a device matrix the cotangent is written to (cholqr2; it may be
Qbar itself) or accumulated into (project), so a chain of rules needs no
extra N x k buffers or additions.
"""
from __future__ import annotations

import numpy as np

from . import kernels
from ._lib import ArgumentError, DimensionMismatch
from .device_api import DeviceMatrix, copy_region
from .panelblas import DeviceOperator, apply_operator, assert_square_operator, cholqr2, project


def _device_copy(backend, A: DeviceMatrix) -> DeviceMatrix:
    out = backend.alloc_device(A.dtype, A.shape)
    copy_region(out, A, backend.current_queue)
    return out


def rrule_cholqr2(backend, Y: DeviceMatrix, form: str = "fp64"):
    """(Q, R) = cholqr2!(copy(Y)) and its pullback."""
    if not isinstance(Y, DeviceMatrix):
        raise ArgumentError(f"the cholqr2! rule takes a device-resident matrix, got {type(Y).__name__}")
    N, k = Y.shape
    Q = _device_copy(backend, Y)
    R = backend.alloc_device(np.complex128, (k, k))
    kernels.cholqr2_resident(backend, Q, R, wait=True, form=form)

    def pullback(Qbar: DeviceMatrix | None, Rbar: DeviceMatrix | None = None, *, into: DeviceMatrix | None = None):
        if Qbar is None and Rbar is None:
            return None
        Ybar = into if into is not None else backend.alloc_device(np.complex128, (N, k))
        return kernels.cholqr2_adjoint(backend, Ybar, Y, R, Qbar, Rbar)

    return (Q, R), pullback


def rrule_project(backend, Q: DeviceMatrix, G: DeviceOperator):
    """S = Q^H (G Q) (project on a resident matrix) and its pullback."""
    if not isinstance(Q, DeviceMatrix):
        raise ArgumentError(f"the project rule takes a device-resident matrix, got {type(Q).__name__}")
    N, k = Q.shape
    assert_square_operator(G, N)
    GQ = backend.alloc_device(np.complex128, (N, k))
    apply_operator(backend, GQ, G, Q)
    S = backend.alloc_device(np.complex128, (k, k))
    kernels.gram_accumulate(backend, S, Q, GQ, 1.0, 0.0)

    def pullback(Sbar: DeviceMatrix | None, *, into: DeviceMatrix | None = None):
        if Sbar is None:
            return None, None
        if Sbar.shape != (k, k):
            raise DimensionMismatch(f"Sbar must be {k}x{k}, got {Sbar.shape}")
        GhQ = None
        if not G.hermitian:
            GhQ = backend.alloc_device(np.complex128, (N, k))
            apply_operator(backend, GhQ, G.adjoint(), Q)
        accumulate = into is not None
        Qbar = into if accumulate else backend.alloc_device(np.complex128, (N, k))
        kernels.project_adjoint(backend, Qbar, GQ, Sbar, GhQ, accumulate=accumulate)
        return Qbar, None

    return S, pullback


def rrule(f, *args, backend=None, **kwargs):
    """ChainRulesCore.rrule(f, args...) for f in (cholqr2, project) on device
    matrices; None for any other function (no rule)."""
    if f is cholqr2 or f is rrule_cholqr2:
        (Y,) = args
        return rrule_cholqr2(backend or _backend_of(Y), Y, **kwargs)
    if f is project or f is rrule_project:
        Q, G = args
        return rrule_project(backend or _backend_of(Q), Q, G)
    return None


def _backend_of(A) -> object:
    from .device_api import b200_backend
    return getattr(A, "backend", None) or b200_backend()
