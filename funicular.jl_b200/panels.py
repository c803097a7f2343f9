"""Panels and panel matrices, and their movement between the host tier and the
device (src/panels.jl).

A PanelMatrix is N x k, cut into column panels of width w with a ragged last
one (src/panels.jl:24-92). Each panel lives in a block of page-locked host
memory from the plan's pool, unless it is a ghost panel, whose values are a
function of the seed and the column index and are generated where they are
needed. Movement is one pitched 2-D copy per panel, or per panel slice for a
block of rows (src/panels.jl:373-458); a narrowed host eltype crosses the bus
narrow and is widened on the device by convert_copy (src/panels.jl:365-371).
"""
from __future__ import annotations

import numpy as np

from . import kernels
from ._lib import ArgumentError, DimensionMismatch
from .device_api import DeviceMatrix, copy_region
from .plan import (ResidencyPlan, alloc_host_storage, panel_bytes, release_host_block, resolve_panel_width)


class Panel:
    """One column panel (src/panels.jl:1-12)."""

    __slots__ = ("data", "home", "width", "dirty", "epoch", "pins", "hold")

    def __init__(self, data, home, width):
        self.data = data          # HostStorage, or None for a ghost panel or a released one
        self.home = home          # GhostHome for a ghost panel, else None
        self.width = width
        self.dirty = False
        self.epoch = 0
        self.pins = 0
        self.hold = None          # event the last copies touching the panel finish on

    def storage(self) -> np.ndarray:
        return self.data.array


def host_storage_eltype(plan: ResidencyPlan, dtype) -> np.dtype:
    """host_storage_eltype (src/panels.jl:94-101)."""
    dtype = np.dtype(dtype)
    if plan.host_eltype is None:
        return dtype
    S = plan.host_eltype
    if dtype.kind == "c" and S.kind != "c":
        raise ArgumentError(f"host_eltype {S} cannot hold the imaginary part of a {dtype} panel. Narrowing a complex "
                            "compute eltype means a narrower complex one")
    return S


class PanelMatrix:
    """PanelMatrix{T}(undef, N, k; plan, w) and PanelMatrix(A; plan, w)
    (src/panels.jl:24-92). Not an array: collect it with to_array()."""

    def __init__(self, N: int, k: int, w: int, panels, plan: ResidencyPlan, dtype, ghost=None):
        self.N, self.k, self.w = int(N), int(k), int(w)
        self.panels = panels
        self.plan = plan
        self.dtype = np.dtype(dtype)
        self.ghost = ghost

    @classmethod
    def undef(cls, dtype, N: int, k: int, *, plan: ResidencyPlan, w=None) -> "PanelMatrix":
        dtype = np.dtype(dtype)
        if N <= 0:
            raise ArgumentError(f"N must be positive, got {N}")
        if k <= 0:
            raise ArgumentError(f"k must be positive, got {k}")
        width = resolve_panel_width(plan, N, k, dtype, override=w)
        S = host_storage_eltype(plan, dtype)
        blockbytes = panel_bytes(N, width, S)
        panels = []
        try:
            for j in range(-(-k // width)):
                cols = min((j + 1) * width, k) - j * width
                panels.append(Panel(alloc_host_storage(plan, S, (N, cols), blockbytes), None, cols))
        except BaseException:
            for p in panels:
                release_host_block(plan, p.data.block)
            raise
        return cls(N, k, width, panels, plan, dtype)

    @classmethod
    def from_array(cls, A, *, plan: ResidencyPlan, w=None) -> "PanelMatrix":
        A = np.asarray(A)
        if A.ndim != 2:
            raise ArgumentError("a PanelMatrix is built from a two-dimensional array")
        pm = cls.undef(A.dtype, A.shape[0], A.shape[1], plan=plan, w=w)
        pm.copy_from(A)
        return pm

    @property
    def shape(self):
        return (self.N, self.k)

    def npanels(self) -> int:
        return len(self.panels)

    def panelrange(self, j: int) -> range:
        """Columns of panel j (0-based)."""
        return range(j * self.w, j * self.w + self.panels[j].width)

    def panelwidth(self, j: int) -> int:
        return self.panels[j].width

    def is_ghost(self) -> bool:
        return self.ghost is not None

    def assert_writable(self):
        """assert_writable (src/ghosts.jl:81-84)."""
        if self.is_ghost():
            raise ArgumentError(
                "this is a ghost matrix: its panels are regenerated from a seed rather than stored, so anything "
                "written to one would be lost the moment that panel left host memory. Write into a panel matrix of "
                "its own instead")

    def copy_from(self, A) -> "PanelMatrix":
        """copyto!(pm, A) for a dense host matrix (src/panels.jl:242-270), or
        copyto!(dest, src) for a panel matrix source of the same N and k and
        any panel width (src/panels.jl:317-320), a ghost included."""
        self.assert_writable()
        if isinstance(A, PanelMatrix):
            if A is self:
                raise ArgumentError("copycols! cannot copy a panel matrix into itself, since the two ranges may "
                                    "overlap and a column would then be read after it had already been "
                                    "overwritten. Copy into a matrix of its own and copy that back")
            if (A.N, A.k) != (self.N, self.k):
                raise DimensionMismatch(f"the source is {A.N}×{A.k} and the destination is {self.N}×{self.k}, and "
                                        "a whole-matrix copy moves column j of the source into column j of the "
                                        "destination. Use copycols! to copy part of one matrix into part of another")
            A = A.to_array()
        A = np.asarray(A)
        if A.shape != self.shape:
            raise DimensionMismatch(f"cannot copy a {A.shape} matrix into a {self.shape} panel matrix")
        for j, p in enumerate(self.panels):
            cols = self.panelrange(j)
            p.storage()[...] = A[:, cols.start:cols.stop]
            p.dirty = True
            p.epoch += 1
        return self

    def to_array(self) -> np.ndarray:
        """Matrix(pm) (src/panels.jl:330-359): the whole matrix on the host,
        in the compute eltype."""
        out = np.empty(self.shape, dtype=self.dtype, order="F")
        if self.is_ghost():
            self.ghost.collect_into(self, out)
            return out
        for j, p in enumerate(self.panels):
            wait_hold(self.plan, p)
            cols = self.panelrange(j)
            out[:, cols.start:cols.stop] = p.storage()
        return out

    def __repr__(self):
        kind = "ghost " if self.is_ghost() else ""
        return f"{self.N}x{self.k} {kind}PanelMatrix{{{self.dtype}}} in {self.npanels()} panels of width {self.w}"


def assert_conformal(X: PanelMatrix, Y: PanelMatrix):
    if X.shape != Y.shape or X.w != Y.w:
        raise ArgumentError(f"panel matrices {X.shape} w={X.w} and {Y.shape} w={Y.w} are not conformal: an "
                            "operation over both needs the same size and the same panel width")


def assert_same_panels(X: PanelMatrix, Y: PanelMatrix):
    if X.k != Y.k or X.w != Y.w:
        raise ArgumentError(f"a panel sweep over two matrices needs the same k and panel width, got k={X.k}, "
                            f"w={X.w} and k={Y.k}, w={Y.w}")


def assert_same_rows(X: PanelMatrix, Y: PanelMatrix):
    if X.N != Y.N:
        raise ArgumentError(f"a row sweep over two matrices needs the same number of rows, got {X.N} and {Y.N}")


# ---- movement (src/panels.jl:365-458) --------------------------------------

def convert_staged(backend, dst, src, queue):
    """convert_staged! (src/panels.jl:365-371): the widening or narrowing half
    of a narrowed transfer, on the same queue as the copy."""
    if queue is None:
        kernels.convert_copy(backend, dst, src)
        backend.sync_all()
        return None
    return backend.submit(queue, lambda: kernels.convert_copy(backend, dst, src))


def materialize(dst: DeviceMatrix, pm: PanelMatrix, j: int, queue=None, via=None, rows=None):
    """materialize! (src/panels.jl:373-382,427-431): panel j (or its `rows`)
    into the device buffer dst. A ghost panel is generated on the device."""
    panel = pm.panels[j]
    if pm.is_ghost():
        return pm.ghost.generate(pm, j, dst, queue, rows)
    if panel.data is None:
        raise ArgumentError("this panel has no host memory behind it: it was released")
    src = panel.storage() if rows is None else panel.storage()[rows.start:rows.stop]
    if tuple(dst.shape) != tuple(src.shape):
        raise DimensionMismatch(f"device buffer is {tuple(dst.shape)} but the host panel is {src.shape}; a ragged "
                                "last panel needs a view of the staging buffer")
    backend = pm.plan.backend
    if via is None:
        return backend.h2d(dst, src, queue=queue)
    backend.h2d(via, src, queue=queue)
    return convert_staged(backend, dst, via, queue)


def writeback(pm: PanelMatrix, j: int, src: DeviceMatrix, queue=None, via=None, rows=None):
    """writeback! (src/panels.jl:386-398,433-441)."""
    pm.assert_writable()
    panel = pm.panels[j]
    dst = panel.storage() if rows is None else panel.storage()[rows.start:rows.stop]
    if tuple(dst.shape) != tuple(src.shape):
        raise DimensionMismatch(f"device buffer is {tuple(src.shape)} but the host panel is {dst.shape}")
    backend = pm.plan.backend
    if via is not None:
        convert_staged(backend, via, src, queue)
        src = via
    event = backend.d2h(dst, src, queue=queue)
    panel.dirty = True
    panel.epoch += 1
    return event


def materialize_rows(dst: DeviceMatrix, pm: PanelMatrix, rows: range, queue=None, via=None):
    """materialize_rows! (src/panels.jl:437-445): a row block of every panel,
    one 2-D copy each, into the buffer's matching columns."""
    landing = dst if via is None else via
    event = None
    for j in range(pm.npanels()):
        cols = pm.panelrange(j)
        event = materialize(landing.view(slice(None), slice(cols.start, cols.stop)), pm, j, queue, rows=rows)
    if via is None:
        return event
    return convert_staged(pm.plan.backend, dst, via, queue)


def writeback_rows(pm: PanelMatrix, src: DeviceMatrix, rows: range, queue=None, via=None):
    """writeback_rows! (src/panels.jl:447-458)."""
    leaving = src
    if via is not None:
        convert_staged(pm.plan.backend, via, src, queue)
        leaving = via
    event = None
    for j in range(pm.npanels()):
        cols = pm.panelrange(j)
        event = writeback(pm, j, leaving.view(slice(None), slice(cols.start, cols.stop)), queue, rows=rows)
    return event


def to_device(pm: PanelMatrix, dst: DeviceMatrix, queue=None):
    """Every panel into one N x k device buffer (the backend's resident form)."""
    event = None
    for j in range(pm.npanels()):
        cols = pm.panelrange(j)
        event = materialize(dst.view(slice(None), slice(cols.start, cols.stop)), pm, j, queue)
    return event


def from_device(pm: PanelMatrix, src: DeviceMatrix, queue=None):
    event = None
    for j in range(pm.npanels()):
        cols = pm.panelrange(j)
        event = writeback(pm, j, src.view(slice(None), slice(cols.start, cols.stop)), queue)
    return event


def wait_hold(plan, panel) -> None:
    """Waits for whatever copy last read or wrote the panel's host memory
    (its hold event), before the host reads the panel or gives its block
    back: the wait of spill! (src/panels.jl:512-520)."""
    if panel.hold is not None:
        plan.backend.sync_event(panel.hold)
        panel.hold = None


def free(pm: PanelMatrix) -> None:
    """free! (src/panels.jl:540-555): gives every panel's host block back."""
    for p in pm.panels:
        if p.data is not None:
            wait_hold(pm.plan, p)
            release_host_block(pm.plan, p.data.block)
            p.data = None
