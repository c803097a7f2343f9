"""GhostPanels: panel matrices whose panels are computed instead of stored
(src/ghosts.jl).

With the default generator a ghost panel, or any block of its rows, is filled
in device memory by kernels.ghost_fill straight into the staging buffer the
sweep hands out: nothing is generated on the host and nothing crosses the bus
(the reference generates on the host producer task and uploads,
src/ghosts.jl:97-122). Entry (row, col) depends on the seed, the row and the
column in the full matrix only, so every panel width and every row block cut
gives the same matrix. A user generator f(dst, rng, col) keeps the
reference's host contract: it fills one whole host column of the storage
eltype from an rng seeded by (seed, col), and the column is uploaded.
"""
from __future__ import annotations

import numpy as np

from . import kernels
from ._lib import ArgumentError
from .panels import Panel, PanelMatrix, host_storage_eltype
from .plan import resolve_panel_width


class GhostHome:
    """GhostHome (src/ghosts.jl:65-68): the generator and the columns a panel holds."""

    __slots__ = ("source", "cols")

    def __init__(self, source, cols: range):
        self.source, self.cols = source, cols


class GhostSource:
    """GhostSource (src/ghosts.jl:58): seed, size, width and generator."""

    def __init__(self, generator, seed: int, N: int, k: int, w: int):
        self.generator = generator
        self.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.N, self.k, self.w = N, k, w

    def column_rng(self, col: int) -> np.random.Generator:
        """A stream keyed by the seed and the column alone (src/ghosts.jl:93-100)."""
        return np.random.Generator(np.random.Philox(key=(self.seed << 64) | (int(col) & 0xFFFFFFFFFFFFFFFF)))

    # -- hooks PanelMatrix movement calls ---------------------------------
    def generate(self, pm: PanelMatrix, j: int, dst, queue, rows):
        """materialize! of ghost panel j (or its `rows`) into the device view dst."""
        backend = pm.plan.backend
        cols = pm.panelrange(j)
        row0 = 0 if rows is None else rows.start
        S = host_storage_eltype(pm.plan, pm.dtype)
        if self.generator is None:
            work = lambda: kernels.ghost_fill(backend, dst, row0, cols.start, self.seed, S)
            if queue is None:
                work()
                backend.sync_all()
                return None
            return backend.submit(queue, work)
        host = self.host_columns(S, cols)
        block = host if rows is None else host[rows.start:rows.stop]
        if block.dtype == dst.dtype:
            return backend.h2d(dst, np.asfortranarray(block), queue=queue)
        return backend.h2d(dst, np.asfortranarray(block.astype(dst.dtype)), queue=queue)

    def host_columns(self, S, cols: range) -> np.ndarray:
        """generate_panel! (src/ghosts.jl:97-103) for a user generator."""
        out = np.empty((self.N, len(cols)), dtype=S, order="F")
        for c, col in enumerate(cols):
            # The generator sees the column's 1-based index in the full matrix,
            # as the reference's does.
            self.generator(out[:, c], self.column_rng(col), col + 1)
        return out

    def collect_into(self, pm: PanelMatrix, out: np.ndarray) -> None:
        """Matrix(Ω) for a ghost: the whole matrix, in the compute eltype."""
        S = host_storage_eltype(pm.plan, pm.dtype)
        if self.generator is not None:
            out[...] = self.host_columns(S, range(0, pm.k)).astype(pm.dtype)
            return
        backend = pm.plan.backend
        device = backend.alloc_device(pm.dtype, (pm.N, pm.k))
        kernels.ghost_fill(backend, device, 0, 0, self.seed, S)
        backend.d2h(out, device)


def GhostPanels(dtype, N: int, k: int, *, plan, seed=0, w=None, generator=None) -> PanelMatrix:
    """GhostPanels([f!], T, N, k; plan, seed=0, w=nothing) (src/ghosts.jl:53-63).

    An N x k read-only panel matrix whose panels are generated on demand. With
    no generator, entries are standard normal (complex: real and imaginary
    parts of variance 1/2), generated on the device. `generator(dst, rng, col)`
    fills one host column of the storage eltype instead, col 1-based."""
    if N <= 0:
        raise ArgumentError(f"N must be positive, got {N}")
    if k <= 0:
        raise ArgumentError(f"k must be positive, got {k}")
    dtype = np.dtype(dtype)
    width = resolve_panel_width(plan, N, k, dtype, override=w)
    source = GhostSource(generator, seed, int(N), int(k), width)
    panels = []
    for j in range(-(-int(k) // width)):
        cols = range(j * width, min((j + 1) * width, int(k)))
        panels.append(Panel(None, GhostHome(source, cols), len(cols)))
    return PanelMatrix(N, k, width, panels, plan, dtype, ghost=source)


def isghost(pm: PanelMatrix) -> bool:
    """Whether pm is a GhostPanels matrix (regenerated from its seed, never stored)."""
    return pm.is_ghost()
