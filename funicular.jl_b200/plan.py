"""ResidencyPlan: the owner of every byte the host layer allocates (src/plan.jl).

The device pool is keyed by (eltype, shape), checked against the budget before
it allocates, and never frees (src/plan.jl:9-15,159-185): a sweep checks its
staging buffers out and back in, so after the first sweep of a shape nothing is
allocated. The host pool hands out 64-byte aligned blocks of page-locked slabs
that grow by doubling up to the host budget (src/plan.jl:17-27,192-320). The
panel-width and row-block arithmetic is the reference's (src/plan.jl:112-157).
The disk tier, spilling and eviction are not part of this backend.
"""
from __future__ import annotations

import math
import threading
from collections import defaultdict

import numpy as np

from ._lib import ArgumentError
from .device_api import SLAB_ALIGN, B200Backend

GiB = 1024 ** 3
FEED_DEPTH = 2  # src/plan.jl:7


def human_readable_bytes(n: int) -> str:
    """src/device_api.jl:301-311."""
    if n < 1024:
        return f"{n} B"
    x = n / 1024
    for unit in ("KiB", "MiB", "GiB", "TiB"):
        if x < 1024 or unit == "TiB":
            return f"{round(x, 2)} {unit}"
        x /= 1024
    return f"{n} B"


def align_up(n: int, a: int) -> int:
    return -(-n // a) * a


class DevicePool:
    def __init__(self, budget: int):
        self.budget = int(budget)
        self.allocated = 0
        self.available = defaultdict(list)


class HostBlock:
    __slots__ = ("slab", "offset", "nbytes")

    def __init__(self, slab: int, offset: int, nbytes: int):
        self.slab, self.offset, self.nbytes = slab, offset, nbytes


class HostPool:
    def __init__(self, budget: int):
        self.budget = int(budget)
        self.reserved = 0
        self.slabs = []
        self.cursors = []
        self.free = defaultdict(list)
        self.lock = threading.RLock()


class HostStorage:
    """A panel's host memory: a view of a slab block (src/tiers.jl)."""

    __slots__ = ("array", "slab", "block")

    def __init__(self, array, slab, block):
        self.array, self.slab, self.block = array, slab, block


class ResidencyPlan:
    """ResidencyPlan(; device_budget, host_budget, backend, ...) (src/plan.jl:29-87)."""

    def __init__(self, *, device_budget, host_budget, backend=None, workspace_bytes=0, nbuffers=2,
                 target_panel_bytes=2 * GiB, panel_width=None, host_eltype=None):
        dev = int(math.floor(device_budget))
        host = int(math.floor(host_budget))
        work = int(math.floor(workspace_bytes))
        if work < 0:
            raise ArgumentError(f"workspace_bytes must be nonnegative, got {work}")
        if nbuffers < 1:
            raise ArgumentError(f"nbuffers must be at least 1, got {nbuffers}")
        if target_panel_bytes < 1:
            raise ArgumentError(f"target_panel_bytes must be positive, got {target_panel_bytes}")
        if host <= 0:
            raise ArgumentError(f"host_budget must be positive, got {host}")
        if dev <= work:
            raise ArgumentError(
                f"device_budget of {human_readable_bytes(dev)} does not cover the operator workspace of "
                f"{human_readable_bytes(work)}, leaving nothing for panel buffers. Raise device_budget or report "
                "a smaller workspace_bytes")
        if panel_width is not None and int(panel_width) < 1:
            raise ArgumentError(f"panel_width must be positive, got {panel_width}")
        self.backend = backend if backend is not None else B200Backend(0)
        self.device_budget = dev
        self.host_budget = host
        self.workspace_bytes = work
        self.nbuffers = int(nbuffers)
        self.target_panel_bytes = int(math.floor(target_panel_bytes))
        self.panel_width = None if panel_width is None else int(panel_width)
        self.host_eltype = None if host_eltype is None else np.dtype(host_eltype)
        self.devicepool = DevicePool(dev - work)
        self.hostpool = HostPool(host)

    def __repr__(self):
        return (f"ResidencyPlan({type(self.backend).__name__}, device {human_readable_bytes(self.device_budget)}, "
                f"host {human_readable_bytes(self.host_budget)})")


def panel_bytes(N: int, w: int, dtype) -> int:
    return int(N) * int(w) * np.dtype(dtype).itemsize


def device_bytes_required(N, w, dtype, nbuffers=2, extra_buffers=0, workspace_bytes=0) -> int:
    return (int(nbuffers) + int(extra_buffers)) * panel_bytes(N, w, dtype) + int(workspace_bytes)


def choose_panel_width(N, k, dtype, *, device_budget, nbuffers=2, extra_buffers=0, workspace_bytes=0,
                       target_panel_bytes=2 * GiB) -> int:
    """choose_panel_width (src/plan.jl:112-123)."""
    if N <= 0:
        raise ArgumentError(f"N must be positive, got {N}")
    if k <= 0:
        raise ArgumentError(f"k must be positive, got {k}")
    buffers = int(nbuffers) + int(extra_buffers)
    if buffers < 1:
        raise ArgumentError(f"nbuffers + extra_buffers must be at least 1, got {buffers}")
    column = int(N) * np.dtype(dtype).itemsize
    available = int(math.floor(device_budget)) - int(math.floor(workspace_bytes))
    per_buffer = available // buffers
    if per_buffer < column:
        raise ArgumentError(
            f"device budget of {human_readable_bytes(int(device_budget))} leaves {human_readable_bytes(available)} "
            f"after a {human_readable_bytes(int(workspace_bytes))} operator workspace, so "
            f"{human_readable_bytes(per_buffer)} for each of {buffers} panel buffers, but a single column of {N} "
            f"{np.dtype(dtype)} entries needs {human_readable_bytes(column)}. Raise device_budget, lower nbuffers, "
            "or narrow the compute eltype")
    w = min(int(k), max(1, min(int(math.floor(target_panel_bytes)), per_buffer) // column))
    npanels = -(-int(k) // w)
    return -(-int(k) // npanels)


def row_block_height(N: int, k: int, w: int) -> int:
    """row_block_height (src/plan.jl:133)."""
    return max(1, min(int(N), (int(N) * int(w)) // int(k)))


def resolve_panel_width(plan: ResidencyPlan, N, k, dtype, override=None, extra_buffers=0) -> int:
    """resolve_panel_width (src/plan.jl:135-157)."""
    requested = plan.panel_width if override is None else override
    if requested is None:
        return choose_panel_width(N, k, dtype, device_budget=plan.device_budget, nbuffers=plan.nbuffers,
                                  extra_buffers=extra_buffers, workspace_bytes=plan.workspace_bytes,
                                  target_panel_bytes=plan.target_panel_bytes)
    w = int(requested)
    if not (1 <= w <= k):
        raise ArgumentError(f"panel width {w} must lie in 1:{k}")
    needed = device_bytes_required(N, w, dtype, plan.nbuffers, extra_buffers, plan.workspace_bytes)
    if needed > plan.device_budget:
        buffers = plan.nbuffers + int(extra_buffers)
        fits = choose_panel_width(N, k, dtype, device_budget=plan.device_budget, nbuffers=plan.nbuffers,
                                  extra_buffers=extra_buffers, workspace_bytes=plan.workspace_bytes,
                                  target_panel_bytes=plan.device_budget)
        raise ArgumentError(
            f"panel width {w} needs {human_readable_bytes(needed)} on the device ({buffers} buffers of "
            f"{human_readable_bytes(panel_bytes(N, w, dtype))} plus {human_readable_bytes(plan.workspace_bytes)} of "
            f"operator workspace) but device_budget is {human_readable_bytes(plan.device_budget)}. Use panel_width "
            f"<= {fits} or raise device_budget")
    return w


def checkout_device_buffers(plan: ResidencyPlan, dtype, dims, count: int):
    """checkout_device_buffers! (src/plan.jl:159-177)."""
    dtype = np.dtype(dtype)
    if not plan.backend.supports_eltype(dtype):
        raise ArgumentError(f"backend {type(plan.backend).__name__} cannot compute in {dtype}: the B200 kernels "
                            "compute in ComplexF64, with narrower types only as host storage")
    return _checkout(plan, dtype, dims, count)


def checkout_staging_storage(plan: ResidencyPlan, dtype, dims, count: int):
    """Buffers in a storage eltype (no compute), for narrowed host tiers."""
    return _checkout(plan, np.dtype(dtype), dims, count)


def _checkout(plan, dtype, dims, count):
    pool = plan.devicepool
    dims = (int(dims[0]), int(dims[1]))
    cache = pool.available[(dtype.str, dims)]
    nbytes = dims[0] * dims[1] * dtype.itemsize
    out = []
    for _ in range(count):
        if cache:
            out.append(cache.pop())
            continue
        if pool.allocated + nbytes > pool.budget:
            for b in out:
                cache.append(b)
            raise ArgumentError(
                f"device pool is full: a {dims[0]}x{dims[1]} {dtype} buffer needs {human_readable_bytes(nbytes)}, "
                f"{human_readable_bytes(pool.allocated)} is already allocated and the pool caps at "
                f"{human_readable_bytes(pool.budget)} (device_budget {human_readable_bytes(plan.device_budget)} minus "
                f"{human_readable_bytes(plan.workspace_bytes)} of operator workspace). Reduce the panel width, lower "
                "nbuffers, or raise device_budget")
        out.append(plan.backend.alloc_device(dtype, dims))
        pool.allocated += nbytes
    return out


def device_bytes_to_add(plan: ResidencyPlan, dtype, requests) -> int:
    """Bytes the pool would have to allocate to hand out `requests`, a list of
    (dims, count): buffers of those dims it already holds, given back by
    earlier checkouts, cost nothing."""
    dtype = np.dtype(dtype)
    pool = plan.devicepool
    total = 0
    for dims, count in requests:
        dims = (int(dims[0]), int(dims[1]))
        held = len(pool.available[(dtype.str, dims)])
        total += max(0, int(count) - held) * dims[0] * dims[1] * dtype.itemsize
    return total


def checkin_device_buffers(plan: ResidencyPlan, buffers) -> None:
    """checkin_device_buffers! (src/plan.jl:179-185)."""
    for b in buffers:
        plan.devicepool.available[(b.dtype.str, tuple(b.shape))].append(b)


def device_bytes_allocated(plan: ResidencyPlan) -> int:
    """Bytes the plan's device pool holds (src/plan.jl:159-185): every buffer
    it has checked out so far, in use or free, counted against device_budget."""
    return plan.devicepool.allocated


def _take_host_block(plan: ResidencyPlan, n: int):
    pool = plan.hostpool
    with pool.lock:
        reusable = pool.free[n]
        if reusable:
            return reusable.pop()
        for i, slab in enumerate(pool.slabs):
            if pool.cursors[i] + n <= slab.nbytes:
                block = HostBlock(i, pool.cursors[i], n)
                pool.cursors[i] += n
                return block
        remaining = pool.budget - pool.reserved
        if remaining < n:
            return None
        # Slabs double so page-locking is amortized (src/plan.jl:232-241).
        slab = plan.backend.alloc_host_slab(min(remaining, max(n, pool.reserved)))
        pool.slabs.append(slab)
        pool.cursors.append(0)
        pool.reserved += slab.nbytes
        block = HostBlock(len(pool.slabs) - 1, 0, n)
        pool.cursors[-1] += n
        return block


def acquire_host_block(plan: ResidencyPlan, nbytes: int) -> HostBlock:
    """acquire_host_block! (src/plan.jl:193-208), without a disk tier to spill to."""
    n = align_up(int(nbytes), SLAB_ALIGN)
    block = _take_host_block(plan, n)
    if block is None:
        pool = plan.hostpool
        raise ArgumentError(
            f"host tier is full: a {human_readable_bytes(n)} panel block does not fit in the "
            f"{human_readable_bytes(pool.budget - pool.reserved)} left of the {human_readable_bytes(pool.budget)} "
            "host_budget. Raise host_budget, or reduce k or the panel width")
    return block


def release_host_block(plan: ResidencyPlan, block: HostBlock) -> None:
    with plan.hostpool.lock:
        plan.hostpool.free[block.nbytes].append(block)


def alloc_host_storage(plan: ResidencyPlan, dtype, dims, blockbytes=None) -> HostStorage:
    """alloc_host_storage! (src/plan.jl:316-320)."""
    dtype = np.dtype(dtype)
    nbytes = dims[0] * dims[1] * dtype.itemsize if blockbytes is None else blockbytes
    block = acquire_host_block(plan, max(nbytes, 1))
    slab = plan.hostpool.slabs[block.slab]
    return HostStorage(slab.matrix(dtype, (int(dims[0]), int(dims[1])), block.offset), slab, block)


def _hostpool(x) -> HostPool:
    return x.hostpool if isinstance(x, ResidencyPlan) else x


def host_bytes_reserved(pool) -> int:
    """Page-locked bytes the host pool holds (src/plan.jl:322-334); takes the
    pool or its plan."""
    return _hostpool(pool).reserved


def host_bytes_free(pool) -> int:
    """Bytes of given-back host blocks waiting in the pool for reuse
    (src/plan.jl:322-334); takes the pool or its plan."""
    return sum(b.nbytes for blocks in _hostpool(pool).free.values() for b in blocks)


def host_bytes_in_use(pool) -> int:
    """Bytes of host blocks handed out and not given back (src/plan.jl:322-334);
    takes the pool or its plan."""
    return sum(_hostpool(pool).cursors) - host_bytes_free(pool)
