"""The device API of the B200 backend: the contract of src/device_api.jl:5-138
implemented over libfunicular_b200.

`B200Backend` plays the role `CUDABackend` plays in ext/FunicularCUDAExt.jl:
device arrays, page-locked host slabs, non-blocking queues, device-side event
waits and pitched 2-D copies. Device arrays are `DeviceMatrix` objects, a
pointer with a shape and a leading dimension, whose views carry an offset and
the parent's pitch (the region_pointer/copy_shape idea of
ext/FunicularCUDAExt.jl:154-182). Host arrays are Fortran-ordered numpy
arrays, page-locked when they come from `alloc_host_slab`.
"""
from __future__ import annotations

import ctypes
import threading
import weakref
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch, call, check, load

SLAB_ALIGN = 64  # src/device_api.jl:140

_ELTYPE_CODES = {
    np.dtype(np.complex128): _lib.FB_C128,
    np.dtype(np.complex64): _lib.FB_C64,
    np.dtype(np.float64): _lib.FB_F64,
    np.dtype(np.float32): _lib.FB_F32,
}


def eltype_code(dtype) -> int:
    try:
        return _ELTYPE_CODES[np.dtype(dtype)]
    except KeyError:
        raise ArgumentError(f"the B200 backend stores ComplexF64, ComplexF32, Float64 and Float32, got {dtype}")


class _DeviceAllocation:
    """Owns one device allocation; freed when the last view goes."""

    def __init__(self, nbytes: int):
        p = ctypes.c_void_p()
        call("fb_alloc_device", ctypes.byref(p), ctypes.c_size_t(nbytes))
        self.ptr = p.value or 0
        self.nbytes = nbytes
        self._finalizer = weakref.finalize(self, _free_device, self.ptr)


def _free_device(ptr):
    if ptr:
        try:
            load().fb_free_device(ctypes.c_void_p(ptr))
        except Exception:
            pass


@dataclass(eq=False)
class DeviceMatrix:
    """A column-major device matrix or a view of one."""

    ptr: int
    shape: tuple
    ld: int
    dtype: np.dtype
    owner: object = None

    @property
    def rows(self) -> int:
        return self.shape[0]

    @property
    def cols(self) -> int:
        return self.shape[1]

    @property
    def itemsize(self) -> int:
        return self.dtype.itemsize

    @property
    def size(self) -> int:
        return self.shape[0] * self.shape[1]

    def __len__(self):
        return self.shape[0]

    def view(self, rows=slice(None), cols=slice(None)) -> "DeviceMatrix":
        r0, r1, rs = rows.indices(self.shape[0])
        c0, c1, cs = cols.indices(self.shape[1])
        if rs != 1 or cs != 1:
            raise ArgumentError("a device view takes unit-stride ranges of rows and columns")
        r1, c1 = max(r1, r0), max(c1, c0)
        ptr = self.ptr + (r0 + c0 * self.ld) * self.itemsize
        return DeviceMatrix(ptr, (r1 - r0, c1 - c0), self.ld, self.dtype,
                            self.owner if self.owner is not None else self)

    def __getitem__(self, key):
        rows, cols = key
        if isinstance(rows, int):
            rows = slice(rows, rows + 1)
        if isinstance(cols, int):
            cols = slice(cols, cols + 1)
        return self.view(rows, cols)

    def to_host(self) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype, order="F")
        if out.size:
            copy_region(out, self, None)
        return out

    def same_view(self, other: "DeviceMatrix") -> bool:
        return (self.ptr == other.ptr and self.ld == other.ld and self.shape == other.shape
                and self.dtype == other.dtype)


def host_region(a: np.ndarray):
    """(pointer, rows, cols, ld) of a host array whose columns are contiguous."""
    if a.ndim == 1:
        if a.strides[0] != a.itemsize:
            raise ArgumentError("a copy needs its columns contiguous")
        return a.ctypes.data, a.shape[0], 1, a.shape[0]
    if a.ndim != 2:
        raise ArgumentError(f"Funicular copies panels and blocks of them, which are at most two-dimensional, got a {a.ndim}-dimensional array")
    if a.shape[0] > 1 and a.strides[0] != a.itemsize:
        raise ArgumentError(f"a copy needs its columns contiguous but this array has a stride of {a.strides[0] // a.itemsize} between neighbouring rows")
    ld = a.strides[1] // a.itemsize if a.shape[1] > 1 else max(a.shape[0], 1)
    return a.ctypes.data, a.shape[0], a.shape[1], ld


def region(a):
    if isinstance(a, DeviceMatrix):
        return a.ptr, a.rows, a.cols, a.ld
    return host_region(a)


def copy_region(dst, src, queue) -> None:
    """copy_region! (ext/FunicularCUDAExt.jl:138-152): one pitched 2-D copy."""
    dptr, drows, dcols, dld = region(dst)
    sptr, srows, scols, sld = region(src)
    if (drows, dcols) != (srows, scols):
        raise DimensionMismatch(f"copy between a {(drows, dcols)} destination and a {(srows, scols)} source")
    isz = np.dtype(dst.dtype).itemsize
    if drows == 0 or dcols == 0:
        return
    call("fb_copy2d", ctypes.c_void_p(dptr), ctypes.c_size_t(dld * isz), ctypes.c_void_p(sptr),
         ctypes.c_size_t(sld * isz), ctypes.c_size_t(drows * isz), ctypes.c_size_t(dcols),
         ctypes.c_void_p(queue.handle if queue is not None else None))


class Queue:
    """make_queue: a non-blocking stream (ext/FunicularCUDAExt.jl:63-81)."""

    def __init__(self):
        h = ctypes.c_void_p()
        call("fb_queue_create", ctypes.byref(h))
        self.handle = h.value
        self._finalizer = weakref.finalize(self, _destroy_queue, self.handle)

    def __repr__(self):
        return f"Queue(0x{self.handle:x})"


def _destroy_queue(h):
    try:
        lib = load()
        lib.fb_queue_sync(ctypes.c_void_p(h))
        lib.fb_queue_destroy(ctypes.c_void_p(h))
    except Exception:
        pass


class Event:
    """record_event's token: a timing-free CUDA event."""

    def __init__(self, handle):
        self.handle = handle
        self._finalizer = weakref.finalize(self, _destroy_event, handle)

    def query(self) -> bool:
        done = ctypes.c_int(0)
        call("fb_event_query", ctypes.c_void_p(self.handle), ctypes.byref(done))
        return bool(done.value)


def _destroy_event(h):
    try:
        load().fb_event_destroy(ctypes.c_void_p(h))
    except Exception:
        pass


class Graph:
    """A captured sequence of the library's launches (fb_graph_capture_end),
    replayed with one launch."""

    def __init__(self, handle):
        self.handle = handle
        self._finalizer = weakref.finalize(self, _destroy_graph, handle)

    def launch(self, queue) -> None:
        call("fb_graph_launch", ctypes.c_void_p(self.handle), ctypes.c_void_p(queue.handle if queue else None))


def _destroy_graph(h):
    try:
        load().fb_graph_destroy(ctypes.c_void_p(h))
    except Exception:
        pass


class HostSlab:
    """alloc_host_slab's result (src/device_api.jl:144-163): page-locked host
    memory, 64-byte aligned, handing out Fortran-ordered matrix views."""

    def __init__(self, nbytes: int):
        p = ctypes.c_void_p()
        call("fb_alloc_host_slab", ctypes.byref(p), ctypes.c_size_t(int(nbytes) + SLAB_ALIGN))
        base = p.value
        pad = (-base) % SLAB_ALIGN
        self.base = base
        self.ptr = base + pad
        self.nbytes = int(nbytes)
        self._finalizer = weakref.finalize(self, _free_slab, base)

    def matrix(self, dtype, dims, offset: int = 0) -> np.ndarray:
        dtype = np.dtype(dtype)
        nbytes = int(np.prod(dims)) * dtype.itemsize
        if offset < 0:
            raise ArgumentError(f"slab offset must be nonnegative, got {offset}")
        if offset + nbytes > self.nbytes:
            raise ArgumentError(f"a {nbytes} B view at offset {offset} does not fit in a {self.nbytes} B host slab")
        buf = (ctypes.c_char * max(nbytes, 1)).from_address(self.ptr + offset)
        buf._slab = self  # the view keeps its slab alive
        return np.frombuffer(buf, dtype=dtype, count=int(np.prod(dims))).reshape(dims, order="F")


def _free_slab(base):
    try:
        load().fb_free_host_slab(ctypes.c_void_p(base))
    except Exception:
        pass


class B200Backend:
    """Device backend on one B200 (one process per GPU)."""

    def __init__(self, device: int = 0):
        load()
        n = _lib.device_count()
        if n == 0:
            raise _lib.DeviceError("no CUDA device is visible, and the B200 backend has no CPU fallback")
        if not (0 <= device < n):
            raise ArgumentError(f"device {device} is not one of the {n} visible devices")
        self.device = device
        call("fb_set_device", device)
        self._local = threading.local()
        self._ws_lock = threading.Lock()
        self._ws = None
        self._ws_bytes = 0
        self._ws_event = None
        self.device_bytes_allocated = 0

    # -- device API ------------------------------------------------------
    def devicetype(self, dtype):
        return DeviceMatrix

    def supports_eltype(self, dtype) -> bool:
        # The kernels compute in ComplexF64; the narrower types exist only as
        # storage that convert_copy widens.
        return np.dtype(dtype) == np.complex128

    def transfers_are_real(self) -> bool:
        return True

    def alloc_device(self, dtype, dims) -> DeviceMatrix:
        dtype = np.dtype(dtype)
        eltype_code(dtype)
        rows, cols = (dims[0], dims[1]) if len(dims) == 2 else (dims[0], 1)
        nbytes = max(rows * cols * dtype.itemsize, dtype.itemsize)
        owner = _DeviceAllocation(nbytes)
        self.device_bytes_allocated += nbytes
        return DeviceMatrix(owner.ptr, (rows, cols), max(rows, 1), dtype, owner)

    def alloc_host_slab(self, nbytes: int) -> HostSlab:
        return HostSlab(nbytes)

    def make_queue(self) -> Queue:
        return Queue()

    def make_sweep_queues(self):
        return Queue(), Queue(), Queue()

    @property
    def current_queue(self):
        return getattr(self._local, "queue", None)

    def submit(self, queue: Queue, work):
        """submit! (ext/FunicularCUDAExt.jl:86-89): runs work() now on the
        calling thread, with every kernel it launches through this backend
        landing on `queue`."""
        previous = self.current_queue
        self._local.queue = queue
        try:
            work()
        finally:
            self._local.queue = previous
        return self.record_event(queue)

    def record_event(self, queue) -> Event:
        h = ctypes.c_void_p()
        call("fb_event_record", ctypes.c_void_p(queue.handle if queue else None), ctypes.byref(h))
        return Event(h.value)

    def wait_event(self, queue, event) -> None:
        if event is None:
            return
        call("fb_queue_wait_event", ctypes.c_void_p(queue.handle if queue else None), ctypes.c_void_p(event.handle))

    def sync_queue(self, queue) -> None:
        call("fb_queue_sync", ctypes.c_void_p(queue.handle if queue else None))

    def sync_event(self, event) -> None:
        if event is not None:
            call("fb_event_sync", ctypes.c_void_p(event.handle))

    def sync_all(self) -> None:
        call("fb_sync_all")

    def h2d(self, dst, src, queue=None):
        return self._copy(dst, src, queue)

    def d2h(self, dst, src, queue=None):
        return self._copy(dst, src, queue)

    def _copy(self, dst, src, queue):
        if tuple(dst.shape) != tuple(src.shape):
            raise DimensionMismatch(f"copy between a {tuple(dst.shape)} destination and a {tuple(src.shape)} source")
        if np.dtype(dst.dtype) != np.dtype(src.dtype):
            return self._converting_copy(dst, src, queue)
        copy_region(dst, src, queue)
        return self.record_event(queue) if queue is not None else None

    def _converting_copy(self, dst, src, queue):
        """converting_copy! (ext/FunicularCUDAExt.jl:195-212): outside a sweep
        a bare copy across eltypes stages through a device buffer and waits."""
        from .kernels import convert_copy
        q = queue if queue is not None else self.make_queue()
        if isinstance(dst, DeviceMatrix) and isinstance(src, DeviceMatrix):
            self.submit(q, lambda: convert_copy(self, dst, src))
        elif isinstance(dst, DeviceMatrix):
            staging = self.alloc_device(src.dtype, src.shape)
            copy_region(staging, src, q)
            self.submit(q, lambda: convert_copy(self, dst, staging))
        else:
            staging = self.alloc_device(dst.dtype, dst.shape)
            self.submit(q, lambda: convert_copy(self, staging, src))
            copy_region(dst, staging, q)
        self.sync_queue(q)
        return self.record_event(q) if queue is not None else None

    def capture(self, queue, work) -> Graph:
        """Runs work() with every launch on `queue` captured instead of run, and
        returns the graph that replays them. Scratch used inside must not move
        afterwards: pass kernels their own workspace."""
        call("fb_graph_capture_begin", ctypes.c_void_p(queue.handle))
        previous = self.current_queue
        self._local.queue = queue
        handle = ctypes.c_void_p()
        try:
            work()
        finally:
            self._local.queue = previous
            status = load().fb_graph_capture_end(ctypes.c_void_p(queue.handle), ctypes.byref(handle))
        check(status, "fb_graph_capture_end")
        return Graph(handle.value)

    # -- helpers -----------------------------------------------------------
    def todevice(self, a: np.ndarray) -> DeviceMatrix:
        a = np.asarray(a)
        if a.ndim == 1:
            a = a.reshape(-1, 1)
        d = self.alloc_device(a.dtype, a.shape)
        if a.size:
            copy_region(d, np.asfortranarray(a), None)
        return d

    def workspace(self, nbytes: int):
        """A device scratch buffer of at least nbytes for a kernel about to be
        enqueued on the current queue. One buffer serves every queue: a new
        user's queue first waits for the last user's event, so the reuse is
        ordered on the device and the host never waits. The buffer only grows,
        so after the first calls of a given size nothing is allocated."""
        queue = self.current_queue
        with self._ws_lock:
            if nbytes > self._ws_bytes:
                if self._ws_event is not None:
                    self.sync_event(self._ws_event)
                size = max(int(nbytes), 2 * self._ws_bytes, 1 << 20)
                size = (size + 255) // 256 * 256
                self._ws = _DeviceAllocation(size)
                self._ws_bytes = size
                self.device_bytes_allocated += size
                self._ws_event = None
            elif self._ws_event is not None:
                self.wait_event(queue, self._ws_event)
            return self._ws.ptr, self._ws_bytes

    def workspace_release(self) -> None:
        """Records that the kernels just enqueued on the current queue are the
        last users of the workspace."""
        with self._ws_lock:
            self._ws_event = self.record_event(self.current_queue)

    def queue_handle(self):
        q = self.current_queue
        return ctypes.c_void_p(q.handle if q is not None else None)


def b200_backend(device: int = 0) -> B200Backend:
    """Funicular.cuda_backend's counterpart (src/device_api.jl:173)."""
    return B200Backend(device)
