"""The kernel overrides of the B200 backend: the four functions of
src/kernels.jl that a vendor backend specialises (the pattern of
ext/FunicularMetalExt.jl:187-189), plus the device hooks the reference does
not have yet: the k x k Cholesky with its shifted retry (cholesky_upper,
src/panelblas.jl:148-155) and the whole device-resident cholqr2!.

Every function checks shapes the way the reference does (DimensionMismatch)
before anything reaches the device, then makes one C call whose kernels land on
the backend's current queue (the one `submit` set), or on the default stream
outside a sweep.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, DimensionMismatch, NotPositiveDefinite, call, z128
from .device_api import DeviceMatrix, eltype_code

EPS64 = float(np.finfo(np.float64).eps)


def _vp(x):
    return ctypes.c_void_p(x)


def _need_complex128(*mats):
    for m in mats:
        if not isinstance(m, DeviceMatrix):
            raise ArgumentError(f"the B200 kernels take device matrices, got {type(m).__name__}")
        if m.dtype != np.complex128:
            raise ArgumentError(f"the B200 kernels compute in ComplexF64, got {m.dtype}")


def convert_copy(backend, dst: DeviceMatrix, src: DeviceMatrix) -> DeviceMatrix:
    """convert_copy! (src/kernels.jl:14-20)."""
    if tuple(dst.shape) != tuple(src.shape):
        raise DimensionMismatch(f"copy between a {tuple(dst.shape)} destination and a {tuple(src.shape)} source")
    if dst.size == 0:
        return dst
    call("fb_convert_copy", _vp(dst.ptr), eltype_code(dst.dtype), ctypes.c_int64(dst.ld),
         _vp(src.ptr), eltype_code(src.dtype), ctypes.c_int64(src.ld),
         ctypes.c_int64(dst.rows), ctypes.c_int64(dst.cols), backend.queue_handle())
    return dst


def gram_accumulate(backend, C: DeviceMatrix, A: DeviceMatrix, B: DeviceMatrix, alpha, beta) -> DeviceMatrix:
    """gram_accumulate! (src/kernels.jl:40): C <- alpha A^H B + beta C, with
    beta == 0 overwriting whatever C held."""
    _need_complex128(C, A, B)
    if not (A.rows == B.rows and tuple(C.shape) == (A.cols, B.cols)):
        raise DimensionMismatch(f"cannot accumulate the {A.shape}' times {B.shape} product into a {C.shape} matrix")
    if C.size == 0:
        return C
    lib = _lib.load()
    hermitian = 1 if A.same_view(B) else 0
    need = ctypes.c_size_t(0)
    call("fb_zgram_workspace_size", ctypes.c_int64(A.rows), A.cols, B.cols, hermitian, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    try:
        status = lib.fb_zgram(_vp(C.ptr), C.ld, _vp(A.ptr), max(A.ld, 1), _vp(B.ptr), max(B.ld, 1),
                              A.rows, A.cols, B.cols, z128(alpha), z128(beta), _vp(ws), ws_bytes,
                              backend.queue_handle())
    finally:
        backend.workspace_release()
    _lib.check(status, "gram_accumulate!")
    return C


def gram_tc(backend, C: DeviceMatrix, A: DeviceMatrix, alpha=1.0, beta=0.0) -> DeviceMatrix:
    """The tensor-core form of gram_accumulate!(C, A, A, alpha, beta): C <- alpha
    A^H A + beta C through an Ozaki split of A into 8-bit slices on the integer
    tensor cores (k <= 64)."""
    _need_complex128(C, A)
    if tuple(C.shape) != (A.cols, A.cols):
        raise DimensionMismatch(f"cannot accumulate the Gram matrix of a {A.shape} block into a {C.shape} matrix")
    if C.size == 0:
        return C
    need = ctypes.c_size_t(0)
    call("fb_zgram_tc_workspace_size", ctypes.c_int64(A.rows), A.cols, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    try:
        status = _lib.load().fb_zgram_tc(_vp(C.ptr), C.ld, _vp(A.ptr), max(A.ld, 1), A.rows, A.cols, z128(alpha),
                                         z128(beta), _vp(ws), ws_bytes, backend.queue_handle())
    finally:
        backend.workspace_release()
    _lib.check(status, "gram (tensor cores)")
    return C


def rdiv_upper(backend, Y: DeviceMatrix, R: DeviceMatrix) -> DeviceMatrix:
    """rdiv_upper! (src/kernels.jl:108): Y <- Y R^-1, R upper triangular."""
    _need_complex128(Y, R)
    if not (R.rows == R.cols == Y.cols):
        raise DimensionMismatch(f"a {Y.shape} block cannot be divided by a {R.shape} triangular factor")
    if Y.size == 0:
        return Y
    need = ctypes.c_size_t(0)
    call("fb_ztrsm_workspace_size", Y.cols, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value) if need.value else (None, 0)
    try:
        status = _lib.load().fb_ztrsm_right_upper(_vp(Y.ptr), ctypes.c_int64(Y.ld), ctypes.c_int64(Y.rows), Y.cols,
                                                  _vp(R.ptr), ctypes.c_int64(R.ld), _vp(ws), ws_bytes,
                                                  backend.queue_handle())
    finally:
        if need.value:
            backend.workspace_release()
    _lib.check(status, "rdiv_upper!")
    return Y


def rightmul_gemm(backend, dst: DeviceMatrix, A: DeviceMatrix, C: DeviceMatrix) -> DeviceMatrix:
    """rightmul_gemm! (src/kernels.jl:73): dst <- A C."""
    _need_complex128(dst, A, C)
    if not (A.cols == C.rows and tuple(dst.shape) == (A.rows, C.cols)):
        raise DimensionMismatch(f"cannot multiply a {A.shape} block by a {C.shape} factor into a {dst.shape} matrix")
    if dst.size == 0:
        return dst
    call("fb_zgemm_right", _vp(dst.ptr), ctypes.c_int64(dst.ld), _vp(A.ptr), ctypes.c_int64(max(A.ld, 1)),
         ctypes.c_int64(A.rows), A.cols, _vp(C.ptr), ctypes.c_int64(max(C.ld, 1)), C.cols, backend.queue_handle())
    return dst


def cholesky_upper_device(backend, G: DeviceMatrix, N: int, k: int, U: DeviceMatrix,
                          Rin: DeviceMatrix | None = None, Rout: DeviceMatrix | None = None,
                          forced_unit_roundoff: float | None = None):
    """cholesky_upper(G, N, k) (src/panelblas.jl:148-155) on the device. Writes
    U; with Rin, also Rout = U Rin. Returns (shifted, shift). Waits for the
    queue, since the caller branches on `shifted`. With forced_unit_roundoff
    = u it factors G + s I at once, s = 11 (N k + k (k+1)) u ||G||_F: the
    first pass of the shifted CholeskyQR3."""
    _need_complex128(G, U)
    if G.shape != (k, k) or U.shape != (k, k):
        raise DimensionMismatch(f"cholesky_upper: a {k}x{k} factor of a {G.shape} matrix into {U.shape}")
    need = ctypes.c_size_t(0)
    call("fb_zpotrf_workspace_size", k, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    shifted = ctypes.c_int(0)
    shift = ctypes.c_double(0.0)
    lib = _lib.load()
    rin = (_vp(Rin.ptr if Rin is not None else None), Rin.ld if Rin is not None else k)
    rout = (_vp(Rout.ptr if Rout is not None else None), Rout.ld if Rout is not None else k)
    try:
        if forced_unit_roundoff is None:
            status = lib.fb_zpotrf_shifted(_vp(U.ptr), U.ld, _vp(G.ptr), G.ld, k, N, *rin, *rout,
                                           ctypes.byref(shifted), ctypes.byref(shift), _vp(ws), ws_bytes,
                                           backend.queue_handle())
        else:
            shifted.value = 1
            status = lib.fb_zpotrf_forced_shift(_vp(U.ptr), U.ld, _vp(G.ptr), G.ld, k, N, *rin, *rout,
                                                float(forced_unit_roundoff), ctypes.byref(shift), _vp(ws),
                                                ws_bytes, backend.queue_handle())
    finally:
        backend.workspace_release()
    if status == _lib.FB_ENOTSPD:
        raise NotPositiveDefinite(_lib.last_error())
    _lib.check(status, "cholesky_upper")
    return bool(shifted.value), float(shift.value)


def cholqr2_workspace_bytes(N: int, k: int) -> int:
    """Device scratch the resident cholqr2! chain needs for an N x k matrix."""
    need = ctypes.c_size_t(0)
    call("fb_zcholqr2_workspace_size", ctypes.c_int64(N), k, ctypes.byref(need))
    return need.value


UNIT_ROUNDOFF = {np.dtype(np.complex128): 2.0 ** -53, np.dtype(np.complex64): 2.0 ** -24}


def cholqr2_resident(backend, Y: DeviceMatrix, R: DeviceMatrix, wait: bool = True, form: str = "fp64",
                     unit_roundoff: float = UNIT_ROUNDOFF[np.dtype(np.complex128)]):
    """cholqr2! (src/panelblas.jl:130-139) on a matrix already in device
    memory: Y becomes Q in place and R (k x k) is written. With wait=True the
    call returns (passes, shifts) and raises if a Gram matrix stayed
    indefinite; with wait=False it only enqueues. form="tc" computes the Gram
    matrices on the integer tensor cores (k <= 64); form="shifted3" is the
    shifted CholeskyQR3 (pass 1 shifted by 11 (N k + k (k+1)) u ||G||_F with
    u = unit_roundoff, three passes); form="auto" takes the form the
    autotuner chose for this shape ("fp64" when untuned)."""
    if form not in ("fp64", "tc", "shifted3", "auto"):
        raise ArgumentError(f"cholqr2! form is 'fp64', 'tc', 'shifted3' or 'auto', got {form!r}")
    _need_complex128(Y, R)
    N, k = Y.shape
    if form == "auto":
        from . import autotune
        form = autotune.form_for(N, k)
    if R.shape != (k, k):
        raise DimensionMismatch(f"cholqr2! of an {N}x{k} matrix writes a {k}x{k} R, got {R.shape}")
    need = ctypes.c_size_t(0)
    call("fb_zcholqr2_workspace_size", ctypes.c_int64(N), k, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    lib = _lib.load()
    info = ctypes.c_int(0)
    passes = ctypes.c_int(0)
    try:
        out = (ctypes.byref(info) if wait else None, ctypes.byref(passes) if wait else None,
               _vp(ws), ws_bytes, backend.queue_handle())
        if form == "shifted3":
            status = lib.fb_zcholqr3_shifted(_vp(Y.ptr), Y.ld, N, k, _vp(R.ptr), R.ld, float(unit_roundoff), *out)
        else:
            entry = lib.fb_zcholqr2_tc if form == "tc" else lib.fb_zcholqr2
            status = entry(_vp(Y.ptr), Y.ld, N, k, _vp(R.ptr), R.ld, *out)
    finally:
        backend.workspace_release()
    if not wait:
        _lib.check(status, "cholqr2!")
        return None
    shifts = (ctypes.c_double * 3)()
    if status == _lib.FB_OK:
        status = lib.fb_zcholqr2_query(_vp(ws), None, None, shifts)
    if status == _lib.FB_ENOTSPD:
        raise NotPositiveDefinite(_lib.last_error())
    _lib.check(status, "cholqr2!")
    return passes.value, tuple(shifts)


def cholqr2_staged(backend, panels, D: DeviceMatrix, R: DeviceMatrix, unit_roundoff: float = 0.0):
    """cholqr2! end to end on a matrix held in page-locked host panels (a
    list of N x w_p column-major arrays in column order, all complex128 or
    all complex64 for a narrowed tier, e.g. a PanelMatrix's host storage): the
    panels go up in row blocks while the first Gram consumes them (widened on
    the device), the FP64 chain runs on the device (D is the N x k complex128
    staging copy), and the last solve's row blocks come back into the panels
    as they are solved (narrowed on the device). unit_roundoff > 0 runs the
    shifted CholeskyQR3 instead. R (device) is written. Returns (passes,
    shifts); raises NotPositiveDefinite, leaving the panels as they were,
    when a Gram matrix stays indefinite. For complex128 panels, the same bits
    as cholqr2_resident on D."""
    _need_complex128(D, R)
    N, k = D.shape
    if R.shape != (k, k):
        raise DimensionMismatch(f"cholqr2! of an {N}x{k} matrix writes a {k}x{k} R, got {R.shape}")
    arrays = [np.asarray(a) for a in panels]
    host_dtype = arrays[0].dtype if arrays else np.dtype(np.complex128)
    if host_dtype not in (np.complex128, np.complex64):
        raise ArgumentError(f"host panels are ComplexF64 or ComplexF32, got {host_dtype}")
    for a in arrays:
        if a.dtype != host_dtype or a.ndim != 2 or a.shape[0] != N or not a.flags.f_contiguous:
            raise DimensionMismatch(f"a host panel of an {N}-row matrix must be N x w column major of one eltype, "
                                    f"got {a.shape} {a.dtype}")
    if sum(a.shape[1] for a in arrays) != k:
        raise DimensionMismatch(f"the panels hold {sum(a.shape[1] for a in arrays)} columns, the matrix {k}")
    host_type = _lib.FB_C128 if host_dtype == np.complex128 else _lib.FB_C64
    n = len(arrays)
    ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in arrays])
    lds = (ctypes.c_int64 * n)(*[N for _ in arrays])
    cols = (ctypes.c_int * n)(*[a.shape[1] for a in arrays])
    need = ctypes.c_size_t(0)
    call("fb_zcholqr2_staged_workspace_size", ctypes.c_int64(N), k, host_type, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    lib = _lib.load()
    info = ctypes.c_int(0)
    passes = ctypes.c_int(0)
    try:
        status = lib.fb_zcholqr2_staged(ptrs, host_type, lds, cols, n, _vp(D.ptr), D.ld, N, k, _vp(R.ptr), R.ld,
                                        float(unit_roundoff), ctypes.byref(info), ctypes.byref(passes), _vp(ws),
                                        ws_bytes, backend.queue_handle())
        shifts = (ctypes.c_double * 3)()
        if status == _lib.FB_OK:
            status = lib.fb_zcholqr2_query(_vp(ws), None, None, shifts)
    finally:
        backend.workspace_release()
    if status == _lib.FB_ENOTSPD:
        raise NotPositiveDefinite(_lib.last_error())
    _lib.check(status, "cholqr2!")
    return passes.value, tuple(shifts)


def ghost_fill(backend, dst: DeviceMatrix, row0: int, col0: int, seed: int, value_dtype) -> DeviceMatrix:
    """The device fill behind GhostPanels (generate_panel!, src/ghosts.jl:97-103,
    plus the upload that followed it): dst <- the ghost block whose top left
    entry is (row0, col0) of the matrix seeded by `seed`, its values rounded to
    `value_dtype` (the host storage eltype) and stored in dst's eltype."""
    if not isinstance(dst, DeviceMatrix):
        raise ArgumentError(f"the ghost fill writes a device matrix, got {type(dst).__name__}")
    if dst.size == 0:
        return dst
    call("fb_ghost_fill", _vp(dst.ptr), eltype_code(dst.dtype), ctypes.c_int64(dst.ld), ctypes.c_int64(dst.rows),
         ctypes.c_int64(dst.cols), ctypes.c_int64(row0), ctypes.c_int64(col0),
         ctypes.c_uint64(int(seed) & 0xFFFFFFFFFFFFFFFF), eltype_code(value_dtype), backend.queue_handle())
    return dst


def laplace7_apply(backend, dst: DeviceMatrix, src: DeviceMatrix, grid, shift) -> DeviceMatrix:
    """dst <- (-Lap_7 + shift I) src, column by column, on the grid (nx, ny, nz):
    the matrix-free operator of the streamed range finder."""
    _need_complex128(dst, src)
    nx, ny, nz = (int(g) for g in grid)
    n = nx * ny * nz
    if src.rows != n or tuple(dst.shape) != tuple(src.shape):
        raise DimensionMismatch(f"the {nx}x{ny}x{nz} Laplacian maps {n}-row panels, got {src.shape} -> {dst.shape}")
    if dst.size == 0:
        return dst
    call("fb_zlaplace7_apply", _vp(dst.ptr), ctypes.c_int64(dst.ld), _vp(src.ptr), ctypes.c_int64(src.ld),
         nx, ny, nz, dst.cols, z128(shift), backend.queue_handle())
    return dst


BATCH_SCHEDULES = ("auto", "persistent", "lanes")


def batch_schedule(shapes, form: str = "fp64", schedule: str = "auto") -> str:
    """The schedule a batch of (N, k) runs on: "persistent" (one persistent
    kernel launch for the whole batch; FP64 form, every k <= 64) or "lanes"
    (each instance's chain on one of eight forked streams, any k, either
    form). "auto" takes the persistent kernel wherever it applies."""
    if schedule not in BATCH_SCHEDULES:
        raise ArgumentError(f"a batch schedule is one of {BATCH_SCHEDULES}, got {schedule!r}")
    fits = form == "fp64" and all(int(k) <= 64 for _, k in shapes)
    if schedule == "persistent" and not fits:
        raise ArgumentError("the persistent batch kernel runs the FP64 form with every k <= 64")
    if schedule == "auto":
        return "persistent" if fits else "lanes"
    return schedule


def cholqr2_batched_workspace_bytes(shapes, form: str = "fp64", schedule: str = "auto") -> int:
    """Device scratch for a batch of cholqr2! instances of the given (N, k)
    on the schedule `batch_schedule` picks."""
    n = len(shapes)
    Ns = (ctypes.c_int64 * max(n, 1))(*[int(s[0]) for s in shapes])
    ks = (ctypes.c_int * max(n, 1))(*[int(s[1]) for s in shapes])
    need = ctypes.c_size_t(0)
    entry = ("fb_zcholqr2_batched_persistent_workspace_size"
             if batch_schedule(shapes, form, schedule) == "persistent" else "fb_zcholqr2_batched_workspace_size")
    call(entry, ctypes.cast(Ns, ctypes.c_void_p), ctypes.cast(ks, ctypes.c_void_p), n, ctypes.byref(need))
    return need.value


def cholqr2_batched(backend, Ys, Rs, form: str = "fp64", wait: bool = True, workspace=None,
                    schedule: str = "auto"):
    """cholqr2! of many independent device matrices Ys[i] (N_i x k_i), R_i into
    Rs[i], enqueued on the current queue as one persistent kernel launch or on
    eight stream lanes (`schedule`, see batch_schedule). With wait=True it
    returns the list of passes and raises NotPositiveDefinite if an instance's
    Gram stayed indefinite. `workspace` = (pointer, bytes) of caller-owned
    scratch, which a captured graph needs (the backend's shared scratch may
    move), sized by cholqr2_batched_workspace_bytes with the same form and
    schedule; by default the backend's is used."""
    if form not in ("fp64", "tc"):
        raise ArgumentError(f"cholqr2! form is 'fp64' or 'tc', got {form!r}")
    if len(Ys) != len(Rs):
        raise DimensionMismatch(f"a batch needs one R per Y, got {len(Ys)} and {len(Rs)}")
    n = len(Ys)
    for Y, R in zip(Ys, Rs):
        _need_complex128(Y, R)
        if R.shape != (Y.cols, Y.cols):
            raise DimensionMismatch(f"cholqr2! of an {Y.shape} matrix writes a {Y.cols}x{Y.cols} R, got {R.shape}")
    if n == 0:
        return []
    shapes = [Y.shape for Y in Ys]
    schedule = batch_schedule(shapes, form, schedule)
    arr = lambda ctype, vals: (ctype * n)(*vals)
    Yp = arr(ctypes.c_void_p, [Y.ptr for Y in Ys])
    ldy = arr(ctypes.c_int64, [Y.ld for Y in Ys])
    Ns = arr(ctypes.c_int64, [Y.rows for Y in Ys])
    ks = arr(ctypes.c_int, [Y.cols for Y in Ys])
    Rp = arr(ctypes.c_void_p, [R.ptr for R in Rs])
    ldr = arr(ctypes.c_int64, [R.ld for R in Rs])
    cast = lambda a: ctypes.cast(a, ctypes.c_void_p)
    own = workspace is None
    if own:
        ws, ws_bytes = backend.workspace(cholqr2_batched_workspace_bytes(shapes, form, schedule))
    else:
        ws, ws_bytes = workspace
    lib = _lib.load()
    try:
        if schedule == "persistent":
            status = lib.fb_zcholqr2_batched_persistent(cast(Yp), cast(ldy), cast(Ns), cast(ks), cast(Rp),
                                                        cast(ldr), n, _vp(ws), ws_bytes, backend.queue_handle())
        else:
            status = lib.fb_zcholqr2_batched(cast(Yp), cast(ldy), cast(Ns), cast(ks), cast(Rp), cast(ldr), n,
                                             1 if form == "tc" else 0, _vp(ws), ws_bytes, backend.queue_handle())
    finally:
        if own:
            backend.workspace_release()
    _lib.check(status, "cholqr2! batch")
    if not wait:
        return None
    if backend.current_queue is not None:
        backend.sync_queue(backend.current_queue)
    else:
        backend.sync_all()
    info = (ctypes.c_int * n)()
    passes = (ctypes.c_int * n)()
    status = lib.fb_zcholqr2_batched_query(_vp(ws), n, cast(info), cast(passes))
    if status == _lib.FB_ENOTSPD:
        raise NotPositiveDefinite(_lib.last_error())
    _lib.check(status, "cholqr2! batch")
    return list(passes)


# ---- differentiation: the pullbacks of cholqr2! and project ---------------------

def cholqr2_adjoint(backend, Ybar: DeviceMatrix, Y: DeviceMatrix, R: DeviceMatrix,
                    Qbar: DeviceMatrix | None = None, Rbar: DeviceMatrix | None = None) -> DeviceMatrix:
    """The pullback of (Q, R) = cholqr2!(Y): Ybar <- (Qbar + Q H) R^-H with
    H = copyltu(R Rbar^H - Qbar^H Q), Q recomputed from the original Y and R
    inside the products. Qbar or Rbar None is a zero cotangent; Ybar may be
    Qbar itself."""
    _need_complex128(Ybar, Y, R, *(m for m in (Qbar, Rbar) if m is not None))
    N, k = Y.shape
    if Ybar.shape != (N, k) or R.shape != (k, k):
        raise DimensionMismatch(f"the cholqr2! pullback of an {N}x{k} Y takes a {k}x{k} R and writes an {N}x{k} "
                                f"Ybar, got R {R.shape} and Ybar {Ybar.shape}")
    if Qbar is not None and Qbar.shape != (N, k):
        raise DimensionMismatch(f"Qbar must be {N}x{k}, got {Qbar.shape}")
    if Rbar is not None and Rbar.shape != (k, k):
        raise DimensionMismatch(f"Rbar must be {k}x{k}, got {Rbar.shape}")
    if Ybar.size == 0:
        return Ybar
    need = ctypes.c_size_t(0)
    call("fb_zcholqr2_adjoint_workspace_size", ctypes.c_int64(N), k, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    try:
        call("fb_zcholqr2_adjoint", _vp(Ybar.ptr), Ybar.ld, _vp(Y.ptr), Y.ld, _vp(R.ptr), R.ld,
             _vp(Qbar.ptr if Qbar is not None else None), Qbar.ld if Qbar is not None else 0,
             _vp(Rbar.ptr if Rbar is not None else None), Rbar.ld if Rbar is not None else 0,
             ctypes.c_int64(N), k, _vp(ws), ws_bytes, backend.queue_handle())
    finally:
        backend.workspace_release()
    return Ybar


def project_adjoint(backend, Qbar: DeviceMatrix, GQ: DeviceMatrix, Sbar: DeviceMatrix,
                    GhQ: DeviceMatrix | None = None, accumulate: bool = False) -> DeviceMatrix:
    """The pullback of S = project(Q, G) = Q^H (G Q) with respect to Q:
    Qbar <- [Qbar +] (G Q) Sbar^H + (G^H Q) Sbar, from the operator images
    GQ and GhQ; GhQ None means G is Hermitian."""
    _need_complex128(Qbar, GQ, Sbar, *(m for m in (GhQ,) if m is not None))
    N, k = GQ.shape
    if Qbar.shape != (N, k) or Sbar.shape != (k, k) or (GhQ is not None and GhQ.shape != (N, k)):
        raise DimensionMismatch(f"the project pullback maps a {k}x{k} Sbar and {N}x{k} images to an {N}x{k} Qbar, "
                                f"got Sbar {Sbar.shape}, Qbar {Qbar.shape}")
    if Qbar.size == 0:
        return Qbar
    need = ctypes.c_size_t(0)
    call("fb_zproject_adjoint_workspace_size", k, ctypes.byref(need))
    ws, ws_bytes = backend.workspace(need.value)
    try:
        call("fb_zproject_adjoint", _vp(Qbar.ptr), Qbar.ld, _vp(GQ.ptr), GQ.ld,
             _vp(GhQ.ptr if GhQ is not None else None), GhQ.ld if GhQ is not None else 0,
             _vp(Sbar.ptr), Sbar.ld, ctypes.c_int64(N), k, 1 if accumulate else 0, _vp(ws), ws_bytes,
             backend.queue_handle())
    finally:
        backend.workspace_release()
    return Qbar


def hband_apply(backend, dst: DeviceMatrix, src: DeviceMatrix, Dg: DeviceMatrix) -> DeviceMatrix:
    """dst <- G src for the Hermitian band G stored by diagonals in Dg
    (N x (kd + 1), column d the d-th superdiagonal)."""
    _need_complex128(dst, src, Dg)
    N = Dg.rows
    if src.rows != N or tuple(dst.shape) != tuple(src.shape):
        raise DimensionMismatch(f"a {N}x{N} band operator maps {N}-row panels, got {src.shape} -> {dst.shape}")
    if dst.size == 0:
        return dst
    call("fb_zhband_apply", _vp(dst.ptr), ctypes.c_int64(dst.ld), _vp(src.ptr), ctypes.c_int64(src.ld),
         _vp(Dg.ptr), ctypes.c_int64(Dg.ld), ctypes.c_int64(N), Dg.cols - 1, dst.cols, backend.queue_handle())
    return dst
