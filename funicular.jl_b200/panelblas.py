"""The panel BLAS on the B200 backend (src/panelblas.jl): gram, panelmul!,
cholqr2!, project, rightmul!, with the reference's traversals and
accumulation rules, and the device-resident cholqr2! where the matrix fits.
"""
from __future__ import annotations

import numpy as np

from . import kernels
from ._lib import ArgumentError, DimensionMismatch
from .device_api import DeviceMatrix
from .executor import PanelSteps, RowSteps, readpanels, rowtraversal, sweep, updatepanels, writepanels
from .panels import PanelMatrix, assert_conformal, assert_same_panels, assert_same_rows, from_device, to_device
from .plan import checkin_device_buffers, checkout_device_buffers, row_block_height


def shared_plan(X: PanelMatrix, Y: PanelMatrix):
    """shared_plan (src/panelblas.jl:4-8)."""
    if X.dtype != Y.dtype:
        raise ArgumentError(f"panel matrices in one operation must share their compute eltype, got {X.dtype} and "
                            f"{Y.dtype}. Narrowing belongs on the storage tiers, not here")
    if X.plan is not Y.plan:
        raise ArgumentError("panel matrices in one operation must belong to the same ResidencyPlan, since the plan "
                            "is what owns the staging buffers the operation runs through. Build both matrices from "
                            "one plan")
    return X.plan


def carry(step: int) -> complex:
    """carry (src/panelblas.jl:59): the first step overwrites, later ones add."""
    return 0.0 if step == 0 else 1.0


def collect_small(device: DeviceMatrix, plan) -> np.ndarray:
    """collect_small (src/panelblas.jl:61-65)."""
    host = np.empty(device.shape, dtype=device.dtype, order="F")
    plan.backend.d2h(host, device)
    return host


def gram(X: PanelMatrix, Y: PanelMatrix | None = None, *, nbuffers=None) -> np.ndarray:
    """gram(X[, Y]; nbuffers) (src/panelblas.jl:33-53): X^H Y accumulated on
    the device one row block at a time, copied to the host once."""
    Y = X if Y is None else Y
    plan = shared_plan(X, Y)
    assert_conformal(X, Y)
    backend = plan.backend
    (acc,) = checkout_device_buffers(plan, X.dtype, (X.k, X.k), 1)
    try:
        traversal = rowtraversal(X)
        if X is Y:
            sweep(lambda step, Xb: kernels.gram_accumulate(backend, acc, Xb, Xb, 1.0, carry(step)),
                  readpanels(X), nbuffers=nbuffers, traversal=traversal)
        else:
            sweep(lambda step, Xb, Yb: kernels.gram_accumulate(backend, acc, Xb, Yb, 1.0, carry(step)),
                  readpanels(X), readpanels(Y), nbuffers=nbuffers, traversal=traversal)
        return collect_small(acc, plan)
    finally:
        checkin_device_buffers(plan, [acc])


# ---- operators (src/operator.jl) -------------------------------------------

class DeviceOperator:
    """A linear operator applied to device panels. `apply(backend, dst, src)`
    writes G src into dst on the backend's current queue; an operator that is
    panel-capable takes a whole N x w panel, otherwise it is applied one
    column at a time (apply_operator!, src/operator.jl:80-87)."""

    panel_capable = True
    shape = (0, 0)
    # Whether G^H = G, which lets the pullback of project skip applying G^H.
    hermitian = False

    def apply(self, backend, dst: DeviceMatrix, src: DeviceMatrix):
        raise NotImplementedError

    def adjoint(self) -> "DeviceOperator":
        """G^H, which the pullback of project applies when G is not Hermitian."""
        if self.hermitian:
            return self
        raise ArgumentError(f"{type(self).__name__} has no adjoint; the pullback of project needs G^H")


class DenseOperator(DeviceOperator):
    """A dense m x n matrix resident on the device; applying it is the
    backend's product kernel."""

    def __init__(self, backend, G: np.ndarray):
        G = np.asfortranarray(np.asarray(G, dtype=np.complex128))
        self.backend = backend
        self.host = G
        self.G = backend.todevice(G)
        self.shape = G.shape
        self.hermitian = G.shape[0] == G.shape[1] and bool(np.array_equal(G, G.conj().T))

    def apply(self, backend, dst, src):
        kernels.rightmul_gemm(backend, dst, self.G, src)

    def adjoint(self):
        return self if self.hermitian else DenseOperator(self.backend, self.host.conj().T)


class Laplacian7(DeviceOperator):
    """G = -Lap_7 + shift I on an nx x ny x nz grid, matrix-free on the device
    (the operator of the streamed range finder): grid point (x, y, z) is row
    x + nx (y + ny z), unit spacing, zero outside the grid."""

    def __init__(self, grid, shift=0.0):
        self.grid = tuple(int(g) for g in grid)
        if len(self.grid) != 3 or min(self.grid) < 1:
            raise ArgumentError(f"a 7-point Laplacian needs a 3-D grid of positive sizes, got {grid}")
        self.shift = complex(shift)
        n = self.grid[0] * self.grid[1] * self.grid[2]
        self.shape = (n, n)

    def apply(self, backend, dst, src):
        kernels.laplace7_apply(backend, dst, src, self.grid, self.shift)

    @property
    def hermitian(self):
        return self.shift.imag == 0

    def adjoint(self):
        return Laplacian7(self.grid, self.shift.conjugate())


class HermitianBand(DeviceOperator):
    """A Hermitian N x N operator with kd superdiagonals, held on the device
    by diagonals: Dg is N x (kd + 1) with Dg[i, d] = G[i, i + d] (the imaginary
    part of the main diagonal and the entries past the matrix are ignored).
    The operator of the differentiation workload."""

    hermitian = True

    def __init__(self, backend, Dg):
        if isinstance(Dg, DeviceMatrix):
            self.Dg = Dg
        else:
            Dg = np.asfortranarray(np.asarray(Dg, dtype=np.complex128))
            if Dg.ndim != 2 or Dg.shape[1] < 1:
                raise ArgumentError(f"band storage is N x (kd + 1), got shape {Dg.shape}")
            self.Dg = backend.todevice(Dg)
        self.kd = self.Dg.cols - 1
        self.shape = (self.Dg.rows, self.Dg.rows)

    @classmethod
    def ghost(cls, backend, N: int, kd: int, seed: int, scale: float = 1.0) -> "HermitianBand":
        """The seeded band: entry (i, d) of the storage is scale times the
        complex Gaussian of a ComplexF64 GhostPanels matrix (seed) at row i,
        column d, filled on the device."""
        Dg = backend.alloc_device(np.complex128, (N, kd + 1))
        kernels.ghost_fill(backend, Dg, 0, 0, seed, np.complex128)
        if scale != 1.0:
            S = backend.todevice(np.eye(kd + 1, dtype=np.complex128) * scale)
            out = backend.alloc_device(np.complex128, (N, kd + 1))
            kernels.rightmul_gemm(backend, out, Dg, S)
            Dg = out
        return cls(backend, Dg)

    def apply(self, backend, dst, src):
        kernels.hband_apply(backend, dst, src, self.Dg)


class ColumnOperator(DeviceOperator):
    """Wraps an operator so it is applied column by column (the reference's
    ColumnOperator test wrapper, test/operators.jl)."""

    panel_capable = False

    def __init__(self, inner: DeviceOperator):
        self.inner = inner
        self.shape = inner.shape

    def apply(self, backend, dst, src):
        self.inner.apply(backend, dst, src)

    @property
    def hermitian(self):
        return self.inner.hermitian

    def adjoint(self):
        return self if self.hermitian else ColumnOperator(self.inner.adjoint())


def apply_operator(backend, Y: DeviceMatrix, G: DeviceOperator, X: DeviceMatrix):
    """apply_operator! / columnwise_apply! (src/operator.jl:80-87)."""
    if G.panel_capable:
        G.apply(backend, Y, X)
    else:
        for c in range(X.cols):
            G.apply(backend, Y.view(slice(None), slice(c, c + 1)), X.view(slice(None), slice(c, c + 1)))
    return Y


def assert_operator_shape(G, m, n):
    """assert_operator_shape (src/operator.jl:74-78)."""
    rows, cols = G.shape
    if (rows, cols) != (m, n):
        raise ArgumentError(f"operator is {rows}x{cols} but it reads columns of an {n}-row matrix and writes columns "
                            f"of an {m}-row one, so it has to be {m}x{n}. Either the operator or one of the two "
                            "matrices has the wrong row count")


def assert_square_operator(G, N):
    """assert_square_operator (src/operator.jl:68-72)."""
    rows, cols = G.shape
    if not rows == cols == N:
        raise ArgumentError(f"operator is {rows}x{cols} but the panel matrices have {N} rows. Funicular applies an "
                            "operator to whole columns, so it must be square and match N")


def panelmul(Y: PanelMatrix, G: DeviceOperator, X: PanelMatrix, *, nbuffers=None) -> PanelMatrix:
    """panelmul!(Y, G, X; nbuffers) (src/panelblas.jl:91-100)."""
    plan = shared_plan(X, Y)
    if X is Y:
        raise ArgumentError("panelmul! cannot write its output over its input: the operator is applied panel by "
                            "panel and would read columns it has already overwritten")
    assert_same_panels(X, Y)
    assert_operator_shape(G, Y.N, X.N)
    backend = plan.backend
    sweep(lambda j, Xb, Yb: apply_operator(backend, Yb, G, Xb), readpanels(X), writepanels(Y), nbuffers=nbuffers)
    return Y


# ---- cholqr2! (src/panelblas.jl:130-169) --------------------------------------

def cholesky_upper(plan, G_dev: DeviceMatrix, N: int, k: int, U_dev: DeviceMatrix, forced_unit_roundoff=None):
    """The device hook standing in for cholesky_upper (src/panelblas.jl:148-155):
    returns shifted, with U_dev holding the factor. forced_unit_roundoff
    shifts at once (the first pass of the shifted CholeskyQR3)."""
    shifted, _ = kernels.cholesky_upper_device(plan.backend, G_dev, N, k, U_dev,
                                               forced_unit_roundoff=forced_unit_roundoff)
    return shifted


def gram_rows(Y: PanelMatrix, G_dev: DeviceMatrix, *, nbuffers=None) -> DeviceMatrix:
    """The Gram sweep of cholqr_pass! (src/panelblas.jl:143): G = Y^H Y
    accumulated over row blocks, first block overwriting."""
    backend = Y.plan.backend
    sweep(lambda step, Yb: kernels.gram_accumulate(backend, G_dev, Yb, Yb, 1.0, carry(step)),
          readpanels(Y), nbuffers=nbuffers, traversal=rowtraversal(Y))
    return G_dev


def rdiv_rows(Y: PanelMatrix, R_dev: DeviceMatrix, *, nbuffers=None, next_gram: DeviceMatrix | None = None) -> PanelMatrix:
    """rdiv_rows! (src/panelblas.jl:157-169) with the factor already on the
    device. With next_gram, each solved row block, still on the device, is
    also accumulated into next_gram as the next pass's Gram sweep would
    accumulate it after reading the block back: the same blocks in the same
    order with the same first-step overwrite, so the same bits, one upload
    sweep fewer."""
    backend = Y.plan.backend

    def solve(step, Yb):
        kernels.rdiv_upper(backend, Yb, R_dev)
        if next_gram is not None:
            kernels.gram_accumulate(backend, next_gram, Yb, Yb, 1.0, carry(step))

    sweep(solve, updatepanels(Y), nbuffers=nbuffers, traversal=rowtraversal(Y))
    return Y


def solves_what_it_stores(Y: PanelMatrix) -> bool:
    """Whether a row block on the device after the solve holds exactly what
    the host panels will hold: true unless the host tier narrows (a
    ComplexF32 tier rounds the block on its way down, and the next pass's
    Gram is of the rounded values)."""
    from .panels import host_storage_eltype
    return np.dtype(host_storage_eltype(Y.plan, Y.dtype)) == np.dtype(Y.dtype)


def cholqr2_streamed(Y: PanelMatrix, *, nbuffers=None, forced_unit_roundoff=None) -> np.ndarray:
    """cholqr2! through row sweeps (src/panelblas.jl:130-146): two passes, a
    third when either of the first two shifted, each pass
    (cholqr_pass!, src/panelblas.jl:141-146) a Gram, its factor and the
    solve, the k x k factor staying on the device. The first Gram is its own
    sweep; a later pass's Gram is taken inside the previous pass's solve
    sweep when the host tier stores the solved blocks unrounded, else by a
    sweep of its own as the reference takes it. A pass knows whether another
    follows once its factor is known, before its solve: a fourth never runs.
    With forced_unit_roundoff the first pass is shifted at once, so all three
    run: the shifted CholeskyQR3. When a factor fails, Y holds the previous
    pass's Q."""
    Y.assert_writable()
    plan = Y.plan
    fuse = solves_what_it_stores(Y)
    G_dev, U_dev = checkout_device_buffers(plan, Y.dtype, (Y.k, Y.k), 2)
    try:
        gram_rows(Y, G_dev, nbuffers=nbuffers)
        R, npasses, p = None, 2, 0
        while p < npasses:
            if cholesky_upper(plan, G_dev, Y.N, Y.k, U_dev, forced_unit_roundoff if p == 0 else None):
                npasses = 3
            more = p + 1 < npasses
            rdiv_rows(Y, U_dev, nbuffers=nbuffers, next_gram=G_dev if more and fuse else None)
            if more and not fuse:
                gram_rows(Y, G_dev, nbuffers=nbuffers)
            Rp = collect_small(U_dev, plan)
            R = Rp if R is None else Rp @ R
            p += 1
        return R
    finally:
        checkin_device_buffers(plan, [G_dev, U_dev])


def fits_on_device(Y: PanelMatrix) -> bool:
    """Whether the whole matrix, its R and the chain's scratch fit in what the
    plan's device pool has left."""
    from .plan import device_bytes_to_add
    pool = Y.plan.devicepool
    need = (device_bytes_to_add(Y.plan, Y.dtype, [((Y.N, Y.k), 1), ((Y.k, Y.k), 1)])
            + kernels.cholqr2_workspace_bytes(Y.N, Y.k))
    return pool.allocated + need <= pool.budget


def cholqr2_resident(Y: PanelMatrix, form: str = "fp64", unit_roundoff=None) -> np.ndarray:
    """The backend's cholqr2! when Y fits on the device: every panel goes up
    once, the whole two- or three-pass chain runs on the device
    (kernels.cholqr2_resident), Q comes back down once. Two host-device
    crossings of the matrix instead of the five of the streamed form. When a
    Gram matrix stays indefinite the error is raised before anything is
    written back, so Y keeps its values."""
    plan = Y.plan
    backend = plan.backend
    (D,) = checkout_device_buffers(plan, Y.dtype, (Y.N, Y.k), 1)
    (Rd,) = checkout_device_buffers(plan, Y.dtype, (Y.k, Y.k), 1)
    try:
        q = backend.make_queue()
        for p in Y.panels:
            if p.hold is not None:
                backend.wait_event(q, p.hold)
        from .panels import host_storage_eltype
        S = np.dtype(host_storage_eltype(plan, Y.dtype))
        if form in ("fp64", "shifted3") and Y.dtype == np.complex128 and S in (np.complex128, np.complex64):
            # The staged form: the upload overlaps the first Gram and the
            # download the last solve, narrow tiers widened and narrowed on
            # the device block by block.
            u = 0.0 if form == "fp64" else (unit_roundoff if unit_roundoff is not None
                                            else kernels.UNIT_ROUNDOFF[np.dtype(np.complex128)])
            backend.submit(q, lambda: kernels.cholqr2_staged(backend, [p.storage() for p in Y.panels], D, Rd,
                                                             unit_roundoff=u))
            R = np.empty((Y.k, Y.k), dtype=Y.dtype, order="F")
            backend.d2h(R, Rd, queue=q)
            backend.sync_queue(q)
            for p in Y.panels:
                p.hold = None
                p.dirty = True
                p.epoch += 1
            return R
        to_device(Y, D, q)
        # Waits for the chain and raises NotPositiveDefinite if it stopped.
        extra = {} if unit_roundoff is None else {"unit_roundoff": unit_roundoff}
        backend.submit(q, lambda: kernels.cholqr2_resident(backend, D, Rd, wait=True, form=form, **extra))
        from_device(Y, D, q)
        R = np.empty((Y.k, Y.k), dtype=Y.dtype, order="F")
        backend.d2h(R, Rd, queue=q)
        backend.sync_queue(q)
        for p in Y.panels:
            p.hold = None
        return R
    finally:
        checkin_device_buffers(plan, [D, Rd])


def cholqr2(Y: PanelMatrix, *, nbuffers=None, resident=None) -> np.ndarray:
    """cholqr2!(Y; nbuffers) (src/panelblas.jl:130-139): Y becomes Q in place
    and R (k x k, host) comes back. Device-resident when Y fits the plan's
    device budget, streamed through row sweeps otherwise; `resident` forces
    one or the other."""
    Y.assert_writable()
    if resident is None:
        resident = fits_on_device(Y)
    if resident:
        return cholqr2_resident(Y)
    return cholqr2_streamed(Y, nbuffers=nbuffers)


def storage_unit_roundoff(Y: PanelMatrix) -> float:
    """The unit roundoff of what Y holds between passes: its host storage
    eltype's (ComplexF32 for a narrowed tier), else the compute eltype's."""
    from .panels import host_storage_eltype
    S = host_storage_eltype(Y.plan, Y.dtype)
    return kernels.UNIT_ROUNDOFF.get(np.dtype(S), kernels.UNIT_ROUNDOFF[np.dtype(np.complex128)])


def cholqr3(Y: PanelMatrix, *, nbuffers=None, resident=None, unit_roundoff=None) -> np.ndarray:
    """The shifted CholeskyQR3 (Fukaya et al., SIAM J. Sci. Comput. 2020), the
    north-star addition for the ComplexF32 storage tier: Y becomes Q in place
    and R = R3 R2 R1 comes back. Pass 1 factors G + s I with
    s = 11 (N k + k (k+1)) u ||G||_F whatever G's definiteness, passes 2 and
    3 are plain. u defaults to the unit roundoff of Y's storage (2^-24 for a
    ComplexF32 host tier, 2^-53 otherwise). Device-resident when Y fits,
    streamed through row sweeps otherwise, like cholqr2."""
    Y.assert_writable()
    u = storage_unit_roundoff(Y) if unit_roundoff is None else float(unit_roundoff)
    if resident is None:
        resident = fits_on_device(Y)
    if resident:
        return cholqr2_resident(Y, form="shifted3", unit_roundoff=u)
    return cholqr2_streamed(Y, nbuffers=nbuffers, forced_unit_roundoff=u)


# ---- project (src/panelblas.jl:268-301) ---------------------------------------

PROJECT_SCHEDULES = ("resident", "two-sweep", "nested")


def project_schedule(Q: PanelMatrix) -> str:
    """The cheapest project schedule the plan affords: 'resident' when Q and
    G Q fit the device budget together (Q crosses the bus once), 'two-sweep'
    when the host has room for an N x k matrix Z (panelmul!(Z, G, Q) then
    gram(Q, Z), src/panelblas.jl:250-261: three crossings of the matrix),
    else the reference's nested schedule (p (p + 1) panel uploads)."""
    from .panels import host_storage_eltype
    from .plan import device_bytes_to_add, host_bytes_in_use
    pool = Q.plan.devicepool
    if pool.allocated + device_bytes_to_add(Q.plan, Q.dtype, [((Q.N, Q.k), 2), ((Q.k, Q.k), 1)]) <= pool.budget:
        return "resident"
    host_bytes = Q.N * Q.k * np.dtype(host_storage_eltype(Q.plan, Q.dtype)).itemsize
    if Q.plan.hostpool.budget - host_bytes_in_use(Q.plan) >= host_bytes + 64 * Q.npanels():
        return "two-sweep"
    return "nested"


def project(Q: PanelMatrix, G: DeviceOperator, *, nbuffers=None, schedule=None) -> np.ndarray:
    """project(Q, G; nbuffers) (src/panelblas.jl:268-301): S = Q^H (G Q).
    schedule None takes project_schedule(Q); 'nested' is the reference's
    block-column schedule, 'two-sweep' its documented replacement when a
    second N x k matrix fits on the host (src/panelblas.jl:258-260,
    docs/src/porting.md:42-44), 'resident' the device-resident form: Q up
    once, G applied to all of Q, one cross Gram on the device."""
    assert_square_operator(G, Q.N)
    schedule = project_schedule(Q) if schedule is None else schedule
    if schedule not in PROJECT_SCHEDULES:
        raise ArgumentError(f"project schedule is one of {PROJECT_SCHEDULES}, got {schedule!r}")
    if schedule == "resident":
        return project_resident(Q, G)
    if schedule == "two-sweep":
        try:
            Z = PanelMatrix.undef(Q.dtype, Q.N, Q.k, plan=Q.plan, w=Q.w)
        except ArgumentError:
            # The host tier could not hold Z after all (its blocks are cut
            # for other sizes): the nested schedule needs no second matrix.
            return project_nested(Q, G, nbuffers=nbuffers)
        return project_two_sweep(Q, G, Z, nbuffers=nbuffers)
    return project_nested(Q, G, nbuffers=nbuffers)


def project_resident(Q: PanelMatrix, G: DeviceOperator) -> np.ndarray:
    """Q^H (G Q) with Q and G Q resident: every panel goes up once (a ghost is
    generated on the device), the operator is applied to the whole N x k
    matrix, and one cross Gram forms S."""
    plan = Q.plan
    backend = plan.backend
    D, Z = checkout_device_buffers(plan, Q.dtype, (Q.N, Q.k), 2)
    (acc,) = checkout_device_buffers(plan, Q.dtype, (Q.k, Q.k), 1)
    try:
        q = backend.make_queue()
        for p in Q.panels:
            if p.hold is not None:
                backend.wait_event(q, p.hold)
        to_device(Q, D, q)

        def work():
            apply_operator(backend, Z, G, D)
            kernels.gram_accumulate(backend, acc, D, Z, 1.0, 0.0)

        backend.submit(q, work)
        S = np.empty((Q.k, Q.k), dtype=Q.dtype, order="F")
        backend.d2h(S, acc, queue=q)
        backend.sync_queue(q)
        return S
    finally:
        checkin_device_buffers(plan, [D, Z, acc])


def project_two_sweep(Q: PanelMatrix, G: DeviceOperator, Z: PanelMatrix, *, nbuffers=None) -> np.ndarray:
    """panelmul!(Z, G, Q) into the host matrix Z (cut like Q), then
    gram(Q, Z): two sweeps (src/panelblas.jl:258-260); Z is given back
    afterwards."""
    from .panels import free
    try:
        panelmul(Z, G, Q, nbuffers=nbuffers)
        return gram(Q, Z, nbuffers=nbuffers)
    finally:
        free(Z)


def project_nested(Q: PanelMatrix, G: DeviceOperator, *, nbuffers=None) -> np.ndarray:
    """The reference's schedule: Q^H (G Q) block column by block column,
    p(p+1) steps, one extra N x w image buffer."""
    plan = Q.plan
    backend = plan.backend
    p = Q.npanels()
    panels, labels = [], []
    for j in range(p):
        panels.append(j)
        labels.append((True, j, j))
        for i in range(p):
            panels.append(i)
            labels.append((False, i, j))
    (image,) = checkout_device_buffers(plan, Q.dtype, (Q.N, Q.w), 1)
    (acc,) = checkout_device_buffers(plan, Q.dtype, (Q.k, Q.k), 1)
    try:
        def step(label, Qb):
            applying, i, j = label
            GQj = image.view(slice(None), slice(0, Q.panelwidth(j)))
            if applying:
                apply_operator(backend, GQj, G, Qb)
            else:
                ri, rj = Q.panelrange(i), Q.panelrange(j)
                block = acc.view(slice(ri.start, ri.stop), slice(rj.start, rj.stop))
                kernels.gram_accumulate(backend, block, Qb, GQj, 1.0, 0.0)

        sweep(step, readpanels(Q), nbuffers=nbuffers, traversal=PanelSteps(panels, labels))
        return collect_small(acc, plan)
    finally:
        checkin_device_buffers(plan, [image, acc])


# ---- rightmul! (src/panelblas.jl:203-245) -------------------------------------

def rightmul(dest: PanelMatrix, src: PanelMatrix | np.ndarray, C=None, *, nbuffers=None) -> PanelMatrix:
    """rightmul!(Y, C) in place (k x k C) or rightmul!(dest, src, C)."""
    if C is None:
        Y, C = dest, np.asarray(src)
        if C.shape != (Y.k, Y.k):
            raise ArgumentError(f"rightmul!(Y, C) writes the product back into Y, which has {Y.k} columns and "
                                f"cannot grow or shrink, so C must be {Y.k}x{Y.k}, got {C.shape}. Use "
                                "rightmul!(dest, Y, C) when the column count changes")
        plan = Y.plan
        backend = plan.backend
        traversal = rowtraversal(Y)
        (factor,) = checkout_device_buffers(plan, Y.dtype, (Y.k, Y.k), 1)
        (scratch,) = checkout_device_buffers(plan, Y.dtype, traversal.buffer_dims(Y), 1)
        try:
            backend.h2d(factor, np.asfortranarray(C.astype(Y.dtype)))

            def step(_, Yb):
                product = scratch.view(slice(0, Yb.rows), slice(None))
                kernels.rightmul_gemm(backend, product, Yb, factor)
                kernels.convert_copy(backend, Yb, product)

            sweep(step, updatepanels(Y), nbuffers=nbuffers, traversal=traversal)
        finally:
            checkin_device_buffers(plan, [factor, scratch])
        return Y
    if dest is src:
        raise ArgumentError("rightmul!(dest, src, C) needs two different matrices, since one of them streams up "
                            "while the other streams down and a single matrix cannot do both in one sweep")
    C = np.asarray(C)
    if C.shape != (src.k, dest.k):
        raise ArgumentError(f"rightmul!(dest, src, C) computes src * C, so C must be {src.k}x{dest.k}, got {C.shape}")
    plan = shared_plan(src, dest)
    assert_same_rows(src, dest)
    backend = plan.backend
    height = min(row_block_height(src.N, src.k, src.w), row_block_height(dest.N, dest.k, dest.w))
    (factor,) = checkout_device_buffers(plan, dest.dtype, (src.k, dest.k), 1)
    try:
        backend.h2d(factor, np.asfortranarray(C.astype(dest.dtype)))
        sweep(lambda _, sb, db: kernels.rightmul_gemm(backend, db, sb, factor), readpanels(src), writepanels(dest),
              nbuffers=nbuffers, traversal=RowSteps(src.N, height))
    finally:
        checkin_device_buffers(plan, [factor])
    return dest
