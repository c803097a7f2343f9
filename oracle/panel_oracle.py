"""CPU oracle for the panel linear algebra hot path.

TEST INFRASTRUCTURE ONLY. This module restates, in numpy and scipy's LAPACK,
what Funicular.jl's CPU reference backend computes for the functions on the
hot path, step for step in the reference's order. Only tests/, the smoke check
in __graft_entry__.py and bench.py's CPU-baseline leg may import it, and only
to check or time the reference's algorithm; the B200 backend never calls it.

Where the reference's arithmetic lives:
  * its own code: row-block traversal, the accumulation rule of gram, the pass
    structure and shift rule of cholqr2!, the step order of project. These
    are restated below, each function citing the lines it follows.
  * Julia's LinearAlgebra, which calls OpenBLAS and LAPACK (zgemm, ztrsm,
    zpotrf). No Manifest pins a version (Project.toml:34 asks for julia 1.10).
    The stand-in here is the OpenBLAS/LAPACK that scipy bundles; both are
    reference-LAPACK zpotrf/ztrsm semantics.

Parity pin. The reference publishes no golden vectors for this path; its own
tests check it against dense LinearAlgebra within blastol = 100 eps sqrt(N k)
and orthogonality_bound = 100 N k eps (test/setup.jl:170-172), and check
several results for bitwise equality. tests/test_oracle.py restates those
known-answer tests against this oracle, which is how the oracle is pinned.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.linalg.blas as blas
import scipy.linalg.lapack as lapack

EPS = {np.dtype(np.complex128): 2.0 ** -52, np.dtype(np.float64): 2.0 ** -52,
       np.dtype(np.complex64): 2.0 ** -23, np.dtype(np.float32): 2.0 ** -23}


class OracleArgumentError(ValueError):
    pass


# ---- plan arithmetic: src/plan.jl ------------------------------------------

def row_block_height(N: int, k: int, w: int) -> int:
    """row_block_height (src/plan.jl:133)."""
    return max(1, min(N, (N * w) // k))


def row_steps(N: int, height: int):
    """RowSteps(N, height) (src/executor.jl:33-36): unit ranges as (start, stop)."""
    h = max(1, min(int(height), int(N)))
    return [(top, min(top + h, N)) for top in range(0, N, h)]


def row_blocks(N: int, k: int, w: int):
    """rowtraversal (src/executor.jl:38)."""
    return row_steps(N, row_block_height(N, k, w))


def panel_ranges(k: int, w: int):
    """Column ranges of the panels of an N x k matrix cut at width w
    (src/panels.jl:66-69): ragged last panel."""
    return [(j * w, min((j + 1) * w, k)) for j in range((k + w - 1) // w)]


def choose_panel_width(N, k, itemsize, device_budget, nbuffers=2, extra_buffers=0,
                       workspace_bytes=0, target_panel_bytes=2 * 1024 ** 3):
    """choose_panel_width (src/plan.jl:112-123)."""
    if N <= 0:
        raise OracleArgumentError(f"N must be positive, got {N}")
    if k <= 0:
        raise OracleArgumentError(f"k must be positive, got {k}")
    buffers = nbuffers + extra_buffers
    if buffers < 1:
        raise OracleArgumentError("nbuffers + extra_buffers must be at least 1")
    column = N * itemsize
    available = int(math.floor(device_budget)) - int(math.floor(workspace_bytes))
    per_buffer = available // buffers
    if per_buffer < column:
        raise OracleArgumentError("device budget too small for one column")
    w = min(k, max(1, min(int(math.floor(target_panel_bytes)), per_buffer) // column))
    npanels = -(-k // w)
    return -(-k // npanels)


# ---- kernels: src/kernels.jl ------------------------------------------------

def gram_accumulate(C, A, B, alpha, beta):
    """gram_accumulate! (src/kernels.jl:22-55): C <- alpha A^H B + beta C, a
    zero beta overwriting C (NaN-safe)."""
    if A.shape[0] == 0:
        C[...] = 0 if beta == 0 else beta * C
        return C
    if np.iscomplexobj(A) and A.dtype == np.complex128:
        # mul!(C, A', B, alpha, beta) reaches zgemm('C', 'N', ...)
        out = blas.zgemm(alpha, A, B, beta=beta, c=None if beta == 0 else np.asfortranarray(C), trans_a=2)
        C[...] = out
        return C
    prod = A.conj().T @ B
    C[...] = alpha * prod if beta == 0 else alpha * prod + beta * C
    return C


def rdiv_upper(Y, R):
    """rdiv_upper! (src/kernels.jl:90-124) as rdiv!(Y, UpperTriangular(R)),
    which LinearAlgebra sends to BLAS ztrsm (Right, Upper, NoTrans, NonUnit)."""
    if Y.size == 0:
        return Y
    trsm = blas.ztrsm if np.iscomplexobj(Y) else blas.dtrsm
    if Y.flags.f_contiguous and Y.dtype == R.dtype:
        trsm(1.0, np.asfortranarray(R), Y, side=1, lower=0, trans_a=0, diag=0, overwrite_b=1)
    else:
        Y[...] = trsm(1.0, np.asfortranarray(R), np.asfortranarray(Y), side=1, lower=0, trans_a=0, diag=0)
    return Y


def rightmul_gemm(dst, A, C):
    """rightmul_gemm! (src/kernels.jl:57-88)."""
    dst[...] = A @ C
    return dst


# ---- panel BLAS: src/panelblas.jl --------------------------------------------

def _staging(h, cols, dtype):
    """A sweep's staging buffer (src/executor.jl:177-182): one row block,
    column major, as the CPU backend's "device" array."""
    return np.empty((h, cols), dtype=dtype, order="F")


def gram(X, Y=None, w=None):
    """gram(X[, Y]) (src/panelblas.jl:33-53): C = X^H Y accumulated one row
    block at a time, the first block overwriting (carry, :59). Each block is
    first copied into a staging buffer, as materialize_rows! does
    (src/panels.jl:437-445)."""
    N, k = X.shape
    w = k if w is None else w
    same = Y is None or Y is X
    Y = X if Y is None else Y
    C = np.empty((k, Y.shape[1]), dtype=X.dtype)
    blocks = row_blocks(N, k, w)
    h = blocks[0][1] - blocks[0][0]
    xs = _staging(h, k, X.dtype)
    ys = xs if same else _staging(h, Y.shape[1], Y.dtype)
    for step, (r0, r1) in enumerate(blocks):
        n = r1 - r0
        Xb = xs if n == h else xs[:n]
        np.copyto(Xb, X[r0:r1])
        if same:
            Yb = Xb
        else:
            Yb = ys if n == h else ys[:n]
            np.copyto(Yb, Y[r0:r1])
        gram_accumulate(C, Xb, Yb, 1.0, 0.0 if step == 0 else 1.0)
    return C


def cholesky_upper(G, N, k):
    """cholesky_upper (src/panelblas.jl:148-155): zpotrf on the upper
    triangle; on failure factor G + s I with s = 11 N k eps ||G||_F, and raise
    if that fails too. Returns (U, shifted)."""
    potrf = lapack.zpotrf if np.iscomplexobj(G) else lapack.dpotrf
    U, info = potrf(np.asfortranarray(G), lower=0, clean=1)
    if info == 0:
        return np.triu(U), False
    eps = EPS[np.dtype(G.dtype)]
    shift = 11 * N * k * eps * np.linalg.norm(G)
    U, info = potrf(np.asfortranarray(G + shift * np.eye(k)), lower=0, clean=1)
    if info != 0:
        raise OracleArgumentError(
            f"the {k}x{k} Gram matrix is not positive definite even after a shift of {shift}")
    return np.triu(U), True


def rdiv_rows(Y, R, w=None):
    """rdiv_rows! (src/panelblas.jl:157-169): Y <- Y R^-1 one row block at a
    time."""
    N, k = Y.shape
    w = k if w is None else w
    blocks = row_blocks(N, k, w)
    h = blocks[0][1] - blocks[0][0]
    ys = _staging(h, k, Y.dtype)
    for r0, r1 in blocks:
        n = r1 - r0
        Yb = ys if n == h else ys[:n]
        np.copyto(Yb, Y[r0:r1])
        rdiv_upper(Yb, R)
        np.copyto(Y[r0:r1], Yb)
    return Y


def cholqr_pass(Y, w=None):
    """cholqr_pass! (src/panelblas.jl:141-146)."""
    N, k = Y.shape
    G = gram(Y, w=w)
    R, shifted = cholesky_upper(G, N, k)
    rdiv_rows(Y, R, w)
    return R, shifted


def cholqr2(Y, w=None):
    """cholqr2! (src/panelblas.jl:130-139): two passes, a third if either
    shifted, R = R2 R1 (R3 R2 R1). Y is overwritten with Q. Returns
    (R, passes)."""
    R, s1 = cholqr_pass(Y, w)
    R2, s2 = cholqr_pass(Y, w)
    R = R2 @ R
    passes = 2
    if s1 or s2:
        R3, _ = cholqr_pass(Y, w)
        R = R3 @ R
        passes = 3
    return R, passes


def cholqr3_shifted(Y, u, w=None, storage=None):
    """The shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Zhang, Yamamoto,
    SIAM J. Sci. Comput. 2020) the north-star backend adds; not in the
    reference. Pass 1 factors G + s I with s = 11 (N k + k (k+1)) u ||G||_F
    unconditionally, passes 2 and 3 are cholqr_pass (src/panelblas.jl:141-146),
    R = R3 R2 R1. With storage (a numpy dtype) Y is rounded to it after every
    pass, as a narrowed host tier holds it between passes. Returns R."""
    N, k = Y.shape
    G = gram(Y, w=w)
    shift = 11 * (N * k + k * (k + 1)) * u * np.linalg.norm(G)
    potrf = lapack.zpotrf if np.iscomplexobj(G) else lapack.dpotrf
    R, info = potrf(np.asfortranarray(G + shift * np.eye(k)), lower=0, clean=1)
    if info != 0:
        raise OracleArgumentError(f"the {k}x{k} Gram matrix is not positive definite even after a shift of {shift}")
    R = np.triu(R)
    rdiv_rows(Y, R, w)
    if storage is not None:
        Y[...] = Y.astype(storage)
    for _ in range(2):
        R2, _ = cholqr_pass(Y, w)
        if storage is not None:
            Y[...] = Y.astype(storage)
        R = R2 @ R
    return R


def panelmul(G, X, w=None):
    """panelmul!(Y, G, X) (src/panelblas.jl:91-100): Y[:, panel] = G X[:, panel]."""
    k = X.shape[1]
    w = k if w is None else w
    Y = np.empty((G.shape[0], k), dtype=X.dtype)
    for c0, c1 in panel_ranges(k, w):
        Y[:, c0:c1] = G @ X[:, c0:c1]
    return Y


def project(Q, G, w=None):
    """project(Q, G) (src/panelblas.jl:268-301): for each panel j, apply G to
    Q_j, then fill block column j with Q_i^H (G Q_j) for every panel i."""
    N, k = Q.shape
    w = k if w is None else w
    S = np.empty((k, k), dtype=Q.dtype)
    ranges = panel_ranges(k, w)
    for (c0, c1) in ranges:
        image = G @ Q[:, c0:c1]
        for (r0, r1) in ranges:
            gram_accumulate(S[r0:r1, c0:c1], Q[:, r0:r1], image, 1.0, 0.0)
    return S


# ---- error measures the north star reports ------------------------------------

def orthogonality_error(Q):
    """||Q^H Q - I||_F."""
    k = Q.shape[1]
    return float(np.linalg.norm(Q.conj().T @ Q - np.eye(k)))


def reconstruction_error(Y, Q, R):
    """||Y - Q R|| / ||Y|| (Frobenius)."""
    return float(np.linalg.norm(Y - Q @ R) / np.linalg.norm(Y))


def blastol(dtype, N, k):
    """test/setup.jl:170."""
    return 100 * EPS[np.dtype(dtype)] * math.sqrt(N * k)


def orthogonality_bound(dtype, N, k):
    """test/setup.jl:172."""
    return 100 * N * k * EPS[np.dtype(dtype)]


def laplacian7(grid, shift):
    """-Lap_7 + shift I on an nx x ny x nz grid as a sparse matrix: unit
    spacing, zero outside the grid, point (x, y, z) at row x + nx (y + ny z).
    The streamed range finder's operator, stated as a Kronecker sum of 1-D
    second differences."""
    import scipy.sparse as sp
    nx, ny, nz = grid

    def d2(n):
        return sp.diags([-np.ones(n - 1), 2 * np.ones(n), -np.ones(n - 1)], [-1, 0, 1], shape=(n, n))

    I = sp.identity
    L = (sp.kron(I(nz), sp.kron(I(ny), d2(nx))) + sp.kron(I(nz), sp.kron(d2(ny), I(nx)))
         + sp.kron(d2(nz), sp.kron(I(ny), I(nx))))
    return (L + shift * I(nx * ny * nz)).tocsr().astype(np.complex128)


# ---- differentiation: the pullbacks behind the rrules --------------------------
# The reference has no rrule (Project.toml:6-9 has no ChainRulesCore), so
# nothing in it pins these; they are the textbook reverse-mode rules of the
# functions above, pinned in tests/test_adjoint_oracle.py by central finite
# differences of cholqr2 and project as defined in this module.

def copyltu(M):
    """The Hermitian matrix with M's strictly lower triangle, its conjugate
    transpose above the diagonal and Re diag(M) on the diagonal."""
    L = np.tril(M, -1)
    return L + L.conj().T + np.diag(np.diag(M).real)


def cholqr2_adjoint(Y, R, Qbar=None, Rbar=None):
    """The pullback of (Q, R) = cholqr2!(Y) (src/panelblas.jl:130-146), which
    is the thin QR factorization with a positive real diagonal in R: for a
    real loss, Ybar = (Qbar + Q H) R^-H with H = copyltu(R Rbar^H - Qbar^H Q).
    Q is recomputed from Y and R (Q = Y R^-1), as the device kernel does."""
    import scipy.linalg as sla
    N, k = Y.shape
    Q = sla.solve_triangular(R, Y.T, trans="T", lower=False).T  # Y R^-1
    M = np.zeros((k, k), dtype=np.complex128)
    if Rbar is not None:
        M += R @ Rbar.conj().T
    if Qbar is not None:
        M -= Qbar.conj().T @ Q
    Z = Q @ copyltu(M)
    if Qbar is not None:
        Z = Z + Qbar
    # Z R^-H: solve X R^H = Z, i.e. R X^H = Z^H.
    return sla.solve_triangular(R, Z.conj().T, lower=False).conj().T


def project_adjoint(Q, G, Sbar):
    """The pullback of S = project(Q, G) = Q^H (G Q) (src/panelblas.jl:268-301)
    with respect to Q: Qbar = (G Q) Sbar^H + (G^H Q) Sbar."""
    GhT = G.conj().T
    return (G @ Q) @ Sbar.conj().T + (GhT @ Q) @ Sbar


def hermitian_band(Dg):
    """The sparse N x N Hermitian matrix stored by diagonals in Dg (N x
    (kd + 1), Dg[i, d] = G[i, i + d]; the imaginary part of the main diagonal
    and the entries past the matrix ignored)."""
    import scipy.sparse as sp
    N, kd1 = Dg.shape
    diags, offs = [Dg[:, 0].real.astype(np.complex128)], [0]
    for d in range(1, kd1):
        if d >= N:
            break
        diags += [Dg[:N - d, d], Dg[:N - d, d].conj()]
        offs += [d, -d]
    return sp.diags(diags, offs, shape=(N, N), format="csr", dtype=np.complex128)


def range_finder_loss(Y, W, G, w=None):
    """The differentiation workload's loss: real(tr(W^H Q)) + ||S||_F^2 with
    (Q, R) = cholqr2!(copy(Y)) and S = project(Q, G)."""
    Q = np.array(Y, dtype=np.complex128, order="F", copy=True)
    cholqr2(Q, w)
    S = project(Q, G, w)
    return float(np.real(np.vdot(W, Q)) + np.linalg.norm(S) ** 2)


def range_finder_gradient(Y, W, G):
    """Ybar of range_finder_loss: Qbar = W + (G Q)(2 S)^H + (G^H Q)(2 S), then
    the cholqr2! pullback (Rbar = 0)."""
    Q = np.array(Y, dtype=np.complex128, order="F", copy=True)
    R, _ = cholqr2(Q)
    S = project(Q, G)
    Qbar = W + project_adjoint(Q, G, 2 * S)
    return cholqr2_adjoint(Y, R, Qbar, None)
