"""Pins the CPU oracle to the reference's own known-answer tests for this path.

The reference has no golden vectors for gram, cholqr2!, project or the
kernels: its tests compare against dense LinearAlgebra within blastol and
orthogonality_bound (test/setup.jl:170-172) and demand bitwise equality in a
few places. Each test here restates one of those, on the oracle, with the
reference's sizes (N = 40, k = 23, widths 23, 12, 7, 1).
"""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

BLAS_WIDTHS = (23, 12, 7, 1)  # test/test_panelblas.jl:1


@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_gram_against_dense(oracle, w):
    # test/test_panelblas.jl:3-15
    rng = np.random.default_rng(1)
    N, k = 40, 23
    A, B = randmatrix(rng, N, k), randmatrix(rng, N, k)
    tol = oracle.blastol(np.complex128, N, k)
    np.testing.assert_allclose(oracle.gram(A, B, w), A.conj().T @ B, rtol=tol)
    np.testing.assert_allclose(oracle.gram(A, w=w), A.conj().T @ A, rtol=tol)
    assert np.array_equal(oracle.gram(A, A, w), oracle.gram(A, w=w))


def test_row_blocks_cover_the_matrix(oracle):
    # row_block_height (src/plan.jl:133) and RowSteps (src/executor.jl:33-36)
    assert oracle.row_block_height(40, 23, 7) == 12
    assert oracle.row_blocks(40, 23, 7) == [(0, 12), (12, 24), (24, 36), (36, 40)]
    assert oracle.row_block_height(40, 23, 1) == 1
    assert oracle.row_block_height(40, 23, 23) == 40
    assert oracle.row_block_height(2 ** 20, 32, 8) == 2 ** 18
    assert oracle.row_block_height(10 ** 7, 64, 16) == 2_500_000


def test_choose_panel_width_known_answers(oracle):
    # test/test_plan.jl restated: evening out and the budget cap.
    assert oracle.choose_panel_width(10, 1000, 16, device_budget=2 * 999 * 10 * 16) == 500
    assert oracle.choose_panel_width(100, 8, 16, device_budget=2 ** 30) == 8
    with pytest.raises(oracle.OracleArgumentError):
        oracle.choose_panel_width(10 ** 6, 4, 16, device_budget=1000)


@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_cholqr2_orthonormalizes(oracle, w):
    # test/test_panelblas.jl:297-310
    rng = np.random.default_rng(2)
    N, k = 40, 23
    A = randmatrix(rng, N, k)
    Y = A.copy(order="F")
    R, passes = oracle.cholqr2(Y, w)
    assert passes == 2
    assert R.shape == (k, k)
    np.testing.assert_allclose(R, np.triu(R))
    assert np.linalg.norm(Y.conj().T @ Y - np.eye(k), 2) <= oracle.orthogonality_bound(np.complex128, N, k)
    np.testing.assert_allclose(Y @ R, A, rtol=oracle.blastol(np.complex128, N, k))


@pytest.mark.parametrize("kappa", (1e2, 1e6, 1e10))
def test_cholqr2_survives_conditioning(oracle, kappa):
    # test/test_panelblas.jl:312-325
    rng = np.random.default_rng(3)
    N, k, w = 40, 23, 7
    A = conditioned(rng, N, k, kappa)
    Y = A.copy(order="F")
    R, passes = oracle.cholqr2(Y, w)
    shifted = kappa > 1 / np.sqrt(2.0 ** -52)
    bound = 1e-8 if shifted else oracle.orthogonality_bound(np.complex128, N, k)
    assert np.linalg.norm(Y.conj().T @ Y - np.eye(k), 2) <= bound
    assert np.linalg.norm(Y @ R - A) <= 1e-10 * np.linalg.norm(A)
    assert passes == (3 if shifted else 2)


def test_shift_fires_only_when_it_has_to(oracle):
    # test/test_panelblas.jl:327-345
    rng = np.random.default_rng(4)
    N, k = 40, 23
    healthy = randmatrix(rng, N, k)
    G = healthy.conj().T @ healthy
    _, shifted = oracle.cholesky_upper(G, N, k)
    assert not shifted
    singular = G.copy()
    singular[:, -1] = 0
    singular[-1, :] = 0
    U, shifted = oracle.cholesky_upper(singular, N, k)
    assert shifted
    np.testing.assert_allclose(U, np.triu(U))
    with pytest.raises(oracle.OracleArgumentError):
        oracle.cholesky_upper(-G, N, k)


@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_project_against_dense(oracle, w):
    # test/test_panelblas.jl:347-360
    rng = np.random.default_rng(5)
    N, k = 40, 23
    G = randmatrix(rng, N, N)
    A = randmatrix(rng, N, k)
    np.testing.assert_allclose(oracle.project(A, G, w), A.conj().T @ G @ A,
                               rtol=oracle.blastol(np.complex128, N, k))


def test_project_matches_panelmul_then_gram(oracle):
    # test/test_panelblas.jl:362-373
    rng = np.random.default_rng(6)
    N, k, w = 40, 23, 7
    G = randmatrix(rng, N, N)
    A = randmatrix(rng, N, k)
    Z = oracle.panelmul(G, A, w)
    np.testing.assert_allclose(oracle.project(A, G, w), oracle.gram(A, Z, w),
                               rtol=oracle.blastol(np.complex128, N, k))


def test_kernels_against_dense(oracle):
    # test/test_kernels.jl:32-110, including the NaN-filled output
    rng = np.random.default_rng(7)
    A, B = randmatrix(rng, 12, 5), randmatrix(rng, 12, 4)
    C = np.full((5, 4), np.nan + 0j)
    oracle.gram_accumulate(C, A, B, 1.0, 0.0)
    np.testing.assert_allclose(C, A.conj().T @ B, rtol=oracle.blastol(np.complex128, 12, 5))
    oracle.gram_accumulate(C, A, B, 1.0, 1.0)
    np.testing.assert_allclose(C, 2 * (A.conj().T @ B), rtol=oracle.blastol(np.complex128, 12, 5))
    Y = randmatrix(rng, 7, 5)
    R = np.triu(randmatrix(rng, 5, 5) + 4 * np.eye(5))
    Z = Y.copy(order="F")
    oracle.rdiv_upper(Z, R)
    np.testing.assert_allclose(Z, Y @ np.linalg.inv(R), rtol=oracle.blastol(np.complex128, 7, 5))


# ---- the shifted CholeskyQR3 (the ComplexF32 storage tier's orthonormalization)

@pytest.mark.parametrize("kappa", [1e4, 1e7, 1e12])
def test_cholqr3_shifted_orthonormalizes_past_cholqr2_range(oracle, kappa):
    # The shift makes pass 1 succeed for condition numbers far past what the
    # unshifted CholeskyQR2 handles (about 1e8 in FP64).
    from conftest import conditioned
    rng = np.random.default_rng(int(np.log10(kappa)))
    A = conditioned(rng, 3000, 24, kappa)
    Q = A.copy(order="F")
    R = oracle.cholqr3_shifted(Q, 2.0 ** -53)
    assert oracle.orthogonality_error(Q) < 1e-13
    assert oracle.reconstruction_error(A, Q, R) < 1e-14
    assert np.allclose(np.tril(R, -1), 0)


def test_cholqr3_shifted_with_complex64_storage(oracle):
    from conftest import conditioned
    rng = np.random.default_rng(5)
    A = conditioned(rng, 4000, 16, 1e5).astype(np.complex64).astype(np.complex128)
    Q = A.copy(order="F")
    R = oracle.cholqr3_shifted(Q, 2.0 ** -24, storage=np.complex64)
    assert np.array_equal(Q, Q.astype(np.complex64).astype(np.complex128))
    assert oracle.orthogonality_error(Q) < 1e-5
    assert oracle.reconstruction_error(A, Q, R) < 1e-6
