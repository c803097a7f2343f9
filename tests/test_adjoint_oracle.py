"""The oracle's pullbacks of cholqr2! and project against central finite
differences of the oracle's own forward functions. The reference has no rrule
and so no known answers for these; finite differences of the restated forward
path are what pins them before they check the device kernels."""
import numpy as np
import pytest

from conftest import randmatrix


def fd_error(loss, grad, Y, rng, directions=8, h=1e-6):
    """|| fd - <grad, D> || / || <grad, D> || over random complex directions."""
    fd, an = [], []
    for _ in range(directions):
        D = randmatrix(rng, *Y.shape) * 2
        fd.append((loss(Y + h * D) - loss(Y - h * D)) / (2 * h))
        an.append(np.real(np.vdot(grad, D)))
    fd, an = np.array(fd), np.array(an)
    return np.linalg.norm(fd - an) / np.linalg.norm(an)


@pytest.mark.parametrize("N,k", [(40, 1), (200, 5), (500, 12)])
def test_cholqr2_adjoint_of_Q_matches_finite_differences(oracle, N, k):
    rng = np.random.default_rng(N + k)
    Y = randmatrix(rng, N, k)
    W = randmatrix(rng, N, k)

    def loss(Ym):
        Q = np.array(Ym, order="F", copy=True)
        oracle.cholqr2(Q)
        return np.real(np.vdot(W, Q))

    Q = np.array(Y, order="F", copy=True)
    R, _ = oracle.cholqr2(Q)
    assert fd_error(loss, oracle.cholqr2_adjoint(Y, R, W, None), Y, rng) < 1e-6


def test_cholqr2_adjoint_of_R_matches_finite_differences(oracle):
    rng = np.random.default_rng(3)
    N, k = 300, 7
    Y = randmatrix(rng, N, k)
    B = randmatrix(rng, k, k)  # the lower triangle of a cotangent of R plays no part

    def loss(Ym):
        Q = np.array(Ym, order="F", copy=True)
        R, _ = oracle.cholqr2(Q)
        return np.real(np.vdot(B, R))

    Q = np.array(Y, order="F", copy=True)
    R, _ = oracle.cholqr2(Q)
    assert fd_error(loss, oracle.cholqr2_adjoint(Y, R, None, B), Y, rng) < 1e-6
    # Only the upper triangle and the real diagonal of Rbar reach Ybar.
    Bu = np.triu(B) - 1j * np.diag(np.diag(B).imag)
    full, upper = oracle.cholqr2_adjoint(Y, R, None, B), oracle.cholqr2_adjoint(Y, R, None, Bu)
    assert np.linalg.norm(full - upper) <= 1e-13 * np.linalg.norm(full)


def test_project_adjoint_matches_finite_differences(oracle):
    rng = np.random.default_rng(4)
    N, k = 120, 6
    Q = randmatrix(rng, N, k)
    G = randmatrix(rng, N, N)
    Sbar = randmatrix(rng, k, k)

    def loss(Qm):
        return np.real(np.vdot(Sbar, oracle.project(Qm, G)))

    assert fd_error(loss, oracle.project_adjoint(Q, G, Sbar), Q, rng) < 1e-7


def test_hermitian_band_is_hermitian_and_banded(oracle):
    rng = np.random.default_rng(5)
    N, kd = 50, 7
    Dg = randmatrix(rng, N, kd + 1)
    G = oracle.hermitian_band(Dg).toarray()
    assert np.array_equal(G, G.conj().T)
    i, j = np.nonzero(G)
    assert np.max(np.abs(i - j)) == kd
    assert G[3, 3 + 2] == Dg[3, 2] and G[3 + 2, 3] == np.conj(Dg[3, 2])
    assert G[4, 4] == Dg[4, 0].real


def test_range_finder_gradient_matches_finite_differences(oracle):
    rng = np.random.default_rng(6)
    N, k, kd = 400, 8, 6
    Y = randmatrix(rng, N, k)
    W = randmatrix(rng, N, k)
    G = oracle.hermitian_band(randmatrix(rng, N, kd + 1) * 4)
    g = oracle.range_finder_gradient(Y, W, G)
    assert fd_error(lambda Ym: oracle.range_finder_loss(Ym, W, G), g, Y, rng, directions=12) < 1e-6
