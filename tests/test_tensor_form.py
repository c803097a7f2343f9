"""The tensor-core form of the Gram (fb_zgram_tc): an Ozaki split into 8-bit
slices on the integer tensor cores, checked against the oracle's FP64 Gram
and the FP64 tensor-core path, on shapes and scalings that exercise its
column scales, rescaling and int32 headroom drains.

Every entry keeps at least 47 bits relative to its column maximum and every
slice product that reaches that level is kept, so the Gram matrix is within
FP64-like bounds of the oracle's, relative to sqrt(G_ii G_jj)."""
import numpy as np
import pytest

from conftest import randmatrix

pytestmark = pytest.mark.gpu

TC_RTOL = 1e-13


def gram_tc(fb, backend, A, alpha=1.0, beta=0.0, C0=None):
    D = backend.todevice(np.asfortranarray(A))
    k = A.shape[1]
    C = backend.todevice(np.asfortranarray(C0)) if C0 is not None else backend.alloc_device(np.complex128, (k, k))
    fb.kernels.gram_tc(backend, C, D, alpha, beta)
    backend.sync_all()
    return C.to_host()


def relerr(G, ref):
    """Largest entry error relative to sqrt(G_ii G_jj) of the reference."""
    d = np.sqrt(np.abs(np.diag(ref)).real)
    scale = np.outer(d, d)
    scale[scale == 0] = 1.0
    return float(np.max(np.abs(G - ref) / scale))


@pytest.mark.parametrize("N,k", [(1, 1), (15, 3), (16, 64), (17, 64), (1000, 64), (5000, 23), (33333, 17),
                                 (300000, 64), (100000, 1)])
def test_gram_tc_matches_the_oracle(fb, backend, oracle, N, k):
    rng = np.random.default_rng(N * 131 + k)
    A = randmatrix(rng, N, k)
    G = gram_tc(fb, backend, A)
    ref = oracle.gram(A)
    assert relerr(G, ref) < 1e-14 * max(1.0, np.sqrt(N) / 100)


def test_gram_tc_is_exactly_hermitian_and_deterministic(fb, backend):
    rng = np.random.default_rng(7)
    A = randmatrix(rng, 54321, 64)
    G1 = gram_tc(fb, backend, A)
    G2 = gram_tc(fb, backend, A)
    assert G1.tobytes() == G2.tobytes()
    assert np.array_equal(G1, G1.conj().T)
    assert np.all(np.diag(G1).imag == 0)


def test_gram_tc_graded_columns(fb, backend, oracle):
    # Column scales from 1 to 1e-12: each column is sliced against its own scale.
    rng = np.random.default_rng(11)
    A = randmatrix(rng, 20000, 48) * (10.0 ** -np.linspace(0, 12, 48))
    assert relerr(gram_tc(fb, backend, A), oracle.gram(A)) < TC_RTOL


def test_gram_tc_rows_that_grow_force_rescaling(fb, backend, oracle):
    # Magnitudes grow by 2^40 down the rows, so every CTA keeps meeting
    # entries above its current scale and drains before rescaling.
    rng = np.random.default_rng(12)
    N, k = 400000, 32
    A = randmatrix(rng, N, k) * (2.0 ** (40 * np.arange(N) / N))[:, None]
    assert relerr(gram_tc(fb, backend, A), oracle.gram(A)) < TC_RTOL


def test_gram_tc_long_columns_drain_for_int32_headroom(fb, backend, oracle):
    # More than 8192 rows per CTA: the accumulators drain for headroom. A large
    # mean keeps every integer sum one-signed, the worst case for overflow.
    rng = np.random.default_rng(13)
    N, k = 2_000_000, 64
    A = (rng.standard_normal((N, k)) + 1j * rng.standard_normal((N, k))) / np.sqrt(2)
    A = np.asfortranarray(A + 3.0)
    assert relerr(gram_tc(fb, backend, A), oracle.gram(A)) < TC_RTOL


def test_gram_tc_agrees_with_the_fp64_tensor_path(fb, backend):
    rng = np.random.default_rng(14)
    A = randmatrix(rng, 100000, 64)
    D = backend.todevice(A)
    C = backend.alloc_device(np.complex128, (64, 64))
    fb.kernels.gram_accumulate(backend, C, D, D, 1.0, 0.0)
    backend.sync_all()
    assert relerr(gram_tc(fb, backend, A), C.to_host()) < TC_RTOL


def test_gram_tc_alpha_beta_zero_columns_and_nonfinite(fb, backend):
    rng = np.random.default_rng(15)
    A = randmatrix(rng, 777, 9)
    A[:, 4] = 0
    ref = A.conj().T @ A
    nan = np.full((9, 9), np.nan + 1j * np.nan)
    # beta == 0 overwrites whatever C held, NaN included.
    G = gram_tc(fb, backend, A, 2.0, 0.0, nan)
    assert relerr(G, 2 * ref) < TC_RTOL
    assert np.all(G[:, 4] == 0) and np.all(G[4, :] == 0)
    C0 = randmatrix(rng, 9, 9)
    assert relerr(gram_tc(fb, backend, A, 1.0, 1.0, C0) - C0, ref) < TC_RTOL
    assert np.all(gram_tc(fb, backend, np.zeros((100, 5), dtype=np.complex128)) == 0)
    B = A.copy()
    B[100, 2] = np.nan
    assert np.all(np.isnan(gram_tc(fb, backend, B)))


def test_gram_tc_rejects_wide_matrices(fb, backend):
    D = backend.alloc_device(np.complex128, (100, 65))
    C = backend.alloc_device(np.complex128, (65, 65))
    with pytest.raises(fb.ArgumentError):
        fb.kernels.gram_tc(backend, C, D)


# ---- cholqr2! in the tensor-core form ----------------------------------------

def run_cholqr2_tc(fb, backend, A):
    k = A.shape[1]
    Y = backend.todevice(np.asfortranarray(A))
    R = backend.alloc_device(np.complex128, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, Y, R, form="tc")
    return Y.to_host(), R.to_host(), passes


@pytest.mark.parametrize("kappa", [1e2, 1e6])
def test_cholqr2_tc_meets_the_accuracy_targets(fb, backend, oracle, kappa):
    # ||Q^H Q - I||_F <= 1e-12 and ||Y - Q R|| / ||Y|| <= 1e-13, the targets
    # of the tensor-core form.
    from conftest import conditioned
    rng = np.random.default_rng(int(np.log10(kappa)))
    A = conditioned(rng, 200000, 64, kappa)
    Q, R, passes = run_cholqr2_tc(fb, backend, A)
    assert passes == 2
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(A, Q, R) <= 1e-13
    Rref, _ = oracle.cholqr2(A.copy(order="F"), w=64)
    assert np.linalg.norm(R - Rref) <= 1e-10 * np.linalg.norm(Rref)


def test_cholqr2_tc_takes_the_shifted_third_pass(fb, backend, oracle):
    from conftest import conditioned
    rng = np.random.default_rng(99)
    A = conditioned(rng, 50000, 32, 1e10)
    Q, R, passes = run_cholqr2_tc(fb, backend, A)
    assert passes == 3
    assert np.linalg.norm(Q.conj().T @ Q - np.eye(32), 2) <= 1e-8
    assert oracle.reconstruction_error(A, Q, R) <= 1e-10
