"""The shifted CholeskyQR3 (fb_zcholqr3_shifted, fb_zpotrf_forced_shift,
funicular_b200.cholqr3): the orthonormalization the north-star backend adds
for the ComplexF32 storage tier, against the oracle's restatement
(oracle.cholqr3_shifted), device-resident and streamed, with FP64 and with
ComplexF32 host storage."""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu

MiB = 2 ** 20
U64, U32 = 2.0 ** -53, 2.0 ** -24


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("N,k,kappa", [(50_000, 32, 1e4), (50_000, 32, 1e7), (30_000, 24, 1e12), (100_000, 128, 1e7),
                                       (7, 3, 1e2)])
def test_resident_chain_matches_the_oracle(fb, backend, oracle, N, k, kappa):
    rng = np.random.default_rng(N + k)
    A = conditioned(rng, N, k, kappa)
    Y = backend.todevice(A)
    R = backend.alloc_device(np.complex128, (k, k))
    passes, shifts = fb.kernels.cholqr2_resident(backend, Y, R, form="shifted3", unit_roundoff=U64)
    assert passes == 3
    assert shifts[0] > 0
    Q, Rh = Y.to_host(), R.to_host()
    Qo = A.copy(order="F")
    Ro = oracle.cholqr3_shifted(Qo, U64)
    assert oracle.orthogonality_error(Q) <= 1e-13
    assert oracle.reconstruction_error(A, Q, Rh) <= 1e-14
    assert np.all(np.tril(Rh, -1) == 0)
    if kappa <= 1e7:
        # R and Q are determined by A to about kappa eps.
        assert rel(Rh, Ro) <= 1e-14 * kappa + 1e-13
        assert rel(Q, Qo) <= 1e-14 * kappa + 1e-13


def test_the_forced_shift_matches_the_formula(fb, backend, oracle):
    rng = np.random.default_rng(3)
    N, k = 20_000, 12
    A = randmatrix(rng, N, k)
    G = A.conj().T @ A
    Gd = backend.todevice(np.asfortranarray(G))
    U = backend.alloc_device(np.complex128, (k, k))
    shifted, shift = fb.kernels.cholesky_upper_device(backend, Gd, N, k, U, forced_unit_roundoff=U32)
    assert shifted
    expect = 11 * (N * k + k * (k + 1)) * U32 * np.linalg.norm(G)
    assert abs(shift - expect) <= 1e-13 * expect
    Uh = U.to_host()
    assert rel(Uh.conj().T @ Uh, G + shift * np.eye(k)) <= 1e-14


@pytest.mark.parametrize("resident", [True, False])
def test_complex64_host_storage(fb, make_plan_gpu, oracle, resident):
    rng = np.random.default_rng(11 + resident)
    N, k, w = 20_000, 16, 4
    A = conditioned(rng, N, k, 1e5).astype(np.complex64)
    plan = make_plan_gpu(host_eltype=np.complex64, panel_width=w,
                         device_budget=(256 * MiB if resident else 2 * N * w * 16 + 8 * MiB))
    Y = fb.PanelMatrix.from_array(A.astype(np.complex128), plan=plan)
    R = fb.cholqr3(Y, resident=resident)
    Q = Y.to_array()
    A64 = A.astype(np.complex128)
    # What the panels hold is ComplexF32; the orthogonality and the
    # reconstruction are those of single-precision storage.
    assert np.array_equal(Q, Q.astype(np.complex64).astype(np.complex128))
    assert oracle.orthogonality_error(Q) <= 1e-5
    assert oracle.reconstruction_error(A64, Q, R) <= 1e-6
    if not resident:
        Qo = A64.copy(order="F")
        Ro = oracle.cholqr3_shifted(Qo, U32, w=w, storage=np.complex64)
        assert rel(R, Ro) <= 1e-6


def test_unit_roundoff_is_checked(fb, backend):
    Y = backend.alloc_device(np.complex128, (100, 4))
    R = backend.alloc_device(np.complex128, (4, 4))
    with pytest.raises(fb.ArgumentError):
        fb.kernels.cholqr2_resident(backend, Y, R, form="shifted3", unit_roundoff=0.0)


@pytest.fixture
def make_plan_gpu(fb, backend):
    def make(**kw):
        kw.setdefault("host_budget", 256 * MiB)
        return fb.ResidencyPlan(backend=backend, **kw)
    return make
