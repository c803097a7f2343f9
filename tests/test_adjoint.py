"""The pullbacks of cholqr2! and project on the device (fb_zcholqr2_adjoint,
fb_zproject_adjoint), the Hermitian band operator and the rrules built on
them, against the oracle's pullbacks, and at the differentiation workload's
full size (N = 2^22, k = 64) against central finite differences of the
device forward pass."""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def oracle_R(oracle, Y):
    Q = np.array(Y, order="F", copy=True)
    R, _ = oracle.cholqr2(Q)
    return np.asfortranarray(R)


@pytest.mark.parametrize("N,k", [(1, 1), (37, 3), (1000, 16), (5000, 17), (100000, 64), (3000, 65), (2000, 100)])
def test_cholqr2_adjoint_matches_the_oracle(fb, backend, oracle, N, k):
    rng = np.random.default_rng(N + 7 * k)
    Y = randmatrix(rng, N, k)
    R = oracle_R(oracle, Y)
    Qbar = randmatrix(rng, N, k)
    Rbar = randmatrix(rng, k, k)
    d = lambda a: backend.todevice(a)
    Ybar = backend.alloc_device(np.complex128, (N, k))
    fb.kernels.cholqr2_adjoint(backend, Ybar, d(Y), d(R), d(Qbar), d(Rbar))
    backend.sync_all()
    assert rel(Ybar.to_host(), oracle.cholqr2_adjoint(Y, R, Qbar, Rbar)) < 1e-12


def test_cholqr2_adjoint_one_cotangent_at_a_time_and_in_place(fb, backend, oracle):
    rng = np.random.default_rng(1)
    N, k = 20000, 24
    Y = randmatrix(rng, N, k)
    R = oracle_R(oracle, Y)
    Qbar = randmatrix(rng, N, k)
    Rbar = randmatrix(rng, k, k)
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    out = backend.alloc_device(np.complex128, (N, k))
    fb.kernels.cholqr2_adjoint(backend, out, Yd, Rd, backend.todevice(Qbar), None)
    backend.sync_all()
    assert rel(out.to_host(), oracle.cholqr2_adjoint(Y, R, Qbar, None)) < 1e-12
    fb.kernels.cholqr2_adjoint(backend, out, Yd, Rd, None, backend.todevice(Rbar))
    backend.sync_all()
    assert rel(out.to_host(), oracle.cholqr2_adjoint(Y, R, None, Rbar)) < 1e-12
    # Ybar written over Qbar.
    Qd = backend.todevice(Qbar)
    fb.kernels.cholqr2_adjoint(backend, Qd, Yd, Rd, Qd, backend.todevice(Rbar))
    backend.sync_all()
    assert rel(Qd.to_host(), oracle.cholqr2_adjoint(Y, R, Qbar, Rbar)) < 1e-12


def test_cholqr2_adjoint_is_deterministic(fb, backend, oracle):
    rng = np.random.default_rng(2)
    N, k = 300000, 64
    Y = randmatrix(rng, N, k)
    Yd, Rd = backend.todevice(Y), backend.todevice(oracle_R(oracle, Y))
    Qd = backend.todevice(randmatrix(rng, N, k))
    a = backend.alloc_device(np.complex128, (N, k))
    b = backend.alloc_device(np.complex128, (N, k))
    fb.kernels.cholqr2_adjoint(backend, a, Yd, Rd, Qd, None)
    fb.kernels.cholqr2_adjoint(backend, b, Yd, Rd, Qd, None)
    backend.sync_all()
    assert a.to_host().tobytes() == b.to_host().tobytes()


@pytest.mark.parametrize("kappa", [1e4, 1e7])
def test_cholqr2_adjoint_of_ill_conditioned_inputs(fb, backend, oracle, kappa):
    # R^-1 is formed explicitly on the device and applied by substitution in
    # the oracle: the two agree to about eps cond(R).
    rng = np.random.default_rng(int(np.log10(kappa)))
    N, k = 50000, 32
    Y = conditioned(rng, N, k, kappa)
    R = oracle_R(oracle, Y)
    Qbar = randmatrix(rng, N, k)
    Ybar = backend.alloc_device(np.complex128, (N, k))
    fb.kernels.cholqr2_adjoint(backend, Ybar, backend.todevice(Y), backend.todevice(R), backend.todevice(Qbar), None)
    backend.sync_all()
    assert rel(Ybar.to_host(), oracle.cholqr2_adjoint(Y, R, Qbar, None)) < 1e-15 * kappa + 1e-12


def test_cholqr2_adjoint_refuses_overlap_and_bad_shapes(fb, backend):
    Y = backend.alloc_device(np.complex128, (100, 4))
    R = backend.alloc_device(np.complex128, (4, 4))
    with pytest.raises(fb.ArgumentError):
        fb.kernels.cholqr2_adjoint(backend, Y, Y, R, None, None)
    with pytest.raises(fb.DimensionMismatch):
        fb.kernels.cholqr2_adjoint(backend, backend.alloc_device(np.complex128, (100, 5)), Y, R)
    big = backend.alloc_device(np.complex128, (100, 8))
    with pytest.raises(fb.ArgumentError):
        # Ybar overlapping Qbar without being it.
        fb.kernels.cholqr2_adjoint(backend, big.view(slice(None), slice(0, 4)), Y, R,
                                   big.view(slice(None), slice(2, 6)), None)


@pytest.mark.parametrize("hermitian", [True, False])
@pytest.mark.parametrize("k", [5, 64, 70])
def test_project_adjoint_matches_the_oracle(fb, backend, oracle, hermitian, k):
    rng = np.random.default_rng(k + hermitian)
    N = 3000
    Q = randmatrix(rng, N, k)
    G = randmatrix(rng, N, N)
    if hermitian:
        G = G + G.conj().T
    Sbar = randmatrix(rng, k, k)
    GQ = backend.todevice(G @ Q)
    GhQ = None if hermitian else backend.todevice(G.conj().T @ Q)
    ref = oracle.project_adjoint(Q, G, Sbar)
    Qbar = backend.todevice(np.full((N, k), np.nan + 0j))
    fb.kernels.project_adjoint(backend, Qbar, GQ, backend.todevice(Sbar), GhQ, accumulate=False)
    backend.sync_all()
    assert rel(Qbar.to_host(), ref) < 1e-13
    base = randmatrix(rng, N, k)
    Qbar = backend.todevice(base)
    fb.kernels.project_adjoint(backend, Qbar, GQ, backend.todevice(Sbar), GhQ, accumulate=True)
    backend.sync_all()
    assert rel(Qbar.to_host(), base + ref) < 1e-13


# The last two walk several row tiles a CTA (one CTA an SM, 256 rows a tile),
# with partial column stages and a ragged last tile.
@pytest.mark.parametrize("N,kd,cols", [(1000, 5, 3), (50, 64, 7), (4096, 0, 4), (20000, 64, 9), (200_003, 64, 20),
                                       (90_001, 17, 33)])
def test_hermitian_band_apply_matches_the_oracle(fb, backend, oracle, N, kd, cols):
    rng = np.random.default_rng(N + kd)
    Dg = randmatrix(rng, N, kd + 1)
    X = randmatrix(rng, N, cols)
    G = fb.HermitianBand(backend, Dg)
    Y = backend.alloc_device(np.complex128, (N, cols))
    G.apply(backend, Y, backend.todevice(X))
    backend.sync_all()
    assert rel(Y.to_host(), oracle.hermitian_band(Dg) @ X) < 1e-14


def test_hermitian_band_apply_with_a_wide_band_stride(fb, backend, oracle):
    # Dg's columns 2^25 entries apart: the kernel's band offsets no longer fit
    # 32 bits and it forms them in 64.
    rng = np.random.default_rng(77)
    N, kd, cols, ld = 3001, 2, 5, 1 << 25
    Dg = randmatrix(rng, N, kd + 1)
    store = backend.alloc_device(np.complex128, (ld, kd + 1))
    view = store.view(slice(0, N), slice(None))
    backend.h2d(view, Dg)
    X = randmatrix(rng, N, cols)
    Y = backend.alloc_device(np.complex128, (N, cols))
    fb.kernels.hband_apply(backend, Y, backend.todevice(X), view)
    backend.sync_all()
    assert rel(Y.to_host(), oracle.hermitian_band(Dg) @ X) < 1e-14


def range_finder_rrule(fb, backend, Yd, Wd, G):
    """L = real(tr(W^H Q)) + ||S||_F^2 and its gradient through the rules."""
    (Q, R), back_c = fb.rrule(fb.cholqr2, Yd, backend=backend)
    S, back_p = fb.rrule(fb.project, Q, G, backend=backend)
    Sh = S.to_host()
    T = backend.alloc_device(np.complex128, (Q.cols, Q.cols))
    fb.kernels.gram_accumulate(backend, T, Wd, Q, 1.0, 0.0)
    loss = float(np.real(np.trace(T.to_host())) + np.linalg.norm(Sh) ** 2)
    Qbar = backend.alloc_device(np.complex128, Q.shape)
    fb.device_api.copy_region(Qbar, Wd, None)
    back_p(backend.todevice(2 * Sh), into=Qbar)
    Ybar = back_c(Qbar, None, into=Qbar)
    return loss, Ybar


@pytest.mark.parametrize("hermitian", [True, False])
def test_range_finder_rrule_matches_the_oracle_gradient(fb, backend, oracle, hermitian):
    rng = np.random.default_rng(8 + hermitian)
    N, k, kd = 16384, 64, 64
    Y = randmatrix(rng, N, k)
    W = randmatrix(rng, N, k)
    if hermitian:
        Dg = randmatrix(rng, N, kd + 1) * 4
        G = fb.HermitianBand(backend, Dg)
        Gs = oracle.hermitian_band(Dg)
    else:
        grid = (32, 32, 16)
        G = fb.Laplacian7(grid, 0.5 + 0.1j)
        Gs = oracle.laplacian7(grid, 0.5 + 0.1j)
    loss, Ybar = range_finder_rrule(fb, backend, backend.todevice(Y), backend.todevice(W), G)
    backend.sync_all()
    assert abs(loss - oracle.range_finder_loss(Y, W, Gs)) <= 1e-12 * abs(loss)
    assert rel(Ybar.to_host(), oracle.range_finder_gradient(Y, W, Gs)) < 1e-11


def test_rrule_of_anything_else_is_none(fb, backend):
    assert fb.rrule(fb.gram, None, backend=backend) is None


def test_range_finder_gradient_at_full_size_matches_finite_differences(fb, backend):
    # The differentiation workload: N = 2^22, k = 64, G Hermitian with 64
    # superdiagonals; 32 random directions, central differences of step 1e-6.
    N, k, kd = 1 << 22, 64, 64
    ghost = lambda dst, seed: fb.kernels.ghost_fill(backend, dst, 0, 0, seed, np.complex128)
    YD = backend.alloc_device(np.complex128, (N, 2 * k))
    Yd, Dd = YD.view(slice(None), slice(0, k)), YD.view(slice(None), slice(k, 2 * k))
    Wd = backend.alloc_device(np.complex128, (N, k))
    ghost(Yd, 0xC5)
    ghost(Wd, 0xC6)
    G = fb.HermitianBand.ghost(backend, N, kd, seed=0xC7, scale=float(np.sqrt(N / ((2 * kd + 1) * k))))
    loss0, Ybar = range_finder_rrule(fb, backend, Yd, Wd, G)

    Q = backend.alloc_device(np.complex128, (N, k))
    R = backend.alloc_device(np.complex128, (k, k))
    GQ = backend.alloc_device(np.complex128, (N, k))
    S = backend.alloc_device(np.complex128, (k, k))
    T = backend.alloc_device(np.complex128, (k, k))

    def loss(C):
        fb.kernels.rightmul_gemm(backend, Q, YD, C)   # Y +- h D
        passes, _ = fb.kernels.cholqr2_resident(backend, Q, R)
        assert passes == 2
        G.apply(backend, GQ, Q)
        fb.kernels.gram_accumulate(backend, S, Q, GQ, 1.0, 0.0)
        fb.kernels.gram_accumulate(backend, T, Wd, Q, 1.0, 0.0)
        return float(np.real(np.trace(T.to_host())) + np.linalg.norm(S.to_host()) ** 2)

    h = 1e-6
    I = np.eye(k, dtype=np.complex128)
    Cp, Cm = backend.todevice(np.vstack([I, h * I])), backend.todevice(np.vstack([I, -h * I]))
    fd, an = [], []
    for i in range(32):
        ghost(Dd, 0x1000 + i)
        fd.append((loss(Cp) - loss(Cm)) / (2 * h))
        fb.kernels.gram_accumulate(backend, T, Ybar, Dd, 1.0, 0.0)
        an.append(float(np.real(np.trace(T.to_host()))))
    fd, an = np.array(fd), np.array(an)
    assert abs(loss(backend.todevice(np.vstack([I, 0 * I]))) - loss0) <= 1e-12 * abs(loss0)
    assert np.linalg.norm(fd - an) / np.linalg.norm(an) < 1e-6
