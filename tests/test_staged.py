"""cholqr2! end to end on host panels (fb_zcholqr2_staged): the upload of
row blocks overlapped with pass 1's Gram and the last solve's row blocks
going down as they are solved. The result must equal the device-resident
chain's (fb_zcholqr2) on the same matrix to the bit: the Gram's row chunks
are only grouped into blocks, never re-cut, and the solve is row by row.
The reference runs cholqr2! as src/panelblas.jl:130-146 with the panels
moved by src/panels.jl:365-458."""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu

MiB = 1 << 20


def staged_and_resident(fb, backend, A, w):
    N, k = A.shape
    nbytes = N * k * 16
    plan = fb.ResidencyPlan(device_budget=2 * nbytes + 64 * MiB, host_budget=nbytes + 64 * MiB, backend=backend)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    R = fb.cholqr2(Y, resident=True)
    Q = Y.to_array()
    fb.free(Y)
    D = backend.todevice(A)
    Rd = backend.alloc_device(np.complex128, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, D, Rd)
    return Q, R, D.to_host(), Rd.to_host(), passes


@pytest.mark.parametrize("N,k,w,kappa", [(300_007, 64, 16, 1e6), (200_003, 40, 24, 1e3), (1_000_000, 32, 8, 1e2),
                                         (50_000, 96, 32, 1e4), (123_457, 24, 24, 1e10)])
def test_staged_cholqr2_equals_the_resident_chain_to_the_bit(fb, backend, N, k, w, kappa):
    rng = np.random.default_rng(N + k)
    A = conditioned(rng, N, k, kappa)
    blocks = fb._lib.staged_blocks(N, k)
    assert blocks >= 1
    Q, R, Qd, Rd, passes = staged_and_resident(fb, backend, A, w)
    assert passes == (3 if kappa > 1e8 else 2)
    np.testing.assert_array_equal(Q, Qd)
    np.testing.assert_array_equal(R, Rd)


def test_staged_cholqr2_uses_several_blocks_on_a_tall_matrix(fb):
    assert fb._lib.staged_blocks(10_000_000, 64) == 8


def test_staged_cholqr2_leaves_the_panels_alone_when_it_fails(fb, backend):
    rng = np.random.default_rng(5)
    N, k = 100_000, 16
    A = randmatrix(rng, N, k)
    A[777, 3] = np.nan
    plan = fb.ResidencyPlan(device_budget=64 * MiB, host_budget=64 * MiB, backend=backend)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=8)
    with pytest.raises(fb.NotPositiveDefinite):
        fb.cholqr2(Y, resident=True)
    np.testing.assert_array_equal(Y.to_array(), A)
    fb.free(Y)


@pytest.mark.parametrize("N,k,w", [(250_001, 64, 16), (100_003, 128, 32)])
def test_staged_shifted_cholqr3_on_a_complexf32_tier_equals_the_resident_chain(fb, backend, N, k, w):
    """The narrowed tier (src/panels.jl:94-122): ComplexF32 panels go up,
    are widened on the device block by block, the shifted CholeskyQR3 runs in
    FP64, and Q is narrowed on the device on the way back; the same as the
    resident chain on the widened input, Q then rounded to ComplexF32."""
    rng = np.random.default_rng(N)
    A = conditioned(rng, N, k, 1e4)
    nbytes = N * k * 16
    plan = fb.ResidencyPlan(device_budget=2 * nbytes + 64 * MiB, host_budget=nbytes + 64 * MiB, backend=backend,
                            host_eltype=np.complex64)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    stored = Y.to_array()
    R = fb.cholqr3(Y, resident=True)
    Q = Y.to_array()
    fb.free(Y)
    D = backend.todevice(np.asfortranarray(stored))
    Rd = backend.alloc_device(np.complex128, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, D, Rd, form="shifted3", unit_roundoff=2.0 ** -24)
    assert passes == 3
    np.testing.assert_array_equal(R, Rd.to_host())
    np.testing.assert_array_equal(Q, D.to_host().astype(np.complex64).astype(np.complex128))
