"""Parity of the device kernels against the CPU oracle, through the C ABI.

Mirrors test/test_kernels.jl (whole buffers, the ragged views a sweep hands
over, NaN-filled outputs, shape errors) and adds the shapes the tiling has to
get right: widths that are not multiples of 4 or 64, row counts around the
32-row stage, and the folded Hermitian case. Floating point tolerance is the
reference's blastol = 100 eps sqrt(N k) (test/setup.jl:170) unless stated.
"""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu


def nanbuffer(backend, shape):
    return backend.todevice(np.full(shape, np.nan + 1j * np.nan, dtype=np.complex128, order="F"))


@pytest.mark.parametrize("rows,kA,kB", [(12, 5, 4), (1, 1, 1), (31, 7, 9), (33, 23, 23), (1000, 64, 64),
                                        (4097, 65, 3), (300, 130, 70), (0, 4, 4)])
def test_gram_accumulate_general(fb, backend, oracle, rows, kA, kB):
    rng = np.random.default_rng(rows * 1000 + kA)
    A, B = randmatrix(rng, rows, kA), randmatrix(rng, rows, kB)
    Ad, Bd = backend.todevice(A), backend.todevice(B)
    C = nanbuffer(backend, (kA, kB))
    fb.kernels.gram_accumulate(backend, C, Ad, Bd, 1.0, 0.0)
    tol = oracle.blastol(np.complex128, max(rows, 1), kA)
    np.testing.assert_allclose(C.to_host(), A.conj().T @ B, rtol=tol, atol=tol)
    fb.kernels.gram_accumulate(backend, C, Ad, Bd, 1.0, 1.0)
    np.testing.assert_allclose(C.to_host(), 2 * (A.conj().T @ B), rtol=tol, atol=tol)
    fb.kernels.gram_accumulate(backend, C, Ad, Bd, 0.5 - 2j, 3.0)
    np.testing.assert_allclose(C.to_host(), (6.5 - 2j) * (A.conj().T @ B), rtol=tol, atol=tol)


@pytest.mark.parametrize("rows,k", [(40, 23), (2048, 64), (1000, 1), (777, 96), (513, 130), (33, 8)])
def test_gram_hermitian_is_exact_mirror(fb, backend, oracle, rows, k):
    rng = np.random.default_rng(k)
    A = randmatrix(rng, rows, k)
    Ad = backend.todevice(A)
    C = nanbuffer(backend, (k, k))
    fb.kernels.gram_accumulate(backend, C, Ad, Ad, 1.0, 0.0)
    G = C.to_host()
    np.testing.assert_allclose(G, A.conj().T @ A, rtol=oracle.blastol(np.complex128, rows, k))
    assert np.array_equal(G, G.conj().T)
    assert np.all(np.diag(G).imag == 0)


def test_gram_is_deterministic(fb, backend):
    rng = np.random.default_rng(11)
    A = randmatrix(rng, 100_003, 64)
    B = randmatrix(rng, 100_003, 40)
    Ad, Bd = backend.todevice(A), backend.todevice(B)
    outs = []
    for _ in range(3):
        C = nanbuffer(backend, (64, 40))
        fb.kernels.gram_accumulate(backend, C, Ad, Bd, 1.0, 0.0)
        H = nanbuffer(backend, (64, 64))
        fb.kernels.gram_accumulate(backend, H, Ad, Ad, 1.0, 0.0)
        outs.append((C.to_host(), H.to_host()))
    for c, h in outs[1:]:
        assert np.array_equal(c, outs[0][0]) and np.array_equal(h, outs[0][1])


def test_gram_views(fb, backend, oracle):
    # test/test_kernels.jl:55-59: a block of the accumulator against views.
    rng = np.random.default_rng(12)
    A, B = randmatrix(rng, 12, 5), randmatrix(rng, 12, 4)
    Ad, Bd = backend.todevice(A), backend.todevice(B)
    C = backend.todevice(np.zeros((5, 4), dtype=np.complex128, order="F"))
    fb.kernels.gram_accumulate(backend, C.view(slice(0, 3), slice(0, 2)), Ad.view(slice(0, 6), slice(0, 3)),
                               Bd.view(slice(0, 6), slice(0, 2)), 1.0, 0.0)
    H = C.to_host()
    np.testing.assert_allclose(H[:3, :2], A[:6, :3].conj().T @ B[:6, :2], rtol=oracle.blastol(np.complex128, 6, 3))
    assert np.all(H[3:, :] == 0) and np.all(H[:, 2:] == 0)
    # A view of the same buffer on both sides is the folded Hermitian case.
    X = backend.todevice(randmatrix(rng, 50, 10))
    Xh = X.to_host()
    D = nanbuffer(backend, (6, 6))
    v = X.view(slice(5, 45), slice(2, 8))
    fb.kernels.gram_accumulate(backend, D, v, v, 1.0, 0.0)
    np.testing.assert_allclose(D.to_host(), Xh[5:45, 2:8].conj().T @ Xh[5:45, 2:8],
                               rtol=oracle.blastol(np.complex128, 40, 6))
    with pytest.raises(fb.DimensionMismatch):
        fb.kernels.gram_accumulate(backend, C, Ad, Bd.view(slice(None), slice(0, 2)), 1.0, 0.0)


@pytest.mark.parametrize("rows,k", [(7, 5), (1, 1), (129, 16), (1000, 23), (5000, 64), (300, 65), (257, 100),
                                   (3000, 128), (2001, 129), (1500, 200), (100, 257)])
def test_rdiv_upper(fb, backend, oracle, rows, k):
    rng = np.random.default_rng(rows + k)
    Y = randmatrix(rng, rows, k)
    R = np.asfortranarray(np.triu(randmatrix(rng, k, k) + 4 * np.eye(k)))
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd, Rd)
    expect = Y.copy(order="F")
    oracle.rdiv_upper(expect, R)
    np.testing.assert_allclose(Yd.to_host(), expect, rtol=oracle.blastol(np.complex128, rows, k))


def test_rdiv_upper_strided_block(fb, backend, oracle):
    # test/test_kernels.jl:103-107: the ragged last block, a view with a row stride.
    rng = np.random.default_rng(13)
    Y = randmatrix(rng, 7, 5)
    R = np.asfortranarray(np.triu(randmatrix(rng, 5, 5) + 4 * np.eye(5)))
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd.view(slice(0, 3)), Rd)
    H = Yd.to_host()
    expect = Y[:3].copy(order="F")
    oracle.rdiv_upper(expect, R)
    np.testing.assert_allclose(H[:3], expect, rtol=oracle.blastol(np.complex128, 7, 5))
    assert np.array_equal(H[3:], Y[3:])
    with pytest.raises(fb.DimensionMismatch):
        fb.kernels.rdiv_upper(backend, Yd, Rd.view(slice(0, 4), slice(0, 4)))


def test_rdiv_upper_complex_diagonal(fb, backend, oracle):
    rng = np.random.default_rng(14)
    Y = randmatrix(rng, 64, 12)
    R = np.asfortranarray(np.triu(randmatrix(rng, 12, 12)) + np.diag(2 + 1.5j * np.arange(12)))
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd, Rd)
    expect = Y.copy(order="F")
    oracle.rdiv_upper(expect, R)
    np.testing.assert_allclose(Yd.to_host(), expect, rtol=1e-13)


@pytest.mark.parametrize("rows,s,r", [(12, 5, 4), (1000, 64, 64), (77, 3, 100), (500, 80, 7), (9, 1, 1),
                                      (100_003, 64, 64), (20_001, 200, 130), (5000, 17, 64), (4097, 64, 9)])
def test_rightmul_gemm(fb, backend, oracle, rows, s, r):
    rng = np.random.default_rng(rows + s + r)
    A, C = randmatrix(rng, rows, s), randmatrix(rng, s, r)
    Ad, Cd = backend.todevice(A), backend.todevice(C)
    D = nanbuffer(backend, (rows, r))
    fb.kernels.rightmul_gemm(backend, D, Ad, Cd)
    np.testing.assert_allclose(D.to_host(), A @ C, rtol=oracle.blastol(np.complex128, rows, s))


def test_rightmul_gemm_ragged_block(fb, backend, oracle):
    # test/test_kernels.jl:79-84
    rng = np.random.default_rng(15)
    A, C = randmatrix(rng, 12, 5), randmatrix(rng, 5, 4)
    Ad, Cd = backend.todevice(A), backend.todevice(C)
    D = backend.todevice(np.zeros((12, 4), dtype=np.complex128, order="F"))
    fb.kernels.rightmul_gemm(backend, D.view(slice(0, 7)), Ad.view(slice(0, 7)), Cd)
    H = D.to_host()
    np.testing.assert_allclose(H[:7], A[:7] @ C, rtol=oracle.blastol(np.complex128, 12, 5))
    assert np.all(H[7:] == 0)


def test_convert_copy(fb, backend):
    # test/test_kernels.jl:5-30 with ComplexF32 as the narrowed type.
    rng = np.random.default_rng(16)
    A = randmatrix(rng, 9, 5)
    src = backend.todevice(A)
    narrow = backend.alloc_device(np.complex64, (9, 5))
    fb.kernels.convert_copy(backend, narrow, src)
    assert np.array_equal(narrow.to_host(), A.astype(np.complex64))
    wide = backend.alloc_device(np.complex128, (9, 5))
    fb.kernels.convert_copy(backend, wide, narrow)
    assert np.array_equal(wide.to_host(), A.astype(np.complex64).astype(np.complex128))
    dst = backend.todevice(np.zeros((9, 5), dtype=np.complex128, order="F"))
    fb.kernels.convert_copy(backend, dst.view(slice(None), slice(0, 2)), src.view(slice(None), slice(3, 5)))
    fb.kernels.convert_copy(backend, dst.view(slice(0, 3), slice(2, 5)), src.view(slice(6, 9), slice(0, 3)))
    H = dst.to_host()
    assert np.array_equal(H[:, :2], A[:, 3:5]) and np.array_equal(H[:3, 2:5], A[6:9, :3])
    with pytest.raises(fb.DimensionMismatch):
        fb.kernels.convert_copy(backend, dst, src.view(slice(None), slice(0, 3)))


def test_cholesky_upper_device(fb, backend, oracle):
    # test/test_panelblas.jl:327-345 on the device hook.
    rng = np.random.default_rng(17)
    N, k = 40, 23
    healthy = randmatrix(rng, N, k)
    G = np.asfortranarray(healthy.conj().T @ healthy)
    U = backend.alloc_device(np.complex128, (k, k))
    shifted, _ = fb.kernels.cholesky_upper_device(backend, backend.todevice(G), N, k, U)
    assert not shifted
    Uo, _ = oracle.cholesky_upper(G, N, k)
    np.testing.assert_allclose(U.to_host(), Uo, rtol=1e-13, atol=1e-13 * np.abs(Uo).max())
    singular = G.copy(order="F")
    singular[:, -1] = 0
    singular[-1, :] = 0
    shifted, shift = fb.kernels.cholesky_upper_device(backend, backend.todevice(singular), N, k, U)
    Uo, shifted_o = oracle.cholesky_upper(singular, N, k)
    assert shifted and shifted_o
    np.testing.assert_allclose(shift, 11 * N * k * 2.0 ** -52 * np.linalg.norm(singular), rtol=1e-12)
    np.testing.assert_allclose(U.to_host(), Uo, rtol=1e-10, atol=1e-10 * np.abs(Uo).max())
    with pytest.raises(fb.NotPositiveDefinite):
        fb.kernels.cholesky_upper_device(backend, backend.todevice(np.asfortranarray(-G)), N, k, U)


@pytest.mark.parametrize("k", [1, 5, 64, 100, 130])
def test_cholesky_product(fb, backend, oracle, k):
    rng = np.random.default_rng(k + 100)
    A = randmatrix(rng, 4 * k + 3, k)
    G = np.asfortranarray(A.conj().T @ A)
    Rin = np.asfortranarray(np.triu(randmatrix(rng, k, k) + 3 * np.eye(k)))
    U = backend.alloc_device(np.complex128, (k, k))
    Rout = nanbuffer(backend, (k, k))
    fb.kernels.cholesky_upper_device(backend, backend.todevice(G), A.shape[0], k, U,
                                     backend.todevice(Rin), Rout)
    Uo, _ = oracle.cholesky_upper(G, A.shape[0], k)
    np.testing.assert_allclose(U.to_host(), Uo, rtol=1e-12, atol=1e-12 * np.abs(Uo).max())
    expect = Uo @ Rin
    np.testing.assert_allclose(Rout.to_host(), expect, rtol=1e-12, atol=1e-12 * np.abs(expect).max())


@pytest.mark.parametrize("N,k", [(40, 23), (2 ** 16, 32), (100_000, 64), (5000, 100), (3, 3), (200_000, 128),
                                 (20_000, 150)])
def test_cholqr2_resident_matches_oracle(fb, backend, oracle, N, k):
    rng = np.random.default_rng(N + k)
    A = randmatrix(rng, N, k)
    Y = backend.todevice(A)
    R = nanbuffer(backend, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, Y, R)
    Q, Rh = Y.to_host(), R.to_host()
    Qo = A.copy(order="F")
    Ro, passes_o = oracle.cholqr2(Qo)
    assert passes == passes_o == 2
    assert oracle.orthogonality_error(Q) <= max(1e-12, oracle.orthogonality_bound(np.complex128, N, k))
    assert oracle.reconstruction_error(A, Q, Rh) <= 1e-13
    assert np.linalg.norm(Rh - Ro) <= 1e-12 * np.linalg.norm(Ro)
    assert np.linalg.norm(Q - Qo) <= 1e-12 * np.linalg.norm(Qo)
    assert np.all(np.tril(Rh, -1) == 0)


@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_cholqr2_resident_conditioning(fb, backend, oracle, kappa):
    # test/test_panelblas.jl:312-325 on the resident chain, including the
    # device-side decision to run the third pass.
    rng = np.random.default_rng(int(np.log10(kappa)))
    N, k = 4000, 23
    A = conditioned(rng, N, k, kappa)
    Y = backend.todevice(A)
    R = backend.alloc_device(np.complex128, (k, k))
    passes, shifts = fb.kernels.cholqr2_resident(backend, Y, R)
    Q, Rh = Y.to_host(), R.to_host()
    Qo = A.copy(order="F")
    _, passes_o = oracle.cholqr2(Qo)
    shifted = kappa > 1 / np.sqrt(2.0 ** -52)
    assert passes == passes_o == (3 if shifted else 2)
    bound = 1e-8 if shifted else oracle.orthogonality_bound(np.complex128, N, k)
    assert np.linalg.norm(Q.conj().T @ Q - np.eye(k), 2) <= bound
    assert np.linalg.norm(Q @ Rh - A) <= 1e-10 * np.linalg.norm(A)


def test_cholqr2_resident_refuses_dependent_columns(fb, backend):
    rng = np.random.default_rng(18)
    A = randmatrix(rng, 500, 6)
    A[:, 3] = A[:, 1]
    A[:, 4] = 0
    A = -np.asfortranarray(A)
    Y = backend.todevice(A)
    R = backend.alloc_device(np.complex128, (6, 6))
    # A zero column is rescued by the shift; an exactly duplicated one too
    # (the Gram matrix stays semidefinite), so this must not raise.
    fb.kernels.cholqr2_resident(backend, Y, R)
    # An indefinite Gram cannot come out of Y^H Y, so force one through the
    # factorization hook instead.
    G = -np.eye(6, dtype=np.complex128)
    U = backend.alloc_device(np.complex128, (6, 6))
    with pytest.raises(fb.NotPositiveDefinite):
        fb.kernels.cholesky_upper_device(backend, backend.todevice(np.asfortranarray(G)), 500, 6, U)


@pytest.mark.parametrize("k", [8, 23, 64])
def test_rdiv_upper_ill_conditioned_diagonal_block(fb, backend, oracle, k):
    # A diagonal 8 x 8 block of R whose condition number is far past what an
    # explicit block inverse tolerates: the kernel must fall back to plain
    # substitution and match ztrsm to working accuracy.
    rng = np.random.default_rng(k + 7)
    rows = 1000
    Y = randmatrix(rng, rows, k)
    R = np.asfortranarray(np.triu(randmatrix(rng, k, k)) + np.diag(np.full(k, 2.0)))
    R[1, 1] = 1e-7
    R[0, 1] = 3.0
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd, Rd)
    expect = Y.copy(order="F")
    oracle.rdiv_upper(expect, R)
    X = Yd.to_host()
    # Substitution is backward stable: its residual is eps |X| |R|, which the
    # 1e-7 pivot makes large; the device must do as well as ztrsm does.
    res, res_ref = np.linalg.norm(X @ R - Y), np.linalg.norm(expect @ R - Y)
    assert res <= 10 * res_ref + 1e-14 * np.linalg.norm(Y)
    assert np.linalg.norm(X - expect) <= 1e-7 * np.linalg.norm(expect)


def test_rdiv_upper_reconstructs_to_working_accuracy(fb, backend, oracle):
    # The blocked tensor-core solve multiplies by inverses of 8 x 8 diagonal
    # blocks; for a triangular factor of a Gram matrix with condition 1e12
    # (cholqr2!'s first pass on C2-like data) X R must still equal Y to 1e-13.
    rng = np.random.default_rng(99)
    rows, k = 20000, 64
    from conftest import conditioned
    A = conditioned(rng, rows, k, 1e6)
    R, _ = oracle.cholesky_upper(A.conj().T @ A, rows, k)
    Ad, Rd = backend.todevice(A), backend.todevice(np.asfortranarray(R))
    fb.kernels.rdiv_upper(backend, Ad, Rd)
    X = Ad.to_host()
    assert np.linalg.norm(X @ R - A) <= 1e-13 * np.linalg.norm(A)
    # And X is the substitution's result to within what any backward-stable
    # solve's forward error allows (about cond_1(R) eps).
    expect = A.copy(order="F")
    oracle.rdiv_upper(expect, R)
    cond = np.linalg.norm(R, 1) * np.linalg.norm(np.linalg.inv(R), 1)
    assert np.linalg.norm(X - expect) <= 1e-15 * cond * np.linalg.norm(expect)


@pytest.mark.parametrize("k", [40, 64])
def test_cholqr2_resident_matches_oracle_at_kappa_1e6(fb, backend, oracle, k):
    # The C2 conditioning: pass 1's factor is past the product by the inverse,
    # so the blocked solve runs. R stays within 1e-12 of the oracle's (whose
    # pass-1 solve is substitution); Q, which Y determines only to about
    # kappa eps, within that (the measured difference is near 1.3e-11).
    rng = np.random.default_rng(k + 500)
    N = 100_000
    A = conditioned(rng, N, k, 1e6)
    Qo = A.copy(order="F")
    Ro, passes_o = oracle.cholqr2(Qo)
    Y = backend.todevice(A)
    R = nanbuffer(backend, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, Y, R)
    Q, Rh = Y.to_host(), R.to_host()
    assert passes == passes_o == 2
    assert np.linalg.norm(Q - Qo) <= 1e6 * 2.0 ** -52 * np.linalg.norm(Qo)
    assert np.linalg.norm(Rh - Ro) <= 1e-12 * np.linalg.norm(Ro)
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(A, Q, Rh) <= 1e-13


@pytest.mark.parametrize("k,scale", [(64, 0.01), (37, 0.01), (64, 0.5), (8, 3.0)])
def test_rdiv_upper_both_tensor_core_paths(fb, backend, oracle, k, scale):
    # scale 0.01: R within 1 % of the identity, cond_1 well under 16, so the
    # solve is one product by inv(R); scale 0.5 and 3.0: larger off-diagonal
    # entries push cond_1 past 16 and the blocked solve takes over.
    rng = np.random.default_rng(k + int(100 * scale))
    rows = 3001
    Y = randmatrix(rng, rows, k)
    R = np.asfortranarray(np.eye(k) + scale * np.triu(randmatrix(rng, k, k)))
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd, Rd)
    expect = Y.copy(order="F")
    oracle.rdiv_upper(expect, R)
    X = Yd.to_host()
    cond = np.linalg.norm(R, 1) * np.linalg.norm(np.linalg.inv(R), 1)
    np.testing.assert_allclose(X, expect, rtol=0, atol=1e-14 * cond * np.abs(expect).max())
    assert np.linalg.norm(X @ R - Y) <= 1e-14 * np.linalg.norm(Y) * max(1.0, np.sqrt(cond))


@pytest.mark.parametrize("k", [8, 24, 37, 40, 56, 64])
def test_rdiv_upper_blocked_solve_over_many_sweeps(fb, backend, oracle, k):
    # Enough rows that every warp solves several 8-row units in turn (the
    # grid covers about 3e4 rows a sweep), with odd and even counts of 8-column
    # blocks: the Y prefetch runs from one unit into the next.
    rng = np.random.default_rng(k + 1000)
    rows = 300_001
    Y = randmatrix(rng, rows, k)
    R = np.asfortranarray(np.eye(k) + 0.5 * np.triu(randmatrix(rng, k, k)))
    Yd, Rd = backend.todevice(Y), backend.todevice(R)
    fb.kernels.rdiv_upper(backend, Yd, Rd)
    expect = Y.copy(order="F")
    oracle.rdiv_upper(expect, R)
    X = Yd.to_host()
    cond = np.linalg.norm(R, 1) * np.linalg.norm(np.linalg.inv(R), 1)
    np.testing.assert_allclose(X, expect, rtol=0, atol=1e-14 * cond * np.abs(expect).max())
    assert np.linalg.norm(X @ R - Y) <= 1e-14 * np.linalg.norm(Y) * max(1.0, np.sqrt(cond))


@pytest.mark.parametrize("k", [24, 40])
def test_cholqr2_resident_odd_block_counts(fb, backend, oracle, k):
    rng = np.random.default_rng(k)
    N = 200_003
    A = conditioned(rng, N, k, 1e3)
    Y = backend.todevice(A)
    R = nanbuffer(backend, (k, k))
    fb.kernels.cholqr2_resident(backend, Y, R)
    Q, Rh = Y.to_host(), R.to_host()
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(A, Q, Rh) <= 1e-13


@pytest.mark.parametrize("kappa", [1e4, 1e7])
def test_cholqr2_resident_k128_conditioned(fb, backend, oracle, kappa):
    # Past 64 columns the triangular solves go by 64-column blocks, each
    # diagonal block choosing its own path; the result keeps the accuracy
    # targets of the plain form.
    rng = np.random.default_rng(int(np.log10(kappa)) + 128)
    N, k = 100_000, 128
    A = conditioned(rng, N, k, kappa)
    Y = backend.todevice(A)
    R = nanbuffer(backend, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, Y, R)
    Q, Rh = Y.to_host(), R.to_host()
    Qo = A.copy(order="F")
    _, passes_o = oracle.cholqr2(Qo)
    assert passes == passes_o
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(A, Q, Rh) <= 1e-13
