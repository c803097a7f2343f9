"""Batched cholqr2! as one persistent kernel (fb_zcholqr2_batched_persistent):
every instance against the oracle's cholqr2! (src/panelblas.jl:130-139), the
same bits run to run and whatever else is in the batch, the three solve
paths and the device-side third pass, a failing instance stopping only its
own chain, a captured graph, and batches past one launch's 384 instances."""
import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu

SHAPES = [(1000, 16), (5000, 32), (20000, 64), (77, 7), (16, 16), (123457, 64), (40000, 23), (3000, 1),
          (700001, 64), (33, 33), (9000, 57), (260000, 8)]


def run(fb, backend, mats, **kw):
    Ys = [backend.todevice(A) for A in mats]
    Rs = [backend.todevice(np.full((A.shape[1],) * 2, np.nan + 1j * np.nan, order="F")) for A in mats]
    passes = fb.kernels.cholqr2_batched(backend, Ys, Rs, schedule="persistent", **kw)
    return passes, [Y.to_host() for Y in Ys], [R.to_host() for R in Rs]


def orthogonality(Q):
    return np.linalg.norm(Q.conj().T @ Q - np.eye(Q.shape[1]))


def test_persistent_batch_matches_the_oracle(fb, backend, oracle):
    rng = np.random.default_rng(11)
    mats = [randmatrix(rng, N, k) for N, k in SHAPES]
    passes, Qs, Rs = run(fb, backend, mats)
    assert passes == [2] * len(mats)
    for A, Q, R in zip(mats, Qs, Rs):
        N, k = A.shape
        Qo = A.copy(order="F")
        Ro, passes_o = oracle.cholqr2(Qo)
        assert passes_o == 2
        assert oracle.orthogonality_error(Q) <= max(1e-12, oracle.orthogonality_bound(np.complex128, N, k))
        assert oracle.reconstruction_error(A, Q, R) <= 1e-13
        assert np.linalg.norm(R - Ro) <= 1e-12 * np.linalg.norm(Ro)
        assert np.linalg.norm(Q - Qo) <= 1e-12 * np.linalg.norm(Qo)
        assert np.all(np.tril(R, -1) == 0)


def test_persistent_bits_depend_only_on_the_instance(fb, backend):
    rng = np.random.default_rng(12)
    mats = [randmatrix(rng, N, k) for N, k in SHAPES]
    _, Q1, R1 = run(fb, backend, mats)
    _, Q2, R2 = run(fb, backend, mats)
    assert all(a.tobytes() == b.tobytes() for a, b in zip(Q1 + R1, Q2 + R2))
    # Alone, or in another batch in another order: the same bits.
    for i in (2, 5, 8):
        _, Qa, Ra = run(fb, backend, [mats[i]])
        assert Qa[0].tobytes() == Q1[i].tobytes() and Ra[0].tobytes() == R1[i].tobytes()
    _, Qr, Rr = run(fb, backend, mats[::-1])
    assert all(a.tobytes() == b.tobytes() for a, b in zip(Qr[::-1] + Rr[::-1], Q1 + R1))


def test_persistent_agrees_with_the_lanes(fb, backend):
    rng = np.random.default_rng(13)
    mats = [randmatrix(rng, N, k) for N, k in SHAPES[:8]]
    _, Qp, Rp = run(fb, backend, mats)
    Ys = [backend.todevice(A) for A in mats]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in mats]
    fb.kernels.cholqr2_batched(backend, Ys, Rs, schedule="lanes")
    for Q, R, Y, Rl in zip(Qp, Rp, Ys, Rs):
        assert np.linalg.norm(Q - Y.to_host()) <= 1e-12 * np.linalg.norm(Q)
        assert np.linalg.norm(R - Rl.to_host()) <= 1e-12 * np.linalg.norm(R)


@pytest.mark.parametrize("kappa", [1e6, 1e10])
def test_persistent_conditioning_and_third_pass(fb, backend, oracle, kappa):
    # kappa = 1e6: pass 1 solves by blocks (cond_1(R) past the product by the
    # inverse); 1e10: the first Gram is shifted, a third pass runs, and the
    # 8 x 8 diagonal blocks are too ill-conditioned to invert (substitution).
    rng = np.random.default_rng(int(np.log10(kappa)))
    shapes = [(30000, 64), (4000, 23), (2500, 8), (50000, 40)]
    mats = [conditioned(rng, N, k, kappa) for N, k in shapes]
    passes, Qs, Rs = run(fb, backend, mats)
    shifted = kappa > 1 / np.sqrt(2.0 ** -52)
    # Whether the unshifted Cholesky of a numerically singular Gram matrix
    # fails is decided by rounding when only a few of its pivots lie below the
    # rounding noise, as in the reference (which shifts only on failure): the
    # 8-column instance at kappa = 1e10 has two such pivots, so a summation
    # order other than the oracle's may factor it unshifted, and both counts
    # are valid there. The wider instances have four or more and must shift.
    robust = [A.shape[1] >= 16 for A in mats]
    for A, Q, R, p, rob in zip(mats, Qs, Rs, passes, robust):
        N, k = A.shape
        _, passes_o = oracle.cholqr2(A.copy(order="F"))
        assert passes_o == (3 if shifted else 2)
        assert p == passes_o if rob else p in (2, 3)
        bound = 1e-8 if shifted else oracle.orthogonality_bound(np.complex128, N, k)
        assert np.linalg.norm(Q.conj().T @ Q - np.eye(k), 2) <= bound
        assert np.linalg.norm(Q @ R - A) <= 1e-10 * np.linalg.norm(A)
    # The lanes take the same paths: the same passes, and Q as close as two
    # summation orders of the first Gram allow (Q moves by about kappa eps).
    Ys = [backend.todevice(A) for A in mats]
    Rl = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in mats]
    passes_l = fb.kernels.cholqr2_batched(backend, Ys, Rl, schedule="lanes")
    for Q, Y, p, pl, rob in zip(Qs, Ys, passes, passes_l, robust):
        if rob:
            assert p == pl
        if p == pl:
            assert np.linalg.norm(Q - Y.to_host()) <= 1e-15 * kappa * np.linalg.norm(Q)


def test_persistent_failure_stops_only_its_instance(fb, backend):
    rng = np.random.default_rng(14)
    bad = randmatrix(rng, 4000, 4)
    bad[:, 2] = np.nan
    mats = [randmatrix(rng, 6000, 4), bad, randmatrix(rng, 90000, 32)]
    Ys = [backend.todevice(A) for A in mats]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in mats]
    with pytest.raises(fb.NotPositiveDefinite, match="instance 1"):
        fb.kernels.cholqr2_batched(backend, Ys, Rs, schedule="persistent")
    for i in (0, 2):
        assert orthogonality(Ys[i].to_host()) <= 1e-12
    # The failing instance's rows are left as they were (pass 1 failed).
    assert np.array_equal(np.isnan(Ys[1].to_host()), np.isnan(bad))


def test_persistent_batch_replays_as_one_graph(fb, backend):
    rng = np.random.default_rng(15)
    mats = [randmatrix(rng, N, k) for N, k in SHAPES]
    _, Qe, Re = run(fb, backend, mats)
    Ys = [backend.todevice(A) for A in mats]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in mats]
    nbytes = fb.kernels.cholqr2_batched_workspace_bytes([A.shape for A in mats], schedule="persistent")
    ws = backend.alloc_device(np.complex128, (nbytes // 16 + 16, 1))
    aligned = (ws.ptr + 255) // 256 * 256
    q = backend.make_queue()
    graph = backend.capture(q, lambda: fb.kernels.cholqr2_batched(
        backend, Ys, Rs, wait=False, workspace=(aligned, nbytes), schedule="persistent"))
    for _ in range(3):
        for A, Y in zip(mats, Ys):
            backend.h2d(Y, A)
        graph.launch(q)
        backend.sync_queue(q)
        for Y, R, Q0, R0 in zip(Ys, Rs, Qe, Re):
            assert Y.to_host().tobytes() == Q0.tobytes()
            assert R.to_host().tobytes() == R0.tobytes()


def test_persistent_batch_past_one_launch(fb, backend):
    # 400 instances: two launches of the kernel (384 and 16 instances).
    rng = np.random.default_rng(16)
    shapes = [(int(N), int(k)) for N, k in zip(rng.integers(100, 3000, 400), rng.integers(1, 65, 400))]
    mats = [randmatrix(rng, N, k) for N, k in shapes]
    passes, Qs, Rs = run(fb, backend, mats)
    assert passes == [2] * len(mats)
    for A, Q, R in zip(mats, Qs, Rs):
        k = A.shape[1]
        assert orthogonality(Q) <= 1e-12
        assert np.linalg.norm(Q @ R - A) <= 1e-13 * np.linalg.norm(A) * np.sqrt(k)
