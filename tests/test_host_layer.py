"""The host layers over the B200 backend, mirroring the reference's own suites
(test/test_executor.jl, test/test_panelblas.jl, test/test_ghosts.jl,
test/test_cuda.jl): sweeps over column panels and row blocks at nbuffers 1
and 2, the panel BLAS against dense products and against the oracle, the
resident and streamed cholqr2!, and GhostPanels filled on the device against
the oracle's C restatement, bit for bit."""
import numpy as np
import pytest

from conftest import conditioned, randmatrix
from oracle import ghost as ghost_oracle

pytestmark = pytest.mark.gpu

BLAS_WIDTHS = (23, 12, 7, 1)
EPS = np.finfo(np.float64).eps
MiB = 2 ** 20


def blastol(N, k):
    return 100 * EPS * np.sqrt(N * k)


def orthogonality_bound(N, k):
    return 100 * N * k * EPS


def close(a, b, rtol):
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


@pytest.fixture
def plan(fb, backend):
    return fb.ResidencyPlan(device_budget=64 * MiB, host_budget=64 * MiB, backend=backend)


@pytest.fixture
def make_plan(fb, backend):
    def make(**kw):
        kw.setdefault("device_budget", 64 * MiB)
        kw.setdefault("host_budget", 64 * MiB)
        return fb.ResidencyPlan(backend=backend, **kw)
    return make


@pytest.fixture
def rng():
    return np.random.default_rng(20240611)


# ---- sweeps (test/test_executor.jl) -------------------------------------------

def collect_sweep(fb, backend, X, nb, traversal=None):
    """Copies every step's buffer into one device matrix and brings it back."""
    D = backend.alloc_device(np.complex128, X.shape)
    if traversal is None:
        def f(j, Xb):
            cols = X.panelrange(j)
            fb.kernels.convert_copy(backend, D.view(slice(None), slice(cols.start, cols.stop)), Xb)
    else:
        def f(step, Xb):
            rows = traversal.blocks[step]
            fb.kernels.convert_copy(backend, D.view(slice(rows.start, rows.stop), slice(None)), Xb)
    fb.sweep(f, fb.readpanels(X), nbuffers=nb, traversal=traversal)
    return D.to_host()


@pytest.mark.parametrize("w", [23, 7, 1])
@pytest.mark.parametrize("nb", [1, 2])
def test_read_only_sweep_sees_every_panel(fb, backend, plan, rng, w, nb):
    A = randmatrix(rng, 40, 23)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    assert np.array_equal(collect_sweep(fb, backend, X, nb), A)
    assert np.array_equal(collect_sweep(fb, backend, X, nb, fb.rowtraversal(X)), A)
    assert np.array_equal(X.to_array(), A)


@pytest.mark.parametrize("w", [23, 7, 1])
@pytest.mark.parametrize("nb", [1, 2])
def test_read_write_sweeps(fb, backend, plan, rng, w, nb):
    A = randmatrix(rng, 40, 23)
    halves = {}

    def half(width):
        if width not in halves:
            halves[width] = backend.todevice(np.eye(width, dtype=np.complex128) * 0.5)
        return halves[width]

    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    fb.sweep(lambda j, Xb: fb.kernels.rdiv_upper(backend, Xb, half(Xb.cols)), fb.updatepanels(X), nbuffers=nb)
    assert np.array_equal(X.to_array(), 2 * A)
    fb.sweep(lambda s, Xb: fb.kernels.rdiv_upper(backend, Xb, half(Xb.cols)), fb.updatepanels(X), nbuffers=nb,
             traversal=fb.rowtraversal(X))
    assert np.array_equal(X.to_array(), 4 * A)
    assert all(p.dirty and p.epoch >= 3 for p in X.panels)


@pytest.mark.parametrize("w", [23, 7, 1])
@pytest.mark.parametrize("nb", [1, 2])
def test_produce_sweep(fb, backend, plan, rng, w, nb):
    A = randmatrix(rng, 40, 23)
    D = backend.todevice(A)
    Y = fb.PanelMatrix.undef(np.complex128, 40, 23, plan=plan, w=w)

    def f(j, Yb):
        cols = Y.panelrange(j)
        fb.kernels.convert_copy(backend, Yb, D.view(slice(None), slice(cols.start, cols.stop)))

    fb.sweep(f, fb.writepanels(Y), nbuffers=nb)
    assert np.array_equal(Y.to_array(), A)


def test_panel_functions_run_on_the_sweeps_queue(fb, backend, plan, rng):
    X = fb.PanelMatrix.from_array(randmatrix(rng, 40, 23), plan=plan, w=7)
    seen = []
    fb.sweep(lambda j, Xb: seen.append(backend.current_queue), fb.readpanels(X))
    assert len(seen) == X.npanels() and all(q is not None for q in seen) and len({id(q) for q in seen}) == 1
    assert backend.current_queue is None


def test_narrowed_host_storage_streams_through_the_sweep(fb, backend, make_plan, rng):
    A = randmatrix(rng, 40, 23)
    plan = make_plan(host_eltype=np.complex64)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=7)
    stored = A.astype(np.complex64).astype(np.complex128)
    assert np.array_equal(collect_sweep(fb, backend, X, 2), stored)
    assert np.array_equal(collect_sweep(fb, backend, X, 1, fb.rowtraversal(X)), stored)
    Y = fb.PanelMatrix.undef(np.complex128, 40, 23, plan=plan, w=7)
    D = backend.todevice(A)
    fb.sweep(lambda j, Yb: fb.kernels.convert_copy(backend, Yb, D.view(slice(None), slice(j * 7, j * 7 + Yb.cols))),
             fb.writepanels(Y))
    assert np.array_equal(Y.to_array(), stored)


def test_sweeps_give_their_buffers_back_and_allocate_nothing_after_warmup(fb, backend, plan, rng):
    A = randmatrix(rng, 40, 23)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=7)
    Y = fb.PanelMatrix.from_array(randmatrix(rng, 40, 23), plan=plan, w=7)
    Z = fb.PanelMatrix.undef(np.complex128, 40, 12, plan=plan, w=5)
    dense = fb.DenseOperator(backend, randmatrix(rng, 40, 40))
    C, D = randmatrix(rng, 23, 12), randmatrix(rng, 23, 23)

    def everything():
        fb.gram(X, Y)
        fb.project(X, dense)
        fb.rightmul(Z, X, C)
        fb.rightmul(Y, D)
        fb.cholqr2(Y, resident=False)
        fb.cholqr2(Y, resident=True)

    everything()
    before = (fb.device_bytes_allocated(plan), backend.device_bytes_allocated)
    everything()
    assert (fb.device_bytes_allocated(plan), backend.device_bytes_allocated) == before
    assert all(p.pins == 0 for m in (X, Y, Z) for p in m.panels)


def test_a_failing_panel_function_surfaces_and_frees_its_buffers(fb, backend, plan, rng):
    X = fb.PanelMatrix.from_array(randmatrix(rng, 40, 23), plan=plan, w=7)
    collect_sweep(fb, backend, X, 2)
    before = fb.device_bytes_allocated(plan)

    def boom(j, Xb):
        if j == 1:
            raise RuntimeError("panel function failed")

    with pytest.raises(RuntimeError, match="panel function failed"):
        fb.sweep(boom, fb.readpanels(X))
    assert all(p.pins == 0 for p in X.panels)
    collect_sweep(fb, backend, X, 2)
    assert fb.device_bytes_allocated(plan) == before


def test_sweep_validation(fb, plan, make_plan, rng):
    X = fb.PanelMatrix.from_array(randmatrix(rng, 10, 20), plan=plan, w=7)
    Y = fb.PanelMatrix.from_array(randmatrix(rng, 10, 20), plan=plan, w=5)
    noop = lambda *a: None
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop)
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop, fb.readpanels(X), fb.readpanels(X))
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop, fb.readpanels(X), nbuffers=0)
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop, fb.readpanels(X), fb.readpanels(Y))
    other = fb.PanelMatrix.from_array(randmatrix(rng, 10, 20), plan=make_plan(), w=7)
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop, fb.readpanels(X), fb.readpanels(other))
    with pytest.raises(fb.ArgumentError):
        fb.sweep(noop, fb.updatepanels(X), traversal=fb.PanelSteps([0, 1, 0]))
    fb.sweep(noop, fb.readpanels(X), traversal=fb.PanelSteps([0, 1, 0]))


@pytest.mark.parametrize("N", [12, 13, 1])
@pytest.mark.parametrize("h", [1, 3, 5, 20])
def test_row_blocks_tile_the_rows_exactly(fb, N, h):
    blocks = fb.RowSteps(N, h).blocks
    assert [i for b in blocks for i in b] == list(range(N))
    assert all(len(b) == min(h, N) for b in blocks[:-1])


def test_a_custom_traversal_labels_its_steps(fb, backend, plan, rng):
    X = fb.PanelMatrix.from_array(randmatrix(rng, 10, 20), plan=plan, w=7)
    seen = []
    fb.sweep(lambda label, Xb: seen.append((label, Xb.cols)), fb.readpanels(X),
             traversal=fb.PanelSteps([2, 0, 2], ["a", "b", "c"]))
    assert seen == [("a", 6), ("b", 7), ("c", 6)]


# ---- panel BLAS (test/test_panelblas.jl) --------------------------------------

@pytest.mark.parametrize("w", BLAS_WIDTHS)
@pytest.mark.parametrize("nb", [1, 2])
def test_gram_against_dense(fb, plan, rng, w, nb):
    N, k = 40, 23
    A, B = randmatrix(rng, N, k), randmatrix(rng, N, k)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    Y = fb.PanelMatrix.from_array(B, plan=plan, w=w)
    tol = blastol(N, k)
    assert close(fb.gram(X, Y, nbuffers=nb), A.conj().T @ B, tol)
    assert close(fb.gram(X, nbuffers=nb), A.conj().T @ A, tol)
    assert np.array_equal(fb.gram(X, X, nbuffers=nb), fb.gram(X, nbuffers=nb))
    assert np.array_equal(X.to_array(), A)


@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_gram_is_the_same_to_the_bit_at_nbuffers_1_and_2(fb, plan, rng, w):
    A, B = randmatrix(rng, 40, 23), randmatrix(rng, 40, 23)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    Y = fb.PanelMatrix.from_array(B, plan=plan, w=w)
    assert np.array_equal(fb.gram(X, Y, nbuffers=1), fb.gram(X, Y, nbuffers=2))
    assert np.array_equal(fb.gram(X, nbuffers=1), fb.gram(X, nbuffers=2))


def test_gram_matches_the_oracles_row_block_order(fb, oracle, make_plan, rng):
    # A long matrix, so the rows cut into several blocks and the carry rule runs.
    N, k, w = 5000, 16, 4
    A = randmatrix(rng, N, k)
    plan = make_plan(device_budget=2 * N * w * 16 + 8 * MiB, panel_width=w)
    X = fb.PanelMatrix.from_array(A, plan=plan)
    assert len(fb.rowtraversal(X).blocks) == 4
    G = fb.gram(X)
    ref = oracle.gram(A, w=w)
    assert close(G, ref, blastol(N, k))


def test_gram_with_narrowed_host_storage(fb, make_plan, rng):
    A = randmatrix(rng, 40, 23)
    X = fb.PanelMatrix.from_array(A, plan=make_plan(host_eltype=np.complex64), w=7)
    stored = A.astype(np.complex64).astype(np.complex128)
    assert close(fb.gram(X), stored.conj().T @ stored, blastol(40, 23))


def test_gram_rejects_mismatched_operands(fb, plan, make_plan):
    X = fb.PanelMatrix.undef(np.complex128, 10, 20, plan=plan, w=7)
    with pytest.raises(fb.ArgumentError):
        fb.gram(X, fb.PanelMatrix.undef(np.complex128, 10, 20, plan=plan, w=5))
    with pytest.raises(fb.ArgumentError):
        fb.gram(X, fb.PanelMatrix.undef(np.complex128, 10, 20, plan=make_plan(), w=7))


@pytest.mark.parametrize("w", BLAS_WIDTHS)
@pytest.mark.parametrize("nb", [1, 2])
def test_panelmul_against_dense(fb, backend, plan, rng, w, nb):
    N, k = 40, 23
    A, G = randmatrix(rng, N, k), randmatrix(rng, N, N)
    dense = fb.DenseOperator(backend, G)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    Y = fb.PanelMatrix.undef(np.complex128, N, k, plan=plan, w=w)
    tol = blastol(N, k)
    assert close(fb.panelmul(Y, dense, X, nbuffers=nb).to_array(), G @ A, tol)
    assert close(fb.panelmul(Y, fb.ColumnOperator(dense), X, nbuffers=nb).to_array(), G @ A, tol)


@pytest.mark.parametrize("mn", [(40, 25), (25, 40)])
def test_panelmul_with_a_rectangular_operator(fb, backend, plan, rng, mn):
    m, n = mn
    k, w = 23, 7
    A, G = randmatrix(rng, n, k), randmatrix(rng, m, n)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    Y = fb.PanelMatrix.undef(np.complex128, m, k, plan=plan, w=w)
    assert close(fb.panelmul(Y, fb.DenseOperator(backend, G), X).to_array(), G @ A, blastol(max(m, n), k))


def test_panelmul_rejects_an_operator_that_does_not_fit(fb, backend, plan, rng):
    X = fb.PanelMatrix.undef(np.complex128, 10, 20, plan=plan, w=7)
    Y = fb.PanelMatrix.undef(np.complex128, 10, 20, plan=plan, w=7)
    for G in (randmatrix(rng, 10, 9), randmatrix(rng, 11, 11)):
        with pytest.raises((fb.ArgumentError, fb.DimensionMismatch)):
            fb.panelmul(Y, fb.DenseOperator(backend, G), X)
    with pytest.raises(fb.ArgumentError):
        fb.panelmul(X, fb.DenseOperator(backend, randmatrix(rng, 10, 10)), X)


@pytest.mark.parametrize("r", [12, 23, 31])
@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_rightmul_out_of_place_against_dense(fb, plan, rng, r, w):
    N, s = 40, 23
    A, C = randmatrix(rng, N, s), randmatrix(rng, s, r)
    src = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    dest = fb.PanelMatrix.undef(np.complex128, N, r, plan=plan, w=min(max(w - 3, 1), r))
    assert fb.rightmul(dest, src, C) is dest
    assert close(dest.to_array(), A @ C, blastol(N, max(s, r)))
    assert np.array_equal(src.to_array(), A)


@pytest.mark.parametrize("w", BLAS_WIDTHS)
@pytest.mark.parametrize("nb", [1, 2])
def test_rightmul_in_place_against_dense(fb, plan, rng, w, nb):
    N, k = 40, 23
    A, C = randmatrix(rng, N, k), randmatrix(rng, k, k)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    assert fb.rightmul(Y, C, nbuffers=nb) is Y
    assert close(Y.to_array(), A @ C, blastol(N, k))


@pytest.mark.parametrize("w", BLAS_WIDTHS)
def test_rightmul_is_the_same_to_the_bit_at_nbuffers_1_and_2(fb, make_plan, rng, w):
    N, s, r = 40, 23, 12
    A, C, D = randmatrix(rng, N, s), randmatrix(rng, s, r), randmatrix(rng, s, s)
    produced, inplace = [], []
    for nb in (1, 2):
        p = make_plan()
        src = fb.PanelMatrix.from_array(A, plan=p, w=w)
        dest = fb.PanelMatrix.undef(np.complex128, N, r, plan=p, w=min(max(w - 3, 1), r))
        produced.append(fb.rightmul(dest, src, C, nbuffers=nb).to_array())
        inplace.append(fb.rightmul(fb.PanelMatrix.from_array(A, plan=p, w=w), D, nbuffers=nb).to_array())
    assert np.array_equal(*produced) and np.array_equal(*inplace)


def test_rightmul_rejects_factors_and_matrices_that_do_not_fit(fb, plan, make_plan, rng):
    N, s, r, w = 20, 12, 8, 5
    Y = fb.PanelMatrix.from_array(randmatrix(rng, N, s), plan=plan, w=w)
    dest = fb.PanelMatrix.undef(np.complex128, N, r, plan=plan, w=4)
    ghost = fb.GhostPanels(np.complex128, N, s, plan=plan, w=w)
    bad = [(Y, randmatrix(rng, s, r)), (Y, randmatrix(rng, r, s)), (dest, Y, randmatrix(rng, s, s)),
           (Y, Y, randmatrix(rng, s, s)), (ghost, randmatrix(rng, s, s)), (ghost, Y, randmatrix(rng, s, s)),
           (dest, fb.PanelMatrix.undef(np.complex128, N + 1, s, plan=plan, w=w), randmatrix(rng, s, r)),
           (dest, fb.PanelMatrix.undef(np.complex128, N, s, plan=make_plan(), w=w), randmatrix(rng, s, r))]
    for args in bad:
        with pytest.raises(fb.ArgumentError):
            fb.rightmul(*args)


@pytest.mark.parametrize("resident", [True, False])
@pytest.mark.parametrize("w", BLAS_WIDTHS)
@pytest.mark.parametrize("nb", [1, 2])
def test_cholqr2_orthonormalizes(fb, plan, rng, resident, w, nb):
    N, k = 40, 23
    A = randmatrix(rng, N, k)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    R = fb.cholqr2(Y, nbuffers=nb, resident=resident)
    Q = Y.to_array()
    assert R.shape == (k, k) and np.array_equal(R, np.triu(R))
    assert np.linalg.norm(Q.conj().T @ Q - np.eye(k), 2) <= orthogonality_bound(N, k)
    assert close(Q @ R, A, blastol(N, k))


@pytest.mark.parametrize("resident", [True, False])
@pytest.mark.parametrize("kappa", [1e2, 1e6, 1e10])
def test_cholqr2_survives_kappa(fb, plan, rng, resident, kappa):
    N, k, w = 40, 23, 7
    A = conditioned(rng, N, k, kappa)
    Y = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    R = fb.cholqr2(Y, resident=resident)
    Q = Y.to_array()
    shifted = kappa > 1 / np.sqrt(EPS)
    bound = 1e-8 if shifted else orthogonality_bound(N, k)
    assert np.linalg.norm(Q.conj().T @ Q - np.eye(k), 2) <= bound
    assert np.linalg.norm(Q @ R - A) <= 1e-10 * np.linalg.norm(A)


def test_cholqr2_streamed_matches_the_oracle(fb, oracle, make_plan, rng):
    N, k, w = 5000, 16, 4
    A = conditioned(rng, N, k, 1e5)
    plan = make_plan(device_budget=2 * N * w * 16 + 8 * MiB, panel_width=w)
    Y = fb.PanelMatrix.from_array(A, plan=plan)
    R = fb.cholqr2(Y, resident=False)
    Q = Y.to_array()
    Rref, passes = oracle.cholqr2(A.copy(order="F"), w)
    assert passes == 2
    assert close(R, Rref, 1e-10)
    assert oracle.orthogonality_error(Q) <= orthogonality_bound(N, k)


def separate_sweeps(fb, Y, forced_unit_roundoff=None):
    """cholqr2! with every pass's Gram a sweep of its own, read back from the
    host panels (the reference's order, src/panelblas.jl:141-146)."""
    pb, plan = fb.panelblas, Y.plan
    G = plan.backend.alloc_device(np.complex128, (Y.k, Y.k))
    U = plan.backend.alloc_device(np.complex128, (Y.k, Y.k))
    R, npasses, p = None, 2, 0
    while p < npasses:
        pb.gram_rows(Y, G)
        if pb.cholesky_upper(plan, G, Y.N, Y.k, U, forced_unit_roundoff if p == 0 else None):
            npasses = 3
        pb.rdiv_rows(Y, U)
        Rp = pb.collect_small(U, plan)
        R = Rp if R is None else Rp @ R
        p += 1
    return R, npasses


@pytest.mark.parametrize("kappa,forced,passes", [(1e5, None, 2), (1e5, 2.0 ** -24, 3), (1e13, None, 3)])
def test_streamed_gram_taken_in_the_solve_sweep_has_the_bits_of_its_own_sweep(fb, make_plan, rng, kappa, forced,
                                                                                 passes):
    N, k, w = 5000, 16, 4
    A = conditioned(rng, N, k, kappa)
    plan = make_plan(device_budget=2 * N * w * 16 + 8 * MiB, panel_width=w)
    Y = fb.PanelMatrix.from_array(A, plan=plan)
    R = fb.cholqr2(Y, resident=False) if forced is None else fb.cholqr3(Y, resident=False, unit_roundoff=forced)
    Y2 = fb.PanelMatrix.from_array(A, plan=plan)
    R2, n = separate_sweeps(fb, Y2, forced)
    assert n == passes
    assert np.array_equal(R, R2)
    assert np.array_equal(Y.to_array(), Y2.to_array())


def test_cholqr2_refuses_an_indefinite_gram_and_a_ghost(fb, plan, rng):
    A = randmatrix(rng, 40, 6)
    A[:, 3] = 0
    for resident in (True, False):
        Y = fb.PanelMatrix.from_array(A, plan=plan, w=2)
        # A zero column survives the shift (the factor is then rank deficient),
        # so the orthonormality is not promised; the call must still return.
        R = fb.cholqr2(Y, resident=resident)
        assert np.all(np.isfinite(R))
    with pytest.raises(fb.ArgumentError):
        fb.cholqr2(fb.GhostPanels(np.complex128, 40, 6, plan=plan, w=2))


@pytest.mark.parametrize("w", BLAS_WIDTHS)
@pytest.mark.parametrize("nb", [1, 2])
def test_project_against_dense(fb, backend, plan, rng, w, nb):
    N, k = 40, 23
    G, A = randmatrix(rng, N, N), randmatrix(rng, N, k)
    dense = fb.DenseOperator(backend, G)
    Q = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    ref = A.conj().T @ G @ A
    tol = blastol(N, k)
    for schedule in (None,) + fb.panelblas.PROJECT_SCHEDULES:
        assert close(fb.project(Q, dense, nbuffers=nb, schedule=schedule), ref, tol), schedule
        assert close(fb.project(Q, fb.ColumnOperator(dense), nbuffers=nb, schedule=schedule), ref, tol), schedule
    assert np.array_equal(Q.to_array(), A)


def test_project_schedule_follows_the_budgets(fb, backend, make_plan, rng):
    """Resident when Q and G Q fit the device budget, two sweeps when only a
    second matrix fits on the host, nested (the reference's) when neither;
    all three give the same S."""
    N, k, w = 20_000, 48, 4
    L = fb.Laplacian7((50, 40, 10), 0.5 + 0.1j)
    A = randmatrix(rng, N, k)
    nbytes = N * k * 16
    # Room for the sweeps' staging buffers (the pool keeps those of both of
    # the two-sweep schedule's sweeps, 10.3 MB), not for Q and G Q together.
    small = 12 * MiB
    cases = {"resident": make_plan(device_budget=4 * nbytes, host_budget=4 * nbytes, panel_width=w),
             "two-sweep": make_plan(device_budget=small, host_budget=4 * nbytes, panel_width=w),
             "nested": make_plan(device_budget=small, host_budget=nbytes + MiB, panel_width=w)}
    results = {}
    for want, p in cases.items():
        Q = fb.PanelMatrix.from_array(A, plan=p)
        assert fb.panelblas.project_schedule(Q) == want
        results[want] = fb.project(Q, L)
    tol = blastol(N, k)
    assert close(results["two-sweep"], results["nested"], tol)
    assert close(results["resident"], results["nested"], tol)


def test_project_matches_panelmul_followed_by_gram(fb, backend, plan, rng):
    N, k, w = 40, 23, 7
    dense = fb.DenseOperator(backend, randmatrix(rng, N, N))
    Q = fb.PanelMatrix.from_array(randmatrix(rng, N, k), plan=plan, w=w)
    Z = fb.PanelMatrix.undef(np.complex128, N, k, plan=plan, w=w)
    fb.panelmul(Z, dense, Q)
    assert close(fb.project(Q, dense), fb.gram(Q, Z), blastol(N, k))


def test_repeated_calls_keep_their_schedule(fb, backend, make_plan, rng):
    """The plan's pool keeps the buffers a resident call checked out; a
    second call of the same shape reuses them and stays resident."""
    N, k, w = 20_000, 12, 4
    nbytes = N * k * 16
    p = make_plan(device_budget=2 * nbytes + 4 * MiB, host_budget=4 * nbytes, panel_width=w)
    Q = fb.PanelMatrix.from_array(randmatrix(rng, N, k), plan=p)
    L = fb.Laplacian7((50, 40, 10), 0.5)
    for _ in range(3):
        assert fb.panelblas.project_schedule(Q) == "resident"
        fb.project(Q, L)
    Y = fb.PanelMatrix.from_array(randmatrix(rng, N, k), plan=make_plan(device_budget=nbytes + 64 * MiB,
                                                                         host_budget=2 * nbytes, panel_width=w))
    for _ in range(3):
        assert fb.panelblas.fits_on_device(Y)
        fb.cholqr2(Y)


def test_project_follows_the_operators_adjoint(fb, backend, plan, rng):
    N, k, w = 40, 23, 7
    G = randmatrix(rng, N, N)
    Q = fb.PanelMatrix.from_array(randmatrix(rng, N, k), plan=plan, w=w)
    tol = blastol(N, k)
    S = fb.project(Q, fb.DenseOperator(backend, G))
    assert close(fb.project(Q, fb.DenseOperator(backend, G.conj().T)), S.conj().T, tol)
    H = np.triu(G) + np.triu(G, 1).conj().T
    H[np.diag_indices(N)] = H.diagonal().real
    SH = fb.project(Q, fb.DenseOperator(backend, H))
    assert close(SH, SH.conj().T, tol)


# ---- ghosts (test/test_ghosts.jl) ----------------------------------------------

@pytest.mark.parametrize("dtype,value", [(np.complex128, np.complex128), (np.complex128, np.complex64),
                                         (np.complex64, np.complex64), (np.float64, np.float64),
                                         (np.float32, np.float32)])
def test_device_fill_matches_the_oracle_bit_for_bit(fb, backend, dtype, value):
    rows, cols, row0, col0, seed = 3001, 5, 12345, 7, 0xDEADBEEF
    D = backend.alloc_device(dtype, (rows, cols))
    fb.kernels.ghost_fill(backend, D, row0, col0, seed, value)
    backend.sync_all()
    ref = ghost_oracle.ghost_block(dtype, rows, cols, row0, col0, seed, value)
    got = D.to_host()
    assert got.dtype == np.dtype(dtype)
    assert got.tobytes(order="F") == ref.tobytes(order="F")


def test_device_fill_writes_only_its_view(fb, backend):
    big = np.full((50, 9), 7 + 7j)
    D = backend.todevice(big)
    fb.kernels.ghost_fill(backend, D.view(slice(3, 40), slice(2, 6)), 3, 2, 11, np.complex128)
    got = D.to_host()
    ref = ghost_oracle.ghost_block(np.complex128, 50, 9, 0, 0, 11)
    assert np.array_equal(got[3:40, 2:6], ref[3:40, 2:6])
    mask = np.ones_like(big, dtype=bool)
    mask[3:40, 2:6] = False
    assert np.all(got[mask] == 7 + 7j)


@pytest.mark.parametrize("w", [8, 7, 1])
def test_a_ghost_matrix_regenerates_the_same_entries(fb, plan, make_plan, w):
    N, k = 24, 8
    G = fb.GhostPanels(np.complex128, N, k, plan=plan, seed=0xDEADBEEF, w=w)
    assert G.shape == (N, k) and G.npanels() == -(-k // w)
    A = G.to_array()
    assert np.array_equal(A, G.to_array())
    assert np.array_equal(A, fb.GhostPanels(np.complex128, N, k, plan=make_plan(), seed=0xDEADBEEF, w=w).to_array())
    assert not np.array_equal(A, fb.GhostPanels(np.complex128, N, k, plan=make_plan(), seed=0xDEADBEEF + 1,
                                                w=w).to_array())
    assert 0.5 < np.linalg.norm(A) / np.sqrt(N * k) < 2
    assert np.linalg.matrix_rank(A) == min(N, k)
    assert np.array_equal(A, ghost_oracle.ghost_block(np.complex128, N, k, 0, 0, 0xDEADBEEF))


def test_the_same_seed_gives_the_same_matrix_at_every_width_and_traversal(fb, backend, make_plan):
    N, k = 40, 23
    ref = fb.GhostPanels(np.complex128, N, k, plan=make_plan(), seed=0xDEADBEEF, w=23).to_array()
    for w in (23, 12, 7, 1):
        G = fb.GhostPanels(np.complex128, N, k, plan=make_plan(), seed=0xDEADBEEF, w=w)
        assert np.array_equal(G.to_array(), ref)
        for nb in (1, 2):
            assert np.array_equal(collect_sweep(fb, backend, G, nb), ref)
        rows = fb.RowSteps(N, 9)
        assert np.array_equal(collect_sweep(fb, backend, G, 2, rows), ref)


def test_the_generator_sees_each_columns_index_in_the_full_matrix(fb, plan):
    def gen(dst, rng, col):
        dst[:] = col
    G = fb.GhostPanels(np.complex128, 12, 7, plan=plan, w=3, generator=gen)
    assert np.array_equal(G.to_array(), np.tile(np.arange(1, 8), (12, 1)).astype(np.complex128))


@pytest.mark.parametrize("w", [23, 7, 1])
def test_a_per_column_generator_is_free_of_the_panel_boundaries(fb, backend, make_plan, w):
    def gen(dst, rng, col):
        dst[:] = rng.standard_normal(len(dst)) + 1j * rng.standard_normal(len(dst))
        dst /= np.linalg.norm(dst)
    G = fb.GhostPanels(np.complex128, 40, 23, plan=make_plan(), seed=0xDEADBEEF, w=w, generator=gen)
    A = G.to_array()
    assert np.allclose(np.linalg.norm(A, axis=0), 1)
    ref = fb.GhostPanels(np.complex128, 40, 23, plan=make_plan(), seed=0xDEADBEEF, w=23, generator=gen).to_array()
    assert np.array_equal(A, ref)
    assert np.array_equal(collect_sweep(fb, backend, G, 2), ref)


def test_a_ghost_matrix_narrows_its_host_storage(fb, make_plan):
    plan = make_plan(host_eltype=np.complex64)
    G = fb.GhostPanels(np.complex128, 40, 7, plan=plan, seed=5, w=3)
    A = G.to_array()
    assert A.dtype == np.complex128
    assert np.array_equal(A, A.astype(np.complex64).astype(np.complex128))
    assert np.array_equal(A, ghost_oracle.ghost_block(np.complex128, 40, 7, 0, 0, 5, np.complex64))


@pytest.mark.parametrize("w", [4, 3])
def test_a_ghost_matrix_feeds_the_operator_sweeps(fb, backend, plan, rng, w):
    m, n, k = 40, 25, 10
    Gm = randmatrix(rng, m, n)
    ghost = fb.GhostPanels(np.complex128, n, k, plan=plan, seed=0xDEADBEEF, w=w)
    Omega = ghost.to_array()
    Y = fb.PanelMatrix.undef(np.complex128, m, k, plan=plan, w=w)
    fb.panelmul(Y, fb.DenseOperator(backend, Gm), ghost)
    assert close(Y.to_array(), Gm @ Omega, blastol(m, k))
    assert close(fb.gram(ghost), Omega.conj().T @ Omega, blastol(n, k))
    C = randmatrix(rng, k, 6)
    dest = fb.PanelMatrix.undef(np.complex128, n, 6, plan=plan, w=3)
    assert close(fb.rightmul(dest, ghost, C).to_array(), Omega @ C, blastol(n, k))
    assert np.array_equal(ghost.to_array(), Omega)


def test_a_ghost_matrix_refuses_to_be_written_to(fb, backend, plan):
    ghost = fb.GhostPanels(np.complex128, 20, 6, plan=plan, w=2)
    with pytest.raises(fb.ArgumentError):
        fb.sweep(lambda *a: None, fb.updatepanels(ghost))
    with pytest.raises(fb.ArgumentError):
        fb.sweep(lambda *a: None, fb.writepanels(ghost))
    with pytest.raises(fb.ArgumentError):
        fb.panelmul(ghost, fb.DenseOperator(backend, np.eye(20)),
                    fb.PanelMatrix.undef(np.complex128, 20, 6, plan=plan, w=2))


# ---- the matrix-free Laplacian operator ---------------------------------------

@pytest.mark.parametrize("grid", [(5, 4, 3), (7, 1, 1), (1, 1, 1), (3, 6, 2), (33, 17, 9)])
def test_laplacian_matches_the_sparse_operator(fb, backend, oracle, rng, grid):
    n = grid[0] * grid[1] * grid[2]
    shift = 0.5 + 0.1j
    X = randmatrix(rng, n, 5)
    D = backend.todevice(X)
    Y = backend.alloc_device(np.complex128, (n, 5))
    fb.Laplacian7(grid, shift).apply(backend, Y, D)
    backend.sync_all()
    ref = oracle.laplacian7(grid, shift) @ X
    assert np.linalg.norm(Y.to_host() - ref) <= 1e-15 * np.linalg.norm(ref) * 10


def test_laplacian_refuses_aliasing_and_wrong_shapes(fb, backend, rng):
    D = backend.todevice(randmatrix(rng, 60, 3))
    with pytest.raises(fb.ArgumentError):
        fb.Laplacian7((5, 4, 3), 0.5).apply(backend, D, D)
    with pytest.raises(fb.DimensionMismatch):
        fb.Laplacian7((5, 4, 2), 0.5).apply(backend, backend.alloc_device(np.complex128, (60, 3)), D)
    with pytest.raises(fb.ArgumentError):
        fb.Laplacian7((5, 0, 2), 0.5)


@pytest.mark.parametrize("w", [7, 1])
def test_panelmul_and_project_with_the_laplacian(fb, backend, oracle, plan, rng, w):
    grid, shift = (6, 5, 4), 0.5 + 0.1j
    n, k = 120, 23
    G = fb.Laplacian7(grid, shift)
    L = oracle.laplacian7(grid, shift)
    A = randmatrix(rng, n, k)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
    Y = fb.PanelMatrix.undef(np.complex128, n, k, plan=plan, w=w)
    tol = blastol(n, k)
    assert close(fb.panelmul(Y, G, X).to_array(), L @ A, tol)
    assert close(fb.panelmul(Y, fb.ColumnOperator(G), X).to_array(), L @ A, tol)
    assert close(fb.project(X, G), A.conj().T @ (L @ A), tol)
    ghost = fb.GhostPanels(np.complex128, n, k, plan=plan, seed=0xDEADBEEF, w=w)
    Omega = ghost.to_array()
    assert close(fb.panelmul(Y, G, ghost).to_array(), L @ Omega, tol)
