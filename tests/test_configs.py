"""The configurations the north star names, run through the public API at
their stated sizes where the oracle finishes in seconds.

C1: cholqr2! on a PanelMatrix{ComplexF64} with N = 2^20, k = 32 and panel
width 8, whose entries come from GhostPanels(ComplexF64, N, k; seed =
0xdeadbeef) (src/panelblas.jl:130-139 on src/ghosts.jl:53-63 inputs). The
ghost matrix is filled on the device; its entries are checked bit for bit
against the oracle's C restatement of the fill, and Q and R against the
oracle's cholqr2! on those entries.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C1_N, C1_K, C1_W, C1_SEED = 1 << 20, 32, 8, 0xDEADBEEF


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def c1_entries():
    from oracle import ghost
    return ghost.ghost_block(np.complex128, C1_N, C1_K, 0, 0, C1_SEED)


@pytest.fixture(scope="module")
def c1_oracle(oracle, c1_entries):
    Qo = c1_entries.copy(order="F")
    Ro, passes = oracle.cholqr2(Qo, C1_W)
    return Qo, Ro, passes


@pytest.mark.parametrize("resident", [True, False])
def test_c1_ghost_panels_through_cholqr2_match_the_oracle(fb, backend, oracle, c1_entries, c1_oracle, resident):
    nbytes = C1_N * C1_K * 16
    # resident: the device budget holds the matrix, so cholqr2 runs the device
    # chain; streamed: a budget of about half of it (two staging row blocks of
    # 2^18 rows), so every pass streams through row sweeps: the Gram and the
    # solve, a later pass's Gram taken inside the previous solve sweep.
    budget = 4 * nbytes if resident else nbytes // 2 + (32 << 20)
    plan = fb.ResidencyPlan(device_budget=budget, host_budget=2 * nbytes + (64 << 20), backend=backend)
    Omega = fb.GhostPanels(np.complex128, C1_N, C1_K, plan=plan, seed=C1_SEED, w=C1_W)
    Y = fb.PanelMatrix.undef(np.complex128, C1_N, C1_K, plan=plan, w=C1_W)
    Y.copy_from(Omega)  # copyto!(Y, Omega)
    np.testing.assert_array_equal(Y.to_array(), c1_entries)
    R = fb.cholqr2(Y, resident=resident)
    Q = Y.to_array()
    Qo, Ro, passes = c1_oracle
    assert passes == 2
    assert rel(R, Ro) <= 1e-12
    assert rel(Q, Qo) <= 1e-12
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(c1_entries, Q, R) <= 1e-13
    fb.free(Y)


def test_copying_a_panel_matrix_into_itself_or_a_wrong_shape_is_refused(fb, backend):
    plan = fb.ResidencyPlan(device_budget=1 << 26, host_budget=1 << 26, backend=backend)
    Y = fb.PanelMatrix.undef(np.complex128, 1000, 8, plan=plan, w=4)
    with pytest.raises(fb.ArgumentError):
        Y.copy_from(Y)
    Omega = fb.GhostPanels(np.complex128, 1000, 6, plan=plan, seed=1, w=3)
    with pytest.raises(fb.DimensionMismatch):
        Y.copy_from(Omega)
    with pytest.raises(fb.ArgumentError):
        Omega.copy_from(Y)
    fb.free(Y)
