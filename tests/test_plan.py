"""The plan's arithmetic and pools (test/test_plan.jl), on a stand-in backend
that hands out host memory, so these run without a GPU."""
import numpy as np
import pytest


class FakeDevice:
    def __init__(self, dtype, dims):
        self.dtype = np.dtype(dtype)
        self.shape = tuple(dims)


class FakeSlab:
    def __init__(self, nbytes):
        self.nbytes = int(nbytes)
        self.buf = np.zeros(self.nbytes + 64, dtype=np.uint8)
        self.base = (-self.buf.ctypes.data) % 64

    def matrix(self, dtype, dims, offset=0):
        dtype = np.dtype(dtype)
        n = int(np.prod(dims)) * dtype.itemsize
        assert offset + n <= self.nbytes
        start = self.base + offset
        return self.buf[start:start + n].view(dtype).reshape(dims, order="F")


class FakeBackend:
    def supports_eltype(self, dtype):
        return np.dtype(dtype) == np.complex128

    def alloc_device(self, dtype, dims):
        return FakeDevice(dtype, dims)

    def alloc_host_slab(self, nbytes):
        return FakeSlab(nbytes)


@pytest.fixture
def plan_mod(fb):
    import importlib
    return importlib.import_module(fb.__name__ + ".plan")


def make_plan(fb, **kw):
    kw.setdefault("device_budget", 64 * 2 ** 20)
    kw.setdefault("host_budget", 64 * 2 ** 20)
    return fb.ResidencyPlan(backend=FakeBackend(), **kw)


C128 = np.complex128


def test_plan_construction(fb):
    plan = make_plan(fb, workspace_bytes=2 ** 20)
    assert plan.device_budget == 64 * 2 ** 20
    assert plan.devicepool.budget == 64 * 2 ** 20 - 2 ** 20
    assert "ResidencyPlan" in repr(plan)
    for bad in (dict(nbuffers=0), dict(host_budget=0), dict(workspace_bytes=-1),
                dict(device_budget=2 ** 20, workspace_bytes=2 ** 20), dict(panel_width=0),
                dict(target_panel_bytes=0)):
        with pytest.raises(fb.ArgumentError):
            make_plan(fb, **bad)


def test_panel_width_arithmetic(fb, plan_mod):
    p = plan_mod
    assert p.panel_bytes(1000, 8, C128) == 1000 * 8 * 16
    assert p.device_bytes_required(1000, 8, C128, nbuffers=2, workspace_bytes=7) == 2 * 1000 * 8 * 16 + 7
    assert p.choose_panel_width(100, 64, C128, device_budget=1 << 30) == 64
    assert p.choose_panel_width(100, 64, C128, device_budget=2 * 2 * 100 * 16) == 2
    assert p.choose_panel_width(100, 1000, C128, device_budget=2 * 999 * 100 * 16) == 500
    assert p.choose_panel_width(100, 64, C128, device_budget=1 << 30, target_panel_bytes=8 * 100 * 16) == 8
    assert p.choose_panel_width(100, 64, C128, device_budget=1 << 30, target_panel_bytes=1) == 1
    for args in ((100, 64, C128, 100 * 16), (0, 64, C128, 1 << 30), (100, 0, C128, 1 << 30)):
        with pytest.raises(fb.ArgumentError):
            p.choose_panel_width(*args[:3], device_budget=args[3])


def test_panel_width_properties(plan_mod):
    p = plan_mod
    rng = np.random.default_rng(0xdeadbeef)
    for _ in range(400):
        N = int(rng.integers(1, 5001))
        k = int(rng.integers(1, 2001))
        T = [np.complex64, np.complex128, np.float64][int(rng.integers(0, 3))]
        nbuffers = int(rng.integers(1, 3))
        extra = int(rng.integers(0, 3))
        workspace = int(rng.integers(0, (1 << 20) + 1))
        column = N * np.dtype(T).itemsize
        budget = workspace + (nbuffers + extra) * column * int(rng.integers(1, 2001))
        target = [1, 1 << 10, 1 << 20, 2 * 1024 ** 3][int(rng.integers(0, 4))]
        w = p.choose_panel_width(N, k, T, device_budget=budget, nbuffers=nbuffers, extra_buffers=extra,
                                 workspace_bytes=workspace, target_panel_bytes=target)
        per_buffer = (budget - workspace) // (nbuffers + extra)
        uncapped = min(k, per_buffer // column)
        capped = min(k, max(1, min(target, per_buffer) // column))
        assert 1 <= w <= uncapped
        assert p.device_bytes_required(N, w, T, nbuffers, extra, workspace) <= budget
        assert -(-k // w) == -(-k // capped)
        assert w == 1 or p.panel_bytes(N, w, T) <= max(target, column)


def test_plan_width_resolution(fb, plan_mod):
    p = plan_mod
    plan = make_plan(fb, device_budget=2 * 64 * 100 * 16)
    assert p.resolve_panel_width(plan, 100, 256, C128) == 64
    assert p.resolve_panel_width(plan, 100, 256, C128, override=17) == 17
    assert p.resolve_panel_width(plan, 100, 256, C128, extra_buffers=2) == 32
    for o in (0, 257, 128):
        with pytest.raises(fb.ArgumentError):
            p.resolve_panel_width(plan, 100, 256, C128, override=o)
    fixed = make_plan(fb, device_budget=1 << 30, panel_width=13)
    assert p.resolve_panel_width(fixed, 100, 256, C128) == 13
    assert p.resolve_panel_width(fixed, 100, 256, C128, override=8) == 8
    with pytest.raises(fb.ArgumentError) as err:
        p.resolve_panel_width(plan, 100, 256, C128, override=128)
    assert "device_budget" in str(err.value) and "panel_width <= 64" in str(err.value)


def test_row_block_height(fb):
    # h = clamp(fld(N w, k), 1, N) (src/plan.jl:133)
    assert fb.row_block_height(10 ** 7, 64, 16) == 2_500_000
    assert fb.row_block_height(2 ** 20, 32, 8) == 262_144
    assert fb.row_block_height(5, 100, 1) == 1
    assert fb.row_block_height(40, 23, 23) == 40


def test_device_pool(fb, plan_mod):
    p = plan_mod
    plan = make_plan(fb, device_budget=5 * 64 * 16 + 64)
    buffers = p.checkout_device_buffers(plan, C128, (64, 1), 2)
    assert len(buffers) == 2 and buffers[0] is not buffers[1]
    assert p.device_bytes_allocated(plan) == 2 * 64 * 16
    p.checkin_device_buffers(plan, buffers)
    again = p.checkout_device_buffers(plan, C128, (64, 1), 2)
    assert {id(b) for b in again} == {id(b) for b in buffers}
    assert p.device_bytes_allocated(plan) == 2 * 64 * 16
    nested = p.checkout_device_buffers(plan, C128, (64, 1), 3)
    assert not ({id(b) for b in nested} & {id(b) for b in again})
    assert p.device_bytes_allocated(plan) == 5 * 64 * 16
    with pytest.raises(fb.ArgumentError):
        p.checkout_device_buffers(plan, C128, (64, 1), 1)
    # Storage eltypes come from the staging pool, the compute one must be supported.
    narrow = p.checkout_staging_storage(plan, np.complex64, (4, 1), 1)
    assert narrow[0].dtype == np.complex64
    with pytest.raises(fb.ArgumentError):
        p.checkout_device_buffers(plan, np.complex64, (4, 1), 1)


def test_device_bytes_to_add_counts_buffers_the_pool_holds(fb, plan_mod):
    """A residency check asks what a call would add to the pool: buffers of
    the right dims given back by an earlier call are reused, not counted
    again (otherwise a second call of the same shape would take a slower
    schedule than the first)."""
    p = plan_mod
    plan = make_plan(fb, device_budget=10 * 64 * 16)
    assert p.device_bytes_to_add(plan, C128, [((64, 1), 2), ((4, 4), 1)]) == 2 * 64 * 16 + 16 * 16
    held = p.checkout_device_buffers(plan, C128, (64, 1), 2)
    p.checkin_device_buffers(plan, held)
    assert p.device_bytes_to_add(plan, C128, [((64, 1), 2), ((4, 4), 1)]) == 16 * 16
    assert p.device_bytes_to_add(plan, C128, [((64, 1), 3)]) == 64 * 16


def test_host_pool(fb, plan_mod):
    p = plan_mod
    plan = make_plan(fb, host_budget=4 * 2 ** 20)
    pool = plan.hostpool
    blocks = [p.alloc_host_storage(plan, C128, (2 ** 16, 1)) for _ in range(4)]
    assert all(s.array.shape == (2 ** 16, 1) for s in blocks)
    assert fb.host_bytes_reserved(pool) == pool.budget
    assert fb.host_bytes_in_use(pool) == 4 * 2 ** 20
    assert fb.host_bytes_free(pool) == 0
    with pytest.raises(fb.ArgumentError):
        p.alloc_host_storage(plan, C128, (2 ** 16, 1))
    p.release_host_block(plan, blocks[1].block)
    assert fb.host_bytes_free(pool) == 2 ** 20
    assert fb.host_bytes_in_use(pool) == 3 * 2 ** 20
    reused = p.alloc_host_storage(plan, C128, (2 ** 16, 1))
    assert reused.block is blocks[1].block
    assert fb.host_bytes_free(pool) == 0
    blocks[2].array[...] = 1
    blocks[3].array[...] = 2
    assert blocks[2].block.slab == blocks[3].block.slab
    assert np.all(blocks[2].array == 1)


def test_host_pool_grows_in_slabs(fb, plan_mod):
    p = plan_mod
    plan = make_plan(fb, host_budget=8 * 2 ** 20)
    pool = plan.hostpool
    assert fb.host_bytes_reserved(pool) == 0
    p.alloc_host_storage(plan, C128, (2 ** 16, 1))
    assert fb.host_bytes_reserved(pool) == 2 ** 20
    for _ in range(7):
        p.alloc_host_storage(plan, C128, (2 ** 16, 1))
    assert fb.host_bytes_reserved(pool) == 8 * 2 ** 20
    assert len(pool.slabs) == 4


def test_panel_matrix_layout_without_a_device(fb):
    # PanelMatrix construction and host round trips touch only the host pool.
    plan = make_plan(fb)
    rng = np.random.default_rng(1)
    A = np.asfortranarray(rng.random((40, 23)) + 1j * rng.random((40, 23)))
    for w in (23, 12, 7, 1):
        X = fb.PanelMatrix.from_array(A, plan=plan, w=w)
        assert X.npanels() == -(-23 // w)
        assert X.panels[-1].width == 23 - (X.npanels() - 1) * w
        assert np.array_equal(X.to_array(), A)
    with pytest.raises(fb.ArgumentError):
        fb.PanelMatrix.undef(C128, 0, 3, plan=plan)
    with pytest.raises(fb.ArgumentError):
        fb.PanelMatrix.undef(C128, 3, 0, plan=plan)


def test_narrowed_host_storage_without_a_device(fb):
    plan = make_plan(fb, host_eltype=np.complex64)
    A = np.asfortranarray(np.arange(12.0).reshape(4, 3) * (1 + 1j) / 3)
    X = fb.PanelMatrix.from_array(A, plan=plan, w=2)
    assert X.dtype == np.complex128
    assert X.panels[0].storage().dtype == np.complex64
    assert np.array_equal(X.to_array(), A.astype(np.complex64).astype(np.complex128))
    # The streamed cholqr2 takes a later pass's Gram inside the previous solve
    # sweep only where the panels store the solved values unrounded.
    assert not fb.panelblas.solves_what_it_stores(X)
    assert fb.panelblas.solves_what_it_stores(fb.PanelMatrix.from_array(A, plan=make_plan(fb), w=2))
    real_plan = make_plan(fb, host_eltype=np.float32)
    with pytest.raises(fb.ArgumentError):
        fb.PanelMatrix.undef(C128, 4, 3, plan=real_plan)


def test_ghost_construction_is_validated(fb):
    plan = make_plan(fb)
    with pytest.raises(fb.ArgumentError):
        fb.GhostPanels(C128, 0, 3, plan=plan)
    with pytest.raises(fb.ArgumentError):
        fb.GhostPanels(C128, 3, 0, plan=plan)
    G = fb.GhostPanels(C128, 24, 8, plan=plan, seed=0xdeadbeef, w=3)
    assert G.is_ghost() and G.npanels() == 3 and G.shape == (24, 8)
    with pytest.raises(fb.ArgumentError):
        G.assert_writable()
