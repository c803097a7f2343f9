"""The autotuner (funicular_b200.autotune) and the library's tuning table:
every Gram chunk shift it may choose gives a correct Gram, the bits are
reproducible for a fixed table, the workspace size follows the table, and
tuned shapes keep the accuracy targets."""
import ctypes

import numpy as np
import pytest

from conftest import randmatrix

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def clean_table(fb):
    fb.autotune.clear()
    yield
    fb.autotune.clear()


def ws_size(fb, N, k):
    need = ctypes.c_size_t(0)
    fb._lib.call("fb_zgram_workspace_size", ctypes.c_int64(N), k, k, 1, ctypes.byref(need))
    return need.value


@pytest.mark.parametrize("N,k", [(100_000, 64), (12_345, 16), (300_000, 128)])
def test_every_chunk_shift_gives_the_gram(fb, backend, oracle, N, k):
    rng = np.random.default_rng(N + k)
    A = randmatrix(rng, N, k)
    Ad = backend.todevice(A)
    ref = oracle.gram(A)
    tol = oracle.blastol(np.complex128, N, k)
    sizes = set()
    for s in fb.autotune.GRAM_SHIFTS:
        fb.autotune.set_gram_shift(N, k, s)
        sizes.add(ws_size(fb, N, k))
        C1 = backend.alloc_device(np.complex128, (k, k))
        C2 = backend.alloc_device(np.complex128, (k, k))
        fb.kernels.gram_accumulate(backend, C1, Ad, Ad, 1.0, 0.0)
        fb.kernels.gram_accumulate(backend, C2, Ad, Ad, 1.0, 0.0)
        backend.sync_all()
        G1, G2 = C1.to_host(), C2.to_host()
        assert G1.tobytes() == G2.tobytes()
        np.testing.assert_allclose(G1, ref, rtol=tol, atol=tol * np.abs(ref).max())
    assert len(sizes) > 1  # the chunk count, and so the scratch, follows the table


def test_tune_records_a_choice_and_keeps_the_targets(fb, backend, oracle):
    N, k = 40_000, 32
    rec = fb.autotune.tune(backend, N, k)
    assert rec["gram_shift"] in fb.autotune.GRAM_SHIFTS
    assert fb.autotune.gram_shift(N, k) == rec["gram_shift"]
    assert rec["form"] in ("fp64", "tc") and fb.autotune.form_for(N, k) == rec["form"]
    assert set(rec["gram_ms"]) == {str(s) for s in fb.autotune.GRAM_SHIFTS}
    rng = np.random.default_rng(4)
    A = randmatrix(rng, N, k)
    Y = backend.todevice(A)
    R = backend.alloc_device(np.complex128, (k, k))
    passes, _ = fb.kernels.cholqr2_resident(backend, Y, R, form="auto")
    assert passes == 2
    Q = Y.to_host()
    assert oracle.orthogonality_error(Q) <= 1e-12
    assert oracle.reconstruction_error(A, Q, R.to_host()) <= 1e-13


def test_tune_shapes_covers_each_class_once(fb, backend):
    recs = fb.autotune.tune_shapes(backend, [(10_000, 16), (12_000, 16), (20_000, 16), (10_000, 32)], forms=False)
    assert sorted((r["class"], r["k"]) for r in recs) == [(13, 16), (13, 32), (14, 16)]
    assert [r["N"] for r in recs if (r["class"], r["k"]) == (13, 16)] == [12_000]


def test_batch_lanes_are_tunable_and_keep_the_bits(fb, backend):
    rng = np.random.default_rng(9)
    shapes = [(20_000, 16), (5_000, 32), (60_000, 64), (9_000, 8), (30_000, 24)]
    mats = [randmatrix(rng, N, k) for N, k in shapes]
    outs = {}
    for lanes in (1, 3, 16):
        fb.autotune.set_batch_lanes(lanes)
        assert fb.autotune.batch_lanes() == lanes
        Ys = [backend.todevice(A) for A in mats]
        Rs = [backend.alloc_device(np.complex128, (k, k)) for _, k in shapes]
        passes = fb.kernels.cholqr2_batched(backend, Ys, Rs, schedule="lanes")
        assert passes == [2] * len(shapes)
        outs[lanes] = b"".join(Y.to_host().tobytes() + R.to_host().tobytes() for Y, R in zip(Ys, Rs))
    assert outs[1] == outs[3] == outs[16]
    rec = fb.autotune.tune_batch_lanes(backend, Ys, Rs)
    assert rec["lanes"] in fb.autotune.BATCH_LANES and fb.autotune.batch_lanes() == rec["lanes"]
    with pytest.raises(fb.ArgumentError):
        fb.autotune.set_batch_lanes(17)
