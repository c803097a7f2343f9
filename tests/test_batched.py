"""Batched cholqr2! on stream lanes (fb_zcholqr2_batched): many independent
instances of uneven N and k in one enqueued sequence, each bitwise equal to
its own fb_zcholqr2 call, and the whole batch replayed as one captured
graph."""
import ctypes

import numpy as np
import pytest

from conftest import conditioned, randmatrix

pytestmark = pytest.mark.gpu

SHAPES = [(1000, 16), (5000, 32), (20000, 64), (77, 7), (16, 16), (123457, 64), (40000, 23), (3000, 1)]


def instances(rng):
    return [randmatrix(rng, N, k) for N, k in SHAPES]


@pytest.mark.parametrize("form", ["fp64", "tc"])
def test_batch_equals_one_call_per_instance(fb, backend, oracle, form):
    rng = np.random.default_rng(5)
    As = instances(rng)
    Ys = [backend.todevice(A) for A in As]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in As]
    passes = fb.kernels.cholqr2_batched(backend, Ys, Rs, form=form, schedule="lanes")
    assert passes == [2] * len(As)
    for A, Y, R in zip(As, Ys, Rs):
        Y1 = backend.todevice(A)
        R1 = backend.alloc_device(np.complex128, R.shape)
        fb.kernels.cholqr2_resident(backend, Y1, R1, form=form)
        assert Y.to_host().tobytes() == Y1.to_host().tobytes()
        assert R.to_host().tobytes() == R1.to_host().tobytes()
        Q = Y.to_host()
        assert oracle.orthogonality_error(Q) <= 1e-12
        assert oracle.reconstruction_error(A, Q, R.to_host()) <= 1e-13


def test_batch_reports_each_instance(fb, backend):
    rng = np.random.default_rng(6)
    As = [randmatrix(rng, 3000, 16), conditioned(rng, 3000, 16, 1e10), randmatrix(rng, 500, 8)]
    Ys = [backend.todevice(A) for A in As]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in As]
    assert fb.kernels.cholqr2_batched(backend, Ys, Rs, schedule="lanes") == [2, 3, 2]
    # An indefinite instance (a column of NaN) stops its own chain only.
    bad = randmatrix(rng, 400, 4)
    bad[:, 2] = np.nan
    As2 = [randmatrix(rng, 600, 4), bad]
    Ys2 = [backend.todevice(A) for A in As2]
    Rs2 = [backend.alloc_device(np.complex128, (4, 4)) for _ in As2]
    with pytest.raises(fb.NotPositiveDefinite, match="instance 1"):
        fb.kernels.cholqr2_batched(backend, Ys2, Rs2, schedule="lanes")
    Q0 = Ys2[0].to_host()
    assert np.linalg.norm(Q0.conj().T @ Q0 - np.eye(4)) <= 1e-12


@pytest.mark.parametrize("form", ["fp64", "tc"])
def test_a_captured_batch_replays_as_one_graph(fb, backend, form):
    rng = np.random.default_rng(7)
    As = instances(rng)
    Ys = [backend.todevice(A) for A in As]
    Rs = [backend.alloc_device(np.complex128, (A.shape[1],) * 2) for A in As]
    eager_Y = [backend.todevice(A) for A in As]
    eager_R = [backend.alloc_device(np.complex128, R.shape) for R in Rs]
    fb.kernels.cholqr2_batched(backend, eager_Y, eager_R, form=form, schedule="lanes")
    nbytes = fb.kernels.cholqr2_batched_workspace_bytes([A.shape for A in As], form, "lanes")
    ws = backend.alloc_device(np.complex128, (nbytes // 16 + 16, 1))
    aligned = (ws.ptr + 255) // 256 * 256
    q = backend.make_queue()
    graph = backend.capture(q, lambda: fb.kernels.cholqr2_batched(
        backend, Ys, Rs, form=form, wait=False, workspace=(aligned, nbytes), schedule="lanes"))
    for _ in range(2):
        for A, Y in zip(As, Ys):
            backend.h2d(Y, A)
        graph.launch(q)
        backend.sync_queue(q)
        for Y, R, Ye, Re in zip(Ys, Rs, eager_Y, eager_R):
            assert Y.to_host().tobytes() == Ye.to_host().tobytes()
            assert R.to_host().tobytes() == Re.to_host().tobytes()
