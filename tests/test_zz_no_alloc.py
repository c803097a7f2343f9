"""fb_zgram_static, the Gram entry point that allocates nothing.

It exists for callers that have no device memory to hand over as a workspace
(a host whose allocator has promised every device byte to a budgeted pool, or
one that must not pay for cudaMalloc inside a pipelined sweep), so it keeps its
scratch in a fixed array inside the library. This test calls it through the C
ABI and checks it against fb_zgram, the workspace-taking entry point, bit for
bit, twice in a row, so that the second call also shows the shared scratch
carries nothing over from the first, and checks that repeated calls leave the
device's free memory unchanged. The file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from conftest import randmatrix

pytestmark = pytest.mark.gpu


def _vp(x):
    return ctypes.c_void_p(x)


def gram_static(fb, C, A, B, alpha, beta):
    lib = fb._lib.load()
    status = lib.fb_zgram_static(_vp(C.ptr), C.ld, _vp(A.ptr), A.ld, _vp(B.ptr), B.ld, A.rows, A.cols, B.cols,
                                 fb._lib.z128(alpha), fb._lib.z128(beta), None)
    fb._lib.check(status, "fb_zgram_static")


def gram_with_workspace(fb, backend, C, A, B, alpha, beta):
    lib = fb._lib.load()
    herm = 1 if A.same_view(B) else 0
    need = ctypes.c_size_t(0)
    fb._lib.call("fb_zgram_workspace_size", ctypes.c_int64(A.rows), A.cols, B.cols, herm, ctypes.byref(need))
    ws = backend.alloc_device(np.complex128, (max(need.value // 16 + 1, 1), 1))
    status = lib.fb_zgram(_vp(C.ptr), C.ld, _vp(A.ptr), A.ld, _vp(B.ptr), B.ld, A.rows, A.cols, B.cols,
                          fb._lib.z128(alpha), fb._lib.z128(beta), _vp(ws.ptr), need.value, None)
    fb._lib.check(status, "fb_zgram")
    fb._lib.call("fb_sync_all")


# Shapes: a folded 64-column Gram, a cross Gram of ragged widths, a 128-column
# Gram (three 64 x 64 tiles), and narrow panels over many rows, whose many
# row chunks each keep a partial tile of only 8 x 8 or 16 x 16 entries.
@pytest.mark.parametrize("rows,kA,kB,same", [(200_003, 64, 64, True), (4099, 23, 9, False), (50_000, 128, 128, True),
                                             (200_003, 8, 8, True), (1_000_000, 16, 16, True),
                                             (1_000_000, 8, 16, False)])
def test_static_scratch_matches_the_workspace_entry_point(fb, backend, rows, kA, kB, same):
    rng = np.random.default_rng(rows + kA)
    for call in range(2):
        A = randmatrix(rng, rows, kA)
        B = A if same else randmatrix(rng, rows, kB)
        Ad = backend.todevice(A)
        Bd = Ad if same else backend.todevice(B)
        expect = backend.todevice(np.zeros((kA, kB), dtype=np.complex128, order="F"))
        got = backend.todevice(np.full((kA, kB), np.nan + 0j, dtype=np.complex128, order="F"))
        gram_with_workspace(fb, backend, expect, Ad, Bd, 1.0, 0.0)
        gram_static(fb, got, Ad, Bd, 1.0, 0.0)
        fb._lib.call("fb_sync_all")
        # Same partial tiles, same reduction order: the same bits.
        np.testing.assert_array_equal(got.to_host(), expect.to_host())
        # beta = 1 accumulates onto what the first product left, as fb_zgram does.
        gram_with_workspace(fb, backend, expect, Ad, Bd, 0.5, 1.0)
        gram_static(fb, got, Ad, Bd, 0.5, 1.0)
        fb._lib.call("fb_sync_all")
        np.testing.assert_array_equal(got.to_host(), expect.to_host())


def test_static_scratch_call_allocates_no_device_memory(fb, backend):
    import torch

    rows, k = 300_000, 64
    rng = np.random.default_rng(7)
    Ad = backend.todevice(randmatrix(rng, rows, k))
    C = backend.alloc_device(np.complex128, (k, k))
    gram_static(fb, C, Ad, Ad, 1.0, 0.0)  # warm: the kernels are loaded by now
    fb._lib.call("fb_sync_all")
    free_before, _ = torch.cuda.mem_get_info(0)
    for _ in range(3):
        gram_static(fb, C, Ad, Ad, 1.0, 0.0)
    fb._lib.call("fb_sync_all")
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before


def test_static_scratch_refuses_shapes_that_do_not_fit(fb, backend):
    rows, k = 100_000, 448
    need = ctypes.c_size_t(0)
    fb._lib.call("fb_zgram_workspace_size", ctypes.c_int64(rows), k, k, 1, ctypes.byref(need))
    assert need.value > 32 << 20  # a Hermitian 448 x 448 Gram over 1e5 rows: 28 tiles x 21 chunks on a B200
    A = backend.alloc_device(np.complex128, (rows, k))
    C = backend.alloc_device(np.complex128, (k, k))
    lib = fb._lib.load()
    before = fb._lib.kernel_launches()
    status = lib.fb_zgram_static(_vp(C.ptr), C.ld, _vp(A.ptr), A.ld, _vp(A.ptr), A.ld, rows, k, k,
                                 fb._lib.z128(1.0), fb._lib.z128(0.0), None)
    assert status == fb._lib.FB_ENOMEM
    assert "33554432" in fb._lib.last_error()
    assert fb._lib.kernel_launches() == before
