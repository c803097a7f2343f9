"""The C ABI: the library loads on a machine without a GPU, exports every
function its header declares, and turns bad arguments into the statuses the
reference's exceptions map onto, before touching the device."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "funicular_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fb_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_device_api_and_kernels():
    names = declared_functions()
    for required in ("fb_alloc_device", "fb_alloc_host_slab", "fb_queue_create", "fb_event_record",
                     "fb_queue_wait_event", "fb_queue_sync", "fb_event_sync", "fb_sync_all", "fb_copy2d",
                     "fb_convert_copy", "fb_zgram", "fb_ztrsm_right_upper", "fb_zgemm_right",
                     "fb_zpotrf_shifted", "fb_zcholqr2"):
        assert required in names


def test_library_exports_every_declared_symbol(fb):
    lib = fb._lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), f"{name} is declared in the header but not exported"
        assert name in fb._lib.SIGNATURES, f"{name} has no ctypes signature"


def test_binding_declares_nothing_the_header_lacks(fb):
    assert set(fb._lib.SIGNATURES) <= set(declared_functions())


def test_abi_version(fb):
    assert fb._lib.load().fb_abi_version() == 1


def test_device_count_without_a_gpu_is_not_an_error(fb):
    assert fb._lib.device_count() >= 0


def test_shape_errors_map_to_dimension_mismatch(fb):
    lib = fb._lib.load()
    z = fb._lib.z128(1.0)
    status = lib.fb_zgram(None, 1, None, 1, None, 1, -1, 2, 2, z, z, None, 0, None)
    assert status == fb._lib.FB_EDIM
    assert "negative" in fb._lib.last_error()
    with pytest.raises(fb.DimensionMismatch):
        fb._lib.check(status)
    assert lib.fb_ztrsm_right_upper(None, 1, -3, 2, None, 1, None, 0, None) == fb._lib.FB_EDIM
    assert lib.fb_zgemm_right(None, 1, None, 1, 4, -1, None, 1, 2, None) == fb._lib.FB_EDIM


def test_leading_dimension_is_checked(fb):
    lib = fb._lib.load()
    z = fb._lib.z128(1.0)
    fake = ctypes.c_void_p(1 << 20)
    status = lib.fb_zgram(fake, 4, fake, 3, fake, 8, 8, 4, 4, z, z, fake, 1 << 20, None)
    assert status == fb._lib.FB_EDIM
    assert "leading dimension" in fb._lib.last_error()


def test_empty_work_is_a_no_op(fb):
    lib = fb._lib.load()
    z = fb._lib.z128(1.0)
    assert lib.fb_zgram(None, 1, None, 1, None, 1, 10, 0, 3, z, z, None, 0, None) == fb._lib.FB_OK
    assert lib.fb_ztrsm_right_upper(None, 1, 0, 3, None, 1, None, 0, None) == fb._lib.FB_OK
    assert lib.fb_copy2d(None, 16, None, 16, 0, 4, None) == fb._lib.FB_OK


def test_workspace_queries(fb):
    lib = fb._lib.load()
    n = ctypes.c_size_t(0)
    assert lib.fb_zpotrf_workspace_size(64, ctypes.byref(n)) == fb._lib.FB_OK and n.value > 0
    assert lib.fb_zgram_workspace_size(100, 4, 5, 1, ctypes.byref(n)) == fb._lib.FB_EDIM
    assert lib.fb_zcholqr2_workspace_size(-1, 4, ctypes.byref(n)) == fb._lib.FB_EINVAL


def test_bad_eltype_and_complex_to_real_are_refused(fb):
    lib = fb._lib.load()
    fake = ctypes.c_void_p(1 << 20)
    assert lib.fb_convert_copy(fake, 9, 4, fake, 0, 4, 4, 4, None) == fb._lib.FB_EINVAL
    assert lib.fb_convert_copy(fake, fb._lib.FB_F64, 4, fake, fb._lib.FB_C128, 4, 4, 4, None) == fb._lib.FB_EINVAL
    assert "complex" in fb._lib.last_error()


def test_cholqr2_rejects_empty_and_misaligned(fb):
    lib = fb._lib.load()
    assert lib.fb_zcholqr2(None, 1, 0, 4, None, 4, None, None, None, 0, None) == fb._lib.FB_EINVAL
    odd = ctypes.c_void_p((1 << 20) + 8)
    assert lib.fb_zcholqr2(odd, 8, 8, 4, odd, 4, None, None, None, 0, None) == fb._lib.FB_EINVAL
    assert "aligned" in fb._lib.last_error()


def test_errors_are_per_thread(fb):
    import threading
    lib = fb._lib.load()
    lib.fb_ztrsm_right_upper(None, 1, -3, 2, None, 1, None, 0, None)
    seen = []
    t = threading.Thread(target=lambda: seen.append(fb._lib.last_error()))
    t.start()
    t.join()
    assert seen == [""]
    assert fb._lib.last_error() != ""


def test_tuning_table_is_host_state(fb, tmp_path):
    # The autotuner's table lives in the library's host memory: it can be set,
    # read, saved, loaded and cleared without a GPU.
    fb.autotune.clear()
    assert fb.autotune.gram_shift(10_000, 16) == 0
    fb.autotune.set_gram_shift(10_000, 16, 2)
    assert fb.autotune.gram_shift(16_383, 16) == 2      # same class: floor(log2 N) = 13
    assert fb.autotune.gram_shift(16_384, 16) == 0      # next class
    assert fb.autotune.gram_shift(10_000, 32) == 0
    fb.autotune._records[(13, 16)] = {"N": 10_000, "k": 16, "class": 13, "gram_shift": 2, "form": "tc"}
    fb.autotune._forms[(13, 16)] = "tc"
    path = tmp_path / "tune.json"
    fb.autotune.save(str(path))
    fb.autotune.clear()
    assert fb.autotune.gram_shift(10_000, 16) == 0 and fb.autotune.form_for(10_000, 16) == "fp64"
    fb.autotune.load(str(path))
    assert fb.autotune.gram_shift(10_000, 16) == 2 and fb.autotune.form_for(10_000, 16) == "tc"
    with pytest.raises(fb.ArgumentError):
        fb.autotune.set_gram_shift(10_000, 16, 9)
    fb.autotune.clear()


def test_newer_entry_points_check_arguments_without_a_gpu(fb):
    # Every check below fires before anything reaches a device: the pointers
    # are fake (aligned, distinct), never dereferenced.
    lib = fb._lib.load()
    E = fb._lib
    a, b, c, d = 0x10000000, 0x20000000, 0x30000000, 0x40000000
    n = ctypes.c_size_t(0)
    # The cholqr2! pullback.
    assert lib.fb_zcholqr2_adjoint_workspace_size(-1, 4, ctypes.byref(n)) == E.FB_EINVAL
    assert lib.fb_zcholqr2_adjoint(None, 8, b, 8, c, 4, None, 0, None, 0, 8, 4, None, 0, None) == E.FB_EINVAL
    assert lib.fb_zcholqr2_adjoint(a, 8, b, 8, c, 4, None, 0, None, 0, -1, 4, None, 0, None) == E.FB_EDIM
    assert lib.fb_zcholqr2_adjoint(a, 7, b, 8, c, 4, None, 0, None, 0, 8, 4, None, 0, None) == E.FB_EDIM
    assert lib.fb_zcholqr2_adjoint(a + 8, 8, b, 8, c, 4, None, 0, None, 0, 8, 4, None, 0, None) == E.FB_EINVAL
    assert lib.fb_zcholqr2_adjoint(a, 8, a + 16 * 8, 8, c, 4, None, 0, None, 0, 8, 4, None, 0, None) == E.FB_EINVAL
    assert "overlaps" in E.last_error()
    assert lib.fb_zcholqr2_adjoint(a, 8, b, 8, c, 4, d, 8, None, 0, 8, 4, None, 0, None) == E.FB_ENOMEM
    # The project pullback.
    assert lib.fb_zproject_adjoint(None, 8, b, 8, None, 0, c, 4, 8, 4, 0, None, 0, None) == E.FB_EINVAL
    assert lib.fb_zproject_adjoint(a, 8, b, 8, None, 0, c, 4, -8, 4, 0, None, 0, None) == E.FB_EDIM
    assert lib.fb_zproject_adjoint(a, 8, a, 8, None, 0, c, 4, 8, 4, 0, None, 0, None) == E.FB_EINVAL
    # The band operator.
    assert lib.fb_zhband_apply(a, 8, b, 8, c, 8, -1, 2, 4, None) == E.FB_EINVAL
    assert lib.fb_zhband_apply(a, 7, b, 8, c, 8, 8, 2, 4, None) == E.FB_EDIM
    assert lib.fb_zhband_apply(a + 8, 8, b, 8, c, 8, 8, 2, 4, None) == E.FB_EINVAL
    assert lib.fb_zhband_apply(a, 8, a + 16, 8, c, 8, 8, 2, 4, None) == E.FB_EINVAL
    # The shifted CholeskyQR3 and its forced-shift factorization.
    for u in (0.0, 1.5, float("nan")):
        assert lib.fb_zcholqr3_shifted(a, 8, 8, 4, c, 4, u, None, None, None, 0, None) == E.FB_EINVAL
        assert lib.fb_zpotrf_forced_shift(a, 4, b, 4, 4, 8, None, 4, None, 4, u, None, None, 0, None) == E.FB_EINVAL
    # The batch.
    assert lib.fb_zcholqr2_batched(None, None, None, None, None, None, 0, 0, None, 0, None) == E.FB_OK
    assert lib.fb_zcholqr2_batched(None, None, None, None, None, None, 2, 0, None, 0, None) == E.FB_EINVAL
    Ns = (ctypes.c_int64 * 2)(100, 0)
    ks = (ctypes.c_int * 2)(4, 4)
    assert lib.fb_zcholqr2_batched_workspace_size(ctypes.cast(Ns, ctypes.c_void_p), ctypes.cast(ks, ctypes.c_void_p),
                                                   2, ctypes.byref(n)) == E.FB_EINVAL
    assert "instance 1" in E.last_error()
    # The persistent batch: the same argument checks, and k past 64 refused.
    assert lib.fb_zcholqr2_batched_persistent(None, None, None, None, None, None, 0, None, 0, None) == E.FB_OK
    assert lib.fb_zcholqr2_batched_persistent(None, None, None, None, None, None, 2, None, 0, None) == E.FB_EINVAL
    cast = lambda x: ctypes.cast(x, ctypes.c_void_p)
    assert lib.fb_zcholqr2_batched_persistent_workspace_size(cast(Ns), cast(ks), 2, ctypes.byref(n)) == E.FB_EINVAL
    Ns2 = (ctypes.c_int64 * 2)(100, 5000)
    ks2 = (ctypes.c_int * 2)(64, 65)
    assert lib.fb_zcholqr2_batched_persistent_workspace_size(cast(Ns2), cast(ks2), 2, ctypes.byref(n)) == E.FB_ENOTSUP
    assert "instance 1" in E.last_error()
    assert lib.fb_zcholqr2_batched_persistent_workspace_size(cast(Ns2), cast(ks2), 1, ctypes.byref(n)) == E.FB_OK
    assert n.value > 0
    # The tuning table.
    assert lib.fb_tune_set_batch_lanes(0) == E.FB_EINVAL
    assert lib.fb_tune_set_batch_lanes(17) == E.FB_EINVAL
    assert lib.fb_tune_set_gram_chunks(100, 4, 9) == E.FB_EINVAL
    assert lib.fb_tune_set_gram_chunks(0, 4, 1) == E.FB_EINVAL


def test_static_gram_scratch_holds_every_gram_of_at_most_128_columns(fb):
    """fb_zgram_static keeps its partial tiles in a 32 MiB array. A partial
    tile takes tw_a x tw_b entries, so narrow panels over many rows (many row
    chunks, few entries each) stay small; the documented bound is that every
    Gram of at most 128 columns a side fits on a 148-SM B200 (the SM count the
    library assumes without a device)."""
    if fb._lib.device_count() > 0:
        pytest.skip("the bound is stated for the 148 SMs the library assumes without a device")
    need = ctypes.c_size_t(0)
    worst = 0
    for rows in (1000, 16_384, 200_003, 1_000_000, 10_000_000, 40_001_688, 1 << 30):
        for kA in range(1, 129):
            for kB in sorted({kA, 1, 8, 16, 64, 128}):
                for herm in ((0, 1) if kA == kB else (0,)):
                    fb._lib.call("fb_zgram_workspace_size", ctypes.c_int64(rows), kA, kB, herm,
                                 ctypes.byref(need))
                    worst = max(worst, need.value)
    assert worst <= 32 << 20
