"""The ghost generator's C restatement on its own: Philox4x32-10 against the
published known-answer vectors, the series ln / cos / sin against libm, and
the properties GhostPanels promises (test/test_ghosts.jl:1-28)."""
import numpy as np
import pytest

from oracle import ghost


def test_philox_known_answers():
    # Known-answer vectors published with Philox4x32-10 (Random123).
    assert ghost.philox4x32_10((0, 0, 0, 0), (0, 0)) == (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)
    assert ghost.philox4x32_10((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2) == (0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                         0x6D5451FD)
    assert ghost.philox4x32_10((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0)) == \
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)


def test_series_ln_is_within_two_ulps():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.random(20000), [1.0, 2.0 ** -53, 0.5, 0.7071067811865476, 1 - 2.0 ** -53, 3.5, 1e300]])
    got = np.array([ghost.ln(float(x)) for x in xs])
    ref = np.log(xs)
    ulps = np.abs(got - ref) / np.spacing(np.maximum(np.abs(ref), 1e-300))
    assert ghost.ln(1.0) == 0.0
    assert ulps.max() <= 2.0


def test_series_cos_sin_are_accurate():
    rng = np.random.default_rng(1)
    us = np.concatenate([rng.random(20000), np.arange(16) / 16, [1 - 2.0 ** -53]])
    got = np.array([ghost.cos_sin_2pi(float(u)) for u in us])
    assert np.abs(got[:, 0] - np.cos(2 * np.pi * us)).max() < 2e-15
    assert np.abs(got[:, 1] - np.sin(2 * np.pi * us)).max() < 2e-15


def test_ghost_entries_are_standard_normal():
    A = ghost.ghost_block(np.complex128, 4096, 8, 0, 0, 0xDEADBEEF)
    assert abs(A.real.mean()) < 0.03 and abs(A.imag.mean()) < 0.03
    assert abs(A.real.var() - 0.5) < 0.03 and abs(A.imag.var() - 0.5) < 0.03
    R = ghost.ghost_block(np.float64, 4096, 8, 0, 0, 0xDEADBEEF)
    assert abs(R.mean()) < 0.03 and abs(R.var() - 1.0) < 0.05
    assert np.linalg.matrix_rank(A[:24]) == 8


def test_ghost_blocks_are_cut_free():
    # One seed means one matrix, whatever rows and columns a block covers.
    whole = ghost.ghost_block(np.complex128, 40, 23, 0, 0, 7)
    assert np.array_equal(ghost.ghost_block(np.complex128, 13, 5, 11, 9, 7), whole[11:24, 9:14])
    assert not np.array_equal(ghost.ghost_block(np.complex128, 40, 23, 0, 0, 8), whole)
    # Rows past 2^32 and columns past 2^32 reach the high counter words.
    far = ghost.ghost_block(np.complex128, 2, 2, 2 ** 32 - 1, 2 ** 32 - 1, 7)
    assert np.all(np.isfinite(far)) and len(set(far.ravel().tolist())) == 4


def test_narrowed_values_are_single_precision_values():
    wide = ghost.ghost_block(np.complex128, 64, 3, 0, 0, 3)
    narrow = ghost.ghost_block(np.complex128, 64, 3, 0, 0, 3, value_dtype=np.complex64)
    assert np.array_equal(narrow, wide.astype(np.complex64).astype(np.complex128))
