"""Shared fixtures. Tests marked `gpu` need a B200 and the built library; the
rest run on any machine."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200) and the built library")


@pytest.fixture(scope="session")
def fb():
    """The package, imported as funicular_b200."""
    return __graft_entry__.load()


@pytest.fixture(scope="session")
def oracle():
    from oracle import panel_oracle
    return panel_oracle


@pytest.fixture(scope="session")
def backend(fb):
    if fb._lib.device_count() == 0:
        pytest.fail("a gpu test ran without a visible CUDA device")
    return fb.B200Backend(0)


def randmatrix(rng, N, k, dtype=np.complex128):
    """randmatrix (test/setup.jl:148-149): entries uniform on -1/2..1/2, real
    and imaginary parts alike."""
    if np.dtype(dtype).kind == "c":
        a = (rng.random((N, k)) - 0.5) + 1j * (rng.random((N, k)) - 0.5)
    else:
        a = rng.random((N, k)) - 0.5
    return np.asfortranarray(a.astype(dtype))


def conditioned(rng, N, k, kappa, dtype=np.complex128):
    """conditioned(T, N, k, kappa) (test/test_panelblas.jl:284): orthonormal
    left factor, log-spaced singular values from 1 to 1/kappa, unitary right
    factor."""
    U, _ = np.linalg.qr(randmatrix(rng, N, k, dtype))
    V, _ = np.linalg.qr(randmatrix(rng, k, k, dtype))
    s = 10.0 ** np.linspace(0, -np.log10(kappa), k)
    return np.asfortranarray((U * s) @ V.conj().T)
