"""The autotuner: tile shapes and forms chosen per (N, k, dtype) by timing
candidates on the device. No counterpart in the reference.

Two choices are tuned per shape class (floor(log2 N), k), and one per batch;
the compute dtype is always ComplexF64, the storage dtype does not change the
kernels:

- the Gram's row-chunk count (its tile shape along the rows), a shift of the
  built-in one-wave count held in the library's own table
  (fb_tune_set_gram_chunks), which every Gram launch of that class reads:
  the FP64 Gram of gram_accumulate!, of both cholqr2! forms' FP64 passes, of
  the batch and of the pullbacks;
- the form of the device-resident cholqr2! ("fp64" or "tc", k <= 64), read
  by kernels.cholqr2_resident(form="auto");
- the number of stream lanes a batch of cholqr2! instances is spread over
  (fb_tune_set_batch_lanes), timed on the caller's own batch.

Candidates are timed on the host clock around a synchronized run of several
launches, on scratch matrices filled by the ghost generator, so tuning
allocates and synchronizes: do it before a sweep, not inside one. A shape's
results are reproducible to the bit for a fixed table; changing the Gram's
entry changes its reduction order. `save`/`load` keep a table across
processes as JSON.
"""
from __future__ import annotations

import ctypes
import json
import time

import numpy as np

from . import _lib, kernels
from ._lib import ArgumentError, call

GRAM_SHIFTS = (-1, 0, 1, 2, 3)
_forms: dict[tuple[int, int], str] = {}
_records: dict[tuple[int, int], dict] = {}


def shape_class(N: int) -> int:
    """floor(log2 N), the library's class of a row count."""
    if N < 1:
        raise ArgumentError(f"N must be positive, got {N}")
    return int(N).bit_length() - 1


def gram_shift(N: int, k: int) -> int:
    out = ctypes.c_int(0)
    call("fb_tune_get_gram_chunks", ctypes.c_int64(N), int(k), ctypes.byref(out))
    return out.value


def set_gram_shift(N: int, k: int, shift: int) -> None:
    call("fb_tune_set_gram_chunks", ctypes.c_int64(N), int(k), int(shift))


def form_for(N: int, k: int) -> str:
    """The tuned cholqr2! form of this shape, "fp64" when untuned."""
    return _forms.get((shape_class(N), int(k)), "fp64")


BATCH_LANES = (1, 2, 4, 8, 12, 16)
_lanes_record: dict = {}


def batch_lanes() -> int:
    out = ctypes.c_int(0)
    call("fb_tune_get_batch_lanes", ctypes.byref(out))
    return out.value


def set_batch_lanes(lanes: int) -> None:
    call("fb_tune_set_batch_lanes", int(lanes))


def clear() -> None:
    """Forgets every tuned choice: Gram shifts, forms, and the batch lanes (back to 8)."""
    call("fb_tune_clear")
    set_batch_lanes(8)
    _forms.clear()
    _records.clear()
    _lanes_record.clear()


def _time(backend, fn, reps: int) -> float:
    fn()
    backend.sync_all()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    backend.sync_all()
    return 1e3 * (time.perf_counter() - t0) / reps


def tune(backend, N: int, k: int, *, forms: bool = True, reps: int | None = None, seed: int = 0x70E) -> dict:
    """Tunes the shape class of (N, k) on the device and records the choices.
    Returns the record: the chosen shift and form and every candidate's time
    in ms per call."""
    N, k = int(N), int(k)
    if N < 1 or k < 1:
        raise ArgumentError(f"cannot tune an {N}x{k} shape")
    if reps is None:
        reps = max(3, min(50, int(2e8 // max(N * k * k, 1))))
    Y = backend.alloc_device(np.complex128, (N, k))
    G = backend.alloc_device(np.complex128, (k, k))
    kernels.ghost_fill(backend, Y, 0, 0, seed, np.complex128)
    gram_ms = {}
    for s in GRAM_SHIFTS:
        set_gram_shift(N, k, s)
        gram_ms[s] = _time(backend, lambda: kernels.gram_accumulate(backend, G, Y, Y, 1.0, 0.0), reps)
    # The fastest, and the built-in count unless another is clearly faster.
    best = min(gram_ms, key=gram_ms.get)
    if gram_ms[best] > 0.97 * gram_ms[0]:
        best = 0
    set_gram_shift(N, k, best)
    record = {"N": N, "k": k, "class": shape_class(N), "gram_shift": best,
              "gram_ms": {str(s): v for s, v in gram_ms.items()}}
    if forms and k <= 64:
        R = backend.alloc_device(np.complex128, (k, k))
        form_ms = {}
        for form in ("fp64", "tc"):
            kernels.ghost_fill(backend, Y, 0, 0, seed, np.complex128)
            form_ms[form] = _time(backend, lambda: kernels.cholqr2_resident(backend, Y, R, wait=False, form=form),
                                  max(3, reps // 4))
        choice = "tc" if form_ms["tc"] < 0.97 * form_ms["fp64"] else "fp64"
        _forms[(shape_class(N), k)] = choice
        record.update(form=choice, cholqr2_ms=form_ms)
    _records[(shape_class(N), k)] = record
    return record


def tune_shapes(backend, shapes, **kw) -> list[dict]:
    """Tunes every shape class among (N, k) pairs, each at its largest N."""
    largest: dict[tuple[int, int], int] = {}
    for N, k in shapes:
        key = (shape_class(int(N)), int(k))
        largest[key] = max(largest.get(key, 0), int(N))
    return [tune(backend, N, k, **kw) for (_, k), N in sorted(largest.items())]


def tune_batch_lanes(backend, Ys, Rs, *, reps: int = 3) -> dict:
    """Times the batch (Ys[i] -> Q, Rs[i]; the matrices are overwritten) at
    each lane count and keeps the fastest. Returns the record."""
    ms = {}
    for lanes in BATCH_LANES:
        set_batch_lanes(lanes)
        ms[lanes] = _time(backend, lambda: kernels.cholqr2_batched(backend, Ys, Rs, wait=False, schedule="lanes"), reps)
    best = min(ms, key=ms.get)
    if ms[best] > 0.97 * ms[8]:
        best = 8
    set_batch_lanes(best)
    _lanes_record.clear()
    _lanes_record.update(lanes=best, ms={str(l): v for l, v in ms.items()}, instances=len(Ys))
    return dict(_lanes_record)


def records() -> list[dict]:
    return [dict(r) for _, r in sorted(_records.items())]


def save(path: str) -> None:
    with open(path, "w") as f:
        json.dump({"version": 1, "records": records(), "batch": dict(_lanes_record)}, f, indent=1)


def load(path: str) -> None:
    """Applies a saved table: Gram shifts into the library, forms here."""
    with open(path) as f:
        data = json.load(f)
    if data.get("version") != 1:
        raise ArgumentError(f"{path} is not an autotuning table of this version")
    for r in data["records"]:
        N, k = int(r["N"]), int(r["k"])
        set_gram_shift(N, k, int(r["gram_shift"]))
        if "form" in r:
            if r["form"] not in ("fp64", "tc"):
                raise ArgumentError(f"unknown form {r['form']!r} in {path}")
            _forms[(shape_class(N), k)] = r["form"]
        _records[(shape_class(N), k)] = dict(r)
    if data.get("batch"):
        set_batch_lanes(int(data["batch"]["lanes"]))
        _lanes_record.update(data["batch"])
