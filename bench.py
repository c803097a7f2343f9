#!/usr/bin/env python
"""cholqr2! throughput on the B200 backend.

Workload (one step): cholqr2! of a device-resident ComplexF64 matrix with
N = 10^7 rows and k = 64 columns (panel width 16, so the reference's row
blocks are 2.5e6 rows), Y = U diag(s) V^H with U a seeded complex Gaussian made
orthonormal, V a seeded 64 x 64 Haar unitary and s log-spaced from 1 to 1e-6.
The metric is GB/s of algorithmic traffic, 96 N k bytes per cholqr2! (two
passes of Gram read + TRSM read + TRSM write), over the device time of the
step; the inputs (10.24 GB) are larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N under torchrun every rank runs its own replica (one matrix per
GPU, no collective on the data path) and `value` is the bytes of all ranks over
the slowest rank's time. --impl reference times the reference algorithm on the
host cores instead (the CPU oracle, since Funicular.jl is Julia and Julia is
not available here), on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cholqr2! GB/s & % roofline, tensor vs FP64 form at ||QᴴQ-I||<=1e-12"
UNIT = "GB/s"
N_DEFAULT, K_DEFAULT, W_PANEL = 10_000_000, 64, 16
CPU_SAMPLE_ROWS = 1 << 21

# DRAM bytes per row each kernel moved in its committed ncu capture (N = 5e5,
# k = 64, profiles/*_N5e5_k64_ncu.md), scaled here to the bench's N.
NCU_BYTES_PER_ROW = {"gram_partial+reduce": (512.085760e6 + 3.649536e6) / 5e5,
                     "trsm_inverse": (512.097536e6 + 452.634880e6) / 5e5,
                     "trsm_blocked": (512.105728e6 + 452.283904e6) / 5e5}
NCU_CAPTURE_K = 64


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=("ours", "reference"), default="ours")
    p.add_argument("--N", type=int, default=N_DEFAULT)
    p.add_argument("--k", type=int, default=K_DEFAULT)
    p.add_argument("--e2e-steps", type=int, default=3)
    p.add_argument("--skip-cpu-baseline", action="store_true")
    p.add_argument("--batch", type=int, default=256,
                   help="instances of the batched cholqr2! measurement (0 skips it)")
    p.add_argument("--wide-N", type=int, default=10_000_000,
                   help="rows of the k = 128 configuration (0 skips it)")
    p.add_argument("--rf-k", type=int, default=64, help="columns of the streamed range finder (0 skips it)")
    p.add_argument("--rf-budget-gb", type=float, default=40.0, help="device budget of the streamed range finder, GB")
    p.add_argument("--project-k", type=int, default=64,
                   help="columns of the device-resident project on the 215^3 Laplacian (0 skips it)")
    p.add_argument("--c1-N", type=int, default=1 << 20,
                   help="rows of the GhostPanels configuration (k = 32, panel width 8; 0 skips it)")
    p.add_argument("--skip-full-compare", action="store_true",
                   help="skip the full-size comparison of R and Q with the oracle's in the CPU leg")
    p.add_argument("--adjoint-N", type=int, default=1 << 22,
                   help="rows of the differentiation workload (0 skips it)")
    p.add_argument("--only", choices=("gram", "gram_tc", "trsm_blocked", "trsm_inverse", "ghost_fill", "laplace",
                                      "cholqr2", "cholqr2_adjoint", "project_adjoint", "hband", "adjoint_step",
                                      "batch"),
                   default=None,
                   help="launch one kernel of the step on the workload, the timed launches inside an NVTX range "
                        "named 'only' (what a profiler capture selects), and print its time")
    return p.parse_args()


def alg_bytes(N, k):
    return 96 * N * k  # 2 passes x (Gram read + TRSM read + TRSM write) x 16 B


def alg_flops(N, k):
    return 16 * N * k * k  # 2 passes x (Hermitian Gram 4Nk^2 + TRSM 4Nk^2)


def workload_config(N, k, extra=None):
    cfg = {
        "workload": f"cholqr2! device-resident, N={N}, k={k}, panel width {W_PANEL}, ComplexF64, "
                    "Y = U diag(logspace(0,-6,k)) V^H (seeded U Gaussian orthonormalized, V Haar)",
        "N": N, "k": k, "panel_width": W_PANEL, "form": "fp64",
        "l2": "inputs larger than L2 (10.24 GB vs 126 MB), no flush",
        "parallelism": "replicas (one matrix per GPU)",
    }
    if extra:
        cfg.update(extra)
    return cfg


# ---------------------------------------------------------------------------
# CPU side: the reference algorithm restated by the oracle, on host cores.

def cpu_threads():
    try:
        from threadpoolctl import threadpool_info
        n = [i.get("num_threads", 0) for i in threadpool_info() if i.get("internal_api") in ("openblas", "mkl", "blis")]
        if n:
            return max(n)
    except Exception:
        pass
    return os.cpu_count() or 1


def cpu_cholqr2_rate(Y0: np.ndarray, steps: int, warmup: int):
    """Times the oracle's cholqr2! (the reference's row-block order, BLAS and
    LAPACK on every host core) on Y0; returns (GB/s, seconds per step)."""
    from oracle import panel_oracle as oracle
    N, k = Y0.shape
    Y = Y0.copy(order="F")
    for _ in range(warmup):
        oracle.cholqr2(Y, W_PANEL)
    times = []
    for _ in range(steps):
        np.copyto(Y, Y0)
        t0 = time.perf_counter()
        oracle.cholqr2(Y, W_PANEL)
        times.append(time.perf_counter() - t0)
    sec = statistics.mean(times)
    return alg_bytes(N, k) / sec / 1e9, sec


def compare_c1_with_oracle(A, Q, R):
    """The oracle's cholqr2! (the reference's CPU backend path) on the ghost
    matrix's entries from the C restatement of the fill, against the device
    path's Q and R: the entries bit for bit, Q and R to 1e-12 relative."""
    from oracle import ghost as ghost_oracle
    from oracle import panel_oracle as oracle
    N, k = A.shape
    entries = ghost_oracle.ghost_block(np.complex128, N, k, 0, 0, C1_SEED)
    same_entries = bool(np.array_equal(entries, A))
    Qo = entries.copy(order="F")
    t0 = time.perf_counter()
    Ro, passes = oracle.cholqr2(Qo, C1_W)
    sec = time.perf_counter() - t0
    return {"entries_bitwise_equal": same_entries, "oracle_passes": passes, "oracle_s": sec,
            "q_rel": float(np.linalg.norm(Q - Qo) / np.linalg.norm(Qo)),
            "r_rel": float(np.linalg.norm(R - Ro) / np.linalg.norm(Ro)),
            "orthogonality_fro": oracle.orthogonality_error(Q),
            "reconstruction_rel": oracle.reconstruction_error(entries, Q, R),
            "oracle_orthogonality_fro": oracle.orthogonality_error(Qo), "bound_rel": 1e-12,
            "bound_orthogonality": 1e-12, "bound_reconstruction": 1e-13}


def compare_full_size_with_oracle(fb, backend, torch, Yt0, Yt, Y, R, queue, stream, N, k):
    """One cholqr2! of the full-size workload on the device and the oracle's
    on the same host copy of Y (all host cores): R and Q relative
    differences. Y's condition number is 1e6, so both factors are determined
    by Y only to about kappa * eps: the differences are reported against that
    scale, not against 1e-12."""
    from oracle import panel_oracle as oracle
    with torch.cuda.stream(stream):
        Yt.copy_(Yt0)
    stream.synchronize()
    backend.submit(queue, lambda: fb.kernels.cholqr2_resident(backend, Y, R))
    Q = Y.to_host()
    Rh = R.to_host()
    Yh = np.asfortranarray(wrap(fb, Yt0, N, k).to_host())
    t0 = time.perf_counter()
    Ro, passes = oracle.cholqr2(Yh, W_PANEL)
    sec = time.perf_counter() - t0
    out = {"N": N, "k": k, "oracle_s": sec, "oracle_passes": passes, "kappa": 1e6,
           "r_rel": float(np.linalg.norm(Rh - Ro) / np.linalg.norm(Ro)),
           "q_rel": float(np.linalg.norm(Q - Yh) / np.linalg.norm(Yh)),
           "oracle_orthogonality_fro": oracle.orthogonality_error(Yh),
           "scale_kappa_eps": 1e6 * 2.0 ** -52}
    del Q, Yh
    return out


def synthetic_host_sample(rows, k, seed=0xDEADBEEF):
    """The workload's matrix family on the host, for the CPU-side sample."""
    rng = np.random.default_rng(seed)
    G = (rng.standard_normal((rows, k)) + 1j * rng.standard_normal((rows, k))) / np.sqrt(2)
    U, _ = np.linalg.qr(G)
    V = haar_unitary(k, seed + 1)
    s = 10.0 ** np.linspace(0, -6, k)
    return np.asfortranarray((U * s) @ V.conj().T)


def haar_unitary(k, seed):
    rng = np.random.default_rng(seed)
    Z = (rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k))) / np.sqrt(2)
    Q, R = np.linalg.qr(Z)
    d = np.diag(R)
    return Q * (d / np.abs(d))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    k = args.k
    rows = min(args.N, CPU_SAMPLE_ROWS)
    Y0 = synthetic_host_sample(rows, k)
    steps = max(1, args.steps)
    gbs, sec = cpu_cholqr2_rate(Y0, steps=steps, warmup=max(0, min(args.warmup, 1)))
    cores = cpu_threads()
    sample = f"{rows} of the {args.N} rows (k={k}), {steps} timed steps of {sec:.3f} s"
    line = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args.N, k, {"cpu_sample_rows": rows}),
        "cpu_baseline": {"value": gbs, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": gbs, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "Funicular.jl is Julia, which is not installed; this is the CPU oracle's restatement of its "
                "CPU backend path (row-block order, zgemm/ztrsm/zpotrf from OpenBLAS/LAPACK).",
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU side.

class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
        0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
        0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
    }

    def __init__(self, device_index):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._thread = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._handle = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._handle, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # reported, not fatal
            self._nvml = None
            self.error = str(e)

    def _run(self):
        nv = self._nvml
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._handle, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksEventReasons(self._handle)
                for bit, name in self.REASONS.items():
                    if mask & bit and name != "gpu_idle":
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self._nvml is not None:
            self._thread = threading.Thread(target=self._run, daemon=True)
            self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons),
                    "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def run_batched(args, fb, backend, torch, device, world, max_over_ranks, barrier, hbm_peak, fp64_peak):
    """The batched range finder's orthonormalization: args.batch independent
    cholqr2! instances, N log-uniform on [1e4, 2e6], k drawn from {16, 32, 64}
    (seeded), on both batch schedules: the persistent kernel (the whole batch
    as one launch) and the eight stream lanes, each timed eagerly and as one
    captured CUDA graph, then the lanes again after the autotuner. Inputs are
    seeded complex Gaussians, refilled before each schedule's checked run;
    the timed steps orthonormalize in place (the later steps see orthonormal
    columns, which moves the same bytes through the same kernels)."""
    rng = np.random.default_rng(0xBA7C4)
    count = args.batch
    Ns = np.exp(rng.uniform(np.log(1e4), np.log(2e6), count)).astype(np.int64)
    ks = rng.choice([16, 32, 64], count)
    tensors = [torch.empty((int(k), int(N)), dtype=torch.complex128, device=device) for N, k in zip(Ns, ks)]

    def refill():
        gen = torch.Generator(device=device)
        gen.manual_seed(0xBA7C4)
        for t in tensors:
            t.copy_(torch.randn(t.shape, dtype=torch.complex128, device=device, generator=gen))
        torch.cuda.synchronize()

    Ys = [wrap(fb, t, int(N), int(k)) for t, N, k in zip(tensors, Ns, ks)]
    Rs = [backend.alloc_device(np.complex128, (int(k), int(k))) for k in ks]
    shapes = [(int(N), int(k)) for N, k in zip(Ns, ks)]
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    keep = []

    def workspace(schedule):
        nbytes = fb.kernels.cholqr2_batched_workspace_bytes(shapes, schedule=schedule)
        buf = backend.alloc_device(np.complex128, (nbytes // 16 + 32, 1))
        keep.append(buf)
        return ((buf.ptr + 255) // 256 * 256, nbytes)

    def timed(step):
        for _ in range(max(1, args.warmup)):
            step()
        backend.sync_queue(queue)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            step()
        b.record(stream)
        b.synchronize()
        return max_over_ranks(a.elapsed_time(b) / args.steps)

    alg = float(sum(96.0 * N * k for N, k in zip(Ns, ks)))
    # The batch's roofline: each instance at the slower of its HBM time
    # (96 N k bytes) and its FP64 time (16 N k^2 flops), summed.
    roof_ms = float(sum(max(96.0 * N * k / (hbm_peak * 1e9), 16.0 * N * k * k / (fp64_peak * 1e12))
                        for N, k in zip(Ns, ks))) * 1e3
    out = {}
    for schedule in ("persistent", "lanes"):
        ws = workspace(schedule)
        refill()
        passes = []
        backend.submit(queue, lambda: passes.extend(fb.kernels.cholqr2_batched(backend, Ys, Rs, workspace=ws,
                                                                                schedule=schedule)))
        worst = 0.0
        for t in tensors:
            Q = t.t()
            worst = max(worst, float(torch.linalg.matrix_norm(Q.conj().t() @ Q - torch.eye(
                Q.shape[1], dtype=Q.dtype, device=device))))
        enqueue = lambda: fb.kernels.cholqr2_batched(backend, Ys, Rs, wait=False, workspace=ws, schedule=schedule)
        ms_eager = timed(lambda: backend.submit(queue, enqueue))
        graph = backend.capture(queue, enqueue)
        ms_graph = timed(lambda: graph.launch(queue))
        del graph
        out[schedule] = {"ms_per_step_eager": ms_eager, "ms_per_step_graph": ms_graph,
                         "value_graph": whole_job_gbs(alg, world, ms_graph),
                         "value_eager": whole_job_gbs(alg, world, ms_eager),
                         "roofline_frac_graph": roof_ms / ms_graph, "passes_max": max(passes),
                         "orthogonality_fro_max": worst}
    out["persistent"]["launch"] = ("fb_zcholqr2_batched_persistent: a memset and one persistent kernel launch "
                                   "(one CTA per SM taking Gram, factor and solve jobs from a ticket counter)")
    out["lanes"]["launch"] = "fb_zcholqr2_batched: each instance's chain on one of eight stream lanes"
    # The lanes after the autotuner has chosen the Gram's row chunks for each
    # shape class of the batch (each class tuned at its largest N) and the
    # lane count.
    t0 = time.perf_counter()
    tuned = fb.autotune.tune_shapes(backend, shapes, forms=False)
    lanes = fb.autotune.tune_batch_lanes(backend, Ys, Rs)
    tune_s = time.perf_counter() - t0
    ws_t = workspace("lanes")
    enqueue_t = lambda: fb.kernels.cholqr2_batched(backend, Ys, Rs, wait=False, workspace=ws_t, schedule="lanes")
    graph_t = backend.capture(queue, enqueue_t)
    ms_tuned = timed(lambda: graph_t.launch(queue))
    passes_t = []
    backend.submit(queue, lambda: passes_t.extend(fb.kernels.cholqr2_batched(backend, Ys, Rs, workspace=ws_t,
                                                                              schedule="lanes")))
    shifts = sorted({r["gram_shift"] for r in tuned})
    fb.autotune.clear()
    del graph_t, tensors, Ys
    out["lanes"]["tuned"] = {"ms_per_step_graph": ms_tuned, "value_graph": whole_job_gbs(alg, world, ms_tuned),
                             "shape_classes": len(tuned), "gram_shifts_chosen": shifts, "lanes": lanes["lanes"],
                             "ms_by_lanes_eager": lanes["ms"], "tuning_s": tune_s, "passes_max": max(passes_t)}
    p = out["persistent"]
    return {"instances": count, "N_range": [int(Ns.min()), int(Ns.max())], "k_values": [16, 32, 64],
            "alg_bytes_per_step": alg, "ms_per_step_graph": p["ms_per_step_graph"],
            "ms_per_step_eager": p["ms_per_step_eager"], "value_graph": p["value_graph"],
            "value_eager": p["value_eager"], "unit": UNIT, "schedule": "persistent",
            "roofline": {"ms": roof_ms, "frac_graph": roof_ms / p["ms_per_step_graph"],
                         "frac_eager": roof_ms / p["ms_per_step_eager"],
                         "rule": "sum over instances of max(96 N k / HBM peak, 16 N k^2 / FP64 peak)"},
            "persistent": out["persistent"], "lanes": out["lanes"]}


C1_K, C1_W, C1_SEED = 32, 8, 0xDEADBEEF


def run_c1(args, fb, backend, torch, device, world, max_over_ranks, barrier, hbm_peak, fp64_peak):
    """The GhostPanels configuration: cholqr2! of a PanelMatrix{ComplexF64}
    with N = 2^20 rows, k = 32 columns and panel width 8, copied from
    GhostPanels(ComplexF64, N, k; seed = 0xdeadbeef) (filled on the device).
    End to end through the public API (copyto!(Y, Omega), then cholqr2(Y) on
    the page-locked host panels, resident since Y fits), and the device chain
    alone with the ghost fill restoring Y before each step, outside the step's
    event pair. Returns the record and the host input, Q and R for the
    oracle comparison of the CPU leg."""
    N, k, w = args.c1_N, C1_K, C1_W
    nbytes = N * k * 16
    plan = fb.ResidencyPlan(device_budget=4 * nbytes + fb.GiB, host_budget=2 * nbytes + 64 * 2 ** 20,
                            backend=backend)
    Omega = fb.GhostPanels(np.complex128, N, k, plan=plan, seed=C1_SEED, w=w)
    Y = fb.PanelMatrix.undef(np.complex128, N, k, plan=plan, w=w)
    Y.copy_from(Omega)
    A = Y.to_array()
    times = []
    for i in range(args.e2e_steps + 1):
        Y.copy_from(A)
        barrier()
        t0 = time.perf_counter()
        R = fb.cholqr2(Y)
        dt = time.perf_counter() - t0
        if i > 0:
            times.append(dt)
    Q = Y.to_array()
    ms_e2e = max_over_ranks(1e3 * sum(times) / max(1, len(times)))
    fb.free(Y)

    # The device chain alone: the ghost fill regenerates Y, then one event
    # pair around cholqr2!.
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    D = backend.alloc_device(np.complex128, (N, k))
    Rd = backend.alloc_device(np.complex128, (k, k))

    def fill():
        backend.submit(queue, lambda: fb.kernels.ghost_fill(backend, D, 0, 0, C1_SEED, np.complex128))

    def step():
        backend.submit(queue, lambda: fb.kernels.cholqr2_resident(backend, D, Rd, wait=False))

    for _ in range(max(3, args.warmup)):
        fill()
        step()
    backend.sync_queue(queue)
    barrier()
    pairs = []
    for _ in range(args.steps):
        fill()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        pairs.append((a, b))
    pairs[-1][1].synchronize()
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in pairs)) / args.steps
    roof_ms = max(alg_bytes(N, k) / (hbm_peak * 1e9), alg_flops(N, k) / (fp64_peak * 1e12)) * 1e3
    record = {
        "workload": f"cholqr2! of PanelMatrix{{ComplexF64}} N={N}, k={k}, panel width {w}, copied from "
                    f"GhostPanels seed {C1_SEED:#x} (device fill)",
        "ms_per_step": ms, "value": whole_job_gbs(alg_bytes(N, k), world, ms), "unit": UNIT,
        "step_roofline": {"ms_roofline": roof_ms, "frac": roof_ms / ms},
        "e2e": {"ms_per_step": ms_e2e, "value": whole_job_gbs(alg_bytes(N, k), world, ms_e2e), "unit": UNIT,
                "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + k * k * 16,
                "path": "Y.copy_from(A); funicular_b200.cholqr2(Y) on page-locked host panels"},
    }
    del D, Rd
    return record, (A, Q, R)


def run_wide(args, fb, backend, torch, device, world, max_over_ranks, barrier, fp64_peak):
    """The wide configuration: plain FP64 cholqr2! at N = args.wide_N (10^7),
    k = 128, on Y = U diag(s) V^H with condition numbers 1e4 and 1e7 (s
    log-spaced). The triangular solves go by 64-column blocks. Each kappa: one
    checked run (passes, ||Q^H Q - I||_F, ||Y - QR||/||Y||), then the timed
    loop on the result, as in the main step."""
    N, k = args.wide_N, 128
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    out = {"workload": f"cholqr2! FP64, N={N}, k={k}, ComplexF64 resident", "runs": []}
    for kappa in (1e4, 1e7):
        Yt0 = build_workload(fb, backend, torch, device, N, k, seed=0xC3 + int(np.log10(kappa)), kappa=kappa)
        Yt = Yt0.clone()
        torch.cuda.synchronize()
        Y = wrap(fb, Yt, N, k)
        R = backend.alloc_device(np.complex128, (k, k))
        checked = {}
        backend.submit(queue, lambda: checked.update(r=fb.kernels.cholqr2_resident(backend, Y, R)))
        passes, _ = checked["r"]
        orth, orth_cublas, recon = accuracy(fb, backend, torch, Yt0, Yt, R, N, k)
        del Yt0
        step = lambda: backend.submit(queue, lambda: fb.kernels.cholqr2_resident(backend, Y, R, wait=False))
        for _ in range(args.warmup):
            step()
        backend.sync_queue(queue)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            step()
        b.record(stream)
        b.synchronize()
        ms = max_over_ranks(a.elapsed_time(b) / args.steps)
        bound_ms = alg_flops(N, k) / (fp64_peak * 1e12) * 1e3
        out["runs"].append({"kappa": kappa, "passes": passes, "ms_per_step": ms,
                            "value": whole_job_gbs(alg_bytes(N, k), world, ms), "unit": UNIT,
                            "tflops": alg_flops(N, k) / (ms * 1e-3) / 1e12, "fp64_roofline_frac": bound_ms / ms,
                            "orthogonality_fro": orth, "orthogonality_fro_cublas": orth_cublas,
                            "reconstruction_rel": recon})
        del Yt, Y
    return out


def run_wide_storage(args, fb, backend, torch, device, world, max_over_ranks, barrier):
    """The wide configuration's storage comparison, end to end through the
    public API on page-locked host panels (N = args.wide_N, k = 128,
    kappa = 1e7): cholqr2 with ComplexF64 host storage, and the shifted
    CholeskyQR3 (cholqr3) with a ComplexF32 host tier, which halves the bytes
    that cross the bus. Both run the device-resident FP64 chain; each call
    uploads the panels (widened on the device), orthonormalizes, and writes
    Q back (narrowed on the device). Accuracy of what the panels hold after
    the call is measured on the device against the stored input."""
    N, k = args.wide_N, 128
    Yt0 = build_workload(fb, backend, torch, device, N, k, seed=0xC37, kappa=1e7)
    Yhost = np.asfortranarray(wrap(fb, Yt0, N, k).to_host())
    del Yt0
    out = {"workload": f"N={N}, k={k}, kappa=1e7, device-resident chain, host panels page-locked", "runs": []}
    for storage, fn, name in ((np.complex128, fb.cholqr2, "cholqr2, ComplexF64 storage"),
                              (np.complex64, fb.cholqr3, "shifted cholqr3, ComplexF32 storage")):
        itemsize = np.dtype(storage).itemsize
        nbytes = N * k * itemsize
        plan = fb.ResidencyPlan(device_budget=N * k * 16 + 8 * fb.GiB, host_budget=nbytes + 64 * 2 ** 20,
                                backend=backend, panel_width=32,
                                host_eltype=None if storage == np.complex128 else storage)
        Ypm = fb.PanelMatrix.from_array(Yhost, plan=plan)
        # The stored input (rounded to the storage eltype), widened on the device.
        q = backend.make_queue()
        Reft = torch.empty((k, N), dtype=torch.complex128, device=device)
        fb.panels.to_device(Ypm, wrap(fb, Reft, N, k), q)
        backend.sync_queue(q)
        times = []
        for i in range(3):
            if i:
                Ypm.copy_from(Yhost)
            barrier()
            t0 = time.perf_counter()
            R = fn(Ypm, resident=True)
            times.append(time.perf_counter() - t0)
        # Accuracy of the panels' Q (in their storage precision) in FP64.
        Qt = torch.empty_like(Reft)
        Qd = wrap(fb, Qt, N, k)
        fb.panels.to_device(Ypm, Qd, q)
        backend.sync_queue(q)
        G = backend.alloc_device(np.complex128, (k, k))
        fb.kernels.gram_accumulate(backend, G, Qd, Qd, 1.0, 0.0)
        orth = float(np.linalg.norm(G.to_host() - np.eye(k)))
        QRt = torch.empty_like(Reft)
        fb.kernels.rightmul_gemm(backend, wrap(fb, QRt, N, k), Qd, backend.todevice(np.asfortranarray(R)))
        backend.sync_all()
        QRt.sub_(Reft)
        recon = float(torch.linalg.vector_norm(QRt).item() / torch.linalg.vector_norm(Reft).item())
        del Qt, Qd, QRt, Reft
        ms = max_over_ranks(1e3 * sum(times[1:]) / len(times[1:]))
        out["runs"].append({"call": name, "storage": np.dtype(storage).name, "ms_per_call": ms,
                            "bus_bytes_per_call": 2 * nbytes, "value": world * alg_bytes(N, k) / (ms * 1e-3) / 1e9,
                            "unit": UNIT, "orthogonality_fro": orth, "reconstruction_rel": recon,
                            "clock": "host wall clock around the synchronous call, 2 calls after one warm-up"})
        fb.free(Ypm)
        del Ypm, plan
    return out


def measure_pcie(torch, device):
    """Page-locked copy bandwidth of this box, best of a few 1 GiB copies each
    way (cudaMemcpyAsync through torch): the streamed path's roofline."""
    n = 1 << 30
    h = torch.empty(n, dtype=torch.uint8, pin_memory=True)
    d = torch.empty(n, dtype=torch.uint8, device=device)
    out = {}
    for name, fn in (("h2d", lambda: d.copy_(h, non_blocking=True)), ("d2h", lambda: h.copy_(d, non_blocking=True))):
        fn()
        torch.cuda.synchronize()
        best = None
        for _ in range(3):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            b.synchronize()
            ms = a.elapsed_time(b)
            best = ms if best is None else min(best, ms)
        out[name] = n / (best * 1e-3) / 1e9
    del h, d
    return out


def run_range_finder(args, fb, backend, torch, device, world, max_over_ranks, barrier):
    """The streamed range finder (config C4, scaled): G = -Lap_7 + (0.5+0.1i) I
    on the 342^3 grid (N = 40 001 688) applied matrix-free, X = GhostPanels
    (filled on the device), Y = panelmul(G, X), cholqr2 of Y through row
    sweeps, S = project(Y, G), with the plan's device budget below the matrix
    so every panel streams through page-locked host memory. k = args.rf_k and
    the budget are scaled down from 256 and 40 GB so one step fits the bench:
    project moves p (p + 1) panels, quadratic in the panel count. Each phase is
    timed on the host clock around its synchronous call; the bytes that cross
    the bus are counted from the panel widths and set against the measured
    page-locked copy bandwidth."""
    grid = (342, 342, 342)
    N = grid[0] * grid[1] * grid[2]
    k = args.rf_k
    # Host blocks are whole panels of the plan's width (the last one too);
    # room for Y and for project's second matrix Z (the two-sweep schedule).
    budget = int(args.rf_budget_gb * 1e9)
    plan = fb.ResidencyPlan(device_budget=budget, host_budget=int(2.1 * N * k * 16) + 4 * fb.GiB, backend=backend)
    X = fb.GhostPanels(np.complex128, N, k, plan=plan, seed=0xC4)
    Y = fb.PanelMatrix.undef(np.complex128, N, k, plan=plan, w=X.w)
    G = fb.Laplacian7(grid, 0.5 + 0.1j)
    pcie = measure_pcie(torch, device)

    schedule = fb.panelblas.project_schedule(Y)

    def step():
        t = [time.perf_counter()]
        fb.panelmul(Y, G, X)
        t.append(time.perf_counter())
        R = fb.cholqr2(Y, resident=False)
        t.append(time.perf_counter())
        S = fb.project(Y, G, schedule=schedule)
        t.append(time.perf_counter())
        return [1e3 * (t[i + 1] - t[i]) for i in range(3)], R, S

    barrier()
    step()
    barrier()
    ms, R, S = step()
    ms = [max_over_ranks(x) for x in ms]
    widths = [Y.panelwidth(j) for j in range(Y.npanels())]
    p = len(widths)
    col = 16 * N
    passes = 2  # the third pass runs only after a shift, and the Gram of G X is well conditioned here
    # Host to device and back, per phase: panelmul writes Y (X is generated on
    # the device); cholqr2 reads Y once for the first Gram and once per pass
    # for the solve, which also takes the next pass's Gram (twice per pass on
    # a narrowed host tier), and writes it once per pass; project in two
    # sweeps reads Y, writes Z = G Y, then reads both (the nested schedule
    # uploads p (p + 1) panels).
    if schedule == "two-sweep":
        up_project, down_project = 3 * col * k, col * k
    elif schedule == "resident":
        up_project, down_project = col * k, 0
    else:
        up_project, down_project = col * sum(widths) + col * p * sum(widths), 0
    cholqr2_reads = passes + 1 if fb.panelblas.solves_what_it_stores(Y) else 2 * passes
    up = {"panelmul": 0, "cholqr2": cholqr2_reads * col * k, "project": up_project}
    down = {"panelmul": col * k, "cholqr2": passes * col * k, "project": down_project}
    Gq = fb.gram(Y)
    orth = float(np.linalg.norm(Gq - np.eye(k)))
    total_ms = sum(ms)
    total_bus = sum(up.values()) + sum(down.values())
    # The link carries both directions at once: a phase's bound is its slower
    # direction's bytes over that direction's measured bandwidth. The three
    # calls run one after another, so the step's bound is the sum over the
    # phases; the bound if every phase's traffic could overlap every other's
    # is reported beside it.
    phase_ms = {ph: 1e3 * max(up[ph] / (pcie["h2d"] * 1e9), down[ph] / (pcie["d2h"] * 1e9)) for ph in up}
    bound_ms = sum(phase_ms.values())
    overlapped_ms = 1e3 * max(sum(up.values()) / (pcie["h2d"] * 1e9), sum(down.values()) / (pcie["d2h"] * 1e9))
    out = {"workload": f"streamed range finder, 342^3 Laplacian (N={N}), k={k}, {p} panels of width {max(widths)}, "
                       f"device budget {budget / 1e9:.1f} GB for a {col * k / 1e9:.1f} GB matrix, "
                       f"project schedule {schedule}",
           "project_schedule": schedule,
           "ms": {"panelmul": ms[0], "cholqr2_streamed": ms[1], "project": ms[2], "step": total_ms},
           "bus_bytes_up": up, "bus_bytes_down": down, "bus_gbs": total_bus / (total_ms * 1e-3) / 1e9,
           "pcie_measured_gbs": pcie, "ms_pcie_bound": bound_ms, "pcie_roofline_frac": bound_ms / total_ms,
           "ms_pcie_bound_by_phase": phase_ms,
           "pcie_frac_by_phase": {ph: phase_ms[ph] / v for ph, v in zip(("panelmul", "cholqr2", "project"), ms)},
           "ms_pcie_bound_phases_overlapped": overlapped_ms,
           "orthogonality_fro": orth, "r_finite": bool(np.isfinite(R).all()), "s_finite": bool(np.isfinite(S).all()),
           "clock": "host wall clock around each synchronous call, the second of two steps"}
    fb.free(Y)
    del X, Y, plan
    return out


def run_project(args, fb, backend, torch, device, world, max_over_ranks, barrier, hbm_peak, fp64_peak):
    """project(Q, G) = Q^H (G Q) device-resident (src/panelblas.jl:268-301 in
    its two-sweep form): Q is N x k with N = 215^3 = 9 938 375 (the C2 size on
    a cube), k = args.project_k, G = -Lap_7 + (0.5+0.1i) I. Timed on the
    device: the operator applied to all of Q, the cross Gram Q^H (G Q) (the
    projection proper: 32 N k bytes, 8 N k^2 flops), and both; end to end:
    project() on a PanelMatrix in page-locked host panels (Q up once, G
    applied, one cross Gram, S to the host)."""
    grid = (215, 215, 215)
    N = grid[0] * grid[1] * grid[2]
    k = args.project_k
    G = fb.Laplacian7(grid, 0.5 + 0.1j)
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    Q = backend.alloc_device(np.complex128, (N, k))
    Z = backend.alloc_device(np.complex128, (N, k))
    S = backend.alloc_device(np.complex128, (k, k))
    backend.submit(queue, lambda: fb.kernels.ghost_fill(backend, Q, 0, 0, 0x9A0, np.complex128))

    def timed(fn):
        for _ in range(max(3, args.warmup)):
            backend.submit(queue, fn)
        backend.sync_queue(queue)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            backend.submit(queue, fn)
        b.record(stream)
        b.synchronize()
        return max_over_ranks(a.elapsed_time(b) / args.steps)

    ms_apply = timed(lambda: G.apply(backend, Z, Q))
    ms_gram = timed(lambda: fb.kernels.gram_accumulate(backend, S, Q, Z, 1.0, 0.0))
    ms_both = timed(lambda: (G.apply(backend, Z, Q), fb.kernels.gram_accumulate(backend, S, Q, Z, 1.0, 0.0)))
    flops, nbytes = 8 * N * k * k, 32 * N * k
    roof_ms = max(nbytes / (hbm_peak * 1e9), flops / (fp64_peak * 1e12)) * 1e3
    # End to end through the public API.
    Qh = np.asfortranarray(Q.to_host())
    del Q, Z
    release_device_memory(torch)
    plan = fb.ResidencyPlan(device_budget=3 * N * k * 16 + fb.GiB, host_budget=N * k * 16 + 64 * 2 ** 20,
                            backend=backend, panel_width=16)
    Qpm = fb.PanelMatrix.from_array(Qh, plan=plan)
    schedule = fb.panelblas.project_schedule(Qpm)
    times = []
    for i in range(4):
        barrier()
        t0 = time.perf_counter()
        Sh = fb.project(Qpm, G)
        if i:
            times.append(time.perf_counter() - t0)
    ms_e2e = max_over_ranks(1e3 * sum(times) / len(times))
    fb.free(Qpm)
    del Qh, Qpm, plan
    return {"workload": f"project(Q, G), N={N} (215^3 Laplacian, shift 0.5+0.1i), k={k}, device-resident",
            "cross_gram": {"ms": ms_gram, "tflops": flops / (ms_gram * 1e-3) / 1e12,
                           "gbs": nbytes / (ms_gram * 1e-3) / 1e9, "ms_roofline": roof_ms, "frac": roof_ms / ms_gram,
                           "per_launch": "8 N k^2 flops, 32 N k bytes (Q and G Q read)"},
            "apply": {"ms": ms_apply, "gbs": 32 * N * k / (ms_apply * 1e-3) / 1e9,
                      "hbm_frac": 32 * N * k / (ms_apply * 1e-3) / 1e9 / hbm_peak,
                      "per_launch": "32 N k bytes (Q read, G Q written)"},
            "ms_apply_plus_gram": ms_both,
            "e2e": {"ms_per_call": ms_e2e, "schedule": schedule, "h2d_bytes": N * k * 16,
                    "path": "funicular_b200.project(PanelMatrix, Laplacian7) on page-locked host panels",
                    "s_finite": bool(np.isfinite(Sh).all())}}


def run_adjoint(args, fb, backend, torch, device, world, max_over_ranks, barrier):
    """The differentiation workload: N = args.adjoint_N (2^22), k = 64, the
    loss real(tr(W^H Q)) + ||S||_F^2 with (Q, R) = cholqr2!(Y) and
    S = Q^H (G Q), G Hermitian with 64 superdiagonals. Y, W and the band are
    seeded device ghost fills (complex Gaussians), the band scaled by
    sqrt(N / (129 k)) so that both terms of the loss are of the same order.
    One step is the forward pass and the pullbacks the rrules run, on
    preallocated buffers: copy Y, cholqr2!, G Q, 2 Q^H (G Q) (Sbar), W^H Q,
    copy W into Qbar, the project pullback accumulated into Qbar, the cholqr2!
    pullback written over Qbar. The gradient is checked against central
    differences in 4 random directions (the tests use 32)."""
    N, k, kd = args.adjoint_N, 64, 64
    ghost = lambda dst, seed: fb.kernels.ghost_fill(backend, dst, 0, 0, seed, np.complex128)
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    alloc = lambda r, c: backend.alloc_device(np.complex128, (r, c))
    YD = alloc(N, 2 * k)
    Y, D = YD.view(slice(None), slice(0, k)), YD.view(slice(None), slice(k, 2 * k))
    W, Q, GQ, Qbar = alloc(N, k), alloc(N, k), alloc(N, k), alloc(N, k)
    R, Sbar, T = alloc(k, k), alloc(k, k), alloc(k, k)
    ghost(Y, 0xC5)
    ghost(W, 0xC6)
    G = fb.HermitianBand.ghost(backend, N, kd, seed=0xC7, scale=float(np.sqrt(N / ((2 * kd + 1) * k))))
    copy = fb.device_api.copy_region
    K = fb.kernels

    def forward(src):
        copy(Q, src, queue)
        K.cholqr2_resident(backend, Q, R, wait=False)
        G.apply(backend, GQ, Q)
        K.gram_accumulate(backend, Sbar, Q, GQ, 2.0, 0.0)
        K.gram_accumulate(backend, T, W, Q, 1.0, 0.0)

    def backward():
        copy(Qbar, W, queue)
        K.project_adjoint(backend, Qbar, GQ, Sbar, None, accumulate=True)
        K.cholqr2_adjoint(backend, Qbar, Y, R, Qbar, None)

    def loss():
        backend.sync_queue(queue)
        return float(np.real(np.trace(T.to_host())) + np.linalg.norm(Sbar.to_host() / 2) ** 2)

    def timed(fn, reps):
        for _ in range(max(1, args.warmup)):
            backend.submit(queue, fn)
        backend.sync_queue(queue)
        barrier()
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            backend.submit(queue, fn)
        b.record(stream)
        b.synchronize()
        return max_over_ranks(a.elapsed_time(b) / reps)

    reps = max(3, min(args.steps, 10))
    ms_step = timed(lambda: (forward(Y), backward()), reps)
    ms_forward = timed(lambda: forward(Y), reps)
    ms_cholqr2_pullback = timed(lambda: K.cholqr2_adjoint(backend, GQ, Y, R, Qbar, None), reps)
    ms_project_pullback = timed(lambda: K.project_adjoint(backend, Qbar, GQ, Sbar, None, accumulate=True), reps)
    ms_band = timed(lambda: G.apply(backend, GQ, Q), reps)
    # The gradient, then central differences of the loss through the same
    # forward kernels: Y +- h D is one product of [Y D] by [I; +-h I].
    backend.submit(queue, lambda: (forward(Y), backward()))
    loss0 = loss()
    h = 1e-6
    I = np.eye(k, dtype=np.complex128)
    Cp, Cm = backend.todevice(np.vstack([I, h * I])), backend.todevice(np.vstack([I, -h * I]))
    Yh = alloc(N, k)
    fd, an = [], []
    for i in range(4):
        backend.submit(queue, lambda: ghost(D, 0x1000 + i))
        vals = []
        for C in (Cp, Cm):
            backend.submit(queue, lambda: (K.rightmul_gemm(backend, Yh, YD, C), forward(Yh)))
            vals.append(loss())
        fd.append((vals[0] - vals[1]) / (2 * h))
        backend.submit(queue, lambda: K.gram_accumulate(backend, T, Qbar, D, 1.0, 0.0))
        backend.sync_queue(queue)
        an.append(float(np.real(np.trace(T.to_host()))))
    fd, an = np.array(fd), np.array(an)
    fd_err = float(np.linalg.norm(fd - an) / np.linalg.norm(an))
    flops_cp = 20.0 * N * k * k           # Qbar^H Y, Qbar R^-H (triangular), Y (R^-1 H R^-H)
    flops_pp = 8.0 * N * k * k            # (G Q)(Sbar + Sbar^H)
    flops_band = 8.0 * N * k * (2 * kd + 1)
    del YD, W, Q, GQ, Qbar, Yh, G
    return {
        "workload": f"rrule through cholqr2! and project, N={N}, k={k}, G Hermitian band kd={kd}",
        "ms_per_step": ms_step, "ms_forward": ms_forward, "loss": loss0,
        "fd_rel_error": fd_err, "fd_directions": 4, "fd_step": h, "bound_fd": 1e-6,
        "cholqr2_pullback": {"ms": ms_cholqr2_pullback, "tflops": flops_cp / (ms_cholqr2_pullback * 1e-3) / 1e12,
                             "gbs": 80.0 * N * k / (ms_cholqr2_pullback * 1e-3) / 1e9,
                             "per_launch": "20 N k^2 flops, 80 N k bytes (Qbar, Y read twice, Ybar written)"},
        "project_pullback": {"ms": ms_project_pullback, "tflops": flops_pp / (ms_project_pullback * 1e-3) / 1e12,
                             "gbs": 48.0 * N * k / (ms_project_pullback * 1e-3) / 1e9,
                             "per_launch": "8 N k^2 flops, 48 N k bytes (G Q read, Qbar read and written)"},
        "band_apply": {"ms": ms_band, "tflops": flops_band / (ms_band * 1e-3) / 1e12,
                       "per_launch": "8 N k (2 kd + 1) flops"},
    }


def release_device_memory(torch) -> None:
    """Frees what dropped Python references held: the backend's buffers (their
    finalizers run on collection) and the blocks torch's allocator caches."""
    import gc
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def reduce_max_over_ranks(x: float, world: int, device) -> float:
    """The largest of the ranks' values: the whole job takes as long as its
    slowest rank. An all-reduce over the default process group (NCCL on the
    GPUs, gloo in the CPU tests)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_gbs(bytes_per_rank: float, world: int, ms: float) -> float:
    """Weak scaling: every rank orthonormalizes its own matrix, so the job moves
    world times the bytes of one rank in the slowest rank's time."""
    return world * bytes_per_rank / (ms * 1e-3) / 1e9


def measure_fp64_peak(torch, device):
    """cuBLAS ZGEMM (complex FP64, the arithmetic of this path) through torch,
    best of a few 4096^3 products: the FP64 roofline denominator."""
    n = 4096
    a = torch.randn(n, n, dtype=torch.complex128, device=device)
    b = torch.randn(n, n, dtype=torch.complex128, device=device)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del a, b
    return 8 * n ** 3 / (best * 1e-3) / 1e12


def wrap(fb, tensor, rows, cols):
    """A column-major DeviceMatrix over a (cols, rows) row-major torch tensor."""
    import numpy as _np
    return fb.DeviceMatrix(tensor.data_ptr(), (rows, cols), rows, _np.dtype(_np.complex128), tensor)


def build_workload(fb, backend, torch, device, N, k, seed, kappa=1e6):
    """Y = U diag(s) V^H on the device, s log-spaced from 1 to 1/kappa. U: a
    seeded complex Gaussian made orthonormal by the backend's own cholqr2!;
    V: seeded Haar unitary."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    Ut = torch.randn((k, N), dtype=torch.complex128, device=device, generator=gen)
    U = wrap(fb, Ut, N, k)
    Rtmp = backend.alloc_device(np.complex128, (k, k))
    fb.kernels.cholqr2_resident(backend, U, Rtmp)
    V = haar_unitary(k, seed + 1)
    s = 10.0 ** np.linspace(0, -np.log10(kappa), k)
    C = backend.todevice(np.asfortranarray(s[:, None] * V.conj().T))
    Yt = torch.empty((k, N), dtype=torch.complex128, device=device)
    Y = wrap(fb, Yt, N, k)
    fb.kernels.rightmul_gemm(backend, Y, U, C)
    backend.sync_all()
    del U, Ut
    return Yt


def accuracy(fb, backend, torch, Yt0, Qt, R, N, k):
    """||Q^H Q - I||_F (with the backend's Gram) and ||Y - Q R||_F / ||Y||_F."""
    Q = wrap(fb, Qt, N, k)
    G = backend.alloc_device(np.complex128, (k, k))
    fb.kernels.gram_accumulate(backend, G, Q, Q, 1.0, 0.0)
    orth = float(np.linalg.norm(G.to_host() - np.eye(k)))
    # The same measure with cuBLAS ZGEMM, which shares no code with the backend.
    Qm = Qt.t()
    orth_cublas = float(np.linalg.norm((Qm.conj().t() @ Qm).cpu().numpy() - np.eye(k)))
    QRt = torch.empty_like(Qt)
    fb.kernels.rightmul_gemm(backend, wrap(fb, QRt, N, k), Q, R)
    backend.sync_all()
    QRt.sub_(Yt0)
    recon = float(torch.linalg.vector_norm(QRt).item() / torch.linalg.vector_norm(Yt0).item())
    del QRt
    return orth, orth_cublas, recon


def run_ours(args):
    import torch
    import torch.distributed as dist

    import __graft_entry__
    fb = __graft_entry__.load()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=device)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max_over_ranks(x, world, device)

    N, k = args.N, args.k
    backend = fb.B200Backend(local)
    fp64_peak = measure_fp64_peak(torch, device)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    hbm_source = "MEASURED_PEAKS.json" if os.path.exists(peaks_path) else "fallback"

    Yt0 = build_workload(fb, backend, torch, device, N, k, seed=0xDEADBEEF + rank)
    Yt = Yt0.clone()
    # torch works on its own stream and the backend on a non-blocking queue:
    # nothing orders the two, so wait here for the copy to land.
    torch.cuda.synchronize()
    Y = wrap(fb, Yt, N, k)
    R = backend.alloc_device(np.complex128, (k, k))

    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)

    # One checked run on the true Y: accuracy and the number of passes.
    checked = {}
    backend.submit(queue, lambda: checked.update(r=fb.kernels.cholqr2_resident(backend, Y, R)))
    passes, _ = checked["r"]
    orth, orth_cublas, recon = accuracy(fb, backend, torch, Yt0, Yt, R, N, k)

    def step():
        backend.submit(queue, lambda: fb.kernels.cholqr2_resident(backend, Y, R, wait=False))

    def restore():
        # Every step orthonormalizes the configured input, not the Q the
        # previous step left: a device-to-device copy of the pristine Y on the
        # queue, outside the step's event pair.
        with torch.cuda.stream(stream):
            Yt.copy_(Yt0)

    def timed_steps(fn, count, with_launches=False):
        """count steps, each on a freshly restored Y, every step bracketed by
        its own CUDA-event pair on the queue; returns (summed ms, launches)."""
        pairs = []
        launches_before = fb._lib.kernel_launches()
        for _ in range(count):
            restore()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            pairs.append((a, b))
        pairs[-1][1].synchronize()
        return sum(a.elapsed_time(b) for a, b in pairs), fb._lib.kernel_launches() - launches_before

    for _ in range(args.warmup):
        restore()
        step()
    backend.sync_queue(queue)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()

    with ClockSampler(local) as clocks:
        ms_total, launches = timed_steps(step, args.steps)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ms_total = max_over_ranks(ms_total)
    ms_step = ms_total / args.steps
    value = whole_job_gbs(alg_bytes(N, k) * args.steps, world, ms_total)

    # The tensor-core form of the same step: every Gram on the integer tensor
    # cores (Ozaki slices), Cholesky and triangular solves in FP64. One checked
    # run on the true Y for its accuracy, then the same timed loop.
    tensor_form = None
    if k <= 64:
        Yt.copy_(Yt0)
        torch.cuda.synchronize()
        Rtc = backend.alloc_device(np.complex128, (k, k))
        checked_tc = {}
        backend.submit(queue, lambda: checked_tc.update(
            r=fb.kernels.cholqr2_resident(backend, Y, Rtc, form="tc")))
        passes_tc, _ = checked_tc["r"]
        orth_tc, orth_tc_cublas, recon_tc = accuracy(fb, backend, torch, Yt0, Yt, Rtc, N, k)

        def step_tc():
            backend.submit(queue, lambda: fb.kernels.cholqr2_resident(backend, Y, Rtc, wait=False, form="tc"))

        for _ in range(args.warmup):
            restore()
            step_tc()
        backend.sync_queue(queue)
        barrier()
        ms_tc_total, _ = timed_steps(step_tc, args.steps)
        barrier()
        ms_tc = max_over_ranks(ms_tc_total) / args.steps
        tensor_form = {
            "ms_per_step": ms_tc, "value": world * alg_bytes(N, k) / (ms_tc * 1e-3) / 1e9, "unit": UNIT,
            "speedup_vs_fp64_form": ms_step / ms_tc, "passes": passes_tc,
            "orthogonality_fro": orth_tc, "orthogonality_fro_cublas": orth_tc_cublas,
            "reconstruction_rel": recon_tc, "bound_orthogonality": 1e-12, "bound_reconstruction": 1e-13,
            "gram": "7 signed 8-bit slices per entry against a power-of-two column scale, 28 int8 products",
        }

    # Per-kernel durations, same shapes as inside the step, same queue.
    def time_kernel(fn, reps):
        fn()
        backend.sync_queue(queue)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / reps

    G = backend.alloc_device(np.complex128, (k, k))
    reps = max(3, min(args.steps, 20))
    gram_ms = time_kernel(lambda: backend.submit(queue, lambda: fb.kernels.gram_accumulate(backend, G, Y, Y, 1.0, 0.0)), reps)
    gram_tc_ms = (time_kernel(lambda: backend.submit(queue, lambda: fb.kernels.gram_tc(backend, G, Y, 1.0, 0.0)), reps)
                  if k <= 64 else None)
    # The two triangular solves of the step: pass 1 divides by the factor of
    # the ill-conditioned input (the blocked solve), pass 2 by a factor within
    # O(eps) of the identity (one product by its inverse). The first is timed
    # with the R of the checked run (its condition is the input's), restoring
    # Y between launches is not needed: the work does not depend on the values.
    Rid = backend.todevice(np.asfortranarray(np.eye(k, dtype=np.complex128)))
    R1 = backend.todevice(np.asfortranarray(R.to_host()))
    trsm_ms = time_kernel(lambda: backend.submit(queue, lambda: fb.kernels.rdiv_upper(backend, Y, Rid)), reps)
    trsm_blocked_ms = time_kernel(lambda: backend.submit(queue, lambda: fb.kernels.rdiv_upper(backend, Y, R1)), reps)
    # rightmul_gemm! (src/kernels.jl:73, the product behind rightmul! and the
    # dense operator): Z <- Y C with a dense k x k C, into a second N x k
    # buffer. 8 N k^2 flops (a full complex product), 32 N k bytes.
    Zt = torch.empty_like(Yt)
    torch.cuda.synchronize()
    Zm = wrap(fb, Zt, N, k)
    rightmul_ms = time_kernel(lambda: backend.submit(queue, lambda: fb.kernels.rightmul_gemm(backend, Zm, Y, R1)),
                              reps)
    del Zm, Zt
    # The GhostPanels device fill (the C1 input generator), over the same
    # N x k block: 16 N k bytes written per launch, nothing read. It runs last
    # because it overwrites Y.
    ghost_ms = time_kernel(lambda: backend.submit(
        queue, lambda: fb.kernels.ghost_fill(backend, Y, 0, 0, 0xDEADBEEF, np.complex128)), reps)
    kernel_flops = 4 * N * k * k  # each of them, algorithmic
    kernels = {
        "gram_partial+reduce": {"ms": gram_ms, "tflops": kernel_flops / (gram_ms * 1e-3) / 1e12,
                                "gbs": 16 * N * k / (gram_ms * 1e-3) / 1e9},
        "trsm_inverse": {"ms": trsm_ms, "tflops": kernel_flops / (trsm_ms * 1e-3) / 1e12,
                         "gbs": 32 * N * k / (trsm_ms * 1e-3) / 1e9},
        "trsm_blocked": {"ms": trsm_blocked_ms, "tflops": kernel_flops / (trsm_blocked_ms * 1e-3) / 1e12,
                         "gbs": 32 * N * k / (trsm_blocked_ms * 1e-3) / 1e9},
    }
    dominant = max(kernels, key=lambda name: kernels[name]["ms"])
    kernels["rightmul_gemm"] = {"ms": rightmul_ms, "tflops": 8 * N * k * k / (rightmul_ms * 1e-3) / 1e12,
                                "gbs": 32 * N * k / (rightmul_ms * 1e-3) / 1e9,
                                "fp64_frac": 8 * N * k * k / (rightmul_ms * 1e-3) / 1e12 / fp64_peak,
                                "per_launch": f"8 N k^2 = {8 * N * k * k:.3e} flops, 32 N k bytes"}
    if gram_tc_ms is not None:
        kernels["gram_tensor_cores"] = {"ms": gram_tc_ms, "tflops": kernel_flops / (gram_tc_ms * 1e-3) / 1e12,
                                        "gbs": 16 * N * k / (gram_tc_ms * 1e-3) / 1e9,
                                        "int8_tops": 28 * 2 * 128 * 64 * 2 * N / (gram_tc_ms * 1e-3) / 1e12}
    ghost_gbs = 16 * N * k / (ghost_ms * 1e-3) / 1e9
    kernels["ghost_fill"] = {"ms": ghost_ms, "gbs": ghost_gbs, "hbm_frac": ghost_gbs / hbm_peak,
                             "per_launch": f"16 N k = {16 * N * k:.3e} bytes written"}
    dk = kernels[dominant]
    traffic = NCU_BYTES_PER_ROW[dominant] * N if k == NCU_CAPTURE_K else None
    roofline = {
        "bound": "fp64", "achieved": dk["tflops"], "peak": fp64_peak, "unit": "TFLOP/s",
        "frac": dk["tflops"] / fp64_peak, "traffic": traffic, "kernel": dominant,
        "traffic_source": "ncu dram bytes of the N=5e5 capture (profiles/*_N5e5_k64_ncu.md), scaled by N/5e5",
        "peak_source": "cuBLAS ZGEMM 4096^3 measured in this run (FP64 has no entry in MEASURED_PEAKS.json)",
        "per_launch": f"4 N k^2 = {kernel_flops:.3e} flops per launch",
    }
    step_flops_bound = alg_flops(N, k) / (fp64_peak * 1e12) * 1e3
    step_bytes_bound = alg_bytes(N, k) / (hbm_peak * 1e9) * 1e3
    step_roofline = {
        "ms_fp64_bound": step_flops_bound, "ms_hbm_bound": step_bytes_bound,
        "ms_roofline": max(step_flops_bound, step_bytes_bound), "ms_measured": ms_step,
        "frac": max(step_flops_bound, step_bytes_bound) / ms_step,
        "achieved_tflops": alg_flops(N, k) / (ms_step * 1e-3) / 1e12,
        "hbm_peak_gbs": hbm_peak, "hbm_peak_source": hbm_source, "fp64_peak_tflops": fp64_peak,
    }

    def section(run, *extra):
        # Each section allocates both through the backend and through torch;
        # what a finished section held goes back to the device before the
        # next one (torch's caching allocator would otherwise keep it).
        out = run(args, fb, backend, torch, device, world, max_over_ranks, barrier, *extra)
        release_device_memory(torch)
        return out

    c1, c1_outputs = section(run_c1, hbm_peak, fp64_peak) if args.c1_N > 0 else (None, None)
    batched = section(run_batched, hbm_peak, fp64_peak) if args.batch > 0 else None
    wide = section(run_wide, fp64_peak) if args.wide_N > 0 else None
    if wide is not None and args.e2e_steps > 0:
        wide["storage"] = section(run_wide_storage)
    range_finder = section(run_range_finder) if args.rf_k > 0 else None
    project = section(run_project, hbm_peak, fp64_peak) if args.project_k > 0 else None
    adjoint = section(run_adjoint) if args.adjoint_N > 0 else None
    if adjoint is not None:
        fp = adjoint["cholqr2_pullback"]["tflops"]
        adjoint["cholqr2_pullback"]["fp64_frac"] = fp / fp64_peak
        adjoint["project_pullback"]["fp64_frac"] = adjoint["project_pullback"]["tflops"] / fp64_peak
        adjoint["band_apply"]["fp64_frac"] = adjoint["band_apply"]["tflops"] / fp64_peak

    # End to end through the public API, the call a user makes: a PanelMatrix
    # whose panels sit in page-locked host memory, and cholqr2 on it. Each
    # step uploads the panels, runs the device-resident chain, writes Q back
    # into the panels and returns R on the host; the call is synchronous, so
    # it is timed on the host clock (max over ranks). The panels are restored
    # to Y before each step, outside the timed region.
    e2e = None
    if args.e2e_steps > 0:
        nbytes = N * k * 16
        Yhost = np.asfortranarray(wrap(fb, Yt0, N, k).to_host())
        plan = fb.ResidencyPlan(device_budget=nbytes + 4 * fb.GiB, host_budget=nbytes + 64 * 2 ** 20,
                                backend=backend, panel_width=W_PANEL)
        Ypm = fb.PanelMatrix.from_array(Yhost, plan=plan)
        times = []
        for i in range(args.e2e_steps + 1):
            Ypm.copy_from(Yhost)
            barrier()
            t0 = time.perf_counter()
            Rh = fb.cholqr2(Ypm, resident=True)
            dt = time.perf_counter() - t0
            if i > 0:  # the first call checks out the plan's buffers
                times.append(dt)
        Qcheck = Ypm.panels[0].storage()[:4096]
        ok = bool(np.isfinite(Rh).all() and np.isfinite(Qcheck).all())
        ms_e2e = max_over_ranks(1e3 * sum(times) / len(times))
        e2e = {"value": world * alg_bytes(N, k) / (ms_e2e * 1e-3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes + k * k * 16,
               "ms_per_step": ms_e2e, "steps": args.e2e_steps, "finite": ok,
               "path": "funicular_b200.cholqr2(PanelMatrix) on page-locked host panels: panels up, "
                       "device-resident chain, Q back into the panels, R returned to the host",
               "clock": "host wall clock around the synchronous call"}
        fb.free(Ypm)
        del Yhost, Ypm, plan

    cpu = None
    full_compare = None
    if rank == 0 and world == 1 and not args.skip_cpu_baseline:
        rows = min(N, CPU_SAMPLE_ROWS)
        sample = np.asfortranarray(wrap(fb, Yt0, N, k).view(slice(0, rows)).to_host())
        gbs, sec = cpu_cholqr2_rate(sample, steps=2, warmup=0)
        cpu = {"value": gbs, "unit": UNIT, "cores": cpu_threads(), "kind": "port",
               "sample": f"first {rows} rows of the workload (k={k}), 2 timed steps of {sec:.3f} s each"}
        del sample
        # The oracle as the checker: the GhostPanels configuration's Q and R
        # against the oracle's on the same entries (its C restatement of the
        # ghost fill), and the full-size workload's R and Q against the
        # oracle's full-size run.
        if c1_outputs is not None:
            c1["oracle"] = compare_c1_with_oracle(*c1_outputs)
        if not args.skip_full_compare:
            full_compare = compare_full_size_with_oracle(fb, backend, torch, Yt0, Yt, Y, R, queue, stream, N, k)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(N, k),
        "roofline": roofline, "step_roofline": step_roofline, "kernels": kernels,
        "accuracy": {"orthogonality_fro": orth, "orthogonality_fro_cublas": orth_cublas,
                     "reconstruction_rel": recon, "passes": passes,
                     "bound_orthogonality": 1e-12, "bound_reconstruction": 1e-13,
                     "vs_oracle_full_size": full_compare},
        "c1": c1,
        "tensor_form": tensor_form, "batched": batched, "wide": wide, "range_finder": range_finder, "adjoint": adjoint,
        "project": project,
        "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks.summary(), "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_only(args):
    """One kernel of the step on the workload, for profiling: `warmup` launches,
    then `steps` launches inside the NVTX range 'only', timed with events."""
    import torch

    import __graft_entry__
    fb = __graft_entry__.load()
    device = torch.device("cuda", 0)
    torch.cuda.set_device(device)
    N, k = args.N, args.k
    backend = fb.B200Backend(0)
    if args.only == "laplace":
        return run_only_laplace(args, fb, backend, torch, device)
    if args.only == "batch":
        return run_only_batch(args, fb, backend, torch, device)
    if args.only in ("cholqr2_adjoint", "project_adjoint", "hband", "adjoint_step"):
        return run_only_adjoint(args, fb, backend, torch, device)
    Yt = build_workload(fb, backend, torch, device, N, k, seed=0xDEADBEEF)
    Y = wrap(fb, Yt, N, k)
    # The first pass's factor: the Cholesky factor of Y^H Y (Y is Yt^T).
    G = torch.conj(Yt) @ Yt.t()
    R1 = backend.todevice(np.asfortranarray(torch.linalg.cholesky(G).conj().t().cpu().numpy()))
    Rid = backend.todevice(np.asfortranarray(np.eye(k, dtype=np.complex128)))
    Gd = backend.alloc_device(np.complex128, (k, k))
    torch.cuda.synchronize()
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    launch = {
        "gram": lambda: fb.kernels.gram_accumulate(backend, Gd, Y, Y, 1.0, 0.0),
        "gram_tc": lambda: fb.kernels.gram_tc(backend, Gd, Y, 1.0, 0.0),
        "trsm_blocked": lambda: fb.kernels.rdiv_upper(backend, Y, R1),
        "trsm_inverse": lambda: fb.kernels.rdiv_upper(backend, Y, Rid),
        "ghost_fill": lambda: fb.kernels.ghost_fill(backend, Y, 0, 0, 0xDEADBEEF, np.complex128),
        "cholqr2": lambda: fb.kernels.cholqr2_resident(backend, Y, Gd, wait=False),
    }[args.only]
    for _ in range(args.warmup):
        backend.submit(queue, launch)
    backend.sync_queue(queue)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("only")
    a.record(stream)
    for _ in range(args.steps):
        backend.submit(queue, launch)
    b.record(stream)
    torch.cuda.nvtx.range_pop()
    b.synchronize()
    print(json.dumps({"only": args.only, "N": N, "k": k, "steps": args.steps,
                      "ms_per_launch": a.elapsed_time(b) / args.steps}), flush=True)
    return 0


def run_only_adjoint(args, fb, backend, torch, device):
    """The differentiation kernels on N = args.N rows, k = args.k, inputs
    filled by the ghost generator: `cholqr2_adjoint` (cross Gram, prep, fused
    product), `project_adjoint` (Hermitian G), `hband` (G Q with kd = 64), or
    `adjoint_step` (the whole forward pass and both pullbacks of the
    differentiation workload)."""
    N, k, kd = args.N, args.k, 64
    alloc = lambda r, c: backend.alloc_device(np.complex128, (r, c))
    Y, Qbar, GQ, Q = alloc(N, k), alloc(N, k), alloc(N, k), alloc(N, k)
    R, S = alloc(k, k), alloc(k, k)
    fb.kernels.ghost_fill(backend, Y, 0, 0, 0xC5, np.complex128)
    fb.kernels.ghost_fill(backend, Qbar, 0, 0, 0xC6, np.complex128)
    fb.device_api.copy_region(Q, Y, None)
    fb.kernels.cholqr2_resident(backend, Q, R)
    G = fb.HermitianBand.ghost(backend, N, kd, seed=0xC7, scale=float(np.sqrt(N / ((2 * kd + 1) * k))))
    G.apply(backend, GQ, Q)
    fb.kernels.gram_accumulate(backend, S, Q, GQ, 2.0, 0.0)
    backend.sync_all()
    Ybar = alloc(N, k)
    K = fb.kernels

    def step():
        fb.device_api.copy_region(Q, Y, queue)
        K.cholqr2_resident(backend, Q, R, wait=False)
        G.apply(backend, GQ, Q)
        K.gram_accumulate(backend, S, Q, GQ, 2.0, 0.0)
        fb.device_api.copy_region(Ybar, Qbar, queue)
        K.project_adjoint(backend, Ybar, GQ, S, None, accumulate=True)
        K.cholqr2_adjoint(backend, Ybar, Y, R, Ybar, None)

    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    launch = {
        "cholqr2_adjoint": lambda: K.cholqr2_adjoint(backend, Ybar, Y, R, Qbar, None),
        "project_adjoint": lambda: K.project_adjoint(backend, Ybar, GQ, S, None, accumulate=True),
        "hband": lambda: G.apply(backend, GQ, Q),
        "adjoint_step": step,
    }[args.only]
    for _ in range(args.warmup):
        backend.submit(queue, launch)
    backend.sync_queue(queue)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("only")
    a.record(stream)
    for _ in range(args.steps):
        backend.submit(queue, launch)
    b.record(stream)
    torch.cuda.nvtx.range_pop()
    b.synchronize()
    print(json.dumps({"only": args.only, "N": N, "k": k, "kd": kd, "steps": args.steps,
                      "ms_per_launch": a.elapsed_time(b) / args.steps}), flush=True)
    return 0


def run_only_batch(args, fb, backend, torch, device):
    """The persistent batch kernel on args.batch instances drawn as the bench's
    batch section draws them (N log-uniform on [1e4, 2e6], k from {16, 32, 64},
    the same seed): one launch per step."""
    rng = np.random.default_rng(0xBA7C4)
    Ns = np.exp(rng.uniform(np.log(1e4), np.log(2e6), args.batch)).astype(np.int64)
    ks = rng.choice([16, 32, 64], args.batch)
    gen = torch.Generator(device=device)
    gen.manual_seed(0xBA7C4)
    tensors = [torch.randn((int(k), int(N)), dtype=torch.complex128, device=device, generator=gen)
               for N, k in zip(Ns, ks)]
    Ys = [wrap(fb, t, int(N), int(k)) for t, N, k in zip(tensors, Ns, ks)]
    Rs = [backend.alloc_device(np.complex128, (int(k), int(k))) for k in ks]
    shapes = [(int(N), int(k)) for N, k in zip(Ns, ks)]
    nbytes = fb.kernels.cholqr2_batched_workspace_bytes(shapes, schedule="persistent")
    buf = backend.alloc_device(np.complex128, (nbytes // 16 + 32, 1))
    ws = ((buf.ptr + 255) // 256 * 256, nbytes)
    torch.cuda.synchronize()
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    launch = lambda: fb.kernels.cholqr2_batched(backend, Ys, Rs, wait=False, workspace=ws, schedule="persistent")
    for _ in range(args.warmup):
        backend.submit(queue, launch)
    backend.sync_queue(queue)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("only")
    a.record(stream)
    for _ in range(args.steps):
        backend.submit(queue, launch)
    b.record(stream)
    torch.cuda.nvtx.range_pop()
    b.synchronize()
    ms = a.elapsed_time(b) / args.steps
    print(json.dumps({"only": "batch", "instances": args.batch, "bytes_on_device": int(sum(16 * N * k for N, k in shapes)),
                      "alg_bytes": float(sum(96.0 * N * k for N, k in shapes)), "ms_per_launch": ms}), flush=True)
    return 0


def run_only_laplace(args, fb, backend, torch, device):
    """The streamed range finder's operator, -Lap_7 + (0.5+0.1i) I on a 342^3
    grid (N = 40 001 688), applied to one panel of min(k, 16) columns: 32 bytes
    per entry of algorithmic traffic (read once, write once)."""
    grid = (342, 342, 342)
    n = grid[0] * grid[1] * grid[2]
    w = min(args.k, 16)
    gen = torch.Generator(device=device)
    gen.manual_seed(0xDEADBEEF)
    Xt = torch.randn((w, n), dtype=torch.complex128, device=device, generator=gen)
    Yt = torch.empty_like(Xt)
    torch.cuda.synchronize()
    X, Y = wrap(fb, Xt, n, w), wrap(fb, Yt, n, w)
    G = fb.Laplacian7(grid, 0.5 + 0.1j)
    queue = backend.make_queue()
    stream = torch.cuda.ExternalStream(queue.handle, device=device)
    for _ in range(args.warmup):
        backend.submit(queue, lambda: G.apply(backend, Y, X))
    backend.sync_queue(queue)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("only")
    a.record(stream)
    for _ in range(args.steps):
        backend.submit(queue, lambda: G.apply(backend, Y, X))
    b.record(stream)
    torch.cuda.nvtx.range_pop()
    b.synchronize()
    ms = a.elapsed_time(b) / args.steps
    print(json.dumps({"only": "laplace", "grid": grid, "N": n, "cols": w, "steps": args.steps, "ms_per_launch": ms,
                      "gbs": 32 * n * w / (ms * 1e-3) / 1e9}), flush=True)
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.only is not None:
        return run_only(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
