#!/usr/bin/env python3
"""Benchmark: detected symbols/s of APSM training + detection on one B200.

Workload (one "step" = one frame): 16QAM, K = 8 users, N = 16 antennas,
P = 1000 pilots, S = 8000 data symbols, window 80, dictionary 1000 entries,
FP32; every user is trained on the frame's pilots from a fresh state and then
detects the frame's data.  Metric: detected symbols/s = users x S / frame time.
Seeded synthetic frames (Rayleigh channel, Rapp PA, AWGN at 20 dB); the
reference publishes no dataset for this path.

  value   device-resident inputs: train + detect kernels only
  e2e     the public C ABI with host buffers (apsm_train / apsm_detect):
          H2D of the frame and D2H of the estimates inside the timed region

``--impl reference`` times the reference algorithm on the host CPU cores
(the reference has no CPU implementation of APSM, so this is the repository's
FP32 C restatement of it, OpenMP over all host threads) on a bounded sample of
the same workload, plus the reference's own CUDA library on this GPU when it
was built (``reference_cuda``).

With torchrun (N > 1) every rank runs an independent replica (detectors do
not shard and need no collective); value = all ranks' symbols / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "detected symbols/s (APSM train + detect per frame, all users)"
UNIT = "symbols/s"
WORKLOAD = {"workload": "16QAM K=8 users N=16 P=1000 S=8000 window=80 dictionary=1000 FP32 train+detect per frame",
            "users": 8, "antennas": 16, "pilots": 1000, "data_symbols": 8000, "window": 80, "dictionary": 1000,
            "snr_db": 20, "l2": "flushed between timed steps (256 MiB write)"}


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons)}


# ---------------------------------------------------------------- B200 arm --
def algorithmic_sweep_bytes(users: int, P: int, D: int) -> int:
    """Minimum HBM bytes of one training sweep launch: the pilot rows (2P x D),
    their norms, each user's targets and coefficients (read + write) and
    linear weights."""
    rows = 2 * P
    return 4 * (rows * D + rows + users * (rows + 2 * rows + 2 * D))


def run_b200(args, rank: int, world: int) -> dict | None:
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    frame = synth.config1_frame(seed=1 + rank)
    cfg = dict(synth.CONFIG1_ALGORITHM)
    if args.detect_version:
        cfg["detectVersion"] = args.detect_version
    U, N = frame.tx_train.shape[0], frame.rx_train.shape[0]
    P, S = frame.rx_train.shape[1], frame.rx_data.shape[1]
    det = L.NomaDetectorFactory.build(cfg, N, num_users=U)
    stream = torch.cuda.ExternalStream(det.stream)
    rx = torch.from_numpy(frame.rx_train).cuda()
    tx = torch.from_numpy(frame.tx_train).cuda()
    rxd = torch.from_numpy(frame.rx_data).cuda()
    est = torch.empty((U, S), dtype=torch.complex64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # pack pilots, gather targets, kernel columns, sweep, pack data, detect
    # (+ operand packing x2, coefficients, reduction for the tensor-core detect)
    launches_per_step = 10 if cfg.get("detectVersion", "").startswith("gram") else 6

    def step():
        det.reset_state()
        det.train_device(rx, tx)
        det.detect_device(rxd, est)

    for _ in range(args.warmup):
        step()
    det.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sweep_ms, detect_ms = [], []
    clocks = ClockSampler(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[i][0].record(stream)
        step()
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
        s_ms, d_ms = det.last_kernel_ms()
        sweep_ms.append(s_ms)
        detect_ms.append(d_ms)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)

    # ---- e2e through the host C ABI (pinned host buffers, H2D/D2H inside) ----
    h_rx = torch.from_numpy(frame.rx_train).pin_memory()
    h_tx = torch.from_numpy(frame.tx_train).pin_memory()
    h_rxd = torch.from_numpy(frame.rx_data).pin_memory()
    h_est = torch.empty((U, S), dtype=torch.complex64).pin_memory()
    lib = det._lib
    import ctypes

    def e2e_step():
        det.reset_state()
        lib.apsm_train(det._h, h_rx.data_ptr(), h_tx.data_ptr(), P, None)
        lib.apsm_detect(det._h, h_rxd.data_ptr(), S, h_est.data_ptr(), None)

    for _ in range(args.warmup):
        e2e_step()
    ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev2[i][0].record(stream)
        e2e_step()
        with torch.cuda.stream(stream):
            ev2[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_ms = sum(a.elapsed_time(b) for a, b in ev2)
    est_ok = np.isfinite(h_est.numpy()).all()

    # ---- max over ranks ----
    t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    total_ms, e2e_ms = float(t[0]), float(t[1])
    if rank != 0:
        return None

    symbols = world * U * S
    ms_step = total_ms / args.steps
    sweep = float(np.median(sweep_ms))
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    alg_bytes = algorithmic_sweep_bytes(U, P, 2 * N)
    achieved = alg_bytes / (sweep * 1e-3) / 1e9
    ser = float(np.mean([L.symbol_error_rate(h_est.numpy()[u], frame.tx_data[u], frame.modulation)
                         for u in range(U)]))
    return {
        "metric": METRIC, "value": symbols / (ms_step * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded NOMA frames; no public dataset)",
        "config": dict(WORKLOAD, parallelism=f"replicas x{world}", detect_version=cfg.get("detectVersion", "balanced")),
        "e2e": {"value": symbols / (e2e_ms / args.steps * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": int(h_rx.numel() * 8 + h_tx.numel() * 8 + h_rxd.numel() * 8),
                "d2h_bytes_per_step": int(h_est.numel() * 8), "ms_per_step": e2e_ms / args.steps},
        "gpu_launches": launches_per_step * args.steps,
        "roofline": {"bound": "hbm", "kernel": "train_exact_kernel (training sweep)", "achieved": achieved,
                     "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
                     # dram read + write of one sweep launch on this workload, ncu
                     # (profiles/train_sweep_kernel_config1_frame.md): the kernel columns
                     "traffic": 9772544,
                     "algorithmic_bytes_per_launch": alg_bytes, "launch_ms": sweep,
                     "note": "sweep is a chain of P dependent steps; latency-bound, see DESIGN.md",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        "stage_ms": {"sweep": sweep, "detect": float(np.median(detect_ms))},
        "ser_mean": ser, "estimates_finite": bool(est_ok),
        "clocks": clk,
    }


# ----------------------------------------------------------- reference arm --
def cpu_baseline(sample_users: int = 1) -> dict:
    """The FP32 restatement of the reference algorithm on the host cores,
    on a bounded sample of the workload (sample_users of the frame's users)."""
    from libapsm_b200 import synth
    from oracle import oracle as O

    threads = O.set_threads(os.cpu_count() or 1)
    frame = synth.config1_frame(seed=1)
    cfg = dict(synth.CONFIG1_ALGORITHM)
    S = frame.rx_data.shape[1]
    t0 = time.perf_counter()
    for u in range(sample_users):
        d = O.OracleDetector(cfg, frame.rx_train.shape[0], O.F32)
        d.train(frame.rx_train, frame.tx_train[u])
        d.detect(frame.rx_data)
    dt = time.perf_counter() - t0
    return {"value": sample_users * S / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{sample_users} of 8 users of one frame (train 1000 pilots + detect 8000 symbols each), "
                      f"{dt:.2f} s"}


def reference_cuda(warmup: int, steps: int) -> dict | None:
    """The reference library (built from its sources for sm_100a) on this GPU,
    as its CLI's -p mode runs it: one detector and host thread per user."""
    from libapsm_b200 import synth
    from oracle import oracle as O

    if not O.reference_available():
        return None
    try:
        import torch

        if not torch.cuda.is_available():
            return None
    except Exception:
        return None
    frame = synth.config1_frame(seed=1)
    cfg = dict(synth.CONFIG1_ALGORITHM)
    U, S = frame.tx_train.shape[0], frame.rx_data.shape[1]
    for _ in range(warmup):
        O.reference_users_threaded(cfg, frame.rx_train, frame.tx_train, frame.rx_data)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.reference_users_threaded(cfg, frame.rx_train, frame.tx_train, frame.rx_data)
    dt = (time.perf_counter() - t0) / steps
    return {"value": U * S / dt, "unit": UNIT, "ms_per_step": dt * 1e3,
            "what": "reference CUDA kernels (libapsm built for sm_100a), 8 detectors on 8 host threads, wall clock"}


def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    base = cpu_baseline()
    line = {
        "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": WORKLOAD["users"] * WORKLOAD["data_symbols"] / base["value"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded NOMA frames; no public dataset)", "config": dict(WORKLOAD),
        "impl": "reference", "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    rc = reference_cuda(min(args.warmup, 1), min(args.steps, 3))
    if rc is not None:
        line["reference_cuda"] = rc
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--detect-version", default=None,
                    help="detectVersion of the algorithm config (default: the reference's 'balanced')")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
        if line is not None:
            print(json.dumps(line), flush=True)
        return

    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    line = run_b200(args, rank, world)
    if line is not None and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
