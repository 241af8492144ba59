#!/usr/bin/env python3
"""Benchmark: detected symbols/s of batched APSM detection on one B200, with
the plain per-detector form and the served (per-TTI request) form beside it.

Headline workload (one "step" = one batch): 512 independent detectors (users
x cells), antennas uniform over {4, 8, 16, 32}, pilots over [200, 2000], data
symbols over [1000, 16000], SNR over [10, 25] dB, QPSK or 16QAM, Rapp PA;
window 80, dictionary 2000 entries, the reference's defaults otherwise.  Each
detector is trained from a fresh state on its pilots and detects its data:
all of it one detector-pool batch (one persistent training launch, tensor-core
detection in TF32 hi/lo form, FP32-accurate).  Seeded synthetic frames
(Rayleigh channel, Rapp PA, AWGN); the reference publishes no dataset.

  value    device-resident inputs: the batch's kernels (CUDA events on its stream)
  e2e      the public C ABI with host buffers (apsm_pool_run, APSM_RUN_HOST) in
           page-locked memory: host-to-device copies, kernels, device-to-host copies
  plain    the per-detector form (NomaDetector per user, the reference's API)
           on one 8-user 16QAM frame (N=16, 1000 pilots, 8000 symbols)
  serving  Poisson per-TTI requests (train-append 16-64 pilots / detect
           500-4000 symbols) against 512 resident detectors through the
           request server: p50 / p99 latency and detected symbols/s
  precision  large detection (N=64, dictionary 8192, 16 users, 65536
           symbols) in the exact form and every tensor-core form: time,
           symbols/s, soft-output and decision error against a float64
           evaluation of the same trained model, SER

``--impl reference`` times the reference algorithm on the host cores (the
reference has no CPU implementation of APSM: this is the repository's FP32 C
restatement of it, OpenMP over all host threads) on a bounded sample of the
same workload, plus the reference's own CUDA library on this GPU when it was
built (``reference_cuda``, one NomaDetector per detector as its API runs).

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

METRIC = "detected symbols/s (batched APSM train + detect, 512 heterogeneous detectors)"
UNIT = "symbols/s"
N_DET = 512
# DRAM bytes per algorithmic byte of the batched sweep (ncu capture of the first
# 32 detectors: 367.8 MB read + 4.6 MB written for 361.3 MB algorithmic)
SWEEP_TRAFFIC_PER_ALG_BYTE = (368.360704 + 4.627968) / 361.273728
WORKLOAD = {"workload": "512 detectors: N~U{4,8,16,32}, P~U[200,2000], S~U[1000,16000], SNR~U[10,25] dB, "
                        "QPSK/16QAM, window 80, dictionary 2000, fresh train + detect per step",
            "detectors": N_DET, "window": 80, "dictionary": 2000, "detect": "gram_tf32x3 (FP32-accurate)",
            "l2": "inputs 0.6 GB (> L2) and a 256 MiB write between timed steps"}


# ------------------------------------------------------------------ clocks --
class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML read
    every 10 ms from a thread (the device found by its UUID), else nvidia-smi
    every 100 ms.  Only reads; nothing is set."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.nvml = None
        self.lines: list[str] = []
        self.samples: list[tuple[float, int]] = []  # (SM MHz, reason bits) from NVML
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.index)
        try:
            u = str(props.uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
        except Exception:
            bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.nvml = (nv, h, nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _poll(self):
        nv, h, _ = self.nvml
        while not self.stop_flag.is_set():
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     int(nv.nvmlDeviceGetCurrentClocksThrottleReasons(h))))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.nvml is not None:
            self.stop_flag.set()
            self.t.join(timeout=5)
            nv, _, mx = self.nvml
            bits = [nv.nvmlClocksThrottleReasonHwSlowdown, nv.nvmlClocksThrottleReasonHwThermalSlowdown,
                    nv.nvmlClocksThrottleReasonSwThermalSlowdown, nv.nvmlClocksThrottleReasonSwPowerCap]
            reasons = {n for n, b in zip(self.NAMES, bits) if any(r & b for _, r in self.samples)}
            sm = [c for c, _ in self.samples]
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": float(mx), "samples": len(sm),
                    "reasons": sorted(reasons), "source": "NVML, every 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "samples": len(sm),
                "reasons": sorted(reasons), "source": "nvidia-smi, every 100 ms"}


# ------------------------------------------------------------- replicas --
def replica_totals(symbols: int, total_ms: float, e2e_ms: float, world: int, device="cpu"):
    """Whole-job totals of independent replicas: detected symbols summed over
    the ranks, timed milliseconds as the maximum over the ranks.  Every rank
    calls this (a collective when world > 1)."""
    if world <= 1:
        return symbols, total_ms, e2e_ms
    import torch

    s = torch.tensor([float(symbols)], dtype=torch.float64, device=device)
    t = torch.tensor([total_ms, e2e_ms], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(s, op=torch.distributed.ReduceOp.SUM)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return int(s.item()), float(t[0]), float(t[1])


# ------------------------------------------------------- batched (headline) --
def sweep_algorithmic_bytes(dets, window: int, dict_size: int) -> int:
    """Minimum HBM bytes of one batched training-sweep launch: every kernel-
    column entry it combines (16 B, each read once: pair n against the pairs
    before it), the pilots (8N B per complex sample), targets and
    coefficients (read + write) of every job."""
    total = 0
    for d in dets:
        nP, capP = d.P, dict_size
        cols = sum(min(n, capP) for n in range(nP))
        total += 16 * cols + 8 * d.N * nP + 4 * (2 * nP) * 3
    return total


def sweep_column_entries(dets, dict_size: int) -> int:
    """Kernel-column entries of a batch (pair n against the min(n, capacity)
    pairs before it): each is written once by the column launch and read
    once by the sweep, 16 bytes each way."""
    return sum(sum(min(n, dict_size) for n in range(d.P)) for d in dets)


def latency_roofline(pool, L, dets, ids, dev_in, sweep_ms: float, slots: int, sm_mhz: float | None) -> dict:
    """Step-latency bound of the batched training sweep.  Every job is a chain
    of P dependent steps (one complex pilot enters per step, sampleStep 2); the
    launch runs `slots` chains at once (CTAs per SM x SMs).  The per-step
    latency of a chain running alone on the idle GPU (the longest job, one
    CTA) is measured here; from it follow the longest chain's floor and the
    throughput floor of all steps spread over the slots."""
    k = max(range(len(dets)), key=lambda i: dets[i].P)
    job = pool.prepare([L.PoolJob(ids[k], dev_in[k][0], dev_in[k][1], fresh=True)], device=True)
    alone = []
    for _ in range(4):
        pool.run_prepared(job, mode=1)
        pool.wait()
        alone.append(pool.last_sweep_ms())
    alone_ms = min(alone[1:])
    steps_longest = dets[k].P
    step_us = alone_ms * 1e3 / steps_longest
    total_steps = sum(d.P for d in dets)
    floor_ms = max(steps_longest * step_us, total_steps * step_us / slots) * 1e-3
    out = {"kernel": "batch_sweep_kernel", "sweep_ms": sweep_ms, "steps_total": total_steps,
           "longest_chain_steps": steps_longest, "slots": slots, "step_us_alone": step_us,
           "chain_floor_ms": steps_longest * step_us * 1e-3,
           "throughput_floor_ms": total_steps * step_us / slots * 1e-3,
           "floor_ms": floor_ms, "frac": floor_ms / sweep_ms,
           "step_us_in_batch": sweep_ms * 1e3 * slots / total_steps,
           "note": "floor = max(longest chain, all steps / slots) at the step latency of a chain running alone; "
                   "frac < 1 is what sharing an SM between chains costs"}
    if sm_mhz:
        out["cycles_per_step_alone"] = step_us * sm_mhz
        out["cycles_per_step_in_batch"] = out["step_us_in_batch"] * sm_mhz
    return out


def sfu_roofline(dets, dict_size: int, detect_ms: float, sms: int, sm_mhz: float | None) -> dict:
    """Exponential-unit bound of the batch's detection: per (data symbol,
    dictionary pair) the pair form needs 3 exponentials (one ex2.approx each);
    the denominator is the SFU rate measured on this device by
    apsm_measure_ex2_rate (a kernel of nothing but independent ex2 chains),
    with the nominal 16 per clock per SM beside it.  The stage time includes
    the operand packing."""
    import ctypes

    from libapsm_b200 import _native

    pairs = sum(d.S * min(d.P, dict_size) for d in dets)
    mhz = sm_mhz or 1965.0
    nominal = sms * 16 * mhz * 1e6
    rate, ms = ctypes.c_double(0.0), ctypes.c_float(0.0)
    measured = None
    if _native.load().apsm_measure_ex2_rate(ctypes.byref(rate), ctypes.byref(ms)) == 0 and rate.value > 0:
        measured = rate.value
    peak = measured or nominal
    floor_ms = 3.0 * pairs / peak * 1e3
    return {"kernel": "batch_gram_kernel + operand packing (detection stage)", "pair_evaluations": pairs,
            "exponentials": 3 * pairs, "floor_ms": floor_ms, "stage_ms": detect_ms, "frac": floor_ms / detect_ms,
            "peak_ex2_per_s": peak, "peak_source": "measured (apsm_measure_ex2_rate)" if measured else "nominal",
            "measured_ex2_per_clk_per_sm": (measured / (sms * mhz * 1e6)) if measured else None,
            "nominal_ex2_per_s": nominal, "clock_mhz": mhz}


batched_est_host: list = []  # the last batched run's estimates (rank 0), for the CPU sample's SER


def run_batched(args, rank: int, world: int) -> dict | None:
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    dets = synth.config2_detectors(args.detectors, seed=2 + rank)
    cfg = dict(synth.CONFIG2_ALGORITHM, detectVersion="gram_tf32x3")
    pool = L.DetectorPool(cfg)
    ids = [pool.add(d.N) for d in dets]
    stream = torch.cuda.ExternalStream(pool.stream(0))
    dev_in = [(torch.from_numpy(d.rx_train).cuda(), torch.from_numpy(d.tx_train).cuda(),
               torch.from_numpy(d.rx_data).cuda(), torch.empty(d.S, dtype=torch.complex64, device="cuda"))
              for d in dets]
    jobs = pool.prepare([L.PoolJob(i, x[0], x[1], fresh=True) for i, x in zip(ids, dev_in)] +
                        [L.PoolJob(i, x[2], est=x[3]) for i, x in zip(ids, dev_in)], device=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    for _ in range(args.warmup):
        pool.run_prepared(jobs, mode=1)
    pool.wait()
    # launch shapes chosen by the pool's autotuner on this batch (untimed; changes no result)
    if args.no_autotune:
        shape = {"sweep_ctas_per_sm": 0, "gram_stages": 0, "detect_blocks_per_sm": 0}
    else:
        tuned = pool.autotune(jobs, mode=1)
        shape = {k: tuned[k] for k in ("sweep_ctas_per_sm", "gram_stages", "detect_blocks_per_sm")}

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage = {"train": [], "sweep": [], "detect": []}
    launches = 0
    clocks = ClockSampler(dev)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for i in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            ev[i][0].record(stream)
        pool.run_prepared(jobs, mode=1)
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
        pool.wait()
        t_ms, d_ms = pool.last_ms()
        stage["train"].append(t_ms)
        stage["detect"].append(d_ms)
        stage["sweep"].append(pool.last_sweep_ms())
        launches += pool.last_launches()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clk = clocks.stop()
    total_ms = sum(a.elapsed_time(b) for a, b in ev)

    # SER of the estimates (hard decisions of the reference's Gray map)
    est_batched = [x[3].cpu().numpy() for x in dev_in]
    sers = [L.symbol_error_rate(e, d.tx_data, d.modulation) for d, e in zip(dets, est_batched)]
    sweep = float(np.median(stage["sweep"]))
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    slots = sms * (shape["sweep_ctas_per_sm"] or 2)
    lat = latency_roofline(pool, L, dets, ids, dev_in, sweep, slots, clk.get("sm_mhz"))

    # ---- e2e: host buffers through the C ABI (staging + copies inside) ----
    pinned = []  # page-locked host copies of the frames (the e2e inputs and outputs)

    def pin(a):
        t_ = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        pinned.append(t_)
        return t_.numpy()

    host_jobs = ([L.PoolJob(i, pin(d.rx_train), pin(d.tx_train), fresh=True) for i, d in zip(ids, dets)] +
                 [L.PoolJob(i, pin(d.rx_data), est=pin(np.zeros(d.S, np.complex64))) for i, d in zip(ids, dets)])
    prepared = pool.prepare(host_jobs)
    for _ in range(args.warmup):
        pool.run_prepared(prepared)
    if world > 1:
        torch.distributed.barrier()
    e2e_ms = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pool.run_prepared(prepared)  # apsm_pool_run, APSM_RUN_HOST
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    h2d = sum(d.rx_train.nbytes + d.tx_train.nbytes + d.rx_data.nbytes for d in dets)
    d2h = sum(8 * d.S for d in dets)

    # ---- e2e with pageable host buffers (ordinary numpy arrays, as the reference's std::vector) ----
    page_jobs = ([L.PoolJob(i, np.ascontiguousarray(d.rx_train), np.ascontiguousarray(d.tx_train), fresh=True)
                  for i, d in zip(ids, dets)] +
                 [L.PoolJob(i, np.ascontiguousarray(d.rx_data), est=np.zeros(d.S, np.complex64))
                  for i, d in zip(ids, dets)])
    prepared_pg = pool.prepare(page_jobs)
    for _ in range(2):
        pool.run_prepared(prepared_pg)
    pg_ms = []
    for _ in range(max(2, args.steps // 2)):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pool.run_prepared(prepared_pg)
        pg_ms.append((time.perf_counter() - t0) * 1e3)

    symbols, total_ms, e2e_total = replica_totals(sum(d.S for d in dets), total_ms, sum(e2e_ms), world, "cuda")
    if rank != 0:
        return None

    ms_step = total_ms / args.steps
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak_gbs = float(peaks.get("hbm_gbs", 6650.0))
    alg = sweep_algorithmic_bytes(dets, 80, 2000)
    achieved = alg / (sweep * 1e-3) / 1e9
    col_entries = sweep_column_entries(dets, 2000)
    pilots = sum(d.P for d in dets)
    plain_same = run_plain_same(dets, dev_in, est_batched) if not args.no_extras else None
    batched_est_host[:] = est_batched
    return {
        "metric": METRIC, "value": symbols / (ms_step * 1e-3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded NOMA frames; no public dataset)",
        "config": dict(WORKLOAD, parallelism=f"replicas x{world}", detectors=len(dets),
                       launch_shape=dict(shape, chosen_by="built-in (0 = built-in choice)" if args.no_autotune
                                         else "apsm_pool_autotune")),
        "e2e": {"value": symbols / (e2e_total / args.steps * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_total / args.steps,
                "host_buffers": "page-locked"},
        "e2e_pageable": {"value": symbols / (float(np.median(pg_ms)) * 1e-3), "unit": UNIT,
                         "ms_per_step": float(np.median(pg_ms)), "h2d_bytes_per_step": int(h2d),
                         "d2h_bytes_per_step": int(d2h),
                         "host_buffers": "pageable numpy arrays (staged by the pool's helper threads)"},
        "training_samples_per_s": pilots / (ms_step * 1e-3),
        "training_samples_per_s_train_stage": pilots / (float(np.median(stage["train"])) * 1e-3),
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": "batch_sweep_kernel (training sweep, all 512 jobs)",
                     "achieved": achieved, "peak": peak_gbs, "unit": "GB/s", "frac": achieved / peak_gbs,
                     "traffic": alg * SWEEP_TRAFFIC_PER_ALG_BYTE, "algorithmic_bytes_per_launch": alg,
                     "launch_ms": sweep,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture of the "
                                       "32-detector case (373.0 MB for 361.3 MB algorithmic), scaled to this "
                                       "launch by its algorithmic bytes",
                     "note": "a chain of P dependent steps per detector: bound by step latency (see "
                             "roofline_latency), not HBM; see profiles/",
                     "self_inflicted_bytes": {"kernel_columns_written": 16 * col_entries,
                                              "kernel_columns_read_by_sweep": 16 * col_entries,
                                              "what": "the column launch writes every (pair, earlier pair) "
                                                      "kernel value once and the sweep reads it back: traffic "
                                                      "of the precomputed-column design, not of the algorithm's "
                                                      "inputs"},
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
        "roofline_latency": lat,
        "roofline_sfu": sfu_roofline(dets, 2000, float(np.median(stage["detect"])), sms, clk.get("sm_mhz")),
        "stage_ms": {k: float(np.median(v)) for k, v in stage.items()},
        "ser_mean": float(np.mean(sers)), "clocks": clk,
        "plain_same_workload": plain_same,
    }


# -------------------------------------------------- plain per-detector form --
def run_plain(steps: int = 5, warmup: int = 3, detect_version: str = "balanced", compare: bool = True) -> dict:
    """The reference's per-detector API (NomaDetector per user) on one
    config-1 frame: 8 users, N=16, 1000 pilots, 8000 symbols, FP32 (or the
    detection form `detect_version`); with `compare`, the LLS baselines and
    the reference library's own kernels on the same frame."""
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    frame = synth.config1_frame(seed=1)
    cfg = dict(synth.CONFIG1_ALGORITHM, detectVersion=detect_version)
    U, N = frame.tx_train.shape[0], frame.rx_train.shape[0]
    S = frame.rx_data.shape[1]
    det = L.NomaDetectorFactory.build(cfg, N, num_users=U)
    stream = torch.cuda.ExternalStream(det.stream)
    rx, tx, rxd = (torch.from_numpy(a).cuda() for a in (frame.rx_train, frame.tx_train, frame.rx_data))
    est = torch.empty((U, S), dtype=torch.complex64, device="cuda")

    def step():
        det.reset_state()
        det.train_device(rx, tx)
        det.detect_device(rxd, est)

    for _ in range(warmup):
        step()
    det.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for i in range(steps):
        with torch.cuda.stream(stream):
            ev[i][0].record(stream)
        step()
        with torch.cuda.stream(stream):
            ev[i][1].record(stream)
    torch.cuda.synchronize()
    ms = sum(a.elapsed_time(b) for a, b in ev) / steps
    mod = frame.modulation

    def ser(est_users):
        return float(np.mean([L.symbol_error_rate(est_users[u], frame.tx_data[u], mod) for u in range(U)]))

    out = {"value": U * S / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "ser": ser(est.cpu().numpy()),
           "detect": detect_version,
           "workload": "16QAM K=8 users N=16 P=1000 S=8000 window=80 dictionary=1000, NomaDetector per user "
                       "(exact FP32 sweep + BALANCED-order detect), all 8 users"}
    if not compare:
        det.close()
        return out

    # LLS linear baseline on our own kernels (FP64 normal equations + Cholesky), same frame
    lls = L.NomaDetectorFactory.build({"otype": "LLS"}, N, num_users=U)
    lls.train(frame.rx_train, frame.tx_train)
    lls.detect(frame.rx_data)
    t0 = time.perf_counter()
    lls.train(frame.rx_train, frame.tx_train)
    e_lls, _ = lls.detect(frame.rx_data)
    out["lls"] = {"ser": ser(e_lls.reshape(U, S)), "ms_wall": (time.perf_counter() - t0) * 1e3,
                  "what": "LLS detector on this library's kernels, host buffers, train + detect of all 8 users"}
    lls.close()
    det.close()
    out["reference_cuda"] = reference_cuda_config1(frame, dict(synth.CONFIG1_ALGORITHM))
    return out


def reference_cuda_config1(frame, cfg) -> dict | None:
    """The reference library itself (built from its sources for sm_100a) on the
    same config-1 frame: one NomaDetector per user, as its CLI runs them, with
    the reference's own CUDA-event times (train / detect, noma_detect.cpp:136-138)
    and its cuBLAS LLS baseline (lls_detector.cu:175,217)."""
    import libapsm_b200 as L
    from oracle import oracle as O

    if not O.reference_available():
        return None
    U, N = frame.tx_train.shape[0], frame.rx_train.shape[0]
    mod = frame.modulation
    r = O.ReferenceDetector(cfg, N)  # warm-up (context, module load)
    r.train(frame.rx_train[:, :64], frame.tx_train[0, :64])
    del r
    train_ms = detect_ms = 0.0
    sers = []
    t0 = time.perf_counter()
    for u in range(U):
        r = O.ReferenceDetector(cfg, N)
        train_ms += r.train(frame.rx_train, frame.tx_train[u])
        e, dms = r.detect(frame.rx_data)
        detect_ms += dms
        sers.append(L.symbol_error_rate(e, frame.tx_data[u], mod))
        del r
    wall = time.perf_counter() - t0
    S = frame.rx_data.shape[1]
    out = {"train_ms": train_ms, "detect_ms": detect_ms, "wall_ms": wall * 1e3, "ser": float(np.mean(sers)),
           "value_events": U * S / ((train_ms + detect_ms) * 1e-3), "value_wall": U * S / wall, "unit": UNIT,
           "what": "reference NomaDetector per user (8 users, one after the other); train/detect ms are its own "
                   "CUDA-event times summed over the users"}
    lls_ms, lls_sers = 0.0, []
    for u in range(U):
        r = O.ReferenceDetector({"otype": "LLS"}, N)
        lls_ms += r.train(frame.rx_train, frame.tx_train[u])
        e, dms = r.detect(frame.rx_data)
        lls_ms += dms
        lls_sers.append(L.symbol_error_rate(e, frame.tx_data[u], mod))
        del r
    out["lls"] = {"ser": float(np.mean(lls_sers)), "ms_events": lls_ms,
                  "what": "reference cuBLAS LLS detector (Sgels train, Sgemm detect), 8 users, its own event times"}
    return out


def run_plain_same(dets, dev_in, est_batched) -> dict:
    """The plain per-detector FP32 form on the batched workload itself: one
    NomaDetector (the reference's API) per detector, fresh train + detect of
    the same 512 frames, device-resident inputs, one detector after the
    other (the reference's calls return when their GPU work is done).  SER of
    both forms on the same frames."""
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    cfg = dict(synth.CONFIG2_ALGORITHM)
    handles = {N: L.NomaDetectorFactory.build(cfg, N) for N in sorted({d.N for d in dets})}
    outs = [torch.empty(d.S, dtype=torch.complex64, device="cuda") for d in dets]

    def one(i):
        h = handles[dets[i].N]
        h.reset_state()
        h.train_device(dev_in[i][0], dev_in[i][1])
        h.detect_device(dev_in[i][2], outs[i])
        h.synchronize()

    for i in range(4):  # warm-up (workspaces of each antenna count)
        one(i)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(len(dets)):
        one(i)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    symbols = sum(d.S for d in dets)
    err_p = err_b = diff = 0
    for d, o, eb in zip(dets, outs, est_batched):
        ep = o.cpu().numpy()
        true = d.modulation.hard_decode_int(d.tx_data)
        dp, db = d.modulation.hard_decode_int(ep), d.modulation.hard_decode_int(eb)
        err_p += int(np.sum(dp != true))
        err_b += int(np.sum(db != true))
        diff += int(np.sum(dp != db))
    for h in handles.values():
        h.close()
    ser_p, ser_b = err_p / symbols, err_b / symbols
    return {"value": symbols / secs, "unit": UNIT, "seconds": secs, "ser_plain": ser_p, "ser_batched": ser_b,
            "ser_rel_diff": abs(ser_b - ser_p) / ser_p if ser_p else 0.0, "decisions_differing": diff,
            "symbols": symbols,
            "what": "NomaDetector per detector (exact FP32 sweep + BALANCED-order detect), the 512 frames of the "
                    "batched workload one after the other, device-resident inputs, wall clock with the GPU "
                    "synchronised per detector"}


# ------------------------------------------------- large-detect precision --
PRECISION_FORMS = ("balanced", "gram_tf32x3", "gram_tf32", "gram_bf16x3", "gram_bf16")


def model_fp64(state: dict, variance: float, wL: float, wG: float, rx: np.ndarray) -> np.ndarray:
    """Soft outputs of a trained model (float32 state) evaluated in float64:
    est_u(s) = f_u(x_2s) + i f_u(x_2s+1) with the Dedup rows x_2s = [Re; Im],
    x_2s+1 = [Im; -Re] and f_u(x) = wL <w_u, x> + wG sum_b a_ub exp(-||d_b - x||^2 / (2 variance))."""
    d = state["dictionary"].astype(np.float64)
    a = state["a"].astype(np.float64)
    w = state["w"].astype(np.float64)
    re, im = rx.real.astype(np.float64).T, rx.imag.astype(np.float64).T
    out = np.empty((a.shape[0], rx.shape[1]), dtype=np.complex128)
    dn = (d * d).sum(1)
    for part, x in enumerate((np.hstack([re, im]), np.hstack([im, -re]))):
        for s0 in range(0, x.shape[0], 512):
            xs = x[s0:s0 + 512]
            dist = np.maximum((xs * xs).sum(1)[:, None] + dn[None, :] - 2.0 * xs @ d.T, 0.0)
            f = wL * xs @ w.T + wG * np.exp(-0.5 / variance * dist) @ a.T  # (rows, users)
            if part == 0:
                out[:, s0:s0 + 512] = f.T
            else:
                out[:, s0:s0 + 512] += 1j * f.T
    return out


def run_precision_study(reps: int = 3, sample: int = 2048) -> dict:
    """Large detection in every precision: N=64 antennas (128 real features),
    16 16QAM users at 15 dB behind a Rapp PA (p=3), a dictionary of 8192
    entries filled by 8192 pilots (exact FP32 sweep, all users in one
    launch), 65536 data symbols detected by one trained model in each form
    (the model copied into one detector per form).  Two kernel widths: the
    config-0 width (gaussianKernelVariance 0.5, scaled by N^2: a wide kernel,
    the linear part dominates) and the reference's default 0.05 (exponents of
    a few units: the Gaussian part carries the model).  Soft outputs and decisions
    against a float64 evaluation of the same model on the first `sample`
    symbols; symbol error rates on all symbols."""
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    K, N, P, S = 16, 64, 8192, 65536
    f = synth.generate_frame(3, K=K, N=N, P=P, S=S, modulation="QAM16", snr_db=15.0, rapp_p=3.0)
    rx, tx, rxd = (torch.from_numpy(a).cuda() for a in (f.rx_train, f.tx_train, f.rx_data))
    est = torch.empty((K, S), dtype=torch.complex64, device="cuda")
    mod = f.modulation
    true_dec = mod.hard_decode_int(f.tx_data)
    models = []
    for label, variance in (("0.5 N^2", 0.5), ("0.05 N^2", 0.05)):
        cfg = dict(synth.CONFIG0_ALGORITHM, dictionarySize=8192, gaussianKernelVariance=variance)
        dets = {m: L.NomaDetectorFactory.build(dict(cfg, detectVersion=m), N, num_users=K) for m in PRECISION_FORMS}
        base = dets["balanced"]
        stream = torch.cuda.ExternalStream(base.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
        base.train_device(rx, tx)
        with torch.cuda.stream(stream):
            e1.record(stream)
        base.synchronize()
        train_ms = e0.elapsed_time(e1)
        state = base.get_state()
        ref = model_fp64(state, base.gaussian_variance, 0.5, 0.5, f.rx_data[:, :sample])
        ref_dec = mod.hard_decode_int(ref)
        forms = {}
        for m, det in dets.items():
            if det is not base:
                det.copy_state_from(base)
            st = torch.cuda.ExternalStream(det.stream)
            det.detect_device(rxd, est)  # warm-up (workspace allocation)
            det.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
            for a, b in ev:
                with torch.cuda.stream(st):
                    a.record(st)
                det.detect_device(rxd, est)
                with torch.cuda.stream(st):
                    b.record(st)
            det.synchronize()
            ms = statistics.median(a.elapsed_time(b) for a, b in ev)
            e = est.cpu().numpy()
            es = e[:, :sample].astype(np.complex128)
            err = np.abs(es - ref)
            forms[m] = {
                "detect_ms": round(ms, 3),
                "symbols_per_s": K * S / (ms * 1e-3),
                "soft_max_err_rel": float(err.max() / np.abs(ref).max()),
                "soft_rms_err_rel": float(np.sqrt(np.mean(err ** 2) / np.mean(np.abs(ref) ** 2))),
                "decisions_differing_from_fp64": float(np.mean(mod.hard_decode_int(es) != ref_dec)),
                "ser": float(np.mean(mod.hard_decode_int(e) != true_dec)),
            }
        models.append({"variance": label, "variance_value": base.gaussian_variance, "train_ms": round(train_ms, 3),
                       "ser_fp64_model": float(np.mean(ref_dec != true_dec[:, :sample])), "forms": forms})
        for det in dets.values():
            det.close()
    return {"workload": f"16QAM K={K} users N={N} P={P} S={S} 15 dB Rapp p=3, window 80, dictionary 8192, "
                        "one model per kernel width detected in each form",
            "fp64_sample_symbols": sample, "models": models}


# ------------------------------------------------------------ serving form --
def run_serving(rate_hz: float = 20000.0, duration_s: float = 0.3, n_det: int = N_DET, lanes: int = 8,
                max_batch: int = 16, detect_version: str = "balanced", deadline_s: float = 500e-6) -> dict:
    """Poisson per-TTI requests against resident detectors through the
    request server (continuous batching over `lanes` streams, at most
    `max_batch` requests of one kind per batch), detection in the FP32
    CUDA-core pair form ("balanced") or a tensor-core form ("gram_bf16" ...).
    Request samples sit in
    page-locked host buffers, as a radio front end's DMA buffers would; the
    latency of a request runs from its submission to its completion as the
    server's clock sees them (host samples in, estimates back in host memory).
    Each request carries the 500 us deadline: one not admitted into a batch by
    then is dropped (counted, and as a missed deadline in the percentiles)."""
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth
    from libapsm_b200.server import clock

    pop = synth.config4_population(n_det)
    reqs = synth.config4_requests(pop, rate_hz, duration_s)
    warm_reqs = synth.config4_requests(pop, rate_hz, 0.05, seed=9)
    cfg = dict(synth.CONFIG2_ALGORITHM, detectVersion=detect_version)
    pool = L.DetectorPool(cfg, lanes=lanes)
    ids = [pool.add(p.frame.N) for p in pop]
    pool.run([L.PoolJob(i, p.frame.rx_train, p.frame.tx_train) for i, p in zip(ids, pop)])
    srv = L.DetectorServer(pool, max_batch=max_batch)

    # the largest requests (every lane's scratch and page-locked buffers are grown to a batch
    # of them before timing: growing them allocates, which would stall a timed request)
    big = sorted(range(len(pop)), key=lambda d: -pop[d].frame.N)[: lanes * max_batch]
    big_reqs = [(0.0, d, "detect", 4000) for d in big] + [(0.0, d, "train", 64) for d in big]
    need = sum(8 * (pop[d].frame.N + 1) * n + 512 for (_, d, _, n) in reqs + warm_reqs + big_reqs)
    arena = torch.empty(need, dtype=torch.uint8, pin_memory=True).numpy()
    off = 0

    def pinned(a):
        nonlocal off
        a = np.ascontiguousarray(a)
        v = arena[off:off + a.nbytes].view(a.dtype).reshape(a.shape)
        v[...] = a
        off = (off + a.nbytes + 255) // 256 * 256
        return v

    def job(d, kind, n):
        p = pop[d]
        if kind == "train":
            return L.PoolJob(ids[d], pinned(p.pilots_rx[:, :n]), pinned(p.pilots_tx[:n]))
        return L.PoolJob(ids[d], pinned(p.data_rx[:, :n]), est=pinned(np.zeros(n, np.complex64)))

    # warm-up: every lane's scratch and staging buffers reserved for a batch of the largest
    # requests of each kind, then requests like the timed ones
    for kind in ("detect", "train"):
        big_batch = pool.prepare([job(d, k, n) for (_, d, k, n) in big_reqs if k == kind][:max_batch])
        for lane in range(lanes):
            pool.reserve(big_batch, lane=lane)
    for t in [srv.submit_prepared(srv.make_job(job(d, kind, n))) for (_, d, kind, n) in warm_reqs]:
        srv.wait(t)
    prepared = [(ta, kind, n, srv.make_job(job(d, kind, n))) for (ta, d, kind, n) in reqs]
    b0, j0 = srv.stats()
    srv.set_deadline(deadline_s)  # a request not admitted within the deadline is dropped
    start = clock() + 0.01
    tickets = []
    for (ta, kind, n, prep) in prepared:
        target = start + ta
        while clock() < target:
            pass
        tickets.append(srv.submit_prepared(prep))
    lat, kinds, syms, done, dropped, failed = [], [], 0, [], 0, 0
    for (ta, kind, n, prep), tk in zip(prepared, tickets):
        st = srv.wait_status(tk)
        s0, s1, s2 = srv.times(tk)
        if st != 0:
            dropped += st == L._native.APSM_ERR_DEADLINE
            failed += st != L._native.APSM_ERR_DEADLINE
            lat.append(float("inf"))
            kinds.append(kind)
            continue
        lat.append(s2 - s0)
        kinds.append(kind)
        done.append(s2)
        syms += n if kind == "detect" else 0
    b, jb = srv.stats()
    srv.close()
    pool.close()
    lat_us = np.array(lat) * 1e6
    is_train = np.array([k == "train" for k in kinds])
    pct = lambda x, q: float(np.percentile(x, q)) if len(x) else None
    return {"p50_us": pct(lat_us, 50), "p99_us": pct(lat_us, 99),
            "train_p99_us": pct(lat_us[is_train], 99), "detect_p99_us": pct(lat_us[~is_train], 99),
            "deadline_500us_met": float(np.mean(lat_us <= 500.0)), "symbols_per_s": syms / (max(done) - start),
            "deadline_s": deadline_s, "dropped_at_deadline": int(dropped), "failed": int(failed),
            "requests": len(reqs), "rate_hz": rate_hz, "duration_s": duration_s, "batches": int(b - b0),
            "avg_batch": float((jb - j0) / max(1, b - b0)), "lanes": lanes, "max_batch": max_batch,
            "detect": "FP32 CUDA-core pair form" if detect_version == "balanced" else
                      f"{detect_version} tensor-core pair form",
            "workload": "512 resident detectors (config-2 sizes, dictionarySize 2000); requests alternate "
                        "train-append (16-64 pilots) and detect (500-4000 symbols) per detector; Poisson arrivals; "
                        "request samples in page-locked host buffers"}


# ----------------------------------------------------------- reference arm --
def cpu_sample(per_class: int = 6) -> list:
    """A bounded sample of the batched workload stratified by antenna count:
    the first `per_class` detectors of each antenna class {4, 8, 16, 32} in
    the 512-detector draw (their pilot and data lengths as drawn), as
    (index in the draw, detector) pairs."""
    from libapsm_b200 import synth

    dets = synth.config2_detectors(N_DET, seed=2)
    out = []
    for N in (4, 8, 16, 32):
        out += [(i, d) for i, d in enumerate(dets) if d.N == N][:per_class]
    return out


def cpu_baseline(per_class: int = 6, batched_est: list | None = None) -> dict:
    """The FP32 restatement of the reference algorithm on the host cores
    (OpenMP over all host threads), on a bounded, antenna-stratified sample of
    the batched workload.  Also the share of the full batch's work the sample
    holds, so that its time can be set against the batch's."""
    from libapsm_b200 import synth
    from oracle import oracle as O

    threads = O.set_threads(os.cpu_count() or 1)
    sample = cpu_sample(per_class)
    dets = [d for _, d in sample]
    cfg = dict(synth.CONFIG2_ALGORITHM)
    t0 = time.perf_counter()
    syms = 0
    ests = []
    for d in dets:
        o = O.OracleDetector(cfg, d.N, O.F32)
        o.train(d.rx_train, d.tx_train)
        ests.append(o.detect(d.rx_data))
        syms += d.S
    dt = time.perf_counter() - t0
    P = sum(d.P for d in dets)
    out = {"value": syms / dt, "unit": UNIT, "cores": threads, "kind": "port",
           "training_samples_per_s": P / dt,
           "sample": f"{len(dets)} of the 512 detectors, the first {per_class} of each antenna class "
                     f"(4/8/16/32), train + detect each: {P} pilots, {syms} symbols, {dt:.2f} s"}
    if batched_est is not None:
        # the same frames' SER in the oracle and in the batched run (hard decisions of the Gray map)
        err_o = err_b = diff = 0
        for (i, d), eo in zip(sample, ests):
            true = d.modulation.hard_decode_int(d.tx_data)
            do, db = d.modulation.hard_decode_int(eo), d.modulation.hard_decode_int(batched_est[i])
            err_o += int(np.sum(do != true))
            err_b += int(np.sum(db != true))
            diff += int(np.sum(do != db))
        out["ser_oracle"] = err_o / syms
        out["ser_batched_same_frames"] = err_b / syms
        out["decisions_differing_from_oracle"] = diff
    return out


def reference_cuda(n_sample: int = 16) -> dict | None:
    """The reference library (built from its sources for sm_100a) on this
    GPU: one NomaDetector per detector, train + detect, eight host threads."""
    from concurrent.futures import ThreadPoolExecutor

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
    dets = synth.config2_detectors(n_sample, seed=2)
    cfg = dict(synth.CONFIG2_ALGORITHM)

    def one(d):
        r = O.ReferenceDetector(cfg, d.N)
        r.train(d.rx_train, d.tx_train)
        r.detect(d.rx_data)

    one(dets[0])  # warm-up (context, module load)
    t0 = time.perf_counter()
    with ThreadPoolExecutor(8) as ex:
        list(ex.map(one, dets))
    dt = time.perf_counter() - t0
    return {"value": sum(d.S for d in dets) / dt, "unit": UNIT, "ms": dt * 1e3,
            "what": f"reference CUDA kernels (libapsm built for sm_100a), {n_sample} of the 512 detectors, "
                    "8 host threads, wall clock"}


def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    base = cpu_baseline()
    line = {
        "metric": METRIC, "value": base["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded NOMA frames; no public dataset)",
        "config": dict(WORKLOAD), "impl": "reference", "cpu_baseline": base,
        "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    rc = reference_cuda()
    if rc is not None:
        line["reference_cuda"] = rc
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the plain and serving measurements")
    ap.add_argument("--trace-serving", default="",
                    help="file for the serving pool's batch timeline (APSM_POOL_TRACE; tracing adds latency)")
    ap.add_argument("--detectors", type=int, default=N_DET,
                    help="detectors of the batched workload (the first ones of the same seeded draw; 512 is the "
                         "benchmark, fewer only for profiling captures)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the pool's launch-shape autotuner (profiler runs: its timings are distorted there)")
    ap.add_argument("--precision-only", action="store_true",
                    help="run only the large-detect precision study (N=64, dictionary 8192) and print it")
    ap.add_argument("--serving-only", action="store_true",
                    help="run only the served form (FP32 pair form and BF16 Gram detection) and print it")
    ap.add_argument("--plain-only", action="store_true",
                    help="run only the plain per-detector form on the config-1 frame (8 users, N=16) and print it")
    ap.add_argument("--plain-detect-version", default="balanced",
                    help="detection form of --plain-only (balanced, gram_bf16, gram_bf16x3, gram_tf32, gram_tf32x3)")
    args = ap.parse_args()
    if args.precision_only:
        print(json.dumps({"precision": run_precision_study()}), flush=True)
        return
    if args.plain_only:
        print(json.dumps({"plain": run_plain(steps=max(1, args.steps), warmup=max(1, args.warmup),
                                             detect_version=args.plain_detect_version, compare=False)}), flush=True)
        return
    if args.serving_only:
        print(json.dumps({"serving": run_serving(), "serving_gram_bf16": run_serving(detect_version="gram_bf16")}),
              flush=True)
        return
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
    line = run_batched(args, rank, world)
    if line is not None and not args.no_extras:
        line["plain"] = run_plain()
        if args.trace_serving:
            os.environ["APSM_POOL_TRACE"] = args.trace_serving
        line["serving"] = run_serving()
        os.environ.pop("APSM_POOL_TRACE", None)
        line["serving_gram_bf16"] = run_serving(detect_version="gram_bf16")
        line["serving_p50_us"] = line["serving"]["p50_us"]
        line["serving_p99_us"] = line["serving"]["p99_us"]
        line["serving_deadline_met"] = line["serving"]["deadline_500us_met"]
        ps = line.get("plain_same_workload") or {}
        if ps.get("value"):
            line["batched_over_plain"] = line["value"] / ps["value"]
        line["precision"] = run_precision_study()
    if line is not None and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(batched_est=batched_est_host if len(batched_est_host) == N_DET else None)
    if world > 1:
        import torch

        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
