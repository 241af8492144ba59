"""Detector pool: many resident APSM detectors, batched train/detect.

The reference serves several users by running one detector per user on its
own host thread (its CLI's -p mode, cpp/cli/detect/noma_detect.cpp:109-112),
each call being NomaDetector::train / detect (cpp/lib/noma/noma_detector.cuh:
65-75).  A :class:`DetectorPool` keeps the state of many detectors (users x
cells, each with its own antenna count) resident on the GPU and runs a batch
of their train/detect calls in a handful of launches (include/apsm_b200.h,
``apsm_pool_*``).  Per detector the semantics are those of
``NomaDetector.train`` / ``detect``; training jobs of a batch run before its
detection jobs.

Jobs are :class:`PoolJob` records.  Host jobs take numpy complex64 arrays
(rx antenna-major, shape (N, n)); device jobs (``run_device``) take torch
complex64 CUDA tensors and return once the work is enqueued on the lane's
stream.
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass
from typing import Any, Mapping, Sequence

import numpy as np

from . import _native
from .detector import ApsmError

JOB_TRAIN = 0
JOB_DETECT = 1
JOB_FRESH = 1  # train-job flag: resetState before training


class _CJob(ctypes.Structure):
    _fields_ = [("detector", ctypes.c_uint32), ("kind", ctypes.c_uint32), ("length", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("rx", ctypes.c_void_p), ("tx", ctypes.c_void_p),
                ("est", ctypes.c_void_p)]


@dataclass
class PoolJob:
    """One train (tx given) or detect (tx None) call of one pool detector;
    fresh=True resets the detector before a train job."""

    detector: int
    rx: Any
    tx: Any = None
    est: Any = None
    fresh: bool = False

    @property
    def kind(self) -> int:
        return JOB_TRAIN if self.tx is not None else JOB_DETECT


class DetectorPool:
    def __init__(self, config: Mapping[str, Any] | str, hbm_budget: int = 0, lanes: int = 1):
        lib = _native.load()
        text = config if isinstance(config, str) else json.dumps(dict(config))
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        st = lib.apsm_pool_create(text.encode(), int(hbm_budget), int(lanes), ctypes.byref(h), err, len(err))
        msg = err.value.decode(errors="replace")
        if st == _native.APSM_ERR_INVALID_CONFIG:
            raise ValueError(msg)
        if st != _native.APSM_OK:
            raise ApsmError(st, msg)
        self._lib, self._h, self.lanes = lib, h, int(lanes)
        self.antennas: dict[int, int] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.apsm_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != _native.APSM_OK:
            raise ApsmError(st, self._lib.apsm_pool_last_error(self._h).decode(errors="replace"))

    # ---- detectors ----
    def add(self, num_antennas: int) -> int:
        d = ctypes.c_uint32()
        self._check(self._lib.apsm_pool_add(self._h, int(num_antennas), ctypes.byref(d)))
        self.antennas[d.value] = int(num_antennas)
        return d.value

    def remove(self, detector: int) -> None:
        self._check(self._lib.apsm_pool_remove(self._h, int(detector)))
        self.antennas.pop(detector, None)

    def reset(self, detector: int) -> None:
        self._check(self._lib.apsm_pool_reset(self._h, int(detector)))

    def inject_fault(self, fault: int, count: int = 1) -> None:
        """Host-side fault injection (tests): APSM_FAULT_LANE_ALLOC fails the next
        `count` lane-scratch growths as an allocation would."""
        self._check(self._lib.apsm_pool_inject_fault(self._h, int(fault), int(count)))

    def get_state(self, detector: int) -> tuple[int, np.ndarray, np.ndarray]:
        """(rows in use, a[rows], w[2N])."""
        n = self.antennas[detector]
        a = np.zeros(4 * 4096 + 8, np.float32)
        w = np.zeros(2 * n, np.float32)
        rows = ctypes.c_uint32()
        self._check(self._lib.apsm_pool_get_state(self._h, int(detector), ctypes.byref(rows), a.ctypes.data,
                                                  w.ctypes.data))
        return rows.value, a[: rows.value].copy(), w

    # ---- batches ----
    def _cjobs(self, jobs: Sequence[PoolJob], device: bool):
        arr = (_CJob * max(1, len(jobs)))()
        keep = []
        for i, j in enumerate(jobs):
            n = self.antennas.get(j.detector)
            if n is None:
                raise ValueError(f"unknown detector {j.detector}")
            if device:
                rx, tx, est = j.rx, j.tx, j.est
                length = int(rx.shape[1])
                rxp = rx.data_ptr()
                txp = tx.data_ptr() if tx is not None else None
                if tx is None and est is None:
                    raise ValueError("device detect jobs need an est tensor")
                estp = est.data_ptr() if tx is None else None
            else:
                rx = np.ascontiguousarray(j.rx, dtype=np.complex64)
                if rx.ndim != 2 or rx.shape[0] != n:
                    raise ValueError(f"job {i}: rx must have shape ({n}, n)")
                length = rx.shape[1]
                keep.append(rx)
                rxp = rx.ctypes.data
                txp = estp = None
                if j.tx is not None:
                    tx = np.ascontiguousarray(j.tx, dtype=np.complex64).reshape(-1)
                    if tx.shape[0] != length:
                        raise ValueError(f"job {i}: tx must have {length} pilots")
                    keep.append(tx)
                    txp = tx.ctypes.data
                else:
                    if j.est is None or np.asarray(j.est).shape != (length,) or j.est.dtype != np.complex64:
                        j.est = np.zeros(length, np.complex64)
                    estp = j.est.ctypes.data
            arr[i] = _CJob(int(j.detector), j.kind, length, JOB_FRESH if j.fresh else 0, rxp, txp, estp)
        return arr, keep

    def run(self, jobs: Sequence[PoolJob], lane: int = 0) -> list[np.ndarray | None]:
        """Host buffers; returns each job's estimates (None for train jobs)."""
        arr, keep = self._cjobs(jobs, device=False)
        self._check(self._lib.apsm_pool_run(self._h, int(lane), ctypes.cast(arr, ctypes.c_void_p), len(jobs), 0))
        del keep
        return [j.est if j.kind == JOB_DETECT else None for j in jobs]

    def prepare(self, jobs: Sequence[PoolJob], device: bool = False):
        """The native job list of a batch, for repeated apsm_pool_run calls
        (run_prepared); keeps the host arrays it points to alive."""
        arr, keep = self._cjobs(jobs, device=device)
        return (arr, len(jobs), keep, list(jobs))

    def run_prepared(self, prepared, lane: int = 0, mode: int = 0) -> None:
        """apsm_pool_run on a prepared job list (mode 0: host buffers, 1: device buffers)."""
        arr, n, _, _ = prepared
        self._check(self._lib.apsm_pool_run(self._h, int(lane), ctypes.cast(arr, ctypes.c_void_p), n, int(mode)))

    def run_device(self, jobs: Sequence[PoolJob], lane: int = 0) -> None:
        """Device buffers (torch complex64 CUDA tensors); asynchronous on the lane's stream."""
        arr, _ = self._cjobs(jobs, device=True)
        self._check(self._lib.apsm_pool_run(self._h, int(lane), ctypes.cast(arr, ctypes.c_void_p), len(jobs), 1))

    def reserve(self, prepared, lane: int = 0, mode: int = 0) -> None:
        """apsm_pool_reserve: grow the lane's buffers to this batch's needs now, so that
        no later batch stalls on growing them; runs nothing."""
        arr, n, _, _ = prepared
        self._check(self._lib.apsm_pool_reserve(self._h, int(lane), ctypes.cast(arr, ctypes.c_void_p), n, int(mode)))

    def autotune(self, prepared, lane: int = 0, mode: int = 0) -> dict:
        """apsm_pool_autotune on a prepared batch (mode as in run_prepared): times the
        batch under each candidate launch shape, keeps the fastest for later batches,
        and leaves every detector's state as it was.  Returns the trials and the
        chosen shape."""
        arr, n, _, _ = prepared
        buf = ctypes.create_string_buffer(1 << 14)
        self._check(self._lib.apsm_pool_autotune(self._h, int(lane), ctypes.cast(arr, ctypes.c_void_p), n, int(mode),
                                                  buf, len(buf)))
        return json.loads(buf.value.decode())

    def wait(self, lane: int = 0) -> None:
        self._check(self._lib.apsm_pool_wait(self._h, int(lane)))

    def query(self, lane: int = 0) -> bool:
        r = self._lib.apsm_pool_query(self._h, int(lane))
        if r < 0:
            self._check(-r)
        return r == 1

    def stream(self, lane: int = 0) -> int:
        return self._lib.apsm_pool_stream(self._h, int(lane))

    def last_ms(self, lane: int = 0) -> tuple[float, float]:
        t, d = ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.apsm_pool_last_ms(self._h, int(lane), ctypes.byref(t), ctypes.byref(d)))
        return t.value, d.value

    def set_timing(self, on: bool) -> None:
        """Per-stage GPU events of each batch (default on; needed by last_ms / last_sweep_ms)."""
        self._check(self._lib.apsm_pool_set_timing(self._h, 1 if on else 0))

    def last_sweep_ms(self, lane: int = 0) -> float:
        """GPU time of the last batch's training sweep kernel."""
        v = ctypes.c_float()
        self._check(self._lib.apsm_pool_last_sweep_ms(self._h, int(lane), ctypes.byref(v)))
        return v.value

    def last_launches(self, lane: int = 0) -> int:
        """Kernels the lane's last batch launched."""
        return int(self._lib.apsm_pool_last_launches(self._h, int(lane)))

    def job_bytes(self, job: PoolJob) -> int:
        n = self.antennas[job.detector]
        length = int(job.rx.shape[1])
        cj = _CJob(int(job.detector), job.kind, length, 0, None, None, None)
        del n
        return int(self._lib.apsm_pool_job_bytes(self._h, ctypes.byref(cj)))

    @property
    def budget(self) -> int:
        return int(self._lib.apsm_pool_budget(self._h))

    @property
    def bytes_in_use(self) -> int:
        return int(self._lib.apsm_pool_bytes_in_use(self._h))
