"""Request server: continuous batching of per-TTI requests over a pool.

Reference callers run one detector per user and thread, one frame at a time
(cpp/cli/detect/noma_detect.cpp:100-137).  :class:`DetectorServer` wraps the
native server of include/apsm_b200.h (``apsm_server_*``): requests (one
:class:`~libapsm_b200.pool.PoolJob` each, host buffers) are admitted into
batches on the pool's lanes as lanes free up, per detector in arrival order,
and batches on different lanes overlap on the GPU.  Request times (submission,
admission, completion) come from the native monotonic clock
(:func:`clock`).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from .detector import ApsmError
from .pool import JOB_DETECT, JOB_FRESH, DetectorPool, PoolJob, _CJob


def clock() -> float:
    return float(_native.load().apsm_server_clock())


class DetectorServer:
    def __init__(self, pool: DetectorPool, lanes: int | None = None, max_batch: int = 64):
        self.pool = pool
        self._lib = pool._lib
        h = ctypes.c_void_p()
        st = self._lib.apsm_server_create(pool._h, int(lanes or pool.lanes), int(max_batch), ctypes.byref(h))
        if st != _native.APSM_OK:
            raise ApsmError(st, "apsm_server_create failed")
        self._h = h
        self._keep: dict[int, tuple] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.apsm_server_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def make_job(self, job: PoolJob) -> tuple:
        """Native job record plus the arrays it points to (host buffers)."""
        n = self.pool.antennas[job.detector]
        rx = np.ascontiguousarray(job.rx, dtype=np.complex64)
        if rx.ndim != 2 or rx.shape[0] != n:
            raise ValueError(f"rx must have shape ({n}, n)")
        length = rx.shape[1]
        tx = est = None
        if job.tx is not None:
            tx = np.ascontiguousarray(job.tx, dtype=np.complex64).reshape(-1)
            if tx.shape[0] != length:
                raise ValueError(f"tx must have {length} pilots")
        else:
            if job.est is None or job.est.shape != (length,) or job.est.dtype != np.complex64:
                job.est = np.zeros(length, np.complex64)
            est = job.est
        cj = _CJob(int(job.detector), job.kind, length, JOB_FRESH if job.fresh else 0, rx.ctypes.data,
                   tx.ctypes.data if tx is not None else None, est.ctypes.data if est is not None else None)
        return cj, rx, tx, est

    def submit_prepared(self, prepared: tuple, deadline: float | None = None) -> int:
        """Queue a request; `deadline` seconds after submission (None: the server's
        default, 0: none).  Malformed or oversized requests raise here (no ticket)."""
        t = ctypes.c_uint64()
        dl = -1.0 if deadline is None else float(deadline)
        st = self._lib.apsm_server_submit_deadline(self._h, ctypes.byref(prepared[0]), dl, ctypes.byref(t))
        if st != _native.APSM_OK:
            raise ApsmError(st, "request rejected at submission")
        self._keep[t.value] = prepared
        return t.value

    def submit(self, job: PoolJob, deadline: float | None = None) -> int:
        return self.submit_prepared(self.make_job(job), deadline)

    def set_deadline(self, seconds: float) -> None:
        """Default deadline of later submissions (0: none)."""
        st = self._lib.apsm_server_set_deadline(self._h, float(seconds))
        if st != _native.APSM_OK:
            raise ApsmError(st, "apsm_server_set_deadline")

    def cancel(self, ticket: int) -> int:
        """Cancel a request not admitted yet; the native status (APSM_OK when cancelled)."""
        return int(self._lib.apsm_server_cancel(self._h, ctypes.c_uint64(ticket)))

    def status(self, ticket: int) -> int | None:
        """The finished request's status, None while it is pending."""
        s = ctypes.c_int()
        r = self._lib.apsm_server_poll(self._h, ctypes.c_uint64(ticket), ctypes.byref(s))
        if r < 0:
            raise ValueError(f"unknown ticket {ticket}")
        return s.value if r == 1 else None

    def wait_status(self, ticket: int, timeout: float = 30.0) -> int:
        """Block until the request finished (or timeout): its status, APSM_ERR_TIMEOUT."""
        return int(self._lib.apsm_server_wait(self._h, ctypes.c_uint64(ticket), float(timeout)))

    def counts(self) -> tuple[int, int, int]:
        """Requests dropped at their deadline, cancelled, rejected at submission."""
        d, c, r = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._lib.apsm_server_counts(self._h, ctypes.byref(d), ctypes.byref(c), ctypes.byref(r))
        return d.value, c.value, r.value

    def inject_fault(self, fault: int, count: int = 1) -> None:
        """Host-side fault injection (tests): APSM_FAULT_DROP_REQUEST loses the next
        `count` submitted requests on their way into the queue."""
        st = self._lib.apsm_server_inject_fault(self._h, int(fault), int(count))
        if st != _native.APSM_OK:
            raise ApsmError(st, "apsm_server_inject_fault")

    def wait(self, ticket: int, timeout: float = 30.0) -> np.ndarray | None:
        st = self._lib.apsm_server_wait(self._h, ctypes.c_uint64(ticket), float(timeout))
        if st != _native.APSM_OK:
            raise ApsmError(st, f"request {ticket}")
        prep = self._keep.get(ticket)
        return prep[3] if prep is not None and prep[0].kind == JOB_DETECT else None

    def done(self, ticket: int) -> bool:
        s = ctypes.c_int()
        r = self._lib.apsm_server_poll(self._h, ctypes.c_uint64(ticket), ctypes.byref(s))
        if r < 0:
            raise ValueError(f"unknown ticket {ticket}")
        return r == 1

    def times(self, ticket: int) -> tuple[float, float, float]:
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st = self._lib.apsm_server_times(self._h, ctypes.c_uint64(ticket), ctypes.byref(a), ctypes.byref(b),
                                         ctypes.byref(c))
        if st != _native.APSM_OK:
            raise ApsmError(st, f"request {ticket}")
        return a.value, b.value, c.value

    def release(self, ticket: int) -> None:
        self._lib.apsm_server_release(self._h, ctypes.c_uint64(ticket))
        self._keep.pop(ticket, None)

    def stats(self) -> tuple[int, int]:
        b, j = ctypes.c_uint64(), ctypes.c_uint64()
        self._lib.apsm_server_stats(self._h, ctypes.byref(b), ctypes.byref(j))
        return b.value, j.value
