"""Host-side mirror of the reference's detector API over the B200 C ABI.

Reference interface (fraunhoferhhi/libapsm):
  NomaDetectorFactory::build(json algorithmConfig, uint32_t numAntennas)
      cpp/lib/noma/noma_detector_factory.cu:57-65
  NomaDetector::train(rxSigTraining [N][P], txSigTraining [P]) -> float ms
  NomaDetector::detect(rxSigData [N][S], estData&) -> float ms
  NomaDetector::resetState()
      cpp/lib/noma/noma_detector.cuh:65-75

Here the same calls are ``NomaDetectorFactory.build(config, num_antennas)``,
``det.train(rx, tx) -> ms``, ``det.detect(rx) -> (est, ms)`` and
``det.reset_state()``.  Complex sample matrices are numpy complex64 arrays,
antenna-major (shape (N, n)) exactly like ComplexSampleMatrix.  A detector
built with ``num_users=K`` trains K users that share the received signal
(the reference CLI's -p mode): tx has shape (K, P) and detect returns (K, S).

Errors: configuration problems raise ``ValueError`` (the reference throws
std::invalid_argument), everything else raises ``ApsmError``.  Nothing here
computes on the CPU: every train/detect runs the CUDA kernels of
libapsm_b200.so, and a missing library is an error.
"""
from __future__ import annotations

import ctypes
import json
from typing import Any, Mapping

import numpy as np

from . import _native


class ApsmError(RuntimeError):
    """A non-configuration failure reported by the native library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_native.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def _as_complex_matrix(x: Any, rows: int | None, name: str) -> np.ndarray:
    a = np.asarray(x)
    if a.ndim == 1 and rows is not None and rows == 1:
        a = a[None, :]
    if a.ndim != 2:
        raise ValueError(f"{name} must be a 2-D complex array (antennas x samples)")
    if rows is not None and a.shape[0] != rows:
        raise ValueError(f"{name} has {a.shape[0]} rows, expected {rows}")
    return np.ascontiguousarray(a, dtype=np.complex64)


class NomaDetector:
    """APSM (or LLS) detector on one B200; see the module docstring."""

    def __init__(self, config: Mapping[str, Any] | str, num_antennas: int, num_users: int = 1):
        lib = _native.load()
        text = config if isinstance(config, str) else json.dumps(dict(config))
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        st = lib.apsm_create(text.encode(), int(num_antennas), int(num_users), ctypes.byref(handle), err, len(err))
        msg = err.value.decode(errors="replace")
        if st == _native.APSM_ERR_INVALID_CONFIG or st == _native.APSM_ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        if st != _native.APSM_OK:
            raise ApsmError(st, msg)
        self._lib = lib
        self._h = handle
        self.config = json.loads(text)
        self.num_antennas = int(num_antennas)
        self.num_users = int(num_users)

    # -- lifetime -------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.apsm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int) -> None:
        if st == _native.APSM_OK:
            return
        msg = self._lib.apsm_last_error(self._h).decode(errors="replace")
        if st == _native.APSM_ERR_INVALID_ARGUMENT:
            raise ValueError(msg)
        raise ApsmError(st, msg)

    # -- the reference API ------------------------------------------------
    def train(self, rx_sig_training: Any, tx_sig_training: Any, val_set: tuple | None = None) -> float:
        """NomaDetector::train: rx (N, P) complex, tx (P,) or (users, P). Returns GPU ms.

        val_set = (history, rx_val, tx_val) mirrors the reference's NomaValSet
        (noma_train_history.cuh:99): ``history`` is a NomaTrainHistory that
        receives, for the model after every training step, EVM / SER / BER of
        the training symbols and of the validation set rx_val (N, S) / tx_val
        (S,) or (users, S).  With several users the history keeps user 0's
        rows; ``history.per_user`` holds all of them."""
        rx = _as_complex_matrix(rx_sig_training, self.num_antennas, "rxSigTraining")
        P = rx.shape[1]
        tx = _as_complex_matrix(np.atleast_2d(tx_sig_training), self.num_users, "txSigTraining")
        if tx.shape[1] != P:
            raise ValueError(f"txSigTraining has {tx.shape[1]} samples, rxSigTraining {P}")
        if P == 0:
            raise ValueError("no training samples")
        ms = ctypes.c_float(0.0)
        if val_set is None:
            self._check(self._lib.apsm_train(self._h, rx.ctypes.data, tx.ctypes.data, P, ctypes.byref(ms)))
            return float(ms.value)
        history, rx_val, tx_val = val_set
        rxv = _as_complex_matrix(rx_val, self.num_antennas, "rxSigVal")
        S = rxv.shape[1]
        txv = _as_complex_matrix(np.atleast_2d(tx_val), self.num_users, "txSigVal")
        if txv.shape[1] != S:
            raise ValueError(f"txSigVal has {txv.shape[1]} samples, rxSigVal {S}")
        steps = int(self._lib.apsm_train_steps(self._h, P))
        out = np.zeros((self.num_users, max(steps, 1), 6), dtype=np.float32)
        n = ctypes.c_uint32(0)
        self._check(self._lib.apsm_train_history(self._h, rx.ctypes.data, tx.ctypes.data, P, rxv.ctypes.data,
                                                 txv.ctypes.data, S, int(history.bit_per_symbol),
                                                 float(history.modulation_scale), out.ctypes.data, steps,
                                                 ctypes.byref(n), ctypes.byref(ms)))
        # the library writes users x n x 6 contiguously
        flat = out.reshape(-1)[: self.num_users * n.value * 6].reshape(self.num_users, n.value, 6)
        history.extend(flat)
        return float(ms.value)

    def detect(self, rx_sig_data: Any) -> tuple[np.ndarray, float]:
        """NomaDetector::detect: rx (N, S) complex -> (estData, GPU ms).

        estData has shape (S,) for a single-user detector, (users, S) otherwise."""
        rx = _as_complex_matrix(rx_sig_data, self.num_antennas, "rxSigData")
        S = rx.shape[1]
        est = np.zeros((self.num_users, S), dtype=np.complex64)
        ms = ctypes.c_float(0.0)
        if S:
            self._check(self._lib.apsm_detect(self._h, rx.ctypes.data, S, est.ctypes.data, ctypes.byref(ms)))
        return (est[0] if self.num_users == 1 else est), float(ms.value)

    def reset_state(self) -> None:
        """NomaDetector::resetState."""
        self._check(self._lib.apsm_reset(self._h))

    # -- device-resident calls (torch tensors already on the GPU) --------
    def train_device(self, rx, tx, stream: int | None = None) -> None:
        """Enqueue training on device buffers: rx (N, P) complex64, tx (users, P) complex64."""
        self._check(self._lib.apsm_train_device(self._h, rx.data_ptr(), tx.data_ptr(), int(rx.shape[-1]),
                                                stream or None))

    def detect_device(self, rx, est, stream: int | None = None) -> None:
        """Enqueue detection: rx (N, S) complex64 -> est (users, S) complex64 (device buffers)."""
        self._check(self._lib.apsm_detect_device(self._h, rx.data_ptr(), int(rx.shape[-1]), est.data_ptr(),
                                                 stream or None))

    def last_kernel_ms(self) -> tuple[float, float]:
        """GPU ms of the last training sweep kernel and the last detection kernel (-1 if not run)."""
        a, b = ctypes.c_float(), ctypes.c_float()
        self._check(self._lib.apsm_last_kernel_ms(self._h, ctypes.byref(a), ctypes.byref(b)))
        return float(a.value), float(b.value)

    def synchronize(self) -> None:
        self._check(self._lib.apsm_synchronize(self._h))

    @property
    def stream(self) -> int:
        return int(self._lib.apsm_stream(self._h) or 0)

    @property
    def gaussian_variance(self) -> float:
        """Effective Gaussian variance (N^2-scaled, or the heuristic's value after training)."""
        v = ctypes.c_float(0.0)
        self._check(self._lib.apsm_gaussian_variance(self._h, ctypes.byref(v)))
        return float(v.value)

    def compute_norm_ratio(self, user: int = 0) -> float:
        """ApsmNomaDetector::computeNormRatio: wL |w|^2 / (wG a^T K a) of the user's model."""
        r = ctypes.c_float(0.0)
        self._check(self._lib.apsm_norm_ratio(self._h, int(user), ctypes.byref(r)))
        return float(r.value)

    # -- model snapshot ---------------------------------------------------
    def rows(self) -> int:
        return int(self._lib.apsm_rows(self._h))

    def get_state(self) -> dict[str, np.ndarray]:
        """Dictionary rows (rows, 2N), coefficients (users, rows), linear weights (users, 2N)."""
        rows = self.rows()
        D = 2 * self.num_antennas
        dic = np.zeros((rows, D), dtype=np.float32)
        a = np.zeros((self.num_users, rows), dtype=np.float32)
        w = np.zeros((self.num_users, D), dtype=np.float32)
        self._check(self._lib.apsm_get_state(self._h, dic.ctypes.data if rows else None,
                                             a.ctypes.data if rows else None, w.ctypes.data))
        return {"dictionary": dic, "a": a, "w": w}

    def copy_state_from(self, other: "NomaDetector") -> None:
        """Take over the trained state of another detector of the same sizes
        (apsm_copy_state): one model, evaluated in this detector's detection form."""
        self._check(self._lib.apsm_copy_state(self._h, other._h))


class NomaDetectorFactory:
    """NomaDetectorFactory::build (cpp/lib/noma/noma_detector_factory.cu:57-65)."""

    @staticmethod
    def build(algorithm_config: Mapping[str, Any] | str, num_antennas: int, num_users: int = 1) -> NomaDetector:
        return NomaDetector(algorithm_config, num_antennas, num_users)


def version() -> str:
    return _native.load().apsm_version().decode()
