"""TEST INFRASTRUCTURE ONLY — the oracle is the checker, never the product.

Python access to the two checkers built by oracle/Makefile:

* ``OracleDetector`` — the CPU restatement of the reference APSM path
  (oracle/apsm_oracle.c): FP32 in the reference's evaluation order, or FP64.
* ``ReferenceDetector`` / ``reference_users_threaded`` — the reference library
  itself (fraunhoferhhi/libapsm compiled from its sources for sm_100a,
  oracle/_ref/libapsm_ref.so); needs a GPU.

Parameter handling restates ApsmNomaDetectorFactory::build
(cpp/lib/apsm/apsm_noma_detector.cu:348-383: defaults, strict keys) and the
constructor's variance scaling by N^2 (:79-80).  Only tests/, the smoke test
and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
from pathlib import Path
from typing import Any, Mapping

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
ORACLE_SO = REF_DIR / "liboracle.so"
REF_SO = REF_DIR / "libapsm_ref.so"

F32, F64 = 0, 1

_VALID = ("otype", "llsInitialization", "trainingShuffle", "gaussianKernelWeight", "gaussianKernelVariance",
          "windowSize", "sampleStep", "trainPasses", "startWithFullWindow", "dictionarySize", "normConstraint", "eB",
          "detectVersion")


class OracleParams(ctypes.Structure):
    _fields_ = [("linear_weight", ctypes.c_float), ("gaussian_weight", ctypes.c_float),
                ("gaussian_variance", ctypes.c_float), ("eB", ctypes.c_float), ("window_size", ctypes.c_uint32),
                ("sample_step", ctypes.c_uint32), ("train_passes", ctypes.c_uint32),
                ("start_full_window", ctypes.c_uint32), ("dictionary_size", ctypes.c_uint32),
                ("norm_constraint", ctypes.c_float)]


def reference_params(config: Mapping[str, Any], num_antennas: int) -> OracleParams:
    """apsm_parameters as the reference factory + constructor leave them."""
    for k in sorted(config):
        if k not in _VALID:
            raise ValueError(f"Invalid key: {k}")
    f32 = np.float32
    wG = f32(config.get("gaussianKernelWeight", 0.5))
    p = OracleParams()
    p.gaussian_weight = wG
    p.linear_weight = f32(1) - wG
    var = f32(config.get("gaussianKernelVariance", 0.05))
    if var != 0:
        var = f32(var * f32(num_antennas * num_antennas))
    p.gaussian_variance = var
    p.eB = f32(config.get("eB", 0.001))
    p.window_size = int(config.get("windowSize", 20))
    p.sample_step = int(config.get("sampleStep", 2))
    p.train_passes = int(config.get("trainPasses", 1))
    p.start_full_window = int(bool(config.get("startWithFullWindow", False)))
    p.dictionary_size = int(config.get("dictionarySize", 685))
    p.norm_constraint = f32(config.get("normConstraint", 0.0))
    return p


_oracle_lib = None


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)


def _load_oracle() -> ctypes.CDLL:
    global _oracle_lib
    if _oracle_lib is None:
        if not ORACLE_SO.exists():
            build_oracle()
        lib = ctypes.CDLL(str(ORACLE_SO))
        P = ctypes.c_void_p
        lib.apsm_oracle_create.restype = P
        lib.apsm_oracle_create.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_uint32, ctypes.c_int]
        lib.apsm_oracle_destroy.argtypes = [P]
        lib.apsm_oracle_reset.argtypes = [P]
        lib.apsm_oracle_set_threads.argtypes = [ctypes.c_int]
        lib.apsm_oracle_set_threads.restype = ctypes.c_int
        lib.apsm_oracle_train.argtypes = [P, P, P, ctypes.c_uint32]
        lib.apsm_oracle_train.restype = ctypes.c_int
        lib.apsm_oracle_train_history.argtypes = [P, P, P, ctypes.c_uint32, P, P, ctypes.c_uint32, ctypes.c_uint32,
                                                  ctypes.c_float, P, ctypes.c_uint32, P]
        lib.apsm_oracle_train_history.restype = ctypes.c_int
        lib.apsm_oracle_norm_ratio.argtypes = [P]
        lib.apsm_oracle_norm_ratio.restype = ctypes.c_float
        lib.apsm_oracle_detect.argtypes = [P, P, ctypes.c_uint32, P]
        lib.apsm_oracle_detect.restype = ctypes.c_int
        lib.apsm_oracle_rows.argtypes = [P]
        lib.apsm_oracle_rows.restype = ctypes.c_uint32
        lib.apsm_oracle_get_state.argtypes = [P, P, P, P, P]
        lib.apsm_oracle_set_state.argtypes = [P, ctypes.c_uint32, P, P, P]
        lib.apsm_oracle_set_state.restype = ctypes.c_int
        lib.apsm_oracle_set_variance.argtypes = [P, ctypes.c_float]
        lib.apsm_oracle_shuffle_permutation.argtypes = [ctypes.c_uint32, P]
        lib.apsm_oracle_set_w.argtypes = [P, P]
        _oracle_lib = lib
    return _oracle_lib


def set_threads(n: int) -> int:
    return int(_load_oracle().apsm_oracle_set_threads(int(n)))


def shuffle_permutation(P: int) -> np.ndarray:
    """trainingShuffle order (noma_detector.cu:59-74): shuffled[i] = original[perm[i]]."""
    perm = np.zeros(P, dtype=np.int32)
    _load_oracle().apsm_oracle_shuffle_permutation(P, perm.ctypes.data)
    return perm


def variance_heuristic(rx: np.ndarray) -> np.float32:
    """computeGaussianVarianceHeuristic (apsm_noma_detector.cu:193-218), float arithmetic."""
    rx = np.asarray(rx, np.complex64)
    N, P = rx.shape
    nd = []
    for i in range(P - 1):
        acc = np.zeros(P - i - 1, np.float32)
        for k in range(N):
            acc = (acc + np.abs(rx[k, i] - rx[k, i + 1:]).astype(np.float32)).astype(np.float32)
        nd.append(np.sqrt(acc).astype(np.float32))
    nd = np.sort(np.concatenate(nd)) if nd else np.zeros(0, np.float32)
    idx = int(np.float32(len(nd)) * np.float32(0.7))
    v = np.float32(np.float64(nd[idx]) * P ** (-1.0 / 5.0))
    return np.float32(v * v)


def dedup_rows(rx: np.ndarray) -> np.ndarray:
    """Real rows of the Dedup embedding (cuda_matrix_device.cuh:180-188):
    row 2n = [Re y_n; Im y_n], row 2n+1 = [Im y_n; -Re y_n]."""
    rx = np.asarray(rx)
    N, n = rx.shape
    out = np.empty((2 * n, 2 * N), dtype=np.float64)
    out[0::2, :N] = rx.real.T
    out[0::2, N:] = rx.imag.T
    out[1::2, :N] = rx.imag.T
    out[1::2, N:] = -rx.real.T
    return out


def lls_weights(rx: np.ndarray, tx: np.ndarray) -> np.ndarray:
    """LLS detector training (lls_detector.cu:136-179) in FP64: least squares
    of the Dedup system, targets (Re x_n, Im x_n) interleaved."""
    A = dedup_rows(rx)
    t = np.asarray(tx).reshape(-1)
    y = np.empty(2 * t.size)
    y[0::2], y[1::2] = t.real, t.imag
    return np.linalg.lstsq(A, y, rcond=None)[0]


def lls_detect(rx: np.ndarray, w: np.ndarray) -> np.ndarray:
    """LLS detection (lls_detector.cu:181-218): est = A w as complex symbols."""
    f = dedup_rows(rx) @ w
    return (f[0::2] + 1j * f[1::2]).astype(np.complex64)


class OracleDetector:
    """CPU restatement of one reference ApsmNomaDetector (single user)."""

    def __init__(self, config: Mapping[str, Any], num_antennas: int, precision: int = F32):
        self._lib = _load_oracle()
        self.params = reference_params(config, num_antennas)
        self.shuffle = bool(config.get("trainingShuffle", False))
        self.lls_init = bool(config.get("llsInitialization", False))
        self.N = int(num_antennas)
        self._h = self._lib.apsm_oracle_create(ctypes.byref(self.params), self.N, int(precision))
        if not self._h:
            raise ValueError("oracle: invalid parameters")

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.apsm_oracle_destroy(self._h)
            self._h = None

    def reset_state(self):
        self._lib.apsm_oracle_reset(self._h)

    def train(self, rx: np.ndarray, tx: np.ndarray, val_set: tuple | None = None) -> np.ndarray | None:
        """Train on rx (N, P) / tx (P,).  With val_set = (rx_val, tx_val, bits_per_symbol, modulation_scale)
        the reference's per-step history is recorded and returned as (steps, 6): train EVM, SER, BER,
        validation EVM, SER, BER (NomaTrainHistory, noma_train_history.cu:65-248)."""
        rx = np.ascontiguousarray(rx, dtype=np.complex64)
        tx = np.ascontiguousarray(np.asarray(tx).reshape(-1), dtype=np.complex64)
        assert rx.shape == (self.N, tx.shape[0])
        if self.lls_init:
            # llsInitialization (apsm_noma_detector.cu:98-99, 321-346): w = w_lls / wL, unshuffled pilots
            w = lls_weights(rx, tx).astype(np.float32) / np.float32(self.params.linear_weight)
            self._lib.apsm_oracle_set_w(self._h, np.ascontiguousarray(w, dtype=np.float64).ctypes.data)
        if self.shuffle:
            perm = shuffle_permutation(tx.shape[0])
            rx = np.ascontiguousarray(rx[:, perm])
            tx = np.ascontiguousarray(tx[perm])
        if self.params.gaussian_variance == 0:
            self.params.gaussian_variance = variance_heuristic(rx)
            self._lib.apsm_oracle_set_variance(self._h, self.params.gaussian_variance)
        if val_set is not None:
            rxv, txv, bps, scale = val_set
            rxv = np.ascontiguousarray(rxv, dtype=np.complex64)
            txv = np.ascontiguousarray(np.asarray(txv).reshape(-1), dtype=np.complex64)
            assert rxv.shape == (self.N, txv.shape[0])
            cap = 2 * tx.shape[0] * max(1, self.params.train_passes) + 1
            hist = np.zeros((cap, 6), dtype=np.float32)
            n = ctypes.c_uint32(0)
            st = self._lib.apsm_oracle_train_history(self._h, rx.ctypes.data, tx.ctypes.data, tx.shape[0],
                                                     rxv.ctypes.data, txv.ctypes.data, txv.shape[0], int(bps),
                                                     float(scale), hist.ctypes.data, cap, ctypes.byref(n))
            if st != 0:
                raise RuntimeError(f"oracle train (history) failed: {st}")
            return hist[:n.value].copy()
        if self._lib.apsm_oracle_train(self._h, rx.ctypes.data, tx.ctypes.data, tx.shape[0]) != 0:
            raise RuntimeError("oracle train failed")
        return None

    def detect(self, rx: np.ndarray) -> np.ndarray:
        rx = np.ascontiguousarray(rx, dtype=np.complex64)
        S = rx.shape[1]
        est = np.zeros(S, dtype=np.complex64)
        self._lib.apsm_oracle_detect(self._h, rx.ctypes.data, S, est.ctypes.data)
        return est

    def rows(self) -> int:
        return int(self._lib.apsm_oracle_rows(self._h))

    def norm_ratio(self) -> float:
        """computeNormRatio (apsm_noma_detector.cu:220-311) of the current model."""
        return float(self._lib.apsm_oracle_norm_ratio(self._h))

    def get_state(self) -> dict[str, np.ndarray]:
        r = self.rows()
        D = 2 * self.N
        dic = np.zeros((r, D)); y = np.zeros(r); a = np.zeros(r); w = np.zeros(D)
        self._lib.apsm_oracle_get_state(self._h, dic.ctypes.data, y.ctypes.data, a.ctypes.data, w.ctypes.data)
        return {"dictionary": dic, "y": y, "a": a, "w": w}

    def set_state(self, dictionary: np.ndarray, a: np.ndarray, w: np.ndarray) -> None:
        dic = np.ascontiguousarray(dictionary, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        w = np.ascontiguousarray(w, dtype=np.float64)
        if self._lib.apsm_oracle_set_state(self._h, dic.shape[0], dic.ctypes.data, a.ctypes.data, w.ctypes.data):
            raise ValueError("oracle: state larger than the dictionary")


# ------------------------------------------------------- reference library --

_ref_lib = None


def reference_available() -> bool:
    return REF_SO.exists()


def _load_ref() -> ctypes.CDLL:
    global _ref_lib
    if _ref_lib is None:
        lib = ctypes.CDLL(str(REF_SO))
        P = ctypes.c_void_p
        lib.ref_create.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.POINTER(P), ctypes.c_char_p, ctypes.c_size_t]
        lib.ref_create.restype = ctypes.c_int
        lib.ref_train.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(ctypes.c_float)]
        lib.ref_train.restype = ctypes.c_int
        lib.ref_detect.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint32, P, ctypes.POINTER(ctypes.c_float)]
        lib.ref_detect.restype = ctypes.c_int
        lib.ref_train_history.argtypes = [P, P, P, ctypes.c_uint32, ctypes.c_uint32, P, P, ctypes.c_uint32,
                                          ctypes.c_uint32, ctypes.c_float, P, ctypes.c_uint32, P,
                                          ctypes.POINTER(ctypes.c_float)]
        lib.ref_train_history.restype = ctypes.c_int
        lib.ref_norm_ratio.argtypes = [P, ctypes.POINTER(ctypes.c_float)]
        lib.ref_norm_ratio.restype = ctypes.c_int
        lib.ref_reset.argtypes = [P]
        lib.ref_destroy.argtypes = [P]
        lib.ref_run_users_threaded.argtypes = [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, P, P,
                                               ctypes.c_uint32, P, ctypes.c_uint32, P, ctypes.c_char_p,
                                               ctypes.c_size_t]
        lib.ref_run_users_threaded.restype = ctypes.c_int
        _ref_lib = lib
    return _ref_lib


class ReferenceDetector:
    """The reference's NomaDetector (built from its own sources), on the GPU."""

    def __init__(self, config: Mapping[str, Any] | str, num_antennas: int):
        self._lib = _load_ref()
        text = config if isinstance(config, str) else json.dumps(dict(config))
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if self._lib.ref_create(text.encode(), int(num_antennas), ctypes.byref(h), err, len(err)) != 0:
            raise ValueError(err.value.decode())
        self._h = h
        self.N = int(num_antennas)

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ref_destroy(self._h)
            self._h = None

    def train(self, rx: np.ndarray, tx: np.ndarray) -> float:
        rx = np.ascontiguousarray(rx, dtype=np.complex64)
        tx = np.ascontiguousarray(np.asarray(tx).reshape(-1), dtype=np.complex64)
        ms = ctypes.c_float()
        if self._lib.ref_train(self._h, rx.ctypes.data, tx.ctypes.data, self.N, tx.shape[0], ctypes.byref(ms)):
            raise RuntimeError("reference train failed")
        return ms.value

    def train_history(self, rx: np.ndarray, tx: np.ndarray, rx_val: np.ndarray, tx_val: np.ndarray, bps: int,
                      scale: float, max_steps: int = 1 << 16) -> tuple[np.ndarray, float]:
        """train() with a NomaValSet: (steps, 6) history and the train time (ms)."""
        rx = np.ascontiguousarray(rx, dtype=np.complex64)
        tx = np.ascontiguousarray(np.asarray(tx).reshape(-1), dtype=np.complex64)
        rxv = np.ascontiguousarray(rx_val, dtype=np.complex64)
        txv = np.ascontiguousarray(np.asarray(tx_val).reshape(-1), dtype=np.complex64)
        out = np.zeros((max_steps, 6), dtype=np.float32)
        n = ctypes.c_uint32()
        ms = ctypes.c_float()
        st = self._lib.ref_train_history(self._h, rx.ctypes.data, tx.ctypes.data, self.N, tx.shape[0],
                                         rxv.ctypes.data, txv.ctypes.data, txv.shape[0], int(bps), float(scale),
                                         out.ctypes.data, max_steps, ctypes.byref(n), ctypes.byref(ms))
        if st:
            raise RuntimeError(f"reference train (history) failed: {st}")
        return out[:n.value].copy(), ms.value

    def detect(self, rx: np.ndarray) -> tuple[np.ndarray, float]:
        rx = np.ascontiguousarray(rx, dtype=np.complex64)
        S = rx.shape[1]
        est = np.zeros(S, dtype=np.complex64)
        ms = ctypes.c_float()
        if self._lib.ref_detect(self._h, rx.ctypes.data, self.N, S, est.ctypes.data, ctypes.byref(ms)):
            raise RuntimeError("reference detect failed")
        return est, ms.value

    def norm_ratio(self) -> float:
        """ApsmNomaDetector::computeNormRatio of the reference detector."""
        v = ctypes.c_float()
        if self._lib.ref_norm_ratio(self._h, ctypes.byref(v)):
            raise RuntimeError("reference norm ratio failed")
        return v.value

    def reset_state(self):
        self._lib.ref_reset(self._h)


def reference_users_threaded(config: Mapping[str, Any], rx_train: np.ndarray, tx_train: np.ndarray,
                             rx_data: np.ndarray) -> np.ndarray:
    """The reference CLI's -p mode: one detector + host thread per user."""
    lib = _load_ref()
    rx_train = np.ascontiguousarray(rx_train, dtype=np.complex64)
    rx_data = np.ascontiguousarray(rx_data, dtype=np.complex64)
    tx = np.ascontiguousarray(tx_train, dtype=np.complex64)
    U, P = tx.shape
    N, S = rx_data.shape
    est = np.zeros((U, S), dtype=np.complex64)
    err = ctypes.create_string_buffer(512)
    rc = lib.ref_run_users_threaded(json.dumps(dict(config)).encode(), N, U, rx_train.ctypes.data, tx.ctypes.data,
                                    P, rx_data.ctypes.data, S, est.ctypes.data, err, len(err))
    if rc:
        raise RuntimeError(f"reference -p run failed ({rc}): {err.value.decode()}")
    return est
