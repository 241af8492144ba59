"""Seeded synthetic NOMA uplink frames (the workload generator).

The reference ships captured testbed data but no channel model, so the
benchmark configurations are generated here:
  * K users send i.i.d. uniform symbols of the reference's Gray-mapped
    constellations (unit average energy, ``Modulation``).
  * Each user's signal passes a Rapp power amplifier
        |out| = |in| / (1 + (|in| / A_sat)^(2p))^(1/(2p)),  phase kept,
    driven ``backoff_db`` below saturation power (input scaled by
    A_sat * 10^(-backoff/20)).
  * Flat Rayleigh channel H (N x K, i.i.d. CN(0, 1)), fixed per frame.
  * AWGN per antenna at ``snr_db`` relative to the mean received signal power
    of the frame.
Pilots are the first P symbols of the frame, data the next S.  The generator
is numpy's PCG64 (``numpy.random.default_rng(seed)``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .modulation import Modulation


@dataclass
class Frame:
    rx_train: np.ndarray  # (N, P) complex64
    rx_data: np.ndarray   # (N, S) complex64
    tx_train: np.ndarray  # (K, P) complex64 (constellation symbols, unit energy)
    tx_data: np.ndarray   # (K, S) complex64
    H: np.ndarray         # (N, K) complex128
    modulation: Modulation
    snr_db: float


def rapp(x: np.ndarray, p: float, a_sat: float = 1.0) -> np.ndarray:
    r = np.abs(x)
    return x / (1.0 + (r / a_sat) ** (2 * p)) ** (1.0 / (2 * p))


def generate_frame(seed: int, K: int, N: int, P: int, S: int, modulation: str = "QPSK", snr_db: float = 20.0,
                   rapp_p: float = 2.0, backoff_db: float = 3.0, a_sat: float = 1.0) -> Frame:
    rng = np.random.default_rng(seed)
    mod = Modulation(modulation)
    T = P + S
    ints = rng.integers(0, 1 << mod.bps, size=(K, T))
    sym = mod.symbol_bits(ints).astype(np.complex128)               # (K, T)
    drive = a_sat * 10.0 ** (-backoff_db / 20.0)
    pa = rapp(sym * drive, rapp_p, a_sat)
    H = (rng.standard_normal((N, K)) + 1j * rng.standard_normal((N, K))) / np.sqrt(2.0)
    clean = H @ pa                                                  # (N, T)
    p_sig = float(np.mean(np.abs(clean) ** 2))
    sigma2 = p_sig / 10.0 ** (snr_db / 10.0)
    noise = np.sqrt(sigma2 / 2.0) * (rng.standard_normal((N, T)) + 1j * rng.standard_normal((N, T)))
    rx = (clean + noise).astype(np.complex64)
    tx = sym.astype(np.complex64)
    return Frame(rx_train=np.ascontiguousarray(rx[:, :P]), rx_data=np.ascontiguousarray(rx[:, P:]),
                 tx_train=np.ascontiguousarray(tx[:, :P]), tx_data=np.ascontiguousarray(tx[:, P:]),
                 H=H, modulation=mod, snr_db=snr_db)


# Workloads of the benchmark configurations (sizes as specified for each).
def config0_frame(seed: int = 0) -> Frame:
    """K=6 QPSK users, N=8, 20 dB, Rapp p=2 / 3 dB back-off, 600 pilots, 1800 data symbols."""
    return generate_frame(seed, K=6, N=8, P=600, S=1800, modulation="QPSK", snr_db=20.0, rapp_p=2.0)


def config1_frame(seed: int = 1) -> Frame:
    """K=8 16QAM users, N=16, 20 dB, 1000 pilots, 8000 data symbols."""
    return generate_frame(seed, K=8, N=16, P=1000, S=8000, modulation="QAM16", snr_db=20.0, rapp_p=2.0)


CONFIG0_ALGORITHM = {"otype": "APSM", "windowSize": 80, "gaussianKernelVariance": 0.5, "eB": 0.01}
CONFIG1_ALGORITHM = {"otype": "APSM", "windowSize": 80, "gaussianKernelVariance": 0.5, "eB": 0.01,
                     "dictionarySize": 1000}


# Batched workload: many independent detectors (users x cells).  Keys a
# configuration does not set keep the reference's defaults
# (apsm_parameters.cuh:68-86): gaussianKernelVariance 0.05, eB 0.001.
CONFIG2_ALGORITHM = {"otype": "APSM", "windowSize": 80, "dictionarySize": 2000}


@dataclass
class DetectorFrame:
    """One detector's frame: the cell's received pilots/data and its user's symbols."""

    rx_train: np.ndarray  # (N, P) complex64
    tx_train: np.ndarray  # (P,) complex64
    rx_data: np.ndarray   # (N, S) complex64
    tx_data: np.ndarray   # (S,) complex64
    modulation: Modulation
    snr_db: float

    @property
    def N(self) -> int:
        return self.rx_train.shape[0]

    @property
    def P(self) -> int:
        return self.rx_train.shape[1]

    @property
    def S(self) -> int:
        return self.rx_data.shape[1]


def config2_detectors(n: int = 512, seed: int = 2, users_per_cell: int = 4,
                      pilots: tuple[int, int] = (200, 2000), data: tuple[int, int] = (1000, 16000)) -> list[DetectorFrame]:
    """n detectors: antennas uniform over {4, 8, 16, 32}, pilots uniform over
    [200, 2000], data symbols over [1000, 16000], SNR over [10, 25] dB, QPSK or
    16QAM with probability 1/2, Rapp PA p=2 at 3 dB back-off; detector i's
    frame is drawn with seed 1000 * seed + i (its cell has users_per_cell
    users, the detector detects user 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        N = int(rng.choice([4, 8, 16, 32]))
        P = int(rng.integers(pilots[0], pilots[1] + 1))
        S = int(rng.integers(data[0], data[1] + 1))
        snr = float(rng.uniform(10.0, 25.0))
        mod = "QPSK" if rng.random() < 0.5 else "QAM16"
        f = generate_frame(1000 * seed + i, K=users_per_cell, N=N, P=P, S=S, modulation=mod, snr_db=snr, rapp_p=2.0)
        out.append(DetectorFrame(f.rx_train, np.ascontiguousarray(f.tx_train[0]), f.rx_data,
                                 np.ascontiguousarray(f.tx_data[0]), f.modulation, snr))
    return out


@dataclass
class ServedDetector:
    """A resident detector of the serving workload: the frame it is first
    trained on, then one pilot chunk and one data chunk that its per-TTI
    requests take prefixes of (same channel)."""

    frame: DetectorFrame
    pilots_rx: np.ndarray   # (N, 64) complex64
    pilots_tx: np.ndarray   # (64,) complex64
    data_rx: np.ndarray     # (N, 4000) complex64
    data_tx: np.ndarray     # (4000,) complex64


def config4_population(n: int = 512, seed: int = 4, users_per_cell: int = 4) -> list[ServedDetector]:
    """Detectors of the serving workload, sizes as config2_detectors: each is
    trained on its frame's pilots first; its TTIs append 16-64 pilots and
    detect 500-4000 symbols."""
    out = []
    for d in config2_detectors(n, seed=seed, users_per_cell=users_per_cell, data=(4000, 4000)):
        # the frame's data symbols feed the TTIs: first 64 as pilots, the rest as data
        out.append(ServedDetector(d, d.rx_data[:, :64].copy(), d.tx_data[:64].copy(),
                                  np.ascontiguousarray(d.rx_data), np.ascontiguousarray(d.tx_data)))
    return out


def config4_requests(pop: list[ServedDetector], rate_hz: float, duration_s: float, seed: int = 5):
    """Poisson arrivals at rate_hz over duration_s: (arrival time, detector
    index, kind, length) with each detector alternating train (16-64 new
    pilots) and detect (500-4000 symbols), starting with a train."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    phase = np.zeros(len(pop), np.int8)
    while True:
        t += float(rng.exponential(1.0 / rate_hz))
        if t >= duration_s:
            break
        d = int(rng.integers(0, len(pop)))
        if phase[d] == 0:
            out.append((t, d, "train", int(rng.integers(16, 65))))
        else:
            out.append((t, d, "detect", int(rng.integers(500, 4001))))
        phase[d] ^= 1
    return out
