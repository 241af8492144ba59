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
