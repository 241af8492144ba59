"""Constellations, hard decisions and error metrics of the reference CLI.

Restates cpp/cli/common/modulation.{hpp,cpp} and the metric helpers of
cpp/cli/common/util.cpp so that detector outputs are scored exactly as the
reference scores them:
  map_1d / map / encode      modulation.cpp:107-151 (Gray code, points at -L+1..L-1 step 2)
  demap_1d / demap / hardDecode  modulation.cpp:68-105
  getScale / getRevScale     modulation.hpp:157-204 (QPSK 1/sqrt(2), QAMx 1/sqrt((2^(b+1)-2)/3))
  bit errors                 util.cpp:112-141
  EVM                        util.cpp:143-192
Symbol errors are counted from hard decisions (any decoded bit wrong), not
with the CLI's printSymbolErrors whose imaginary-axis edge tests are inverted
(util.cpp:90-95 vs :81-85); ``cli_symbol_errors`` reproduces that printout
for comparison.
"""
from __future__ import annotations

import math

import numpy as np

BITS = {"OFF": 0, "BPSK": 1, "QPSK": 2, "QAM16": 4, "QAM64": 6, "QAM256": 8, "QAM1024": 10, "QAM4096": 12,
        "QAM16384": 14}


class Modulation:
    def __init__(self, name: str):
        key = name.upper()
        if key not in BITS:
            raise ValueError(f"Unsupported modulation: {key}")
        self.name = key
        self.bps = BITS[key]

    # modulation.hpp: scale converts integer grid -> unit energy (float)
    @property
    def scale(self) -> float:
        if self.bps == 0:
            return 0.0
        if self.bps <= 2:
            return float(np.float32(1.0 / math.sqrt(self.bps)))
        return float(np.float32(1.0 / math.sqrt(((2 << self.bps) - 2) // 3)))

    @property
    def rev_scale(self) -> float:
        if self.bps == 0:
            return 0.0
        if self.bps <= 2:
            return float(np.float32(math.sqrt(self.bps)))
        return float(np.float32(math.sqrt(((2 << self.bps) - 2) // 3)))

    @property
    def points_1d(self) -> int:
        return 2 if self.bps == 1 else 1 << (self.bps // 2)

    # ---- mapping --------------------------------------------------------
    @staticmethod
    def _map_1d(bits: np.ndarray, L: int) -> np.ndarray:
        g = bits.astype(np.int64).copy()
        b = bits.astype(np.int64).copy()
        while np.any(b):
            b >>= 1
            g ^= b
        return 2 * g - L + 1

    @staticmethod
    def _demap_1d(x: np.ndarray, L: int) -> np.ndarray:
        # float arithmetic of demap_1d; round() of C rounds half away from zero
        v = ((np.asarray(x, np.float32) + np.float32(L - 1)) / np.float32(2.0)).astype(np.float64)
        xi = np.where(v >= 0, np.floor(v + 0.5), np.ceil(v - 0.5)).astype(np.int64)
        xi = np.clip(xi, 0, L - 1)
        return xi ^ (xi >> 1)

    def symbol_bits(self, symbols_int: np.ndarray) -> np.ndarray:
        """Symbol index (bps-bit integer, MSB first) -> complex64 constellation point (unit energy)."""
        s = np.asarray(symbols_int, dtype=np.int64)
        if self.bps == 1:
            re = self._map_1d(s, 2).astype(np.float32)
            pts = re + 0j
        else:
            h = self.bps // 2
            L = 1 << h
            re = self._map_1d(s >> h, L).astype(np.float32)
            im = self._map_1d(s & (L - 1), L).astype(np.float32)
            pts = re + 1j * im
        return (pts * np.float32(self.scale)).astype(np.complex64)

    def encode(self, bits: np.ndarray) -> np.ndarray:
        """Modulation::encode: bit vector (MSB first per symbol) -> symbols."""
        b = np.asarray(bits, dtype=np.int64).reshape(-1, self.bps)
        weights = 1 << np.arange(self.bps - 1, -1, -1)
        return self.symbol_bits((b * weights).sum(axis=1))

    def hard_decode_int(self, est: np.ndarray) -> np.ndarray:
        """Symbol index decided for each estimate (demap of est * revScale)."""
        z = np.asarray(est, dtype=np.complex64) * np.float32(self.rev_scale)
        if self.bps == 1:
            return self._demap_1d(z.real, 2)
        h = self.bps // 2
        L = 1 << h
        return (self._demap_1d(z.real, L) << h) | self._demap_1d(z.imag, L)

    def hard_decode(self, est: np.ndarray) -> np.ndarray:
        """Modulation::hardDecode: bit vector, MSB first per symbol."""
        ints = self.hard_decode_int(est)
        shifts = np.arange(self.bps - 1, -1, -1)
        return ((ints[..., None] >> shifts) & 1).astype(np.uint8).reshape(*ints.shape[:-1], -1)

    def boundary_distance(self, est: np.ndarray) -> np.ndarray:
        """Distance (in unit-energy units) of each soft estimate to the nearest decision boundary."""
        z = np.asarray(est, dtype=np.complex128) * self.rev_scale
        L = self.points_1d

        def d1(v):
            # boundaries at even integers between -L+2 .. L-2 (grid coordinates)
            b = np.clip(np.round(v / 2.0) * 2.0, -L + 2, L - 2)
            return np.abs(v - b)

        if self.bps == 1:
            return d1(z.real) / self.rev_scale
        return np.minimum(d1(z.real), d1(z.imag)) / self.rev_scale


def symbol_error_rate(est: np.ndarray, ref: np.ndarray, mod: Modulation) -> float:
    e = mod.hard_decode_int(est)
    r = mod.hard_decode_int(ref)
    return float(np.mean(e != r))


def bit_error_rate(est: np.ndarray, ref: np.ndarray, mod: Modulation) -> float:
    """util.cpp:112-141 (printBitErrors), as a fraction."""
    return float(np.mean(mod.hard_decode(est) != mod.hard_decode(ref)))


def evm(est: np.ndarray, ref: np.ndarray) -> float:
    """util.cpp:143-192 (printEvm): sqrt(mean |est - ref|^2)."""
    d = np.abs(np.asarray(est, np.complex64) - np.asarray(ref, np.complex64)).astype(np.float32)
    return float(np.sqrt(np.sum(d * d, dtype=np.float32) / np.float32(d.size)))


def cli_symbol_errors(est: np.ndarray, ref: np.ndarray, mod: Modulation) -> int:
    """printSymbolErrors (util.cpp:62-110) including its inverted imaginary edge tests."""
    s = mod.scale
    mx = 1.0 if mod.bps == 1 else ((1 << (mod.bps // 2)) - 1) * s
    n = 0
    for y, t in zip(np.asarray(est), np.asarray(ref)):
        if np.isnan(abs(y)):
            n += 1
        elif (abs(y.real - t.real) > s and not (y.real > mx and t.real > mx - s)
              and not (y.real < -mx and t.real < -mx + s)):
            n += 1
        elif (abs(y.imag - t.imag) > s and not (y.imag > mx and t.imag < mx - s)
              and not (y.imag < -mx and t.imag > -mx + s) and mod.bps > 1):
            n += 1
    return n
