"""NOMA_detect: the reference's command line tool over the B200 detector.

Usage (``python -m libapsm_b200.cli`` takes the arguments of the reference's
``NOMA_detect``, cpp/cli/detect/noma_detect.cpp:59-148):

  -s/--synchronized-data FILE   rxSigTraining / rxSigData ([samples, antennas, 2])
  -r/--reference-data FILE      mod_training / mod_data (integer grid, scaled by
                                the modulation's scale on load)
  -rs/--random-seed SEED        reference symbols drawn like the reference CLI
                                (overrides -r; 6 users, 685 pilots, 3840 data)
  -d/--detected-data FILE       writes estSigData ([samples, 1, 2])
  -cf/--config-file FILE | -cs/--config-string JSON
                                {"algorithm": {...}, "modulation": "QAM16",
                                 "user": 0, "antennas": {"otype": "all"}}
  -o/--output-mode SER|BER|EVM|scripting
  -th/--train-history-file CSV  per-step train/validation EVM, SER, BER
  -p/--parallel-processing      all six users (one multi-user detector)

Behaviour follows the reference tool:
  * antenna selection, jsonGetAntennaPattern / selectAntennas
    (cpp/cli/common/util.cpp:194-289); the pattern is a 16-bit set whose
    bit i is the (M-1-i)-th of the first M <= 16 characters of "pattern";
  * reference data from a seed: std::mt19937(seed) feeding
    std::bernoulli_distribution(0.5) (one bit per two 32-bit draws through
    std::generate_canonical<double, 53>), mapped by Modulation::encode and
    split into users of 685 + 3840 symbols (util.cpp:291-325, util.hpp:66-104);
  * printouts of printSymbolErrors / printBitErrors / printEvm / printErrors
    (util.cpp:58-192), including the symbol-error printout's inverted
    imaginary-edge tests and "scripting" printing only "ber,ser,evm";
  * the "Train time = ... ms, detect time = ... ms" line and -d output of the
    single-user path; -p prints the errors of each of the six users.
The detector runs on the GPU through libapsm_b200.NomaDetector; with -p the
six users share one detector whose training updates all users in the same
kernels (the reference builds six detectors and trains them on six threads).
"""
from __future__ import annotations

import argparse
import json
import math
import random
import sys
from typing import IO, Sequence

import numpy as np

from . import binfile
from .modulation import Modulation

MAX_ANTENNAS = 16
DEFAULT_NUM_USERS = 6
# CONSTANTS of cpp/cli/common/util.hpp:66-104: (5 short OFDM symbols) / 16 and (4 slots) / 16
DEFAULT_TRAINING_SAMPLES = 5 * (2048 + 144) // 16
DEFAULT_DATA_SAMPLES = 4 * (1 * (2048 + 160) + 6 * (2048 + 144)) // 16
DEFAULT_CONFIG = '{ "algorithm": { "otype": "APSM" } }'

OUTPUT_MODES = ("BER", "SER", "EVM", "SCRIPTING")


# ---------------------------------------------------------------------------
# antenna patterns (util.cpp:194-289)
# ---------------------------------------------------------------------------
def pattern_from_string(text: str) -> list[bool]:
    """std::bitset<16>(text): the first M = min(16, len) characters, the last of them is bit 0."""
    m = min(MAX_ANTENNAS, len(text))
    bits = [False] * MAX_ANTENNAS
    for i in range(m):
        c = text[m - 1 - i]
        if c not in "01":
            raise ValueError("bitset::_M_copy_from_ptr")
        bits[i] = c == "1"
    return bits


def pattern_first(number: int) -> list[bool]:
    bits = [False] * MAX_ANTENNAS
    for i in range(number):
        bits[i] = True
    return bits


def pattern_equidistant(number: int) -> list[bool]:
    bits = [False] * MAX_ANTENNAS
    for i in range(number):
        bits[i * MAX_ANTENNAS // number] = True
    return bits


def pattern_random(number: int) -> list[bool]:
    """Like antennaPatternRandom: seeded from the OS entropy source, not reproducible."""
    idx = list(range(MAX_ANTENNAS))
    random.SystemRandom().shuffle(idx)
    bits = [False] * MAX_ANTENNAS
    for i in range(number):
        bits[idx[i]] = True
    return bits


def antenna_pattern(config: dict) -> list[bool]:
    """jsonGetAntennaPattern (util.cpp:194-216)."""
    for key in config:
        if key not in ("otype", "pattern", "number"):
            raise ValueError("Invalid key: " + key)
    otype = config.get("otype")
    number = int(config.get("number", 16))
    if otype == "all":
        return [True] * MAX_ANTENNAS
    if otype == "pattern":
        return pattern_from_string(config.get("pattern", "11111111111111111111"))
    if otype == "equidistant":
        return pattern_equidistant(number)
    if otype == "random":
        return pattern_random(number)
    if otype == "first":
        return pattern_first(number)
    raise ValueError(f"Invalid antenna scheme: {otype}")


def select_antennas(m: np.ndarray, pattern: Sequence[bool]) -> np.ndarray:
    """selectAntennas (util.cpp:274-289): rows idx < min(rows, 16) whose bit is set."""
    n = min(m.shape[0], len(pattern))
    keep = [i for i in range(n) if pattern[i]]
    return np.ascontiguousarray(m[keep])


# ---------------------------------------------------------------------------
# reference data from a seed (util.cpp:291-325)
# ---------------------------------------------------------------------------
def random_bits(seed: int, n: int) -> np.ndarray:
    """std::bernoulli_distribution(0.5) over std::mt19937(seed): bit = canonical < 0.5, where the
    canonical double is (g0 + g1 * 2^32) / 2^64 of two consecutive 32-bit outputs."""
    rs = np.random.RandomState(seed & 0xFFFFFFFF)  # init_genrand(seed): the std::mt19937 seeding
    raw = rs._bit_generator.random_raw(2 * n).astype(np.uint64)
    s = raw[0::2].astype(np.float64) + raw[1::2].astype(np.float64) * 4294967296.0
    u = s / 18446744073709551616.0
    u = np.where(u >= 1.0, np.nextafter(1.0, 0.0), u)
    return (u < 0.5).astype(np.uint8)


def random_reference_data(seed: int, modulation: Modulation, users: int = DEFAULT_NUM_USERS,
                          train: int = DEFAULT_TRAINING_SAMPLES,
                          data: int = DEFAULT_DATA_SAMPLES) -> tuple[np.ndarray, np.ndarray]:
    """generateReferenceData: one bit stream, user u takes symbols [u (T+D), (u+1)(T+D))."""
    if modulation.bps == 0:
        raise ValueError("modulation OFF carries no symbols")
    sym = modulation.encode(random_bits(seed, (train + data) * users * modulation.bps))
    sym = sym.reshape(users, train + data)
    return np.ascontiguousarray(sym[:, :train]), np.ascontiguousarray(sym[:, train:])


# ---------------------------------------------------------------------------
# printouts (util.cpp:58-192)
# ---------------------------------------------------------------------------
def print_symbol_errors(est: np.ndarray, ref: np.ndarray, mod: Modulation, out: IO[str]) -> float:
    s = np.float32(mod.scale)
    mx = np.float32(1.0) if mod.bps == 1 else np.float32(((1 << (mod.bps // 2)) - 1)) * s
    errors = 0
    chars = []
    for k, (y, t) in enumerate(zip(np.asarray(est, np.complex64), np.asarray(ref, np.complex64))):
        if k % 80 == 0:
            chars.append("\n")
        yr, yi, tr, ti = np.float32(y.real), np.float32(y.imag), np.float32(t.real), np.float32(t.imag)
        if math.isnan(abs(complex(y))):
            errors += 1
            chars.append("n")
        elif abs(yr - tr) > s and not (yr > mx and tr > mx - s) and not (yr < -mx and tr < -mx + s):
            errors += 1
            chars.append("r")
        elif (abs(yi - ti) > s and not (yi > mx and ti < mx - s) and not (yi < -mx and ti > -mx + s)
              and mod.bps > 1):
            errors += 1
            chars.append("i")
        else:
            chars.append(".")
    total = len(est)
    pct = float(np.float32(100.0 * errors / total)) if total else float("nan")
    out.write("".join(chars) + f" symbol errors: {errors} of {total} - {pct:.2f} percent\n")
    return pct


def print_bit_errors(est: np.ndarray, ref: np.ndarray, mod: Modulation, out: IO[str]) -> float:
    eb = mod.hard_decode(np.asarray(est, np.complex64)).reshape(-1)
    tb = mod.hard_decode(np.asarray(ref, np.complex64)).reshape(-1)
    chars = []
    bps = mod.bps
    for i in range(eb.size):
        if i % (bps * 80) == 0:
            chars.append("\n")
        if i % bps == 0:
            chars.append(" ")
        chars.append("x" if eb[i] != tb[i] else ".")
    errors = int(np.count_nonzero(eb != tb))
    pct = float(np.float32(100.0 * errors / eb.size)) if eb.size else float("nan")
    out.write("".join(chars) + f" bit errors: {errors} of {eb.size} - {pct:.2f} percent\n")
    return pct


_BARS = [" ", "▁", "▂", "▃", "▄", "▅", "▆", "▇"]


def print_evm(est: np.ndarray, ref: np.ndarray, out: IO[str]) -> float:
    err = np.abs(np.asarray(est, np.complex64) - np.asarray(ref, np.complex64)).astype(np.float32)
    chars = []
    for k, e in enumerate(err):
        if k % 80 == 0:
            chars.append("\n")
        level = e / np.float32(0.5) * np.float32(8)
        chars.append(_BARS[int(level)] if level < 8 else "█")
    sq = np.cumsum(err * err, dtype=np.float32)[-1] if err.size else np.float32(0)
    value = float(np.sqrt(np.float32(sq / np.float32(err.size)))) if err.size else float("nan")
    out.write("".join(chars) + f" EVM: {value:.4f}\n")
    return value


class _Null:
    def write(self, _s: str) -> int:
        return 0


def print_errors(mode: str, est: np.ndarray, ref: np.ndarray, mod: Modulation, out: IO[str]) -> None:
    """printErrors (util.cpp:156-192)."""
    if mode == "BER":
        print_bit_errors(est, ref, mod, out)
    elif mode == "SER":
        print_symbol_errors(est, ref, mod, out)
    elif mode == "EVM":
        print_evm(est, ref, out)
    else:
        quiet = _Null()
        ber = print_bit_errors(est, ref, mod, quiet)
        ser = print_symbol_errors(est, ref, mod, quiet)
        e = print_evm(est, ref, quiet)
        out.write(f"{ber:.6f},{ser:.6f},{e:.6f}\n")


def _cout_float(v: float) -> str:
    """operator<<(float) with the stream's default format (%g, 6 significant digits)."""
    return f"{v:g}"


# ---------------------------------------------------------------------------
# the tool
# ---------------------------------------------------------------------------
def make_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(
        prog="NOMA_detect",
        description="This tool runs the training and detection algorithms. The algorithm configuration is "
                    "passed in JSON format either as string or in a file.")
    p.add_argument("-s", "--synchronized-data", required=True,
                   help="synchronized data file containing received training and data signals")
    p.add_argument("-r", "--reference-data", help="reference data file")
    p.add_argument("-rs", "--random-seed", type=int,
                   help="random seed for generation of data (this overrides the --reference-data argument)")
    p.add_argument("-d", "--detected-data", help="detected (estimated) data file")
    p.add_argument("-cf", "--config-file", help="filename for JSON file containing the algorithm configuration")
    p.add_argument("-cs", "--config-string", default=DEFAULT_CONFIG,
                   help="JSON string containing the algorithm configuration")
    p.add_argument("-o", "--output-mode", default="SER",
                   help='print mode for error metric (BER, SER, EVM, scripting = only "ber,ser,evm")')
    p.add_argument("-th", "--train-history-file", default="",
                   help="filename for training history CSV-file (test set will be used as validation set)")
    p.add_argument("-p", "--parallel-processing", action="store_true", help="process all users in parallel")
    return p


def load_config(args: argparse.Namespace) -> dict:
    if args.config_file:
        with open(args.config_file) as f:
            return json.load(f)
    return json.loads(args.config_string)


def output_mode(text: str) -> str:
    mode = text.upper()
    if mode not in OUTPUT_MODES:
        raise ValueError("Invalid print mode: " + text)
    return mode


def load_inputs(args: argparse.Namespace, config: dict):
    """(rxSigTraining, rxSigData, txSigTraining, txSigData) as complex64 matrices."""
    synced = binfile.read(args.synchronized_data)
    rx_train = binfile.complex_matrix(synced["rxSigTraining"])
    rx_data = binfile.complex_matrix(synced["rxSigData"])
    mod = Modulation(config.get("modulation", "QAM16"))
    if args.random_seed is not None:
        tx_train, tx_data = random_reference_data(args.random_seed, mod)
    elif args.reference_data:
        ref = binfile.read(args.reference_data)
        tx_train = binfile.complex_matrix(ref["mod_training"], mod.scale)
        tx_data = binfile.complex_matrix(ref["mod_data"], mod.scale)
    else:
        raise ValueError("Neither --random-seed/-rs nor --reference-data/-r was specified")
    return rx_train, rx_data, tx_train, tx_data


def run(args: argparse.Namespace, out: IO[str]) -> int:
    from .detector import NomaDetectorFactory
    from .history import NomaTrainHistory

    config = load_config(args)
    rx_train, rx_data, tx_train, tx_data = load_inputs(args, config)
    mode = output_mode(args.output_mode)
    user = int(config.get("user", 0))
    mod = Modulation(config.get("modulation", "QAM16"))
    pattern = antenna_pattern(config.get("antennas", {"otype": "all"}))
    rx_train = select_antennas(rx_train, pattern)
    rx_data = select_antennas(rx_data, pattern)
    n_ant = sum(pattern)
    if rx_train.shape[0] != n_ant:
        raise ValueError(f"the antenna pattern selects {n_ant} antennas, the synchronized data holds "
                         f"{rx_train.shape[0]} of them")
    if "algorithm" not in config:
        raise ValueError("the configuration has no \"algorithm\" object")
    text_out = _Null() if mode == "SCRIPTING" else out

    if args.parallel_processing:
        users = DEFAULT_NUM_USERS
        if tx_train.shape[0] < users:
            raise ValueError(f"parallel processing detects {users} users, the reference data holds "
                             f"{tx_train.shape[0]}")
        with NomaDetectorFactory.build(config["algorithm"], n_ant, users) as det:
            det.train(rx_train, tx_train[:users])
            est, _ = det.detect(rx_data)
        for u in range(users):
            print_errors(mode, est[u], tx_data[u], mod, out if mode == "SCRIPTING" else text_out)
        return 0

    if not 0 <= user < tx_train.shape[0]:
        raise ValueError(f"user {user} is not in the reference data ({tx_train.shape[0]} users)")
    history = NomaTrainHistory(mod.bps, mod.scale) if args.train_history_file else None
    with NomaDetectorFactory.build(config["algorithm"], n_ant) as det:
        val_set = (history, rx_data, tx_data[user]) if history is not None else None
        train_ms = det.train(rx_train, tx_train[user], val_set=val_set)
        est, detect_ms = det.detect(rx_data)
    text_out.write(f"Train time = {_cout_float(train_ms)} ms, detect time = {_cout_float(detect_ms)} ms\n")
    print_errors(mode, est, tx_data[user], mod, out)
    if args.detected_data:
        binfile.write(args.detected_data, {"estSigData": binfile.to_array(est[None, :])})
    if history is not None:
        history.to_csv(args.train_history_file)
    return 0


def main(argv: Sequence[str] | None = None, out: IO[str] | None = None) -> int:
    args = make_parser().parse_args(argv)
    return run(args, out or sys.stdout)


if __name__ == "__main__":
    sys.exit(main())
