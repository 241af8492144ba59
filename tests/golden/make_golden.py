#!/usr/bin/env python3
"""Generate the golden fixtures of the parity tests (test infrastructure).

The reference has no tests and stores no expected outputs, so the fixtures
are produced by running the reference library itself — fraunhoferhhi/libapsm
compiled from its sources for sm_100a by oracle/Makefile (oracle/_ref/
libapsm_ref.so) — through its public API (NomaDetectorFactory::build ->
train -> detect) on a B200.

  python tests/golden/make_golden.py capture
      (where the reference tree is mounted) extracts a small slice of the
      reference's captured testbed data, cpp/data/offline, into
      tests/golden/captured_qpsk_inputs.npz
  python tests/golden/make_golden.py run --out DIR
      (on a GPU box) runs the reference library on every case and writes
      DIR/golden_<case>.npz: inputs, config and the reference's estimates.
  python tests/golden/make_golden.py normratio --out DIR
      (on a GPU box) trains the reference on every golden_<case>.npz and
      writes DIR/golden_norm_ratio.npz: its computeNormRatio per case.
  python tests/golden/make_golden.py history --out DIR
      (on a GPU box) trains the reference with a validation set and writes
      DIR/golden_history_<case>.npz: inputs, config, the per-step history.

Synthetic cases use libapsm_b200.synth with fixed seeds; 2S is a multiple of
32 in every case (the reference BALANCED detect mis-handles a partial last
block, see tests/test_parity_gpu.py), and so is 2P in the history cases, whose
training-set metrics run that detection on the pilots.
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

def _reference_dir() -> Path:
    """The fraunhoferhhi/libapsm checkout whose captured data and library this
    script runs (environment variable APSM_REFERENCE_DIR)."""
    import os

    d = os.environ.get("APSM_REFERENCE_DIR")
    if not d:
        raise SystemExit("make_golden.py: set APSM_REFERENCE_DIR to the libapsm checkout (its cpp/data/offline "
                         "holds the captured frames)")
    p = Path(d) / "cpp" / "data" / "offline"
    if not p.is_dir():
        raise SystemExit(f"make_golden.py: {p} not found: APSM_REFERENCE_DIR must be the libapsm checkout")
    return p

CASES = {
    "qpsk_small": (dict(seed=101, K=2, N=4, P=64, S=64, modulation="QPSK"),
                   {"otype": "APSM", "windowSize": 8, "gaussianKernelVariance": 0.5, "eB": 0.01}),
    "qam16_defaults": (dict(seed=102, K=3, N=8, P=120, S=112, modulation="QAM16"), {"otype": "APSM"}),
    "config0_like": (dict(seed=103, K=6, N=8, P=300, S=304, modulation="QPSK"),
                     {"otype": "APSM", "windowSize": 80, "gaussianKernelVariance": 0.5, "eB": 0.01}),
    "sfw_step1": (dict(seed=104, K=3, N=6, P=100, S=96, modulation="QAM16"),
                  {"otype": "APSM", "windowSize": 15, "startWithFullWindow": True, "sampleStep": 1,
                   "gaussianKernelVariance": 0.3, "eB": 0.005}),
    "passes2": (dict(seed=105, K=3, N=6, P=100, S=96, modulation="QAM16"),
                {"otype": "APSM", "windowSize": 10, "trainPasses": 2, "dictionarySize": 100}),
    "shuffle_var0": (dict(seed=106, K=3, N=6, P=100, S=96, modulation="QAM16"),
                     {"otype": "APSM", "windowSize": 10, "trainingShuffle": True, "gaussianKernelVariance": 0.0}),
    "wG08_detect_oldfast": (dict(seed=107, K=4, N=16, P=200, S=208, modulation="QAM16"),
                            {"otype": "APSM", "windowSize": 40, "gaussianKernelWeight": 0.8,
                             "gaussianKernelVariance": 0.2, "eB": 0.02, "detectVersion": "oldfast"}),
    # normConstraint (apsm_train.cu:142-145, 190-256): 0.05 is below the unconstrained model's
    # RKHS norm (0.14), so the coefficients are scaled back after most steps
    "norm_constraint": (dict(seed=108, K=3, N=8, P=96, S=96, modulation="QAM16"),
                        {"otype": "APSM", "windowSize": 10, "gaussianKernelVariance": 0.5,
                         "normConstraint": 0.05}),
}
CAPTURED_CFG = {"otype": "APSM", "windowSize": 80}  # the README example's algorithm config
USER = 1


def capture() -> None:
    """Slice of the captured QPSK (time-domain) data: 8 equidistant antennas,
    user 1, first 160 pilots and 192 data symbols, tx scaled by 1/sqrt(2)
    (loadData with Modulation::getScale, binary_load.cpp:55-81)."""
    from libapsm_b200 import binfile

    rx = binfile.read(_reference_dir() / "rx" / "time" / "rxData_QPSK_alltx_converted.bin")
    tx = binfile.read(_reference_dir() / "tx" / "NOMA_signals_qpsk_complex.bin")
    ant = [i * 16 // 8 for i in range(8)]  # antennaPatternEquidistant(8), util.cpp:264-272
    scale = np.float32(1.0 / np.sqrt(2.0))
    rxt = binfile.complex_matrix(rx["rxSigTraining"])[ant, :160]
    rxd = binfile.complex_matrix(rx["rxSigData"])[ant, :192]
    txt = binfile.complex_matrix(tx["mod_training"], scale)[:, :160]
    txd = binfile.complex_matrix(tx["mod_data"], scale)[:, :192]
    np.savez_compressed(HERE / "captured_qpsk_inputs.npz", rx_train=rxt, rx_data=rxd, tx_train=txt, tx_data=txd,
                        source="cpp/data/offline/rx/time/rxData_QPSK_alltx_converted.bin + "
                               "cpp/data/offline/tx/NOMA_signals_qpsk_complex.bin")
    print("wrote", HERE / "captured_qpsk_inputs.npz")


def run(out: Path, only: set[str] | None = None) -> None:
    from libapsm_b200 import synth
    from oracle import oracle as O

    out.mkdir(parents=True, exist_ok=True)
    todo = []
    for name, (fr, cfg) in CASES.items():
        if only and name not in only:
            continue
        f = synth.generate_frame(fr["seed"], K=fr["K"], N=fr["N"], P=fr["P"], S=fr["S"], modulation=fr["modulation"],
                                 snr_db=20)
        todo.append((name, cfg, f.rx_train, f.tx_train, f.rx_data, f.tx_data, fr["modulation"]))
    cap = np.load(HERE / "captured_qpsk_inputs.npz")
    if not only or "captured_qpsk" in only:
        todo.append(("captured_qpsk", CAPTURED_CFG, cap["rx_train"], cap["tx_train"], cap["rx_data"],
                     cap["tx_data"], "QPSK"))
    for name, cfg, rxt, txt, rxd, txd, mod in todo:
        r = O.ReferenceDetector(cfg, rxt.shape[0])
        tms = r.train(rxt, txt[USER])
        est, dms = r.detect(rxd)
        r2 = O.ReferenceDetector(cfg, rxt.shape[0])
        r2.train(rxt, txt[USER])
        est2, _ = r2.detect(rxd)
        spread = float(np.max(np.abs(est - est2)))
        np.savez_compressed(out / f"golden_{name}.npz", config=json.dumps(cfg), user=USER, modulation=mod,
                            rx_train=rxt, tx_train=txt[USER], rx_data=rxd, tx_data=txd[USER], est_ref=est,
                            ref_run_to_run=spread, ref_train_ms=tms, ref_detect_ms=dms)
        print(f"{name}: ref train {tms:.3f} ms detect {dms:.3f} ms, run-to-run max |d| {spread:.2e}")
    if only and "lls" not in only:
        return
    # LLS reference outputs on one case (the reference's cuBLAS least-squares detector)
    name, cfg, rxt, txt, rxd, txd, mod = todo[2]
    r = O.ReferenceDetector({"otype": "LLS"}, rxt.shape[0])
    r.train(rxt, txt[USER])
    est, _ = r.detect(rxd)
    np.savez_compressed(out / "golden_lls_config0_like.npz", config=json.dumps({"otype": "LLS"}), user=USER,
                        modulation=mod, rx_train=rxt, tx_train=txt[USER], rx_data=rxd, tx_data=txd[USER], est_ref=est)
    print("lls: done")


# Training-history cases: (frame, algorithm config, modulation).  The reference
# records EVM / SER / BER of the training rows and a validation set after every
# step (NomaValSet, apsm_train.cu:147-156).
HISTORY_CASES = {
    "qpsk_small": (dict(seed=201, K=2, N=4, P=64, S=64, modulation="QPSK"),
                   {"otype": "APSM", "windowSize": 8, "gaussianKernelVariance": 0.5, "eB": 0.01}),
    "qam16_sfw_step1": (dict(seed=202, K=3, N=6, P=112, S=96, modulation="QAM16"),
                        {"otype": "APSM", "windowSize": 15, "startWithFullWindow": True, "sampleStep": 1,
                         "gaussianKernelVariance": 0.3, "eB": 0.005}),
    "qam16_passes2_shuffle": (dict(seed=203, K=3, N=6, P=96, S=96, modulation="QAM16"),
                              {"otype": "APSM", "windowSize": 10, "trainPasses": 2, "dictionarySize": 96,
                               "trainingShuffle": True}),
    "bpsk_var0": (dict(seed=204, K=2, N=4, P=128, S=64, modulation="BPSK"),
                  {"otype": "APSM", "windowSize": 6, "gaussianKernelVariance": 0.0}),
    "qam16_norm": (dict(seed=205, K=3, N=8, P=96, S=96, modulation="QAM16"),
                   {"otype": "APSM", "windowSize": 10, "gaussianKernelVariance": 0.5, "normConstraint": 0.05}),
}
# 2P and 2S are multiples of 32 (see the module docstring).  A case with more
# pilots than the dictionary holds (2P > 2 dictionarySize) is kept apart as
# race_<case>.npz: there the reference's result depends on a data race
# (tests/test_reference_eviction.py).
RACE_CASES = {
    "bpsk_evict": (dict(seed=204, K=2, N=4, P=120, S=64, modulation="BPSK"),
                   {"otype": "APSM", "windowSize": 6, "dictionarySize": 30, "gaussianKernelVariance": 0.4}),
}


def history(out: Path, only: set[str] | None = None) -> None:
    from libapsm_b200 import synth
    from libapsm_b200.modulation import Modulation
    from oracle import oracle as O

    out.mkdir(parents=True, exist_ok=True)
    todo = []
    for name, (fr, cfg) in HISTORY_CASES.items():
        if only and name not in only:
            continue
        f = synth.generate_frame(fr["seed"], K=fr["K"], N=fr["N"], P=fr["P"], S=fr["S"], modulation=fr["modulation"],
                                 snr_db=20)
        todo.append((name, cfg, f.rx_train, f.tx_train[USER], f.rx_data, f.tx_data[USER], fr["modulation"]))
    cap = np.load(HERE / "captured_qpsk_inputs.npz")
    if not only or "captured_qpsk" in only:
        todo.append(("captured_qpsk", CAPTURED_CFG, cap["rx_train"], cap["tx_train"][USER], cap["rx_data"],
                     cap["tx_data"][USER], "QPSK"))
    for name, (fr, cfg) in RACE_CASES.items():
        if only and name not in only:
            continue
        f = synth.generate_frame(fr["seed"], K=fr["K"], N=fr["N"], P=fr["P"], S=fr["S"], modulation=fr["modulation"],
                                 snr_db=20)
        todo.append(("race:" + name, cfg, f.rx_train, f.tx_train[USER], f.rx_data, f.tx_data[USER],
                     fr["modulation"]))
    for name, cfg, rxt, txt, rxd, txd, mod in todo:
        m = Modulation(mod)
        r = O.ReferenceDetector(cfg, rxt.shape[0])
        hist, tms = r.train_history(rxt, txt, rxd, txd, m.bps, m.scale)
        est, _ = r.detect(rxd)
        fname = f"race_{name[5:]}.npz" if name.startswith("race:") else f"golden_history_{name}.npz"
        np.savez_compressed(out / fname, config=json.dumps(cfg), modulation=mod,
                            rx_train=rxt, tx_train=txt, rx_data=rxd, tx_data=txd, hist_ref=hist, est_ref=est,
                            ref_train_ms=tms)
        print(f"history {name}: {hist.shape[0]} steps, ref train {tms:.3f} ms, last {hist[-1]}")


def norm_ratio(out: Path) -> None:
    """computeNormRatio of the reference after training on each golden_<case>.npz."""
    from oracle import oracle as O

    vals = {}
    for f in sorted(HERE.glob("golden_*.npz")):
        name = f.stem[len("golden_"):]
        if name.startswith(("lls", "history", "norm_ratio")):
            continue
        d = np.load(f)
        cfg = json.loads(str(d["config"]))
        r = O.ReferenceDetector(cfg, d["rx_train"].shape[0])
        r.train(d["rx_train"], d["tx_train"])
        vals[name] = np.float32(r.norm_ratio())
        print(f"norm ratio {name}: {vals[name]}")
    np.savez(out / "golden_norm_ratio.npz", **vals)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("mode", choices=["capture", "run", "history", "normratio"])
    ap.add_argument("--out", default=str(HERE))
    ap.add_argument("--cases", default="", help="comma-separated case names (default: all)")
    a = ap.parse_args()
    only = set(filter(None, a.cases.split(","))) or None
    if a.mode == "capture":
        capture()
    elif a.mode == "run":
        run(Path(a.out), only)
    elif a.mode == "normratio":
        norm_ratio(Path(a.out))
    else:
        history(Path(a.out), only)
