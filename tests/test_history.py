"""Training history: NomaDetector::train with a validation set (NomaValSet,
cpp/lib/noma/noma_train_history.cuh:64-99), which records after every training
step the EVM, SER and BER of the training symbols and of a validation set
(apsm_train.cu:147-156, noma_train_history.cu:65-248).

Golden fixtures hold the reference library's own history (fraunhoferhhi/libapsm
built from its sources, run on a B200 by tests/golden/make_golden.py history).
The CPU oracle is pinned against them; the B200 path is checked against both.

Tolerances: EVM to 2e-4 relative (sums of squares in another order, estimates
equal to ~1e-5); SER and BER are counts of decisions, which can flip for an
estimate within rounding of a decision boundary: per step at most one symbol
(SER) and two bits (BER) apart, in at most 3% of the steps."""
import json
from pathlib import Path

import numpy as np
import pytest

import libapsm_b200 as L

HERE = Path(__file__).resolve().parent
HIST = sorted((HERE / "golden").glob("golden_history_*.npz"))


def load(p):
    d = np.load(p)
    return {k: d[k] for k in d.files}, json.loads(str(d["config"]))


def assert_history_close(h, ref, n_train, n_val, bps):
    h = np.asarray(h, np.float64)
    ref = np.asarray(ref, np.float64)
    assert h.shape == ref.shape, (h.shape, ref.shape)
    if h.size == 0:
        return
    for c in (0, 3):
        np.testing.assert_allclose(h[:, c], ref[:, c], rtol=2e-4, atol=1e-6)
    bad = 0
    for c, n in ((1, n_train), (2, n_train * bps), (4, n_val), (5, n_val * bps)):
        diff = np.abs(np.rint(h[:, c] * n) - np.rint(ref[:, c] * n))
        limit = 1 if c in (1, 4) else 2
        assert diff.max() <= limit, (c, diff.max())
        bad += int(np.count_nonzero(diff))
    assert bad <= max(1, int(0.03 * h.shape[0])), bad


def oracle_history(oracle_mod, cfg, rxt, txt, rxd, txd, mod):
    # the oracle restates the reference, which has no trainVersion key
    cfg = {k: v for k, v in cfg.items() if k != "trainVersion"}
    o = oracle_mod.OracleDetector(cfg, rxt.shape[0], oracle_mod.F32)
    h = o.train(rxt, txt, val_set=(rxd, txd, mod.bps, mod.scale))
    return h, o


def test_history_fixtures_present():
    assert len(HIST) >= 5, "history fixtures missing: run tests/golden/make_golden.py history on a GPU box"


@pytest.mark.parametrize("path", HIST, ids=[p.stem for p in HIST])
def test_oracle_history_reproduces_reference(oracle_mod, path):
    d, cfg = load(path)
    mod = L.Modulation(str(d["modulation"]))
    h, _ = oracle_history(oracle_mod, cfg, d["rx_train"], d["tx_train"], d["rx_data"], d["tx_data"], mod)
    assert_history_close(h, d["hist_ref"], d["tx_train"].size, d["tx_data"].size, mod.bps)


def test_oracle_history_last_step_is_the_trained_model(oracle_mod):
    f = L.synth.generate_frame(11, K=2, N=4, P=48, S=40, modulation="QAM16", snr_db=25)
    mod = L.Modulation("QAM16")
    cfg = {"otype": "APSM", "windowSize": 6, "gaussianKernelVariance": 0.4}
    h, o = oracle_history(oracle_mod, cfg, f.rx_train, f.tx_train[0], f.rx_data, f.tx_data[0], mod)
    assert h.shape == (48, 6)  # 2P rows, sampleStep 2
    est = o.detect(f.rx_data)
    evm = float(np.sqrt(np.mean(np.abs(est - f.tx_data[0]) ** 2)))
    assert abs(h[-1, 3] - evm) <= 1e-5 * max(evm, 1e-3)
    assert h[-1, 4] == pytest.approx(L.symbol_error_rate(est, f.tx_data[0], mod), abs=1 / 40 + 1e-7)


def test_history_csv_format(tmp_path):
    hist = L.NomaTrainHistory(2, 0.70710677)
    hist.extend(np.array([[[0.5, 0.25, 0.125, 1.5, 0.0, 1e-7], [0.25, 0, 0, 0.75, 0.5, 0.25]]], np.float32))
    out = tmp_path / "h.csv"
    hist.to_csv(str(out))
    lines = out.read_text().splitlines()
    assert lines[0] == "step,train_evm,train_ser,train_ber,val_evm,val_ser,val_ber"
    assert lines[1] == "0,0.5,0.25,0.125,1.5,0,1e-07"
    assert lines[2] == "1,0.25,0,0,0.75,0.5,0.25"
    np.testing.assert_array_equal(hist.evm_val, [1.5, 0.75])


# ----------------------------------------------------------------- GPU --

CASES = {
    "qpsk_w8": (dict(seed=301, K=2, N=4, P=64, S=48, modulation="QPSK"),
                {"otype": "APSM", "windowSize": 8, "gaussianKernelVariance": 0.5, "eB": 0.01}),
    "qam16_defaults": (dict(seed=302, K=3, N=8, P=120, S=96, modulation="QAM16"), {"otype": "APSM"}),
    "qam16_incremental": (dict(seed=303, K=3, N=8, P=120, S=80, modulation="QAM16"),
                          {"otype": "APSM", "windowSize": 12, "trainVersion": "incremental"}),
    "qam64_evict_step3": (dict(seed=304, K=2, N=6, P=150, S=64, modulation="QAM64"),
                          {"otype": "APSM", "windowSize": 9, "sampleStep": 3, "dictionarySize": 40,
                           "gaussianKernelVariance": 0.2}),
    "bpsk_sfw": (dict(seed=305, K=2, N=4, P=90, S=70, modulation="BPSK"),
                 {"otype": "APSM", "windowSize": 7, "startWithFullWindow": True}),
    "n64_shuffle": (dict(seed=306, K=4, N=64, P=96, S=64, modulation="QPSK"),
                    {"otype": "APSM", "windowSize": 10, "trainingShuffle": True}),
    "qam16_norm_evict": (dict(seed=307, K=3, N=8, P=120, S=64, modulation="QAM16"),
                         {"otype": "APSM", "windowSize": 10, "gaussianKernelVariance": 0.5, "dictionarySize": 50,
                          "normConstraint": 0.05}),
}


def frame(fr):
    return L.synth.generate_frame(fr["seed"], K=fr["K"], N=fr["N"], P=fr["P"], S=fr["S"],
                                  modulation=fr["modulation"], snr_db=20)


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_b200_history_matches_oracle(oracle_mod, name):
    fr, cfg = CASES[name]
    f = frame(fr)
    mod = L.Modulation(fr["modulation"])
    ref, _ = oracle_history(oracle_mod, cfg, f.rx_train, f.tx_train[1], f.rx_data, f.tx_data[1], mod)
    det = L.NomaDetectorFactory.build(cfg, fr["N"])
    hist = L.NomaTrainHistory(mod.bps, mod.scale)
    det.train(f.rx_train, f.tx_train[1], val_set=(hist, f.rx_data, f.tx_data[1]))
    assert_history_close(hist.steps, ref, fr["P"], fr["S"], mod.bps)


@pytest.mark.gpu
@pytest.mark.parametrize("path", HIST, ids=[p.stem for p in HIST])
def test_b200_history_reproduces_reference(path):
    d, cfg = load(path)
    mod = L.Modulation(str(d["modulation"]))
    det = L.NomaDetectorFactory.build(cfg, d["rx_train"].shape[0])
    hist = L.NomaTrainHistory(mod.bps, mod.scale)
    det.train(d["rx_train"], d["tx_train"], val_set=(hist, d["rx_data"], d["tx_data"]))
    assert_history_close(hist.steps, d["hist_ref"], d["tx_train"].size, d["tx_data"].size, mod.bps)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["qam16_defaults", "qam16_incremental", "qam64_evict_step3"])
def test_b200_history_leaves_training_unchanged(name):
    fr, cfg = CASES[name]
    f = frame(fr)
    mod = L.Modulation(fr["modulation"])
    plain = L.NomaDetectorFactory.build(cfg, fr["N"])
    plain.train(f.rx_train, f.tx_train[0])
    withh = L.NomaDetectorFactory.build(cfg, fr["N"])
    hist = L.NomaTrainHistory(mod.bps, mod.scale)
    withh.train(f.rx_train, f.tx_train[0], val_set=(hist, f.rx_data, f.tx_data[0]))
    a, b = plain.get_state(), withh.get_state()
    for k in a:
        np.testing.assert_array_equal(a[k], b[k])
    est_a, _ = plain.detect(f.rx_data)
    est_b, _ = withh.detect(f.rx_data)
    np.testing.assert_array_equal(est_a, est_b)
    # the last step's validation metrics are those of the trained model
    evm = float(np.sqrt(np.mean(np.abs(est_b.astype(np.complex128) - f.tx_data[0]) ** 2)))
    assert abs(float(hist.evm_val[-1]) - evm) <= 1e-4 * evm


@pytest.mark.gpu
def test_b200_history_multi_user_matches_single_users():
    fr, cfg = CASES["qam16_defaults"]
    f = frame(fr)
    mod = L.Modulation(fr["modulation"])
    multi = L.NomaDetectorFactory.build(cfg, fr["N"], num_users=3)
    hm = L.NomaTrainHistory(mod.bps, mod.scale)
    multi.train(f.rx_train, f.tx_train, val_set=(hm, f.rx_data, f.tx_data))
    assert hm.per_user.shape == (3, fr["P"], 6)
    for u in range(3):
        det = L.NomaDetectorFactory.build(cfg, fr["N"])
        h1 = L.NomaTrainHistory(mod.bps, mod.scale)
        det.train(f.rx_train, f.tx_train[u], val_set=(h1, f.rx_data, f.tx_data[u]))
        np.testing.assert_allclose(hm.per_user[u], h1.steps, rtol=1e-6, atol=1e-7)


@pytest.mark.gpu
def test_b200_history_second_call_appends(oracle_mod):
    fr, cfg = CASES["qam64_evict_step3"]
    f = frame(fr)
    mod = L.Modulation(fr["modulation"])
    half = fr["P"] // 2
    o = oracle_mod.OracleDetector(cfg, fr["N"], oracle_mod.F32)
    det = L.NomaDetectorFactory.build(cfg, fr["N"])
    for sl in (slice(0, half), slice(half, fr["P"])):
        ref = o.train(f.rx_train[:, sl], f.tx_train[0, sl], val_set=(f.rx_data, f.tx_data[0], mod.bps, mod.scale))
        hist = L.NomaTrainHistory(mod.bps, mod.scale)
        det.train(f.rx_train[:, sl], f.tx_train[0, sl], val_set=(hist, f.rx_data, f.tx_data[0]))
        assert_history_close(hist.steps, ref, sl.stop - sl.start, fr["S"], mod.bps)


@pytest.mark.gpu
def test_b200_history_lls_records_nothing():
    f = frame(CASES["qpsk_w8"][0])
    det = L.NomaDetectorFactory.build({"otype": "LLS"}, 4)
    hist = L.NomaTrainHistory(2, L.Modulation("QPSK").scale)
    det.train(f.rx_train, f.tx_train[0], val_set=(hist, f.rx_data, f.tx_data[0]))
    assert hist.steps.shape == (0, 6)
