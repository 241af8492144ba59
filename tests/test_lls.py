"""LLS linear detector (reference: cpp/lib/noma/lls_detector.cu) and APSM's
llsInitialization (cpp/lib/apsm/apsm_noma_detector.cu:98-99, 321-346):
against an FP64 least-squares restatement, the reference library's own output
(golden fixture), and the reference library run live on the GPU."""
import json
from pathlib import Path

import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import synth

GOLDEN_LLS = Path(__file__).resolve().parent / "golden" / "golden_lls_config0_like.npz"


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def test_lls_restatement_matches_reference_golden(oracle_mod):
    if not GOLDEN_LLS.exists():
        pytest.skip("LLS golden fixture not generated")
    d = np.load(GOLDEN_LLS)
    w = oracle_mod.lls_weights(d["rx_train"], d["tx_train"])
    est = oracle_mod.lls_detect(d["rx_data"], w)
    assert rel(est, d["est_ref"]) < 1e-4


def test_lls_config_rejects_apsm_keys(native_lib):
    with pytest.raises(ValueError, match="Invalid key: windowSize"):
        L.NomaDetectorFactory.build({"otype": "LLS", "windowSize": 80}, 8)


@pytest.mark.gpu
def test_lls_matches_fp64_least_squares(oracle_mod):
    f = synth.generate_frame(41, K=4, N=8, P=300, S=512, modulation="QAM16")
    det = L.NomaDetectorFactory.build({"otype": "LLS"}, 8, num_users=4)
    det.train(f.rx_train, f.tx_train)
    est, _ = det.detect(f.rx_data)
    for u in range(4):
        ref = oracle_mod.lls_detect(f.rx_data, oracle_mod.lls_weights(f.rx_train, f.tx_train[u]))
        assert rel(est[u], ref) < 1e-4
        assert L.symbol_error_rate(est[u], f.tx_data[u], f.modulation) == L.symbol_error_rate(
            ref, f.tx_data[u], f.modulation)


@pytest.mark.gpu
def test_lls_matches_reference_golden():
    if not GOLDEN_LLS.exists():
        pytest.skip("LLS golden fixture not generated")
    d = np.load(GOLDEN_LLS)
    det = L.NomaDetectorFactory.build({"otype": "LLS"}, d["rx_train"].shape[0])
    det.train(d["rx_train"], d["tx_train"])
    est, _ = det.detect(d["rx_data"])
    assert rel(est, d["est_ref"]) < 1e-4


@pytest.mark.gpu
def test_lls_initialization_matches_oracle_and_reference(oracle_mod):
    f = synth.generate_frame(42, K=3, N=8, P=200, S=256, modulation="QAM16")
    cfg = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "llsInitialization": True}
    det = L.NomaDetectorFactory.build(cfg, 8)
    det.train(f.rx_train, f.tx_train[1])
    est, _ = det.detect(f.rx_data)
    o = oracle_mod.OracleDetector(cfg, 8, oracle_mod.F32)
    o.train(f.rx_train, f.tx_train[1])
    assert rel(est, o.detect(f.rx_data)) < 1e-4
    if oracle_mod.reference_available():
        r = oracle_mod.ReferenceDetector(cfg, 8)
        r.train(f.rx_train, f.tx_train[1])
        er, _ = r.detect(f.rx_data)
        assert rel(est, er) < 1e-4


@pytest.mark.gpu
def test_lls_large_features_many_users(oracle_mod):
    # 128 real features, 16 users (right-hand sides): the in-house FP64 normal-equation
    # solve against the FP64 least-squares restatement
    f = synth.generate_frame(42, K=16, N=64, P=500, S=300, modulation="QAM16", snr_db=15)
    det = L.NomaDetectorFactory.build({"otype": "LLS"}, 64, num_users=16)
    det.train(f.rx_train, f.tx_train)
    est, _ = det.detect(f.rx_data)
    for u in (0, 7, 15):
        ref = oracle_mod.lls_detect(f.rx_data, oracle_mod.lls_weights(f.rx_train, f.tx_train[u]))
        assert rel(est[u], ref) < 1e-4


@pytest.mark.gpu
def test_lls_too_few_pilots_is_an_error():
    f = synth.generate_frame(43, K=2, N=16, P=10, S=20, modulation="QPSK")
    det = L.NomaDetectorFactory.build({"otype": "LLS"}, 16)
    with pytest.raises(ValueError, match="at least as many"):
        det.train(f.rx_train, f.tx_train[0])
