"""The CPU oracle (test infrastructure): parameter handling, FP32 vs FP64
agreement, schedule semantics, and the reference's modulation / metrics."""
import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import synth
from libapsm_b200.modulation import Modulation, cli_symbol_errors


def test_reference_params_defaults(oracle_mod):
    p = oracle_mod.reference_params({"otype": "APSM"}, 8)
    assert p.window_size == 20 and p.sample_step == 2 and p.train_passes == 1
    assert p.dictionary_size == 685 and not p.start_full_window
    assert np.float32(p.gaussian_weight) == np.float32(0.5)
    assert np.float32(p.linear_weight) == np.float32(0.5)
    # gaussianKernelVariance 0.05 scaled by N^2 (apsm_noma_detector.cu:79-80)
    assert np.float32(p.gaussian_variance) == np.float32(np.float32(0.05) * np.float32(64))
    assert np.float32(p.eB) == np.float32(0.001)
    with pytest.raises(ValueError, match="Invalid key"):
        oracle_mod.reference_params({"otype": "APSM", "bogus": 1}, 8)


@pytest.mark.parametrize("cfg,seed,N,P,S,mod", [
    ({"otype": "APSM", "windowSize": 5, "gaussianKernelVariance": 0.5, "eB": 0.01}, 1, 4, 40, 64, "QPSK"),
    ({"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "sampleStep": 1}, 2, 6, 90, 64, "QAM16"),
    ({"otype": "APSM", "windowSize": 20, "startWithFullWindow": True}, 3, 8, 120, 64, "QPSK"),
    ({"otype": "APSM", "windowSize": 10, "dictionarySize": 40}, 4, 4, 100, 64, "QPSK"),  # ring wraps
])
def test_oracle_f32_matches_f64(oracle_mod, cfg, seed, N, P, S, mod):
    f = synth.generate_frame(seed, K=3, N=N, P=P, S=S, modulation=mod, snr_db=20)
    d32 = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32)
    d64 = oracle_mod.OracleDetector(cfg, N, oracle_mod.F64)
    d32.train(f.rx_train, f.tx_train[0])
    d64.train(f.rx_train, f.tx_train[0])
    e32, e64 = d32.detect(f.rx_data), d64.detect(f.rx_data)
    scale = np.max(np.abs(e64))
    assert np.max(np.abs(e32 - e64)) <= 1e-5 * scale
    assert d32.rows() == d64.rows() == min(2 * P, 2 * cfg.get("dictionarySize", 685))


def test_oracle_dictionary_is_dedup_of_pilots(oracle_mod):
    """Dictionary rows follow the reference's Dedup embedding (cuda_matrix_device.cuh:180-188, 288-296)."""
    f = synth.generate_frame(9, K=2, N=3, P=10, S=4)
    o = oracle_mod.OracleDetector({"otype": "APSM", "windowSize": 2}, 3)
    o.train(f.rx_train, f.tx_train[1])
    st = o.get_state()
    y = f.rx_train
    for n in range(10):
        np.testing.assert_array_equal(st["dictionary"][2 * n], np.concatenate([y[:, n].real, y[:, n].imag]))
        np.testing.assert_array_equal(st["dictionary"][2 * n + 1], np.concatenate([y[:, n].imag, -y[:, n].real]))
        assert st["y"][2 * n] == np.float32(f.tx_train[1, n].real)
        assert st["y"][2 * n + 1] == np.float32(f.tx_train[1, n].imag)


def test_oracle_window_semantics(oracle_mod):
    """With eB huge no projection fires (c = 0): coefficients stay 0.  With one
    step (P = 1) exactly the two new rows are updated."""
    f = synth.generate_frame(3, K=1, N=2, P=6, S=4)
    o = oracle_mod.OracleDetector({"otype": "APSM", "eB": 1e9}, 2)
    o.train(f.rx_train, f.tx_train[0])
    assert np.all(o.get_state()["a"] == 0)
    o = oracle_mod.OracleDetector({"otype": "APSM", "eB": 0.0}, 2)
    o.train(f.rx_train[:, :1], f.tx_train[0, :1])
    st = o.get_state()
    assert st["a"].shape == (2,) and np.all(st["a"] != 0)


def test_shuffle_permutation_is_a_permutation(oracle_mod):
    p = oracle_mod.shuffle_permutation(1000)
    assert sorted(p.tolist()) == list(range(1000))
    assert not np.array_equal(p, np.arange(1000))
    np.testing.assert_array_equal(p, oracle_mod.shuffle_permutation(1000))  # fixed seed {1..8}


# ------------------------------------------------------------ modulation --

@pytest.mark.parametrize("name", ["BPSK", "QPSK", "QAM16", "QAM64", "QAM256"])
def test_modulation_roundtrip(name):
    m = Modulation(name)
    rng = np.random.default_rng(0)
    bits = rng.integers(0, 2, size=(200 * m.bps,))
    sym = m.encode(bits)
    np.testing.assert_array_equal(m.hard_decode(sym), bits)
    # unit average energy over the full constellation
    allsym = m.symbol_bits(np.arange(1 << m.bps))
    assert abs(np.mean(np.abs(allsym) ** 2) - 1.0) < 1e-6


def test_modulation_gray_neighbours():
    m = Modulation("QAM16")
    pts = m.symbol_bits(np.arange(16)) * m.rev_scale
    for i in range(16):
        for j in range(16):
            if abs(abs(pts[i] - pts[j]) - 2.0) < 1e-4:  # nearest neighbours differ in one bit
                assert bin(i ^ j).count("1") == 1


def test_modulation_reference_values():
    # map_1d (modulation.cpp:107-120): Gray-coded bits -> -L+1..L-1
    m = Modulation("QAM16")
    assert np.float32(m.scale) == np.float32(1 / np.sqrt(10))
    q = Modulation("QPSK")
    np.testing.assert_allclose(q.symbol_bits(np.arange(4)) * np.sqrt(2),
                               [-1 - 1j, -1 + 1j, 1 - 1j, 1 + 1j], atol=1e-6)
    np.testing.assert_array_equal(Modulation._map_1d(np.arange(4), 4), [-3, -1, 3, 1])


def test_metrics():
    m = Modulation("QPSK")
    rng = np.random.default_rng(1)
    sym = m.symbol_bits(rng.integers(0, 4, 500))
    assert L.symbol_error_rate(sym, sym, m) == 0.0
    assert L.bit_error_rate(-sym, sym, m) == 1.0
    assert L.evm(sym, sym) == 0.0
    assert cli_symbol_errors(sym, sym, m) == 0


def test_synth_deterministic_and_shaped():
    a = synth.generate_frame(11, K=3, N=4, P=20, S=30, modulation="QAM16", snr_db=15)
    b = synth.generate_frame(11, K=3, N=4, P=20, S=30, modulation="QAM16", snr_db=15)
    np.testing.assert_array_equal(a.rx_train, b.rx_train)
    assert a.rx_train.shape == (4, 20) and a.rx_data.shape == (4, 30)
    assert a.tx_train.shape == (3, 20) and a.rx_train.dtype == np.complex64
