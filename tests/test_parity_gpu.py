"""GPU parity of the B200 detector (through the C ABI) against the FP32 oracle
(the reference's evaluation order on the CPU), the FP64 oracle, and the
reference library built from its sources, on seeded synthetic frames.

Tolerances (FP32 form): soft outputs within 1e-4 relative to the largest
soft-output magnitude of the frame; hard decisions identical except where a
soft output lies within 1e-4 of a decision boundary.  Measured agreement is
~3e-7 (oracle) and ~2e-6 (reference; its own run-to-run spread is ~5e-7
because it adds the linear-weight updates with float atomics)."""
import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import synth

pytestmark = pytest.mark.gpu

RTOL = 1e-4


def assert_soft_close(est, ref, rtol=RTOL):
    est = np.asarray(est)
    ref = np.asarray(ref)
    assert est.shape == ref.shape
    if ref.size == 0:
        return
    scale = max(float(np.max(np.abs(ref))), 1e-30)
    err = float(np.max(np.abs(est - ref)))
    assert err <= rtol * scale, f"max |est - ref| = {err:.3e} > {rtol:.0e} * {scale:.3e}"


def assert_hard_equal(est, ref, mod):
    e = mod.hard_decode_int(est)
    r = mod.hard_decode_int(ref)
    near = np.minimum(mod.boundary_distance(est), mod.boundary_distance(ref)) < 1e-4
    bad = (e != r) & ~near
    assert not np.any(bad), f"{int(bad.sum())} hard decisions differ away from a boundary"


def run_product(cfg, f, u=0, users=None):
    N = f.rx_train.shape[0]
    if users is None:
        det = L.NomaDetectorFactory.build(cfg, N)
        det.train(f.rx_train, f.tx_train[u])
    else:
        det = L.NomaDetectorFactory.build(cfg, N, num_users=users)
        det.train(f.rx_train, f.tx_train[:users])
    est, _ = det.detect(f.rx_data)
    return det, est


def run_oracle(oracle_mod, cfg, f, u=0, prec=None, second=None):
    N = f.rx_train.shape[0]
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32 if prec is None else prec)
    o.train(f.rx_train, f.tx_train[u])
    if second is not None:
        o.train(second.rx_train, second.tx_train[u])
    return o, o.detect(f.rx_data)


BASE = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01}

CASES = [
    ("tiny", dict(BASE, windowSize=5), (5, 2, 4, 40, 50, "QPSK")),
    ("N1", dict(BASE, windowSize=4), (6, 2, 1, 30, 33, "QPSK")),
    ("P1", dict(BASE), (7, 2, 4, 1, 10, "QPSK")),
    ("S1", dict(BASE), (8, 2, 4, 50, 1, "QPSK")),
    ("defaults", {"otype": "APSM"}, (9, 3, 8, 120, 64, "QAM16")),
    ("sfw", dict(BASE, startWithFullWindow=True), (10, 3, 6, 150, 100, "QAM16")),
    ("step1", dict(BASE, sampleStep=1), (10, 3, 6, 150, 100, "QAM16")),
    ("step3", dict(BASE, sampleStep=3), (10, 3, 6, 151, 100, "QAM16")),
    ("passes2", dict(BASE, trainPasses=2, dictionarySize=150), (10, 3, 6, 150, 100, "QAM16")),
    ("passes0", dict(BASE, trainPasses=0), (10, 3, 6, 150, 100, "QAM16")),
    ("wrap", dict(BASE, dictionarySize=60), (10, 3, 6, 150, 100, "QAM16")),
    ("window>P", dict(BASE, windowSize=200, dictionarySize=300), (10, 3, 6, 150, 100, "QAM16")),
    ("wG0.8", dict(BASE, gaussianKernelWeight=0.8), (11, 3, 6, 150, 100, "QAM16")),
    ("wG1", dict(BASE, gaussianKernelWeight=1.0), (11, 3, 6, 150, 100, "QAM16")),
    ("wG0", dict(BASE, gaussianKernelWeight=0.0), (11, 3, 6, 150, 100, "QAM16")),
    ("var0", dict(BASE, gaussianKernelVariance=0.0), (12, 3, 6, 150, 100, "QAM16")),
    ("shuffle", dict(BASE, trainingShuffle=True), (12, 3, 6, 150, 100, "QAM16")),
    ("N64", dict(BASE, windowSize=16), (13, 4, 64, 100, 70, "QAM16")),
    ("N16-oldfast", dict(BASE, windowSize=40, detectVersion="oldfast"), (14, 4, 16, 300, 200, "QAM64")),
    ("config0", synth.CONFIG0_ALGORITHM, (0, 6, 8, 600, 1800, "QPSK")),
    # normConstraint: every bound below is active (the unconstrained model's RKHS norm is larger)
    ("norm", dict(BASE, windowSize=10, normConstraint=0.05), (108, 3, 8, 96, 96, "QAM16")),
    ("norm-w80", dict(BASE, windowSize=80, normConstraint=0.1), (15, 3, 8, 300, 100, "QAM16")),
    ("norm-wrap", dict(BASE, dictionarySize=60, normConstraint=0.05), (10, 3, 6, 150, 100, "QAM16")),
    ("norm-N32", dict(BASE, windowSize=12, normConstraint=0.003), (16, 3, 32, 100, 64, "QAM16")),
    ("norm-passes2", dict(BASE, windowSize=10, trainPasses=2, dictionarySize=96, normConstraint=0.05),
     (108, 3, 8, 96, 96, "QAM16")),
]


@pytest.mark.parametrize("name,cfg,frame", CASES, ids=[c[0] for c in CASES])
def test_product_matches_oracle_fp32(oracle_mod, name, cfg, frame):
    seed, K, N, P, S, mod = frame
    f = synth.generate_frame(seed, K=K, N=N, P=P, S=S, modulation=mod, snr_db=20)
    det, est = run_product(cfg, f)
    o, eo = run_oracle(oracle_mod, cfg, f)
    assert det.rows() == o.rows()
    assert_soft_close(est, eo, rtol=1e-5)
    assert_hard_equal(est, eo, f.modulation)
    st, so = det.get_state(), o.get_state()
    np.testing.assert_array_equal(st["dictionary"], so["dictionary"].astype(np.float32))
    assert_soft_close(st["a"][0], so["a"], rtol=1e-5)
    assert_soft_close(st["w"][0], so["w"], rtol=1e-5)


def test_product_matches_oracle_fp64_config0(oracle_mod):
    f = synth.config0_frame()
    _, est = run_product(synth.CONFIG0_ALGORITHM, f)
    _, e64 = run_oracle(oracle_mod, synth.CONFIG0_ALGORITHM, f, prec=oracle_mod.F64)
    assert_soft_close(est, e64, rtol=1e-5)


def test_second_train_call_appends(oracle_mod):
    f = synth.generate_frame(20, K=3, N=6, P=150, S=100, modulation="QAM16")
    g = synth.generate_frame(21, K=3, N=6, P=70, S=10, modulation="QAM16")
    for cfg in (BASE, dict(BASE, dictionarySize=100), dict(BASE, dictionarySize=100, normConstraint=0.05)):
        det = L.NomaDetectorFactory.build(cfg, 6)
        det.train(f.rx_train, f.tx_train[0])
        det.train(g.rx_train, g.tx_train[0])
        est, _ = det.detect(f.rx_data)
        o, eo = run_oracle(oracle_mod, cfg, f, second=g)
        assert det.rows() == o.rows()
        assert_soft_close(est, eo, rtol=1e-5)


def test_reset_state_gives_fresh_detector():
    f = synth.generate_frame(22, K=2, N=4, P=80, S=64)
    det = L.NomaDetectorFactory.build(BASE, 4)
    det.train(f.rx_train, f.tx_train[0])
    e1, _ = det.detect(f.rx_data)
    det.reset_state()
    assert det.rows() == 0
    e0, _ = det.detect(f.rx_data)
    assert np.all(e0 == 0)  # untrained model: zero coefficients
    det.train(f.rx_train, f.tx_train[0])
    e2, _ = det.detect(f.rx_data)
    np.testing.assert_array_equal(e1, e2)  # deterministic


def test_norm_constraint_binds_and_multi_user_equals_single():
    f = synth.generate_frame(108, K=3, N=8, P=96, S=96, modulation="QAM16", snr_db=20)
    cfg = dict(BASE, windowSize=10, normConstraint=0.05)
    _, free = run_product(dict(BASE, windowSize=10), f)
    _, bound = run_product(cfg, f)
    assert float(np.max(np.abs(free - bound))) > 1e-3  # the bound changes the model
    _, est = run_product(cfg, f, users=3)
    for u in range(3):
        _, e1 = run_product(cfg, f, u=u)
        np.testing.assert_array_equal(est[u], e1)


def test_norm_constraint_with_incremental_sweep_runs_the_exact_sweep():
    # normConstraint rescales every coefficient after each step (apsm_train.cu:142-145), which the
    # incremental sweep's running sums do not follow: such detectors train with the exact sweep
    f = synth.generate_frame(108, K=3, N=8, P=96, S=96, modulation="QAM16")
    cfg = dict(BASE, windowSize=10, normConstraint=0.05)
    _, e_exact = run_product(cfg, f)
    _, e_inc = run_product(dict(cfg, trainVersion="incremental"), f)
    np.testing.assert_array_equal(e_inc, e_exact)


def test_multi_user_equals_single_user_runs():
    f = synth.config1_frame()
    cfg = synth.CONFIG1_ALGORITHM
    _, est = run_product(cfg, f, users=8)
    for u in (0, 5, 7):
        _, e1 = run_product(cfg, f, u=u)
        np.testing.assert_array_equal(est[u], e1)


def test_device_entry_points_match_host_entry_points():
    import torch

    f = synth.generate_frame(23, K=3, N=8, P=200, S=256, modulation="QAM16")
    det = L.NomaDetectorFactory.build(BASE, 8, num_users=3)
    det.train(f.rx_train, f.tx_train)
    e_host, _ = det.detect(f.rx_data)
    det2 = L.NomaDetectorFactory.build(BASE, 8, num_users=3)
    rx = torch.from_numpy(f.rx_train).cuda()
    tx = torch.from_numpy(f.tx_train).cuda()
    rxd = torch.from_numpy(f.rx_data).cuda()
    est = torch.zeros((3, 256), dtype=torch.complex64, device="cuda")
    det2.train_device(rx, tx)
    det2.detect_device(rxd, est)
    det2.synchronize()
    np.testing.assert_array_equal(est.cpu().numpy(), e_host)


# ------------------------------------------------ reference library on the GPU --

def _ref(oracle_mod):
    if not oracle_mod.reference_available():
        pytest.skip("reference library not built (oracle/Makefile ref)")
    return oracle_mod


# The reference's BALANCED detect skips feature loads in its last block when
# fewer than D of that block's 32 samples exist (early return before the
# block barrier, apsm_detect.cu:852-853 + :765): those samples come out wrong.
# Parity frames therefore use 2S that is a multiple of 32.
REF_CASES = [
    ("small", dict(BASE, windowSize=5), (5, 2, 4, 40, 48, "QPSK")),
    ("shuffle", dict(BASE, trainingShuffle=True), (12, 3, 6, 150, 96, "QAM16")),
    ("var0", dict(BASE, gaussianKernelVariance=0.0), (12, 3, 6, 150, 96, "QAM16")),
    ("sfw-step1", dict(BASE, startWithFullWindow=True, sampleStep=1), (10, 3, 6, 150, 96, "QAM16")),
    ("passes2", dict(BASE, trainPasses=2, dictionarySize=150), (10, 3, 6, 150, 96, "QAM16")),
    ("config0", synth.CONFIG0_ALGORITHM, (0, 6, 8, 600, 1808, "QPSK")),
]


@pytest.mark.parametrize("name,cfg,frame", REF_CASES, ids=[c[0] for c in REF_CASES])
def test_product_matches_reference_library(oracle_mod, name, cfg, frame):
    O = _ref(oracle_mod)
    seed, K, N, P, S, mod = frame
    f = synth.generate_frame(seed, K=K, N=N, P=P, S=S, modulation=mod, snr_db=20)
    _, est = run_product(cfg, f, u=1)
    r = O.ReferenceDetector(cfg, N)
    r.train(f.rx_train, f.tx_train[1])
    er, _ = r.detect(f.rx_data)
    assert_soft_close(est, er)
    assert_hard_equal(est, er, f.modulation)


def test_product_matches_reference_all_users_config1(oracle_mod):
    O = _ref(oracle_mod)
    f = synth.config1_frame()
    cfg = synth.CONFIG1_ALGORITHM
    _, est = run_product(cfg, f, users=8)
    er = O.reference_users_threaded(cfg, f.rx_train, f.tx_train, f.rx_data)
    for u in range(8):
        assert_soft_close(est[u], er[u])
        assert_hard_equal(est[u], er[u], f.modulation)
        ser_b = L.symbol_error_rate(est[u], f.tx_data[u], f.modulation)
        ser_r = L.symbol_error_rate(er[u], f.tx_data[u], f.modulation)
        assert abs(ser_b - ser_r) <= 2.0 / f.tx_data.shape[1]


# ------------------------------------------------ incremental training sweep --
# "trainVersion": "incremental" keeps each window row's Gaussian sum up to date
# instead of re-summing it in the reference's order; the FP32 bar (1e-4
# relative) applies.

INC_CASES = [c for c in CASES if "normConstraint" not in c[1]]  # normConstraint: exact sweep only


@pytest.mark.parametrize("name,cfg,frame", INC_CASES, ids=[c[0] for c in INC_CASES])
def test_incremental_sweep_matches_oracle(oracle_mod, name, cfg, frame):
    seed, K, N, P, S, mod = frame
    f = synth.generate_frame(seed, K=K, N=N, P=P, S=S, modulation=mod, snr_db=20)
    det, est = run_product(dict(cfg, trainVersion="incremental"), f)
    o, eo = run_oracle(oracle_mod, cfg, f)
    assert det.rows() == o.rows()
    assert_soft_close(est, eo)
    assert_hard_equal(est, eo, f.modulation)


def test_incremental_sweep_second_train_and_users(oracle_mod):
    f = synth.generate_frame(20, K=3, N=6, P=150, S=100, modulation="QAM16")
    g = synth.generate_frame(21, K=3, N=6, P=70, S=10, modulation="QAM16")
    for cfg in (BASE, dict(BASE, dictionarySize=100)):
        det = L.NomaDetectorFactory.build(dict(cfg, trainVersion="incremental"), 6, num_users=3)
        det.train(f.rx_train, f.tx_train)
        det.train(g.rx_train, g.tx_train)
        est, _ = det.detect(f.rx_data)
        for u in range(3):
            o = oracle_mod.OracleDetector(cfg, 6, oracle_mod.F32)
            o.train(f.rx_train, f.tx_train[u])
            o.train(g.rx_train, g.tx_train[u])
            assert_soft_close(est[u], o.detect(f.rx_data))


def test_incremental_sweep_config1_all_users(oracle_mod):
    f = synth.config1_frame()
    cfg = synth.CONFIG1_ALGORITHM
    _, est = run_product(dict(cfg, trainVersion="incremental"), f, users=8)
    for u in (0, 7):
        _, eo = run_oracle(oracle_mod, cfg, f, u=u)
        assert_soft_close(est[u], eo)
        assert_hard_equal(est[u], eo, f.modulation)


# ------------------------------------------- coefficient rings in global memory --
# Dictionaries whose coefficient ring does not fit the exact sweep's shared
# memory (N = 64 with dictionarySize 8192: a 32768-entry ring beside 256 window
# rows of 132 floats) keep one private ring per CTA in global memory.  The
# summation order is unchanged, so the FP32 bar is the exact sweep's own.
# APSM_TRAIN_GLOBAL_RING=1 selects that form for any size, so the eviction,
# multi-pass and normConstraint paths are covered at sizes the oracle finishes.

GLOBAL_RING_CASES = [c for c in CASES if c[0] in ("wrap", "passes2", "sfw", "window>P", "N64", "norm-wrap",
                                                   "norm-passes2", "config0")]


@pytest.mark.parametrize("name,cfg,frame", GLOBAL_RING_CASES, ids=[c[0] for c in GLOBAL_RING_CASES])
def test_global_coefficient_ring_matches_oracle(oracle_mod, monkeypatch, name, cfg, frame):
    monkeypatch.setenv("APSM_TRAIN_GLOBAL_RING", "1")
    seed, K, N, P, S, mod = frame
    f = synth.generate_frame(seed, K=K, N=N, P=P, S=S, modulation=mod, snr_db=20)
    det, est = run_product(cfg, f)
    o, eo = run_oracle(oracle_mod, cfg, f)
    assert det.rows() == o.rows()
    assert_soft_close(est, eo, rtol=1e-5)
    assert_hard_equal(est, eo, f.modulation)
    assert_soft_close(det.get_state()["a"][0], o.get_state()["a"], rtol=1e-5)


def test_global_coefficient_ring_users_and_append(oracle_mod, monkeypatch):
    monkeypatch.setenv("APSM_TRAIN_GLOBAL_RING", "1")
    f = synth.generate_frame(20, K=3, N=6, P=150, S=100, modulation="QAM16")
    g = synth.generate_frame(21, K=3, N=6, P=70, S=10, modulation="QAM16")
    cfg = dict(BASE, dictionarySize=100)
    det = L.NomaDetectorFactory.build(cfg, 6, num_users=3)
    det.train(f.rx_train, f.tx_train)
    det.train(g.rx_train, g.tx_train)
    est, _ = det.detect(f.rx_data)
    for u in range(3):
        o = oracle_mod.OracleDetector(cfg, 6, oracle_mod.F32)
        o.train(f.rx_train, f.tx_train[u])
        o.train(g.rx_train, g.tx_train[u])
        assert_soft_close(est[u], o.detect(f.rx_data), rtol=1e-5)


def test_large_dictionary_n64_matches_oracle(oracle_mod):
    # precision-study sizes (N = 64, dictionarySize 8192) with a short pilot
    # sequence: the shape search itself falls back to global rings here
    cfg = dict(BASE, windowSize=80, dictionarySize=8192)
    f = synth.generate_frame(31, K=4, N=64, P=240, S=200, modulation="QAM16", snr_db=15)
    det, est = run_product(cfg, f, users=4)
    for u in (0, 3):
        _, eo = run_oracle(oracle_mod, cfg, f, u=u)
        assert_soft_close(est[u], eo, rtol=1e-5)
        assert_hard_equal(est[u], eo, f.modulation)
