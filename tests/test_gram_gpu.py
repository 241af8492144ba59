"""Tensor-core detection forms of the single detector (detectVersion gram_*)
against a float64 evaluation of the same trained model.

One detector trains in the exact FP32 form; its state is copied
(apsm_copy_state) into one detector per Gram form, and every form's soft
outputs are compared with the FP64 oracle holding the same state
(apsm_oracle_set_state).  The bound for each form, relative to the largest
soft-output magnitude of the frame, follows from its operand precision: the
cross term x.d carries a relative error of about 2^-8 (bf16), 2^-11 (tf32),
2^-16 (bf16x3) or 2^-21 (tf32x3) of |x||d|, which reaches the Gaussian term
scaled by 2 |ew| |x||d|; the single-product forms recompute the entries where
that bound is large exactly, which keeps them within 2e-3."""
import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import synth

pytestmark = pytest.mark.gpu

BASE = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01}
# relative soft-output bound of each form (the exact form is its own FP32 bar)
BOUNDS = {"balanced": 1e-5, "gram_tf32x3": 2e-5, "gram_bf16x3": 1e-4, "gram_tf32": 2e-3, "gram_bf16": 2e-3}

CASES = [  # name, (seed, K users, N, P, S, modulation), users detected, extra config
    ("N8-u1", (40, 3, 8, 150, 300, "QPSK"), 1, {}),
    ("N16-u3", (41, 4, 16, 200, 257, "QAM16"), 3, {}),
    ("N32-u4", (42, 4, 32, 300, 129, "QAM16"), 4, {"dictionarySize": 200}),
    ("N64-u16", (43, 16, 64, 200, 160, "QAM16"), 16, {"windowSize": 40}),
]


def oracle_fp64(oracle_mod, cfg, N, state, u, rx):
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F64)
    o.set_state(state["dictionary"], state["a"][u], state["w"][u])
    return o.detect(rx)


@pytest.mark.parametrize("name,frame,users,extra", CASES, ids=[c[0] for c in CASES])
def test_gram_forms_match_fp64_model(oracle_mod, name, frame, users, extra):
    seed, K, N, P, S, mod = frame
    f = synth.generate_frame(seed, K=K, N=N, P=P, S=S, modulation=mod, snr_db=20)
    cfg = dict(BASE, **extra)
    base = L.NomaDetectorFactory.build(cfg, N, num_users=users)
    base.train(f.rx_train, f.tx_train[:users])
    state = base.get_state()
    refs = [oracle_fp64(oracle_mod, cfg, N, state, u, f.rx_data) for u in range(users)]
    scale = max(float(np.max(np.abs(r))) for r in refs)
    for form, bound in BOUNDS.items():
        det = L.NomaDetectorFactory.build(dict(cfg, detectVersion=form), N, num_users=users)
        if form != "balanced":
            det.copy_state_from(base)
            st = det.get_state()
            np.testing.assert_array_equal(st["dictionary"], state["dictionary"])
            np.testing.assert_array_equal(st["a"], state["a"])
            np.testing.assert_array_equal(st["w"], state["w"])
        else:
            det = base
        est, _ = det.detect(f.rx_data)
        est = est.reshape(users, S)
        err = max(float(np.max(np.abs(est[u] - refs[u]))) for u in range(users)) / scale
        print(f"{name} {form}: max soft error {err:.3e} of the largest soft output")
        assert err <= bound, (form, err)


def test_copy_state_rejects_mismatched_detectors():
    a = L.NomaDetectorFactory.build(BASE, 8, num_users=2)
    for other in (L.NomaDetectorFactory.build(BASE, 4, num_users=2),
                  L.NomaDetectorFactory.build(BASE, 8, num_users=1),
                  L.NomaDetectorFactory.build(dict(BASE, dictionarySize=100), 8, num_users=2),
                  L.NomaDetectorFactory.build(dict(BASE, gaussianKernelWeight=0.7), 8, num_users=2),
                  L.NomaDetectorFactory.build(dict(BASE, gaussianKernelVariance=0.25), 8, num_users=2)):
        with pytest.raises(ValueError):
            other.copy_state_from(a)


def test_copy_state_takes_heuristic_variance_and_continues_training(oracle_mod):
    # a detector whose variance comes from the heuristic hands it over with the model;
    # the copy then trains on exactly as the original would
    f = synth.generate_frame(44, K=2, N=8, P=120, S=200, modulation="QAM16")
    g = synth.generate_frame(45, K=2, N=8, P=60, S=10, modulation="QAM16")
    cfg = dict(BASE, gaussianKernelVariance=0.0, dictionarySize=100)
    a = L.NomaDetectorFactory.build(cfg, 8)
    a.train(f.rx_train, f.tx_train[0])
    b = L.NomaDetectorFactory.build(cfg, 8)
    b.copy_state_from(a)
    assert b.gaussian_variance == a.gaussian_variance
    a.train(g.rx_train, g.tx_train[0])
    b.train(g.rx_train, g.tx_train[0])
    np.testing.assert_array_equal(a.detect(f.rx_data)[0], b.detect(f.rx_data)[0])


def test_bf16_two_product_form_matches_one_product(monkeypatch):
    # 4+ users in the BF16 form contract on the tensor cores (kernel values and
    # coefficients in BF16); APSM_GRAM_ONE_PRODUCT=1 keeps the users' sums on the
    # CUDA cores.  Both stay within the BF16 bound of the float64 model; against each
    # other they agree to the BF16 rounding of the second product.
    f = synth.generate_frame(46, K=8, N=32, P=400, S=700, modulation="QAM16", snr_db=15)
    cfg = dict(BASE, detectVersion="gram_bf16")
    base = L.NomaDetectorFactory.build(BASE, 32, num_users=8)
    base.train(f.rx_train, f.tx_train)
    two = L.NomaDetectorFactory.build(cfg, 32, num_users=8)
    two.copy_state_from(base)
    monkeypatch.setenv("APSM_GRAM_ONE_PRODUCT", "1")
    one = L.NomaDetectorFactory.build(cfg, 32, num_users=8)
    one.copy_state_from(base)
    e2, _ = two.detect(f.rx_data)
    e1, _ = one.detect(f.rx_data)
    scale = float(np.max(np.abs(e1)))
    err = float(np.max(np.abs(e2 - e1))) / scale
    assert 0 < err < 1e-3, err
    for _ in range(2):  # repeatable
        np.testing.assert_array_equal(two.detect(f.rx_data)[0], e2)
