"""ApsmNomaDetector::computeNormRatio (cpp/lib/apsm/apsm_noma_detector.cu:
220-311): the ratio wL |w|^2 / (wG sum_ij a_i a_j k(d_i, d_j)) of a trained
model's linear to Gaussian norm.  tests/golden/golden_norm_ratio.npz holds the
reference library's value after training on each golden_<case>.npz (written by
tests/golden/make_golden.py normratio on a B200).  The oracle restates the
reference's summation order (1e-5); the B200 kernel uses the same order on a
model whose coefficients agree with the reference's to ~1e-6 (1e-4)."""
import json
from pathlib import Path

import numpy as np
import pytest

import libapsm_b200 as L

GOLDEN = Path(__file__).resolve().parent / "golden"
FIXTURE = GOLDEN / "golden_norm_ratio.npz"


def cases():
    if not FIXTURE.exists():
        return []
    return sorted(np.load(FIXTURE).files)


def load(name):
    d = np.load(GOLDEN / f"golden_{name}.npz")
    return d, json.loads(str(d["config"]))


def test_norm_ratio_fixture_present():
    assert len(cases()) >= 8, "run tests/golden/make_golden.py normratio on a GPU box"


@pytest.mark.parametrize("name", cases())
def test_oracle_norm_ratio_reproduces_reference(oracle_mod, name):
    d, cfg = load(name)
    o = oracle_mod.OracleDetector(cfg, d["rx_train"].shape[0], oracle_mod.F32)
    o.train(d["rx_train"], d["tx_train"])
    ref = float(np.load(FIXTURE)[name])
    assert o.norm_ratio() == pytest.approx(ref, rel=1e-5)


@pytest.mark.gpu
@pytest.mark.parametrize("name", cases())
def test_b200_norm_ratio_reproduces_reference(oracle_mod, name):
    d, cfg = load(name)
    det = L.NomaDetectorFactory.build(cfg, d["rx_train"].shape[0])
    det.train(d["rx_train"], d["tx_train"])
    ref = float(np.load(FIXTURE)[name])
    assert det.compute_norm_ratio() == pytest.approx(ref, rel=1e-4)
    o = oracle_mod.OracleDetector(cfg, d["rx_train"].shape[0], oracle_mod.F32)
    o.train(d["rx_train"], d["tx_train"])
    assert det.compute_norm_ratio() == pytest.approx(o.norm_ratio(), rel=1e-5)


@pytest.mark.gpu
def test_b200_norm_ratio_per_user_and_lls_refused():
    f = L.synth.generate_frame(41, K=3, N=6, P=120, S=32, modulation="QAM16")
    cfg = {"otype": "APSM", "windowSize": 12, "gaussianKernelVariance": 0.4}
    multi = L.NomaDetectorFactory.build(cfg, 6, num_users=3)
    multi.train(f.rx_train, f.tx_train)
    for u in range(3):
        single = L.NomaDetectorFactory.build(cfg, 6)
        single.train(f.rx_train, f.tx_train[u])
        assert multi.compute_norm_ratio(u) == pytest.approx(single.compute_norm_ratio(), rel=1e-6)
    with pytest.raises(ValueError):
        multi.compute_norm_ratio(3)
    lls = L.NomaDetectorFactory.build({"otype": "LLS"}, 6)
    lls.train(f.rx_train, f.tx_train[0])
    with pytest.raises(L.ApsmError):
        lls.compute_norm_ratio()

