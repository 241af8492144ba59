"""Golden fixtures: estimates of the reference library itself (fraunhoferhhi/
libapsm built from its sources, run on a B200 by tests/golden/make_golden.py)
on seeded synthetic frames and on a slice of the reference's captured testbed
data.  The CPU oracle is pinned against them (no GPU needed); the B200
detector is checked against them on the GPU.

Tolerance: 1e-4 relative to the largest estimate magnitude (the FP32 bar);
the reference's own run-to-run spread, stored in each fixture, is ~5e-7."""
import json
from pathlib import Path

import numpy as np
import pytest

import libapsm_b200 as L

GOLDEN = sorted((Path(__file__).resolve().parent / "golden").glob("golden_*.npz"))
APSM = [p for p in GOLDEN if "lls" not in p.name and "norm_ratio" not in p.name]


def load(p):
    d = np.load(p)
    return {k: d[k] for k in d.files}, json.loads(str(d["config"]))


def close(est, ref, rtol=1e-4):
    scale = max(float(np.max(np.abs(ref))), 1e-30)
    return float(np.max(np.abs(est - ref))) <= rtol * scale


def test_golden_fixtures_present():
    assert len(APSM) >= 7, "golden fixtures missing: run tests/golden/make_golden.py run on a GPU box"


@pytest.mark.parametrize("path", APSM, ids=[p.stem for p in APSM])
def test_oracle_fp32_reproduces_reference(oracle_mod, path):
    d, cfg = load(path)
    N = d["rx_train"].shape[0]
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F32)
    o.train(d["rx_train"], d["tx_train"])
    est = o.detect(d["rx_data"])
    assert close(est, d["est_ref"], 1e-5), float(np.max(np.abs(est - d["est_ref"])))
    mod = L.Modulation(str(d["modulation"]))
    np.testing.assert_array_equal(mod.hard_decode_int(est), mod.hard_decode_int(d["est_ref"]))


@pytest.mark.parametrize("path", APSM, ids=[p.stem for p in APSM])
def test_oracle_fp64_close_to_reference(oracle_mod, path):
    d, cfg = load(path)
    o = oracle_mod.OracleDetector(cfg, d["rx_train"].shape[0], oracle_mod.F64)
    o.train(d["rx_train"], d["tx_train"])
    assert close(o.detect(d["rx_data"]), d["est_ref"], 1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("path", APSM, ids=[p.stem for p in APSM])
def test_b200_reproduces_reference(path):
    d, cfg = load(path)
    det = L.NomaDetectorFactory.build(cfg, d["rx_train"].shape[0])
    det.train(d["rx_train"], d["tx_train"])
    est, _ = det.detect(d["rx_data"])
    assert close(est, d["est_ref"]), float(np.max(np.abs(est - d["est_ref"])))
    mod = L.Modulation(str(d["modulation"]))
    assert L.symbol_error_rate(est, d["tx_data"], mod) == L.symbol_error_rate(d["est_ref"], d["tx_data"], mod)
