"""Tensor-core detection of points that coincide with dictionary rows.

Detection evaluates k(x, d) = exp(-||x - d||^2 / (2 s^2)) against every
dictionary row d; the reference forms the difference basis - data feature by
feature (cpp/lib/apsm/apsm_detect.cu:760-790), so points that coincide with a
row cost it no accuracy.  The Gram forms write ||x - d||^2 = ||x||^2 +
||d||^2 - 2 x.d, whose three terms cancel for x = d: the split forms (bf16x3,
tf32x3) carry the cross term to ~FP32 accuracy, the single-product forms (bf16,
tf32) flag the entries whose rounding error bound is large and recompute their
distance exactly.

The data detected here ARE the training pilots (exact duplicates of the
dictionary rows) or the pilots plus 1e-3 noise per component (near
duplicates).  Every Gram form is compared with a float64 evaluation of the same
trained model: within 2e-3 of the largest soft output for the single-product
forms, 1e-4 for the split forms, in the single detector (one- and two-product
kernels) and in the detector pool (pair form).
"""
import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import synth

pytestmark = pytest.mark.gpu

BOUND = {"gram_bf16": 2e-3, "gram_tf32": 2e-3, "gram_bf16x3": 1e-4, "gram_tf32x3": 1e-4}
BASE = {"otype": "APSM", "windowSize": 40, "eB": 0.001}


def _points(rx_train, kind):
    if kind == "exact":
        return rx_train.copy()
    rng = np.random.default_rng(5)
    noise = 1e-3 * (rng.standard_normal(rx_train.shape) + 1j * rng.standard_normal(rx_train.shape))
    return (rx_train + noise).astype(np.complex64)


def _fp64(oracle_mod, cfg, N, dictionary, a, w, rx):
    o = oracle_mod.OracleDetector(cfg, N, oracle_mod.F64)
    o.set_state(dictionary, a, w)
    return o.detect(rx)


# N antennas, users detected, gaussianKernelVariance (x N^2 by the detector)
SINGLE = [(3, 1, 0.05), (4, 2, 0.05), (8, 3, 0.5), (16, 8, 0.05), (32, 4, 0.05), (64, 16, 0.05)]


@pytest.mark.parametrize("kind", ["exact", "near"])
@pytest.mark.parametrize("N,users,var", SINGLE, ids=[f"N{n}-u{u}-v{v}" for n, u, v in SINGLE])
def test_single_detector_duplicates(oracle_mod, N, users, var, kind):
    P = 256
    f = synth.generate_frame(60 + N, K=max(users, 2), N=N, P=P, S=16, modulation="QAM16", snr_db=20)
    cfg = dict(BASE, gaussianKernelVariance=var, dictionarySize=P)
    base = L.NomaDetectorFactory.build(cfg, N, num_users=users)
    base.train(f.rx_train, f.tx_train[:users])
    state = base.get_state()
    x = _points(f.rx_train, kind)
    refs = [_fp64(oracle_mod, cfg, N, state["dictionary"], state["a"][u], state["w"][u], x) for u in range(users)]
    scale = max(float(np.max(np.abs(r))) for r in refs)
    for form, bound in BOUND.items():
        det = L.NomaDetectorFactory.build(dict(cfg, detectVersion=form), N, num_users=users)
        det.copy_state_from(base)
        est, _ = det.detect(x)
        est = est.reshape(users, P)
        err = max(float(np.max(np.abs(est[u] - refs[u]))) for u in range(users)) / scale
        print(f"N={N} users={users} var={var} {kind} {form}: {err:.3e}")
        assert err <= bound, (form, err)


POOL_SPECS = [2, 3, 4, 8, 16, 32]


@pytest.mark.parametrize("kind", ["exact", "near"])
@pytest.mark.parametrize("var", [0.05, 0.5], ids=["narrow", "wide"])
@pytest.mark.parametrize("form", sorted(BOUND))
def test_pool_duplicates(oracle_mod, form, var, kind):
    from libapsm_b200 import DetectorPool, PoolJob

    P = 200
    cfg = dict(BASE, gaussianKernelVariance=var, dictionarySize=P, detectVersion=form)
    pool = DetectorPool(cfg)
    dets, frames = [], []
    for i, N in enumerate(POOL_SPECS):
        dets.append(pool.add(N))
        frames.append(synth.generate_frame(500 + i, K=3, N=N, P=P, S=16, modulation="QAM16", snr_db=20))
    pool.run([PoolJob(d, f.rx_train, f.tx_train[0]) for d, f in zip(dets, frames)])
    xs = [_points(f.rx_train, kind) for f in frames]
    outs = pool.run([PoolJob(d, x) for d, x in zip(dets, xs)])
    for d, N, f, x, est in zip(dets, POOL_SPECS, frames, xs, outs):
        rows, a, w = pool.get_state(d)
        assert rows == 2 * P
        ref = _fp64(oracle_mod, cfg, N, oracle_mod.dedup_rows(f.rx_train), a.astype(np.float64),
                    w.astype(np.float64), x)
        err = float(np.max(np.abs(est - ref))) / float(np.max(np.abs(ref)))
        print(f"pool {form} var={var} {kind} N={N}: {err:.3e}")
        assert err <= BOUND[form], (N, err)
