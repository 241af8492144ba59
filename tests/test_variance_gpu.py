"""computeGaussianVarianceHeuristic (cpp/lib/apsm/apsm_noma_detector.cu:193-218),
used when gaussianKernelVariance is 0: host code in the reference, a GPU
pair-distance kernel plus an exact radix select here.  Checked against the
host formula (oracle.variance_heuristic, the reference's float arithmetic) to
one unit in the last place."""
import numpy as np
import pytest

import libapsm_b200 as L


@pytest.mark.gpu
@pytest.mark.parametrize("seed,N,P", [(51, 4, 2), (52, 6, 150), (53, 16, 685), (54, 32, 1200)])
def test_b200_variance_heuristic_matches_host_formula(oracle_mod, seed, N, P):
    # computeGaussianVarianceHeuristic (apsm_noma_detector.cu:193-218) runs on the GPU here;
    # the distances are those of the host formula, the order statistic exact
    f = L.synth.generate_frame(seed, K=3, N=N, P=P, S=8, modulation="QAM16")
    det = L.NomaDetectorFactory.build({"otype": "APSM", "gaussianKernelVariance": 0.0, "windowSize": 4}, N)
    assert det.gaussian_variance == 0.0
    det.train(f.rx_train, f.tx_train[0])
    ref = oracle_mod.variance_heuristic(f.rx_train)
    got = np.float32(det.gaussian_variance)
    assert abs(int(got.view(np.int32)) - int(np.float32(ref).view(np.int32))) <= 1, (got, ref)


@pytest.mark.gpu
def test_b200_configured_variance_is_scaled_by_n_squared():
    det = L.NomaDetectorFactory.build({"otype": "APSM", "gaussianKernelVariance": 0.05}, 8)
    assert det.gaussian_variance == pytest.approx(np.float32(0.05) * np.float32(64), rel=1e-7)
