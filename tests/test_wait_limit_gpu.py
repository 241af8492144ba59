"""Expiry of a bounded wait inside a tensor-core kernel is an error status.

The reference's failure model is CUDA_CHECK: print and exit(EXIT_FAILURE)
(cpp/lib/cuda/cuda_errorhandling.cuh:98-108, :113-134).  Here every barrier
wait of the tensor-core kernels gives up after a limit (2 s), the kernel
records the expiry, stops its work, still waits for its own copies and
tensor-core products, releases tensor memory, and the call returns
APSM_ERR_CUDA.  A limit of 0 makes every wait that is not already complete
give up at once, which drives that path without faulting or hanging the GPU.
The handle must stay usable: once the limit is restored the same call gives
the same estimates as before.
"""
import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import _native, synth

pytestmark = pytest.mark.gpu


@pytest.fixture
def lib():
    lib = _native.load()
    saved = lib.apsm_wait_limit_ns()
    yield lib
    lib.apsm_set_wait_limit_ns(saved)


@pytest.mark.parametrize("form", ["gram_bf16", "gram_tf32x3"])
def test_single_detector_wait_expiry_is_an_error_and_recoverable(lib, form):
    N, users = 16, 4
    f = synth.generate_frame(70, K=4, N=N, P=300, S=2048, modulation="QAM16", snr_db=20)
    cfg = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "dictionarySize": 300,
           "detectVersion": form}
    det = L.NomaDetectorFactory.build(cfg, N, num_users=users)
    det.train(f.rx_train, f.tx_train[:users])
    good, _ = det.detect(f.rx_data)
    lib.apsm_set_wait_limit_ns(0)
    with pytest.raises(L.ApsmError) as ei:
        det.detect(f.rx_data)
    assert ei.value.status == _native.APSM_ERR_CUDA
    assert "bounded wait" in str(ei.value)
    lib.apsm_set_wait_limit_ns(2_000_000_000)
    again, _ = det.detect(f.rx_data)
    np.testing.assert_array_equal(again, good)


def test_pool_wait_expiry_is_an_error_and_recoverable(lib):
    from libapsm_b200 import DetectorPool, PoolJob

    cfg = {"otype": "APSM", "windowSize": 20, "gaussianKernelVariance": 0.5, "eB": 0.01, "dictionarySize": 400,
           "detectVersion": "gram_tf32x3"}
    pool = DetectorPool(cfg)
    frames = [synth.generate_frame(80 + i, K=2, N=N, P=200, S=1500, modulation="QAM16") for i, N in enumerate((4, 16))]
    dets = [pool.add(N) for N in (4, 16)]
    pool.run([PoolJob(d, f.rx_train, f.tx_train[0]) for d, f in zip(dets, frames)])
    good = pool.run([PoolJob(d, f.rx_data) for d, f in zip(dets, frames)])
    lib.apsm_set_wait_limit_ns(0)
    with pytest.raises(L.ApsmError) as ei:
        pool.run([PoolJob(d, f.rx_data) for d, f in zip(dets, frames)])
    assert ei.value.status == _native.APSM_ERR_CUDA
    lib.apsm_set_wait_limit_ns(2_000_000_000)
    again = pool.run([PoolJob(d, f.rx_data) for d, f in zip(dets, frames)])
    for g, a in zip(good, again):
        np.testing.assert_array_equal(a, g)
