"""Allocation-free detection (apsm_detect_device_noalloc), collected last.

Called through the C ABI it must give the same estimates as
apsm_detect_device on the same trained handle, on two calls in a row (the
first call sets up the fixed scratch), and reject a symbol count above its
fixed scratch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_detect_equals_detect_device(native_lib):
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    f = synth.generate_frame(77, K=3, N=8, P=300, S=700, modulation="QAM16", snr_db=20.0)
    cfg = {"otype": "APSM", "windowSize": 40, "gaussianKernelVariance": 0.5, "eB": 0.01}
    det = L.NomaDetectorFactory.build(cfg, 8, num_users=3)
    det.train(f.rx_train, f.tx_train)
    lib = det._lib
    for rep in range(2):
        for S in (700, 333):
            rxd = torch.from_numpy(np.ascontiguousarray(f.rx_data[:, :S])).cuda()
            ref = torch.empty((3, S), dtype=torch.complex64, device="cuda")
            out = torch.full((3, S), float("nan"), dtype=torch.complex64, device="cuda")
            assert lib.apsm_detect_device(det._h, rxd.data_ptr(), S, ref.data_ptr(), None) == 0
            assert lib.apsm_detect_device_noalloc(det._h, rxd.data_ptr(), S, out.data_ptr(), None) == 0
            det.synchronize()
            assert torch.equal(out, ref), (rep, S)


def test_noalloc_rejects_oversized_batch(native_lib):
    import torch

    import libapsm_b200 as L

    det = L.NomaDetectorFactory.build({"otype": "APSM"}, 16)
    S = 40000  # 2 * S * 32 * 4 bytes > 8 MiB
    rx = torch.zeros((16, S), dtype=torch.complex64, device="cuda")
    est = torch.zeros(S, dtype=torch.complex64, device="cuda")
    st = det._lib.apsm_detect_device_noalloc(det._h, rx.data_ptr(), S, est.data_ptr(), None)
    assert st == 1
    assert b"fixed scratch" in det._lib.apsm_last_error(det._h)
