"""Allocation-free detection (apsm_detect_device_noalloc), collected last.

Called through the C ABI it must give the same estimates as
apsm_detect_device on the same trained handle, on two calls in a row (the
first call sets up the fixed scratch), in both exact detection kernels: the
<= 16-feature form (N = 8) and the wide form with cp.async dictionary tiles
(N = 16 and N = 64), with more than 8 users (a second pass over the users),
and at symbol counts up to the fixed scratch's limit (2 S Dp 4 bytes = 8 MiB:
S = 32768 at N = 16, S = 8192 at N = 64).  A symbol count above the limit is
rejected."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [  # N antennas, users, symbol counts (the largest at the scratch limit where given)
    (8, 3, (700, 333)),
    (16, 12, (32768, 1001)),
    (64, 2, (8192, 257)),
]


@pytest.mark.parametrize("N,users,sizes", CASES, ids=[f"N{c[0]}-u{c[1]}" for c in CASES])
def test_noalloc_detect_equals_detect_device(native_lib, N, users, sizes):
    import torch

    import libapsm_b200 as L
    from libapsm_b200 import synth

    f = synth.generate_frame(77 + N, K=max(users, 2), N=N, P=300, S=max(sizes), modulation="QAM16", snr_db=20.0)
    cfg = {"otype": "APSM", "windowSize": 40, "gaussianKernelVariance": 0.5, "eB": 0.01}
    det = L.NomaDetectorFactory.build(cfg, N, num_users=users)
    det.train(f.rx_train, f.tx_train[:users])
    lib = det._lib
    for rep in range(2):
        for S in sizes:
            rxd = torch.from_numpy(np.ascontiguousarray(f.rx_data[:, :S])).cuda()
            ref = torch.empty((users, S), dtype=torch.complex64, device="cuda")
            out = torch.full((users, S), float("nan"), dtype=torch.complex64, device="cuda")
            assert lib.apsm_detect_device(det._h, rxd.data_ptr(), S, ref.data_ptr(), None) == 0
            assert lib.apsm_detect_device_noalloc(det._h, rxd.data_ptr(), S, out.data_ptr(), None) == 0
            det.synchronize()
            assert torch.equal(out, ref), (rep, S)


def test_noalloc_rejects_oversized_batch(native_lib):
    import torch

    import libapsm_b200 as L

    det = L.NomaDetectorFactory.build({"otype": "APSM"}, 16)
    S = 32769  # 2 * S * 32 * 4 bytes: one symbol past 8 MiB
    rx = torch.zeros((16, S), dtype=torch.complex64, device="cuda")
    est = torch.zeros(S, dtype=torch.complex64, device="cuda")
    st = det._lib.apsm_detect_device_noalloc(det._h, rx.data_ptr(), S, est.data_ptr(), None)
    assert st == 1
    assert b"fixed scratch" in det._lib.apsm_last_error(det._h)
