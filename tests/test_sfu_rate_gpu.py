"""The measured SFU exponential rate that bench.py divides the detection
stage's exponentials by (its roofline denominator): plausible against the
nominal 16 ex2 per clock per SM of an sm_100 SM at the device's clocks."""
import ctypes

import pytest

from libapsm_b200 import _native

pytestmark = pytest.mark.gpu


def test_measured_ex2_rate_is_plausible():
    import torch

    lib = _native.load()
    rate, ms = ctypes.c_double(0.0), ctypes.c_float(0.0)
    assert lib.apsm_measure_ex2_rate(ctypes.byref(rate), ctypes.byref(ms)) == _native.APSM_OK
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    per_clk_sm_at_max = rate.value / (sms * 1.965e9)
    # between a quarter and 1.25x of the nominal 16 per clock per SM at the maximum SM clock
    assert 4.0 < per_clk_sm_at_max < 20.0, per_clk_sm_at_max
    assert ms.value > 0.0
    assert lib.apsm_measure_ex2_rate(None, None) == _native.APSM_ERR_INVALID_ARGUMENT
