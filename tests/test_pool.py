"""Detector pool, host side (no GPU): configuration restrictions are checked
before any device is looked for, and the C ABI exports the pool entry points."""
import ctypes

import pytest


def _create(native_lib, cfg: str):
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(256)
    st = native_lib.apsm_pool_create(cfg.encode(), 0, 1, ctypes.byref(h), err, len(err))
    if st == 0:
        native_lib.apsm_pool_destroy(h)
    return st, err.value.decode()


@pytest.mark.parametrize("cfg,status,msg", [
    ('{"otype":"APSM","foo":1}', 2, "Invalid key: foo"),
    ('{"otype":"LLS"}', 5, "APSM detectors only"),
    ('{"otype":"APSM","llsInitialization":true}', 5, "llsInitialization"),
    ('{"otype":"APSM","gaussianKernelVariance":0}', 5, "gaussianKernelVariance"),
    ('{"otype":"APSM","sampleStep":3}', 5, "even sampleStep"),
    ('{"otype":"APSM","sampleStep":10}', 5, "even sampleStep"),
    ('{"otype":"APSM","windowSize":90,"dictionarySize":80}', 5, "dictionarySize"),
])
def test_pool_config_restrictions(native_lib, cfg, status, msg):
    st, err = _create(native_lib, cfg)
    assert st == status, (st, err)
    assert msg in err


def test_pool_null_arguments(native_lib):
    h = ctypes.c_void_p()
    assert native_lib.apsm_pool_create(None, 0, 1, ctypes.byref(h), None, 0) == 1
    assert native_lib.apsm_pool_create(b'{"otype":"APSM"}', 0, 0, ctypes.byref(h), None, 0) == 1
    assert native_lib.apsm_pool_run(None, 0, None, 0, 0) == 1
    assert native_lib.apsm_pool_query(None, 0) < 0
    assert native_lib.apsm_pool_bytes_in_use(None) == 0


def test_column_prefix_closed_form():
    """The kernel-column offsets use a closed form of sum_m len(m) with
    len(m) = min(m + qP, nP) - max(0, m + 1 - capP); check it against the sum."""
    def closed(n, qP, nP, capP):
        k = min(max(nP - qP, 0), n)
        s1 = k * qP + k * (k - 1) // 2 + (n - k) * nP
        j = max(n - capP, 0)
        return s1 - j * (j + 1) // 2

    for qP, nP, capP in [(20, 300, 400), (80, 1000, 1000), (20, 330, 200), (5, 3, 10), (80, 50, 100)]:
        acc = 0
        for n in range(nP + 1):
            assert closed(n, qP, nP, capP) == acc, (qP, nP, capP, n)
            if n < nP:
                acc += min(n + qP, nP) - max(0, n + 1 - capP)
