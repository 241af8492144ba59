"""C-ABI boundary: exported symbols, configuration validation and error
behaviour of the factory (cpp/lib/apsm/apsm_noma_detector.cu:348-383,
cpp/lib/noma/noma_detector_factory.cu:57-65).  No GPU needed: the library
parses and validates the configuration before it looks for a device."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import HAS_GPU, ROOT


def header_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(apsm_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(native_lib):
    names = header_functions()
    assert "apsm_create" in names and "apsm_train" in names and "apsm_detect" in names
    for n in names:
        assert hasattr(native_lib, n), f"{n} declared in include/ but not exported"


def test_library_is_sm100a_only():
    # every kernel is compiled for sm_100a only (no PTX fallback for other GPUs)
    from libapsm_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.ARCH)


def _create(native_lib, cfg: str, n_ant=4, users=1):
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(256)
    st = native_lib.apsm_create(cfg.encode(), n_ant, users, ctypes.byref(h), err, len(err))
    if st == 0:
        native_lib.apsm_destroy(h)
    return st, err.value.decode()


@pytest.mark.parametrize("cfg,msg", [
    ('{"otype":"APSM","foo":1}', "Invalid key: foo"),
    ('{"otype":"APSM","zeta":1,"alpha":2}', "Invalid key: alpha"),  # sorted-key order, as nlohmann iterates
    ('{"otype":"APSM","detectVersion":"fast"}', "Unknown detect version: fast"),
    ('{"otype":"KNN"}', "Unknown algorithm: KNN"),
    ('{"otype":"LLS","windowSize":3}', "Invalid key: windowSize"),
    ('{"otype":"APSM","windowSize":"x"}', "windowSize"),
    ('{"otype":"APSM",', "JSON parse error"),
    ('[1,2]', "JSON object"),
])
def test_invalid_config_rejected(native_lib, cfg, msg):
    st, err = _create(native_lib, cfg)
    assert st == 2, (st, err)  # APSM_ERR_INVALID_CONFIG
    assert msg in err


def test_invalid_arguments(native_lib):
    h = ctypes.c_void_p()
    assert native_lib.apsm_create(None, 4, 1, ctypes.byref(h), None, 0) == 1
    st, err = _create(native_lib, '{"otype":"APSM"}', n_ant=0)
    assert st == 1
    st, err = _create(native_lib, '{"otype":"APSM"}', n_ant=65)
    assert st == 5 and "num_antennas" in err
    st, err = _create(native_lib, '{"otype":"APSM"}', users=0)
    assert st == 1
    # null handles are rejected, not dereferenced
    assert native_lib.apsm_train(None, None, None, 0, None) == 1
    assert native_lib.apsm_detect(None, None, 0, None, None) == 1
    assert native_lib.apsm_reset(None) == 1
    assert native_lib.apsm_rows(None) == 0
    native_lib.apsm_destroy(None)


def test_python_mirror_raises_value_error_on_bad_config(native_lib):
    from libapsm_b200 import NomaDetectorFactory

    with pytest.raises(ValueError, match="Invalid key: windowsize"):
        NomaDetectorFactory.build({"otype": "APSM", "windowsize": 80}, 8)
    with pytest.raises(ValueError, match="Unknown algorithm"):
        NomaDetectorFactory.build({"otype": "SVM"}, 8)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_valid_config_without_gpu_reports_no_device(native_lib):
    st, err = _create(native_lib, '{"otype":"APSM","windowSize":80}')
    assert st == 6 and "device" in err
    from libapsm_b200 import ApsmError, NomaDetectorFactory

    with pytest.raises(ApsmError):
        NomaDetectorFactory.build({"otype": "APSM"}, 8)


def test_product_path_has_no_cpu_fallback():
    """The package must not import or execute the oracle (the CPU checker)."""
    pat = re.compile(r"^\s*(from\s+oracle|import\s+oracle)|oracle/_ref|liboracle", re.M)
    for p in list((ROOT / "libapsm_b200").rglob("*.py")) + list((ROOT / "libapsm_b200").rglob("*.cu*")):
        assert not pat.search(p.read_text()), f"{p} reaches the oracle"
