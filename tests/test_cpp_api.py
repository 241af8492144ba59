"""The C++ drop-in header (include/apsm_b200.hpp): compiles against the C ABI,
throws std::invalid_argument for configuration errors like the reference
factory, and (GPU) gives the same estimates as the Python mirror."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from tests.conftest import ROOT

SRC = ROOT / "tests" / "cpp" / "cpp_api_check.cpp"


@pytest.fixture(scope="module")
def cpp_check(native_lib, tmp_path_factory):
    exe = tmp_path_factory.mktemp("cpp") / "cpp_api_check"
    subprocess.run(["g++", "-std=c++17", "-O2", f"-I{ROOT / 'include'}", str(SRC), f"-L{ROOT / 'libapsm_b200'}",
                    "-lapsm_b200", f"-Wl,-rpath,{ROOT / 'libapsm_b200'}", "-o", str(exe)], check=True)
    return exe


@pytest.mark.parametrize("cfg,msg", [
    ('{"otype":"APSM","foo":1}', "Invalid key: foo"),
    ('{"otype":"APSM","detectVersion":"x"}', "Unknown detect version: x"),
    ('{"otype":"NN"}', "Unknown algorithm: NN"),
])
def test_cpp_factory_throws_invalid_argument(cpp_check, cfg, msg):
    r = subprocess.run([str(cpp_check), cfg], capture_output=True, text=True)
    assert r.returncode == 3, r.stdout + r.stderr
    assert msg in r.stdout


@pytest.mark.gpu
def test_cpp_api_matches_python_api(cpp_check, tmp_path):
    import libapsm_b200 as L
    from libapsm_b200 import synth

    f = synth.generate_frame(31, K=2, N=8, P=300, S=500, modulation="QAM16")
    cfg = '{"otype":"APSM","windowSize":40,"gaussianKernelVariance":0.5,"eB":0.01}'
    files = {}
    for name, arr in (("rxt", f.rx_train), ("tx", f.tx_train[0]), ("rxd", f.rx_data)):
        p = tmp_path / f"{name}.f32"
        np.ascontiguousarray(arr, dtype=np.complex64).tofile(p)
        files[name] = str(p)
    out = tmp_path / "est.f32"
    r = subprocess.run([str(cpp_check), cfg, "8", "300", "500", files["rxt"], files["tx"], files["rxd"], str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Train time = " in r.stdout
    est_cpp = np.fromfile(out, dtype=np.complex64)
    det = L.NomaDetectorFactory.build(cfg, 8)
    det.train(f.rx_train, f.tx_train[0])
    est_py, _ = det.detect(f.rx_data)
    np.testing.assert_array_equal(est_cpp, est_py)


@pytest.mark.gpu
def test_cpp_api_train_history(cpp_check, tmp_path):
    import libapsm_b200 as L
    from libapsm_b200 import synth

    f = synth.generate_frame(32, K=2, N=4, P=64, S=96, modulation="QPSK")
    cfg = '{"otype":"APSM","windowSize":8,"gaussianKernelVariance":0.5}'
    files = {}
    for name, arr in (("rxt", f.rx_train), ("tx", f.tx_train[0]), ("rxd", f.rx_data), ("txd", f.tx_data[0])):
        p = tmp_path / f"{name}.f32"
        np.ascontiguousarray(arr, dtype=np.complex64).tofile(p)
        files[name] = str(p)
    csv = tmp_path / "h.csv"
    r = subprocess.run([str(cpp_check), cfg, "4", "64", "96", files["rxt"], files["tx"], files["rxd"],
                        str(tmp_path / "est.f32"), files["txd"], str(csv)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    rows = csv.read_text().splitlines()
    assert rows[0] == "step,train_evm,train_ser,train_ber,val_evm,val_ser,val_ber" and len(rows) == 65
    det = L.NomaDetectorFactory.build(cfg, 4)
    hist = L.NomaTrainHistory(2, L.Modulation("QPSK").scale)
    det.train(f.rx_train, f.tx_train[0], val_set=(hist, f.rx_data, f.tx_data[0]))
    got = np.array([[float(v) for v in row.split(",")[1:]] for row in rows[1:]])
    np.testing.assert_allclose(got, hist.steps, rtol=1e-5, atol=1e-6)  # %g keeps 6 digits
