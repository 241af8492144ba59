"""NOMA_detect command line tool (cpp/cli/detect/noma_detect.cpp and
cpp/cli/common/*): argument handling, antenna patterns, seeded reference data,
printouts and end-to-end runs on the reference's captured data."""
import io
import json
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import libapsm_b200 as L
from libapsm_b200 import binfile, cli
from tests.conftest import HAS_GPU

HERE = Path(__file__).resolve().parent


# ------------------------------------------------------- antenna patterns --

def bits_set(p):
    return [i for i, b in enumerate(p) if b]


def test_pattern_string_is_a_bitset_of_16():
    # std::bitset<16>(s): the first min(16, len) characters, the last of them is bit 0
    assert bits_set(cli.pattern_from_string("1")) == [0]
    assert bits_set(cli.pattern_from_string("10")) == [1]
    assert bits_set(cli.pattern_from_string("1000000000000000")) == [15]
    assert bits_set(cli.pattern_from_string("0000000000000101")) == [0, 2]
    # longer strings: characters past the 16th are ignored
    assert bits_set(cli.pattern_from_string("0000000000000001" + "1111")) == [0]
    assert len(bits_set(cli.pattern_from_string("11111111111111111111"))) == 16
    with pytest.raises(ValueError):
        cli.pattern_from_string("10x1")


def test_antenna_schemes():
    assert bits_set(cli.antenna_pattern({"otype": "all"})) == list(range(16))
    assert bits_set(cli.antenna_pattern({"otype": "equidistant", "number": 8})) == list(range(0, 16, 2))
    assert bits_set(cli.antenna_pattern({"otype": "equidistant", "number": 5})) == [0, 3, 6, 9, 12]
    assert bits_set(cli.antenna_pattern({"otype": "first", "number": 3})) == [0, 1, 2]
    assert bits_set(cli.antenna_pattern({"otype": "first"})) == list(range(16))
    assert bits_set(cli.antenna_pattern({"otype": "pattern", "pattern": "0000000000001111"})) == [0, 1, 2, 3]
    assert len(bits_set(cli.antenna_pattern({"otype": "random", "number": 6}))) == 6
    with pytest.raises(ValueError, match="Invalid key: numbr"):
        cli.antenna_pattern({"otype": "first", "numbr": 3})
    with pytest.raises(ValueError, match="Invalid antenna scheme: odd"):
        cli.antenna_pattern({"otype": "odd"})


def test_select_antennas_keeps_rows_in_order():
    m = np.arange(8 * 3).reshape(8, 3).astype(np.complex64)
    out = cli.select_antennas(m, cli.antenna_pattern({"otype": "equidistant", "number": 4}))
    np.testing.assert_array_equal(out, m[[0, 4]])  # rows 8 and 12 do not exist in an 8-antenna file
    np.testing.assert_array_equal(cli.select_antennas(m, cli.antenna_pattern({"otype": "all"})), m)


# -------------------------------------------------- seeded reference data --

MT_PROGRAM = r"""
#include <cstdio>
#include <cstdlib>
#include <random>
int main(int argc, char** argv) {
    std::mt19937 gen(std::strtoul(argv[1], nullptr, 10));
    std::bernoulli_distribution d(0.5);
    for (int i = 0, n = std::atoi(argv[2]); i < n; ++i) std::putchar(d(gen) ? '1' : '0');
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
@pytest.mark.parametrize("seed", [0, 7, 42, 4294967295])
def test_random_bits_match_std_mt19937_bernoulli(tmp_path, seed):
    src = tmp_path / "mt.cpp"
    src.write_text(MT_PROGRAM)
    exe = tmp_path / "mt"
    subprocess.run(["g++", "-O1", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe), str(seed), "5000"], check=True, capture_output=True, text=True).stdout
    expect = np.frombuffer(out.encode(), dtype=np.uint8) - ord("0")
    np.testing.assert_array_equal(cli.random_bits(seed, 5000), expect)


def test_random_reference_data_layout():
    mod = L.Modulation("QAM16")
    tr, da = cli.random_reference_data(3, mod)
    assert tr.shape == (6, 685) and da.shape == (6, 3840)
    bits = cli.random_bits(3, (685 + 3840) * 6 * 4)
    sym = mod.encode(bits).reshape(6, -1)
    np.testing.assert_array_equal(tr, sym[:, :685])
    np.testing.assert_array_equal(da, sym[:, 685:])
    # every symbol is a constellation point
    np.testing.assert_array_equal(mod.symbol_bits(mod.hard_decode_int(da)), da)


# ------------------------------------------------------------- printouts --

def test_symbol_error_printout():
    mod = L.Modulation("QPSK")
    s = np.float32(mod.scale)
    ref = np.array([s + 1j * s, -s + 1j * s, s - 1j * s, -s - 1j * s], np.complex64)
    est = ref.copy()
    est[1] = s + 1j * s                  # real axis wrong
    est[2] = np.complex64(np.nan)        # NaN
    buf = io.StringIO()
    pct = cli.print_symbol_errors(est, ref, mod, buf)
    assert buf.getvalue() == "\n.rn. symbol errors: 2 of 4 - 50.00 percent\n"
    assert pct == 50.0


def test_symbol_error_printout_keeps_the_inverted_imaginary_edge_test():
    # util.cpp:90-95: an estimate beyond the outer imaginary edge of an outer true point counts as an error
    mod = L.Modulation("QPSK")
    s = np.float32(mod.scale)
    ref = np.array([s + 1j * s], np.complex64)
    est = np.array([s + 1j * 3 * s], np.complex64)
    buf = io.StringIO()
    cli.print_symbol_errors(est, ref, mod, buf)
    assert "i symbol errors: 1 of 1" in buf.getvalue()


def test_bit_error_and_evm_printouts():
    mod = L.Modulation("QPSK")
    s = np.float32(mod.scale)
    ref = np.array([s + 1j * s, -s - 1j * s], np.complex64)
    est = np.array([s + 1j * s, s - 1j * s], np.complex64)  # one bit wrong
    buf = io.StringIO()
    assert cli.print_bit_errors(est, ref, mod, buf) == 25.0
    assert buf.getvalue() == "\n .. x. bit errors: 1 of 4 - 25.00 percent\n"
    buf = io.StringIO()
    v = cli.print_evm(est, ref, buf)
    assert v == pytest.approx(1.0, rel=1e-6)  # |error| = 2 scale on one of two symbols
    assert buf.getvalue() == "\n █ EVM: 1.0000\n"


def test_scripting_prints_only_the_three_numbers():
    mod = L.Modulation("QPSK")
    s = np.float32(mod.scale)
    ref = np.array([s + 1j * s, -s - 1j * s], np.complex64)
    est = np.array([s + 1j * s, s - 1j * s], np.complex64)
    buf = io.StringIO()
    cli.print_errors("SCRIPTING", est, ref, mod, buf)
    assert buf.getvalue() == "25.000000,50.000000,1.000000\n"


def test_output_mode_and_missing_reference_are_errors(tmp_path):
    with pytest.raises(ValueError, match="Invalid print mode: XYZ"):
        cli.output_mode("XYZ")
    assert cli.output_mode("scripting") == "SCRIPTING"
    synced = tmp_path / "s.bin"
    binfile.write(synced, {"rxSigTraining": np.zeros((4, 2, 2), np.float32),
                           "rxSigData": np.zeros((4, 2, 2), np.float32)})
    args = cli.make_parser().parse_args(["-s", str(synced)])
    with pytest.raises(ValueError, match="Neither --random-seed/-rs nor --reference-data/-r"):
        cli.load_inputs(args, cli.load_config(args))


def test_default_config_and_config_file(tmp_path):
    args = cli.make_parser().parse_args(["-s", "x"])
    assert cli.load_config(args) == {"algorithm": {"otype": "APSM"}}
    f = tmp_path / "c.json"
    f.write_text(json.dumps({"algorithm": {"otype": "LLS"}, "user": 2}))
    args = cli.make_parser().parse_args(["-s", "x", "-cf", str(f), "-cs", "{}"])
    assert cli.load_config(args) == {"algorithm": {"otype": "LLS"}, "user": 2}  # -cf wins


# ------------------------------------------------------- end-to-end runs --

CAPTURED_CFG = {"algorithm": {"otype": "APSM", "windowSize": 80}, "modulation": "QPSK",
                "antennas": {"otype": "equidistant", "number": 8}, "user": 1}


def captured_files(tmp_path):
    """The captured-data slice as the reference's files: 16 antennas (the 8 equidistant ones
    of the slice, other antennas filled with noise) and integer-grid reference symbols."""
    cap = np.load(HERE / "golden" / "captured_qpsk_inputs.npz")
    mod = L.Modulation("QPSK")
    rng = np.random.default_rng(0)

    def sixteen(m):
        full = (rng.standard_normal((16, m.shape[1])) + 1j * rng.standard_normal((16, m.shape[1]))).astype(np.complex64)
        full[0::2] = m
        return full

    def grid(m):
        g = np.rint(m / np.float32(mod.scale)).astype(np.complex64)
        np.testing.assert_array_equal(binfile.complex_matrix(binfile.to_array(g), mod.scale), m)
        return g

    synced, ref = tmp_path / "synced.bin", tmp_path / "ref.bin"
    binfile.write(synced, {"rxSigTraining": binfile.to_array(sixteen(cap["rx_train"])),
                           "rxSigData": binfile.to_array(sixteen(cap["rx_data"]))})
    binfile.write(ref, {"mod_training": binfile.to_array(grid(cap["tx_train"])),
                        "mod_data": binfile.to_array(grid(cap["tx_data"]))})
    return synced, ref, cap


@pytest.mark.skipif(HAS_GPU, reason="checks the behaviour without a GPU")
def test_cli_without_gpu_fails_loudly(tmp_path):
    synced, ref, _ = captured_files(tmp_path)
    with pytest.raises(L.ApsmError):
        cli.main(["-s", str(synced), "-r", str(ref), "-cs", json.dumps(CAPTURED_CFG)], out=io.StringIO())


@pytest.mark.gpu
def test_cli_reproduces_reference_on_captured_data(tmp_path):
    synced, ref, cap = captured_files(tmp_path)
    gold = np.load(HERE / "golden" / "golden_captured_qpsk.npz")
    out_file = tmp_path / "est.bin"
    buf = io.StringIO()
    assert cli.main(["-s", str(synced), "-r", str(ref), "-cs", json.dumps(CAPTURED_CFG), "-d", str(out_file)],
                    out=buf) == 0
    est = binfile.complex_matrix(binfile.read(out_file)["estSigData"])[0]
    assert binfile.read(out_file)["estSigData"].shape == (192, 1, 2)
    scale = float(np.max(np.abs(gold["est_ref"])))
    assert float(np.max(np.abs(est - gold["est_ref"]))) <= 1e-4 * scale
    lines = buf.getvalue().splitlines()
    assert lines[0].startswith("Train time = ") and " ms, detect time = " in lines[0] and lines[0].endswith(" ms")
    mod = L.Modulation("QPSK")
    errors = L.modulation.cli_symbol_errors(est, cap["tx_data"][1], mod)
    assert lines[-1].endswith(f" symbol errors: {errors} of 192 - {100.0 * errors / 192:.2f} percent")
    marks = "".join(lines[1:]).split(" symbol errors")[0]
    assert len(marks) == 192 and set(marks) <= set(".nri") and marks.count(".") == 192 - errors
    # a line break before every 80 marks (util.cpp:73-74), the first one right after the time line
    assert [len(line) for line in lines[1:-1]] == [0, 80, 80]


@pytest.mark.gpu
def test_cli_train_history_file(tmp_path):
    synced, ref, _ = captured_files(tmp_path)
    csv = tmp_path / "hist.csv"
    buf = io.StringIO()
    cli.main(["-s", str(synced), "-r", str(ref), "-cs", json.dumps(CAPTURED_CFG), "-th", str(csv), "-o", "EVM"],
             out=buf)
    rows = csv.read_text().splitlines()
    assert rows[0] == "step,train_evm,train_ser,train_ber,val_evm,val_ser,val_ber"
    assert len(rows) == 1 + 160  # 160 pilots, sampleStep 2: one step per pilot
    last = [float(v) for v in rows[-1].split(",")]
    evm_line = buf.getvalue().splitlines()[-1]
    assert evm_line.startswith(" EVM: ") or " EVM: " in evm_line
    assert abs(last[4] - float(evm_line.split("EVM: ")[1])) <= 1e-4
    hist_fixture = HERE / "golden" / "golden_history_captured_qpsk.npz"
    if hist_fixture.exists():
        from tests.test_history import assert_history_close

        h = np.array([[float(v) for v in r.split(",")[1:]] for r in rows[1:]], np.float32)
        assert_history_close(h, np.load(hist_fixture)["hist_ref"], 160, 192, 2)


@pytest.mark.gpu
def test_cli_parallel_users_scripting(tmp_path):
    synced, ref, cap = captured_files(tmp_path)
    buf = io.StringIO()
    cfg = dict(CAPTURED_CFG)
    cli.main(["-s", str(synced), "-r", str(ref), "-cs", json.dumps(cfg), "-p", "-o", "scripting"], out=buf)
    lines = buf.getvalue().splitlines()
    assert len(lines) == 6
    mod = L.Modulation("QPSK")
    for u, line in enumerate(lines):
        ber, ser, evm = (float(v) for v in line.split(","))
        det = L.NomaDetectorFactory.build(cfg["algorithm"], 8)
        det.train(cap["rx_train"], cap["tx_train"][u])
        est, _ = det.detect(cap["rx_data"])
        assert ber == pytest.approx(100 * L.bit_error_rate(est, cap["tx_data"][u], mod), abs=0.6)
        assert evm == pytest.approx(L.evm(est, cap["tx_data"][u]), rel=1e-3)
        assert 0.0 <= ser <= 100.0


@pytest.mark.gpu
def test_cli_random_seed_reference_at_default_sizes(tmp_path):
    # -rs: 685 pilots and 3840 data symbols per user drawn like the reference tool; a
    # received signal synthesised from them (16 antennas, 6 users, 25 dB) is detected
    mod = L.Modulation("QPSK")
    tr, da = cli.random_reference_data(12, mod)
    rng = np.random.default_rng(12)
    H = (rng.standard_normal((16, 6)) + 1j * rng.standard_normal((16, 6))) / np.sqrt(2)

    def rx(tx):
        clean = H @ tx
        noise = (rng.standard_normal(clean.shape) + 1j * rng.standard_normal(clean.shape)) * np.sqrt(
            np.mean(np.abs(clean) ** 2) / 10 ** 2.5 / 2)
        return (clean + noise).astype(np.complex64)

    synced = tmp_path / "s.bin"
    binfile.write(synced, {"rxSigTraining": binfile.to_array(rx(tr)), "rxSigData": binfile.to_array(rx(da))})
    cfg = {"algorithm": {"otype": "APSM", "windowSize": 40}, "modulation": "QPSK", "user": 2}
    buf = io.StringIO()
    cli.main(["-s", str(synced), "-rs", "12", "-cs", json.dumps(cfg), "-o", "scripting"], out=buf)
    ber, ser, evm = (float(v) for v in buf.getvalue().split(","))
    assert ser < 10.0 and evm < 0.6
