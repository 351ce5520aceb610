"""The reference program's on-disk formats, pinned against files the
reference itself wrote (tests/golden, made by make_golden.py from the
reference tree): list-directed output of fort.11-14 (rhmc/cheisdwf.f:347,
:387-389), the explicit formats of 'output' (:165-176, :436-453) and the
'con' record (sread/swrite :1455-1489; the single-precision variant of
rhmc/sp_to_dp.f).  No GPU: these are host functions of libchdwf."""
import json
import os
import re

import numpy as np
import pytest

import chiralheisenberg_b200 as chb

GOLD = os.path.join(os.path.dirname(__file__), "golden")
KVOL = 12 * 12 * 12


def test_list_directed_records_match_reference_output():
    """Every record: parse its values, write them again, get the same bytes."""
    data = json.load(open(os.path.join(GOLD, "list_directed.json")))
    n = 0
    for block in data:
        for line in block["lines"]:
            vals = [float(t) for t in line.split()]
            assert len(vals) == len(block["kinds"])
            assert chb.format_list(block["kinds"], vals) == line, (block["source"], line)
            n += 1
    assert n > 1000


def test_list_directed_edge_values():
    # zero, negatives in both forms, the F/E boundary and REAL*8 layout
    assert chb.format_list("f", [0.0]) == "   0.00000000    \n"
    assert chb.format_list("f", [0.1]) == "  0.100000001    \n"
    assert chb.format_list("f", [0.099999994]) == "   9.99999940E-02\n"
    assert chb.format_list("f", [-123.25]) == "  -123.250000    \n"
    assert chb.format_list("f", [1.0e9]) == "   1.00000000E+09\n"
    assert chb.format_list("i", [-7]) == "          -7\n"
    assert chb.format_list("d", [-0.5]) == " -0.50000000000000000     \n"
    assert chb.format_list("d", [1.0e-5]) == "   1.0000000000000001E-005\n"


def _seed_lines(text):
    return [ln for ln in text.splitlines() if ln.startswith(" seed:")]


def test_output_file_layout_matches_reference():
    """'output' records of rhmc/Ls_8/b_0.45/out_1: the seed lines
    (list-directed REAL*8) and every explicit format whose layout the
    current source keeps."""
    text = open(os.path.join(GOLD, "out_1_b0.45.txt")).read()
    for ln in _seed_lines(text):
        seed = float(ln.split()[1])
        # 'seed: ' after the record's leading blank, then separator + G25.17
        assert " seed: " + chb.format_list("d", [seed]) == ln + "\n"
    lines = text.splitlines()
    E, F, I = (lambda w, d, v: chb.format_edit("E", w, d, v),
               lambda w, d, v: chb.format_edit("F", w, d, v),
               lambda w, v: chb.format_edit("I", w, 0, v))
    f32 = lambda x: float(np.float32(x))
    assert lines[1] == " ksize=" + I(3, 12) + " ksizet=" + I(3, 12)
    assert lines[2] == " kthird=" + I(3, 8)
    assert lines[3] == " time step: dt=" + F(6, 4, f32(0.125)) + " trajectory length=" + \
        F(9, 6, f32(8 * f32(0.125)))
    assert lines[4] == " # trajectories=" + I(6, 2500) + " beta=" + F(9, 6, f32(0.45))
    assert lines[6] == " imass=" + I(2, 1)
    assert lines[7] == " Stopping residuals: guidance: " + E(9, 4, f32(1e-6)) + \
        " acceptance: " + E(9, 4, f32(1e-9)) + " estimator: " + E(9, 4, f32(1e-6))
    # format 9022: re-edit the printed values with the format's descriptors
    nums = lambda s: [float(x) for x in re.findall(r"-?\d*\.\d+(?:E[+-]\d+)?|\d+", s)]
    i = lines.index(" averages for last   2500 trajectories")
    a = nums(lines[i + 1])
    assert lines[i + 1] == "  # of acceptances: " + I(6, int(a[0])) + \
        " average trajectory length= " + F(8, 3, a[1])
    a = nums(lines[i + 2])
    assert lines[i + 2] == "  <exp-dH>=" + E(11, 4, a[0]) + " +/-" + E(10, 3, a[1])
    a = nums(lines[i + 3])
    assert lines[i + 3] == "  av. # QMR itr. guidance: " + F(9, 3, a[0]) + "; acceptance: " + \
        F(9, 3, a[1])
    a = nums(lines[i + 4])
    assert lines[i + 4] == "  force: " + F(9, 3, a[0]) + "; pseudofermion: " + F(9, 3, a[1])
    assert lines[i + 5] == ""
    assert lines[i + 6] == "  measurement: " + F(9, 3, nums(lines[i + 6])[0])
    a = nums(lines[i + 8])
    assert lines[i + 8] == "  condmod=" + E(11, 3, a[0]) + " susc=" + E(11, 3, a[1])
    a = nums(lines[i + 9])
    assert lines[i + 9] == " cond components=" + "".join(E(11, 3, v) for v in a)
    assert lines[i + 10] == "  psibarpsi=" + E(11, 3, nums(lines[i + 10])[0])
    a = nums(lines[i + 11])
    assert lines[i + 11] == "  mean square velocity=" + E(10, 3, a[0]) + \
        "; action per site=" + E(10, 3, a[1])
    # '//' closing 9022 and two 9024 records (1x alone writes nothing)
    assert lines[i + 12:i + 16] == ["", "", "", ""]


def test_edit_descriptor_rules():
    assert chb.format_edit("E", 9, 4, 0.0) == ".0000E+00"
    assert chb.format_edit("E", 10, 3, -0.00727) == "-0.727E-02"
    assert chb.format_edit("F", 6, 4, -0.5) == "-.5000"
    assert chb.format_edit("F", 4, 1, 12345.0) == "****"
    assert chb.format_edit("I", 3, 0, 1234) == "***"


def test_con_double_precision_round_trip(tmp_path):
    chi, seed, single = chb.con_read(os.path.join(GOLD, "con_12x12x12.bin"), KVOL)
    assert not single and chi.shape == (3, KVOL) and np.isfinite(chi).all()
    out = tmp_path / "con"
    chb.con_write(str(out), chi, seed)
    # swrite's record is byte-identical to the one the reference wrote
    assert out.read_bytes() == open(os.path.join(GOLD, "con_12x12x12.bin"), "rb").read()


def test_con_single_precision_is_converted(tmp_path):
    raw = open(os.path.join(GOLD, "con_sp_12x12x12.bin"), "rb").read()
    assert int.from_bytes(raw[:4], "little") == 12 * KVOL + 8
    chi, seed, single = chb.con_read(os.path.join(GOLD, "con_sp_12x12x12.bin"), KVOL)
    assert single
    ref = np.frombuffer(raw[4:4 + 12 * KVOL], dtype="<f4").reshape(3, KVOL)
    assert np.array_equal(chi, ref.astype(np.float64))
    assert seed == np.frombuffer(raw[4 + 12 * KVOL:12 + 12 * KVOL], dtype="<f8")[0]
    # the sp_to_dp conversion: a REAL*8 record of the same values
    chb.con_write(str(tmp_path / "condp"), chi, seed)
    chi2, seed2, single2 = chb.con_read(str(tmp_path / "condp"), KVOL)
    assert not single2 and np.array_equal(chi2, chi) and seed2 == seed


def test_con_errors(tmp_path):
    with pytest.raises(FileNotFoundError):
        chb.con_read(str(tmp_path / "missing"), KVOL)
    with pytest.raises(chb.ChdwfError):
        chb.con_read(os.path.join(GOLD, "con_12x12x12.bin"), 8 * 8 * 8)
    (tmp_path / "bad").write_bytes(b"\x10\x00\x00\x00" + b"\x00" * 16 + b"\x11\x00\x00\x00")
    with pytest.raises(chb.ChdwfError):
        chb.con_read(str(tmp_path / "bad"), 1)


def test_run_dir_reports_missing_inputs(tmp_path):
    """The run driver reads midout and the Remez files before it touches a GPU."""
    with pytest.raises(FileNotFoundError):
        chb.run_dir(str(tmp_path), 4, 4, 4)
    (tmp_path / "midout").write_text("0.1 0.45 1.0 0.0 0.0 1 4 5\ndt beta am3 am hpin imass iterl iter2\n")
    with pytest.raises(FileNotFoundError):     # no remez2
        chb.run_dir(str(tmp_path), 4, 4, 4)
    (tmp_path / "midout").write_text("0.1 0.45 x\n")
    with pytest.raises(chb.ChdwfError):
        chb.run_dir(str(tmp_path), 4, 4, 4)
