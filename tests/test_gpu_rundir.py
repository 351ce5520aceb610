"""program dwf3d run in a directory (chdwf_run_dir): the reference's input
files in, its output streams out (rhmc/cheisdwf.f:1-466).  The same chain
run through the Program API must produce byte-identical records."""
import os
import shutil

import numpy as np
import pytest

import chiralheisenberg_b200 as chb

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
L, LT, LS = 4, 4, 4
MIDOUT = (0.1, 0.45, 1.0, 0.0, 0.0, 1, 4, 6)     # dt beta am3 am hpin imass iterl iter2


@pytest.fixture(scope="module")
def run(tmp_path_factory):
    d = tmp_path_factory.mktemp("dwf3d")
    (d / "midout").write_text(" ".join(str(v) for v in MIDOUT) +
                              "\ndt beta am3 am hpin imass iterl iter2\n")
    for name in ("remez2", "remez4", "remez2g"):
        shutil.copyfile(os.path.join(GOLD, name), d / name)
    chb.run_dir(str(d), L, LT, LS)
    # the same chain through the API: cold start (no 'con'), default seed
    dt, beta, am3, am, hpin, imass, iterl, iter2 = MIDOUT
    rz = {k: chb.read_remez(k, n, os.path.join(GOLD, k))
          for k, n in (("remez2", 25), ("remez4", 25), ("remez2g", 12))}
    prog = chb.Program(L, LT, LS, dt, beta, am3, am, hpin, imass, iterl, rz["remez2"],
                       rz["remez4"], rz["remez2g"])
    seed0 = prog.read_con(str(d / "no_such_con"))
    prog.startup(seed0)
    seed1 = prog.seed()
    recs, cfs = [], []
    for _ in range(iter2):
        r = prog.sweep()
        recs.append(r)
        cfs.append(prog.correlators() if r.measured else None)
    out = dict(dir=d, recs=recs, cfs=cfs, chi=prog.get_chi(), seed=prog.seed(), seed0=seed0,
               seed1=seed1, avg=prog.averages())
    prog.close()
    return out


def _lines(d, name):
    return open(d / name).read().splitlines(keepends=True)


def test_control_and_action_streams(run):
    recs = run["recs"]
    assert _lines(run["dir"], "control") == [
        chb.format_list("ddi", [r.dH, r.dS, r.accepted]) for r in recs]
    assert _lines(run["dir"], "fort.11") == [
        chb.format_list("iff", [i + 1, r.gaction, r.paction]) for i, r in enumerate(recs)]


def test_measurement_streams(run):
    recs, d = run["recs"], run["dir"]
    meas = [r for r in recs if r.measured]
    assert len(meas) == MIDOUT[7] // 5
    assert _lines(d, "fort.12") == [chb.format_list("fff", list(r.cond)) for r in meas]
    assert _lines(d, "fort.13") == [chb.format_list("fff", list(r.susc)) for r in meas]
    assert _lines(d, "fort.14") == [chb.format_list("ff", [r.condmod, r.susctot]) for r in meas]
    cf = [c for c in run["cfs"] if c is not None]
    for name, (k, f) in (("fort.5001", (0, 0)), ("fort.5011", (1, 0)), ("fort.5002", (0, 1)),
                         ("fort.5012", (1, 1))):
        want = [chb.format_list("iff", [it, c[k, f, it, 0], c[k, f, it, 1]])
                for c in cf for it in range(LT)]
        assert _lines(d, name) == want


def test_con_checkpoint(run):
    chi, seed, single = chb.con_read(str(run["dir"] / "con"), L * L * LT)
    assert not single
    assert np.array_equal(chi, run["chi"])
    assert seed == run["seed"]


def test_output_file(run):
    text = _lines(run["dir"], "output")
    a = run["avg"]
    assert text[0] == " seed: " + chb.format_list("d", [run["seed0"]])
    assert text[1] == " ksize=" + chb.format_edit("I", 3, 0, L) + " ksizet=" + \
        chb.format_edit("I", 3, 0, LT) + "\n"
    assert text[8] == " seed: " + chb.format_list("d", [run["seed1"]])
    assert text[9] == " averages for last " + chb.format_edit("I", 6, 0, MIDOUT[7]) + \
        " trajectories\n"
    assert text[10] == "  # of acceptances: " + chb.format_edit("I", 6, 0, a.naccp) + \
        " average trajectory length= " + chb.format_edit("F", 8, 3, a.atraj) + "\n"
    assert text[11] == "  <exp-dH>=" + chb.format_edit("E", 11, 4, a.yav) + " +/-" + \
        chb.format_edit("E", 10, 3, a.yyav) + "\n"
    assert text[-1] == " seed: " + chb.format_list("d", [run["seed"]])
    assert text[-6].startswith("  mean square velocity=")
    assert text[-5:-1] == ["\n"] * 4          # '//' of format 9022, two 9024 records
    # averages follow the records
    recs = run["recs"]
    assert a.naccp == sum(r.accepted for r in recs)
    assert a.iter2 == len(recs)
