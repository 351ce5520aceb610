"""Trajectory parity against the single-threaded oracle, over many trajectories.

The fixtures tests/golden/traj_*.json hold every scalar the main loop of
program dwf3d (rhmc/cheisdwf.f:207-399) produced, trajectory by trajectory,
when the oracle ran the chain on one thread (its reductions then follow the
reference's loop order, i.e. the reference at OMP_NUM_THREADS=1).  They are
made by tests/golden/make_traj_golden.py.  Workloads:
  traj_8x8_b0.475  L=Lt=8, Ls=8, beta=0.475, dt=0.1, iterl=10, chi from a
                   seeded N(0, 1/beta), the reference's default seed;
                   12 trajectories;
  traj_12x8_rhmc   L=Lt=12, Ls=8, the reference's shipped input deck
                   rhmc/midout (dt=0.125, beta=0.45, hpin=0.5, iterl=8) and
                   configuration rhmc/_con; 10 trajectories.
The GPU program runs the same chain from the same configuration and seed.

What must agree, and how closely (the numbers in TOL):
  * the random stream: MD step counts, the Metropolis draw x, the final
    seed -- identical;
  * the accept/reject decision sequence -- identical;
  * H0, S0 (before the molecular dynamics): from the same chi (the first
    trajectory) the 25-pole solves at 1e-9 of the GPU and of the oracle give
    H0 to about 1e-14 relative; later trajectories start from chains whose
    chi differ at the REAL*4 level of the momenta (below);
  * H1, S1, hg and dH (after it): the momenta and forces are REAL*4, as in
    the reference, and the GPU's FP64 reductions are summed in another
    order than the oracle's loop, so a force solve's last-bit difference can
    flip a REAL*4 rounding of dSdchi and of pp.  The bound is a small
    multiple of what was measured on a B200 against this 1-thread oracle;
    the reference itself moves dH by up to 1e-5 between 1 and 8 OpenMP
    threads on the 8^3 workload (the oracle's thread-count model);
  * solver iterations within the reference's own thread-count envelope
    (+-5 per solve);
  * REAL*4 observables relative 1e-5, correlators 1e-4 of their maximum.
Set CHDWF_TRAJ_OUT to a file path to write the measured differences as JSON.
"""
import json
import os

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

ITER_ENVELOPE = 5
# Relative bounds (dH also absolutely), about 3x the largest difference
# measured on a B200 over the 12 trajectories at 8^3x8: H0, S0 1.7e-10 (the
# chains' chi drift apart at the REAL*4 level after accepted trajectories;
# from the same chi, trajectory 1, H0 agrees to 5e-15), H1 4.4e-10,
# S1 2.4e-10, hg 6.2e-9, dH 1.35e-5 absolute = 3.9e-10 |H0|.
TOL = {"H0": 5e-10, "S0": 5e-10, "H1": 1.5e-9, "S1": 1.5e-9, "hg": 2e-8, "dH_rel_H0": 1.2e-9}
TOL_DH_ABS = 4e-5
TOL_FIRST_H0 = 1e-13   # trajectory 1 starts from the same chi on both sides
WORKLOADS = ["traj_8x8_b0.475", "traj_12x8_rhmc"]


def _load(name):
    path = os.path.join(GOLDEN, name + ".json")
    if not os.path.exists(path):
        pytest.skip(f"fixture {name}.json not generated")
    return json.load(open(path))


def _initial(cfg):
    kvol = cfg["L"] ** 2 * cfg["Lt"]
    if cfg["chi"] == "gauss12345":
        chi = np.random.default_rng(12345).standard_normal((3, kvol)) / np.sqrt(cfg["beta"])
        return chi, cfg["seed"]
    chi, seed, _ = chb.con_read(os.path.join(GOLDEN, cfg["chi"]), kvol)
    return chi, seed


@pytest.fixture(scope="module", params=WORKLOADS)
def golden_run(request, remez):
    gold = _load(request.param)
    cfg = gold["config"]
    chi, seed = _initial(cfg)
    prog = chb.Program(cfg["L"], cfg["Lt"], cfg["Ls"], cfg["dt"], cfg["beta"], cfg["am3"],
                       cfg["am"], cfg["hpin"], cfg["imass"], cfg["iterl"], remez["remez2"],
                       remez["remez4"], remez["remez2g"])
    prog.set_chi(chi)
    prog.startup(seed)
    prog.set_measure(cfg["iprint"], True)
    recs = []
    for _ in gold["records"]:
        r = prog.sweep()
        d = r.as_dict()
        d["cferm"] = prog.correlators().reshape(-1).tolist() if r.measured else None
        recs.append(d)
    final_seed = prog.seed()
    prog.close()
    diffs = []
    for g, o in zip(recs, gold["records"]):
        d = {f: abs(g[f] - o[f]) / abs(o[f]) for f in ("H0", "S0", "H1", "S1", "hg")}
        d["dH_abs"] = abs(g["dH"] - o["dH"])
        d["dH_rel_H0"] = d["dH_abs"] / abs(o["H0"])
        d["dH_rel_dH"] = d["dH_abs"] / abs(o["dH"]) if o["dH"] else None
        diffs.append(d)
    out = os.environ.get("CHDWF_TRAJ_OUT")
    if out:
        allout = json.load(open(out)) if os.path.exists(out) else {}
        allout[request.param] = diffs
        with open(out, "w") as f:
            json.dump(allout, f, indent=1)
    return request.param, gold, recs, final_seed, diffs


def test_stream_and_decisions_identical(golden_run):
    name, gold, recs, final_seed, _ = golden_run
    for k, (g, o) in enumerate(zip(recs, gold["records"])):
        assert g["nsteps"] == o["nsteps"], (name, k)
        assert g["x"] == o["x"], (name, k)
        assert g["accepted"] == o["accepted"], (name, k)
        assert g["measured"] == o["measured"], (name, k)
    assert final_seed == gold["final_seed"]


def test_hamiltonians_within_measured_envelope(golden_run):
    name, gold, recs, _, diffs = golden_run
    for k, d in enumerate(diffs):
        for f in ("H0", "S0", "H1", "S1", "hg", "dH_rel_H0"):
            assert d[f] <= TOL[f], (name, k, f, d[f])
        assert d["dH_abs"] <= TOL_DH_ABS, (name, k, d["dH_abs"])
    assert diffs[0]["H0"] <= TOL_FIRST_H0 and diffs[0]["S0"] <= TOL_FIRST_H0


def test_iterations_and_single_precision_outputs(golden_run):
    name, gold, recs, _, _ = golden_run
    for g, o in zip(recs, gold["records"]):
        for f in ("it_pf", "it_h0", "it_h1"):
            assert abs(g[f] - o[f]) <= ITER_ENVELOPE, (name, f, g[f], o[f])
        assert g["nforce"] == o["nforce"]
        for f in ("it_guid", "it_force"):
            assert abs(g[f] - o[f]) <= ITER_ENVELOPE * o["nforce"], (name, f)
        for f in ("action", "gaction", "paction", "vel2"):
            assert abs(g[f] - o[f]) <= 1e-5 * abs(o[f]), (name, f, g[f], o[f])
        if o["measured"]:
            assert abs(g["condmod"] - o["condmod"]) <= 1e-5 * abs(o["condmod"])
            assert abs(g["ancgm"] - o["ancgm"]) <= ITER_ENVELOPE
            cg, co = np.array(g["cferm"]), np.array(o["cferm"])
            assert np.abs(cg - co).max() <= 1e-4 * np.abs(co).max()
