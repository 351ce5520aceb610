"""Generate the trajectory fixtures tests/golden/traj_*.json from the oracle.

The oracle (oracle/chdwf_oracle.c, a restatement of program dwf3d,
rhmc/cheisdwf.f:207-399) runs single-threaded, so its reductions follow the
reference's loop order (the reference run with OMP_NUM_THREADS=1).  Each
fixture holds, per trajectory, every scalar the main loop produces (H0, H1,
dH, S0, S1, hg, hp, y, x, decision, MD steps, solver iterations, REAL*4
observables), plus the final seed and a digest of the final chi.  The GPU
trajectory tests run the same chains and compare against these records.

    python tests/golden/make_traj_golden.py [name ...]

Workloads:
  traj_8x8_b0.475   L=Lt=8, Ls=8, beta=0.475, dt=0.1, iterl=10, hpin=0,
                    imass=1, chi from seeded N(0, 1/beta) (numpy default_rng
                    12345), the reference's default seed 693764523745
                    (rhmc/cheisdwf.f:1469); 12 trajectories, measuring every
                    5 (the reference's iprint).
  traj_12x8_rhmc    L=Lt=12, Ls=8 with the reference's shipped input deck
                    rhmc/midout (dt=0.125, beta=0.45, am3=1, am=0, hpin=0.5,
                    imass=1, iterl=8) and configuration rhmc/_con
                    (tests/golden/con_12x12x12.bin, its chi and seed);
                    10 trajectories, measuring every 5.
Remez sets: the shipped remez2, remez4 (25 poles) and remez2g (12 poles).
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import pyoracle as po  # noqa: E402
from conftest import read_con, read_remez  # noqa: E402

FIELDS = ("H0", "H1", "dH", "dS", "S0", "S1", "hg", "hp", "y", "x", "accepted", "nsteps",
          "it_pf", "it_h0", "it_h1", "it_guid", "it_force", "nforce", "action", "gaction",
          "paction", "vel2", "measured", "condmod", "susctot", "ancgm")

WORKLOADS = {
    "traj_8x8_b0.475": dict(L=8, Lt=8, Ls=8, beta=0.475, am3=1.0, dt=0.1, am=0.01, hpin=0.0,
                            imass=1, iterl=10, ntraj=12, iprint=5, chi="gauss12345",
                            seed=693764523745.0),
    "traj_12x8_rhmc": dict(L=12, Lt=12, Ls=8, beta=0.45, am3=1.0, dt=0.125, am=0.0, hpin=0.5,
                           imass=1, iterl=8, ntraj=10, iprint=5, chi="con_12x12x12.bin",
                           seed=None),
}


def initial_chi(cfg):
    kvol = cfg["L"] ** 2 * cfg["Lt"]
    if cfg["chi"] == "gauss12345":
        chi = np.random.default_rng(12345).standard_normal((3, kvol)) / np.sqrt(cfg["beta"])
        return chi, cfg["seed"]
    chi, seed = read_con(os.path.join(HERE, cfg["chi"]), kvol)
    return chi, seed


def chi_digest(chi):
    return hashlib.sha256(np.ascontiguousarray(chi, dtype="<f8").tobytes()).hexdigest()


def oracle_remez(r):
    return po.remez_struct(r["anum"][0], r["anum"][1:], r["aden"], r["bnum"][0], r["bnum"][1:],
                           r["bden"])


def run(name):
    cfg = WORKLOADS[name]
    rz = {"remez2": read_remez("remez2", 25), "remez4": read_remez("remez4", 25),
          "remez2g": read_remez("remez2g", 12)}
    chi, seed = initial_chi(cfg)
    sw = po.Sweeper(cfg["L"], cfg["Lt"], cfg["Ls"], cfg["beta"], cfg["am3"], cfg["dt"],
                    cfg["am"], cfg["hpin"], cfg["imass"], cfg["iterl"],
                    oracle_remez(rz["remez2"]), oracle_remez(rz["remez4"]),
                    oracle_remez(rz["remez2g"]), chi=chi, seed=seed, measure=True, threads=1)
    sw.st.contents.iprint = cfg["iprint"]
    recs = []
    t0 = time.time()
    for k in range(cfg["ntraj"]):
        r = sw.sweep()
        d = {f: getattr(r, f) for f in FIELDS}
        d["cond"] = list(r.cond)
        d["susc"] = list(r.susc)
        if r.measured:
            d["cferm"] = sw.cferm.reshape(-1).tolist()
        recs.append(d)
        print(f"{name}: trajectory {k + 1}/{cfg['ntraj']} dH={r.dH:.6e} acc={r.accepted} "
              f"nsteps={r.nsteps} ({time.time() - t0:.0f} s)", flush=True)
    out = {"workload": name, "config": cfg, "threads": 1, "records": recs,
           "final_seed": po.lib().orc_rranget(po.C.byref(sw.st.contents.rng)),
           "final_chi_sha256": chi_digest(sw.chi.copy().reshape(3, -1)),
           "final_chi_sum": float(np.sum(sw.chi)),
           "generator": "tests/golden/make_traj_golden.py (oracle, 1 thread)"}
    sw.close()
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {name}.json in {time.time() - t0:.0f} s")


if __name__ == "__main__":
    for n in (sys.argv[1:] or list(WORKLOADS)):
        run(n)
