"""Statistical parity with the reference's own production run.

rhmc/Ls_8/b_0.45/out_1 (tests/golden/out_1_b0.45.txt) is the 'output' file
of a 2500-trajectory run of the reference at L=Lt=12, Ls=8, beta=0.45,
dt=0.125, am3=1, am=0, hpin=0, imass=1, iterl=8 (its midout), on the
reference's earlier single-precision build.  It prints:
  acceptances 2194 / 2500                        (out_1:11)
  <exp(dH)> = 1.003 +/- 0.00727                  (out_1:12)
  mean multi-shift iterations: guidance 613.3, acceptance 761.1,
                               force 630.6, pseudofermion 767.2  (out_1:13-14)
  condmod 0.119, mean square velocity 2.99, action per site 65.6 (out_1:18-21)
rhmc/Ls_8/b_0.45/_con (tests/golden/con_sp_12x12x12.bin) is that run's last
configuration, i.e. a configuration thermalised at these parameters, with
its seed.

The GPU program starts from it and runs NTRAJ trajectories of the same
parameters with the shipped Remez sets.  This pins the solver, the force and
the Hamiltonian statistically against numbers the reference produced:
  * acceptance rate within 4 combined binomial standard deviations;
  * <exp(dH)> against the reference's value within 4 combined standard
    errors, and against 1 (the exact value for a reversible, area-preserving
    integrator) within 4 of ours;
  * mean iterations per solve type between 0.80 and 1.00 of the
    reference's: the Lanczos stopping rule is the reference's, and the
    reference's single-precision Lanczos loses orthogonality and needs more
    iterations than FP64, the more so the tighter the tolerance.  Measured
    on a B200: 0.95 (guidance, 1e-6), 0.93 (force, 1e-6), 0.86 (acceptance,
    1e-9), 0.85 (pseudofermion, 1e-9);
  * mean square velocity, action per site and condmod within 5%
    (autocorrelated means over a short run).
Set CHDWF_STAT_OUT to a file path to write the measured summary as JSON.
"""
import json
import math
import os

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

NTRAJ = 400
NTHERM = 10
REF = dict(acc=2194, ntraj=2500, yav=1.003, yav_err=0.00727, guid=613.319, accept=761.103,
           force=630.598, pf=767.234, condmod=0.119, vel2=2.99, action=65.6)


@pytest.fixture(scope="module")
def chain(remez):
    L, Lt, Ls = 12, 12, 8
    chi, seed, single = chb.con_read(os.path.join(GOLDEN, "con_sp_12x12x12.bin"), L * L * Lt)
    assert single
    prog = chb.Program(L, Lt, Ls, 0.125, 0.45, 1.0, 0.0, 0.0, 1, 8, remez["remez2"],
                       remez["remez4"], remez["remez2g"])
    prog.set_chi(chi)
    prog.startup(seed)
    prog.set_measure(5, True)
    for _ in range(NTHERM):
        prog.sweep()
    prog.reset_sums()
    recs = [prog.sweep() for _ in range(NTRAJ)]
    av = prog.averages()
    prog.close()
    return recs, av


def test_statistics_against_reference_run(chain):
    recs, av = chain
    n = len(recs)
    acc = np.array([r.accepted for r in recs], dtype=float)
    y = np.array([r.y for r in recs], dtype=float)
    p, p_ref = acc.mean(), REF["acc"] / REF["ntraj"]
    sp = math.sqrt(p * (1 - p) / n + p_ref * (1 - p_ref) / REF["ntraj"])
    ym, ye = y.mean(), y.std(ddof=1) / math.sqrt(n)
    its = {k: float(getattr(av, f)) for k, f in
           (("guid", "ancg"), ("accept", "ancgh"), ("force", "ancgf"), ("pf", "ancgpf"))}
    summary = dict(ntraj=n, acceptance=p, acceptance_ref=p_ref, acceptance_sigma=sp,
                   yav=ym, yav_err=ye, yav_ref=REF["yav"], yav_ref_err=REF["yav_err"],
                   iterations=its, iterations_ref={k: REF[k] for k in its},
                   vel2=float(av.vel2a), action=float(av.actiona), condmod=float(av.condmoda),
                   atraj=float(av.atraj))
    out = os.environ.get("CHDWF_STAT_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(summary, f, indent=1)
    print(json.dumps(summary))
    assert abs(p - p_ref) <= 4 * sp, (p, p_ref, sp)
    assert abs(ym - REF["yav"]) <= 4 * math.sqrt(ye ** 2 + REF["yav_err"] ** 2), (ym, ye)
    assert abs(ym - 1.0) <= 4 * ye, (ym, ye)
    for k, v in its.items():
        assert 0.80 * REF[k] <= v <= 1.00 * REF[k], (k, v, REF[k])
    assert abs(av.vel2a - REF["vel2"]) <= 0.05 * REF["vel2"]
    assert abs(av.actiona - REF["action"]) <= 0.05 * REF["action"]
    assert abs(av.condmoda - REF["condmod"]) <= 0.05 * REF["condmod"] + 0.01
