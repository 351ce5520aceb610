"""The multi-pseudofermion variant (csrc/ext.cu, chdwf_prog_set_ext): no
counterpart in the reference, checked by identities and against the
reference-mode program.

  * with one field and the reference's own functions (remez4 a for the
    heatbath, remez2 b for the action) the first trajectory starts from the
    same Gaussians and momenta as the reference-mode sweep, so H0 and S0 are
    the same numbers: bit-identical;
  * the force of chdwf_ext_force is the chi-gradient of
    beta sum chi^2 + sum_i Re Phi_i^dag r_act(M^dag M) Phi_i (a central
    difference of the action with Richardson extrapolation, solves at
    1e-12): within 2e-5 of sum |dSdchi| |delta| (dSdchi is REAL*4);
  * the integrators are second order: over the same draws |dH| falls by at
    least 2.5x when dt halves (4x in the limit), for Omelyan and leapfrog;
  * FP32 force solves keep the FP64 chain's decisions; the dH difference is
    printed and bounded by 1e-8 |H0|.
"""
import ctypes as C
import os

import numpy as np
import pytest

import chiralheisenberg_b200 as chb
from chiralheisenberg_b200.remez import read_remez_file

pytestmark = pytest.mark.gpu

DATA = os.path.join(os.path.dirname(chb.__file__), "data")
SEED = 693764523745.0


def ext_sets():
    """(heatbath, action) sets for two fields: x^(1/8) and x^(-1/4), 20 poles."""
    a8, d8, _, _ = read_remez_file(os.path.join(DATA, "remez8_20"), 20)
    _, _, b4, e4 = read_remez_file(os.path.join(DATA, "remez4_20"), 20)
    return (a8, d8), (b4, e4)


def make_prog(remez, L=6, Ls=6, dt=0.1, beta=0.475, seed_chi=99):
    prog = chb.Program(L, L, Ls, dt, beta, 1.0, 0.01, 0.0, 1, 10, remez["remez2"],
                       remez["remez4"], remez["remez2g"])
    chi = np.random.default_rng(seed_chi).standard_normal((3, L ** 3)) / np.sqrt(beta)
    prog.set_chi(chi)
    prog.startup(SEED)
    prog.set_measure(5, False)
    return prog, chi


def test_single_field_reproduces_reference_H0(remez):
    ref, chi = make_prog(remez)
    r0 = ref.sweep()
    ref.close()
    ext, _ = make_prog(remez)
    hb = (remez["remez4"]["anum"], remez["remez4"]["aden"])
    act = (remez["remez2"]["bnum"], remez["remez2"]["bden"])
    ext.set_ext(1, 4, hb, act, integrator="leapfrog")
    e0 = ext.sweep()
    ext.close()
    assert e0.H0 == r0.H0 and e0.S0 == r0.S0, (e0.H0, r0.H0)
    assert e0.it_pf == r0.it_pf and e0.it_h0 == r0.it_h0


def test_ext_force_is_gradient_of_action(remez):
    import torch
    L, Ls, beta = 6, 6, 0.475
    prog, chi = make_prog(remez, L=L, Ls=Ls, beta=beta)
    hb, act = ext_sets()
    prog.set_ext(2, 1, hb, act)
    lib, ctx = prog.lib, prog.context
    kvol = L ** 3
    rng = np.random.default_rng(5)
    gauss = (rng.standard_normal((2, 16 * kvol * Ls)) * np.sqrt(0.5)).astype(np.float32)
    gdev = torch.from_numpy(gauss).cuda()
    pp = np.zeros((3, kvol), np.float32)
    assert lib.chdwf_traj_set_chi(ctx, chi.ctypes.data_as(C.c_void_p)) == 0
    assert lib.chdwf_traj_begin(ctx) == 0
    assert lib.chdwf_traj_set_momenta(ctx, pp.ctypes.data_as(C.c_void_p)) == 0
    for i in range(2):
        it = C.c_int()
        assert lib.chdwf_ext_select_pf(ctx, i) == 0
        assert lib.chdwf_ext_heatbath_dev(ctx, C.c_void_p(gdev[i].data_ptr()), 1e-12, 0.0, 1,
                                          C.byref(it)) == 0

    def action(x):
        x = np.ascontiguousarray(x)
        assert lib.chdwf_traj_set_chi(ctx, x.ctypes.data_as(C.c_void_p)) == 0
        assert lib.chdwf_traj_begin(ctx) == 0
        b = np.zeros(2)
        assert lib.chdwf_ext_bosonic(ctx, b.ctypes.data_as(C.c_void_p)) == 0
        tot = b[1]
        for i in range(2):
            h, it = C.c_double(), C.c_int()
            assert lib.chdwf_ext_select_pf(ctx, i) == 0
            assert lib.chdwf_ext_action(ctx, 1e-12, 0.0, 1, C.byref(h), C.byref(it)) == 0
            tot += h.value
        return tot

    assert lib.chdwf_traj_set_chi(ctx, chi.ctypes.data_as(C.c_void_p)) == 0
    assert lib.chdwf_traj_begin(ctx) == 0
    for i in range(2):
        it = C.c_int()
        assert lib.chdwf_ext_select_pf(ctx, i) == 0
        assert lib.chdwf_ext_force(ctx, 1e-12, 0.0, 1, 1 if i == 0 else 0, C.byref(it)) == 0
    dS = np.empty((3, kvol), np.float32)
    assert lib.chdwf_traj_get_force(ctx, dS.ctypes.data_as(C.c_void_p)) == 0
    delta = rng.standard_normal((3, kvol))

    def central(h):
        return (action(chi + h * delta) - action(chi - h * delta)) / (2 * h)

    # The operator couples chi rounded to REAL*4 (the reference's KIND-less
    # cmplx), which quantises a step below ~1e-4; steps of 4e-3 and 2e-3
    # with Richardson extrapolation remove the h^2 term instead.
    fd = (4 * central(2e-3) - central(4e-3)) / 3
    an = float(np.sum(dS.astype(np.float64) * delta))
    scale = float(np.sum(np.abs(dS) * np.abs(delta)))
    prog.close()
    print(f"directional derivative: difference {fd:.9e}, force {an:.9e}")
    assert abs(fd - an) <= 2e-5 * scale, (fd, an, scale)


@pytest.mark.parametrize("integrator", ["omelyan", "leapfrog"])
def test_ext_integrator_second_order(remez, integrator):
    hb, act = ext_sets()
    dh = {}
    for dt, ns in ((0.1, 4), (0.05, 8)):
        prog, _ = make_prog(remez, dt=dt)
        prog.set_ext(2, ns, hb, act, integrator=integrator)
        dh[dt] = [abs(prog.sweep().dH) for _ in range(3)]
        prog.close()
    ratio = np.mean(dh[0.1]) / np.mean(dh[0.05])
    print(f"{integrator}: |dH| {np.mean(dh[0.1]):.3e} -> {np.mean(dh[0.05]):.3e}, ratio {ratio:.2f}")
    assert ratio >= 2.5


def test_ext_mixed_precision_decisions(remez):
    hb, act = ext_sets()
    recs = {}
    for mode in ("f64", "f32"):
        prog, _ = make_prog(remez)
        prog.set_ext(2, 5, hb, act)
        prog.set_precision(md=mode, accept="f64")
        recs[mode] = [prog.sweep() for _ in range(3)]
        prog.close()
    for a, b in zip(recs["f64"], recs["f32"]):
        print(f"dH fp64 {a.dH:.9e} mixed {b.dH:.9e} diff {abs(a.dH - b.dH):.3e}")
        assert a.accepted == b.accepted
        assert abs(a.dH - b.dH) <= 1e-8 * abs(a.H0)
