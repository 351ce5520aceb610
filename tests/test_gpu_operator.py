"""GPU parity of the FP64 operator against the oracle, through the C ABI.

The kernel evaluates each output element with the same sequence of IEEE
operations as the reference's sweeps (no fused multiply-add), so the
comparison is bit-exact."""
import numpy as np
import pytest

import pyoracle as po
import chiralheisenberg_b200 as chb
from conftest import random_fields

pytestmark = pytest.mark.gpu

CASES = [(4, 4, 4), (3, 5, 2), (8, 8, 8), (6, 4, 7), (12, 12, 8)]


@pytest.mark.parametrize("L,Lt,Ls", CASES)
@pytest.mark.parametrize("imass", [1, 3])
@pytest.mark.parametrize("dag", [False, True])
def test_operator_bit_exact(L, Lt, Ls, imass, dag):
    R, chi = random_fields(L, Lt, Ls, seed=L * 100 + Lt * 10 + Ls)
    hpin = 0.37 if imass == 1 else 0.0
    lat = po.make_lat(L, Lt, Ls, beta=0.475, am3=1.0)
    ref = po.dslash(lat, R, chi, hpin=hpin, imass=imass, dag=dag)
    gl = chb.Lattice(L, Lt, Ls, beta=0.475, am3=1.0)
    out = (gl.dslashd if dag else gl.dslash)(R, chi, hpin=hpin, imass=imass)
    assert np.array_equal(out.view(np.float64), ref.view(np.float64))


@pytest.mark.parametrize("ibound,am3", [(1, 1.0), (-1, 0.7)])
def test_operator_boundary_and_height(ibound, am3):
    L, Lt, Ls = 4, 6, 4
    R, chi = random_fields(L, Lt, Ls, seed=11)
    lat = po.make_lat(L, Lt, Ls, am3=am3, ibound=ibound)
    gl = chb.Lattice(L, Lt, Ls, am3=am3, ibound=ibound)
    for dag in (False, True):
        ref = po.dslash(lat, R, chi, imass=1, dag=dag)
        out = (gl.dslashd if dag else gl.dslash)(R, chi, imass=1)
        assert np.array_equal(out.view(np.float64), ref.view(np.float64))


def test_operator_shipped_configuration(con12):
    """12^3 x 8 with the reference's own chi configuration (rhmc/_con)."""
    chi, _ = con12
    L, Lt, Ls = 12, 12, 8
    R, _ = random_fields(L, Lt, Ls, seed=12)
    lat = po.make_lat(L, Lt, Ls, beta=0.45)
    gl = chb.Lattice(L, Lt, Ls, beta=0.45)
    for dag in (False, True):
        ref = po.dslash(lat, R, chi, hpin=0.5, imass=1, dag=dag)
        out = (gl.dslashd if dag else gl.dslash)(R, chi, hpin=0.5, imass=1)
        assert np.array_equal(out.view(np.float64), ref.view(np.float64))


def test_operator_large_lattice_adjoint():
    """At 24^3 x 24 (oracle too slow for every case): <y,Mx> = <M^dag y,x>
    and linearity M(ax+y) = aMx + My to rounding."""
    L, Lt, Ls = 24, 24, 24
    x, chi = random_fields(L, Lt, Ls, seed=13)
    y, _ = random_fields(L, Lt, Ls, seed=14)
    gl = chb.Lattice(L, Lt, Ls)
    Mx = gl.dslash(x, chi, hpin=0.2)
    Mdy = gl.dslashd(y, chi, hpin=0.2)
    a, b = np.vdot(y, Mx), np.vdot(Mdy, x)
    assert abs(a - b) <= 1e-12 * abs(a)
    Mlin = gl.dslash(2.5 * x + y, chi, hpin=0.2)
    My = gl.dslash(y, chi, hpin=0.2)
    assert np.linalg.norm(Mlin - (2.5 * Mx + My)) <= 1e-13 * np.linalg.norm(Mlin)


# The operator sweep's lattices (L=Lt in {16, 24, 32, 48}, Ls in {16, 24,
# 32}): FP64 M and M^dagger bit-exact against the oracle at the sizes the
# sweep times.  48^3 x 16 (a 226 MB spinor) is checked for M only.
SWEEP_CASES = [(16, 16, False), (16, 16, True), (16, 24, False), (16, 32, True),
               (24, 16, True), (24, 24, False), (24, 24, True), (24, 32, False),
               (32, 16, False), (32, 24, True), (48, 16, False)]


@pytest.mark.parametrize("L,Ls,dag", SWEEP_CASES)
def test_operator_bit_exact_sweep_sizes(L, Ls, dag):
    R, chi = random_fields(L, L, Ls, seed=2024 + L + Ls)
    lat = po.make_lat(L, L, Ls, beta=0.475, am3=1.0)
    ref = po.dslash(lat, R, chi, hpin=0.0, imass=1, dag=dag)
    gl = chb.Lattice(L, L, Ls, beta=0.475, am3=1.0)
    out = (gl.dslashd if dag else gl.dslash)(R, chi, hpin=0.0, imass=1)
    gl.close()
    assert np.array_equal(out.view(np.float64), ref.view(np.float64))
