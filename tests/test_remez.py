"""The Remez generator (chiralheisenberg_b200/remez.py) against the
reference's own rational approximations, and the generated data files.

The reference ships remez2g (rhmc/remez2g, tests/golden/remez2g): 12-pole
approximations of x^(1/2) (a-set) and x^(-1/2) (b-set).  Their relative error
equioscillates on [1e-4, 50] at the level 7.2515e-7, i.e. they are the
minimax approximations there, which are unique.  The generator, run on the
same function, degree and interval, must return the same coefficients: it
does so to the last bits of double precision (bound 1e-13 relative).

The 20-pole files of the multi-pseudofermion variant (data/remez4_20,
data/remez8_20, made by data/make_remez.py) are checked in double precision:
their relative error is below 1e-10 on [1e-4, 50] and alternates in sign at
least 2n+1 times between extrema at the level (the minimax signature).
"""
import os

import numpy as np
import pytest

import chiralheisenberg_b200
from chiralheisenberg_b200.remez import read_remez_file, remez
from conftest import read_remez

DATA = os.path.join(os.path.dirname(chiralheisenberg_b200.__file__), "data")


def test_generator_reproduces_shipped_remez2g():
    r, rinv = remez("1/2", 1e-4, 50.0, 12, digits=60)
    g = read_remez("remez2g", 12)
    assert abs(r.error - 7.2515e-7) < 1e-10
    assert abs(r.a0 / g["anum"][0] - 1) < 1e-13
    assert np.abs(np.array(r.a) / g["anum"][1:] - 1).max() < 1e-13
    assert np.abs(np.array(r.sigma) / g["aden"] - 1).max() < 1e-13
    assert abs(rinv.a0 / g["bnum"][0] - 1) < 1e-13
    assert np.abs(np.array(rinv.a) / g["bnum"][1:] - 1).max() < 1e-13
    assert np.abs(np.array(rinv.sigma) / g["bden"] - 1).max() < 1e-13


def _eval(num, den, x):
    return num[0] + sum(num[k + 1] / (x + den[k]) for k in range(len(den)))


@pytest.mark.parametrize("name,power", [("remez4_20", 0.25), ("remez8_20", 0.125)])
def test_generated_files_are_minimax(name, power):
    an, ad, bn, bd = read_remez_file(os.path.join(DATA, name), 20)
    assert (ad > 0).all() and (bd > 0).all()
    x = np.logspace(-4, np.log10(50.0), 200001)
    for num, den, pw in ((an, ad, power), (bn, bd, -power)):
        e = _eval(num, den, x) / x ** pw - 1
        lev = np.abs(e).max()
        assert lev < 1e-10, lev
        big = np.abs(e) > 0.9 * lev
        signs = np.sign(e[big])
        changes = int(np.sum(signs[1:] != signs[:-1]))
        assert changes >= 2 * 20 + 1, changes
