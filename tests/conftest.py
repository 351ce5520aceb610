"""Shared fixtures for the test suite.

Markers: ``gpu`` -- needs a CUDA device (run with ``-m gpu`` on a B200).
Fixtures read only files committed under tests/golden/ (never the reference
checkout), so the suite runs unchanged on a machine without it.
"""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


def read_remez(name, n):
    """Parse a remez data file: a0, (a_k, sigma_k)*n, b0, (b_k, sigma_k)*n."""
    vals = []
    for line in open(os.path.join(GOLDEN, name)):
        line = line.replace(",", " ").replace("d", "e").replace("D", "e").strip()
        if line:
            vals.append([float(t) for t in line.split()])
    a0 = vals[0][0]
    an = np.array([v[0] for v in vals[1:n + 1]])
    ad = np.array([v[1] for v in vals[1:n + 1]])
    b0 = vals[n + 1][0]
    bn = np.array([v[0] for v in vals[n + 2:2 * n + 2]])
    bd = np.array([v[1] for v in vals[n + 2:2 * n + 2]])
    return {"anum": np.concatenate([[a0], an]), "aden": ad,
            "bnum": np.concatenate([[b0], bn]), "bden": bd}


@pytest.fixture(scope="session")
def remez():
    return {"remez2": read_remez("remez2", 25), "remez4": read_remez("remez4", 25),
            "remez2g": read_remez("remez2g", 12)}


@pytest.fixture(scope="session")
def seed_pins():
    return json.load(open(os.path.join(GOLDEN, "seed_pins.json")))


def read_con(path, kvol):
    """One Fortran unformatted record: chi(kvol,3) real*8 + seed real*8."""
    raw = open(path, "rb").read()
    n = int(np.frombuffer(raw[:4], dtype="<i4")[0])
    assert n == 8 * (3 * kvol + 1), (n, kvol)
    assert int(np.frombuffer(raw[4 + n:8 + n], dtype="<i4")[0]) == n
    vals = np.frombuffer(raw[4:4 + n], dtype="<f8")
    return vals[:-1].reshape(3, kvol).copy(), float(vals[-1])


@pytest.fixture(scope="session")
def con12():
    return read_con(os.path.join(GOLDEN, "con_12x12x12.bin"), 12 ** 3)


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def random_fields(L, Lt, Ls, seed=2024, chi_scale=1.0):
    rng = np.random.default_rng(seed)
    shape = (2, 4, Lt, L, L, Ls)
    R = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    chi = chi_scale * rng.standard_normal((3, L * L * Lt))
    return R, chi
