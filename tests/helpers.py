"""Shared helpers of the test suite."""
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

# Closure cases of the golden fixtures (tests/golden/make_golden.py): name ->
# (turb_model, variables kwargs, oracle Params kwargs).  nu=0.02, dt=0.01, t=0.37.
CASES = {
    "dns": (0, {}, {}),
    "dns_rot": (0, dict(rotate=1, Om=(0.3, -0.2, 0.5)), dict(rotate=1, Om=(0.3, -0.2, 0.5))),
    "smag": (1, {}, {}),
    "smag_rot": (1, dict(rotate=1, Om=(0.1, 0.4, -0.25)), dict(rotate=1, Om=(0.1, 0.4, -0.25))),
    "tmodel": (2, dict(Ct=0.13), dict(Ct=0.13)),
    "tmodel_rot": (2, dict(rotate=1, Om=(0.2, 0.0, 0.3)), dict(rotate=1, Om=(0.2, 0.0, 0.3), Ct=0.1)),
    "stau": ("Static tau-model", dict(dt0=0.05, dt1=0.2), dict(tau_a=0.05, tau_b=0.2)),
    "dtau": ("Dynamic tau-model", {}, {}),
    "dsmag": (7, {}, {}),
    "dsmag_rot": (7, dict(rotate=1, Om=(-0.15, 0.35, 0.2)), dict(rotate=1, Om=(-0.15, 0.35, 0.2))),
    "cm1": (6, {}, {}),
    "budgets": (99, {}, {}),
    "fm1": (3, dict(dt0=0.05), {}),
    "fm1_rot": (3, dict(dt0=0.05, rotate=1, Om=(0.25, -0.1, 0.4)), dict(rotate=1, Om=(0.25, -0.1, 0.4))),
}
NU, DT, T = 0.02, 0.01, 0.37


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b):
    """max-norm relative difference |a-b|_inf / |b|_inf."""
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
