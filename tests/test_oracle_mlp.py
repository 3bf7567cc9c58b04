"""The MLP oracle's analytic gradient agrees with central finite differences
(BF16 rounding switched off for the check)."""
import numpy as np
import pytest

from oracle import mlp_oracle as mo


@pytest.mark.parametrize("act,hidden", [("gelu", 64), ("relu", 64), ("relu", 32)])
def test_mlp_oracle_gradient_matches_finite_differences(monkeypatch, act, hidden):
    monkeypatch.setattr(mo, "bf16", lambda x: np.asarray(x, np.float64))
    rng = np.random.default_rng(0)
    X = rng.standard_normal((40, 10))
    T = rng.standard_normal((40, 6))
    norm = np.r_[np.zeros(10), np.ones(10), np.zeros(6), np.ones(6)]
    P = mo.init_params(1, hidden) + 0.01 * rng.standard_normal(mo.nparams(hidden))
    _, g = mo.loss_and_grad(P, norm, X, T, act=act)
    n = mo.nparams(hidden)
    for i in (0, 5, 10 * hidden + 3, 11 * hidden + 7, n - 7 * hidden, n - 20, n - 1):
        e = np.zeros_like(P)
        e[i] = 1e-6
        fd = (mo.loss_and_grad(P + e, norm, X, T, act=act)[0] - mo.loss_and_grad(P - e, norm, X, T, act=act)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 3.0e-3], dtype=np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) / 3.0e-3 < 2 ** -8


def test_device_gelu_erf_constants_meet_the_published_bound():
    """The device GELU evaluates erf by Abramowitz & Stegun 7.1.26 (|error| <=
    1.5e-7); the constants in the CUDA header must reproduce that bound."""
    import math
    import os
    import re
    from tests.helpers import ROOT
    src = open(os.path.join(ROOT, "pyspectral_b200", "csrc", "psb_mlp.cuh")).read()
    body = src[src.index("struct GeluAS"):]
    body = body[:body.index("};")]
    c = {k: float(v) for k, v in re.findall(r"(p|a[1-5]) = (-?[0-9.]+)f", body)}
    assert set(c) == {"p", "a1", "a2", "a3", "a4", "a5"}
    x = np.linspace(-8, 8, 40001)
    z = np.abs(x) / math.sqrt(2)
    t = 1 / (1 + c["p"] * z)
    poly = t * (c["a1"] + t * (c["a2"] + t * (c["a3"] + t * (c["a4"] + t * c["a5"]))))
    q = poly * np.exp(-0.5 * x * x)
    approx = np.where(x >= 0, 2 - q, q)
    exact = 1 + np.array([math.erf(v / math.sqrt(2)) for v in x])
    assert np.abs(approx - exact).max() < 1.5e-7


def test_device_forward_gelu_erf_constants_meet_the_published_bound():
    """The device forward GELU evaluates erf by Abramowitz & Stegun 7.1.28
    (|error| <= 3e-7); the constants in the CUDA header must meet it."""
    import math
    import os
    import re
    from tests.helpers import ROOT
    src = open(os.path.join(ROOT, "pyspectral_b200", "csrc", "psb_mlp.cuh")).read()
    body = src[src.index("struct GeluAS28"):]
    body = body[:body.index("};")]
    c = {k: float(v) for k, v in re.findall(r"(a[1-6]) = (-?[0-9.]+)f", body)}
    assert set(c) == {"a1", "a2", "a3", "a4", "a5", "a6"}
    z = np.linspace(0, 8, 40001)
    P = 1 + sum(c[f"a{i}"] * z ** i for i in range(1, 7))
    exact = np.array([math.erf(v) for v in z])
    assert np.abs((1 - P ** -16.0) - exact).max() < 3e-7
