"""Host logic of the learned closure's eddy-viscosity targets (CPU)."""
import numpy as np
import torch

from pyspectral_b200.learned import PAIRS, eddy_targets


def _sample(n, seed):
    rs = np.random.RandomState(seed)
    G = rs.standard_normal((n, 3, 3))
    G -= np.trace(G, axis1=1, axis2=2)[:, None, None] / 3 * np.eye(3)  # solenoidal: du_i/dx_i = 0
    X = np.concatenate([G.reshape(n, 9), np.full((n, 1), 0.1)], 1)
    S = 0.5 * (G + G.transpose(0, 2, 1))
    S6 = np.stack([S[:, a, b] for a, b in PAIRS], 1)
    return torch.tensor(X, dtype=torch.float32), S6


def test_eddy_targets_keep_an_eddy_viscosity_stress():
    X, S6 = _sample(64, 0)
    c = np.linspace(0.01, 0.5, 64)[:, None]
    T = torch.tensor(-2 * c * S6, dtype=torch.float32)
    got = eddy_targets(X, T).numpy()
    np.testing.assert_allclose(got, -2 * c * S6, rtol=1e-4, atol=1e-6)


def test_eddy_targets_drop_backscatter_and_the_part_not_aligned_with_s():
    X, S6 = _sample(64, 1)
    T = torch.tensor(+0.3 * S6, dtype=torch.float32)  # backscatter: -tau:S < 0
    assert np.abs(eddy_targets(X, T).numpy()).max() == 0.0
    rs = np.random.RandomState(2)
    T = rs.standard_normal((64, 6))
    got = eddy_targets(X, torch.tensor(T, dtype=torch.float32)).numpy().astype(np.float64)
    w = np.array([1, 1, 1, 2, 2, 2.0])
    nu = np.maximum(0, -(T * S6 * w).sum(1) / (2 * (S6 * S6 * w).sum(1)))
    np.testing.assert_allclose(got, -2 * nu[:, None] * S6, rtol=1e-4, atol=1e-6)
    # forward transfer kept: -got:S = max(0, -T:S); trace zero
    np.testing.assert_allclose(-(got * S6 * w).sum(1), np.maximum(0, -(T * S6 * w).sum(1)), rtol=1e-4, atol=1e-6)
    assert np.abs(got[:, :3].sum(1)).max() < 1e-5
