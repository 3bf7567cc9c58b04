"""CPU checks of the MHD t-model oracle (no reference counterpart): the
structural properties that pin it in place of golden vectors.

* the memory term is solenoidal in both fields;
* it drains exactly the energy of the unresolved tendency,
  <(u,B), PLQL(u,B)> = -|QL(u,B)|^2, which holds only when L is evaluated
  without aliasing and its linearisation is exact (skew-symmetry of the ideal
  MHD operator);
* with B = 0 no magnetic memory arises; at t = 0 the closure is plain MHD,
  whose oracle is pinned to the reference's own outputs."""
import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import golden, rel


def _solenoidal(g, rng):
    N1, N2, N3 = g.N1, g.N2, g.N3
    s = np.stack([np.fft.rfftn(a) for a in rng.standard_normal((3, N1, N2, N3))])
    k1, k2, k3 = g.k1[:, None, None], g.k2[None, :, None], g.k3[None, None, :]
    div = (k1 * s[0] + k2 * s[1] + k3 * s[2]) * g.ksqr_i
    return np.stack([s[0] - k1 * div, s[1] - k2 * div, s[2] - k3 * div]) * g.dealias_mask


def _wsum(a, n3h):
    w = np.full(n3h, 2.0)
    w[0] = 1.0
    w[-1] = 1.0
    return float(np.sum(w * a))


@pytest.mark.parametrize("shape", [(12, 12, 12), (16, 12, 20)])
def test_memory_is_solenoidal_and_drains_the_unresolved_energy(shape):
    N1, N2, N3 = shape
    g = orc.MHDGrid(N1, N2, N3, N1 // 2)
    rng = np.random.default_rng(5)
    st = np.concatenate([_solenoidal(g, rng), _solenoidal(g, rng)])
    mem, QL = orc.mhd_tmodel_memory(g, st, 1.0, 1.0, return_ql=True)
    k1, k2, k3 = g.k1[:, None, None], g.k2[None, :, None], g.k3[None, None, :]
    assert np.abs(k1 * mem[0] + k2 * mem[1] + k3 * mem[2]).max() < 1e-12 * np.abs(mem[:3]).max()
    assert np.abs(k1 * mem[3] + k2 * mem[4] + k3 * mem[5]).max() < 1e-12 * np.abs(mem[3:]).max()
    dE = _wsum(sum((st[i].conj() * mem[i]).real for i in range(6)), N3 // 2 + 1)
    q2 = _wsum(sum(np.abs(QL[i]) ** 2 for i in range(6)), N3 + 1)
    assert q2 > 0
    assert dE == pytest.approx(-q2, rel=1e-11)


def test_no_magnetic_memory_without_field_and_plain_mhd_at_t0():
    N = 12
    g = orc.MHDGrid(N, N, N, N // 2)
    rng = np.random.default_rng(6)
    st = np.concatenate([_solenoidal(g, rng), np.zeros((3, N, N, N // 2 + 1), complex)])
    mem = orc.mhd_tmodel_memory(g, st, 0.1, 0.5)
    assert np.abs(mem[:3]).max() > 0
    assert np.abs(mem[3:]).max() == 0.0
    d = golden("mhd_N12.npz")
    r, _ = orc.rhs_mhd_tmodel(g, d["state"], float(d["nu"]), 0.1, 0.0, force=d["force"])
    assert rel(r, d["rhs"]) < 1e-13
