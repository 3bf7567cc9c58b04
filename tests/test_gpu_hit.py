"""The decaying-turbulence runner (pyspectral_b200.hit) against the oracle.

Every closure of the case -- Smagorinsky, the t-model (memory coefficient
Ct * t with t advanced per step, as the loop of PySpectral/src/PySpec_3d.py:
107-148 does), the static and the dynamic tau-model -- run by the runner for
20 RK4 steps from the seeded isotropic field, and by the oracle from the same
field: the final state, the energy / enstrophy history the runner records
(on the state each step's last stage read, src/PySpec_3d.py:129) and E(k)
at the end agree to 1e-11 in FP64.
"""
import numpy as np
import pytest

from oracle import spectral_oracle as orc

pytestmark = pytest.mark.gpu

N, STEPS, EVERY, DT, NU = 16, 20, 5, 2e-3, 1e-3

# name -> oracle (rhs, field the RHS read); the memory closures read the state
# with its Nyquist modes zeroed (main.uhat), Smagorinsky reads it unchanged
ORACLE = {
    "smag": lambda g, q, t: (orc.rhs_smag(g, q, orc.Params(nu=NU, t=t))[0], q),
    "tmodel": lambda g, q, t: orc.rhs_tmodel(g, q, orc.Params(nu=NU, t=t, Ct=0.1))[::2],
    "tau_static": lambda g, q, t: orc.rhs_staumodel(g, q, orc.Params(nu=NU, t=t, tau_a=0.05, tau_b=0.2))[0:3:2],
    "tau_dynamic": lambda g, q, t: orc.rhs_dtaumodel(g, q, orc.Params(nu=NU, t=t))[0:3:2],
}


def _oracle_run(name, st):
    """Oracle history: (t, energy, enstrophy) every EVERY steps, final state and read field."""
    g = orc.Grid.periodic(N)
    fn = ORACLE[name]
    hist = [(0.0, orc.energy(g, st[:3]), orc.enstrophy(g, st[:3]))]
    q, t, read = st.copy(), 0.0, None
    for s in range(STEPS):
        tt = t
        q, read = orc.advance_rk4(q, lambda x: fn(g, x, tt), DT)
        t += DT
        if (s + 1) % EVERY == 0:
            hist.append((t, orc.energy(g, read[:3]), orc.enstrophy(g, read[:3])))
    return hist, q, read, g


@pytest.mark.parametrize("name", sorted(ORACLE))
def test_hit_runner_matches_oracle(name):
    from pyspectral_b200 import hit

    st = orc.isotropic_state(N, 3, k0=4.0)
    res, main, _ = hit.run_case(N, name, STEPS, precision=64, every=EVERY, dt=DT, nu=NU, state=st)
    hist, q, read, g = _oracle_run(name, st)
    assert res["finite"]
    assert len(res["history"]) == len(hist)
    for h, (t, e, z) in zip(res["history"], hist):
        assert abs(h["t"] - t) < 1e-12
        assert abs(h["energy"] - np.real(e)) <= 1e-11 * abs(np.real(e))
        assert abs(h["enstrophy"] - np.real(z)) <= 1e-11 * abs(np.real(z))
        assert abs(h["dissipation"] - 2 * NU * np.real(z)) <= 1e-11 * abs(2 * NU * np.real(z))
    got = main.Q.cpu().numpy()
    assert np.abs(got[:3] - q[:3]).max() <= 1e-11 * np.abs(q[:3]).max()
    k, E = orc.spectrum(g, read[:3])
    E = np.real(np.asarray(E)).sum(1)
    Eg = np.asarray(res["E_k"])
    assert Eg.shape == E.shape
    assert np.abs(Eg - E).max() <= 1e-11 * np.abs(E).max()


def test_hit_fp32_smagorinsky_tracks_fp64():
    """FP32 fields + Kahan over 200 steps stay within 1e-5 of the FP64 run (energy, fields)."""
    from pyspectral_b200 import hit

    st = orc.isotropic_state(32, 4, k0=4.0)
    r64, m64, _ = hit.run_case(32, "smag", 200, precision=64, every=50, dt=DT, nu=NU, state=st)
    r32, m32, _ = hit.run_case(32, "smag", 200, precision=32, every=50, dt=DT, nu=NU, state=st)
    e64 = np.array([h["energy"] for h in r64["history"]])
    e32 = np.array([h["energy"] for h in r32["history"]])
    assert np.abs(e32 - e64).max() <= 1e-5 * np.abs(e64).max()
    assert hit.rel_diff(m32.Q.cpu().numpy(), m64.Q.cpu().numpy()) < 1e-5
