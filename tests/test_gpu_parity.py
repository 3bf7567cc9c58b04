"""GPU parity: every RHS, the RK4 step and the diagnostics through the public
API (the C ABI underneath) against the reference's own outputs (golden
fixtures) and against the CPU oracle.  FP64 bar: 1e-12 relative (max norm).
FP32 bar: 2e-5 relative to the FP64 result."""
import math

import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import CASES, DT, NU, T, golden, rel

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 2e-5


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _main(name, N, state, precision=64):
    from pyspectral_b200 import Classes as C
    tm, kw, _ = CASES[name]
    grid = C.gridclass.periodic(N)
    kw = dict(kw)
    Om = kw.pop("Om", (0.0, 0.0, 0.0))
    main = C.variables(0, tm, kw.pop("rotate", 0), Om[0], Om[1], Om[2], grid, state[0], state[1], state[2], T, DT,
                       NU, precision=precision, **kw)
    return grid, main


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name", list(CASES))
def test_rhs_matches_reference(N, name):
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(name, N, d["state"])
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), d[f"{name}_rhs"]) < TOL64
    assert rel(np_(main.U), d[f"{name}_uhat"]) < TOL64
    if f"{name}_w0" in d:
        assert rel(np_(main.W0), d[f"{name}_w0"]) < TOL64
    if f"{name}_tau" in d:
        assert main.tau == pytest.approx(float(d[f"{name}_tau"]), rel=1e-11)


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name", list(CASES))
def test_rk4_step_matches_reference(N, name):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(name, N, d["state"])
    advanceQ_RK4(main, grid, None, C.utilitiesClass())
    assert rel(np_(main.Q), d[f"{name}_step"]) < TOL64
    assert rel(np_(main.U), d[f"{name}_step_uhat"]) < TOL64


@pytest.mark.parametrize("N", [12, 16])
def test_diagnostics_match_reference(N):
    from pyspectral_b200 import Classes as C
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main("dns", N, d["state"])
    grid = C.gridclass.periodic(N, kc=int(d["diag_kc"]))
    main.U.copy_(main.Q)
    u = C.utilitiesClass()
    assert u.computeEnergy(main, grid) == pytest.approx(float(d["energy"]), rel=1e-13)
    assert u.computeEnergy_resolved(main, grid) == pytest.approx(float(d["energy_resolved"]), rel=1e-13)
    assert u.computeEnstrophy(main, grid) == pytest.approx(float(d["enstrophy"]), rel=1e-13)
    np.testing.assert_allclose(np.array(u.computeAllStats(main, grid)), d["allstats"], rtol=1e-12)
    k, s = u.computeSpectrum(main, grid)
    np.testing.assert_array_equal(k, d["spectrum_k"])
    assert rel(s, d["spectrum"]) < 1e-13
    k, s = u.computeSpectrum_resolved(main, grid)
    np.testing.assert_array_equal(k, d["spectrum_res_k"])
    assert rel(s, d["spectrum_res"]) < 1e-13
    w = u.computeSGS_DNS(main, grid, None)
    assert rel(np.stack([np_(x[..., 0]) for x in w]), d["sgs_dns_w0"]) < TOL64
    main.cfl = 0.4
    u.compute_dt(main, grid)
    assert main.dt == pytest.approx(float(d["cfl_dt"]), rel=1e-12)


@pytest.mark.parametrize("N", [12, 16])
def test_mhd_matches_reference(N):
    torch = _torch()
    from pyspectral_b200 import mpi as M
    d = golden(f"mhd_N{N}.npz")
    nu, dt = float(d["nu"]), float(d["dt"])
    grid = M.gridclass.periodic(N)
    x = [np.fft.irfftn(d["state"][i], s=(N, N, N), axes=(0, 1, 2)) for i in range(6)]
    main = M.variables("MHD", 0, 0, 0, 0, grid, *x, t=0.0, dt=dt, nu=nu)
    # r2c of the physical fields and of the forcing reproduce the reference's spectra
    assert rel(np_(main.Q), d["state"]) < 1e-13
    assert rel(np_(main.force), d["force"]) < 1e-13
    Q0 = main.Q.clone()
    M.computeRHS_MHD(main, grid, None)
    assert rel(np_(main.Q), d["rhs"]) < TOL64
    main.Q = Q0
    M.advanceQ_RK4(main, grid, None)
    assert rel(np_(main.Q), d["step"]) < TOL64
    main.U.copy_(torch.as_tensor(d["diag_state"], device=main.U.device))
    u = M.utilitiesClass()
    assert u.computeEnergy(main, grid) == pytest.approx(float(d["energy_u"]), rel=1e-13)
    assert u.computeMHDEnergy(main, grid) == pytest.approx(float(d["energy_B"]), rel=1e-13)
    assert rel(u.computeSpectrum(main, grid)[1], d["spectrum_u"]) < 1e-13
    assert rel(u.computeMHDSpectrum(main, grid)[1], d["spectrum_B"]) < 1e-13


@pytest.mark.parametrize("shape", [(16, 24, 12), (24, 16, 32)])
@pytest.mark.parametrize("name", ["dns_rot", "smag", "tmodel", "dsmag", "cm1", "budgets", "fm1"])
def test_noncubic_grid_matches_oracle(shape, name):
    torch = _torch()
    from pyspectral_b200 import Classes as C
    N1, N2, N3 = shape
    rng = np.random.default_rng(7)
    st = (rng.standard_normal((3, N1, N2, N3 // 2 + 1)) + 1j * rng.standard_normal((3, N1, N2, N3 // 2 + 1)))
    st *= np.exp(-0.05 * np.arange(N3 // 2 + 1))
    # Hermitian-consistent via a real-space round trip
    st = np.stack([np.fft.rfftn(np.fft.irfftn(s, s=(N1, N2, N3), axes=(0, 1, 2))) for s in st])
    L = 2 * np.pi
    g = orc.Grid(N1, N2, N3, L / N1, L / N2, L / N3, min(N1, N2, N3) // 2)
    tm, kw, okw = CASES[name]
    p = orc.Params(nu=NU, t=T, dt=DT, **okw)
    fn = {"dns": orc.rhs_nosgs, "smag": orc.rhs_smag, "tmodel": orc.rhs_tmodel, "dsmag": orc.rhs_dsmag,
          "cm1": orc.rhs_cm1, "budgets": orc.rhs_budgets,
          "fm1": lambda g, s, p: orc.rhs_fm1(g, s, p, dt0=0.05)}[name.split("_")[0]]
    ost = np.concatenate([st, np.zeros_like(st)]) if tm in (3, 6) else st
    ref = fn(g, ost, p)[0]
    a1, a2, a3 = (np.arange(n) * (L / n) for n in shape)
    y, x, z = np.meshgrid(a2, a1, a3)
    grid = C.gridclass(N1, N2, N3, x, y, z, min(N1, N2, N3) // 2)
    kw = dict(kw)
    Om = kw.pop("Om", (0.0, 0.0, 0.0))
    main = C.variables(0, tm, kw.pop("rotate", 0), Om[0], Om[1], Om[2], grid, st[0], st[1], st[2], T, DT, NU, **kw)
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), ref) < TOL64
    del torch


@pytest.mark.parametrize("N", [8, 12, 16, 24, 32, 48, 64])
@pytest.mark.parametrize("precision", [64, 32])
def test_plain_transforms_match_numpy(N, precision):
    torch = _torch()
    from pyspectral_b200 import _capi
    ctx = _capi.Context(N, N, N, precision=precision)
    rng = np.random.default_rng(N)
    x = rng.standard_normal((2, N, N, N))
    rd = torch.float64 if precision == 64 else torch.float32
    cd = torch.complex128 if precision == 64 else torch.complex64
    X = torch.as_tensor(x, device="cuda", dtype=rd).contiguous()
    S = torch.empty((2, N, N, N // 2 + 1), device="cuda", dtype=cd)
    ctx.r2c(X, S, 2)
    ref = np.stack([np.fft.rfftn(a) for a in x])
    tol = 1e-14 if precision == 64 else 2e-6
    assert rel(np_(S), ref) < tol
    Y = torch.empty_like(X)
    ctx.c2r(S, Y, 2)
    assert rel(np_(Y), x) < tol


@pytest.mark.parametrize("name", list(CASES))
def test_fp32_rhs_tracks_fp64(name):
    _torch()
    d = golden("serial_N16.npz")
    grid, m64 = _main(name, 16, d["state"], 64)
    grid32, m32 = _main(name, 16, d["state"], 32)
    m64.computeRHS(m64, grid, None, None)
    m32.computeRHS(m32, grid32, None, None)
    assert rel(np_(m32.Q), np_(m64.Q)) < TOL32


def test_tgv_config1_matches_oracle_over_200_steps():
    """Config 1: TGV DNS at 32^3, nu=1/1600, dt=0.01, 200 RK4 steps, FP64:
    energy history and final field against the oracle."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    from pyspectral_b200.initial_conditions import tgv_state
    N, nu, dt, nsteps = 32, 1.0 / 1600, 0.01, 200
    st = np_(tgv_state(N))
    ost = orc.tgv_state(N)
    assert rel(st, ost) < 1e-13
    grid = C.gridclass.periodic(N)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu)
    util = C.utilitiesClass()
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=nu)
    Q = ost
    E_gpu, E_cpu = [], []
    for n in range(nsteps):
        advanceQ_RK4(main, grid, None, util)
        E_gpu.append(util.computeEnergy(main, grid))
        Q, read = orc.advance_rk4(Q, lambda q: orc.rhs_nosgs(g, q, p), dt)
        E_cpu.append(orc.energy(g, read))
    assert rel(np.array(E_gpu), np.array(E_cpu)) < 1e-12
    assert rel(np_(main.Q), Q) < 1e-10
    del torch


def test_tgv64_known_answer_history():
    """The reference's TGV validation case (64^3, nu=1/100, dt=0.010005,
    t in [0, 20]) against its shipped energy history
    (run/TGV_Validate100/benchmark_sol_64.npz).  That history was made with
    settings that are not recorded (it differs from the reference code run
    on the same inputs by ~2.5e-4 already at t=0.1), so the bound over the
    2000 steps is 5e-3 relative; the decay rate must match to 2%."""
    _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    from pyspectral_b200.initial_conditions import tgv_state
    b = golden("tgv64_benchmark.npz")
    t, E = b["t"], b["Energy"]
    N = 64
    dt = t[2] - t[1]
    st = np_(tgv_state(N))
    grid = C.gridclass.periodic(N)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, 0.01)
    util = C.utilitiesClass()
    Es = [util.computeEnergy(main, grid)]
    for n in range(1, len(t)):
        advanceQ_RK4(main, grid, None, util)
        Es.append(util.computeEnergy(main, grid))
    Es = np.array(Es)
    dev = np.abs(Es[1:] - E[1:]) / E[1:]
    print("max rel deviation of E(t) from the shipped history:", dev.max())
    assert dev.max() < 5e-3
    dE = np.diff(Es[1:]) / dt
    dEm = np.diff(E[1:]) / dt
    assert np.abs(dE - dEm).max() < 0.02 * np.abs(dEm).max()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("name", ["smag", "dsmag", "cm1", "fm1", "budgets"])
def test_cuda_graph_replay_equals_eager_steps(precision, name):
    """A captured 3-step graph replayed twice gives bit-identical state to
    6 eager steps (closures whose RHS runs reductions, stored passes or
    memory state included)."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import StepGraph, advance
    d = golden("serial_N16.npz")
    grid, a = _main(name, 16, d["state"], precision)
    grid2, b = _main(name, 16, d["state"], precision)
    g = StepGraph(a, grid, 3)
    g.replay()
    g.replay()
    advance(b, grid2, 6)
    torch.cuda.synchronize()
    assert torch.equal(a.Q, b.Q)
    assert torch.equal(a.U, b.U)
    del C


@pytest.mark.parametrize("tm,fn", [(1, "rhs_smag"), (2, "rhs_tmodel")])
def test_1000_step_histories_and_spectrum_match_oracle(tm, fn):
    """1000 RK4 steps of decaying isotropic turbulence (E(k) ~ k^4 exp(-2k^2/k0^2),
    k0 = 4, seed 1, nu = 1e-3, dt = 2e-3) at 16^3 in FP64: the energy and
    dissipation histories (every step) and the final E(k) against the oracle
    run of the same case.  Smagorinsky, and the t-model with t advancing."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    N, nu, dt, nsteps = 16, 1e-3, 2e-3, 1000
    st = orc.isotropic_state(N, 1, k0=4.0)
    grid = C.gridclass.periodic(N)
    main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu)
    util = C.utilitiesClass()
    g = orc.Grid.periodic(N)
    rhs = getattr(orc, fn)
    Q = st
    E_gpu, D_gpu, E_cpu, D_cpu = [], [], [], []
    t = 0.0
    for n in range(nsteps):
        main.t = t
        advanceQ_RK4(main, grid, None, util)
        ens, en, diss = util.computeAllStats(main, grid)[:3]
        E_gpu.append(en)
        D_gpu.append(diss)
        p = orc.Params(nu=nu, t=t)
        if fn == "rhs_smag":  # (rhs, w0); Smagorinsky reads the state as it is
            step = lambda q: (rhs(g, q, p)[0], q)
        else:  # (rhs, w0, uhat_read)
            step = lambda q: (lambda o: (o[0], o[2]))(rhs(g, q, p))
        Q, read = orc.advance_rk4(Q, step, dt)
        E_cpu.append(orc.energy(g, read))
        D_cpu.append(2 * nu * orc.enstrophy(g, read))
        t += dt
    assert rel(np.array(E_gpu), np.array(E_cpu)) < 1e-10
    assert rel(np.array(D_gpu), np.array(D_cpu)) < 1e-10
    assert E_gpu[-1] < E_gpu[0]  # decaying
    Ek_gpu = np.abs(util.computeSpectrum(main, grid)[1])
    Ek_cpu = np.abs(orc.spectrum(g, read)[1])
    assert rel(Ek_gpu, Ek_cpu) < 1e-9
    del torch
