"""GPU parity at the sizes the benchmarks and the reference's configs run:
64^3 (the headline LES: learned closure in FP32 + Kahan with the shipped
network and tuned launch shapes, plain FP64 Smagorinsky, the t-model on its
2x grid), 128^3 (Smagorinsky, t-model, MHD), the padded transform lengths
(72, 96, 192, 384) on their own, and members of batched ensembles at 48^3
and 64^3 -- all against the CPU oracle, not against another GPU path.

Every transform schedule compiled into the library for the 96- and
192-point lengths is run in every pass it can serve (set by hand through
psb_set_tuned_shape), so a wrong twiddle or index in a schedule that only
these lengths take fails here.

Bars: FP64 1e-12 relative (max norm); FP32 fields 2e-5 against the FP64
oracle; the learned closure (BF16 tensor-core arithmetic) 5e-4 against the
BF16-emulating oracle, its RK4 increments 1e-3.
"""
import json
import os

import numpy as np
import pytest

from oracle import mlp_oracle as mo
from oracle import spectral_oracle as orc
from tests.helpers import ROOT, rel

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 2e-5
TOL_LEARNED = 5e-4
NU, DT = 1e-3, 2e-3

# compiled-in schedules (psb_fft.cuh PSB_FIXED_PLANS) by length
FIXED = {96: [(8, 4, 3), (16, 6), (6, 16), (12, 8), (8, 12)], 192: [(8, 8, 3), (16, 12), (12, 16)],
         48: [(8, 2, 3), (16, 3), (3, 16), (8, 6), (6, 8)], 72: [(8, 3, 3), (6, 12), (12, 6)]}


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    orc.set_workers(os.cpu_count() or 1)
    return torch


def np_(t):
    return t.detach().cpu().numpy()


def _shipped():
    d = np.load(os.path.join(ROOT, "pyspectral_b200", "models", "sgs_mlp.npz"))
    return (d["params"].astype(np.float64), d["norm"].astype(np.float64),
            json.loads(str(d["meta"])).get("act", "gelu"))


def _main(N, closure, precision, st, model=None, t=0.0):
    from pyspectral_b200 import Classes as C
    tm = {"dns": 0, "smag": 1, "tmodel": 2, "learned": "learned"}[closure]
    grid = C.gridclass.periodic(N)
    main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], t, DT, NU, precision=precision, model=model)
    return grid, main


def _rhs(torch, grid, main):
    ctx = grid.ctx(main.precision)
    out = torch.empty_like(main.Q)
    ctx.rhs(main.closure_code(), main.Q, out, main.params())
    torch.cuda.synchronize()
    return np_(out)


def _set_one(ctx, code, k, radices, tiles):
    """Pass k at the first of `tiles` the closure accepts (shared-memory budget,
    pencil bound), the other passes at their default shapes."""
    ctx.autotune_clear(code)
    for tile in tiles:
        shapes = [None] * 5
        shapes[k] = {"tile": tile, "radices": list(radices)}
        try:
            ctx.set_tuned_shapes(code, shapes)
            return tile
        except RuntimeError:
            continue
    return None


def _schedule_sweep(torch, grid, main, ref, tol, L_by_pass):
    """Every compiled schedule of each pass's length, one pass at a time (the
    others at their default shapes), and the tiles each pass accepts."""
    ctx = grid.ctx(main.precision)
    code = main.closure_code()
    ran = 0
    for k, L in enumerate(L_by_pass):
        for rad in FIXED.get(L, []):
            tile = _set_one(ctx, code, k, rad, (4, 2, 1) if k == 2 else (8, 4, 2, 1))
            assert tile is not None, (k, rad)
            got = _rhs(torch, grid, main)
            assert rel(got, ref) < tol, (k, rad, tile, rel(got, ref))
            ran += 1
        for tile in ((1, 2, 8) if k == 2 else (2, 4, 16, 32)):
            if _set_one(ctx, code, k, FIXED[L][0], (tile,)) is None:
                continue  # beyond this closure's shared-memory budget or pencil bound
            got = _rhs(torch, grid, main)
            assert rel(got, ref) < tol, (k, tile, rel(got, ref))
            ran += 1
    ctx.autotune_clear(code)
    return ran


def _learned_ref(N, st, P, nrm, act):
    g = orc.Grid.periodic(N)
    return g, (lambda q: mo.rhs_learned(g, q, NU, P, nrm, 2 * np.pi / N, act=act))


def test_les64_learned_fp32_shipped_model_tuned_and_every_schedule():
    """The headline workload: 64^3, FP32 + Kahan, the shipped width-32 ReLU
    network, shapes from psb_autotune; then every compiled 96-point schedule
    in every pass.  RHS and one RK4 step against the BF16-emulating oracle."""
    torch = _torch()
    from pyspectral_b200.RHSfunctions import advanceQ_RK4, autotune
    from pyspectral_b200.learned import MLPModel
    N = 64
    P, nrm, act = _shipped()
    model = MLPModel.load()
    assert model.act_name == act
    st = orc.isotropic_state(N, 1, k0=4.0)
    st32 = st.astype(np.complex64).astype(np.complex128)  # what the FP32 run holds
    g, rhs_fn = _learned_ref(N, st32, P, nrm, act)
    ref = rhs_fn(st32)
    grid, main = _main(N, "learned", 32, st, model=model)
    autotune(main, grid)
    assert all(s["tile"] > 0 for s in grid.ctx(32).tuned_shapes(main.closure_code()))
    got = _rhs(torch, grid, main)
    assert rel(got, ref) < TOL_LEARNED
    # one RK4 step (Kahan-compensated stages) with the tuned shapes
    advanceQ_RK4(main, grid, None, None)
    Q1, _ = orc.advance_rk4(st32, lambda q: (rhs_fn(q), None), DT)
    assert rel(np_(main.Q).astype(np.complex128) - st32, Q1 - st32) < 1e-3
    # every compiled schedule, pass by pass
    grid, main = _main(N, "learned", 32, st, model=model)
    assert _schedule_sweep(torch, grid, main, ref, TOL_LEARNED, [96] * 5) >= 25


@pytest.mark.parametrize("closure", ["smag", "dns"])
def test_les64_fp64_default_tuned_and_every_schedule(closure):
    """64^3 FP64 (the plain path the headline is compared with): default
    shapes, autotuned shapes and every 96-point schedule, RHS at 1e-12; one
    RK4 step at 1e-12."""
    torch = _torch()
    from pyspectral_b200.RHSfunctions import advanceQ_RK4, autotune
    N = 64
    st = orc.isotropic_state(N, 1, k0=4.0)
    g = orc.Grid.periodic(N)
    fn = orc.rhs_smag if closure == "smag" else orc.rhs_nosgs
    ref = fn(g, st, orc.Params(nu=NU))[0]
    grid, main = _main(N, closure, 64, st)
    assert rel(_rhs(torch, grid, main), ref) < TOL64
    advanceQ_RK4(main, grid, None, None)
    Q1, _ = orc.advance_rk4(st, lambda q: (fn(g, q, orc.Params(nu=NU))[0], None), DT)
    assert rel(np_(main.Q), Q1) < TOL64
    grid, main = _main(N, closure, 64, st)
    autotune(main, grid)
    assert rel(_rhs(torch, grid, main), ref) < TOL64
    assert _schedule_sweep(torch, grid, main, ref, TOL64, [96] * 5) >= 25


def test_autotune_rounds_keeps_state_and_parity():
    """autotune(rounds=3) -- three tuner runs, their shape sets and the default
    timed as whole flushed RK4 steps on a copy of the state -- leaves the state
    and its compensation array untouched and keeps a set under which the
    learned 64^3 FP32 RHS and one RK4 step still match the oracle."""
    torch = _torch()
    from pyspectral_b200.learned import MLPModel
    from pyspectral_b200.RHSfunctions import advanceQ_RK4, autotune
    N = 64
    P, nrm, act = _shipped()
    model = MLPModel.load()
    st = orc.isotropic_state(N, 2, k0=4.0)
    st32 = st.astype(np.complex64).astype(np.complex128)  # what the FP32 run holds
    g, rhs_fn = _learned_ref(N, st32, P, nrm, act)
    ref = rhs_fn(st32)
    grid, main = _main(N, "learned", 32, st, model=model)
    q0, c0 = main.Q.clone(), main.comp.clone()
    ms = autotune(main, grid, rounds=3, confirm_steps=8)
    assert ms is not None and ms > 0
    assert torch.equal(main.Q, q0) and torch.equal(main.comp, c0)
    assert rel(_rhs(torch, grid, main), ref) < TOL_LEARNED
    advanceQ_RK4(main, grid, None, None)
    Q1, _ = orc.advance_rk4(st32, lambda q: (rhs_fn(q), None), DT)
    assert rel(np_(main.Q).astype(np.complex128) - st32, Q1 - st32) < 1e-3


def test_les64_tmodel_fp64_rhs_and_step():
    """t-model at 64^3 (2x grid: 128-point transforms), FP64, t != 0."""
    torch = _torch()
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    N, t = 64, 0.37
    st = orc.isotropic_state(N, 2, k0=4.0)
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=t)
    ref = orc.rhs_tmodel(g, st, p)[0]
    grid, main = _main(N, "tmodel", 64, st, t=t)
    assert rel(_rhs(torch, grid, main), ref) < TOL64
    advanceQ_RK4(main, grid, None, None)
    Q1, _ = orc.advance_rk4(st, lambda q: (orc.rhs_tmodel(g, q, p)[0], None), DT)
    assert rel(np_(main.Q), Q1) < TOL64


@pytest.mark.parametrize("closure", ["smag", "tmodel"])
def test_128_fp64_rhs_matches_oracle(closure):
    """128^3, FP64: Smagorinsky (192-point transforms) and the t-model (256)."""
    torch = _torch()
    N, t = 128, 0.2
    st = orc.isotropic_state(N, 1, k0=4.0)
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=t)
    ref = (orc.rhs_smag if closure == "smag" else orc.rhs_tmodel)(g, st, p)[0]
    grid, main = _main(N, closure, 64, st, t=t)
    assert rel(_rhs(torch, grid, main), ref) < TOL64


def test_128_smag_fp32_every_schedule():
    """128^3 Smagorinsky in FP32: default shapes and every compiled 192-point
    schedule in every pass, against the FP64 oracle at the FP32 bar."""
    torch = _torch()
    N = 128
    st = orc.isotropic_state(N, 1, k0=4.0)
    st32 = st.astype(np.complex64).astype(np.complex128)
    g = orc.Grid.periodic(N)
    ref = orc.rhs_smag(g, st32, orc.Params(nu=NU))[0]
    grid, main = _main(N, "smag", 32, st)
    assert rel(_rhs(torch, grid, main), ref) < TOL32
    assert _schedule_sweep(torch, grid, main, ref, TOL32, [192] * 5) >= 15


def test_48_smag_fp32_every_schedule():
    """48^3 Smagorinsky in FP32 (the ensemble's middle size): default shapes
    and every compiled 72-point schedule in every pass, against the FP64
    oracle at the FP32 bar."""
    torch = _torch()
    N = 48
    st = orc.isotropic_state(N, 4, k0=3.0)
    st32 = st.astype(np.complex64).astype(np.complex128)
    g = orc.Grid.periodic(N)
    ref = orc.rhs_smag(g, st32, orc.Params(nu=NU))[0]
    grid, main = _main(N, "smag", 32, st)
    assert rel(_rhs(torch, grid, main), ref) < TOL32
    assert _schedule_sweep(torch, grid, main, ref, TOL32, [72] * 5) >= 15


def test_128_learned_fp32_rhs_matches_oracle():
    torch = _torch()
    from pyspectral_b200.learned import MLPModel
    N = 128
    P, nrm, act = _shipped()
    st = orc.isotropic_state(N, 3, k0=4.0)
    st32 = st.astype(np.complex64).astype(np.complex128)
    _, rhs_fn = _learned_ref(N, st32, P, nrm, act)
    grid, main = _main(N, "learned", 32, st, model=MLPModel.load())
    assert rel(_rhs(torch, grid, main), rhs_fn(st32)) < TOL_LEARNED


def test_128_mhd_fp64_rhs_matches_oracle():
    """The MHD case at 128^3 (u and B from the k0 = 3 spectrum, seeds 2 and
    3; nu = eta = 2e-3), FP64, plain MHD right-hand side (2/3 rule)."""
    torch = _torch()
    from pyspectral_b200.precision import mhd_case
    N = 128
    grid, main = mhd_case(N, "none", 64)
    state = np_(main.Q)
    rhs = torch.empty_like(main.Q)
    grid.ctx(64).rhs(main.closure_code(), main.Q, rhs, main.params(), read_out=main.U)
    ref, read = orc.rhs_mhd(orc.MHDGrid(N, N, N, N // 2), state, 2e-3)
    assert rel(np_(rhs), ref) < TOL64
    assert rel(np_(main.U), read) < TOL64


@pytest.mark.parametrize("N", [72, 96, 192, 384])
@pytest.mark.parametrize("precision", [64, 32])
def test_plain_transforms_padded_lengths(N, precision):
    """r2c / c2r of the lengths the padded transforms use (3/2 of 48, 64,
    128, 256), against NumPy."""
    torch = _torch()
    from pyspectral_b200 import _capi
    nf = 1 if N == 384 else 2
    ctx = _capi.Context(N, N, N, precision=precision)
    rng = np.random.default_rng(N)
    x = rng.standard_normal((nf, N, N, N))
    rd = torch.float64 if precision == 64 else torch.float32
    cd = torch.complex128 if precision == 64 else torch.complex64
    X = torch.as_tensor(x, device="cuda", dtype=rd).contiguous()
    S = torch.empty((nf, N, N, N // 2 + 1), device="cuda", dtype=cd)
    ctx.r2c(X, S, nf)
    ref = np.stack([np.fft.rfftn(a) for a in x])
    tol = 1e-14 if precision == 64 else 3e-6
    assert rel(np_(S), ref) < tol
    Y = torch.empty_like(X)
    ctx.c2r(S, Y, nf)
    assert rel(np_(Y), x) < tol


def _batch(torch, N, closure, precision, specs, model=None):
    from pyspectral_b200 import _capi
    from pyspectral_b200.ensemble import Batch
    code = {"smag": _capi.SMAG, "learned": _capi.LEARNED}[closure]
    cdt = torch.complex128 if precision == 64 else torch.complex64
    ctx = _capi.Context(N, N, N, precision=precision)
    b = Batch(ctx, code, len(specs))
    states = []
    for r, (seed, k0, nu) in enumerate(specs):
        st = torch.as_tensor(orc.isotropic_state(N, seed, k0=k0), device="cuda").to(cdt).contiguous()
        comp = torch.zeros_like(st) if precision == 32 else None
        p = _capi.make_params(nu=nu, dt=DT, mlp_params=model.params.data_ptr() if model else None,
                              mlp_norm=model.norm.data_ptr() if model else None, les_delta=2 * np.pi / N,
                              mlp_act=model.act if model else 0, mlp_hidden=model.hidden if model else 0)
        b.set_run(r, st, comp, p)
        states.append(st)
    b.autotune()
    b.step(1)
    torch.cuda.synchronize()
    return [np_(s) for s in states]


def test_ensemble_member_48_smag_fp64_matches_oracle():
    """Members of a 48^3 Smagorinsky batch (72-point transforms, autotuned
    batch shapes) advance one RK4 step exactly like the oracle."""
    torch = _torch()
    N = 48
    specs = [(1001, 2.0, 6e-4), (1002, 5.0, 3e-3)]
    out = _batch(torch, N, "smag", 64, specs)
    g = orc.Grid.periodic(N)
    for (seed, k0, nu), q in zip(specs, out):
        st = orc.isotropic_state(N, seed, k0=k0)
        Q1, _ = orc.advance_rk4(st, lambda s: (orc.rhs_smag(g, s, orc.Params(nu=nu))[0], None), DT)
        assert rel(q, Q1) < TOL64


def test_ensemble_member_64_learned_fp32_matches_oracle():
    """A member of a 64^3 learned batch (FP32 + Kahan, shipped network,
    autotuned batch shapes): its RK4 increment against the oracle's."""
    torch = _torch()
    from pyspectral_b200.learned import MLPModel
    N = 64
    P, nrm, act = _shipped()
    specs = [(1040, 3.0, 1e-3), (1041, 4.0, 2e-3)]
    out = _batch(torch, N, "learned", 32, specs, model=MLPModel.load())
    g = orc.Grid.periodic(N)
    seed, k0, nu = specs[0]
    st = orc.isotropic_state(N, seed, k0=k0).astype(np.complex64).astype(np.complex128)
    Q1, _ = orc.advance_rk4(st, lambda s: (mo.rhs_learned(g, s, nu, P, nrm, 2 * np.pi / N, act=act), None), DT)
    assert rel(out[0].astype(np.complex128) - st, Q1 - st) < 1e-3
