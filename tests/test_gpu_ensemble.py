"""Batched ensembles on the GPU: every run of a batch advances exactly like the
same run through the single-run path (FP64: 1e-12 relative), before and after
the autotuner changes the launch shapes, and the ensemble driver runs an
uneven-size ensemble in one CUDA graph."""
import numpy as np
import pytest

from tests.helpers import rel

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def np_(t):
    return t.detach().cpu().numpy()


def _single(torch, N, st, nu, dt, closure, precision, model=None, steps=2):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advance
    tm = {"dns": 0, "smag": 1, "learned": "learned"}[closure]
    grid = C.gridclass.periodic(N)
    main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu, precision=precision,
                       model=model)
    advance(main, grid, steps)
    return np_(main.Q)


def _batch_runs(torch, N, closure, precision, tune, model=None, steps=2, nruns=3):
    from pyspectral_b200 import _capi
    from pyspectral_b200.ensemble import Batch
    from pyspectral_b200.initial_conditions import isotropic_state
    code = {"dns": _capi.DNS, "smag": _capi.SMAG, "learned": _capi.LEARNED}[closure]
    cdt = torch.complex128 if precision == 64 else torch.complex64
    ctx = _capi.Context(N, N, N, precision=precision)
    b = Batch(ctx, code, nruns)
    init, states, nus = [], [], []
    for r in range(nruns):
        st = isotropic_state(N, 10 + r, k0=3.0 + r).to(cdt).contiguous()
        init.append(st.clone())
        nu = 1e-3 * (1 + r)
        comp = torch.zeros_like(st) if precision == 32 else None
        p = _capi.make_params(nu=nu, dt=2e-3, mlp_params=model.params.data_ptr() if model else None,
                              mlp_norm=model.norm.data_ptr() if model else None, les_delta=2 * np.pi / N,
                              mlp_act=model.act if model else 0, mlp_hidden=model.hidden if model else 0)
        b.set_run(r, st, comp, p)
        states.append(st)
        nus.append(nu)
    if tune:
        b.autotune()
        for s, s0 in zip(states, init):
            assert torch.equal(s, s0)  # tuning leaves the states alone
    b.step(steps)
    torch.cuda.synchronize()
    return b, [np_(s) for s in states], [np_(s) for s in init], nus


@pytest.mark.parametrize("closure", ["dns", "smag"])
@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_single_runs_fp64(closure, tune):
    torch = _torch()
    N = 16
    b, out, init, nus = _batch_runs(torch, N, closure, 64, tune)
    for r in range(len(out)):
        ref = _single(torch, N, init[r], nus[r], 2e-3, closure, 64)
        assert rel(out[r], ref) < 1e-12
    sh = b.shapes()
    assert sh["z-fused"]["tile"] >= 1 and np.prod(sh["x-inverse"]["radices"]) == 3 * N // 2


def test_learned_batch_tracks_single_runs_fp32():
    torch = _torch()
    from pyspectral_b200.learned import MLPModel
    model = MLPModel.load()
    N = 32
    b, out, init, nus = _batch_runs(torch, N, "learned", 32, True, model=model)
    for r in range(len(out)):
        ref = _single(torch, N, init[r].astype(np.complex128), nus[r], 2e-3, "learned", 32, model=model)
        assert rel(out[r], ref) < 2e-5


def test_uneven_ensemble_in_one_graph():
    torch = _torch()
    from pyspectral_b200.ensemble import Ensemble, ensemble_specs, time_batched
    from pyspectral_b200.learned import MLPModel
    specs = ensemble_specs(sizes=(16, 24, 32), per_size=3)
    ens = Ensemble(specs, model=MLPModel.load(), learned_N=32, tune=True)
    before = [s.clone() for g in ens.groups for s in g["states"]]
    res = time_batched(ens, 4, graph_steps=2)
    after = [s for g in ens.groups for s in g["states"]]
    assert res["value"] > 0 and res["steps"] == 4
    assert all(bool(torch.isfinite(torch.view_as_real(s)).all()) for s in after)
    assert all(not torch.equal(a, b) for a, b in zip(after, before))
    assert {g["closure"] for g in ens.groups} == {"learned", "smag"}


@pytest.mark.parametrize("closure,precision,tol", [("smag", 64, 1e-12), ("dns", 64, 1e-12), ("learned", 32, 5e-5)])
def test_autotuned_single_run_matches_default_shapes(closure, precision, tol):
    """psb_autotune picks other tiles and radix orders for a single run's
    passes; the RHS and two RK4 steps stay equal to the default shapes' up to
    rounding, and the state is not touched by tuning."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advance, autotune
    from pyspectral_b200.initial_conditions import isotropic_state
    from pyspectral_b200.learned import MLPModel
    N = 32
    model = MLPModel.load() if closure == "learned" else None
    tm = {"dns": 0, "smag": 1, "learned": "learned"}[closure]
    st = isotropic_state(N, 4, k0=3.0)
    out = []
    for tune in (False, True):
        grid = C.gridclass.periodic(N)
        main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 2e-3, 1e-3, precision=precision,
                           model=model)
        if tune:
            q0 = main.Q.clone()
            autotune(main, grid)
            assert torch.equal(main.Q, q0)
            sh = grid.ctx(precision).tuned_shapes(main.closure_code())
            assert all(s["tile"] > 0 for s in sh)
        rhs = torch.empty_like(main.Q)
        grid.ctx(precision).rhs(main.closure_code(), main.Q, rhs, main.params())
        advance(main, grid, 2)
        out.append((np_(rhs), np_(main.Q)))
    assert rel(out[1][0], out[0][0]) < tol
    assert rel(out[1][1], out[0][1]) < tol


def test_set_run_between_steps_on_a_side_stream():
    """Changing a run's parameters between two queued steps on a non-blocking
    stream: the first step runs entirely with the old arguments, the second
    with the new ones (the library drains the stream before it rewrites the
    device argument blocks)."""
    torch = _torch()
    from pyspectral_b200 import _capi
    from pyspectral_b200.ensemble import Batch
    from pyspectral_b200.initial_conditions import isotropic_state
    N, nu = 16, 2e-3
    ctx = _capi.Context(N, N, N, precision=64)
    st0 = isotropic_state(N, 21, k0=3.0).contiguous()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        b = Batch(ctx, _capi.SMAG, 1)
        st = st0.clone()
        b.set_run(0, st, None, _capi.make_params(nu=nu, dt=2e-3))
        b.step(3)
        b.set_run(0, st, None, _capi.make_params(nu=nu, dt=5e-3))
        b.step(2)
    torch.cuda.synchronize()
    ref = _single(torch, N, np_(st0), nu, 2e-3, "smag", 64, steps=3)
    ref = _single(torch, N, ref, nu, 5e-3, "smag", 64, steps=2)
    assert rel(np_(st), ref) < 1e-12


def _persistent_groups(torch, specs, precision, model=None):
    """Batches (one per grid size) of the given (N, closure, seed, nu) runs."""
    from pyspectral_b200 import _capi
    from pyspectral_b200.ensemble import Batch
    from pyspectral_b200.initial_conditions import isotropic_state
    cdt = torch.complex128 if precision == 64 else torch.complex64
    groups = []
    for N, closure, runs in specs:
        ctx = _capi.Context(N, N, N, precision=precision)
        code = {"dns": _capi.DNS, "smag": _capi.SMAG, "learned": _capi.LEARNED}[closure]
        b = Batch(ctx, code, len(runs))
        states = []
        for r, (seed, nu) in enumerate(runs):
            st = isotropic_state(N, seed, k0=3.0).to(cdt).contiguous()
            comp = torch.zeros_like(st) if precision == 32 else None
            m = model if closure == "learned" else None
            p = _capi.make_params(nu=nu, dt=2e-3, mlp_params=m.params.data_ptr() if m else None,
                                  mlp_norm=m.norm.data_ptr() if m else None, les_delta=2 * np.pi / N,
                                  mlp_act=m.act if m else 0, mlp_hidden=m.hidden if m else 0)
            b.set_run(r, st, comp, p)
            states.append((st, comp))
        groups.append((N, closure, b, states))
    return groups


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_persistent_ensemble_matches_batched_steps(precision, tol):
    """One cooperative launch for every batch (sizes 16, 24 and 32; DNS,
    Smagorinsky and the learned closure) advances each run exactly like the
    batched launches (FP64 1e-12; FP32 at the FP32 bar: the two paths may take
    different transform schedules), and no barrier wait gives up."""
    torch = _torch()
    from pyspectral_b200.ensemble import Persistent
    from pyspectral_b200.learned import MLPModel
    model = MLPModel.load()
    spec = [(16, "smag", [(31, 1e-3), (32, 3e-3)]), (24, "dns", [(33, 2e-3)]),
            (32, "learned" if precision == 32 else "smag", [(34, 1e-3), (35, 2e-3), (36, 4e-3)])]
    ga = _persistent_groups(torch, spec, precision, model)
    gb = _persistent_groups(torch, spec, precision, model)
    for _, _, b, _ in ga:
        b.step(3)
    p = Persistent([g[2] for g in gb])
    p.step(2)
    p.step(1)
    torch.cuda.synchronize()
    assert p.status() == 0
    for (_, _, _, sa), (_, _, _, sb) in zip(ga, gb):
        for (a, _), (b_, _) in zip(sa, sb):
            assert rel(np_(b_), np_(a)) < tol


def test_persistent_ensemble_barrier_gives_up_and_returns():
    """With a poll limit of one, the grid barriers give up instead of waiting:
    the launch returns (the call completes, the device stays usable), the
    status word reads 1 once and is then cleared, and a later call with the
    default limit runs normally."""
    torch = _torch()
    from pyspectral_b200.ensemble import Persistent
    spec = [(16, "smag", [(41, 1e-3), (42, 2e-3)])]
    g = _persistent_groups(torch, spec, 64)
    p = Persistent([g[0][2]])
    p.step(1, poll_limit=1)
    torch.cuda.synchronize()
    assert p.status() == 1
    assert p.status() == 0
    g2 = _persistent_groups(torch, spec, 64)
    p2 = Persistent([g2[0][2]])
    p2.step(1)
    ref = _persistent_groups(torch, spec, 64)
    ref[0][2].step(1)
    torch.cuda.synchronize()
    assert p2.status() == 0
    for (a, _), (b_, _) in zip(g2[0][3], ref[0][3]):
        assert rel(np_(a), np_(b_)) < 1e-12


def test_persistent_ensemble_in_a_graph():
    """The uneven ensemble's persistent launch captured in a CUDA graph and
    replayed advances it like the batched graph does."""
    torch = _torch()
    from pyspectral_b200.ensemble import Ensemble, ensemble_specs, time_batched, time_persistent
    from pyspectral_b200.learned import MLPModel
    specs = ensemble_specs(sizes=(16, 24, 32), per_size=2)
    model = MLPModel.load()
    e1 = Ensemble(specs, model=model, learned_N=32, tune=False)
    e2 = Ensemble(specs, model=model, learned_N=32, tune=False)
    r1 = time_batched(e1, 4, graph_steps=2)
    r2 = time_persistent(e2, 4, graph_steps=2)
    assert r2["status"] == 0 and r1["steps"] == r2["steps"] == 4
    for g1, g2 in zip(e1.groups, e2.groups):
        for a, b_ in zip(g1["states"], g2["states"]):
            assert rel(np_(b_), np_(a)) < 2e-5
