"""Right-hand-side routines with the reference's names and signatures.

``computeRHS_X(main, grid, myFFT, utilities)`` evaluates the RHS of the
closure on the GPU and keeps the reference's side effects
(PySpectral/src/RHSfunctions.py): ``main.Q`` becomes the RHS, ``main.uhat``
(``main.U``) holds the state as the RHS read it (Nyquist-zeroed except in
Smagorinsky, :10-12), ``main.w0_*`` holds the closure force and the
tau-models set ``main.tau``.
"""
from __future__ import annotations

import torch

from . import _capi


def _rhs(main, grid, closure):
    ctx = grid.ctx(main.precision)
    rhs = torch.empty_like(main.Q)
    tau = ctx.rhs(closure, main.Q, rhs, main.params(), w0=main.W0, read_out=main.U)
    main.Q = rhs
    return tau


def computeRHS_NOSGS(main, grid, myFFT=None, utilities=None):
    """DNS, src/RHSfunctions.py:3-50."""
    _rhs(main, grid, _capi.DNS)


def computeRHS_SMAG(main, grid, myFFT=None, utilities=None):
    """Smagorinsky (Cs = 0.16), src/RHSfunctions.py:146-237."""
    _rhs(main, grid, _capi.SMAG)


def computeRHS_tmodel(main, grid, myFFT=None, utilities=None):
    """t-model ``w0 = Ct t PLQLu``, src/RHSfunctions.py:240-363."""
    _rhs(main, grid, _capi.TMODEL)


def computeRHS_staumodel(main, grid, myFFT=None, utilities=None):
    """Static tau-model ``tau = max(0, tau_a + tau_b t)``, src/RHSfunctions.py:366-497."""
    main.tau = _rhs(main, grid, _capi.TAU_STATIC)


def computeRHS_Dtaumodel(main, grid, myFFT=None, utilities=None):
    """Dynamic tau-model, src/RHSfunctions.py:592-878 (``main.tau`` before the clamp)."""
    main.tau = _rhs(main, grid, _capi.TAU_DYNAMIC)


def computeRHS_FM1(main, grid, myFFT=None, utilities=None):
    """First-order finite memory model (turb_model 3), src/RHSfunctions.py:882-1024:
    ``main.Q`` holds u and the memory variables of each subintegration and
    becomes their right-hand sides; ``main.w0_*`` view the memory variables
    ``(N1, N2, N3/2+1, dt0_subintegrations)``."""
    _rhs(main, grid, _capi.FM1)


def computeRHS_FM2(main, grid, myFFT=None, utilities=None):
    """Second-order finite memory model (turb_model 4), src/RHSfunctions.py:1025-1286:
    ``main.Q`` holds u and, per subintegration, the memory variables w0 and w1
    (interleaved, src/Classes.py:330-355) and becomes their right-hand sides;
    ``main.w0_*`` and ``main.w1_*`` view the memory variables as read,
    ``(N1, N2, N3/2+1, subintegrations)``.  No rotating form (the reference's
    raises)."""
    if main.rotate:
        raise RuntimeError("computeRHS_FM2: the reference has no rotating form")
    _rhs(main, grid, _capi.FM2)


def computeRHS_Orthogonal(main, grid, myFFT=None, utilities=None):
    """Orthogonal dynamics ('Orthogonal Dynamics'), src/RHSfunctions.py:53-143:
    the DNS right-hand side of u minus that of ``Gf u``."""
    _rhs(main, grid, _capi.ORTHO)


def computeRHS_FM1_2term(main, grid, myFFT=None, utilities=None):
    """Two-term finite memory model (turb_model 5), src/RHSfunctions.py:1288-1410,
    on ``(u, w0, w01)``: the finite memory model with two subintegrations of
    2 dt0 (the same right-hand sides).  No rotating form (the reference's raises)."""
    if main.rotate:
        raise RuntimeError("computeRHS_FM1_2term: the reference has no rotating form")
    _rhs(main, grid, _capi.FM1)


def computeRHS_CM1(main, grid, myFFT=None, utilities=None):
    """First-order complete memory model (turb_model 6),
    src/RHSfunctions.py:1411-1542: ``main.Q`` holds (u, v, w, w0_u, w0_v,
    w0_w) and becomes their six right-hand sides; ``main.w0_*`` the memory
    variables as read (w0_v zero, as the reference's Q2U reads it,
    src/Classes.py:489).  No rotating form (the reference's raises)."""
    _rhs(main, grid, _capi.CM1)


def computeRHS_BUDGETS(main, grid, myFFT=None, utilities=None):
    """DNS with SGS budgets (turb_model 99), src/RHSfunctions.py:1543-1661:
    ``main.Q`` becomes ``unpad_2x(PL u)``, kept as ``main.PLu/v/w``;
    ``main.PLQLu/v/w`` the memory term with the q part split at ``main.kc``."""
    _rhs(main, grid, _capi.BUDGETS)
    main.PLu, main.PLv, main.PLw = main.Q.clone().unbind(0)
    main.PLQLu, main.PLQLv, main.PLQLw = main.W0.unbind(0)


def computeRHS_DSMAG(main, grid, myFFT=None, utilities=None):
    """Dynamic Smagorinsky (turb_model 7), src/RHSfunctions.py:1663-1862:
    ``Cs^2 = <L:M>/<M:M>`` with the test filter ``myFilter(., kc/2)``, then the
    Smagorinsky stress with that coefficient.  The coefficient, a local of the
    reference, is kept as ``main.Cs_sqr``."""
    main.Cs_sqr = _rhs(main, grid, _capi.DSMAG)


def computeRHS_learned(main, grid, myFFT=None, utilities=None):
    """LES with the learned MLP subgrid stress (no reference counterpart;
    takes the place of the Smagorinsky stress of src/RHSfunctions.py:195-212).
    The stress enters with the solenoidal projection -i k_j (u_i u_j + tau_ij)
    projected, like the advection term."""
    _rhs(main, grid, _capi.LEARNED)


def advanceQ_RK4(main, grid, myFFT=None, utilities=None):
    """``advanceQ_RK4`` (src/PySpec_3d.py:96-105): four low-storage stages
    ``Q = Q0 + dt c_i RHS(Q)``, c = [1/4, 1/3, 1/2, 1], fused into the RHS
    epilogues.  ``main.uhat`` ends as the state read by the last stage, which
    is what the reference's per-step diagnostics read (src/PySpec_3d.py:129)."""
    if utilities is not None:
        utilities.preAdvanceQ_hook(main, grid, myFFT)
        utilities.compute_dt(main, grid)
    ctx = grid.ctx(main.precision)
    ctx.step(main.closure_code(), main.Q, main.params(), 1, comp=main.comp, read_out=main.U)
    if utilities is not None:
        utilities.postAdvanceQ_hook(main, grid, myFFT)


def autotune(main, grid, rounds=1, confirm_steps=40, flush_bytes=256 << 20):
    """Tune the launch shapes of main's closure on its current state (no
    reference counterpart; DNS, Smagorinsky and the learned closure).

    The tuner ranks each pass's candidates by that pass's own launch time,
    which its neighbours' overlap and the timing noise blur; its pick varies
    by a few percent of the step between calls.  With ``rounds`` > 1 it runs
    ``rounds`` times from the default shapes, and the distinct shape sets it
    returns, plus the default, are then timed as whole RK4 steps
    (``confirm_steps`` steps each, one at a time on a copy of the state, L2
    flushed with a ``flush_bytes`` write before every step and left out of
    the timing; sets interleaved, median per set); the fastest set is kept.
    The state is untouched.  Returns the kept set's median ms per step (None
    for rounds = 1)."""
    ctx = grid.ctx(main.precision)
    code = main.closure_code()
    if rounds <= 1:
        ctx.autotune(code, main.Q, main.params())
        return None
    sets = []
    for _ in range(rounds):
        ctx.autotune_clear(code)
        ctx.autotune(code, main.Q, main.params())
        s = ctx.tuned_shapes(code)
        if s not in sets:
            sets.append(s)
    ctx.autotune_clear(code)
    sets.append(ctx.tuned_shapes(code))  # the default shapes (tile 0: per-pass default)
    q = main.Q.clone()
    u = main.U.clone()
    comp = main.comp.clone() if main.comp is not None else None
    p = main.params()
    flush = torch.empty(max(1, flush_bytes // 4), dtype=torch.float32, device=main.Q.device)
    times = [[] for _ in sets]
    for _ in range(confirm_steps):
        for i, s in enumerate(sets):
            ctx.autotune_clear(code)
            if any(x["tile"] for x in s):
                ctx.set_tuned_shapes(code, [x if x["tile"] else None for x in s])
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            ctx.step(code, q, p, 1, comp=comp, read_out=u)
            b.record()
            times[i].append((a, b))
            q.copy_(main.Q)  # every set steps the same state
            if comp is not None:
                comp.copy_(main.comp)
    torch.cuda.synchronize()
    med = [float(torch.tensor([a.elapsed_time(b) for a, b in t]).median()) for t in times]
    best = min(range(len(sets)), key=lambda i: med[i])
    ctx.autotune_clear(code)
    if any(x["tile"] for x in sets[best]):
        ctx.set_tuned_shapes(code, [x if x["tile"] else None for x in sets[best]])
    return med[best]


def advance(main, grid, nsteps):
    """``nsteps`` fixed-dt RK4 steps in one call (no per-step host work)."""
    ctx = grid.ctx(main.precision)
    ctx.step(main.closure_code(), main.Q, main.params(), int(nsteps), comp=main.comp, read_out=main.U)


class StepGraph:
    """``nsteps`` fixed-dt RK4 steps captured once into a CUDA graph.

    ``replay()`` advances ``main`` in place exactly like ``advance(main, grid,
    nsteps)`` but with one graph launch.  Kernel arguments (dt, nu, t, closure
    coefficients) are frozen at capture, so this suits closures without an
    explicit time dependence (DNS, Smagorinsky, MHD) or a fixed t; re-capture
    after changing them."""

    def __init__(self, main, grid, nsteps=1):
        import torch
        self.main, self.grid, self.nsteps = main, grid, int(nsteps)
        ctx = grid.ctx(main.precision)
        ctx.prepare(main.closure_code())
        saved = [t.clone() for t in self._state()]
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):  # warm-up outside the capture (sets kernel attributes)
            advance(main, grid, self.nsteps)
        torch.cuda.current_stream().wait_stream(side)
        for t, s in zip(self._state(), saved):
            t.copy_(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            advance(main, grid, self.nsteps)
        torch.cuda.synchronize()

    def _state(self):
        out = [self.main.Q, self.main.U]
        if self.main.comp is not None:
            out.append(self.main.comp)
        return out

    def replay(self):
        self.graph.replay()
