"""Serial-solver objects with the reference's names and signatures.

``gridclass``, ``FFTclass``, ``variables`` and ``utilitiesClass`` mirror
PySpectral/src/Classes.py (:7-545, :548-588, :590-625, :631-1385) for the RHS /
RK4 path.  State lives in CUDA tensors; every computation runs in
libpyspectral_b200 through the C ABI (``_capi``).

One layout difference: the reference packs uhat, vhat, what into the diagonal
of a stride-3 array ``Q[i::3, i::3, i::3]`` (src/Classes.py:30-34).  Here
``main.Q`` is the dense ``(nvars, N1, N2, N3//2+1)`` tensor holding the same
spectra (3, or 3 plus the memory variables of the memory models);
:func:`to_stride3` / :func:`from_stride3` convert for interop.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _capi

TWO_PI = 2.0 * np.pi


def _cdtype(precision):
    return torch.complex128 if precision == 64 else torch.complex64


def _to_dev(a, dtype, device):
    if isinstance(a, torch.Tensor):
        return a.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(a), device=device).to(dtype).contiguous()


def to_stride3(Q):
    """Dense (nvars,N1,N2,N3h) -> the reference's stride-nvars ``Q`` (NumPy):
    field f at ``Q[f::nvars, f::nvars, f::nvars]`` (nvars = 3, or 3 plus the
    memory variables of the memory models)."""
    Q = Q.detach().cpu().numpy() if isinstance(Q, torch.Tensor) else np.asarray(Q)
    nv, N1, N2, N3h = Q.shape
    out = np.zeros((nv * N1, nv * N2, nv * N3h), dtype=Q.dtype)
    for i in range(nv):
        out[i::nv, i::nv, i::nv] = Q[i]
    return out


def from_stride3(Q3, nvars=3):
    """The reference's stride-nvars ``Q`` -> dense (nvars,N1,N2,N3h)."""
    return np.stack([Q3[i::nvars, i::nvars, i::nvars] for i in range(nvars)])


class gridclass:
    """``gridclass(N1,N2,N3,x,y,z,kc,L1,L2,L3)`` (src/Classes.py:548-588).

    ``x, y, z`` are the caller's coordinate arrays; only their spacings are
    used (``dx = x[1,0,0]-x[0,0,0]``, ``Delta = (dx dy dz)^(1/3)``).  The
    wavenumber arrays of the reference are available as lazily built FP64
    tensors (``k1``, ``k2``, ``k3``, ``ksqr``, ``Gf`` ...)."""

    def __init__(self, N1, N2, N3, x, y, z, kc, L1=TWO_PI, L2=TWO_PI, L3=TWO_PI, device=0):
        self.N1, self.N2, self.N3 = int(N1), int(N2), int(N3)
        self.L1, self.L2, self.L3 = float(L1), float(L2), float(L3)
        self.dx = float(x[1, 0, 0] - x[0, 0, 0])
        self.dy = float(y[0, 1, 0] - y[0, 0, 0])
        self.dz = float(z[0, 0, 1] - z[0, 0, 0])
        self.x, self.y, self.z = x, y, z
        self.kc = int(kc)
        self.Delta = (self.dx * self.dy * self.dz) ** (1.0 / 3.0)
        self.device = device
        self._ctx = {}
        self._tabs = None

    @classmethod
    def periodic(cls, N, kc=None, L=TWO_PI, device=0):
        a = np.arange(N) * (L / N)
        y, x, z = np.meshgrid(a, a, a)
        return cls(N, N, N, x, y, z, N // 2 if kc is None else kc, L, L, L, device=device)

    def ctx(self, precision=64) -> _capi.Context:
        c = self._ctx.get(precision)
        if c is None:
            c = _capi.Context(self.N1, self.N2, self.N3, (self.L1, self.L2, self.L3), (self.dx, self.dy, self.dz),
                              self.kc, precision, self.device)
            self._ctx[precision] = c
        return c

    def numpy_k(self):
        """The reference's (N1, N2, N3/2+1) wavenumber arrays k1, k2, k3 as NumPy
        (src/Classes.py:565-570: fftshifted index ranges times 2 pi / L)."""
        N1, N2, N3 = self.N1, self.N2, self.N3
        k1 = np.fft.fftshift(np.linspace(-(N1 // 2), N1 // 2 - 1, N1)) * 2.0 * np.pi / self.L1
        k2 = np.fft.fftshift(np.linspace(-(N2 // 2), N2 // 2 - 1, N2)) * 2.0 * np.pi / self.L2
        k3 = np.linspace(0, N3 // 2, N3 // 2 + 1) * 2.0 * np.pi / self.L3
        K2, K1, K3 = np.meshgrid(k2, k1, k3)
        return K1, K2, K3

    def _tables(self):
        if self._tabs is None:
            N1, N2 = self.N1, self.N2
            dev = torch.device("cuda", self.device)
            K1, K2, K3 = self.numpy_k()
            self._tabs = {n: torch.as_tensor(a, device=dev) for n, a in
                          (("k1", K1), ("k2", K2), ("k3", K3))}
            ks = K1 * K1 + K2 * K2 + K3 * K3 + 1.0e-50
            self._tabs["ksqr"] = torch.as_tensor(ks, device=dev)
            self._tabs["ksqr_i"] = torch.as_tensor(1.0 / ks, device=dev)
            kc = self.kc
            Gf = np.zeros(K1.shape)
            Gf[0:kc, 0:kc, 0:kc] = 1
            Gf[0:kc, N2 - kc + 1:, 0:kc] = 1
            Gf[N1 - kc + 1:, 0:kc, 0:kc] = 1
            Gf[N1 - kc + 1:, N2 - kc + 1:, 0:kc] = 1
            self._tabs["Gf"] = torch.as_tensor(Gf, device=dev)
        return self._tabs

    def __getattr__(self, name):
        if name in ("k1", "k2", "k3", "ksqr", "ksqr_i", "Gf"):
            return self._tables()[name]
        raise AttributeError(name)


class FFTclass:
    """``FFTclass(N1,N2,N3,nthreads)`` (src/Classes.py:590-625).

    The padded plans live in the grid's context; ``nthreads`` is accepted and
    ignored.  ``scale`` is the reference's 3/2-padding scale."""

    def __init__(self, N1, N2, N3, nthreads=1):
        self.N1, self.N2, self.N3 = N1, N2, N3
        self.nthreads = nthreads
        self.scale = math.sqrt((3.0 / 2.0) ** 3 * math.sqrt(N1 * N2 * N3))


class variables:
    """``variables(weave,turb_model,rotate,Om1,Om2,Om3,grid,uhat,vhat,what,t,dt,nu,
    Ct,dt0,dt0_subintegrations,dt1,dt1_subintegrations,cfl,dim)``
    (src/Classes.py:7-229).

    turb_model: 0 (DNS), 1 (Smagorinsky), 2 (t-model), 'Static tau-model',
    'Dynamic tau-model', 'Orthogonal Dynamics', 3 (first-order finite memory model, state
    ``Q = (u, v, w)`` then ``(w0_u, w0_v, w0_w)`` per subintegration; dt0 and
    dt0_subintegrations as in the reference), 4 (second-order finite memory
    model, state ``Q = (u, v, w)`` then per subintegration ``w0`` and ``w1``;
    dt0, dt1 and equal dt0/dt1_subintegrations), 5 (its two-term form, state
    ``(u, w0, w01)``), 6 (first-order complete memory model, state
    ``Q = (u, v, w, w0_u, w0_v, w0_w)``), 7 (dynamic Smagorinsky), 99 (DNS
    with SGS budgets: ``utilitiesClass``'s hooks write ``budget<it>.npz``
    every 20 iterations).  ``precision`` (64 or 32) selects FP64 or FP32
    fields; FP32 runs carry a Kahan compensation array ``comp``."""

    def __init__(self, weave, turb_model, rotate, Om1, Om2, Om3, grid, uhat, vhat, what, t, dt, nu, Ct=-10,
                 dt0=-10, dt0_subintegrations=-10, dt1=-10, dt1_subintegrations=-10, cfl=None, dim=3,
                 precision=64, kahan=None, model=None, les_delta=None):
        from . import RHSfunctions as R
        self.turb_model = turb_model
        self.rotate = int(rotate)
        self.Om1, self.Om2, self.Om3 = float(Om1), float(Om2), float(Om3)
        self.t = float(t)
        self.dt = float(dt)
        self.nu = float(nu)
        self.cfl = -float(dt) if cfl is None else float(cfl)
        self.precision = precision
        self.grid = grid
        self.kc = float(np.amax(np.fft.fftshift(np.linspace(-(grid.N1 // 2), grid.N1 // 2 - 1, grid.N1))
                                * 2.0 * np.pi / grid.L1))
        dev = torch.device("cuda", grid.device)
        cd = _cdtype(precision)
        self.Q = torch.stack([_to_dev(a, cd, dev) for a in (uhat, vhat, what)]).contiguous()
        self.U = self.Q.clone()
        self.nvars = 3
        if turb_model == 6:
            # complete memory model: the memory variables w0_u, w0_v, w0_w are
            # state (src/Classes.py:460-475), initially zero
            self.Q = torch.cat([self.Q, torch.zeros_like(self.Q)]).contiguous()
            self.nvars = 6
        self.fm_dt0, self.fm_nsub = 0.0, 0
        if turb_model == 3:
            # finite memory model: dt0 (default 0.1) split into dt0_subintegrations
            # memory variables (src/Classes.py:233-268), initially zero
            self.fm_dt0 = 0.1 if dt0 == -10 else float(dt0)
            self.fm_nsub = 1 if dt0_subintegrations == -10 else int(dt0_subintegrations)
            self.Q = torch.cat([self.Q] + [torch.zeros_like(self.Q)] * self.fm_nsub).contiguous()
            self.nvars = 3 + 3 * self.fm_nsub
        self.fm_dt1 = 0.0
        if turb_model == 4:
            # second-order finite memory model (src/Classes.py:294-401): dt0 (default
            # 0.1), dt1 (default 0.05); per subintegration the pair w0, w1
            # interleaved after u, initially zero.  The reference's layout needs
            # equal dt0 and dt1 subintegration counts (unequal ones overlap).
            self.fm_dt0 = 0.1 if dt0 == -10 else float(dt0)
            self.fm_dt1 = 0.05 if dt1 == -10 else float(dt1)
            n0 = 1 if dt0_subintegrations == -10 else int(dt0_subintegrations)
            n1 = 1 if dt1_subintegrations == -10 else int(dt1_subintegrations)
            if n0 != n1:
                raise ValueError("turb_model 4: dt0_subintegrations and dt1_subintegrations must be equal")
            self.fm_nsub = n0
            self.Q = torch.cat([self.Q] + [torch.zeros_like(self.Q)] * (2 * self.fm_nsub)).contiguous()
            self.nvars = 3 + 6 * self.fm_nsub
        if turb_model == 5:
            # two-term finite memory model (src/Classes.py:408-454): state (u, w0, w01);
            # it is the finite memory model with two subintegrations of 2 dt0
            self.dt0 = 0.1 if dt0 == -10 else float(dt0)
            self.fm_dt0, self.fm_nsub = 2.0 * self.dt0, 2
            self.Q = torch.cat([self.Q] + [torch.zeros_like(self.Q)] * 2).contiguous()
            self.nvars = 9
        self.Ct = 0.1 if Ct == -10 else float(Ct)
        self.tau_a, self.tau_b = float(dt0), float(dt1)
        self.tau = 0.0
        self.Cs_sqr = 0.0  # dynamic Smagorinsky coefficient of the last RHS (turb_model 7)
        self.kf = None
        use_kahan = (precision == 32) if kahan is None else bool(kahan)
        self.comp = torch.zeros_like(self.Q) if use_kahan else None
        self.W0 = None
        table = {0: R.computeRHS_NOSGS, 1: R.computeRHS_SMAG, 2: R.computeRHS_tmodel, 3: R.computeRHS_FM1,
                 4: R.computeRHS_FM2,
                 "Orthogonal Dynamics": R.computeRHS_Orthogonal,
                 5: R.computeRHS_FM1_2term,
                 "Static tau-model": R.computeRHS_staumodel, "Dynamic tau-model": R.computeRHS_Dtaumodel,
                 6: R.computeRHS_CM1, 7: R.computeRHS_DSMAG, 99: R.computeRHS_BUDGETS,
                 "learned": R.computeRHS_learned}
        if turb_model not in table:
            raise ValueError(f"turb_model {turb_model!r} is not on this path")
        self.computeRHS = table[turb_model]
        # learned closure (no reference counterpart): an MLPModel from pyspectral_b200.learned
        self.model = model
        self.les_delta = float(les_delta) if les_delta else 2.0 * np.pi / grid.N1
        if turb_model == "learned" and model is None:
            from .learned import MLPModel
            self.model = MLPModel.load(device=grid.device)
        if turb_model not in (0, "learned", "Orthogonal Dynamics"):
            self.W0 = torch.zeros_like(self.Q[3:] if turb_model in (3, 4, 5) else self.U)
        if turb_model == "Dynamic tau-model":
            self.kf = int(grid.kc * 2.0 / 3.0)
        if turb_model == "Static tau-model":
            self.kf = int(grid.kc / 2.0)
        if turb_model == 99:
            self.kf = int(self.kc)  # the budget split main.kc = amax(k1) (src/Classes.py:16)
        self.iteration = 0

    # views of the reference's per-component names
    @property
    def uhat(self):
        return self.U[0]

    @property
    def vhat(self):
        return self.U[1]

    @property
    def what(self):
        return self.U[2]

    def _w0(self, c):
        if self.W0 is None:
            return None
        if self.turb_model == 5:  # w0_u, w0_v, w0_w (N1, N2, N3/2+1); w01_* are fields 3..5
            return self.W0[c]
        if self.turb_model == 3:  # FM1: one memory variable per subintegration, (N1, N2, N3/2+1, nsub)
            return self.W0[c::3].permute(1, 2, 3, 0)
        if self.turb_model == 4:  # FM2: w0 of subintegration i is field 6i + c of W0
            return self.W0[c::6].permute(1, 2, 3, 0)
        return self.W0[c].unsqueeze(-1)

    def _w1(self, c):
        if self.turb_model != 4:
            return None
        return self.W0[3 + c::6].permute(1, 2, 3, 0)  # FM2: w1 of subintegration i is field 6i + 3 + c

    @property
    def w1_u(self):
        return self._w1(0)

    @property
    def w1_v(self):
        return self._w1(1)

    @property
    def w1_w(self):
        return self._w1(2)

    @property
    def w0_u(self):
        return self._w0(0)

    @property
    def w0_v(self):
        return self._w0(1)

    @property
    def w0_w(self):
        return self._w0(2)

    # second memory variable of the two-term finite memory model (turb_model 5)
    @property
    def w01_u(self):
        return self.W0[3] if self.turb_model == 5 else None

    @property
    def w01_v(self):
        return self.W0[4] if self.turb_model == 5 else None

    @property
    def w01_w(self):
        return self.W0[5] if self.turb_model == 5 else None

    def U2Q(self):
        self.Q[:3].copy_(self.U)
        if self.turb_model in (3, 4, 5, 6):  # memory models: w0 is state (src/Classes.py:253-259,342-355,432-440,476-482)
            self.Q[3:].copy_(self.W0)

    def Q2U(self):
        self.U.copy_(self.Q[:3])
        if self.turb_model in (3, 4, 5):
            self.W0.copy_(self.Q[3:])
        elif self.turb_model == 6:  # w0_v read from a slice nothing writes (src/Classes.py:489)
            self.W0.copy_(self.Q[3:6])
            self.W0[1].zero_()

    def params(self):
        m = self.model
        return _capi.make_params(nu=self.nu, t=self.t, dt=self.dt, Ct=self.Ct, tau_a=self.tau_a,
                                 tau_b=self.tau_b, kf=self.kf or 0, rotate=self.rotate,
                                 Om=(self.Om1, self.Om2, self.Om3),
                                 mlp_params=m.params.data_ptr() if m is not None else None,
                                 mlp_norm=m.norm.data_ptr() if m is not None else None,
                                 les_delta=self.les_delta, mlp_act=m.act if m is not None else 0,
                                 mlp_hidden=m.hidden if m is not None else 0, fm_dt0=self.fm_dt0,
                                 fm_nsub=self.fm_nsub, fm_dt1=self.fm_dt1)

    def closure_code(self):
        return {0: _capi.DNS, 1: _capi.SMAG, 2: _capi.TMODEL, "Static tau-model": _capi.TAU_STATIC,
                "Dynamic tau-model": _capi.TAU_DYNAMIC, 3: _capi.FM1, 4: _capi.FM2, 5: _capi.FM1, 6: _capi.CM1,
                7: _capi.DSMAG, "Orthogonal Dynamics": _capi.ORTHO,
                99: _capi.BUDGETS,
                "learned": _capi.LEARNED}[self.turb_model]


class utilitiesClass:
    """Diagnostics of src/Classes.py:631-929 (FP64 reductions on the GPU)."""

    def preAdvanceQ_hook(self, main, grid, myFFT):
        """SGS budgets (src/Classes.py:632-637): every 20 iterations of a
        turb_model 99 run keep the state and the SGS force of its filtered field."""
        if main.turb_model == 99 and main.iteration % 20 == 0:
            main.u0 = main.U.clone()
            main.w0_u0, main.w0_v0, main.w0_w0 = self.computeSGS_DNS(main, grid, myFFT)

    def postAdvanceQ_hook(self, main, grid, myFFT, directory="3DSolution"):
        """SGS budgets (src/Classes.py:638-649): ``budget<it>.npz`` with the
        rates of change of the SGS force and of the state over the step, the
        last stage's PLQL (u, v, w) and PL (u).  The step ran fused, so the last
        stage's PL and PLQL are evaluated again from the state it read
        (``main.uhat``), which gives the same values."""
        if not (main.turb_model == 99 and main.iteration % 20 == 0):
            return
        import os
        w0_u, w0_v, w0_w = self.computeSGS_DNS(main, grid, myFFT)
        rhs = torch.empty_like(main.U)
        plql = torch.empty_like(main.U)
        grid.ctx(main.precision).rhs(_capi.BUDGETS, main.U, rhs, main.params(), w0=plql)

        def h(t):
            return t.detach().cpu().numpy().astype(np.complex128)
        os.makedirs(directory, exist_ok=True)
        np.savez_compressed(os.path.join(directory, "budget" + str(main.iteration)),
                            w0_udot=h((w0_u - main.w0_u0) / main.dt), w0_vdot=h((w0_v - main.w0_v0) / main.dt),
                            w0_wdot=h((w0_w - main.w0_w0) / main.dt), u_dot=h((main.U[0] - main.u0[0]) / main.dt),
                            PLQLu=h(plql[0]), PLQLv=h(plql[1]), PLQLw=h(plql[2]), PLu=h(rhs[0]))

    def computeEnergy(self, main, grid):
        return grid.ctx(main.precision).energy(main.U, _capi.NORM_SERIAL)

    def computeEnergy_resolved(self, main, grid):
        return grid.ctx(main.precision).energy(main.U, _capi.FILTER_GF)

    def computeEnstrophy(self, main, grid):
        return grid.ctx(main.precision).enstrophy(main.U, _capi.NORM_SERIAL)

    def compute_dt(self, main, grid):
        if main.cfl > 0:
            main.dt = grid.ctx(main.precision).cfl_dt(main.U, main.cfl, main.nu)
        else:
            main.dt = -main.cfl

    def computeAllStats(self, main, grid):
        enstrophy = self.computeEnstrophy(main, grid)
        energy = self.computeEnergy(main, grid)
        dissipation = 2 * enstrophy * main.nu
        lambda_k = (main.nu ** 3 / dissipation) ** 0.25
        tau_k = (main.nu / dissipation) ** 0.5
        Re_lambda = energy * np.sqrt(20.0 / (3.0 * main.nu * dissipation))
        return enstrophy, energy, dissipation, lambda_k, tau_k, Re_lambda

    def _spectrum(self, main, grid, flags):
        spec = grid.ctx(main.precision).spectrum(main.U, flags)
        return spec.astype(np.complex128)

    def computeSpectrum(self, main, grid):
        spec = self._spectrum(main, grid, _capi.NORM_SERIAL)
        kmax = spec.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), spec

    def computeTransfer(self, main, grid, myFFT=None):
        """``computeTransfer`` (src/Classes.py:988-1040): ``(kdata, Transfer)``
        with Transfer complex like the reference's.  As there, the velocity
        views main.uhat/vhat/what lose their Nyquist modes (the reference
        rebinds them to ``unpad(pad(.))``); the state main.Q is untouched."""
        N1, N2, N3 = grid.N1, grid.N2, grid.N3
        main.U[:, N1 // 2, :, :] = 0
        main.U[:, :, N2 // 2, :] = 0
        main.U[:, :, :, N3 // 2] = 0
        tr = grid.ctx(main.precision).transfer(main.U)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeTransfer_resolved(self, main, grid, myFFT=None):
        """``computeTransfer_resolved`` (src/Classes.py:1093-1150): the transfer
        spectrum of the Gf-filtered velocity (no side effect)."""
        tr = grid.ctx(main.precision).transfer(main.U, flags=_capi.FILTER_GF)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeTransfer_SGS(self, main, grid, myFFT=None):
        """``computeTransfer_SGS`` (src/Classes.py:1206-1239): Re of
        conj(Gf u_i) w0_i per shell, w0 the closure force of the last RHS."""
        if main.W0 is None:
            raise ValueError("computeTransfer_SGS needs a closure that keeps w0 (turb_model != 0)")
        tr = grid.ctx(main.precision).transfer(main.U, w0=main.W0)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeTransfer_2D(self, main, grid, myFFT=None):
        """``computeTransfer_2D`` (src/Classes.py:1043-1092): the transfer of
        the k3 = 0 plane binned by rint(|k_h|), u and v components; the same
        Nyquist side effect on main.uhat/vhat/what as computeTransfer."""
        N1, N2, N3 = grid.N1, grid.N2, grid.N3
        main.U[:, N1 // 2, :, :] = 0
        main.U[:, :, N2 // 2, :] = 0
        main.U[:, :, :, N3 // 2] = 0
        tr = grid.ctx(main.precision).transfer(main.U, flags=_capi.TRANSFER_2D)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeTransfer_resolved_2D(self, main, grid, myFFT=None):
        """``computeTransfer_resolved_2D`` (src/Classes.py:1152-1205)."""
        tr = grid.ctx(main.precision).transfer(main.U, flags=_capi.FILTER_GF | _capi.TRANSFER_2D)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeTransfer_SGS_2D(self, main, grid, myFFT=None):
        """``computeTransfer_SGS_2D`` (src/Classes.py:1241-1270)."""
        if main.W0 is None:
            raise ValueError("computeTransfer_SGS_2D needs a closure that keeps w0 (turb_model != 0)")
        tr = grid.ctx(main.precision).transfer(main.U, w0=main.W0, flags=_capi.TRANSFER_2D)
        kmax = tr.shape[0] - 1
        return np.linspace(0, kmax, kmax + 1), tr

    def computeSpectrum_resolved(self, main, grid):
        spec = self._spectrum(main, grid, _capi.FILTER_GF)
        N1, N2, N3 = grid.N1, grid.N2, grid.N3
        i1 = np.fft.fftfreq(N1, 1.0 / N1)
        i2 = np.fft.fftfreq(N2, 1.0 / N2)
        i3 = np.arange(1, N3 // 2)
        ks = i1[:, None, None] ** 2 + i2[None, :, None] ** 2 + i3[None, None, :] ** 2
        k_m = np.unique(np.rint(np.sqrt(ks.ravel())))
        return k_m, spec

    def computeSGS_DNS(self, main, grid, myFFT):
        w0 = torch.zeros_like(main.U)
        grid.ctx(main.precision).sgs_dns(main.U, w0)
        return w0[0].unsqueeze(-1), w0[1].unsqueeze(-1), w0[2].unsqueeze(-1)
