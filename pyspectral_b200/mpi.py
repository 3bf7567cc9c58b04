"""MHD path of the MPI solver, single GPU, with the reference's names.

Mirrors PySpectral/src_MPI: ``gridclass`` (Classes.py:177-236), ``FFTclass``
(Classes.py:238-265), ``variables`` for ``turb_model='MHD'``
(Classes.py:5-149), ``computeRHS_MHD`` (RHSfunctions.py:95-175),
``advanceQ_RK4`` (time_schemes.py:2-7) and the MHD diagnostics
(Classes.py:269-448).  The right-hand sides run as single-GPU pencil passes
(one run per GPU).  ``FFTclass`` also runs the reference's slab-decomposed
transforms across ranks (``num_processes`` > 1 with a ``torch.distributed``
process group as ``comm``): each rank holds an x slab of the spectra and a y
slab of the physical field, and the Alltoall between the halves is
``all_to_all_single`` (NCCL over NVLink on GPUs).  Spectra are unnormalised
``rfftn`` results, as in the MPI solver.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _capi

TWO_PI = 2.0 * np.pi


def _cdtype(p):
    return torch.complex128 if p == 64 else torch.complex64


def _rdtype(p):
    return torch.float64 if p == 64 else torch.float32


def _on(a, dev, dtype):
    """Host array or tensor -> tensor of `dtype` on `dev`."""
    if isinstance(a, torch.Tensor):
        return a.to(device=dev, dtype=dtype)
    return torch.as_tensor(np.asarray(a), device=dev).to(dtype)


class gridclass:
    def __init__(self, N1, N2, N3, x, y, z, kc, num_processes=1, L1=TWO_PI, L2=TWO_PI, L3=TWO_PI, mpi_rank=0,
                 comm=None, turb_model="MHD", device=0):
        if num_processes != 1:
            raise ValueError("the GPU build runs one rank per run; num_processes must be 1")
        self.N1, self.N2, self.N3 = int(N1), int(N2), int(N3)
        self.Npx, self.Npy = self.N1, self.N2
        self.num_processes, self.mpi_rank, self.comm = 1, 0, comm
        self.L1, self.L2, self.L3 = float(L1), float(L2), float(L3)
        self.x, self.y, self.z = x, y, z
        self.dx = float(x[1, 0, 0] - x[0, 0, 0])
        self.dy = float(y[0, 1, 0] - y[0, 0, 0])
        self.dz = float(z[0, 0, 1] - z[0, 0, 0])
        self.kc = int(kc)
        self.Delta = np.pi / self.kc
        self.device = device
        self._ctx = {}

    @classmethod
    def periodic(cls, N, kc=None, device=0):
        a = np.arange(N) * (TWO_PI / N)
        y, x, z = np.meshgrid(a, a, a)
        return cls(N, N, N, x, y, z, N // 2 if kc is None else kc, device=device)

    def ctx(self, precision=64):
        c = self._ctx.get(precision)
        if c is None:
            c = _capi.Context(self.N1, self.N2, self.N3, (self.L1, self.L2, self.L3), (self.dx, self.dy, self.dz),
                              self.kc, precision, self.device)
            self._ctx[precision] = c
        return c


class FFTclass:
    """``myfft3D`` (unnormalised rfftn) / ``myifft3D`` (normalised irfftn) and
    the in-place 2/3-rule ``dealias``.

    With ``num_processes`` = P > 1 the transforms are the reference's slab
    decomposition (src_MPI/Classes.py:238-258): ``myifft3D(uhat, u)`` takes this
    rank's x slab of the spectra, ``uhat`` (Npx, N2, N3/2+1), and returns its y
    slab of the physical field, ``u`` (N1, Npy, N3), with Npx = N1/P and
    Npy = N2/P; ``myfft3D(u, uhat)`` goes back.  ``comm`` is the
    ``torch.distributed`` process group of the P ranks (None: the default
    group) and ``mpi_rank`` this rank's index in it.  The local halves run in
    the library (``psb_slab_*``); the exchange of P equal blocks between them
    is one ``all_to_all_single`` per transform."""

    def __init__(self, N1, N2, N3, nthreads=1, fft_type=None, Npx=None, Npy=None, num_processes=1, comm=None,
                 mpi_rank=0, grid=None, precision=64):
        self.N1, self.N2, self.N3 = N1, N2, N3
        self.grid = grid
        self.precision = precision
        self._own = None
        self.P = int(num_processes)
        self.comm = comm
        self.mpi_rank = int(mpi_rank)
        if self.P > 1:
            if N1 % self.P or N2 % self.P:
                raise ValueError("N1 and N2 must be multiples of num_processes")
            self.Npx, self.Npy = N1 // self.P, N2 // self.P
            if (Npx is not None and Npx != self.Npx) or (Npy is not None and Npy != self.Npy):
                raise ValueError("Npx, Npy must be N1/num_processes, N2/num_processes")
            self._bufs = None

    def _ctx(self):
        if self.grid is not None:
            return self.grid.ctx(self.precision)
        if self._own is None:
            self._own = _capi.Context(self.N1, self.N2, self.N3, precision=self.precision,
                                      device=torch.cuda.current_device())
        return self._own

    def _exchange_buffers(self, device):
        """send and recv blocks (P, Npx, Npy, N3/2+1) complex, allocated once."""
        if self._bufs is None:
            shape = (self.P, self.Npx, self.Npy, self.N3 // 2 + 1)
            cd = _cdtype(self.precision)
            self._bufs = (torch.empty(shape, dtype=cd, device=device), torch.empty(shape, dtype=cd, device=device))
        return self._bufs

    def _alltoall(self, send, recv):
        """comm.Alltoall(send, recv): block p of send to rank p, block p of recv from rank p."""
        import torch.distributed as dist
        dist.all_to_all_single(torch.view_as_real(recv), torch.view_as_real(send), group=self.comm)

    def myfft3D(self, u, uhat):
        if self.P == 1:
            self._ctx().r2c(u.contiguous(), uhat, 1)
            return uhat
        send, recv = self._exchange_buffers(u.device)
        ctx = self._ctx()
        ctx.slab_fft_xz(self.P, u.contiguous(), send)
        self._alltoall(send, recv)
        ctx.slab_fft_y(self.P, recv, uhat)
        return uhat

    def myifft3D(self, uhat, u):
        if self.P == 1:
            self._ctx().c2r(uhat.contiguous(), u, 1)
            return u
        send, recv = self._exchange_buffers(uhat.device)
        ctx = self._ctx()
        ctx.slab_ifft_y(self.P, uhat.contiguous(), send)
        self._alltoall(send, recv)
        ctx.slab_ifft_xz(self.P, recv, u)
        return u


class variables:
    """MPI ``variables`` for ``turb_model='MHD'`` (src_MPI/Classes.py:82-149),
    0 (Navier-Stokes, :58-80) and 'Orthogonal Dynamics' (:152-174).
    ``u,v,w,B1,B2,B3`` are physical fields (``initDomain='Physical'``) or
    ``uhat..`` spectra (``'Fourier'``, re-symmetrised by a round trip); the B
    fields are ignored by the Navier-Stokes models."""

    def __init__(self, turb_model, rotate, Om1, Om2, Om3, grid, u, v, w, B1, B2, B3, uhat=None, vhat=None,
                 what=None, t=0.0, dt=0.0, nu=0.0, myFFT=None, mpi_rank=0, initDomain="Physical",
                 time_scheme="RK4", precision=64, kahan=None, Bhat=None, forcing=True, closure=None, Ct=0.1):
        if turb_model not in ("MHD", 0, "Orthogonal Dynamics"):
            raise ValueError("turb_model must be 'MHD', 0 or 'Orthogonal Dynamics'")
        if time_scheme not in ("RK4", "Semi-Implicit") or (time_scheme != "RK4" and turb_model != 0):
            raise ValueError("Error, time scheme " + str(time_scheme) + " not implemented for "
                             + str(turb_model) + " (the semi-implicit scheme is turb_model 0's)")
        if closure not in (None, "tmodel"):
            raise ValueError("closure must be None (plain MHD) or 'tmodel'")
        self.closure = closure
        self.Ct = float(Ct)
        self.turb_model, self.rotate = turb_model, int(rotate)
        self.t, self.dt, self.nu = float(t), float(dt), float(nu)
        self.lam = self.nu
        self.precision = precision
        self.time_scheme = time_scheme
        dev = torch.device("cuda", grid.device)
        ctx = grid.ctx(precision)
        N1, N2, N3 = grid.N1, grid.N2, grid.N3
        sh = (N1, N2, N3 // 2 + 1)
        nf = 6 if turb_model == "MHD" else 3
        self.Q = torch.zeros((nf,) + sh, dtype=_cdtype(precision), device=dev)
        if initDomain == "Physical":
            fields = (u, v, w, B1, B2, B3)[:nf]
            phys = torch.stack([_on(a, dev, _rdtype(precision)) for a in fields]).contiguous()
            ctx.r2c(phys, self.Q, nf)
        else:
            src = torch.stack([_on(a, dev, _cdtype(precision)) for a in (uhat, vhat, what)] +
                              ([_on(a, dev, _cdtype(precision)) for a in Bhat] if nf == 6 else []))
            phys = torch.empty((nf, N1, N2, N3), dtype=_rdtype(precision), device=dev)
            ctx.c2r(src.contiguous(), phys, nf)
            ctx.r2c(phys, self.Q, nf)
        self.U = self.Q.clone()
        self.nvars = nf
        self.Om1, self.Om2, self.Om3 = float(Om1), float(Om2), float(Om3)
        self.force = torch.zeros((3,) + sh, dtype=_cdtype(precision), device=dev) if nf == 6 else None
        if forcing and nf == 6:  # kf = 2, f0 = 0.25 (src_MPI/Classes.py:91-94)
            kf, f0 = 2, 0.25
            X = torch.as_tensor(np.asarray(grid.x), device=dev, dtype=torch.float64)
            Y = torch.as_tensor(np.asarray(grid.y), device=dev, dtype=torch.float64)
            Z = torch.as_tensor(np.asarray(grid.z), device=dev, dtype=torch.float64)
            fp = torch.zeros((3, N1, N2, N3), dtype=_rdtype(precision), device=dev)
            fp[0] = (f0 * torch.sin(kf * X) * torch.cos(kf * Y) * torch.cos(kf * Z)).to(fp.dtype)
            fp[1] = (-f0 * torch.cos(kf * X) * torch.sin(kf * Y) * torch.cos(kf * Z)).to(fp.dtype)
            ctx.r2c(fp, self.force, 3)
        use_kahan = (precision == 32) if kahan is None else bool(kahan)
        self.comp = torch.zeros_like(self.Q) if use_kahan else None
        self.computeRHS = {"MHD": computeRHS_MHD, 0: computeRHS_NOSGS,
                           "Orthogonal Dynamics": computeRHS_Ortho}[turb_model]
        self.advanceQ = advanceQ_RK4
        if time_scheme == "Semi-Implicit":
            # H of the last step (src_MPI/Classes.py:49-52 allocates it with np.empty;
            # here it starts at zero)
            self.H = torch.zeros_like(self.Q)
            self.advanceQ = advanceQ_SI

    @property
    def uhat(self):
        return self.U[0]

    @property
    def vhat(self):
        return self.U[1]

    @property
    def what(self):
        return self.U[2]

    @property
    def B1hat(self):
        return self.U[3]

    @property
    def B2hat(self):
        return self.U[4]

    @property
    def B3hat(self):
        return self.U[5]

    def U2Q(self):
        self.Q.copy_(self.U)

    def Q2U(self):
        self.U.copy_(self.Q)

    def closure_code(self):
        if self.turb_model == 0:
            return _capi.MPI_DNS
        if self.turb_model == "Orthogonal Dynamics":
            return _capi.MPI_ORTHO
        return _capi.MHD_TMODEL if self.closure == "tmodel" else _capi.MHD

    def params(self):
        return _capi.make_params(nu=self.nu, eta=self.lam, t=self.t, dt=self.dt, Ct=self.Ct,
                                 force=self.force.data_ptr() if self.force is not None else None,
                                 rotate=self.rotate, Om=(self.Om1, self.Om2, self.Om3))


def computeRHS_MHD(main, grid, myFFT=None):
    """src_MPI/RHSfunctions.py:95-175; ``main.Q`` becomes the RHS and the
    six stored fields are dealiased in place, as in the reference."""
    ctx = grid.ctx(main.precision)
    rhs = torch.empty_like(main.Q)
    ctx.rhs(main.closure_code(), main.Q, rhs, main.params(), read_out=main.U)
    main.Q = rhs


def computeRHS_NOSGS(main, grid, myFFT=None):
    """src_MPI/RHSfunctions.py:22-93 (RK4 form): 2/3-rule Navier-Stokes."""
    computeRHS_MHD(main, grid, myFFT)


def computeRHS_Ortho(main, grid, myFFT=None):
    """src_MPI/RHSfunctions.py:179-268 (RK4 form): the Navier-Stokes RHS of u
    minus that of ``grid.filter(u)``."""
    computeRHS_MHD(main, grid, myFFT)


def advanceQ_RK4(main, grid, myFFT=None):
    """src_MPI/time_schemes.py:2-7."""
    grid.ctx(main.precision).step(main.closure_code(), main.Q, main.params(), 1, comp=main.comp, read_out=main.U)


def advanceQ_SI(main, grid, myFFT=None):
    """src_MPI/time_schemes.py:9-11 with the 'Semi-Implicit' branch of
    computeRHS_NOSGS (src_MPI/RHSfunctions.py:70-93), one fused pass."""
    grid.ctx(main.precision).step_si(main.Q, main.H, main.params(), 1, read_out=main.U)


def advance(main, grid, nsteps):
    grid.ctx(main.precision).step(main.closure_code(), main.Q, main.params(), int(nsteps), comp=main.comp,
                                  read_out=main.U)


class utilitiesClass:
    """MPI diagnostics (src_MPI/Classes.py:269-448), normalised by (N1 N2 N3)^2."""

    def computeEnergy(self, main, grid):
        return grid.ctx(main.precision).energy(main.U[0:3].contiguous(), _capi.NORM_MPI)

    def computeMHDEnergy(self, main, grid):
        return grid.ctx(main.precision).energy(main.U[3:6].contiguous(), _capi.NORM_MPI)

    def computeEnstrophy(self, main, grid):
        return grid.ctx(main.precision).enstrophy(main.U[0:3].contiguous(), _capi.NORM_MPI)

    def computeCrossHelicity(self, main, grid):
        return grid.ctx(main.precision).cross_helicity(main.U[0:3].contiguous(), main.U[3:6].contiguous(),
                                                      _capi.NORM_MPI)

    def computeSpectrum(self, main, grid):
        s = grid.ctx(main.precision).spectrum_mpi(main.U[0:3].contiguous())
        return np.linspace(0, s.shape[0] - 1, s.shape[0]), s

    def computeMHDSpectrum(self, main, grid):
        s = grid.ctx(main.precision).spectrum_mpi(main.U[3:6].contiguous())
        return np.linspace(0, s.shape[0] - 1, s.shape[0]), s
