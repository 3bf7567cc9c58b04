"""Initial conditions on the GPU.

* Taylor-Green vortex, ``uhat = rfftn(u)/sqrt(N^3)``
  (PySpectral/run/TGV_Validate100/inputfile.py:38-44), on the exactly
  periodic grid ``x_i = 2 pi i / N``.
* Decaying isotropic turbulence: random-phase solenoidal field from an energy
  spectrum by the Craya-Herring construction of
  PySpectral/run/HIT/MansourWray/inputfile.py:52-95 (seeded phases drawn with
  NumPy's legacy ``RandomState`` as there), Hermitian-symmetrised by a c2r/r2c
  round trip (as src_MPI/Classes.py:33-45 does) and projected solenoidal.
  The spectrum is E(k) = 16 sqrt(2/pi) u0^2 k^4 / k0^5 exp(-2 (k/k0)^2).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from . import _capi


def periodic_coords(N, L=2 * np.pi):
    a = np.arange(N) * (L / N)
    y, x, z = np.meshgrid(a, a, a)
    return x, y, z


def _ctx64(N, device):
    return _capi.Context(N, N, N, precision=64, device=device)


def tgv_state(N, variant="sin", device=0, ctx=None):
    """(3, N, N, N//2+1) complex128 TGV spectrum."""
    ctx = ctx or _ctx64(N, device)
    dev = torch.device("cuda", device)
    a = torch.arange(N, device=dev, dtype=torch.float64) * (2 * math.pi / N)
    X, Y, Z = torch.meshgrid(a, a, a, indexing="ij")
    if variant == "sin":
        u = torch.sin(X) * torch.cos(Y) * torch.cos(Z)
        v = -torch.cos(X) * torch.sin(Y) * torch.cos(Z)
    else:
        u = torch.cos(X) * torch.sin(Y) * torch.cos(Z)
        v = -torch.sin(X) * torch.cos(Y) * torch.cos(Z)
    phys = torch.stack([u, v, torch.zeros_like(u)]).contiguous()
    spec = torch.empty((3, N, N, N // 2 + 1), dtype=torch.complex128, device=dev)
    ctx.r2c(phys, spec, 3)
    return spec / math.sqrt(N ** 3)


def spectrum_k4(k, k0=4.0, u0=1.0):
    return 16.0 * math.sqrt(2.0 / math.pi) * u0 ** 2 * k ** 4 / k0 ** 5 * torch.exp(-2.0 * (k / k0) ** 2)


def isotropic_phases(N, seed):
    rs = np.random.RandomState(seed)
    sh = (N, N, N // 2 + 1)
    return (rs.rand(*sh) * 2.0 * np.pi, rs.rand(*sh) * 2.0 * np.pi, rs.rand(*sh) * 2.0 * np.pi)


def isotropic_state(N, seed, k0=4.0, u0=1.0, L=2 * np.pi, normalise="sqrtN3", device=0, ctx=None):
    """(3, N, N, N//2+1) complex128 solenoidal random-phase field."""
    ctx = ctx or _ctx64(N, device)
    dev = torch.device("cuda", device)
    th1, th2, phi = (torch.as_tensor(a, device=dev) for a in isotropic_phases(N, seed))
    k1 = torch.as_tensor(np.fft.fftshift(np.linspace(-(N // 2), N // 2 - 1, N)), device=dev)
    k3 = torch.as_tensor(np.linspace(0, N // 2, N // 2 + 1), device=dev)
    K1, K2, K3 = torch.meshgrid(k1, k1, k3, indexing="ij")
    ksqr = K1 ** 2 + K2 ** 2 + K3 ** 2
    kmag = torch.sqrt(ksqr) + 1e-30
    E = spectrum_k4(torch.sqrt(ksqr), k0, u0)
    amp = torch.sqrt(E / (4.0 * math.pi * ksqr + 1e-30))
    alpha = amp * torch.exp(1j * th1) * torch.cos(phi)
    beta = amp * torch.exp(1j * th2) * torch.sin(phi)
    tp = 2.0 * math.pi / L
    kperp = torch.sqrt(K1 ** 2 + K2 ** 2)
    uh = (alpha * kmag * K2 * tp + beta * K1 * tp * K3 * tp) / (kmag * kperp + 1e-30)
    vh = (-alpha * kmag * K1 * tp + beta * K2 * tp * K3 * tp) / (kmag * kperp + 1e-30)
    wh = -beta * kperp / kmag
    st = (torch.stack([uh, vh, wh]) * math.sqrt(N ** 3)).to(torch.complex128).contiguous()
    phys = torch.empty((3, N, N, N), dtype=torch.float64, device=dev)
    ctx.c2r(st, phys, 3)
    ctx.r2c(phys, st, 3)
    kk = (K1 * tp, K2 * tp, K3 * tp)
    ks = kk[0] ** 2 + kk[1] ** 2 + kk[2] ** 2 + 1e-50
    div = (kk[0] * st[0] + kk[1] * st[1] + kk[2] * st[2]) / ks
    st = torch.stack([st[i] - kk[i] * div for i in range(3)]).contiguous()
    if normalise == "none":
        return st * math.sqrt(N ** 3)
    return st
