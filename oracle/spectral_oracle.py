"""CPU oracle for the PySpectral right-hand-side evaluation and RK4 step.

TEST INFRASTRUCTURE ONLY.  This module is the parity checker: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (``pyspectral_b200``) never calls it and fails loudly when
its CUDA library is missing.

It is a from-scratch NumPy restatement of the reference algorithm, written in
FP64 (complex128 / float64) like the reference.  Each function cites the
reference file and lines it restates; paths are relative to the PySpectral
project (``PySpectral/src`` is the serial solver, ``PySpectral/src_MPI`` the MPI
solver that carries the MHD equations).

Parity is pinned: ``tests/test_oracle_golden.py`` checks every routine here
against fixtures produced by executing the unmodified reference sources
(``tests/golden/make_golden.py``) and against the reference's own known-answer
energy history (``run/TGV_Validate100/benchmark_sol_64.npz``).

State layout used throughout: ``state[f, i1, i2, i3]`` complex128 with shape
``(nfields, N1, N2, N3//2+1)``; field order u, v, w (then B1, B2, B3 for MHD).
The reference keeps the same three spectra in the diagonal of a stride-3 array
``Q[0::3,0::3,0::3]`` (``PySpectral/src/Classes.py:30-34``); the dense layout
here holds the identical numbers.
"""
from __future__ import annotations

import math
import os

import numpy as np

try:  # pocketfft with threads when SciPy is present; NumPy otherwise
    import scipy.fft as _fft

    def _rfftn(a, workers=None):
        return _fft.rfftn(a, workers=workers or _WORKERS)

    def _irfftn(a, s, workers=None):
        return _fft.irfftn(a, s=s, workers=workers or _WORKERS)
except Exception:  # pragma: no cover
    def _rfftn(a, workers=None):
        return np.fft.rfftn(a)

    def _irfftn(a, s, workers=None):
        return np.fft.irfftn(a, s=s)

_WORKERS = 1


def set_workers(n: int) -> None:
    """Number of FFT worker threads (the reference's ``nthreads``)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


# --------------------------------------------------------------------------
# Grid / wavenumbers                      PySpectral/src/Classes.py:548-588
# --------------------------------------------------------------------------
class Grid:
    """Wavenumber arrays of ``gridclass`` (``src/Classes.py:548-588``).

    ``dx, dy, dz`` are the spacings of the caller's x, y, z arrays
    (``:561-564``); ``Delta=(dx dy dz)^(1/3)`` (``:581-582``).  ``ksqr`` carries
    the reference's ``+1e-50`` (``:576``)."""

    def __init__(self, N1, N2, N3, dx, dy, dz, kc, L1=2 * np.pi, L2=2 * np.pi, L3=2 * np.pi):
        self.N1, self.N2, self.N3 = N1, N2, N3
        self.L1, self.L2, self.L3 = L1, L2, L3
        self.dx, self.dy, self.dz = dx, dy, dz
        self.kc = kc
        k1 = np.fft.fftshift(np.linspace(-(N1 // 2), N1 // 2 - 1, N1)) * 2.0 * np.pi / L1
        k2 = np.fft.fftshift(np.linspace(-(N2 // 2), N2 // 2 - 1, N2)) * 2.0 * np.pi / L2
        k3 = np.linspace(0, N3 // 2, N3 // 2 + 1) * 2.0 * np.pi / L3
        k1f = np.fft.fftshift(np.linspace(-N1, N1 - 1, 2 * N1)) * 2.0 * np.pi / L1
        k2f = np.fft.fftshift(np.linspace(-N2, N2 - 1, 2 * N2)) * 2.0 * np.pi / L2
        k3f = np.linspace(0, N3, N3 + 1) * 2.0 * np.pi / L3
        self.k1d, self.k2d, self.k3d = k1, k2, k3
        self.k1fd, self.k2fd, self.k3fd = k1f, k2f, k3f
        self.k2, self.k1, self.k3 = np.meshgrid(k2, k1, k3)
        self.k2f, self.k1f, self.k3f = np.meshgrid(k2f, k1f, k3f)
        self.ksqr = self.k1 * self.k1 + self.k2 * self.k2 + self.k3 * self.k3 + 1.0e-50
        self.ksqr_i = 1.0 / self.ksqr
        self.ksqrf = self.k1f * self.k1f + self.k2f * self.k2f + self.k3f * self.k3f + 1.0e-50
        self.ksqrf_i = 1.0 / self.ksqrf
        self.Delta = (dx * dy * dz) ** (1.0 / 3.0)
        # sharp spectral cutoff at kc, Nyquist index excluded (:584-588)
        Gf = np.zeros(self.k1.shape)
        Gf[0:kc, 0:kc, 0:kc] = 1
        Gf[0:kc, N2 - kc + 1:, 0:kc] = 1
        Gf[N1 - kc + 1:, 0:kc, 0:kc] = 1
        Gf[N1 - kc + 1:, N2 - kc + 1:, 0:kc] = 1
        self.Gf = Gf

    @classmethod
    def periodic(cls, N, kc=None, L=2 * np.pi):
        """Cube with the exactly periodic spacing ``dx = L/N``."""
        return cls(N, N, N, L / N, L / N, L / N, N // 2 if kc is None else kc, L, L, L)


# --------------------------------------------------------------------------
# Padding / truncation                     PySpectral/src/padding.py
# --------------------------------------------------------------------------
def pad(uhat):
    """3/2 zero padding, ``src/padding.py:16-25``.  Copies the four corner
    blocks; index N/2 of axes 0 and 1 and the k3=N/2 plane are dropped."""
    N1, N2, N3h = uhat.shape
    h1, h2 = N1 // 2, N2 // 2
    M1, M2 = 3 * N1 // 2, 3 * N2 // 2
    out = np.zeros((M1, M2, N3h + (N3h - 1) // 2), dtype=complex)
    z = slice(0, N3h - 1)
    out[0:h1, 0:h2, z] = uhat[0:h1, 0:h2, z]
    out[0:h1, M2 - h2 + 1:, z] = uhat[0:h1, h2 + 1:, z]
    out[M1 - h1 + 1:, 0:h2, z] = uhat[h1 + 1:, 0:h2, z]
    out[M1 - h1 + 1:, M2 - h2 + 1:, z] = uhat[h1 + 1:, h2 + 1:, z]
    return out


def unpad(upad):
    """Inverse of :func:`pad`, ``src/padding.py:2-13``."""
    M1, M2, M3h = upad.shape
    N1, N2 = int(M1 * 2.0 / 3.0), int(M2 * 2.0 / 3.0)
    N3h = int(M3h * 2.0 / 3.0 + 1)
    h1, h2 = N1 // 2, N2 // 2
    out = np.zeros((N1, N2, N3h), dtype=complex)
    z = slice(0, N3h - 1)
    out[0:h1, 0:h2, z] = upad[0:h1, 0:h2, z]
    out[0:h1, h2 + 1:, z] = upad[0:h1, M2 - h2 + 1:, z]
    out[h1 + 1:, 0:h2, z] = upad[M1 - h1 + 1:, 0:h2, z]
    out[h1 + 1:, h2 + 1:, z] = upad[M1 - h1 + 1:, M2 - h2 + 1:, z]
    return out


def pad_2x(uhat):
    """2x zero padding, ``src/padding.py:41-49`` (keeps index N/2 of axes 0,1
    as the -N/2 mode; drops k3=N/2)."""
    N1, N2, N3h = uhat.shape
    h1, h2 = N1 // 2, N2 // 2
    out = np.zeros((2 * N1, 2 * N2, 2 * N3h - 1), dtype=complex)
    z = slice(0, N3h - 1)
    out[0:h1, 0:h2, z] = uhat[0:h1, 0:h2, z]
    out[0:h1, 2 * N2 - h2:, z] = uhat[0:h1, h2:, z]
    out[2 * N1 - h1:, 0:h2, z] = uhat[h1:, 0:h2, z]
    out[2 * N1 - h1:, 2 * N2 - h2:, z] = uhat[h1:, h2:, z]
    return out


def unpad_2x(upad):
    """Inverse of :func:`pad_2x`, ``src/padding.py:28-38``."""
    M1, M2, M3h = upad.shape
    N1, N2, N3h = M1 // 2, M2 // 2, (M3h + 1) // 2
    h1, h2 = N1 // 2, N2 // 2
    out = np.zeros((N1, N2, N3h), dtype=complex)
    z = slice(0, N3h - 1)
    out[0:h1, 0:h2, z] = upad[0:h1, 0:h2, z]
    out[0:h1, h2:, z] = upad[0:h1, 2 * N2 - h2:, z]
    out[h1:, 0:h2, z] = upad[2 * N1 - h1:, 0:h2, z]
    out[h1:, h2:, z] = upad[2 * N1 - h1:, 2 * N2 - h2:, z]
    return out


def separate_modes(upad):
    """Resolved/unresolved split on the 2x grid, ``src/padding.py:67-79``:
    p = {|k1|,|k2| < N/2, 0 <= k3 < N/2}; q = the rest (Nyquist included)."""
    M1, M2, M3h = upad.shape
    N1, N2, N3h = M1 // 2, M2 // 2, (M3h + 1) // 2
    p = np.zeros_like(upad)
    z = slice(0, M3h - N3h)
    a1, b1 = slice(0, N1 // 2), slice(M1 - N1 // 2 + 1, M1)
    a2, b2 = slice(0, N2 // 2), slice(M2 - N2 // 2 + 1, M2)
    for s1 in (a1, b1):
        for s2 in (a2, b2):
            p[s1, s2, z] = upad[s1, s2, z]
    return p, upad - p


def separate_modes_testfilter(upad, kf):
    """Test-filter split on the 2x grid, ``src/padding.py:52-64``:
    p = {|k1|,|k2| < kf, 0 <= k3 < kf}."""
    M1, M2, _ = upad.shape
    p = np.zeros_like(upad)
    z = slice(0, kf)
    for s1 in (slice(0, kf), slice(M1 - kf + 1, M1)):
        for s2 in (slice(0, kf), slice(M2 - kf + 1, M2)):
            p[s1, s2, z] = upad[s1, s2, z]
    return p, upad - p


# --------------------------------------------------------------------------
# Transforms                               PySpectral/src/Classes.py:590-625
# --------------------------------------------------------------------------
def scale_32(g):
    """``scale`` of ``FFTclass`` (``src/Classes.py:593``)."""
    return math.sqrt((3.0 / 2.0) ** 3 * math.sqrt(g.N1 * g.N2 * g.N3))


def scale_2x(g):
    """``scale`` of the 2x-padded closures (``src/RHSfunctions.py:244``)."""
    return math.sqrt(2.0 ** 3 * math.sqrt(g.N1 * g.N2 * g.N3))


def ifft32(g, X):
    """``ifftT_obj``: c2r on the 3/2 grid with 1/M normalisation
    (pyFFTW ``normalise_idft=True``), ``src/Classes.py:596-599``."""
    return _irfftn(X, s=(3 * g.N1 // 2, 3 * g.N2 // 2, 3 * g.N3 // 2))


def fft32(x):
    """``fft_obj``: unnormalised r2c, ``src/Classes.py:601-605``."""
    return _rfftn(x)


def ifft2x(g, X):
    """``ifftT_obj2`` on the 2x grid, ``src/Classes.py:607-610``."""
    return _irfftn(X, s=(2 * g.N1, 2 * g.N2, 2 * g.N3))


def fft2x(x):
    """``fft_obj2``, ``src/Classes.py:612-615``."""
    return _rfftn(x)


def nyquist_zero(uhat):
    """``unpad(pad(uhat))`` as applied on read at ``src/RHSfunctions.py:10-12``."""
    return unpad(pad(uhat))


def _coriolis_pressure(k1, k2, k3, ksqr_i, u, v, w, Om):
    Om1, Om2, Om3 = Om
    return -2.0 * ksqr_i * 1j * (k1 * (v * Om3 - w * Om2) + k2 * (w * Om1 - u * Om3)
                                 + k3 * (u * Om2 - v * Om1))


def _coriolis_force(u, v, w, Om):
    Om1, Om2, Om3 = Om
    return (2.0 * (v * Om3 - w * Om2), 2.0 * (w * Om1 - u * Om3), 2.0 * (u * Om2 - v * Om1))


class Params:
    """Run parameters carried by the reference's ``variables`` object
    (``src/Classes.py:8-26``) and its driver defaults (``src/PySpec_3d.py:9-72``)."""

    def __init__(self, nu, t=0.0, dt=0.0, rotate=0, Om=(0.0, 0.0, 0.0), Ct=0.1,
                 tau_a=0.0, tau_b=0.0, kf=None):
        self.nu, self.t, self.dt = nu, t, dt
        self.rotate, self.Om = rotate, tuple(Om)
        self.Ct, self.tau_a, self.tau_b, self.kf = Ct, tau_a, tau_b, kf


# --------------------------------------------------------------------------
# Right-hand sides                          PySpectral/src/RHSfunctions.py
# --------------------------------------------------------------------------
def _products_32(g, u, v, w):
    """The six 3/2-dealiased quadratic products (``src/RHSfunctions.py:14-23``)."""
    s = scale_32(g)
    ur = ifft32(g, pad(u)) * s
    vr = ifft32(g, pad(v)) * s
    wr = ifft32(g, pad(w)) * s
    return [unpad(fft32(a * b)) for a, b in ((ur, ur), (vr, vr), (wr, wr), (ur, vr), (ur, wr), (vr, wr))]


def _pressure(k1, k2, k3, ksqr_i, uu, vv, ww, uv, uw, vw):
    return ksqr_i * (-k1 * k1 * uu - k2 * k2 * vv - k3 * k3 * ww - 2.0 * k1 * k2 * uv
                     - 2.0 * k1 * k3 * uw - 2.0 * k2 * k3 * vw)


def _advection(k1, k2, k3, nu, ksqr, phat, P, u, v, w):
    uu, vv, ww, uv, uw, vw = P
    ru = -1j * k1 * uu - 1j * k2 * uv - 1j * k3 * uw - 1j * k1 * phat - nu * ksqr * u
    rv = -1j * k1 * uv - 1j * k2 * vv - 1j * k3 * vw - 1j * k2 * phat - nu * ksqr * v
    rw = -1j * k1 * uw - 1j * k2 * vw - 1j * k3 * ww - 1j * k3 * phat - nu * ksqr * w
    return ru, rv, rw


def rhs_nosgs(g, state, p):
    """DNS right-hand side, ``computeRHS_NOSGS`` (``src/RHSfunctions.py:3-50``).

    Returns ``(rhs, uhat_read)``; ``uhat_read`` is the Nyquist-zeroed state the
    reference rebinds to ``main.uhat`` (``:10-12``)."""
    u, v, w = (nyquist_zero(state[i]) for i in range(3))
    P = _products_32(g, u, v, w)
    k1, k2, k3 = g.k1, g.k2, g.k3
    phat = _pressure(k1, k2, k3, g.ksqr_i, *P)
    if p.rotate == 1:
        phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, u, v, w, p.Om)
    r = list(_advection(k1, k2, k3, p.nu, g.ksqr, phat, P, u, v, w))
    if p.rotate == 1:
        c = _coriolis_force(u, v, w, p.Om)
        r = [r[i] + c[i] for i in range(3)]
    return np.stack(r), np.stack([u, v, w])


def rhs_orthogonal(g, state, p):
    """Orthogonal dynamics, ``computeRHS_Orthogonal`` (``src/RHSfunctions.py:53-143``):
    the DNS right-hand side of the (Nyquist-zeroed) state minus that of
    ``Gf u``, each with its own pressure and Coriolis terms.  Returns
    ``(rhs, uhat_read)``."""
    u, v, w = (nyquist_zero(state[i]) for i in range(3))
    k1, k2, k3 = g.k1, g.k2, g.k3

    def part(a, b, c):
        P = _products_32(g, a, b, c)
        phat = _pressure(k1, k2, k3, g.ksqr_i, *P)
        if p.rotate == 1:
            phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, a, b, c, p.Om)
        return list(_advection(k1, k2, k3, p.nu, g.ksqr, phat, P, a, b, c))
    r = part(u, v, w)
    if p.rotate == 1:
        cf = _coriolis_force(u, v, w, p.Om)
        r = [r[i] + cf[i] for i in range(3)]
    uf, vf, wf = g.Gf * u, g.Gf * v, g.Gf * w
    rf = part(uf, vf, wf)
    r = [r[i] - rf[i] for i in range(3)]
    if p.rotate == 1:
        cf = _coriolis_force(uf, vf, wf, p.Om)
        r = [r[i] - cf[i] for i in range(3)]
    return np.stack(r), np.stack([u, v, w])


def _sgs_divergence(g, tau):
    """Projected divergence of a stress, ``src/RHSfunctions.py:215-222``
    (identical form at ``src/Classes.py:917-927``).  Note the reference's
    projection term is ``1j*k_i * (1j*ksqr_i*k_m k_j tau_jm)``."""
    k1, k2, k3 = g.k1, g.k2, g.k3
    t11, t22, t33, t12, t13, t23 = tau
    proj = 1j * g.ksqr_i * (k1 * k1 * t11 + k2 * k2 * t22 + k3 * k3 * t33 + 2.0 * k1 * k2 * t12
                            + 2.0 * k1 * k3 * t13 + 2.0 * k2 * k3 * t23)
    w0u = -1j * k1 * t11 - 1j * k2 * t12 - 1j * k3 * t13 + 1j * k1 * proj
    w0v = -1j * k1 * t12 - 1j * k2 * t22 - 1j * k3 * t23 + 1j * k2 * proj
    w0w = -1j * k1 * t13 - 1j * k2 * t23 - 1j * k3 * t33 + 1j * k3 * proj
    return np.stack([w0u, w0v, w0w])


def smag_stress(g, u, v, w):
    """Smagorinsky stress in Fourier space, ``src/RHSfunctions.py:174-212``
    (Cs = 0.16 fixed, ``:197``)."""
    s = scale_32(g)
    k1, k2, k3 = g.k1, g.k2, g.k3
    Shat = (1j * k1 * u, 1j * k2 * v, 1j * k3 * w, 0.5 * (1j * k2 * u + 1j * k1 * v),
            0.5 * (1j * k3 * u + 1j * k1 * w), 0.5 * (1j * k3 * v + 1j * k2 * w))
    S = [ifft32(g, pad(x) * s) for x in Shat]
    S11, S22, S33, S12, S13, S23 = S
    Smag = np.sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * S12 * S12 + 2.0 * S13 * S13
                          + 2.0 * S23 * S23))
    nut = 0.16 * g.Delta * 0.16 * g.Delta * np.abs(Smag)
    return [unpad(fft32(-2.0 * nut * x)) for x in S]


def rhs_smag(g, state, p):
    """Smagorinsky right-hand side, ``computeRHS_SMAG``
    (``src/RHSfunctions.py:146-237``).  No Nyquist re-zeroing on read.

    Returns ``(rhs, w0)`` where ``w0`` is the SGS force (``main.w0_*``)."""
    u, v, w = state[0], state[1], state[2]
    P = _products_32(g, u, v, w)
    k1, k2, k3 = g.k1, g.k2, g.k3
    phat = _pressure(k1, k2, k3, g.ksqr_i, *P)
    if p.rotate == 1:
        phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, u, v, w, p.Om)
    w0 = _sgs_divergence(g, smag_stress(g, u, v, w))
    r = list(_advection(k1, k2, k3, p.nu, g.ksqr, phat, P, u, v, w))
    r = [r[i] + w0[i] for i in range(3)]
    if p.rotate == 1:
        c = _coriolis_force(u, v, w, p.Om)
        r = [r[i] + c[i] for i in range(3)]
    return np.stack(r), w0


def myfilter_axes(g, kc):
    """Index masks of ``utilitiesClass.myFilter(uhat, kc)`` (``src/Classes.py:1271-1279``):
    rows ``[0:kc]`` and ``[-kc+1:]`` of axes 1 and 2, ``[0:kc]`` of axis 3,
    with Python slice semantics (so ``kc = 1`` keeps whole rows, since
    ``-kc+1 = 0``).  A fractional ``kc`` is truncated, as the NumPy the
    reference was written for did with float slice bounds."""
    kc = int(kc)

    def rows(n):
        m = np.zeros(n)
        m[0:kc] = 1.0
        m[-kc + 1:] = 1.0
        return m
    m3 = np.zeros(g.N3 // 2 + 1)
    m3[0:kc] = 1.0
    return rows(g.N1), rows(g.N2), m3


def myfilter(g, uhat, kc):
    m1, m2, m3 = myfilter_axes(g, kc)
    return uhat * (m1[:, None, None] * m2[None, :, None] * m3[None, None, :])


def dsmag_cs2(g, u, v, w, return_parts=False):
    """The dynamic coefficient ``Cs_sqr = mean(L:M)/mean(M:M)`` of
    ``computeRHS_DSMAG`` (``src/RHSfunctions.py:1693-1843``): Leonard stress
    ``L = F(u_i u_j) - (F u_i F u_j)``, ``M = -2 Delta^2 (alpha^2 |S~|S~ - F(|S|S))``
    with the test filter ``F = myFilter(., kc/alpha)``, ``alpha = 2``; both
    means taken on the 3/2-padded physical grid, off-diagonal terms weighted 1
    as written at ``:1838-1841``."""
    alpha = 2.0
    kL = g.kc / alpha
    s = scale_32(g)
    k1, k2, k3 = g.k1, g.k2, g.k3
    P = _products_32(g, u, v, w)
    uF, vF, wF = (myfilter(g, x, kL) for x in (u, v, w))
    PF = _products_32(g, uF, vF, wF)
    L = [myfilter(g, P[i], kL) - PF[i] for i in range(6)]

    def strain(a, b, c):
        Sh = (1j * k1 * a, 1j * k2 * b, 1j * k3 * c, 0.5 * (1j * k2 * a + 1j * k1 * b),
              0.5 * (1j * k3 * a + 1j * k1 * c), 0.5 * (1j * k3 * b + 1j * k2 * c))
        S = [ifft32(g, pad(x) * s) for x in Sh]
        S11, S22, S33, S12, S13, S23 = S
        mag = np.sqrt(2.0 * (S11 * S11 + S22 * S22 + S33 * S33 + 2.0 * S12 * S12 + 2.0 * S13 * S13
                             + 2.0 * S23 * S23))
        return S, mag
    S, Smag = strain(u, v, w)
    SF, SmagF = strain(uF, vF, wF)
    SFS = [unpad(fft32(SmagF * x)) for x in SF]
    SSF = [myfilter(g, unpad(fft32(Smag * x)), kL) for x in S]
    M = [-2.0 * g.Delta ** 2 * (alpha ** 2 * SFS[i] - SSF[i]) for i in range(6)]
    Mr = [ifft32(g, pad(x)) * s for x in M]
    Lr = [ifft32(g, pad(x)) * s for x in L]
    num = sum(Mr[i] * Lr[i] for i in range(6))
    den = sum(Mr[i] * Mr[i] for i in range(6))
    cs2 = np.mean(num) / np.mean(den)
    if return_parts:
        return cs2, P, S, Smag
    return cs2


def rhs_dsmag(g, state, p):
    """Dynamic Smagorinsky right-hand side, ``computeRHS_DSMAG``
    (``src/RHSfunctions.py:1663-1862``): the Smagorinsky form of ``:146-237``
    with ``Cs^2`` from :func:`dsmag_cs2` in place of ``0.16^2``.

    Returns ``(rhs, w0, cs2)``."""
    u, v, w = state[0], state[1], state[2]
    cs2, P, S, Smag = dsmag_cs2(g, u, v, w, return_parts=True)
    k1, k2, k3 = g.k1, g.k2, g.k3
    phat = _pressure(k1, k2, k3, g.ksqr_i, *P)
    if p.rotate == 1:
        phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, u, v, w, p.Om)
    nut = cs2 * g.Delta * g.Delta * np.abs(Smag)
    tau = [unpad(fft32(-2.0 * nut * x)) for x in S]
    w0 = _sgs_divergence(g, tau)
    r = list(_advection(k1, k2, k3, p.nu, g.ksqr, phat, P, u, v, w))
    r = [r[i] + w0[i] for i in range(3)]
    if p.rotate == 1:
        c = _coriolis_force(u, v, w, p.Om)
        r = [r[i] + c[i] for i in range(3)]
    return np.stack(r), w0, cs2


def _pl_2x(g, up, vp, wp, nu, rotate, Om):
    """``PLu`` on the 2x grid (``src/RHSfunctions.py:269-315``): returns the
    full-grid PL fields, the physical velocities and the 2x product spectra."""
    s = scale_2x(g)
    ur, vr, wr = ifft2x(g, up * s), ifft2x(g, vp * s), ifft2x(g, wp * s)
    P = [fft2x(a * b) for a, b in ((ur, ur), (vr, vr), (wr, wr), (ur, vr), (ur, wr), (vr, wr))]
    k1, k2, k3 = g.k1f, g.k2f, g.k3f
    phat = _pressure(k1, k2, k3, g.ksqrf_i, *P)
    if rotate == 1:
        phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqrf_i, up, vp, wp, Om)
    PL = _advection(k1, k2, k3, nu, g.ksqrf, phat, P, up, vp, wp)
    return PL, (ur, vr, wr), P, phat


def _plql(g, vel_real, PLq):
    """``PLQLu`` from the q-part of PL (``src/RHSfunctions.py:321-352``
    and ``:451-478``)."""
    s = scale_2x(g)
    ur, vr, wr = vel_real
    qr = [ifft2x(g, x * s) for x in PLq]
    # a[j][i] = unpad_2x(fft(u_j * PL_q,i))
    a = [[unpad_2x(fft2x(vel * q)) for q in qr] for vel in (ur, vr, wr)]
    up_u, up_v, up_w = a[0]
    vp_u, vp_v, vp_w = a[1]
    wp_u, wp_v, wp_w = a[2]
    k1, k2, k3 = g.k1, g.k2, g.k3
    pterm = 2.0 * g.ksqr_i * (k1 * k1 * up_u + k2 * k2 * vp_v + k3 * k3 * wp_w
                              + k1 * k2 * (up_v + vp_u) + k1 * k3 * (up_w + wp_u)
                              + k2 * k3 * (vp_w + wp_v))
    Lu = (-1j * k1 * up_u - 1j * k2 * vp_u - 1j * k3 * wp_u
          - 1j * k1 * up_u - 1j * k2 * up_v - 1j * k3 * up_w + 1j * k1 * pterm)
    Lv = (-1j * k1 * up_v - 1j * k2 * vp_v - 1j * k3 * wp_v
          - 1j * k1 * vp_u - 1j * k2 * vp_v - 1j * k3 * vp_w + 1j * k2 * pterm)
    Lw = (-1j * k1 * up_w - 1j * k2 * vp_w - 1j * k3 * wp_w
          - 1j * k1 * wp_u - 1j * k2 * wp_v - 1j * k3 * wp_w + 1j * k3 * pterm)
    return np.stack([Lu, Lv, Lw])


def _memory_rhs(g, state, p, coef_fn):
    """Shared body of the t-model and tau-models
    (``src/RHSfunctions.py:240-363`` / ``:366-497``)."""
    u, v, w = (nyquist_zero(state[i]) for i in range(3))
    up, vp, wp = pad_2x(u), pad_2x(v), pad_2x(w)
    PL, vel, P, phat = _pl_2x(g, up, vp, wp, p.nu, p.rotate, p.Om)
    PLq = [separate_modes(x)[1] for x in PL]
    PLQL = _plql(g, vel, PLq)
    coef, extra = coef_fn(u, v, w, up, vp, wp, P, phat, PLQL)
    w0 = coef * PLQL
    r = [unpad_2x(PL[i]) + w0[i] for i in range(3)]
    if p.rotate == 1:
        c = _coriolis_force(u, v, w, p.Om)
        r = [r[i] + c[i] for i in range(3)]
    return np.stack(r), w0, np.stack([u, v, w]), PLQL, extra


def rhs_tmodel(g, state, p):
    """t-model, ``computeRHS_tmodel`` (``src/RHSfunctions.py:240-363``):
    ``w0 = Ct * t * PLQLu``.  Returns ``(rhs, w0, uhat_read)``."""
    r, w0, ur, _, _ = _memory_rhs(g, state, p, lambda *a: (p.Ct * p.t, None))
    return r, w0, ur


def rhs_fm1(g, state, p, dt0=0.1, nsub=1):
    """First-order finite memory model, ``computeRHS_FM1``
    (``src/RHSfunctions.py:882-1024``) on the state ``(u, v, w)`` followed by
    ``(w0_u, w0_v, w0_w)`` of each of the ``nsub`` subintegrations:
    ``du/dt = unpad_2x(PL u) + sum_i w0^i``,
    ``dw0^i/dt = -2/d w0^i + (-1)^(i+1) 2 PLQL u + S_i`` with ``d = dt0/nsub``
    and ``S_i`` the running sum of ``:1010-1014`` (not reset between i).

    The reference source calls ``pad_2x_var``, which none of its files
    defines; this restatement (and the fixtures) use ``pad_2x`` there.  With
    rotation the reference adds the Coriolis force to PL on the 2x grid before
    the mode split (``:959-962``); that force lives on the resolved modes only
    (``pad_2x`` of the Nyquist-zeroed state), so PL_q and PLQL are unchanged
    and the force joins the velocity RHS, as in ``_memory_rhs``.

    Returns ``(rhs, w0_read, uhat_read)``, ``w0_read`` the first
    subintegration's memory variables (``main.w0_*[..., 0]``)."""
    r, _, ur, PLQL, _ = _memory_rhs(g, state[:3], p, lambda *a: (0.0, None))
    w = [state[3 + 3 * i:6 + 3 * i] for i in range(nsub)]
    d = dt0 / nsub
    out = [r[c] + np.sum(np.stack([w[i][c] for i in range(nsub)], axis=-1), axis=-1) for c in range(3)]
    run = [np.zeros_like(r[0]) for _ in range(3)]
    for i in range(1, nsub + 1):
        for j in range(1, i):
            for c in range(3):
                run[c] = run[c] + 4.0 / d * (-1.0) ** (i + j + 1) * w[j - 1][c]
        out += [-2.0 / d * w[i - 1][c] + (-1.0) ** (i + 1) * 2.0 * PLQL[c] + run[c] for c in range(3)]
    return np.stack(out), np.stack(w[0]), ur


def fm2_layout(nsub):
    """Field offsets of w0^i and w1^i in the FM2 state with
    ``dt0_subintegrations = dt1_subintegrations = nsub``
    (``src/Classes.py:330-355``: the pairs interleave, w0 from 3, w1 from 6)."""
    return [3 + 6 * i for i in range(nsub)], [6 + 6 * i for i in range(nsub)]


def rhs_fm2(g, state, p, dt0=0.1, dt1=0.05, nsub=1):
    """Second-order finite memory model, ``computeRHS_FM2``
    (``src/RHSfunctions.py:1025-1287``, turb_model 4), cubic grids, equal
    numbers of w0 and w1 subintegrations (unequal ones index past w1 in the
    reference, ``:1252``).  PL and PLQL on the full 2x grid; the products
    ``PL_i (PL_q)_j`` on the 3N grid (``pad`` of the 2x grid); ``PLQL_q u_j``
    on the 2x grid; ``PLQLQL`` as written at ``:1214-1224`` (including the
    sign of the ``PLQLuq_up`` term of the u component).  No rotating form
    (the reference's raises).  Returns ``(rhs, uhat_read)``."""
    if p.rotate == 1:
        raise ValueError("computeRHS_FM2 has no rotating form")
    N1, N2, N3 = g.N1, g.N2, g.N3
    u, v, w = (nyquist_zero(state[i]) for i in range(3))
    s2 = scale_2x(g)
    up, vp, wp = pad_2x(u), pad_2x(v), pad_2x(w)
    ur, vr, wr = ifft2x(g, up * s2), ifft2x(g, vp * s2), ifft2x(g, wp * s2)
    P = [fft2x(a * b) for a, b in ((ur, ur), (vr, vr), (wr, wr), (ur, vr), (ur, wr), (vr, wr))]
    K1, K2, K3 = g.k1f, g.k2f, g.k3f
    phat = _pressure(K1, K2, K3, g.ksqrf_i, *P)
    PL = _advection(K1, K2, K3, p.nu, g.ksqrf, phat, P, up, vp, wp)
    PLq = [separate_modes(x)[1] for x in PL]
    qr = [ifft2x(g, x * s2) for x in PLq]
    a = [[fft2x(vel * q) for q in qr] for vel in (ur, vr, wr)]  # a[j][i] = (u_j PLq_i)^ on 2x
    upu, upv, upw = a[0]
    vpu, vpv, vpw = a[1]
    wpu, wpv, wpw = a[2]
    pt = 2.0 * g.ksqrf_i * (K1 * K1 * upu + K2 * K2 * vpv + K3 * K3 * wpw + K1 * K2 * (upv + vpu)
                            + K1 * K3 * (upw + wpu) + K2 * K3 * (vpw + wpv))
    PLQL2 = [-1j * K1 * upu - 1j * K2 * vpu - 1j * K3 * wpu - 1j * K1 * upu - 1j * K2 * upv - 1j * K3 * upw
             + 1j * K1 * pt,
             -1j * K1 * upv - 1j * K2 * vpv - 1j * K3 * wpv - 1j * K1 * vpu - 1j * K2 * vpv - 1j * K3 * vpw
             + 1j * K2 * pt,
             -1j * K1 * upw - 1j * K2 * vpw - 1j * K3 * wpw - 1j * K1 * wpu - 1j * K2 * wpv - 1j * K3 * wpw
             + 1j * K3 * pt]
    PLQLq = [separate_modes(x)[1] for x in PLQL2]
    # PL x PL_q on the 3N grid
    sc3 = np.sqrt(3.0 ** 3 * np.sqrt(N1 * N2 * N3))

    def i3n(x):
        return _irfftn(pad(x) * sc3, s=(3 * N1, 3 * N2, 3 * N3))
    PLr = [i3n(x) for x in PL]
    PLqr = [i3n(x) for x in PLq]

    def c3n(x, y):
        return unpad_2x(unpad(_rfftn(x * y)))
    # names of the reference: PLa_PLbq = PL_a * (PL_q)_b
    PLu_PLuq, PLv_PLuq, PLw_PLuq = (c3n(PLr[j], PLqr[0]) for j in range(3))
    PLu_PLvq, PLv_PLvq, PLw_PLvq = (c3n(PLr[j], PLqr[1]) for j in range(3))
    PLu_PLwq, PLv_PLwq, PLw_PLwq = (c3n(PLr[j], PLqr[2]) for j in range(3))
    Qr = [ifft2x(g, x * s2) for x in PLQLq]

    def c2(x, y):
        return unpad_2x(fft2x(x * y))
    PLQLuq_up, PLQLvq_up, PLQLwq_up = (c2(Qr[i], ur) for i in range(3))
    PLQLuq_vp, PLQLvq_vp, PLQLwq_vp = (c2(Qr[i], vr) for i in range(3))
    PLQLuq_wp, PLQLvq_wp, PLQLwq_wp = (c2(Qr[i], wr) for i in range(3))
    k1, k2, k3 = g.k1, g.k2, g.k3
    pterm = g.ksqr_i * (k1 * k1 * PLu_PLuq + k2 * k2 * PLv_PLvq + k3 * k3 * PLw_PLwq + k1 * k2 * (PLv_PLuq + PLu_PLvq)
                        + k1 * k3 * (PLu_PLwq + PLw_PLuq) + k2 * k3 * (PLv_PLwq + PLw_PLvq))
    pterm2 = g.ksqr_i * (k1 * k1 * PLQLuq_up + k2 * k2 * PLQLvq_vp + k3 * k3 * PLQLwq_wp
                         + k1 * k2 * (PLQLvq_up + PLQLuq_vp) + k1 * k3 * (PLQLwq_up + PLQLuq_wp)
                         + k2 * k3 * (PLQLwq_vp + PLQLvq_wp))
    qu, qv, qw = (unpad_2x(x) for x in PLQLq)
    nu = p.nu
    QQu = (2. * -1j * k1 * PLu_PLuq - 1j * k2 * PLv_PLuq - 1j * k3 * PLw_PLuq - 1j * k2 * PLu_PLvq - 1j * k3 * PLu_PLwq
           + 2. * 1j * k1 * pterm + -2. * -1j * k1 * PLQLuq_up - 1j * k2 * PLQLvq_up - 1j * k3 * PLQLwq_up
           - 1j * k2 * PLQLuq_vp - 1j * k3 * PLQLuq_wp + 2. * 1j * k1 * pterm2 - nu * g.ksqr * qu)
    QQv = (-1j * k1 * PLu_PLvq - 2. * 1j * k2 * PLv_PLvq - 1j * k3 * PLw_PLvq - 1j * k1 * PLv_PLuq - 1j * k3 * PLv_PLwq
           + 2. * 1j * k2 * pterm + -1j * k1 * PLQLuq_vp - 2. * 1j * k2 * PLQLvq_vp - 1j * k3 * PLQLwq_vp
           - 1j * k1 * PLQLvq_up - 1j * k3 * PLQLvq_wp + 2. * 1j * k2 * pterm2 - nu * g.ksqr * qv)
    QQw = (-1j * k1 * PLu_PLwq - 1j * k2 * PLv_PLwq - 2. * 1j * k3 * PLw_PLwq - 1j * k1 * PLw_PLuq - 1j * k2 * PLw_PLvq
           + 2. * 1j * k3 * pterm + -1j * k1 * PLQLuq_wp - 1j * k2 * PLQLvq_wp - 2. * 1j * k3 * PLQLwq_wp
           - 1j * k1 * PLQLwq_up - 1j * k3 * PLQLwq_vp + 2. * 1j * k3 * pterm2 - nu * g.ksqr * qw)
    PLQL = [unpad_2x(x) for x in PLQL2]
    PLQLQL = [QQu, QQv, QQw]
    o0, o1 = fm2_layout(nsub)
    w0 = [state[o:o + 3] for o in o0]
    w1 = [state[o:o + 3] for o in o1]
    out = np.zeros((3 + 6 * nsub,) + u.shape, dtype=complex)
    for c in range(3):
        out[c] = unpad_2x(PL[c]) + np.sum(np.stack([w0[i][c] for i in range(nsub)], axis=-1), axis=-1)
    d0, d1 = dt0 / nsub, dt1 / nsub
    run = [np.zeros_like(u) for _ in range(3)]
    for i in range(1, nsub + 1):
        for j in range(1, i):
            for c in range(3):
                run[c] = run[c] + 4. / d0 * (-1.) ** (i + j + 1) * w0[j - 1][c]
        for c in range(3):
            out[o0[i - 1] + c] = -2. / d0 * w0[i - 1][c] + (-1.) ** (i + 1) * 2. * PLQL[c] + run[c] + w1[i - 1][c]
    run = [np.zeros_like(u) for _ in range(3)]
    for i in range(1, nsub + 1):
        for j in range(1, i):
            for c in range(3):
                run[c] = run[c] + 4. / d1 * (-1.) ** (i + j + 1) * w1[j - 1][c]
        for c in range(3):
            out[o1[i - 1] + c] = -2. / d1 * w1[i - 1][c] + (-1.) ** (i + 1) * 2. * PLQLQL[c] + run[c]
    return out, np.stack([u, v, w])


def rhs_fm1_2term(g, state, p, dt0=0.1):
    """Two-term first-order finite memory model, ``computeRHS_FM1_2term``
    (``src/RHSfunctions.py:1288-1410``, turb_model 5) on ``(u, w0, w01)``:
    ``du/dt = unpad_2x(PL u) + w0 + w01``, ``dw0/dt = -2/dt0 w0 + 2 PLQL``,
    ``dw01/dt = -2/dt0 w01 - 2 PLQL + 4/dt0 w0``.  ``rotate = 1`` raises in
    the reference (an N-grid Coriolis pressure added to the 2x-grid ``phat``).

    Returns ``(rhs, uhat_read)``."""
    if p.rotate == 1:
        raise ValueError("computeRHS_FM1_2term has no rotating form")
    r, _, ur, PLQL, _ = _memory_rhs(g, state[:3], p, lambda *a: (0.0, None))
    w0, w01 = state[3:6], state[6:9]
    out = [r[c] + w0[c] + w01[c] for c in range(3)]
    out += [-2.0 / dt0 * w0[c] + 2.0 * PLQL[c] for c in range(3)]
    out += [-2.0 / dt0 * w01[c] - 2.0 * PLQL[c] + 4.0 / dt0 * w0[c] for c in range(3)]
    return np.stack(out), ur


def rhs_cm1(g, state, p):
    """First-order complete memory model, ``computeRHS_CM1``
    (``src/RHSfunctions.py:1411-1542``) on the state ``(u, v, w, w0_u, w0_v,
    w0_w)``: ``du/dt = unpad_2x(PL u) + w0``, ``dw0/dt = PLQL u - 250 nu k^2 w0``.

    As in the reference, ``w0_v`` is read as zero: its ``Q2U`` takes it from
    ``Q[3::6, 4::6, 4::6]`` (``src/Classes.py:489``), a slice of the
    interleaved state that nothing writes.  ``rotate = 1`` raises there (an
    N-grid Coriolis pressure added to the 2x-grid ``phat``, ``:1463-1465``).

    Returns ``(rhs, w0_read, uhat_read)``."""
    if p.rotate == 1:
        raise ValueError("computeRHS_CM1 has no rotating form")
    r, _, ur, PLQL, _ = _memory_rhs(g, state[:3], p, lambda *a: (0.0, None))
    w0 = np.stack([state[3], np.zeros_like(state[4]), state[5]])
    rhs = np.concatenate([r + w0, PLQL - 250 * p.nu * g.ksqr * w0])
    return rhs, w0, ur


def budget_kc(g):
    """``main.kc = np.amax(grid.k1)`` (``src/Classes.py:16``), truncated as
    the slices of ``seperateModesBudgets`` take it."""
    return int(np.amax(np.fft.fftshift(np.linspace(-(g.N1 // 2), g.N1 // 2 - 1, g.N1)) * 2.0 * np.pi / g.L1))


def rhs_budgets(g, state, p, kc=None):
    """DNS with SGS budgets, ``computeRHS_BUDGETS`` (``src/RHSfunctions.py:1543-1661``):
    RHS ``= unpad_2x(PL u)``; ``PLQL u`` with the q part split at ``main.kc``
    (``seperateModesBudgets``, ``src/padding.py:81-93``).  ``rotate = 1``
    raises in the reference (an N-grid Coriolis pressure added to the 2x-grid
    ``phat``, ``:1605-1607``).

    Returns ``(rhs, PLQL, uhat_read)``; ``rhs`` is also ``main.PLu/v/w``."""
    if p.rotate == 1:
        raise ValueError("computeRHS_BUDGETS has no rotating form")
    kc = budget_kc(g) if kc is None else kc
    u, v, w = (nyquist_zero(state[i]) for i in range(3))
    PL, vel, _, _ = _pl_2x(g, pad_2x(u), pad_2x(v), pad_2x(w), p.nu, 0, p.Om)
    PLq = [separate_modes_testfilter(x, kc)[1] for x in PL]
    PLQL = _plql(g, vel, PLq)
    return np.stack([unpad_2x(x) for x in PL]), PLQL, np.stack([u, v, w])


def rhs_staumodel(g, state, p):
    """Static tau-model, ``computeRHS_staumodel`` (``src/RHSfunctions.py:366-497``):
    ``tau = max(0, tau_a + tau_b*t)``.  Returns ``(rhs, w0, uhat_read, tau)``
    with ``tau`` before the clamp (``main.tau``, ``:480``)."""
    tau = p.tau_a + p.tau_b * p.t
    r, w0, ur, _, _ = _memory_rhs(g, state, p, lambda *a: (max(0.0, tau), None))
    return r, w0, ur, tau


def test_filter_masks(g, kf):
    """``test_filter`` / ``test_filter_2x`` masks, ``src/Classes.py:131-170``."""
    f1 = (np.abs(g.k1d) < kf).astype(float)
    f2 = (np.abs(g.k2d) < kf).astype(float)
    f3 = (np.abs(g.k3d) < kf).astype(float)
    F1 = (np.abs(g.k1fd) < kf).astype(float)
    F2 = (np.abs(g.k2fd) < kf).astype(float)
    F3 = (np.abs(g.k3fd) < kf).astype(float)
    return (f1[:, None, None] * f2[None, :, None] * f3[None, None, :],
            F1[:, None, None] * F2[None, :, None] * F3[None, None, :])


def _weighted_dot(a, b, nk3):
    """``sum(a[:,:,1:nk3]*conj(b[:,:,1:nk3]*2)) + sum(a[:,:,0]*conj(b[:,:,0]))``."""
    return np.sum(a[:, :, 1:nk3] * np.conj(b[:, :, 1:nk3] * 2)) + np.sum(a[:, :, 0] * np.conj(b[:, :, 0]))


def rhs_dtaumodel(g, state, p):
    """Dynamic tau-model, ``computeRHS_Dtaumodel`` (``src/RHSfunctions.py:592-878``).

    Returns ``(rhs, w0, uhat_read, tau)``; ``tau`` is ``main.tau`` before the
    clamp (``:857-859``).  ``p.kf`` defaults to ``int(kc*2/3)``
    (``src/Classes.py:131``)."""
    kf = p.kf if p.kf is not None else int(g.kc * 2.0 / 3.0)
    G, G2 = test_filter_masks(g, kf)
    N3 = g.N3
    NNN = g.N1 * g.N2 * g.N3
    k1f, k2f, k3f = g.k1f, g.k2f, g.k3f

    def coef(u, v, w, up, vp, wp, P, phat, PLQL):
        uf, vf, wf = G * u, G * v, G * w
        ufp, vfp, wfp = pad_2x(uf), pad_2x(vf), pad_2x(wf)
        PLf, velf, Pf, phatf = _pl_2x(g, ufp, vfp, wfp, p.nu, p.rotate, p.Om)
        PLqf = [separate_modes_testfilter(x, kf)[1] for x in PLf]
        PLQLf = _plql(g, velf, PLqf)
        uu, vv, ww, uv, uw, vw = P
        fuu, fvv, fww, fuv, fuw, fvw = Pf
        # Leonard-type term (:813-819); note the "+1j*k*phat" sign
        Lu = G2 * (-1j * k1f * uu - 1j * k2f * uv - 1j * k3f * uw + 1j * k1f * phat) - \
            G2 * (-1j * k1f * fuu - 1j * k2f * fuv - 1j * k3f * fuw + 1j * k1f * phatf)
        Lv = G2 * (-1j * k1f * uv - 1j * k2f * vv - 1j * k3f * vw + 1j * k2f * phat) - \
            G2 * (-1j * k1f * fuv - 1j * k2f * fvv - 1j * k3f * fvw + 1j * k2f * phatf)
        Lw = G2 * (-1j * k1f * uw - 1j * k2f * vw - 1j * k3f * ww + 1j * k3f * phat) - \
            G2 * (-1j * k1f * fuw - 1j * k2f * fvw - 1j * k3f * fww + 1j * k3f * phatf)
        h = N3 // 2
        LE = (_weighted_dot(Lu, ufp, h) + _weighted_dot(Lv, vfp, h) + _weighted_dot(Lw, wfp, h)) / NNN
        PLQLE_filt = sum(_weighted_dot(G * PLQLf[i], x, h) for i, x in enumerate((uf, vf, wf))) / NNN
        # the reference sums the *unfiltered* PLQL here (:846-852)
        filt_PLQLE = sum(_weighted_dot(PLQL[i], x, h) for i, x in enumerate((uf, vf, wf))) / NNN
        tau = np.abs(LE) / (np.abs(PLQLE_filt) - np.abs(filt_PLQLE) + 1.0e-5)
        return max(0.0, tau), (tau, LE, PLQLE_filt, filt_PLQLE)

    r, w0, ur, _, extra = _memory_rhs(g, state, p, coef)
    return r, w0, ur, extra[0], extra


# --------------------------------------------------------------------------
# MHD (MPI solver, single rank)      PySpectral/src_MPI/RHSfunctions.py:95-175
# --------------------------------------------------------------------------
class MHDGrid:
    """Single-rank ``gridclass`` of the MPI solver (``src_MPI/Classes.py:177-236``).
    Wavenumbers are 1-D; the 2/3-rule masks follow ``:206-218`` exactly,
    including the ``int((N3/2)*2/3)`` cut along k3."""

    def __init__(self, N1, N2, N3, kc, L1=2 * np.pi, L2=2 * np.pi, L3=2 * np.pi, dx=None):
        self.N1, self.N2, self.N3 = N1, N2, N3
        self.L1, self.L2, self.L3 = L1, L2, L3
        self.k1 = np.fft.fftshift(np.linspace(-(N1 // 2), N1 // 2 - 1, N1)) * 2.0 * np.pi / L1
        self.k2 = np.fft.fftshift(np.linspace(-(N2 // 2), N2 // 2 - 1, N2)) * 2.0 * np.pi / L2
        self.k3 = np.linspace(0, N3 // 2, N3 // 2 + 1) * 2.0 * np.pi / L3
        self.ksqr = (self.k1[:, None, None] ** 2 + self.k2[None, :, None] ** 2
                     + self.k3[None, None, :] ** 2 + 1.0e-50)
        self.ksqr_i = 1.0 / self.ksqr
        self.kc = kc
        self.Delta = np.pi / kc
        dx_ = np.ones(N1)
        dy_ = np.ones(N2)
        dz_ = np.ones(N3 // 2 + 1)
        dx_[np.abs(self.k1) >= (N1 // 2) * 2.0 / 3.0 * 2.0 * np.pi / L1] = 0.0
        dy_[np.abs(self.k2) >= (N2 // 2) * 2.0 / 3.0 * 2.0 * np.pi / L2] = 0.0
        if N3 != 2:
            dz_[int((N3 // 2) * 2.0 / 3.0):] = 0.0
        self.dealias_mask = dx_[:, None, None] * dy_[None, :, None] * dz_[None, None, :]


def mhd_forcing(g, x, y, z, kf=2, f0=0.25):
    """Constant forcing of ``src_MPI/Classes.py:91-94`` (unnormalised rfftn)."""
    f = np.zeros((3, g.N1, g.N2, g.N3 // 2 + 1), dtype=complex)
    f[0] = np.fft.rfftn(f0 * np.sin(kf * x) * np.cos(kf * y) * np.cos(kf * z))
    f[1] = np.fft.rfftn(-f0 * np.cos(kf * x) * np.sin(kf * y) * np.cos(kf * z))
    return f


def rhs_mhd(g, state, nu, force=None, eta=None):
    """Incompressible MHD, ``computeRHS_MHD`` (``src_MPI/RHSfunctions.py:95-175``).

    State is ``(u, v, w, B1, B2, B3)`` as unnormalised ``rfftn`` spectra;
    ``eta`` defaults to ``nu`` (``main.lam = main.nu``, ``src_MPI/Classes.py:95``).
    Returns ``(rhs, dealiased_state)``: the reference dealiases the six fields
    in place (``:102-107``; ``dealias`` writes into its argument,
    ``src_MPI/Classes.py:262-264``)."""
    eta = nu if eta is None else eta
    D = g.dealias_mask
    s = [D * state[i] for i in range(6)]
    shape = (g.N1, g.N2, g.N3)
    u, v, w, B1, B2, B3 = (_irfftn(x, s=shape) for x in s)
    NL = [_rfftn(a * b) for a, b in ((u, u), (v, v), (w, w), (u, v), (u, w), (v, w))]
    uxB = [_rfftn(v * B3 - w * B2), _rfftn(w * B1 - u * B3), _rfftn(u * B2 - v * B1)]
    MN = [_rfftn(a * b) for a, b in ((B1, B1), (B2, B2), (B3, B3), (B1, B2), (B1, B3), (B2, B3))]
    k1 = g.k1[:, None, None]
    k2 = g.k2[None, :, None]
    k3 = g.k3[None, None, :]
    phat = _pressure(k1, k2, k3, g.ksqr_i, *NL) - _pressure(k1, k2, k3, g.ksqr_i, *MN)
    f = force if force is not None else np.zeros((3,) + g.ksqr.shape, dtype=complex)
    n0, n1, n2, n3, n4, n5 = NL
    m0, m1, m2, m3, m4, m5 = MN
    r = np.empty((6,) + g.ksqr.shape, dtype=complex)
    r[0] = D * (-1j * k1 * n0 - 1j * k2 * n3 - 1j * k3 * n4 + 1j * k1 * m0 + 1j * k2 * m3 + 1j * k3 * m4
                - 1j * k1 * phat - nu * g.ksqr * s[0] + f[0])
    r[1] = D * (-1j * k1 * n3 - 1j * k2 * n1 - 1j * k3 * n5 + 1j * k1 * m3 + 1j * k2 * m1 + 1j * k3 * m5
                - 1j * k2 * phat - nu * g.ksqr * s[1] + f[1])
    r[2] = D * (-1j * k1 * n4 - 1j * k2 * n5 - 1j * k3 * n2 + 1j * k1 * m4 + 1j * k2 * m5 + 1j * k3 * m2
                - 1j * k3 * phat - nu * g.ksqr * s[2] + f[2])
    r[3] = D * ((1j * k2 * uxB[2] - 1j * k3 * uxB[1]) - eta * g.ksqr * s[3])
    r[4] = D * ((1j * k3 * uxB[0] - 1j * k1 * uxB[2]) - eta * g.ksqr * s[4])
    r[5] = D * ((1j * k1 * uxB[1] - 1j * k2 * uxB[0]) - eta * g.ksqr * s[5])
    return r, np.stack(s)


def rhs_mpi_ns(g, state, nu, rotate=0, Om=(0.0, 0.0, 0.0), ortho=False):
    """Navier-Stokes of the MPI solver, ``computeRHS_NOSGS``
    (``src_MPI/RHSfunctions.py:22-93``): 2/3-rule masks on read and on the
    RHS, products on the N grid, Coriolis after the mask.  ``ortho``:
    ``computeRHS_Ortho`` (``:179-268``), that RHS minus the same of
    ``grid.filter(u)`` (``|k_i| < kc`` per axis, ``src_MPI/Classes.py:219-235``).
    Returns ``(rhs, dealiased_state)``."""
    D = g.dealias_mask
    k1 = g.k1[:, None, None]
    k2 = g.k2[None, :, None]
    k3 = g.k3[None, None, :]
    shape = (g.N1, g.N2, g.N3)

    def part(a):
        u, v, w = (_irfftn(x, s=shape) for x in a)
        NL = [_rfftn(x * y) for x, y in ((u, u), (v, v), (w, w), (u, v), (u, w), (v, w))]
        phat = _pressure(k1, k2, k3, g.ksqr_i, *NL)
        if rotate == 1:
            phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, a[0], a[1], a[2], Om)
        r = [D * x for x in _advection(k1, k2, k3, nu, g.ksqr, phat, NL, a[0], a[1], a[2])]
        c = _coriolis_force(a[0], a[1], a[2], Om) if rotate == 1 else None
        return r, c
    s = [D * state[i] for i in range(3)]
    r, c = part(s)
    if rotate == 1:
        r = [r[i] + c[i] for i in range(3)]
    if ortho:
        kc = g.kc
        fx = (np.abs(g.k1) < kc * 2.0 * np.pi / g.L1).astype(float)
        fy = (np.abs(g.k2) < kc * 2.0 * np.pi / g.L2).astype(float)
        fz = np.ones(g.N3 // 2 + 1)
        fz[kc:] = 0.0
        F = fx[:, None, None] * fy[None, :, None] * fz[None, None, :]
        rf, cf = part([F * x for x in s])
        r = [r[i] - rf[i] for i in range(3)]
        if rotate == 1:
            r = [r[i] - cf[i] for i in range(3)]
    return np.stack(r), np.stack(s)


def step_mpi_si(g, state, H, nu, dt, rotate=0, Om=(0.0, 0.0, 0.0)):
    """One semi-implicit step of the MPI solver's Navier-Stokes, ``advanceQ_SI``
    (``src_MPI/time_schemes.py:9-11``) with the 'Semi-Implicit' branch of
    ``computeRHS_NOSGS`` (``src_MPI/RHSfunctions.py:70-93``): H the masked
    nonlinear term (+ Coriolis),
    ``Q = (Q + dt/2 (3 H - H_old) + dt/2 (-nu k^2 u)) / (1 + nu dt/2 k^2)``.
    Returns ``(Q, H)``."""
    D = g.dealias_mask
    k1 = g.k1[:, None, None]
    k2 = g.k2[None, :, None]
    k3 = g.k3[None, None, :]
    s = [D * state[i] for i in range(3)]
    u, v, w = (_irfftn(x, s=(g.N1, g.N2, g.N3)) for x in s)
    NL = [_rfftn(x * y) for x, y in ((u, u), (v, v), (w, w), (u, v), (u, w), (v, w))]
    phat = _pressure(k1, k2, k3, g.ksqr_i, *NL)
    if rotate == 1:
        phat = phat + _coriolis_pressure(k1, k2, k3, g.ksqr_i, s[0], s[1], s[2], Om)
    n0, n1, n2, n3, n4, n5 = NL
    Hn = [D * (-1j * k1 * n0 - 1j * k2 * n3 - 1j * k3 * n4 - 1j * k1 * phat),
          D * (-1j * k1 * n3 - 1j * k2 * n1 - 1j * k3 * n5 - 1j * k2 * phat),
          D * (-1j * k1 * n4 - 1j * k2 * n5 - 1j * k3 * n2 - 1j * k3 * phat)]
    if rotate == 1:
        c = _coriolis_force(s[0], s[1], s[2], Om)
        Hn = [Hn[i] + c[i] for i in range(3)]
    Hn = np.stack(Hn)
    visc = np.stack([-nu * g.ksqr * s[i] for i in range(3)])
    Q = (state + dt / 2.0 * (3.0 * Hn - H) + dt / 2.0 * visc) / (1.0 + nu * dt / 2.0 * g.ksqr[None])
    return Q, Hn


def _mhd_nonlinear(k1, k2, k3, ksqr_i, P):
    """Nonlinear MHD operator from the nine product spectra
    P = (u_iu_j - B_iB_j for 11,22,33,12,13,23, then u x B): the momentum
    terms with the pressure projection and the induction term of
    ``src_MPI/RHSfunctions.py:117-170``, without dissipation, forcing or mask."""
    n0, n1, n2, n3, n4, n5, x0, x1, x2 = P
    ph = _pressure(k1, k2, k3, ksqr_i, n0, n1, n2, n3, n4, n5)
    return np.stack([
        -1j * k1 * n0 - 1j * k2 * n3 - 1j * k3 * n4 - 1j * k1 * ph,
        -1j * k1 * n3 - 1j * k2 * n1 - 1j * k3 * n5 - 1j * k2 * ph,
        -1j * k1 * n4 - 1j * k2 * n5 - 1j * k3 * n2 - 1j * k3 * ph,
        1j * k2 * x2 - 1j * k3 * x1,
        1j * k3 * x0 - 1j * k1 * x2,
        1j * k1 * x1 - 1j * k2 * x0])


def mhd_tmodel_memory(g, state, Ct, t, return_ql=False):
    """t-model memory term ``Ct t PLQL`` of the MHD system (no reference
    counterpart; the construction of ``computeRHS_tmodel``,
    ``src/RHSfunctions.py:240-363``, applied to ``computeRHS_MHD``,
    ``src_MPI/RHSfunctions.py:95-175``).

    The resolved set p is the 2/3-rule set of the MPI grid, q its complement.
    L(u, B) is the nonlinear MHD operator evaluated without aliasing on the
    2x grid; QL its q part; PLQL the linearisation of L about (u, B) in the
    direction QL, restricted to p:
    momentum products  u_i q_j + q_i u_j - B_i r_j - r_i B_j,
    induction products q x B + u x r, with (q, r) = QL(u, B).
    Spectra use the MPI solver's unnormalised convention on the N grid."""
    N1, N2, N3 = g.N1, g.N2, g.N3
    F1, F2, F3 = 2 * N1, 2 * N2, 2 * N3
    D = g.dealias_mask
    s = [D * state[i] for i in range(6)]
    up_scale = (F1 * F2 * F3) / (N1 * N2 * N3)

    def rows(N):  # N-grid row index -> 2x-grid row index (the N/2 row is masked anyway)
        i = np.arange(N)
        return np.where(i < N // 2, i, i + N)

    r1, r2 = rows(N1), rows(N2)

    def up(x):
        out = np.zeros((F1, F2, F3 // 2 + 1), dtype=complex)
        out[np.ix_(r1, r2, np.arange(N3 // 2 + 1))] = x
        return out

    def down(X):
        return X[np.ix_(r1, r2, np.arange(N3 // 2 + 1))]

    def phys(X):
        return _irfftn(X, s=(F1, F2, F3)) * up_scale

    def spec(a):
        return _rfftn(a) / up_scale

    K1 = (np.fft.fftfreq(F1, 1.0 / F1) * 2.0 * np.pi / g.L1)[:, None, None]
    K2 = (np.fft.fftfreq(F2, 1.0 / F2) * 2.0 * np.pi / g.L2)[None, :, None]
    K3 = (np.arange(F3 // 2 + 1) * 2.0 * np.pi / g.L3)[None, None, :]
    Ki = 1.0 / (K1 ** 2 + K2 ** 2 + K3 ** 2 + 1.0e-50)
    Dp = np.zeros((F1, F2, F3 // 2 + 1))
    Dp[np.ix_(r1, r2, np.arange(N3 // 2 + 1))] = D
    u, v, w, b1, b2, b3 = (phys(up(x)) for x in s)

    def products(u, v, w, b1, b2, b3):
        return [spec(a) for a in (u * u - b1 * b1, v * v - b2 * b2, w * w - b3 * b3, u * v - b1 * b2,
                                  u * w - b1 * b3, v * w - b2 * b3, v * b3 - w * b2, w * b1 - u * b3,
                                  u * b2 - v * b1)]

    QL = (1.0 - Dp) * _mhd_nonlinear(K1, K2, K3, Ki, products(u, v, w, b1, b2, b3))
    q1, q2, q3, r1_, r2_, r3_ = (phys(x) for x in QL)
    lin = [spec(a) for a in (
        2 * u * q1 - 2 * b1 * r1_, 2 * v * q2 - 2 * b2 * r2_, 2 * w * q3 - 2 * b3 * r3_,
        u * q2 + q1 * v - b1 * r2_ - r1_ * b2, u * q3 + q1 * w - b1 * r3_ - r1_ * b3,
        v * q3 + q2 * w - b2 * r3_ - r2_ * b3,
        (q2 * b3 - q3 * b2) + (v * r3_ - w * r2_), (q3 * b1 - q1 * b3) + (w * r1_ - u * r3_),
        (q1 * b2 - q2 * b1) + (u * r2_ - v * r1_))]
    PLQL = Dp * _mhd_nonlinear(K1, K2, K3, Ki, lin)
    mem = Ct * t * np.stack([down(x) for x in PLQL])
    return (mem, QL) if return_ql else mem


def rhs_mhd_tmodel(g, state, nu, Ct, t, force=None, eta=None):
    """``rhs_mhd`` plus the MHD t-model memory term ``mhd_tmodel_memory``."""
    r, s = rhs_mhd(g, state, nu, force=force, eta=eta)
    return r + mhd_tmodel_memory(g, state, Ct, t), s


# --------------------------------------------------------------------------
# Time stepping                         PySpectral/src/PySpec_3d.py:96-105
# --------------------------------------------------------------------------
RK4_CONST = (1.0 / 4, 1.0 / 3, 1.0 / 2, 1.0)


def advance_rk4(state, rhs_fn, dt):
    """Low-storage 4-stage scheme ``Q = Q0 + dt*c_i*RHS(Q)``,
    c = [1/4, 1/3, 1/2, 1] (``src/PySpec_3d.py:96-105``,
    ``src_MPI/time_schemes.py:2-7``).  ``rhs_fn(Q)`` returns ``(rhs, read)``
    where ``read`` is the field the RHS rebinds to ``main.uhat``; the value
    of the last stage is returned with the new state because the reference's
    per-step diagnostics read it (``src/PySpec_3d.py:129``)."""
    Q0 = state.copy()
    Q = state
    read = None
    for c in RK4_CONST:
        rhs, read = rhs_fn(Q)
        Q = Q0 + dt * c * rhs
    return Q, read


# --------------------------------------------------------------------------
# Diagnostics                          PySpectral/src/Classes.py:652-929
# --------------------------------------------------------------------------
def energy(g, uvw):
    """``computeEnergy`` (``src/Classes.py:652-659``): k3=N/2 plane excluded."""
    h = g.N3 // 2
    tot = sum(_weighted_dot(uvw[i], uvw[i], h) for i in range(3))
    return float(np.real(0.5 * tot / (g.N1 * g.N2 * g.N3)))


def energy_resolved(g, uvw):
    """``computeEnergy_resolved`` (``src/Classes.py:666-676``)."""
    return energy(g, np.stack([g.Gf * uvw[i] for i in range(3)]))


def vorticity(g, uvw):
    u, v, w = uvw
    return (1j * g.k2 * w - 1j * g.k3 * v, 1j * g.k3 * u - 1j * g.k1 * w, 1j * g.k1 * v - 1j * g.k2 * u)


def enstrophy(g, uvw):
    """``computeEnstrophy`` (``src/Classes.py:733-744``)."""
    h = g.N3 // 2
    om = vorticity(g, uvw)
    tot = sum(_weighted_dot(x, x, h) for x in om)
    return float(np.real(0.5 * tot / (g.N1 * g.N2 * g.N3)))


def all_stats(g, uvw, nu):
    """``computeAllStats`` (``src/Classes.py:701-731``): returns
    (enstrophy, energy, dissipation, lambda_k, tau_k, Re_lambda)."""
    ens = enstrophy(g, uvw)
    en = energy(g, uvw)
    diss = 2 * ens * nu
    lambda_k = (nu ** 3 / diss) ** 0.25
    tau_k = (nu / diss) ** 0.5
    Re_lambda = en * np.sqrt(20.0 / (3.0 * nu * diss))
    return ens, en, diss, lambda_k, tau_k, Re_lambda


def spectrum(g, uvw, filtered=False):
    """``computeSpectrum`` (``src/Classes.py:762-797``) / ``computeSpectrum_resolved``
    (``:825-844``).  Shell index ``int8(rint(|k|))`` with NumPy negative-index
    wrap (the reference's int8 cast), k3=N/2 plane excluded.  Returns
    ``(kdata, spectrum[kmax+1, 3])`` (complex, like the reference)."""
    N1, N2, N3 = g.N1, g.N2, g.N3
    h = N3 // 2
    if filtered:
        uvw = np.stack([g.Gf * uvw[i] for i in range(3)])
    ks = ((g.k1 * g.L1 / (2 * np.pi)) ** 2 + (g.k2 * g.L2 / (2 * np.pi)) ** 2
          + (g.k3 * g.L3 / (2 * np.pi)) ** 2)
    km = np.rint(np.sqrt(ks[:, :, 1:h]))
    k0 = np.rint(np.sqrt(ks[:, :, 0]))
    kmax = int(np.round(np.amax(km)))
    spec = np.zeros((kmax + 1, 3), dtype=complex)
    bm = km.astype(np.int64).astype(np.int8).ravel()
    b0 = k0.astype(np.int64).astype(np.int8).ravel()
    for i in range(3):
        np.add.at(spec[:, i], bm, (2 * uvw[i][:, :, 1:h] * np.conj(uvw[i][:, :, 1:h])).ravel())
        np.add.at(spec[:, i], b0, (uvw[i][:, :, 0] * np.conj(uvw[i][:, :, 0])).ravel())
    kdata = np.linspace(0, kmax, kmax + 1)
    return kdata, spec / (N1 * N2 * N3)


def transfer(g, uvw, filtered=False, w0=None, two_d=False):
    """``computeTransfer`` (``src/Classes.py:988-1040``): energy transfer
    spectrum sum_i conj(u_i) (-i k_j (u_i u_j)^ - i k_i p^), from the state with
    its Nyquist modes zeroed (``unpad(pad(.))``), binned like ``spectrum``
    (k3 = N/2 excluded, k3 > 0 twice) over N1 N2 N3.  ``filtered``:
    ``computeTransfer_resolved`` (``:1093-1150``), the same of Gf u.  ``w0``:
    ``computeTransfer_SGS`` (``:1206-1239``), Re sum_i conj(Gf u_i) w0_i.
    ``two_d``: the ``*_2D`` variants (``:1043-1092``, ``:1152-1205``,
    ``:1241-1270``): the k3 = 0 plane only, binned by ``rint(sqrt(k1^2+k2^2))``,
    the u and v components only, weight 1.
    Returns ``(kdata, T[kmax+1])`` (complex, like the reference)."""
    N1, N2, N3 = g.N1, g.N2, g.N3
    h = N3 // 2
    if filtered or w0 is not None:
        uvw = [g.Gf * uvw[i] for i in range(3)]
    u, v, w = (nyquist_zero(uvw[i]) for i in range(3))
    if w0 is not None:
        rc = [np.real(np.conj(a) * b) for a, b in zip((u, v, w), w0)]
    else:
        P = _products_32(g, u, v, w)
        uu, vv, ww, uv, uw, vw = P
        k1, k2, k3 = g.k1, g.k2, g.k3
        phat = _pressure(k1, k2, k3, g.ksqr_i, *P)
        rc = [np.conj(u) * (-1j * k1 * uu - 1j * k2 * uv - 1j * k3 * uw - 1j * k1 * phat),
              np.conj(v) * (-1j * k1 * uv - 1j * k2 * vv - 1j * k3 * vw - 1j * k2 * phat),
              np.conj(w) * (-1j * k1 * uw - 1j * k2 * vw - 1j * k3 * ww - 1j * k3 * phat)]
    if two_d:
        kh = np.rint(np.sqrt(g.k1 ** 2 + g.k2 ** 2)[:, :, 0])
        kmax = int(np.round(np.amax(kh)))
        out = np.zeros(kmax + 1, dtype=complex)
        for i in range(2):
            np.add.at(out, kh.astype(np.int64).astype(np.int8).ravel(), rc[i][:, :, 0].ravel())
        return np.linspace(0, kmax, kmax + 1), out / (N1 * N2 * N3)
    r = (rc[0] + rc[1] + rc[2]).astype(complex)
    ks = ((g.k1 * g.L1 / (2 * np.pi)) ** 2 + (g.k2 * g.L2 / (2 * np.pi)) ** 2
          + (g.k3 * g.L3 / (2 * np.pi)) ** 2)
    km = np.rint(np.sqrt(ks[:, :, 1:h]))
    k0 = np.rint(np.sqrt(ks[:, :, 0]))
    kmax = int(np.round(np.amax(km)))
    out = np.zeros(kmax + 1, dtype=complex)
    np.add.at(out, km.astype(np.int64).astype(np.int8).ravel(), (2 * r[:, :, 1:h]).ravel())
    np.add.at(out, k0.astype(np.int64).astype(np.int8).ravel(), r[:, :, 0].ravel())
    return np.linspace(0, kmax, kmax + 1), out / (N1 * N2 * N3)


def compute_dt(g, uvw, cfl, nu, dt_prev):
    """``compute_dt`` (``src/Classes.py:687-698``).  ``cfl <= 0`` means a fixed
    ``dt = -cfl``."""
    if cfl > 0:
        n = math.sqrt(g.N1 * g.N2 * g.N3)
        s = (g.N1, g.N2, g.N3)
        u, v, w = (np.fft.irfftn(uvw[i], s=s, axes=(0, 1, 2)) * n for i in range(3))
        max_vel = np.amax(np.abs(u) / g.dx + np.abs(v) / g.dy + np.abs(w) / g.dz)
        dt = cfl / (max_vel + 1e-10)
        if nu > 0:
            dt = min(dt, 0.634 / (1.0 / g.dx ** 2 + 1.0 / g.dy ** 2 + 1.0 / g.dz ** 2) / nu * cfl / 1.35)
        return dt
    return -cfl


def sgs_dns(g, uvw):
    """``computeSGS_DNS`` (``src/Classes.py:861-929``): sharp-cutoff SGS stress
    ``tau_ij = Gf*(u_i u_j)^ - (Gf u_i Gf u_j)^`` and its projected divergence.
    Returns ``(w0[3], tauhat[6])``."""
    s = scale_32(g)
    u, v, w = uvw
    uf, vf, wf = g.Gf * u, g.Gf * v, g.Gf * w
    r = [ifft32(g, pad(x) * s) for x in (u, v, w)]
    rf = [ifft32(g, pad(x) * s) for x in (uf, vf, wf)]
    pairs = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))
    full = [unpad(fft32(r[a] * r[b])) for a, b in pairs]
    filt = [unpad(fft32(rf[a] * rf[b])) for a, b in pairs]
    tau = [g.Gf * full[i] - filt[i] for i in range(6)]
    return _sgs_divergence(g, tau), np.stack(tau)


def mhd_energy(g, fields3):
    """``computeEnergy`` / ``computeMHDEnergy`` of the MPI solver
    (``src_MPI/Classes.py:269-303``): normalised by (N1 N2 N3)^2."""
    h = g.N3 // 2
    tot = sum(_weighted_dot(fields3[i], fields3[i], h) for i in range(3))
    return float(np.real(0.5 * tot)) / (g.N1 * g.N2 * g.N3) ** 2


def mhd_spectrum(g, fields3):
    """``computeSpectrum`` / ``computeMHDSpectrum`` of the MPI solver
    (``src_MPI/Classes.py:370-448``): int16 shells, k3=N/2 included with
    weight 2, normalised by (N1 N2 N3)^2."""
    N1, N2, N3 = g.N1, g.N2, g.N3
    k1 = (g.k1 * g.L1 / (2 * np.pi))[:, None, None]
    k2 = (g.k2 * g.L2 / (2 * np.pi))[None, :, None]
    k3 = (g.k3 * g.L3 / (2 * np.pi))[None, None, :]
    kmag = np.sqrt(k1 ** 2 + k2 ** 2 + k3 ** 2)
    E = sum(np.real(x * np.conj(x)) for x in fields3)
    E = E.copy()
    E[:, :, 1:] *= 2.0
    kmax = int(np.round(np.sqrt((N1 // 2) ** 2 + (N2 // 2) ** 2 + (N3 // 2) ** 2)))
    bins = np.round(kmag).astype(np.int16).astype(np.int64).ravel()
    spec = np.bincount(bins, E.ravel(), minlength=kmax + 1)[:kmax + 1]
    return np.linspace(0, kmax, kmax + 1), spec / (N1 * N2 * N3) ** 2


def cross_helicity(g, uvw, B):
    """Cross-helicity ``H_c = <u.B>`` with the MPI solver's energy weighting and
    normalisation (no reference counterpart; defined like ``src_MPI/Classes.py:269-285``)."""
    h = g.N3 // 2
    tot = sum(_weighted_dot(uvw[i], B[i], h) for i in range(3))
    return float(np.real(tot)) / (g.N1 * g.N2 * g.N3) ** 2


# --------------------------------------------------------------------------
# Initial conditions
# --------------------------------------------------------------------------
def periodic_coords(N, L=2 * np.pi):
    """Exactly periodic grid ``x_i = L*i/N`` in the reference's meshgrid order
    (``run/TGV_Validate100/inputfile.py:31-38`` uses an off-grid linspace)."""
    a = np.arange(N) * (L / N)
    y, x, z = np.meshgrid(a, a, a)
    return x, y, z


def tgv_state(N, variant="sin"):
    """Taylor-Green vortex, ``uhat = rfftn(u)/sqrt(N^3)``
    (``run/TGV_Validate100/inputfile.py:38-44``).  ``variant="sin"`` is
    u=(sin x cos y cos z, -cos x sin y cos z, 0); ``"cos"`` the reference
    script's (cos x sin y cos z, -sin x cos y cos z, 0)."""
    x, y, z = periodic_coords(N)
    if variant == "sin":
        u = np.sin(x) * np.cos(y) * np.cos(z)
        v = -np.cos(x) * np.sin(y) * np.cos(z)
    else:
        u = np.cos(x) * np.sin(y) * np.cos(z)
        v = -np.sin(x) * np.cos(y) * np.cos(z)
    w = np.zeros_like(u)
    n = np.sqrt(N ** 3)
    return np.stack([np.fft.rfftn(u) / n, np.fft.rfftn(v) / n, np.fft.rfftn(w) / n])


def spectrum_k4(k, k0=4.0, u0=1.0):
    """E(k) = 16 sqrt(2/pi) u0^2 k^4 / k0^5 exp(-2 (k/k0)^2)."""
    return 16.0 * np.sqrt(2.0 / np.pi) * u0 ** 2 * k ** 4 / k0 ** 5 * np.exp(-2.0 * (k / k0) ** 2)


def isotropic_phases(N, seed):
    """Seeded phases theta1, theta2, phi drawn as in
    ``run/HIT/MansourWray/inputfile.py:72-75`` (NumPy legacy seeding)."""
    rs = np.random.RandomState(seed)
    sh = (N, N, N // 2 + 1)
    th1 = rs.rand(*sh) * 2.0 * np.pi
    th2 = rs.rand(*sh) * 2.0 * np.pi
    phi = rs.rand(*sh) * 2.0 * np.pi
    return th1, th2, phi


def isotropic_state(N, seed, k0=4.0, u0=1.0, L=2 * np.pi, phases=None, normalise="sqrtN3"):
    """Random-phase solenoidal field from E(k) by the Craya-Herring construction
    of ``run/HIT/MansourWray/inputfile.py:52-95``, with the spectrum
    :func:`spectrum_k4`.  The raw construction is not Hermitian on the k3=0
    plane, so it is symmetrised by a c2r/r2c round trip (as the MPI solver's
    ``initDomain='Fourier'`` does, ``src_MPI/Classes.py:33-45``) and then
    projected divergence-free.  ``normalise="sqrtN3"`` gives the serial
    solver's ``uhat = rfftn(u)/sqrt(N^3)``; ``"none"`` the MPI solver's
    unnormalised spectra."""
    th1, th2, phi = phases if phases is not None else isotropic_phases(N, seed)
    k1 = np.fft.fftshift(np.linspace(-(N // 2), N // 2 - 1, N))
    k3 = np.linspace(0, N // 2, N // 2 + 1)
    K2, K1, K3 = np.meshgrid(k1, k1, k3)
    ksqr = K1 ** 2 + K2 ** 2 + K3 ** 2
    kmag = np.sqrt(ksqr) + 1e-30
    E = spectrum_k4(np.sqrt(ksqr), k0, u0)
    alpha = np.sqrt(E / (4.0 * np.pi * ksqr + 1e-30)) * np.exp(1j * th1) * np.cos(phi)
    beta = np.sqrt(E / (4.0 * np.pi * ksqr + 1e-30)) * np.exp(1j * th2) * np.sin(phi)
    tp = 2.0 * np.pi / L
    kperp = np.sqrt(K1 ** 2 + K2 ** 2)
    uh = (alpha * kmag * K2 * tp + beta * K1 * tp * K3 * tp) / (kmag * kperp + 1e-30)
    vh = (-alpha * kmag * K1 * tp + beta * K2 * tp * K3 * tp) / (kmag * kperp + 1e-30)
    wh = -beta * kperp / kmag
    n3 = N ** 3
    st = np.stack([uh, vh, wh]) * np.sqrt(n3)
    # Hermitian symmetrisation by a round trip (unit-normalised irfftn/rfftn)
    st = np.stack([np.fft.rfftn(np.fft.irfftn(st[i], s=(N, N, N), axes=(0, 1, 2))) for i in range(3)])
    # divergence-free projection
    kk = (K1 * tp, K2 * tp, K3 * tp)
    ks = kk[0] ** 2 + kk[1] ** 2 + kk[2] ** 2 + 1e-50
    div = (kk[0] * st[0] + kk[1] * st[1] + kk[2] * st[2]) / ks
    st = np.stack([st[i] - kk[i] * div for i in range(3)])
    if normalise == "none":
        return st * np.sqrt(n3)
    return st


# ---- slab-decomposed transforms of the MPI solver ---------------------------
# FFTclass.myifft3D / myfft3D, src_MPI/Classes.py:244-258, split at the
# Alltoall into the two local halves one rank computes.  A rank holds the x
# slab (Npx, N2, N3/2+1) of the spectra and the y slab (N1, Npy, N3) of the
# physical field; blocks are exchanged so that block p of a rank's send
# buffer becomes block (this rank) of rank p's receive buffer.  The whole
# 1/(N1 N2 N3) of numpy's ifft (axis 1) and irfft2 (axes 0, 2) is applied in
# the second inverse half, the y half being an unnormalised inverse DFT (the
# two forms are equal up to round-off).

def slab_ifft_y(uhat, P):
    """x slab (Npx, N2, K) -> send blocks (P, Npx, N2/P, K): inverse DFT along y
    (src_MPI/Classes.py:245-246; the reshape/rollaxis of :246)."""
    Npx, N2, K = uhat.shape
    t = np.fft.ifft(uhat, axis=1) * N2
    return np.ascontiguousarray(t.reshape(Npx, P, N2 // P, K).transpose(1, 0, 2, 3))


def slab_ifft_xz(recv, N2, N3):
    """received blocks (P, Npx, Npy, K) = (N1, Npy, K) -> y slab (N1, Npy, N3):
    irfft2 over x and z (src_MPI/Classes.py:248), times 1/N2."""
    P, Npx, Npy, K = recv.shape
    return np.fft.irfft2(recv.reshape(P * Npx, Npy, K), s=(P * Npx, N3), axes=(0, 2)) / N2


def slab_fft_xz(u):
    """y slab (N1, Npy, N3) -> send (N1, Npy, N3/2+1): rfft2 over x and z
    (src_MPI/Classes.py:252)."""
    return np.fft.rfft2(u, axes=(0, 2))


def slab_fft_y(recv):
    """received blocks (P, Npx, Npy, K) -> x slab (Npx, P Npy, K): the
    rollaxis/reshape of src_MPI/Classes.py:254, then the DFT along y (:255)."""
    P, Npx, Npy, K = recv.shape
    return np.fft.fft(recv.transpose(1, 0, 2, 3).reshape(Npx, P * Npy, K), axis=1)


def slab_alltoall(sends):
    """The Alltoall of one transform over all ranks' send buffers (lists of
    (P, ...) arrays): rank r receives block r of every rank's send, in rank order."""
    P = len(sends)
    return [np.stack([sends[p][r] for p in range(P)]) for r in range(P)]
