"""ctypes binding of the C ABI declared in ``include/pyspectral_b200.h``.

Only plain pointers and sizes cross the boundary.  Tensors are passed as
``data_ptr()`` values; the context queues its work on the caller's current
torch CUDA stream.  There is no CPU fallback: if the shared library is missing
or no GPU is visible every call raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyspectral_b200.so")

PSB_OK = 0
PSB_ERR_NONFINITE = 6
DNS, SMAG, TMODEL, TAU_STATIC, TAU_DYNAMIC, MHD, LEARNED, MHD_TMODEL, DSMAG, CM1, BUDGETS, FM1, ORTHO = (
    0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12)
MPI_DNS, MPI_ORTHO = 13, 14
FM2 = 15
ACT_GELU, ACT_RELU = 0, 1  # hidden activation of the learned closure's MLP
NORM_SERIAL, NORM_MPI, FILTER_GF, TRANSFER_2D = 0, 1, 2, 4

EXPORTS = (
    "psb_ctx_create", "psb_ctx_destroy", "psb_ctx_set_stream", "psb_last_error", "psb_create_error",
    "psb_rhs", "psb_step_rk4", "psb_step_si", "psb_prepare", "psb_energy", "psb_enstrophy", "psb_cross_helicity",
    "psb_spectrum", "psb_spectrum_nbins", "psb_transfer", "psb_spectrum_mpi", "psb_cfl_dt", "psb_sgs_dns",
    "psb_fft_r2c", "psb_fft_c2r", "psb_slab_ifft_y", "psb_slab_ifft_xz", "psb_slab_fft_xz",
    "psb_slab_fft_y", "psb_check_finite", "psb_launch_count", "psb_timing_enable",
    "psb_timing_count", "psb_timing_get", "psb_rhs_dns_noalloc", "psb_mlp_sizes", "psb_mlp_forward",
    "psb_mlp_forward_tc",
    "psb_mlp_grad", "psb_mlp_adam", "psb_physical_fields", "psb_products", "psb_spectral_resample",
    "psb_batch_create", "psb_batch_set_run", "psb_batch_autotune", "psb_batch_step_rk4", "psb_batch_shape",
    "psb_batch_destroy", "psb_autotune", "psb_tuned_shape", "psb_autotune_clear", "psb_set_tuned_shape",
    "psb_ctx_set_tma", "psb_ctx_set_zrr", "psb_device_status", "psb_ensemble_create", "psb_ensemble_step_rk4", "psb_ensemble_status",
    "psb_ensemble_destroy",
)


class Grid(ctypes.Structure):
    _fields_ = [("N1", ctypes.c_int), ("N2", ctypes.c_int), ("N3", ctypes.c_int),
                ("L1", ctypes.c_double), ("L2", ctypes.c_double), ("L3", ctypes.c_double),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("kc", ctypes.c_int)]


class Params(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_double), ("eta", ctypes.c_double), ("t", ctypes.c_double),
                ("dt", ctypes.c_double), ("Ct", ctypes.c_double), ("tau_a", ctypes.c_double),
                ("tau_b", ctypes.c_double), ("kf", ctypes.c_int), ("rotate", ctypes.c_int),
                ("Om1", ctypes.c_double), ("Om2", ctypes.c_double), ("Om3", ctypes.c_double),
                ("force", ctypes.c_void_p), ("mlp_params", ctypes.c_void_p), ("mlp_norm", ctypes.c_void_p),
                ("les_delta", ctypes.c_double), ("mlp_act", ctypes.c_int), ("mlp_hidden", ctypes.c_int),
                ("fm_dt0", ctypes.c_double), ("fm_nsub", ctypes.c_int), ("fm_dt1", ctypes.c_double)]


_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m pyspectral_b200.build`")
    lib = ctypes.CDLL(path)
    vp, ip, dp, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_int
    d = ctypes.c_double
    sig = {
        "psb_ctx_create": ([ctypes.POINTER(Grid), i, i, ctypes.POINTER(vp)], i),
        "psb_ctx_destroy": ([vp], i),
        "psb_ctx_set_stream": ([vp, vp], i),
        "psb_last_error": ([vp], ctypes.c_char_p),
        "psb_create_error": ([], ctypes.c_char_p),
        "psb_rhs": ([vp, i, vp, vp, vp, vp, ctypes.POINTER(Params), dp], i),
        "psb_step_rk4": ([vp, i, vp, vp, vp, ctypes.POINTER(Params), i], i),
        "psb_step_si": ([vp, vp, vp, vp, ctypes.POINTER(Params), i], i),
        "psb_prepare": ([vp, i], i),
        "psb_energy": ([vp, vp, i, dp], i),
        "psb_enstrophy": ([vp, vp, i, dp], i),
        "psb_cross_helicity": ([vp, vp, vp, i, dp], i),
        "psb_spectrum": ([vp, vp, i, dp, i], i),
        "psb_spectrum_nbins": ([vp, i, ip], i),
        "psb_spectrum_mpi": ([vp, vp, dp, i], i),
        "psb_transfer": ([vp, vp, vp, i, dp, i], i),
        "psb_cfl_dt": ([vp, vp, d, d, dp], i),
        "psb_sgs_dns": ([vp, vp, vp, vp], i),
        "psb_fft_r2c": ([vp, vp, vp, i], i),
        "psb_fft_c2r": ([vp, vp, vp, i], i),
        "psb_slab_ifft_y": ([vp, i, vp, vp], i),
        "psb_slab_ifft_xz": ([vp, i, vp, vp], i),
        "psb_slab_fft_xz": ([vp, i, vp, vp], i),
        "psb_slab_fft_y": ([vp, i, vp, vp], i),
        "psb_check_finite": ([vp, vp, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong)], i),
        "psb_launch_count": ([vp, ctypes.POINTER(ctypes.c_ulonglong)], i),
        "psb_timing_enable": ([vp, i], i),
        "psb_timing_count": ([vp, ip], i),
        "psb_timing_get": ([vp, i, ctypes.c_char_p, i, dp, dp], i),
        "psb_rhs_dns_noalloc": ([vp, vp, vp, ctypes.POINTER(Params)], i),
        "psb_autotune": ([vp, i, vp, ctypes.POINTER(Params)], i),
        "psb_tuned_shape": ([vp, i, i, ip, ip, i], i),
        "psb_autotune_clear": ([vp, i], i),
        "psb_set_tuned_shape": ([vp, i, i, i, ip, i], i),
        "psb_ctx_set_tma": ([vp, i], i),
        "psb_ctx_set_zrr": ([vp, i], i),
        "psb_device_status": ([vp, ip], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def make_params(nu=0.0, eta=-1.0, t=0.0, dt=0.0, Ct=0.1, tau_a=0.0, tau_b=0.0, kf=0, rotate=0,
                Om=(0.0, 0.0, 0.0), force=None, mlp_params=None, mlp_norm=None, les_delta=0.0,
                mlp_act=0, mlp_hidden=0, fm_dt0=0.0, fm_nsub=0, fm_dt1=0.0) -> Params:
    return Params(float(nu), float(eta), float(t), float(dt), float(Ct), float(tau_a), float(tau_b), int(kf),
                  int(rotate), float(Om[0]), float(Om[1]), float(Om[2]), force, mlp_params, mlp_norm,
                  float(les_delta), int(mlp_act), int(mlp_hidden), float(fm_dt0), int(fm_nsub), float(fm_dt1))


def state_fields(closure, params):
    """Fields of the state (and RHS) of `closure`: 3 velocity components plus
    the closure's memory variables or magnetic field."""
    if closure in (MHD, MHD_TMODEL, CM1):
        return 6
    if closure == FM1:
        return 3 + 3 * max(1, params.fm_nsub)
    if closure == FM2:
        return 3 + 6 * max(1, params.fm_nsub)
    return 3


class Context:
    """Owns one ``psb_ctx`` (grid + precision + device)."""

    def __init__(self, N1, N2, N3, L=(2 * 3.141592653589793,) * 3, d=None, kc=None, precision=64, device=0):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("pyspectral_b200 needs a CUDA device; none is visible")
        self.lib = load()
        L1, L2, L3 = L
        if d is None:
            d = (L1 / N1, L2 / N2, L3 / N3)
        self.grid = Grid(N1, N2, N3, L1, L2, L3, d[0], d[1], d[2], N1 // 2 if kc is None else int(kc))
        self.precision = precision
        self.device = device
        h = ctypes.c_void_p()
        st = self.lib.psb_ctx_create(ctypes.byref(self.grid), precision, device, ctypes.byref(h))
        if st != PSB_OK:
            raise RuntimeError(f"psb_ctx_create failed ({st}): {self.lib.psb_create_error().decode()}")
        self.h = h
        self.N1, self.N2, self.N3 = N1, N2, N3

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                self.lib.psb_ctx_destroy(h)
            except Exception:
                pass
            self.h = None

    def check(self, st: int, what: str):
        if st != PSB_OK:
            raise RuntimeError(f"{what} failed ({st}): {self.lib.psb_last_error(self.h).decode()}")

    def bind_stream(self):
        import torch
        s = torch.cuda.current_stream(self.device).cuda_stream
        self.lib.psb_ctx_set_stream(self.h, ctypes.c_void_p(s))

    # -- tensor helpers
    def _ptr(self, t, ncomplex=None):
        import torch
        if t is None:
            return None
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("tensors passed to pyspectral_b200 must be contiguous CUDA tensors")
        want = torch.complex128 if self.precision == 64 else torch.complex64
        if t.is_complex() and t.dtype != want:
            raise ValueError(f"expected {want}, got {t.dtype}")
        if ncomplex is not None and t.numel() < ncomplex:
            raise ValueError("tensor too small for the grid")
        return ctypes.c_void_p(t.data_ptr())

    def spec_numel(self, nfields):
        return nfields * self.N1 * self.N2 * (self.N3 // 2 + 1)

    def rhs(self, closure, state, rhs, params, w0=None, read_out=None):
        nf = state_fields(closure, params)
        self.bind_stream()
        tau = ctypes.c_double(0.0)
        st = self.lib.psb_rhs(self.h, closure, self._ptr(state, self.spec_numel(nf)),
                              self._ptr(rhs, self.spec_numel(nf)), self._ptr(w0), self._ptr(read_out),
                              ctypes.byref(params), ctypes.byref(tau))
        self.check(st, "psb_rhs")
        return tau.value

    def step_si(self, state, H, params, nsteps=1, read_out=None):
        """Semi-implicit steps of the MPI solver's Navier-Stokes (3 fields; H in/out)."""
        self.bind_stream()
        st = self.lib.psb_step_si(self.h, self._ptr(state, self.spec_numel(3)), self._ptr(H, self.spec_numel(3)),
                                  self._ptr(read_out), ctypes.byref(params), int(nsteps))
        self.check(st, "psb_step_si")

    def step(self, closure, state, params, nsteps=1, comp=None, read_out=None):
        nf = state_fields(closure, params)
        self.bind_stream()
        st = self.lib.psb_step_rk4(self.h, closure, self._ptr(state, self.spec_numel(nf)), self._ptr(comp),
                                   self._ptr(read_out), ctypes.byref(params), int(nsteps))
        self.check(st, "psb_step_rk4")

    def prepare(self, closure):
        self.check(self.lib.psb_prepare(self.h, closure), "psb_prepare")

    def energy(self, f3, flags=0):
        self.bind_stream()
        out = ctypes.c_double()
        self.check(self.lib.psb_energy(self.h, self._ptr(f3, self.spec_numel(3)), flags, ctypes.byref(out)),
                   "psb_energy")
        return out.value

    def enstrophy(self, f3, flags=0):
        self.bind_stream()
        out = ctypes.c_double()
        self.check(self.lib.psb_enstrophy(self.h, self._ptr(f3, self.spec_numel(3)), flags, ctypes.byref(out)),
                   "psb_enstrophy")
        return out.value

    def cross_helicity(self, u3, b3, flags=NORM_MPI):
        self.bind_stream()
        out = ctypes.c_double()
        self.check(self.lib.psb_cross_helicity(self.h, self._ptr(u3), self._ptr(b3), flags, ctypes.byref(out)),
                   "psb_cross_helicity")
        return out.value

    def spectrum(self, f3, flags=0):
        import numpy as np
        self.bind_stream()
        nb = ctypes.c_int()
        self.check(self.lib.psb_spectrum_nbins(self.h, flags, ctypes.byref(nb)), "psb_spectrum_nbins")
        out = np.zeros((nb.value, 3), dtype=np.float64)
        self.check(self.lib.psb_spectrum(self.h, self._ptr(f3), flags,
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nb.value),
                   "psb_spectrum")
        return out

    def transfer(self, f3, w0=None, flags=0):
        """Complex transfer spectrum (kmax+1 bins) of the 3 fields f3; flags
        FILTER_GF: of the Gf-filtered fields; TRANSFER_2D: the k3 = 0 plane
        binned by |k_h| (u and v); w0: the SGS transfer with w0."""
        import numpy as np
        self.bind_stream()
        nb = ctypes.c_int()
        self.check(self.lib.psb_spectrum_nbins(self.h, int(flags) & TRANSFER_2D, ctypes.byref(nb)),
                   "psb_spectrum_nbins")
        out = np.zeros((nb.value, 2), dtype=np.float64)
        self.check(self.lib.psb_transfer(self.h, self._ptr(f3), self._ptr(w0), int(flags),
                                         out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nb.value),
                   "psb_transfer")
        return out[:, 0] + 1j * out[:, 1]

    def spectrum_mpi(self, f3):
        import numpy as np
        self.bind_stream()
        N1, N2, N3 = self.N1, self.N2, self.N3
        kmax = int(np.round(np.sqrt((N1 // 2) ** 2 + (N2 // 2) ** 2 + (N3 // 2) ** 2)))
        out = np.zeros(kmax + 1, dtype=np.float64)
        self.check(self.lib.psb_spectrum_mpi(self.h, self._ptr(f3), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                             kmax + 1), "psb_spectrum_mpi")
        return out

    def cfl_dt(self, f3, cfl, nu):
        self.bind_stream()
        out = ctypes.c_double()
        self.check(self.lib.psb_cfl_dt(self.h, self._ptr(f3), float(cfl), float(nu), ctypes.byref(out)),
                   "psb_cfl_dt")
        return out.value

    def sgs_dns(self, f3, w0, tau6=None):
        self.bind_stream()
        self.check(self.lib.psb_sgs_dns(self.h, self._ptr(f3), self._ptr(w0), self._ptr(tau6)), "psb_sgs_dns")

    def r2c(self, phys, spec, nfields):
        self.bind_stream()
        self.check(self.lib.psb_fft_r2c(self.h, self._ptr(phys), self._ptr(spec), int(nfields)), "psb_fft_r2c")

    def c2r(self, spec, phys, nfields):
        self.bind_stream()
        self.check(self.lib.psb_fft_c2r(self.h, self._ptr(spec), self._ptr(phys), int(nfields)), "psb_fft_c2r")

    # slab-decomposed transforms (one rank of nprocs; the caller exchanges the blocks)
    def slab_ifft_y(self, nprocs, uhat, send):
        self.bind_stream()
        self.check(self.lib.psb_slab_ifft_y(self.h, int(nprocs), self._ptr(uhat), self._ptr(send)), "psb_slab_ifft_y")

    def slab_ifft_xz(self, nprocs, recv, u):
        self.bind_stream()
        self.check(self.lib.psb_slab_ifft_xz(self.h, int(nprocs), self._ptr(recv), self._ptr(u)), "psb_slab_ifft_xz")

    def slab_fft_xz(self, nprocs, u, send):
        self.bind_stream()
        self.check(self.lib.psb_slab_fft_xz(self.h, int(nprocs), self._ptr(u), self._ptr(send)), "psb_slab_fft_xz")

    def slab_fft_y(self, nprocs, recv, uhat):
        self.bind_stream()
        self.check(self.lib.psb_slab_fft_y(self.h, int(nprocs), self._ptr(recv), self._ptr(uhat)), "psb_slab_fft_y")

    def autotune(self, closure, state, params):
        """Pick the fastest launch shapes of closure's RHS passes on `state`
        (unchanged) and use them for this closure from now on."""
        self.bind_stream()
        self.check(self.lib.psb_autotune(self.h, closure, self._ptr(state), ctypes.byref(params)), "psb_autotune")

    def tuned_shapes(self, closure):
        out = []
        for p in range(5):
            t = ctypes.c_int()
            rad = (ctypes.c_int * 12)()
            self.check(self.lib.psb_tuned_shape(self.h, closure, p, ctypes.byref(t), rad, 12), "psb_tuned_shape")
            out.append({"tile": t.value, "radices": [x for x in rad if x]})
        return out

    def autotune_clear(self, closure):
        self.check(self.lib.psb_autotune_clear(self.h, closure), "psb_autotune_clear")

    def set_tuned_shapes(self, closure, shapes):
        """Use the given launch shapes ([{"tile": t, "radices": [...]}] per pass,
        as tuned_shapes() returns them; None entries keep a pass's shape)."""
        for p, sh in enumerate(shapes):
            if sh is None:
                continue
            rad = list(sh["radices"])
            arr = (ctypes.c_int * max(1, len(rad)))(*rad)
            self.check(self.lib.psb_set_tuned_shape(self.h, closure, p, int(sh["tile"]), arr, len(rad)),
                       "psb_set_tuned_shape")

    def set_tma(self, on: bool):
        """Stage eligible pass inputs with bulk tensor copies (default) or plain loads."""
        self.check(self.lib.psb_ctx_set_tma(self.h, 1 if on else 0), "psb_ctx_set_tma")

    def set_zrr(self, on: bool):
        """Register-direct z pass for two-pass (R1, 16) schedules (default) or the
        shared-memory z pass."""
        self.check(self.lib.psb_ctx_set_zrr(self.h, 1 if on else 0), "psb_ctx_set_zrr")

    def device_status(self):
        """0, or 1 if a bounded wait inside one of this context's kernels gave up
        since the last call (cleared on read; synchronises the stream)."""
        self.bind_stream()
        st = ctypes.c_int()
        self.check(self.lib.psb_device_status(self.h, ctypes.byref(st)), "psb_device_status")
        return st.value

    def launch_count(self):
        n = ctypes.c_ulonglong()
        self.check(self.lib.psb_launch_count(self.h, ctypes.byref(n)), "psb_launch_count")
        return n.value

    def timing(self, on: bool):
        self.check(self.lib.psb_timing_enable(self.h, 1 if on else 0), "psb_timing_enable")

    def timing_records(self):
        """[(kernel name, device ms, compulsory bytes)] of the timed launches."""
        n = ctypes.c_int()
        self.check(self.lib.psb_timing_count(self.h, ctypes.byref(n)), "psb_timing_count")
        out = []
        buf = ctypes.create_string_buffer(128)
        ms, by = ctypes.c_double(), ctypes.c_double()
        for i in range(n.value):
            self.check(self.lib.psb_timing_get(self.h, i, buf, 128, ctypes.byref(ms), ctypes.byref(by)),
                       "psb_timing_get")
            out.append((buf.value.decode(), ms.value, by.value))
        return out

    def count_nonfinite(self, t):
        self.bind_stream()
        n = ctypes.c_longlong()
        st = self.lib.psb_check_finite(self.h, self._ptr(t), t.numel(), ctypes.byref(n))
        if st not in (PSB_OK, PSB_ERR_NONFINITE):
            self.check(st, "psb_check_finite")
        return n.value
