"""Generate the golden fixtures under tests/golden/ from the reference itself.

Run in a container that has the PySpectral sources, naming their checkout
(the directory that holds ``PySpectral/``) by argument or by the
``PYSPECTRAL_REF`` variable; there is no default:

    python tests/golden/make_golden.py /path/to/PySpectral-checkout

The reference is Python 2 code that imports pyFFTW, mpi4py and scipy.weave.
This script executes its unmodified sources under a load-time shim:

* every ``/`` is rewritten by an AST pass into ``_py2div(a, b)`` (floor
  division when both operands are integers, true division otherwise);
* ``np`` is a thin proxy over NumPy 2 that restores ``np.int`` and accepts a
  float ``num`` in ``np.linspace``;
* ``pyfftw`` is a stand-in whose ``FFTW`` object copies into its input buffer,
  runs ``scipy.fft`` (normalised inverse, like pyFFTW's default
  ``normalise_idft=True``) and returns its internal output buffer;
* ``RHSfunctionsWEAVE`` is an empty module; ``mpi4py`` a single-rank stand-in;
* ``utilitiesClass.myFilter`` gets its cutoff truncated to an int: the dynamic
  Smagorinsky model calls it with ``kc/2.`` (``src/RHSfunctions.py:1697``),
  a float slice bound that the NumPy of the reference's day truncated and
  NumPy 2 rejects; ``seperateModesBudgets`` likewise (the budget RHS passes
  the float ``main.kc = np.amax(grid.k1)``, ``src/Classes.py:16``);
* ``pad_2x_var``, called by ``computeRHS_FM1`` but defined in no file of
  the reference, is bound to ``pad_2x`` (the FM1 fixtures hold under that
  assumption only).

``advanceQ_RK4`` lives in the driver script, which runs a whole simulation at
import time, so its four lines (``src/PySpec_3d.py:96-105``) are restated in
:func:`ref_rk4_step`.

Outputs (all FP64, a few hundred KB in total):

* ``serial_N{N}.npz`` -- one RHS evaluation and one RK4 step of every serial
  closure (DNS, Smagorinsky, t-model, static and dynamic tau-model, dynamic
  Smagorinsky, first-order complete memory model, first-order finite memory
  model (one and three subintegrations, and its two-term form), orthogonal
  dynamics (+rotation, kc = N/4), DNS with SGS budgets; DNS,
  Smagorinsky, t-model and dynamic Smagorinsky also with rotation), the
  budget file the hooks write at iteration 20, plus the diagnostics;
* ``mhd_N{N}.npz`` -- one MHD RHS and one RK4 step from the MPI solver;
* ``mpi_ns_N{N}.npz`` -- the MPI solver's Navier-Stokes and orthogonal
  dynamics, with and without rotation, one RHS and one RK4 step;
* ``tgv64_benchmark.npz`` -- the reference's known-answer energy and
  dissipation history (``run/TGV_Validate100/benchmark_sol_64.npz``).
"""
from __future__ import annotations

import ast
import contextlib
import io
import math
import os
import sys
import tempfile
import types

import numpy as np
import scipy.fft

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
from oracle import spectral_oracle as orc  # noqa: E402  (inputs only)

REF = SRC = SRC_MPI = None


def set_reference(path):
    """Point the shim at the reference checkout (the directory holding PySpectral/)."""
    global REF, SRC, SRC_MPI
    if not path or not os.path.isdir(os.path.join(path, "PySpectral", "src")):
        raise SystemExit("make_golden.py: give the reference checkout (the directory holding PySpectral/) "
                         "as the first argument or in PYSPECTRAL_REF")
    REF = path
    SRC = os.path.join(REF, "PySpectral", "src")
    SRC_MPI = os.path.join(REF, "PySpectral", "src_MPI")


# ---------------------------------------------------------------- shim ----
def _py2div(a, b):
    def isint(x):
        if isinstance(x, (bool, int, np.integer)):
            return True
        return isinstance(x, np.ndarray) and np.issubdtype(x.dtype, np.integer)
    if isint(a) and isint(b):
        return a // b
    return a / b


class _DivRewrite(ast.NodeTransformer):
    def visit_BinOp(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            return ast.copy_location(
                ast.Call(func=ast.Name(id="_py2div", ctx=ast.Load()), args=[node.left, node.right],
                         keywords=[]), node)
        return node

    def visit_AugAssign(self, node):
        self.generic_visit(node)
        if isinstance(node.op, ast.Div):
            tgt = node.target
            load = ast.Name(id=tgt.id, ctx=ast.Load()) if isinstance(tgt, ast.Name) else tgt
            return ast.copy_location(ast.Assign(targets=[tgt], value=ast.Call(
                func=ast.Name(id="_py2div", ctx=ast.Load()), args=[load, node.value], keywords=[])), node)
        return node


class _NumpyProxy(types.ModuleType):
    def __init__(self):
        super().__init__("numpy_py2_proxy")
        self.int = int

    def __getattr__(self, name):
        return getattr(np, name)

    @staticmethod
    def linspace(start, stop, num=50, *a, **k):
        return np.linspace(start, stop, int(num), *a, **k)


class _FFTW:
    def __init__(self, inp, out, axes=(0, 1, 2), direction="FFTW_FORWARD", threads=1, **kw):
        self.input_array, self.output_array = inp, out
        self.direction = direction

    def __call__(self, input_array=None):
        if input_array is not None:
            self.input_array[...] = input_array
        if self.direction == "FFTW_BACKWARD":
            self.output_array[...] = scipy.fft.irfftn(self.input_array, s=self.output_array.shape)
        else:
            self.output_array[...] = scipy.fft.rfftn(self.input_array)
        return self.output_array


def _install_stubs():
    pyfftw = types.ModuleType("pyfftw")
    pyfftw.n_byte_align_empty = lambda shape, align, dtype: np.empty(shape, dtype=dtype)
    pyfftw.FFTW = _FFTW
    sys.modules["pyfftw"] = pyfftw
    sys.modules["RHSfunctionsWEAVE"] = types.ModuleType("RHSfunctionsWEAVE")

    class _Comm:
        def Get_size(self):
            return 1

        def Get_rank(self):
            return 0

        def Alltoall(self, send, recv):
            recv[...] = np.asarray(send).reshape(recv.shape)

        def gather(self, x, root=0):
            return [x]

    mpi4py = types.ModuleType("mpi4py")
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.COMM_WORLD = _Comm()
    mpi4py.MPI = mpi
    sys.modules["mpi4py"] = mpi4py
    sys.modules["mpi4py.MPI"] = mpi


def _load(path, name):
    with open(path) as f:
        tree = ast.parse(f.read(), filename=path)
    tree = ast.fix_missing_locations(_DivRewrite().visit(tree))
    mod = types.ModuleType(name)
    mod.__dict__["_py2div"] = _py2div
    mod.__dict__["__name__"] = name
    sys.modules[name] = mod
    code = compile(tree, path, "exec")
    # the sources do "import numpy as np": bind np to the proxy afterwards
    exec(code, mod.__dict__)
    mod.__dict__["np"] = _NumpyProxy()
    return mod


def load_serial():
    _install_stubs()
    for n in ("padding", "RHSfunctions", "Classes"):
        sys.modules.pop(n, None)
    pad = _load(os.path.join(SRC, "padding.py"), "padding")
    rhs = _load(os.path.join(SRC, "RHSfunctions.py"), "RHSfunctions")
    for k, v in pad.__dict__.items():  # "from padding import *"
        if not k.startswith("__"):
            rhs.__dict__.setdefault(k, v)
    # computeRHS_FM1 calls pad_2x_var, which no file of the reference defines
    rhs.__dict__.setdefault("pad_2x_var", pad.pad_2x)
    _split = pad.seperateModesBudgets
    rhs.__dict__["seperateModesBudgets"] = lambda uhat_pad, arrange, kc: _split(uhat_pad, arrange, int(kc))
    cls = _load(os.path.join(SRC, "Classes.py"), "Classes")
    for k, v in rhs.__dict__.items():  # "from RHSfunctions import *"
        if not k.startswith("__") and k != "np":
            cls.__dict__.setdefault(k, v)
    return cls


def load_mpi():
    _install_stubs()
    for n in ("padding", "RHSfunctions", "Classes", "time_schemes"):
        sys.modules.pop(n, None)
    _load(os.path.join(SRC_MPI, "padding.py"), "padding")
    rhs = _load(os.path.join(SRC_MPI, "RHSfunctions.py"), "RHSfunctions")
    ts = _load(os.path.join(SRC_MPI, "time_schemes.py"), "time_schemes")
    cls = _load(os.path.join(SRC_MPI, "Classes.py"), "Classes")
    for src in (rhs, ts):
        for k, v in src.__dict__.items():
            if not k.startswith("__") and k != "np":
                cls.__dict__.setdefault(k, v)
    return cls


# ------------------------------------------------------------ drivers ----
def ref_rk4_step(main, grid, myFFT, utilities):
    """``advanceQ_RK4`` restated from ``src/PySpec_3d.py:96-105``."""
    Q0 = np.zeros(np.shape(main.Q), dtype="complex")
    Q0[:, :, :] = main.Q[:, :, :]
    rk4const = np.array([1.0 / 4, 1.0 / 3, 1.0 / 2, 1.0])
    utilities.preAdvanceQ_hook(main, grid, myFFT)
    utilities.compute_dt(main, grid)
    for i in range(0, 4):
        main.computeRHS(main, grid, myFFT, utilities)
        main.Q = Q0 + main.dt * rk4const[i] * main.Q
    utilities.postAdvanceQ_hook(main, grid, myFFT)


def _diag(Q, nv=3):
    return np.stack([Q[f::nv, f::nv, f::nv] for f in range(nv)])


def serial_case(C, N, state, turb_model, nu, dt, t, rotate=0, Om=(0., 0., 0.), Ct=-10, dt0=-10,
                dt1=-10, kc=None, cfl=None, dt0s=-10, dt1s=-10):
    kc = N // 2 if kc is None else kc
    x, y, z = orc.periodic_coords(N)
    grid = C.gridclass(N, N, N, x, y, z, kc, 2 * np.pi, 2 * np.pi, 2 * np.pi)
    myFFT = C.FFTclass(N, N, N, 1)
    util = C.utilitiesClass()
    _filter = util.myFilter
    util.myFilter = lambda uhat, kc: _filter(uhat, int(kc))
    cfl = -dt if cfl is None else cfl
    with contextlib.redirect_stdout(io.StringIO()):
        main = C.variables(0, turb_model, rotate, Om[0], Om[1], Om[2], grid, state[0].copy(),
                           state[1].copy(), state[2].copy(), t, dt, nu, Ct, dt0, dt0s, dt1, dt1s, cfl, 3)
    main.iteration = 1
    return grid, myFFT, util, main


def gen_serial(N, seed):
    C = load_serial()
    st = orc.isotropic_state(N, seed, k0=3.0)
    st[:, 1:3, 2:4, 1] += 0.05 * (1 + 1j)          # non-Hermitian-free nudge off the analytic IC
    out = {"state": st, "N": N}
    nu, dt, t = 0.02, 0.01, 0.37
    cases = [
        ("dns", 0, {}),
        ("dns_rot", 0, dict(rotate=1, Om=(0.3, -0.2, 0.5))),
        ("smag", 1, {}),
        ("smag_rot", 1, dict(rotate=1, Om=(0.1, 0.4, -0.25))),
        ("tmodel", 2, dict(Ct=0.13)),
        ("tmodel_rot", 2, dict(rotate=1, Om=(0.2, 0.0, 0.3))),
        ("stau", "Static tau-model", dict(dt0=0.05, dt1=0.2)),
        ("dtau", "Dynamic tau-model", {}),
        ("dsmag", 7, {}),
        ("dsmag_rot", 7, dict(rotate=1, Om=(-0.15, 0.35, 0.2))),
        ("dsmag_kc", 7, dict(kc=N // 2 - 1)),         # kc/2 fractional: truncated cutoff
        ("cm1", 6, {}),
        ("budgets", 99, {}),
        ("fm1", 3, dict(dt0=0.05)),
        ("fm1_rot", 3, dict(dt0=0.05, rotate=1, Om=(0.25, -0.1, 0.4))),
        ("fm2", 4, dict(dt0=0.05, dt1=0.03)),
        ("ortho", "Orthogonal Dynamics", dict(kc=N // 4)),   # kc = N/4: Gf u != u
        ("ortho_rot", "Orthogonal Dynamics", dict(kc=N // 4, rotate=1, Om=(0.3, 0.1, -0.2))),
    ]
    for name, tm, kw in cases:
        grid, myFFT, util, main = serial_case(C, N, st, tm, nu, dt, t, **kw)
        with contextlib.redirect_stdout(io.StringIO()):
            main.computeRHS(main, grid, myFFT, util)
        out[f"{name}_rhs"] = _diag(main.Q, getattr(main, "nvars", 3))
        out[f"{name}_uhat"] = np.stack([main.uhat, main.vhat, main.what])
        if hasattr(main, "w0_u"):
            out[f"{name}_w0"] = np.stack([main.w0_u[..., 0], main.w0_v[..., 0], main.w0_w[..., 0]])
        if hasattr(main, "tau"):
            out[f"{name}_tau"] = np.float64(np.real(main.tau))
        if tm == 99:
            out[f"{name}_plql"] = np.stack([main.PLQLu, main.PLQLv, main.PLQLw])
            out[f"{name}_plu"] = np.stack([main.PLu, main.PLv, main.PLw])
        grid, myFFT, util, main = serial_case(C, N, st, tm, nu, dt, t, **kw)
        with contextlib.redirect_stdout(io.StringIO()):
            ref_rk4_step(main, grid, myFFT, util)
        out[f"{name}_step"] = _diag(main.Q, getattr(main, "nvars", 3))
        out[f"{name}_step_uhat"] = np.stack([main.uhat, main.vhat, main.what])
    # the budget hooks (src/Classes.py:632-649) around one step at iteration
    # 20, kc = N/4 so that the SGS force of the filtered field is not trivial
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        os.chdir(tmp)
        os.makedirs("3DSolution")
        try:
            grid, myFFT, util, main = serial_case(C, N, st, 99, nu, dt, t, kc=N // 4)
            main.iteration = 20
            with contextlib.redirect_stdout(io.StringIO()):
                ref_rk4_step(main, grid, myFFT, util)
            with np.load(os.path.join("3DSolution", "budget20.npz")) as b:
                for k in b.files:
                    out["budgetfile_" + k] = b[k]
            out["budgetfile_step"] = _diag(main.Q)
        finally:
            os.chdir(cwd)
    # FM1 with three subintegrations from non-zero memory variables
    w0fm = 0.2 * np.stack([orc.isotropic_state(N, seed + 200 + i, k0=2.0) for i in range(3)])
    out["fm1w_init"] = w0fm
    for stage in ("rhs", "step"):
        grid, myFFT, util, main = serial_case(C, N, st, 3, nu, dt, t, dt0=0.08, dt0s=3)
        for i in range(3):
            main.w0_u[..., i], main.w0_v[..., i], main.w0_w[..., i] = w0fm[i]
        main.U2Q()
        with contextlib.redirect_stdout(io.StringIO()):
            if stage == "rhs":
                main.computeRHS(main, grid, myFFT, util)
                out["fm1w_uhat"] = np.stack([main.uhat, main.vhat, main.what])
            else:
                ref_rk4_step(main, grid, myFFT, util)
        out[f"fm1w_{stage}"] = _diag(main.Q, 12)
    # FM2 with two subintegrations each, from non-zero memory variables
    w2init = 0.2 * np.stack([orc.isotropic_state(N, seed + 400 + i, k0=2.0) for i in range(4)])
    out["fm2w_init"] = w2init                     # w0^1, w0^2, w1^1, w1^2
    for stage in ("rhs", "step"):
        grid, myFFT, util, main = serial_case(C, N, st, 4, nu, dt, t, dt0=0.05, dt1=0.03, dt0s=2, dt1s=2)
        for i in range(2):
            main.w0_u[..., i], main.w0_v[..., i], main.w0_w[..., i] = w2init[i]
            main.w1_u[..., i], main.w1_v[..., i], main.w1_w[..., i] = w2init[2 + i]
        main.U2Q()
        with contextlib.redirect_stdout(io.StringIO()):
            if stage == "rhs":
                main.computeRHS(main, grid, myFFT, util)
                out["fm2w_uhat"] = np.stack([main.uhat, main.vhat, main.what])
            else:
                ref_rk4_step(main, grid, myFFT, util)
        out[f"fm2w_{stage}"] = _diag(main.Q, 15)
    # the two-term FM1 (turb_model 5), fresh and from non-zero memory variables
    w0t = 0.2 * np.stack([orc.isotropic_state(N, seed + 300 + i, k0=2.0) for i in range(2)])
    out["fm2t_init"] = w0t
    for case in ("fm2t", "fm2tw"):
        for stage in ("rhs", "step"):
            grid, myFFT, util, main = serial_case(C, N, st, 5, nu, dt, t, dt0=0.04)
            if case == "fm2tw":
                main.w0_u[:], main.w0_v[:], main.w0_w[:] = w0t[0]
                main.w01_u[:], main.w01_v[:], main.w01_w[:] = w0t[1]
                main.U2Q()
            with contextlib.redirect_stdout(io.StringIO()):
                if stage == "rhs":
                    main.computeRHS(main, grid, myFFT, util)
                    out[f"{case}_uhat"] = np.stack([main.uhat, main.vhat, main.what])
                else:
                    ref_rk4_step(main, grid, myFFT, util)
            out[f"{case}_{stage}"] = _diag(main.Q, 9)
    # CM1 from a state with non-zero memory variables (set, then U2Q)
    w0init = 0.3 * orc.isotropic_state(N, seed + 100, k0=2.0)
    out["cm1w_init"] = w0init
    for stage in ("rhs", "step"):
        grid, myFFT, util, main = serial_case(C, N, st, 6, nu, dt, t)
        for i, a in enumerate((main.w0_u, main.w0_v, main.w0_w)):
            a[..., 0] = w0init[i]
        main.U2Q()
        with contextlib.redirect_stdout(io.StringIO()):
            if stage == "rhs":
                main.computeRHS(main, grid, myFFT, util)
                out["cm1w_w0"] = np.stack([main.w0_u[..., 0], main.w0_v[..., 0], main.w0_w[..., 0]])
                out["cm1w_uhat"] = np.stack([main.uhat, main.vhat, main.what])
            else:
                ref_rk4_step(main, grid, myFFT, util)
        out[f"cm1w_{stage}"] = _diag(main.Q, 6)
    # diagnostics on the input state; kc = N/4 so that the sharp cutoff Gf
    # (and with it the SGS stress of computeSGS_DNS) is not trivial
    out["diag_kc"] = np.int64(N // 4)
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t, kc=N // 4)
    out["energy"] = np.float64(util.computeEnergy(main, grid))
    out["energy_resolved"] = np.float64(util.computeEnergy_resolved(main, grid))
    out["enstrophy"] = np.float64(util.computeEnstrophy(main, grid))
    out["allstats"] = np.array([np.real(v) for v in util.computeAllStats(main, grid)], dtype=np.float64)
    k, spec = util.computeSpectrum(main, grid)
    out["spectrum_k"], out["spectrum"] = k, spec
    k, spec = util.computeSpectrum_resolved(main, grid)
    out["spectrum_res_k"], out["spectrum_res"] = k, spec
    w0u, w0v, w0w = util.computeSGS_DNS(main, grid, myFFT)
    out["sgs_dns_w0"] = np.stack([w0u[..., 0], w0v[..., 0], w0w[..., 0]])
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t, cfl=0.4)
    util.compute_dt(main, grid)
    out["cfl_dt"] = np.float64(main.dt)
    # energy transfer spectrum (src/Classes.py:988-1040) on the input state
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t)
    k, tr = util.computeTransfer(main, grid, myFFT)
    out["transfer_k"], out["transfer"] = np.asarray(k), np.asarray(tr)
    # the k3 = 0-plane variants (:1043-1092, :1152-1205, :1241-1270)
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t)
    k, tr = util.computeTransfer_2D(main, grid, myFFT)
    out["transfer2d_k"], out["transfer2d"] = np.asarray(k), np.asarray(tr)
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t, kc=N // 4)
    k, tr = util.computeTransfer_resolved_2D(main, grid, myFFT)
    out["transfer2d_res"] = np.asarray(tr)
    # resolved transfer (:1093-1150) with kc = N/4, and the SGS transfer
    # (:1206-1239) of the Smagorinsky closure force w0 after one RHS
    grid, myFFT, util, main = serial_case(C, N, st, 0, nu, dt, t, kc=N // 4)
    k, tr = util.computeTransfer_resolved(main, grid, myFFT)
    out["transfer_res"] = np.asarray(tr)
    grid, myFFT, util, main = serial_case(C, N, st, 1, nu, dt, t, kc=N // 4)
    with contextlib.redirect_stdout(io.StringIO()):
        main.computeRHS(main, grid, myFFT, util)
    out["transfer_sgs_u"] = np.stack([main.uhat, main.vhat, main.what])
    out["transfer_sgs_w0"] = np.stack([main.w0_u[..., 0], main.w0_v[..., 0], main.w0_w[..., 0]])
    k, tr = util.computeTransfer_SGS(main, grid, myFFT)
    out["transfer_sgs"] = np.asarray(tr)
    k, tr = util.computeTransfer_SGS_2D(main, grid, myFFT)
    out["transfer2d_sgs"] = np.asarray(tr)
    return out


def gen_mhd(N, seed):
    C = load_mpi()
    comm = sys.modules["mpi4py.MPI"].COMM_WORLD
    x, y, z = orc.periodic_coords(N)
    u = orc.isotropic_state(N, seed, k0=3.0, normalise="none")
    B = orc.isotropic_state(N, seed + 1, k0=3.0, normalise="none") * 0.7
    phys = [np.fft.irfftn(a, s=(N, N, N), axes=(0, 1, 2)) for a in list(u) + list(B)]
    nu, dt = 0.02, 0.005
    out = {"N": N, "nu": nu, "dt": dt}
    res = {}
    for name in ("rhs", "step"):
        with contextlib.redirect_stdout(io.StringIO()):
            grid = C.gridclass(N, N, N, x, y, z, N // 2, 1, 2 * np.pi, 2 * np.pi, 2 * np.pi, 0, comm, "MHD")
            myFFT = C.FFTclass(N, N, N, 1, "pyfftw", N, N, 1, comm, 0)
            uh = np.zeros((N, N, N // 2 + 1), dtype=complex)
            vh, wh = uh.copy(), uh.copy()
            main = C.variables("MHD", 0, 0, 0, 0, grid, phys[0].copy(), phys[1].copy(), phys[2].copy(),
                               phys[3], phys[4], phys[5], uh, vh, wh, 0.0, dt, nu, myFFT, 0,
                               "Physical", "RK4")
        if name == "rhs":
            out["state"] = main.Q.copy()
            out["force"] = main.force.copy()
            main.computeRHS(main, grid, myFFT)
            res["rhs"] = main.Q.copy()
        else:
            main.advanceQ(main, grid, myFFT)
            res["step"] = main.Q.copy()
    out.update(res)
    util = C.utilitiesClass()
    out["energy_u"] = np.float64(util.computeEnergy(main, grid))
    out["energy_B"] = np.float64(util.computeMHDEnergy(main, grid))
    k, s = util.computeSpectrum(main, grid)
    out["spectrum_u"] = s
    k, s = util.computeMHDSpectrum(main, grid)
    out["spectrum_B"] = s
    out["diag_state"] = np.stack([main.uhat, main.vhat, main.what, main.B1hat, main.B2hat, main.B3hat])
    return out


def gen_mpi_ns(N, seed):
    """The MPI solver's Navier-Stokes RHS and RK4 step (turb_model 0 and
    'Orthogonal Dynamics', with and without rotation; kc = N/4 so that the
    filtered field differs)."""
    C = load_mpi()
    comm = sys.modules["mpi4py.MPI"].COMM_WORLD
    x, y, z = orc.periodic_coords(N)
    u = orc.isotropic_state(N, seed, k0=3.0, normalise="none")
    phys = [np.fft.irfftn(a, s=(N, N, N), axes=(0, 1, 2)) for a in u]
    zero = np.zeros((N, N, N))
    nu, dt = 0.02, 0.005
    out = {"N": N, "nu": nu, "dt": dt, "kc": N // 4}
    for name, tm, rot in (("dns", 0, (0, 0., 0., 0.)), ("dns_rot", 0, (1, 0.2, -0.3, 0.4)),
                          ("ortho", "Orthogonal Dynamics", (0, 0., 0., 0.)),
                          ("ortho_rot", "Orthogonal Dynamics", (1, 0.2, -0.3, 0.4))):
        for stage in ("rhs", "step"):
            with contextlib.redirect_stdout(io.StringIO()):
                grid = C.gridclass(N, N, N, x, y, z, N // 4, 1, 2 * np.pi, 2 * np.pi, 2 * np.pi, 0, comm, tm)
                myFFT = C.FFTclass(N, N, N, 1, "pyfftw", N, N, 1, comm, 0)
                uh = np.zeros((N, N, N // 2 + 1), dtype=complex)
                vh, wh = uh.copy(), uh.copy()
                main = C.variables(tm, *rot, grid, phys[0].copy(), phys[1].copy(), phys[2].copy(), zero, zero,
                                   zero, uh, vh, wh, 0.0, dt, nu, myFFT, 0, "Physical", "RK4")
                if stage == "rhs":
                    out["state"] = main.Q.copy()
                    main.computeRHS(main, grid, myFFT)
                    out[f"{name}_uhat"] = np.stack([main.uhat, main.vhat, main.what])
                else:
                    main.advanceQ(main, grid, myFFT)
            out[f"{name}_{stage}"] = main.Q.copy()
    # the semi-implicit scheme (src_MPI/time_schemes.py:9-11), two steps; H is
    # allocated with np.empty there, so it is zeroed before the first step
    for name, rot in (("si", (0, 0., 0., 0.)), ("si_rot", (1, 0.2, -0.3, 0.4))):
        with contextlib.redirect_stdout(io.StringIO()):
            grid = C.gridclass(N, N, N, x, y, z, N // 4, 1, 2 * np.pi, 2 * np.pi, 2 * np.pi, 0, comm, 0)
            myFFT = C.FFTclass(N, N, N, 1, "pyfftw", N, N, 1, comm, 0)
            uh = np.zeros((N, N, N // 2 + 1), dtype=complex)
            vh, wh = uh.copy(), uh.copy()
            main = C.variables(0, *rot, grid, phys[0].copy(), phys[1].copy(), phys[2].copy(), zero, zero,
                               zero, uh, vh, wh, 0.0, dt, nu, myFFT, 0, "Physical", "Semi-Implicit")
            main.H[:] = 0.0
            for k in (1, 2):
                main.advanceQ(main, grid, myFFT)
                out[f"{name}_step{k}"] = main.Q.copy()
                out[f"{name}_H{k}"] = main.H.copy()
    return out


class _ThreadComm:
    """One rank's view of a P-rank communicator whose ranks are threads of this
    process: ``Alltoall(send, recv)`` hands block p of every rank's send buffer
    to rank p (blocks in rank order), as MPI's Alltoall does."""

    def __init__(self, rank, size, shared, barrier):
        self.rank, self.size, self.shared, self.barrier = rank, size, shared, barrier

    def Get_size(self):
        return self.size

    def Get_rank(self):
        return self.rank

    def Alltoall(self, send, recv):
        self.shared[self.rank] = np.array(send).reshape(self.size, -1)
        self.barrier.wait()
        got = np.stack([self.shared[p][self.rank] for p in range(self.size)])
        self.barrier.wait()
        recv[...] = got.reshape(recv.shape)


def gen_slab_fft(shape, seed, P):
    """The MPI solver's slab-decomposed myifft3D / myfft3D (src_MPI/Classes.py:238-258)
    run by P ranks (threads sharing a stand-in communicator) on the slabs of one
    random field: per rank the physical y slab from its spectral x slab, and the
    spectral x slab from its physical y slab."""
    import threading
    C = load_mpi()
    N1, N2, N3 = shape
    rng = np.random.default_rng(seed)
    u = rng.standard_normal(shape)
    uhat = np.fft.rfftn(u)
    Npx, Npy = N1 // P, N2 // P
    shared, barrier = [None] * P, threading.Barrier(P)
    out = {"u": u, "uhat": uhat}
    res, errs = {}, []

    def rank(r):
        try:
            comm = _ThreadComm(r, P, shared, barrier)
            fft = C.FFTclass(N1, N2, N3, 1, "numpy", Npx, Npy, P, comm, r)
            ur = np.zeros((N1, Npy, N3))
            fft.myifft3D(uhat[r * Npx:(r + 1) * Npx].copy(), ur)
            uh = np.zeros((Npx, N2, N3 // 2 + 1), dtype=complex)
            fft.myfft3D(u[:, r * Npy:(r + 1) * Npy].copy(), uh)
            res[r] = (ur, uh)
        except Exception as e:  # surfaced after the join
            errs.append(e)
            barrier.abort()

    th = [threading.Thread(target=rank, args=(r,)) for r in range(P)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    for r in range(P):
        out[f"P{P}_r{r}_u"], out[f"P{P}_r{r}_uhat"] = res[r]
    return out


def main():
    os.makedirs(HERE, exist_ok=True)
    d = {}
    for P in (2, 4):
        d.update(gen_slab_fft((16, 24, 12), 31, P))
    np.savez_compressed(os.path.join(HERE, "slab_fft.npz"), **d)
    print("slab fft", sorted(d.keys()))
    for N, seed in ((12, 11), (16, 5)):
        d = gen_serial(N, seed)
        np.savez_compressed(os.path.join(HERE, f"serial_N{N}.npz"), **d)
        print("serial", N, sorted(d.keys())[:4], "...")
    for N, seed in ((12, 21), (16, 7)):
        d = gen_mhd(N, seed)
        np.savez_compressed(os.path.join(HERE, f"mhd_N{N}.npz"), **d)
        print("mhd", N)
        d = gen_mpi_ns(N, seed + 50)
        np.savez_compressed(os.path.join(HERE, f"mpi_ns_N{N}.npz"), **d)
        print("mpi ns", N)
    b = np.load(os.path.join(REF, "PySpectral", "run", "TGV_Validate100", "benchmark_sol_64.npz"))
    np.savez_compressed(os.path.join(HERE, "tgv64_benchmark.npz"), t=np.real(b["t"]),
                        Energy=np.real(b["Energy"]), Dissipation=np.real(b["Dissipation"]))
    print("tgv64 benchmark copied")


if __name__ == "__main__":
    set_reference(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYSPECTRAL_REF"))
    main()
