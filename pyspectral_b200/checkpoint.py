"""Checkpoint / restart and the run driver in the reference's ``.npz`` layout.

The reference writes its run into a ``3DSolution`` directory
(PySpectral/src/PySpec_3d.py:85-92,148 and the case scripts' savehooks,
e.g. PySpectral/run/TGV_Validate100/inputfile.py:47-56):

* ``grid.npz``     k1, k2, k3 (the (N1, N2, N3/2+1) wavenumber arrays), x, y, z
* ``runinfo.npz``  turb_model, dt, save_freq, nu
* ``npsol<it>.npz`` uhat, vhat, what, t (compressed), every save_freq steps
* ``stats.npz``    Energy, Dissipation, Energy_resolved, Dissipation_resolved,
  t, Enstrophy

and reads them back with PySpectral/src/postProcessingFunctions.py:5-60
(``variablesFromFile``: uhat/vhat/what, and w0_u/w0_v/w0_w[..., 0] when
turb_model != 0; ``gridFromFile``: k1..k3 and N3 = 2 (shape[2] - 1)).  The
files written here carry exactly those keys, shapes and dtypes, so the
reference's post-processing reads them unchanged.

uhat/vhat/what and t are what the reference saves: ``main.uhat`` after a
step, which is the state the last RK stage read (the reference rebinds it
inside the RHS, src/RHSfunctions.py:10-12), and ``main.t``, the time at the
start of that step (the loop advances its own t after setting main.t).  For an exact restart each solution file
also holds ``Q`` (the state after the step) and, for FP32 runs, ``comp`` (the
Kahan compensation); :func:`restart` uses them, and falls back to
uhat/vhat/what for files written by the reference (its ``initDomain =
'Fourier'`` start, src_MPI/Classes.py:33-45).
"""
from __future__ import annotations

import os
import time

import numpy as np


def _np(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def grid_arrays(grid):
    """The arrays of ``grid.npz`` (src/PySpec_3d.py:90)."""
    k1, k2, k3 = grid.numpy_k()
    return {"k1": k1, "k2": k2, "k3": k3, "x": _np(grid.x), "y": _np(grid.y), "z": _np(grid.z)}


def save_grid(grid, directory="3DSolution"):
    os.makedirs(directory, exist_ok=True)
    np.savez(os.path.join(directory, "grid"), **grid_arrays(grid))


def save_runinfo(directory, turb_model, dt, save_freq, nu):
    """``runinfo.npz`` (src/PySpec_3d.py:92)."""
    os.makedirs(directory, exist_ok=True)
    np.savez(os.path.join(directory, "runinfo"), turb_model=turb_model, dt=dt, save_freq=save_freq, nu=nu)


def solution_arrays(main):
    """uhat, vhat, what and t as the reference saves them, w0_u/w0_v/w0_w
    (N1, N2, N3/2+1, 1) when the closure keeps them, and the exact restart
    state Q (plus comp for FP32 runs)."""
    out = {"uhat": _np(main.uhat).astype(np.complex128), "vhat": _np(main.vhat).astype(np.complex128),
           "what": _np(main.what).astype(np.complex128), "t": np.float64(main.t),
           "Q": _np(main.Q)}
    if getattr(main, "comp", None) is not None:
        out["comp"] = _np(main.comp)
    if getattr(main, "w0_u", None) is not None:
        out["w0_u"] = _np(main.w0_u).astype(np.complex128)
        out["w0_v"] = _np(main.w0_v).astype(np.complex128)
        out["w0_w"] = _np(main.w0_w).astype(np.complex128)
    return out


def savehook(main, grid, iteration, directory="3DSolution"):
    """``npsol<iteration>.npz`` (PySpectral/run/TGV_Validate100/inputfile.py:47-56;
    the VTK output of the reference's savehook is commented out there)."""
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, "npsol" + str(iteration))
    np.savez_compressed(path, **solution_arrays(main))
    return path + ".npz"


def stats_arrays(t_hist, energy, energy_resolved, enstrophy):
    """``stats.npz`` contents; the dissipations are the reference's finite
    differences of the energy histories (src/PySpec_3d.py:145-147)."""
    t_hist = np.asarray(t_hist, dtype=np.float64)
    energy = np.asarray(energy)
    energy_resolved = np.asarray(energy_resolved)
    dt = t_hist[1:] - t_hist[:-1]
    return {"Energy": energy, "Dissipation": 1.0 / dt * (energy[1:] - energy[:-1]),
            "Energy_resolved": energy_resolved,
            "Dissipation_resolved": 1.0 / dt * (energy_resolved[1:] - energy_resolved[:-1]),
            "t": t_hist, "Enstrophy": np.asarray(enstrophy)}


def save_stats(directory, t_hist, energy, energy_resolved, enstrophy):
    os.makedirs(directory, exist_ok=True)
    np.savez(os.path.join(directory, "stats"), **stats_arrays(t_hist, energy, energy_resolved, enstrophy))


def load_solution(path):
    """The arrays of a solution file (ours or the reference's) as a dict."""
    with np.load(path) as d:
        return {k: d[k] for k in d.files}


def restart(path, grid, turb_model, dt, nu, precision=64, **kw):
    """``variables`` continuing from a solution file: the exact state Q (and
    Kahan compensation) when the file has them, else its uhat/vhat/what (a
    file written by the reference), at time t + dt (the file's t is the start
    of the step that produced it)."""
    import torch

    from .Classes import variables
    d = load_solution(path)
    if "Q" in d:
        u, v, w = d["Q"][0], d["Q"][1], d["Q"][2]
    else:
        u, v, w = d["uhat"], d["vhat"], d["what"]
    main = variables(kw.pop("weave", 0), turb_model, kw.pop("rotate", 0), kw.pop("Om1", 0), kw.pop("Om2", 0),
                     kw.pop("Om3", 0), grid, u, v, w, float(d["t"]) + dt, dt, nu, precision=precision, **kw)
    if "Q" in d:
        main.Q.copy_(torch.as_tensor(d["Q"], device=main.Q.device).to(main.Q.dtype))
        main.Q2U()
    if "comp" in d and getattr(main, "comp", None) is not None:
        main.comp.copy_(torch.as_tensor(d["comp"], device=main.comp.device).to(main.comp.dtype))
    return main


def run(main, grid, utilities, et, save_freq, directory="3DSolution", turb_model=None, iteration=0, log=None,
        reference_t0=False):
    """The reference's main loop (src/PySpec_3d.py:107-148): grid and run
    information written first, then ``while t <= et``: set main.t, one RK4
    step, t += dt, the savehook every save_freq iterations, the statistics
    appended; ``stats.npz`` at the end.  Returns the statistics.

    The first entry of the time history is the run's starting time, so that a
    restarted run's ``Dissipation[0]`` is the energy change over its first
    step.  The reference always writes 0 there (``t_hist[0] = 0``,
    src/PySpec_3d.py:117-118); for a run from t = 0 the two agree, and
    ``reference_t0=True`` writes 0 after a restart too, as the reference's
    loop would."""
    from .RHSfunctions import advanceQ_RK4
    save_grid(grid, directory)
    save_runinfo(directory, main.turb_model if turb_model is None else turb_model, main.dt, save_freq, main.nu)
    t = float(main.t)
    energy = [utilities.computeEnergy(main, grid)]
    enstrophy = [utilities.computeEnstrophy(main, grid)]
    energy_res = [utilities.computeEnergy_resolved(main, grid)]
    t_hist = [0.0 if reference_t0 else t]
    t0 = time.time()
    while t <= et:
        main.t = t
        main.iteration = iteration
        advanceQ_RK4(main, grid, None, utilities)
        t += main.dt
        if iteration % save_freq == 0:
            savehook(main, grid, iteration, directory)
        iteration += 1
        ens, en, diss, lam, tauk, re = utilities.computeAllStats(main, grid)
        energy.append(en)
        enstrophy.append(ens)
        energy_res.append(utilities.computeEnergy_resolved(main, grid))
        t_hist.append(t)
        if log is not None:
            log(f"Wall Time= {time.time() - t0:.3f}   t={t:.6g}   Energy = {float(np.real(en)):.10g}  "
                f"eps = {float(np.real(diss)):.6g}")
    main.t = t
    save_stats(directory, t_hist, energy, energy_res, enstrophy)
    return stats_arrays(t_hist, energy, energy_res, enstrophy)
