"""Decaying isotropic turbulence LES: the closures side by side on one field.

The reference's decaying-turbulence case (PySpectral/run/HIT/MansourWray/
inputfile.py, driven by the loop of PySpectral/src/PySpec_3d.py:107-148) run
through this package's public API: one seeded solenoidal field with the
spectrum E(k) = 16 sqrt(2/pi) u0^2 k^4 / k0^5 exp(-2 k^2 / k0^2) (k0 = 4,
u0 = 1, initial_conditions.isotropic_state), advanced by fixed-dt RK4 with
each closure from the same start:

* Smagorinsky (turb_model 1, Cs = 0.16, Delta = the grid spacing) in FP64,
  the reference closure of the case, and in FP32 + Kahan for the precision
  comparison;
* the t-model (turb_model 2, Ct = 0.1, the reference's default), whose
  memory coefficient grows with t: every step is its own call with main.t
  set, as the reference's loop does;
* the static tau-model (tau_a, tau_b = dt0, dt1) and the dynamic tau-model.

For every run: the energy, resolved energy, enstrophy and viscous
dissipation 2 nu Omega (FP64 device reductions, utilitiesClass.computeAllStats,
PySpectral/src/Classes.py:652-744) every `every` steps, E(k) at the end
(computeSpectrum, PySpectral/src/Classes.py:762-797, summed over the three
components), the device time per
step (CUDA events around the stepping only, diagnostics excluded) and
whether the state stayed finite (a run whose energy turns non-finite stops
there and reports the time).  The FP32 Smagorinsky run also reports its
relative difference from the FP64 one (energy history, E(k), final fields).

    python -m pyspectral_b200.hit --N 128 --steps 1000 --out hit128.json
    python -m pyspectral_b200.hit --closures tmodel,tau_static --closure-dt tmodel=1e-3,tau_static=5e-4 --no-fp32
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np
import torch

from . import Classes as C
from .RHSfunctions import advanceQ_RK4
from .initial_conditions import isotropic_state

# name -> (turb_model, keyword arguments of variables)
CLOSURES = {
    "smag": (1, {}),
    "tmodel": (2, {}),
    "tau_static": ("Static tau-model", {"dt0": 0.05, "dt1": 0.2}),
    "tau_dynamic": ("Dynamic tau-model", {}),
    "dns": (0, {}),
}


def make_case(N, closure, precision=64, seed=1, k0=4.0, dt=2e-3, nu=1e-3, device=0, state=None):
    """(grid, main, utilities) of one run from the seeded isotropic field."""
    tm, kw = CLOSURES[closure]
    grid = C.gridclass.periodic(N, device=device)
    st = isotropic_state(N, seed, k0=k0, device=device) if state is None else state
    main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu, precision=precision, **kw)
    return grid, main, C.utilitiesClass()


def _stats(util, main, grid, t):
    ens, en, diss, _, _, _ = util.computeAllStats(main, grid)
    return {"t": t, "energy": float(np.real(en)), "energy_resolved": float(np.real(util.computeEnergy_resolved(main, grid))),
            "enstrophy": float(np.real(ens)), "dissipation": float(np.real(diss))}


def run_case(N, closure, steps, precision=64, every=10, seed=1, k0=4.0, dt=2e-3, nu=1e-3, device=0, state=None):
    """Advance one closure `steps` RK4 steps; returns (result dict, main, grid).

    The statistics of step 0 are taken on the initial state, later ones on the
    state the last stage read (main.uhat), as the reference's loop does."""
    grid, main, util = make_case(N, closure, precision, seed, k0, dt, nu, device, state)
    hist = [_stats(util, main, grid, 0.0)]
    t = 0.0
    dev_ms = 0.0
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    done = 0
    while done < steps:
        chunk = min(every, steps - done)
        torch.cuda.synchronize()
        start.record()
        for _ in range(chunk):
            main.t = t
            main.iteration = done
            advanceQ_RK4(main, grid, None, None)
            t += dt
            done += 1
        stop.record()
        stop.synchronize()
        dev_ms += start.elapsed_time(stop)
        hist.append(_stats(util, main, grid, t))
        if not math.isfinite(hist[-1]["energy"]):
            break  # the run blew up: no further steps
    main.t = t
    k, E = util.computeSpectrum(main, grid)
    finite = bool(torch.isfinite(torch.view_as_real(main.Q)).all().item())
    bad = [h["t"] for h in hist if not math.isfinite(h["energy"])]
    res = {"closure": closure, "N": N, "precision": precision, "steps": steps, "steps_run": done, "dt": dt, "nu": nu,
           "seed": seed, "k0": k0, "ms_per_step": dev_ms / max(1, done),
           "grid_pt_steps_per_s": N ** 3 * done / (dev_ms * 1e-3), "finite": finite,
           "non_finite_at_t": bad[0] if bad else None, "history": hist,
           "E_k": np.real(np.asarray(E)).sum(1).tolist()}
    return res, main, grid


def rel_diff(a, b):
    """max |a - b| / max |b| over arrays of any shape."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--dt", type=float, default=2e-3)
    ap.add_argument("--nu", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--every", type=int, default=10)
    ap.add_argument("--closures", default="smag,tmodel,tau_static,tau_dynamic")
    ap.add_argument("--closure-dt", default="",
                    help="per-closure time steps, e.g. 'tmodel=1e-3,tau_static=5e-4': those runs cover the same "
                         "time (steps * dt) with more, smaller steps")
    ap.add_argument("--no-fp32", action="store_true", help="skip the FP32 + Kahan Smagorinsky comparison")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    t0 = time.time()
    out = {"case": f"decaying isotropic turbulence, {a.N}^3, k0=4, u0=1, nu={a.nu}, dt={a.dt}, {a.steps} RK4 steps",
           "runs": {}}
    finals = {}
    cdt = {k: float(v) for k, v in (x.split("=") for x in a.closure_dt.split(",") if x)}
    for name in a.closures.split(","):
        dt = cdt.get(name, a.dt)
        r = int(round(a.dt / dt))  # steps of this run per step of the case
        res, m, _ = run_case(a.N, name, a.steps * r, 64, a.every * r, a.seed, dt=dt, nu=a.nu)
        out["runs"][f"{name}_fp64" + ("" if r == 1 else f"_dt{dt:g}")] = res
        if name == "smag":
            finals["smag"] = m.Q.cpu().numpy()
        h = res["history"][-1]
        print(f"{name:12s} FP64 dt={dt:g}  {res['ms_per_step']:.3f} ms/step  t={h['t']:.3f}  E={h['energy']:.6f}  "
              f"eps={h['dissipation']:.6f}  finite={res['finite']}  ({time.time() - t0:.0f} s)", flush=True)
        del m
        torch.cuda.empty_cache()
    if not a.no_fp32 and "smag" in finals:
        res, m, _ = run_case(a.N, "smag", a.steps, 32, a.every, a.seed, dt=a.dt, nu=a.nu)
        ref = out["runs"]["smag_fp64"]
        e32 = np.array([h["energy"] for h in res["history"]])
        e64 = np.array([h["energy"] for h in ref["history"]])
        E32, E64 = np.array(res["E_k"]), np.array(ref["E_k"])
        kmax = a.N // 2
        shells = E64[1:kmax] > 1e-12 * E64[1:kmax].max()
        res["vs_fp64"] = {
            "energy_history_max_rel": float(np.abs(e32 - e64).max() / np.abs(e64).max()),
            "E_k_max_rel_shells_with_signal": float((np.abs(E32[1:kmax] - E64[1:kmax]) / E64[1:kmax])[shells].max()),
            "field_max_rel": rel_diff(m.Q.cpu().numpy(), finals["smag"]),
        }
        out["runs"]["smag_fp32"] = res
        print(f"smag         FP32  {res['ms_per_step']:.3f} ms/step  vs FP64: {res['vs_fp64']}", flush=True)
    out["wall_s"] = time.time() - t0
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f, indent=1)
    return out


if __name__ == "__main__":
    main()
