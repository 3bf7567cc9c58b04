"""Precision study: FP32 fields with Kahan-compensated RK4 stage accumulation
against the FP64 run of the same MHD problem.

Problem (the MHD precision case): velocity and magnetic field each drawn from
E(k) = 16 sqrt(2/pi) u0^2 k^4/k0^5 exp(-2 k^2/k0^2) with k0 = 3 and independent
random phases (seeds 2 and 3), both solenoidal; nu = eta = 2e-3; the MHD
t-model closure on both fields (or plain MHD); RK4 with dt = 1e-3.  FP64 stays
only in the energy, cross-helicity and spectrum reductions and the closure's
coefficient, which the library computes in FP64 in both runs.

Every step records the relative error of the FP32 run against the FP64 run:
the fields (max norm over all six spectra), the kinetic and magnetic energies
and the cross-helicity; every `every` steps and at the end also the E(k)
shell spectra of both fields (max relative error over the shells kept by the
2/3 rule whose FP64 energy is above 1e-12 of the spectrum's peak: shells far
below that hold no resolved signal, only rounding noise of the initial
spectrum's Gaussian tail).

    python -m pyspectral_b200.precision [--N 128] [--steps 500] [--out file.json]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np
import torch

from . import _capi
from . import mpi as M
from .initial_conditions import isotropic_state


def mhd_case(N, closure="tmodel", precision=64, k0=3.0, nu=2e-3, dt=1e-3, Ct=0.1, seeds=(2, 3), device=0):
    """(grid, variables) of the MHD precision case at N^3."""
    grid = M.gridclass.periodic(N, device=device)
    u = isotropic_state(N, seeds[0], k0=k0, normalise="none", device=device)
    b = isotropic_state(N, seeds[1], k0=k0, normalise="none", device=device)
    main = M.variables("MHD", 0, 0, 0, 0, grid, None, None, None, None, None, None, uhat=u[0], vhat=u[1],
                       what=u[2], Bhat=[b[0], b[1], b[2]], t=0.0, dt=dt, nu=nu, initDomain="Fourier",
                       precision=precision, forcing=False, closure=None if closure == "none" else closure, Ct=Ct)
    return grid, main


def _shell_spectra(ctx64, Q):
    """E(k) of u and of B, FP64 reductions on the GPU (MPI normalisation)."""
    Eu = ctx64.spectrum_mpi(Q[0:3].contiguous())
    Eb = ctx64.spectrum_mpi(Q[3:6].contiguous())
    return np.asarray(Eu), np.asarray(Eb)


def study(N=128, steps=500, every=50, closure="tmodel", dt=1e-3, device=0, log=print):
    g64, m64 = mhd_case(N, closure, 64, dt=dt, device=device)
    g32, m32 = mhd_case(N, closure, 32, dt=dt, device=device)
    ctx64 = g64.ctx(64)
    kmax = int((N // 2) * 2.0 / 3.0) - 1  # shells inside the 2/3-rule set
    recs, spec = [], []

    def scalars(Q):
        Qd = Q.to(torch.complex128).contiguous()
        eu = ctx64.energy(Qd[0:3].contiguous(), _capi.NORM_MPI)
        eb = ctx64.energy(Qd[3:6].contiguous(), _capi.NORM_MPI)
        hc = ctx64.cross_helicity(Qd[0:3].contiguous(), Qd[3:6].contiguous(), _capi.NORM_MPI)
        return Qd, eu, eb, hc

    def compare(n):
        Q64, eu64, eb64, hc64 = scalars(m64.Q)
        Q32, eu32, eb32, hc32 = scalars(m32.Q)
        r = {"step": n, "t": n * dt,
             "field_rel": float((Q32 - Q64).abs().max() / Q64.abs().max()),
             "Eu_rel": abs(eu32 - eu64) / abs(eu64), "Eb_rel": abs(eb32 - eb64) / abs(eb64),
             "Hc_rel": abs(hc32 - hc64) / max(abs(hc64), 1e-300), "Eu": eu64, "Eb": eb64}
        recs.append(r)
        if n % every == 0 or n == steps:
            Su64, Sb64 = _shell_spectra(ctx64, Q64)
            Su32, Sb32 = _shell_spectra(ctx64, Q32)
            mu = Su64[1:kmax + 1] > 1e-12 * Su64.max()
            mb = Sb64[1:kmax + 1] > 1e-12 * Sb64.max()
            ku = np.abs(Su32[1:kmax + 1] - Su64[1:kmax + 1])[mu] / Su64[1:kmax + 1][mu]
            kb = np.abs(Sb32[1:kmax + 1] - Sb64[1:kmax + 1])[mb] / Sb64[1:kmax + 1][mb]
            spec.append({"step": n, "Ek_u_max_rel": float(ku.max()), "Ek_B_max_rel": float(kb.max()),
                         "shells_u": int(mu.sum()), "shells_B": int(mb.sum())})
            log(f"  step {n:5d}  field {r['field_rel']:.3e}  Eu {r['Eu_rel']:.3e}  Eb {r['Eb_rel']:.3e}  "
                f"E(k) u {ku.max():.3e}  B {kb.max():.3e}")

    compare(0)
    t0 = time.time()
    for n in range(1, steps + 1):
        M.advance(m64, g64, 1)
        M.advance(m32, g32, 1)
        m64.t += dt
        m32.t += dt
        compare(n)
    torch.cuda.synchronize()
    return {"N": N, "steps": steps, "dt": dt, "nu": m64.nu, "closure": closure, "kmax_compared": kmax,
            "per_step": recs, "spectra": spec, "final": {**recs[-1], **spec[-1]}, "wall_s": time.time() - t0}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--every", type=int, default=50)
    ap.add_argument("--closure", choices=["tmodel", "none"], default="tmodel")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    res = study(a.N, a.steps, a.every, a.closure)
    f = res["final"]
    print(json.dumps({"N": a.N, "steps": a.steps, "closure": a.closure, "final": f,
                      "max_field_rel": max(r["field_rel"] for r in res["per_step"]),
                      "max_Ek_u_rel": max(s["Ek_u_max_rel"] for s in res["spectra"]),
                      "max_Ek_B_rel": max(s["Ek_B_max_rel"] for s in res["spectra"]), "wall_s": res["wall_s"]}))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
