"""Learned subgrid closure: data generation, training and deployment.

No counterpart in the reference.  A pointwise MLP 10 -> 64 -> 64 -> 6 maps
the 9 resolved velocity gradients du_i/dx_j and the filter width to the
subgrid stress tau_ij = filter(u_i u_j) - filter(u_i) filter(u_j) that the
Smagorinsky model of PySpectral/src/RHSfunctions.py:195-212 approximates.

* Training data comes from the solver itself: an FP32 DNS (decaying isotropic
  turbulence) is advanced on the GPU; at snapshot times its spectrum is
  sharp-cutoff filtered to the LES grid (the Gf cutoff of
  PySpectral/src/Classes.py:584-588), the products u_i u_j are formed with the
  solver's 3/2-dealiased transforms and filtered the same way, and features and
  targets are sampled at LES grid points.
* Training runs the project's own BF16 tensor-core forward/backward kernel and
  Adam (psb_mlp_grad / psb_mlp_adam).
* Deployment: closure PSB_LEARNED (``variables(..., turb_model='learned')``)
  evaluates the MLP on tensor cores inside the fused z-pass of every RHS.

* Targets: the filtered stress itself (--target stress), or its
  eddy-viscosity form (--target eddy, the default: eddy_targets), which keeps
  the local forward energy transfer of the data and drops backscatter and the
  part of the stress not aligned with the resolved strain.

Command line (the config-4 pipeline; about four minutes on one B200; the
shipped model models/sgs_mlp.npz was made by):

    python -m pyspectral_b200.learned --out pyspectral_b200/models/sgs_mlp.npz --hidden 32 --act relu --target eddy
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import _capi

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "models", "sgs_mlp.npz")
NIN, NH, NOUT = 10, 64, 6


def _lib():
    lib = _capi.load()
    if not hasattr(lib, "_mlp_bound"):
        vp, i, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_double
        lib.psb_mlp_sizes.argtypes = [i, ctypes.POINTER(i), ctypes.POINTER(i)]
        lib.psb_mlp_forward.argtypes = [vp, i, i, vp, vp, vp, i, vp]
        lib.psb_mlp_forward_tc.argtypes = [vp, i, vp, vp, vp, i, vp, vp]
        lib.psb_mlp_grad.argtypes = [vp, i, i, vp, vp, vp, vp, vp, i, vp, vp]
        lib.psb_mlp_adam.argtypes = [vp, i, vp, vp, vp, vp, i, f, f, f, f, f]
        lib.psb_physical_fields.argtypes = [vp, vp, i, vp]
        lib.psb_products.argtypes = [vp, vp, vp]
        lib.psb_spectral_resample.argtypes = [vp, i, i, i, vp, i, i, i, i, i, d, i, vp]
        for n in ("psb_mlp_sizes", "psb_mlp_forward", "psb_mlp_forward_tc", "psb_mlp_grad", "psb_mlp_adam", "psb_physical_fields",
                  "psb_products", "psb_spectral_resample"):
            getattr(lib, n).restype = i
        lib._mlp_bound = True
    return lib


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def nparams(hidden=NH):
    a, b = ctypes.c_int(), ctypes.c_int()
    if _lib().psb_mlp_sizes(int(hidden), ctypes.byref(a), ctypes.byref(b)) != 0:
        raise ValueError(f"hidden width {hidden}: 32 or 64")
    return a.value, b.value


ACTS = {"gelu": _capi.ACT_GELU, "relu": _capi.ACT_RELU}


class MLPModel:
    """FP32 master parameters, normalisation and Adam moments on the device;
    `act` is the hidden activation ("gelu" or "relu"), a property of the
    trained model (recorded in its metadata)."""

    def __init__(self, seed=0, device=0, params=None, norm=None, act="gelu", hidden=NH):
        if act not in ACTS:
            raise ValueError(f"unknown activation {act!r} (expected one of {sorted(ACTS)})")
        if hidden == 32 and act != "relu":
            raise ValueError("width-32 networks are built with ReLU")
        self.act_name = act
        self.act = ACTS[act]
        self.hidden = int(hidden)
        n, nn = nparams(self.hidden)
        dev = torch.device("cuda", device)
        if params is None:
            rs = np.random.RandomState(seed)
            parts = []
            for fan_out, fan_in in ((hidden, NIN), (hidden, hidden), (NOUT, hidden)):
                b = 1.0 / math.sqrt(fan_in)
                parts += [rs.uniform(-b, b, size=fan_out * fan_in), np.zeros(fan_out)]
            params = np.concatenate(parts)
        assert len(params) == n
        self.params = torch.as_tensor(np.asarray(params, np.float32), device=dev).contiguous()
        self.norm = torch.as_tensor(np.asarray(norm if norm is not None else
                                               np.r_[np.zeros(NIN), np.ones(NIN), np.zeros(NOUT), np.ones(NOUT)],
                                               np.float32), device=dev).contiguous()
        assert self.norm.numel() == nn
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.step = 0
        self.device = device
        self.meta = {}

    def fit_norm(self, X, T):
        xm, xs = X.mean(0), X.std(0).clamp_min(1e-12)
        ym, ys = T.mean(0), T.std(0).clamp_min(1e-12)
        self.norm.copy_(torch.cat([xm, 1.0 / xs, ym, ys]).float())

    def save(self, path, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.params.cpu().numpy(), norm=self.norm.cpu().numpy(),
                 meta=json.dumps({**self.meta, **meta, "act": self.act_name, "hidden": self.hidden}))

    @classmethod
    def load(cls, path=DEFAULT_MODEL, device=0):
        d = np.load(path)
        meta = json.loads(str(d["meta"])) if "meta" in d else {}
        m = cls(device=device, params=d["params"], norm=d["norm"], act=meta.get("act", "gelu"),
                hidden=meta.get("hidden", NH))
        m.meta = meta
        return m

    def forward(self, ctx, X):
        Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        ctx.bind_stream()
        ctx.check(_lib().psb_mlp_forward(ctx.h, self.act, self.hidden, _p(self.params), _p(self.norm), _p(X.contiguous()),
                                         X.shape[0], _p(Y)), "psb_mlp_forward")
        return Y

    def forward_tc(self, ctx, X):
        """forward() on the tcgen05 tensor-core kernel (width-64 networks);
        raises if an MMA timed out."""
        if self.hidden != 64:
            raise ValueError("the tcgen05 kernel runs width-64 networks")
        Y = torch.empty((X.shape[0], NOUT), dtype=torch.float32, device=X.device)
        err = torch.zeros(1, dtype=torch.int32, device=X.device)
        ctx.bind_stream()
        ctx.check(_lib().psb_mlp_forward_tc(ctx.h, self.act, _p(self.params), _p(self.norm), _p(X.contiguous()),
                                            X.shape[0], _p(Y), _p(err)), "psb_mlp_forward_tc")
        if int(err.item()):
            raise RuntimeError("psb_mlp_forward_tc: an MMA did not complete")
        return Y

    def grad_of(self, ctx, X, T, idx):
        """(loss, grad) over the points idx (the gradient check entry)."""
        self.grad.zero_()
        loss = torch.zeros(1, dtype=torch.float64, device=X.device)
        ctx.bind_stream()
        ctx.check(_lib().psb_mlp_grad(ctx.h, self.act, self.hidden, _p(self.params), _p(self.norm), _p(X), _p(T), _p(idx),
                                      idx.numel(), _p(self.grad), _p(loss)), "psb_mlp_grad")
        return float(loss.item()), self.grad.clone()

    def train(self, ctx, X, T, steps, batch=16384, lr=2e-3, lr_end=1e-4, beta1=0.9, beta2=0.999, eps=1e-8,
              seed=0, log_every=0):
        """Adam on minibatches drawn without replacement per epoch; cosine lr."""
        lib = _lib()
        g = torch.Generator(device=X.device)
        g.manual_seed(seed)
        npts = X.shape[0]
        loss = torch.zeros(1, dtype=torch.float64, device=X.device)
        perm = torch.randperm(npts, generator=g, device=X.device).to(torch.int32)
        pos = 0
        hist = []
        ctx.bind_stream()
        for s in range(steps):
            if pos + batch > npts:
                perm = torch.randperm(npts, generator=g, device=X.device).to(torch.int32)
                pos = 0
            idx = perm[pos:pos + batch]
            pos += batch
            ctx.check(lib.psb_mlp_grad(ctx.h, self.act, self.hidden, _p(self.params), _p(self.norm), _p(X), _p(T), _p(idx),
                                       idx.numel(), _p(self.grad), _p(loss)), "psb_mlp_grad")
            self.step += 1
            lr_s = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * s / max(1, steps)))
            ctx.check(lib.psb_mlp_adam(ctx.h, self.hidden, _p(self.params), _p(self.m), _p(self.v), _p(self.grad), self.step,
                                       lr_s, beta1, beta2, eps, 0.0), "psb_mlp_adam")
            if log_every and (s + 1) % log_every == 0:
                hist.append((s + 1, float(loss.item()) / log_every))
                loss.zero_()
        return hist


# ---------------------------------------------------------------------------
# spectral helpers
# ---------------------------------------------------------------------------
def resample(src, N, n, kc, scale, precision):
    nf = src.shape[0]
    dst = torch.empty((nf, n, n, n // 2 + 1), dtype=src.dtype, device=src.device)
    st = _lib().psb_spectral_resample(_p(src), N, N, N, _p(dst), n, n, n, nf, int(kc), float(scale), precision,
                                      ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    if st != 0:
        raise RuntimeError(f"psb_spectral_resample failed ({st})")
    return dst


def filtered_state(uhat, N, n, precision):
    """Sharp-cutoff filter of a state-normalised spectrum onto the n^3 grid
    (modes |k_i| < n/2 kept, Nyquist dropped)."""
    return resample(uhat, N, n, n // 2, (n / N) ** 1.5, precision)


def physical(ctx, spec3, what):
    n = ctx.N1
    rd = torch.float64 if ctx.precision == 64 else torch.float32
    out = torch.empty((12 if what else 3, n, n, n), dtype=rd, device=spec3.device)
    ctx.bind_stream()
    ctx.check(_lib().psb_physical_fields(ctx.h, _p(spec3.contiguous()), int(what), _p(out)), "psb_physical_fields")
    return out


def products(ctx, spec3):
    out = torch.empty((6,) + tuple(spec3.shape[1:]), dtype=spec3.dtype, device=spec3.device)
    ctx.bind_stream()
    ctx.check(_lib().psb_products(ctx.h, _p(spec3.contiguous()), _p(out)), "psb_products")
    return out


def sgs_samples(ctx_dns, ctx_les, uhat, precision=32):
    """Features (n^3 x 10) and targets (n^3 x 6) of one DNS snapshot filtered
    onto the LES grid of ctx_les."""
    N, n = ctx_dns.N1, ctx_les.N1
    ub = filtered_state(uhat, N, n, precision)
    f12 = physical(ctx_les, ub, 1)
    P = products(ctx_dns, uhat)
    Pb = filtered_state(P, N, n, precision)
    fuu = torch.cat([physical(ctx_les, Pb[0:3].contiguous(), 0), physical(ctx_les, Pb[3:6].contiguous(), 0)])
    u = f12[0:3]
    tau = torch.stack([fuu[m] - u[a] * u[b] for m, (a, b) in enumerate(PAIRS)])
    delta = 2 * math.pi / n
    X = torch.cat([f12[3:12].reshape(9, -1), torch.full((1, n ** 3), delta, device=uhat.device, dtype=f12.dtype)])
    return X.t().float().contiguous(), tau.reshape(6, -1).t().float().contiguous()


PAIRS = ((0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2))


def eddy_targets(X, T, eps=1e-30):
    """Targets of the eddy-viscosity form: per sample the least-squares eddy
    viscosity of the filtered stress, nu_t = max(0, -(tau:S) / (2 S:S)), and
    the stress -2 nu_t S it implies (S_ij = (du_i/dx_j + du_j/dx_i)/2 from the
    9 gradient features, X[:, 3i+j] = du_i/dx_j; components in the order of T,
    (00, 11, 22, 01, 02, 12)).  The stress keeps the local energy transfer
    -tau:S of the data where it is forward (nu_t > 0) and drops backscatter
    and the part of tau not aligned with S; its trace is zero (the trace of
    tau is a pressure and leaves the projected RHS unchanged)."""
    G = X[:, :9].double().reshape(-1, 3, 3)
    S = 0.5 * (G + G.transpose(1, 2))
    S6 = torch.stack([S[:, a, b] for a, b in PAIRS], 1)
    w = torch.tensor([1.0, 1.0, 1.0, 2.0, 2.0, 2.0], dtype=S6.dtype, device=S6.device)
    tS = (T.double() * S6 * w).sum(1)
    SS = (S6 * S6 * w).sum(1)
    nu_t = torch.clamp(-tS / (2.0 * SS + eps), min=0.0)
    return (-2.0 * nu_t[:, None] * S6).float().contiguous()


# ---------------------------------------------------------------------------
# runs
# ---------------------------------------------------------------------------
def make_run(N, seed, nu, dt, closure=0, precision=32, k0=4.0, device=0, state=None, model=None):
    from . import Classes as C
    from .initial_conditions import isotropic_state
    grid = C.gridclass.periodic(N, device=device)
    st = isotropic_state(N, seed, k0=k0, device=device) if state is None else state
    main = C.variables(0, closure, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu, precision=precision,
                       model=model)
    return grid, main


def energy_spectrum(grid, main):
    """E(k) summed over components (computeSpectrum, src/Classes.py:762-797)."""
    s = grid.ctx(main.precision).spectrum(main.Q[0:3].contiguous())
    return s.sum(1)


def generate(N_dns=256, les=(64, 32), seed=11, nu=5e-4, dt=2e-3, t_snap=(1.0, 8.0, 0.5), npoints=2 ** 22,
             device=0, log=print):
    """Training set from an FP32 DNS: returns (X, T) on the device."""
    from .RHSfunctions import advance
    torch.manual_seed(seed)
    grid, main = make_run(N_dns, seed, nu, dt, 0, 32, device=device)
    cdns = grid.ctx(32)
    cles = {n: _capi.Context(n, n, n, precision=32, device=device) for n in les}
    times = np.arange(t_snap[0], t_snap[1] + 1e-9, t_snap[2])
    Xs, Ts = [], []
    t = 0.0
    t0 = time.time()
    for ts in times:
        nsteps = int(round((ts - t) / dt))
        advance(main, grid, nsteps)
        t += nsteps * dt
        for n in les:
            X, T = sgs_samples(cdns, cles[n], main.Q, 32)
            Xs.append(X)
            Ts.append(T)
        log(f"  snapshot t={t:.2f}  ({time.time() - t0:.1f} s)")
    X = torch.cat(Xs)
    T = torch.cat(Ts)
    if npoints and npoints < X.shape[0]:
        g = torch.Generator(device=X.device)
        g.manual_seed(seed)
        sel = torch.randperm(X.shape[0], generator=g, device=X.device)[:npoints]
        X, T = X[sel].contiguous(), T[sel].contiguous()
    return X, T


def evaluate(model, N_dns=256, n=64, seed=23, nu=5e-4, dt_dns=2e-3, dt_les=4e-3, t0=1.0, les_steps=2000,
             every=250, device=0, log=print):
    """A-posteriori test (config 4): LES from the filtered DNS at t0, advanced
    les_steps; E(k) vs the filtered DNS at the same time for 1 <= k <= n/4,
    at every `every` LES steps and at the end, for the learned closure (FP32),
    Smagorinsky (FP64 and FP32) and no model (FP32)."""
    from .RHSfunctions import advance
    grid, dns = make_run(N_dns, seed, nu, dt_dns, 0, 32, device=device)
    n0 = int(round(t0 / dt_dns))
    advance(dns, grid, n0)
    ub0 = filtered_state(dns.Q, N_dns, n, 32).to(torch.complex128)
    runs = {}
    for name, closure, prec in (("learned_fp32", "learned", 32), ("smagorinsky_fp64", 1, 64),
                                ("smagorinsky_fp32", 1, 32), ("no_model_fp32", 0, 32)):
        g, m = make_run(n, 0, nu, dt_les, closure, prec, device=device, state=ub0, model=model)
        runs[name] = (g, m)
    kmax = n // 4
    ctx_les = runs["learned_fp32"][0].ctx(32)
    hist = {name: [] for name in runs}
    times = []
    t1 = time.time()
    done = 0
    ratio = int(round(dt_les / dt_dns))
    Eref = None
    while done < les_steps:
        chunk = min(every, les_steps - done)
        advance(dns, grid, chunk * ratio)
        for name, (g, m) in runs.items():
            advance(m, g, chunk)
        done += chunk
        ref = filtered_state(dns.Q, N_dns, n, 32)
        Eref = ctx_les.spectrum(ref).sum(1)
        times.append(t0 + done * dt_les)
        for name, (g, m) in runs.items():
            E = g.ctx(m.precision).spectrum(m.Q[0:3].contiguous()).sum(1)
            rel = np.abs(E[1:kmax + 1] - Eref[1:kmax + 1]) / Eref[1:kmax + 1]
            hist[name].append({"t": times[-1], "max": float(rel.max()), "mean": float(rel.mean()),
                               "E": E[:kmax + 1].tolist(), "finite": bool(np.isfinite(E).all())})
        log(f"  t={times[-1]:5.2f}  " + "  ".join(f"{k}: {v[-1]['max']:.3f}/{v[-1]['mean']:.3f}"
                                                for k, v in hist.items()))
    torch.cuda.synchronize()
    out = {"t0": t0, "t_end": times[-1], "N_dns": N_dns, "n_les": n, "k_compare": kmax,
           "E_ref": Eref[:kmax + 1].tolist(), "times": times}
    for name, h in hist.items():
        out[name] = {"max_rel_err_k_le_kc_half": h[-1]["max"], "mean_rel_err": h[-1]["mean"], "E": h[-1]["E"],
                     "finite": h[-1]["finite"], "history": [{k: r[k] for k in ("t", "max", "mean")} for r in h]}
    out["wall_s"] = time.time() - t1
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--N-dns", type=int, default=256)
    ap.add_argument("--npoints", type=int, default=2 ** 22)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--les-steps", type=int, default=2000)
    ap.add_argument("--no-eval", action="store_true")
    ap.add_argument("--nu", type=float, default=5e-4, help="viscosity of the DNS and the LES")
    ap.add_argument("--act", choices=sorted(ACTS), default="relu", help="hidden activation of the network")
    ap.add_argument("--hidden", type=int, choices=(32, 64), default=NH, help="hidden width of the network")
    ap.add_argument("--target", choices=("stress", "eddy"), default="eddy",
                    help="fit the filtered stress itself, or its eddy-viscosity form (eddy_targets)")
    ap.add_argument("--eval-only", action="store_true",
                    help="re-run the a-posteriori evaluation of the model at --out and update its metadata")
    a = ap.parse_args()
    t0 = time.time()
    if a.eval_only:
        model = MLPModel.load(a.out)
        meta = dict(model.meta)
        meta["eval"] = evaluate(model, N_dns=a.N_dns, nu=meta.get("nu", a.nu), les_steps=a.les_steps)
        model.save(a.out, **meta)
        with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
            json.dump(meta, f, indent=1)
        print(f"updated {a.out} ({time.time() - t0:.1f} s)")
        return
    print("generating training data ...")
    X, T = generate(N_dns=a.N_dns, nu=a.nu, npoints=a.npoints)
    print(f"  {X.shape[0]} samples ({time.time() - t0:.1f} s)")
    if a.target == "eddy":
        T = eddy_targets(X, T)
    model = MLPModel(seed=0, act=a.act, hidden=a.hidden)
    model.fit_norm(X, T)
    ctx = _capi.Context(64, 64, 64, precision=32)
    hist = model.train(ctx, X, T, a.steps, batch=a.batch, log_every=max(1, a.steps // 20))
    for s, l in hist:
        print(f"  step {s:6d}  loss {l:.5f}")
    meta = {"train_samples": int(X.shape[0]), "train_steps": a.steps, "batch": a.batch,
            "final_loss": hist[-1][1] if hist else None, "N_dns": a.N_dns, "nu": a.nu, "act": a.act,
            "hidden": a.hidden, "target": a.target,
            "spectrum": "E(k)=16 sqrt(2/pi) u0^2 k^4/k0^5 exp(-2 k^2/k0^2), k0=4, u0=1"}
    model.meta = meta
    if not a.no_eval:
        print("a-posteriori evaluation ...")
        meta["eval"] = evaluate(model, N_dns=a.N_dns, nu=a.nu, les_steps=a.les_steps)
    model.save(a.out, **meta)
    with open(os.path.splitext(a.out)[0] + ".json", "w") as f:
        json.dump(meta, f, indent=1)
    print(f"saved {a.out} ({time.time() - t0:.1f} s)")


if __name__ == "__main__":
    main()
