"""Batched ensembles of independent decaying-turbulence runs.

No counterpart in the reference, which advances one run per process
(PySpectral/src/PySpec_3d.py:96-144).  Runs of one grid size, precision and
closure form a batch (``psb_batch``): every pass of an RK4 stage is one launch
over all runs of the batch, with launch shapes picked by the library's
autotuner.  All batches of an ensemble are captured together into one CUDA
graph, so K steps of the whole ensemble are one graph launch.

Ensemble case (uneven sizes): 96 runs, 32 each at 32^3, 48^3 and 64^3; run i
has seed 1000+i, k0 drawn uniformly from {2,3,4,5}, nu log-uniform in
[5e-4, 5e-3]; FP32 fields with Kahan stage accumulation; RK4 with dt = 2e-3.
The learned closure is used where the model was trained (the filter width
of its training data, 2 pi/64); the other sizes fall back to Smagorinsky.

    python -m pyspectral_b200.ensemble [--steps 500] [--per-size 32]

Across GPUs the runs are independent units (the reference's only
decomposition, the slab split of one run with an all-to-all per transform,
src_MPI/Classes.py:244-258, has no counterpart here: every run fits one GPU).
``shard_specs`` bin-packs the runs by cost N^3 log N onto the ranks (longest
first, each to the least-loaded rank), every rank advances its share as its
own ensemble (one process per GPU, its own batches and CUDA graph), and
``gather_stats`` collects the per-run statistics (energy, enstrophy, FP64
reductions on each rank's GPU) on every rank in the original run order with
one all-gather of a few hundred bytes per run -- the only exchange:

    torchrun --nproc-per-node N -m pyspectral_b200.ensemble --steps 500
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import time

import numpy as np
import torch

from . import _capi
from .initial_conditions import isotropic_state

PASSES = ("x-inverse", "y-inverse", "z-fused", "y-forward", "x-forward+epilogue")


def _lib():
    lib = _capi.load()
    if not getattr(lib, "_psb_batch_sigs", False):
        vp, i = ctypes.c_void_p, ctypes.c_int
        for name, args in (("psb_batch_create", [vp, i, i, ctypes.POINTER(vp)]),
                           ("psb_batch_set_run", [vp, i, vp, vp, ctypes.POINTER(_capi.Params)]),
                           ("psb_batch_autotune", [vp]), ("psb_batch_step_rk4", [vp, i]),
                           ("psb_batch_shape", [vp, i, ctypes.POINTER(i), ctypes.POINTER(i), i]),
                           ("psb_batch_destroy", [vp]),
                           ("psb_ensemble_create", [ctypes.POINTER(vp), i, ctypes.POINTER(vp)]),
                           ("psb_ensemble_step_rk4", [vp, i, ctypes.c_uint]),
                           ("psb_ensemble_status", [vp, ctypes.POINTER(i)]),
                           ("psb_ensemble_destroy", [vp])):
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        lib._psb_batch_sigs = True
    return lib


class Batch:
    """``nruns`` runs on one context (grid size + precision) with one closure."""

    def __init__(self, ctx, closure, nruns):
        self.lib = _lib()
        self.ctx = ctx
        self.closure = closure
        self.nruns = nruns
        h = ctypes.c_void_p()
        ctx.check(self.lib.psb_batch_create(ctx.h, closure, nruns, ctypes.byref(h)), "psb_batch_create")
        self.h = h
        self.runs = [None] * nruns

    def set_run(self, r, state, comp, params):
        self.runs[r] = (state, comp, params)  # keep the tensors and params alive
        self.ctx.check(self.lib.psb_batch_set_run(self.h, r, self.ctx._ptr(state), self.ctx._ptr(comp),
                                                  ctypes.byref(params)), "psb_batch_set_run")

    def autotune(self):
        self.ctx.bind_stream()
        self.ctx.check(self.lib.psb_batch_autotune(self.h), "psb_batch_autotune")

    def step(self, nsteps=1):
        self.ctx.bind_stream()
        self.ctx.check(self.lib.psb_batch_step_rk4(self.h, int(nsteps)), "psb_batch_step_rk4")

    def shapes(self):
        out = {}
        for p, name in enumerate(PASSES):
            t = ctypes.c_int()
            rad = (ctypes.c_int * 12)()
            self.ctx.check(self.lib.psb_batch_shape(self.h, p, ctypes.byref(t), rad, 12), "psb_batch_shape")
            out[name] = {"tile": t.value, "radices": [x for x in rad if x]}
        return out

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                self.lib.psb_batch_destroy(h)
            except Exception:
                pass
            self.h = None


class Persistent:
    """Up to four batches (one device, one precision) advanced by one
    cooperative launch per call (``psb_ensemble``): every pass of every RK4
    stage spreads its tiles over all runs of all batches, with a bounded grid
    barrier between passes."""

    def __init__(self, batches):
        self.lib = _lib()
        self.batches = list(batches)
        self.ctx = self.batches[0].ctx
        arr = (ctypes.c_void_p * len(self.batches))(*[b.h.value for b in self.batches])
        h = ctypes.c_void_p()
        self.ctx.check(self.lib.psb_ensemble_create(arr, len(self.batches), ctypes.byref(h)), "psb_ensemble_create")
        self.h = h

    def step(self, nsteps=1, poll_limit=0):
        self.ctx.bind_stream()
        self.ctx.check(self.lib.psb_ensemble_step_rk4(self.h, int(nsteps), int(poll_limit)), "psb_ensemble_step_rk4")

    def status(self):
        """0, or 1 when a grid-barrier wait gave up since the last call (cleared on read)."""
        self.ctx.bind_stream()
        st = ctypes.c_int()
        self.ctx.check(self.lib.psb_ensemble_status(self.h, ctypes.byref(st)), "psb_ensemble_status")
        return st.value

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            try:
                self.lib.psb_ensemble_destroy(h)
            except Exception:
                pass
            self.h = None


def ensemble_specs(sizes=(32, 48, 64), per_size=32, seed0=1000, nu_range=(5e-4, 5e-3), k0s=(2, 3, 4, 5)):
    """Per-run (N, seed, k0, nu) of the ensemble case, reproducible from seed0."""
    rng = np.random.default_rng(seed0)
    specs = []
    i = 0
    for N in sizes:
        for _ in range(per_size):
            k0 = int(rng.choice(k0s))
            nu = float(math.exp(rng.uniform(math.log(nu_range[0]), math.log(nu_range[1]))))
            specs.append({"N": N, "seed": seed0 + i, "k0": k0, "nu": nu})
            i += 1
    return specs


class Ensemble:
    """All runs of an ensemble, grouped into one batch per grid size."""

    def __init__(self, specs, dt=2e-3, precision=32, model=None, learned_N=64, tune=True, device=0):
        self.specs = specs
        self.dt = dt
        self.precision = precision
        self.device = device
        self.model = model
        self.groups = []
        cdt = torch.complex64 if precision == 32 else torch.complex128
        for N in sorted({s["N"] for s in specs}):
            runs = [s for s in specs if s["N"] == N]
            ctx = _capi.Context(N, N, N, precision=precision, device=device)
            ctx64 = _capi.Context(N, N, N, precision=64, device=device)
            use_learned = model is not None and N == learned_N
            closure = _capi.LEARNED if use_learned else _capi.SMAG
            b = Batch(ctx, closure, len(runs))
            states, comps, params = [], [], []
            for r, s in enumerate(runs):
                st = isotropic_state(N, s["seed"], k0=float(s["k0"]), device=device, ctx=ctx64).to(cdt).contiguous()
                comp = torch.zeros_like(st) if precision == 32 else None
                p = _capi.make_params(nu=s["nu"], dt=dt,
                                      mlp_params=model.params.data_ptr() if use_learned else None,
                                      mlp_norm=model.norm.data_ptr() if use_learned else None,
                                      les_delta=2 * math.pi / N, mlp_act=model.act if use_learned else 0,
                                      mlp_hidden=model.hidden if use_learned else 0)
                b.set_run(r, st, comp, p)
                states.append(st)
                comps.append(comp)
                params.append(p)
            if tune:
                b.autotune()
            self.groups.append({"N": N, "ctx": ctx, "batch": b, "states": states, "comps": comps,
                                "closure": "learned" if use_learned else "smag", "runs": runs})
        self.graph = None

    def points(self):
        return sum(s["N"] ** 3 for s in self.specs)

    def step(self, nsteps=1):
        for g in self.groups:
            g["batch"].step(nsteps)

    def capture(self, nsteps=1):
        """One CUDA graph holding nsteps steps of every batch."""
        saved = [[t.clone() for t in g["states"] + [c for c in g["comps"] if c is not None]] for g in self.groups]
        self.step(nsteps)  # outside the capture: kernel attributes and argument blocks
        torch.cuda.synchronize()
        for g, sv in zip(self.groups, saved):
            for t, s in zip(g["states"] + [c for c in g["comps"] if c is not None], sv):
                t.copy_(s)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=side):
            self.step(nsteps)
        torch.cuda.synchronize()
        self.graph_steps = nsteps

    def replay(self):
        self.graph.replay()

    def shapes(self):
        return {g["N"]: g["batch"].shapes() for g in self.groups}

    def persistent(self):
        """The persistent form: every batch of the ensemble in one cooperative
        launch per call (requires one context stream: the launches go on the
        first batch's context's stream, the current torch stream)."""
        if getattr(self, "_pers", None) is None:
            self._pers = Persistent([g["batch"] for g in self.groups])
        return self._pers

    def capture_persistent(self, nsteps=1):
        """One CUDA graph holding one persistent launch of nsteps steps."""
        p = self.persistent()
        saved = [[t.clone() for t in g["states"] + [c for c in g["comps"] if c is not None]] for g in self.groups]
        p.step(nsteps)  # outside the capture: argument blocks and the launch descriptor
        torch.cuda.synchronize()
        for g, sv in zip(self.groups, saved):
            for t, s in zip(g["states"] + [c for c in g["comps"] if c is not None], sv):
                t.copy_(s)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        self.pgraph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.pgraph, stream=side):
            p.step(nsteps)
        torch.cuda.synchronize()
        self.pgraph_steps = nsteps


def time_batched(ens, steps, graph_steps=10):
    """Aggregate grid-pt x steps / s of the whole ensemble, CUDA-graph replays."""
    ens.capture(graph_steps)
    reps = max(1, steps // graph_steps)
    ens.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        ens.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n = reps * graph_steps
    return {"steps": n, "ms": ms, "value": ens.points() * n / (ms / 1e3)}


def time_persistent(ens, steps, graph_steps=10):
    """Aggregate grid-pt x steps / s with one persistent launch per graph
    replay of graph_steps steps."""
    ens.capture_persistent(graph_steps)
    reps = max(1, steps // graph_steps)
    ens.pgraph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        ens.pgraph.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n = reps * graph_steps
    st = ens.persistent().status()
    return {"steps": n, "ms": ms, "value": ens.points() * n / (ms / 1e3), "status": st}


def time_sequential(specs, steps, dt=2e-3, model=None, learned_N=64, device=0):
    """The same runs one after another, each through the single-run path
    (one CUDA graph of `steps` steps per run)."""
    from . import Classes as C
    from .RHSfunctions import StepGraph
    total_ms = 0.0
    pts = 0
    ctxs = {}
    for s in specs:
        N = s["N"]
        if N not in ctxs:
            ctxs[N] = _capi.Context(N, N, N, precision=64, device=device)
        st = isotropic_state(N, s["seed"], k0=float(s["k0"]), device=device, ctx=ctxs[N])
        use_learned = model is not None and N == learned_N
        grid = C.gridclass.periodic(N, device=device)
        main = C.variables(0, "learned" if use_learned else 1, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt,
                           s["nu"], precision=32, model=model if use_learned else None)
        g = StepGraph(main, grid, steps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        pts += N ** 3
        del g
    return {"steps": steps, "ms": total_ms, "value": pts * steps / (total_ms / 1e3)}


def run_cost(spec):
    """Relative cost of one run's step: N^3 log N (the transforms dominate)."""
    n = spec["N"]
    return float(n) ** 3 * math.log(n)


def shard_specs(specs, world):
    """Indices of the runs each of `world` ranks advances: longest-processing-
    time-first bin packing on run_cost (every run assigned exactly once; the
    heaviest rank carries at most 4/3 of the optimum)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(specs)), key=lambda i: (-run_cost(specs[i]), i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(i)
        load[r] += run_cost(specs[i])
    return [sorted(sh) for sh in shards]


def gather_stats(local, group=None):
    """All ranks' per-run records {run index: stats} merged into one list in
    run order (one all-gather of the small host dicts; works over NCCL and
    gloo).  Every run index must appear exactly once across the ranks."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        parts = [local]
    else:
        parts = [None] * dist.get_world_size(group)
        dist.all_gather_object(parts, local, group=group)
    merged = {}
    for part in parts:
        for i, rec in part.items():
            if i in merged:
                raise RuntimeError(f"run {i} reported by two ranks")
            merged[i] = rec
    return [merged[i] for i in sorted(merged)]


def run_stats(ens):
    """Per-run energy and enstrophy of an ensemble's current states (FP64
    reductions on the device), keyed by the run's index in the ensemble's
    spec list."""
    out = {}
    idx = {id(s): i for i, s in enumerate(ens.specs)}
    for g in ens.groups:
        ctx = g["ctx"]
        for s, st in zip(g["runs"], g["states"]):
            out[idx[id(s)]] = {"N": s["N"], "seed": s["seed"], "energy": ctx.energy(st),
                               "enstrophy": ctx.enstrophy(st), "closure": g["closure"]}
    return out


def run_sharded(specs, steps, graph_steps=10, model=None, tune=True, log=print):
    """This rank's share of the ensemble (torchrun / RANK, WORLD_SIZE,
    LOCAL_RANK): advance it in one CUDA graph per graph_steps, time it on the
    device, gather per-run stats and the max-over-ranks time.  Returns the
    whole-job record on every rank."""
    import datetime
    import os
    import torch.distributed as dist
    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    shards = shard_specs(specs, world)
    mine = [specs[i] for i in shards[rank]]
    ens = Ensemble(mine, model=model, tune=tune, device=local)
    res = time_batched(ens, steps, graph_steps)
    stats_local = {shards[rank][j]: rec for j, rec in run_stats(ens).items()}
    ms = res["ms"]
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    stats = gather_stats(stats_local)
    pts = sum(s["N"] ** 3 for s in specs)
    out = {"runs": len(specs), "ranks": world, "steps": res["steps"], "ms_max_over_ranks": ms,
           "value": pts * res["steps"] / (ms / 1e3), "shards": [len(sh) for sh in shards],
           "loads": [sum(run_cost(specs[i]) for i in sh) for sh in shards], "stats": stats}
    if world > 1:
        ens.graph = None
        dist.barrier()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--per-size", type=int, default=32)
    ap.add_argument("--seq-steps", type=int, default=50)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    import os
    from .learned import MLPModel
    model = MLPModel.load(device=int(os.environ.get("LOCAL_RANK", 0)))
    specs = ensemble_specs(per_size=a.per_size)
    if int(os.environ.get("WORLD_SIZE", 1)) > 1:
        import torch.distributed as dist
        res = run_sharded(specs, a.steps, model=model, tune=not a.no_tune)
        if int(os.environ.get("RANK", 0)) == 0:
            print(json.dumps(res))
            if a.out:
                with open(a.out, "w") as fh:
                    json.dump(res, fh)
        dist.destroy_process_group()
        return
    t0 = time.time()
    ens = Ensemble(specs, model=model, tune=not a.no_tune)
    setup_s = time.time() - t0
    batched = time_batched(ens, a.steps)
    persistent = time_persistent(ens, a.steps)
    finite = all(bool(torch.isfinite(torch.view_as_real(s)).all()) for g in ens.groups for s in g["states"])
    seq = time_sequential(specs, a.seq_steps, model=model)
    res = {"runs": len(specs), "sizes": sorted({s["N"] for s in specs}), "batched": batched,
           "persistent": persistent, "sequential": seq, "speedup": batched["value"] / seq["value"],
           "speedup_persistent": persistent["value"] / seq["value"], "shapes": ens.shapes(), "setup_s": setup_s,
           "closures": {g["N"]: g["closure"] for g in ens.groups}, "finite": finite}
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as fh:
            json.dump(res, fh)


if __name__ == "__main__":
    main()
