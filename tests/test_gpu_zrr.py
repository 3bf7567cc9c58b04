"""The register-direct z pass (zpass_rr_kernel; psb_ctx_set_zrr).

For a compiled two-pass schedule (R1, 16) the z pass of the 3/2-padded
Navier-Stokes closures (DNS products, Smagorinsky, learned; FP32) loads the
packed spectra of its inverse transform straight from global memory into
registers and hands the results of its forward transform straight to the
unpack, pairing k3 = q with M - q across the lanes of a 16-lane group by warp
shuffles.  These tests run it at the three lengths it serves (48, 96 and 192
points: (3, 16), (6, 16), (12, 16)) with 2, 4 and 8 pencils per CTA, on grids
one of whose pencil counts is not a multiple of the tile, and hold it to the CPU
oracle and to the shared-memory z pass on the same shapes.

Bars: FP32 fields 2e-5 against the FP64 oracle of the FP32-rounded state, the
learned closure (BF16 tensor-core arithmetic) 5e-4 against the BF16-emulating
oracle; the two z passes within FP32 rounding of each other (5e-6; 2e-4 for
the learned closure, whose BF16 feature rounding can round a few points the
other way).
"""
import numpy as np
import pytest

from oracle import mlp_oracle as mo
from oracle import spectral_oracle as orc
from tests.helpers import rel

pytestmark = pytest.mark.gpu
NU, DT = 1e-3, 2e-3
# (N1, N2, N3): z lengths 48, 96 and 192; 18 x 18 = 324 pencils leaves a ragged last tile at 8 per CTA
SHAPES = [(32, 32, 32), (12, 12, 64), (16, 12, 128)]


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _state(shape, seed):
    N1, N2, N3 = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((3, N1, N2, N3))
    k = np.sqrt(np.add.outer(np.add.outer(np.fft.fftfreq(N1, 1 / N1) ** 2, np.fft.fftfreq(N2, 1 / N2) ** 2),
                             np.fft.rfftfreq(N3, 1 / N3) ** 2))
    st = np.stack([np.fft.rfftn(a) for a in x]) * np.exp(-0.25 * k) / np.sqrt(N1 * N2 * N3)
    return st.astype(np.complex64).astype(np.complex128)  # what an FP32 run holds


def _grids(shape):
    from pyspectral_b200 import Classes as C
    N1, N2, N3 = shape
    L = 2 * np.pi
    kc = min(shape) // 2
    a1, a2, a3 = (np.arange(n) * (L / n) for n in shape)
    y, x, z = np.meshgrid(a2, a1, a3)
    return C.gridclass(N1, N2, N3, x, y, z, kc), orc.Grid(N1, N2, N3, L / N1, L / N2, L / N3, kc)


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("closure", ["dns", "smag", "learned"])
def test_register_direct_zpass_matches_oracle_and_shared_memory_zpass(shape, closure):
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.learned import MLPModel
    st = _state(shape, 11)
    grid, g = _grids(shape)
    model = MLPModel.load() if closure == "learned" else None
    tm = {"dns": 0, "smag": 1, "learned": "learned"}[closure]
    # the learned closure's filter-width feature at the width the shipped network was trained for
    delta = 2 * np.pi / 64
    main = C.variables(0, tm, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, DT, NU, precision=32, model=model,
                       les_delta=delta)
    if closure == "learned":
        ref = mo.rhs_learned(g, st, NU, model.params.cpu().numpy().astype(np.float64),
                             model.norm.cpu().numpy().astype(np.float64), delta, act=model.act_name)
        tol, tol_pair = 5e-4, 2e-4
    else:
        ref = (orc.rhs_nosgs if closure == "dns" else orc.rhs_smag)(g, st, orc.Params(nu=NU))[0]
        tol, tol_pair = 2e-5, 5e-6
    ctx = grid.ctx(32)
    code = main.closure_code()
    M = 3 * shape[2] // 2
    ran = 0
    for tile in (2, 4, 8):
        shapes = [None] * 5
        shapes[2] = {"tile": tile, "radices": [M // 16, 16]}
        ctx.autotune_clear(code)
        try:
            ctx.set_tuned_shapes(code, shapes)
        except RuntimeError:
            continue  # beyond the closure's pencil bound or shared-memory budget
        out = []
        for zrr in (True, False):
            ctx.set_zrr(zrr)
            r = torch.empty_like(main.Q)
            ctx.rhs(code, main.Q, r, main.params())
            torch.cuda.synchronize()
            out.append(r.cpu().numpy().astype(np.complex128))
        ctx.set_zrr(True)
        errs = (tile, rel(out[0], ref), rel(out[1], ref), rel(out[0], out[1]))
        assert errs[1] < tol and errs[3] < tol_pair, errs
        ran += 1
    ctx.autotune_clear(code)
    assert ran >= 2
    assert ctx.device_status() == 0


def test_register_direct_zpass_rk4_step_with_kahan():
    """One FP32 + Kahan RK4 step of the learned closure at 64^3 with the
    register-direct z pass at 4 and 8 pencils per CTA, against the oracle's
    step (increments to 1e-3, as for the tuned headline shapes)."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    from pyspectral_b200.learned import MLPModel
    N = 64
    model = MLPModel.load()
    st = orc.isotropic_state(N, 1, k0=4.0)
    st32 = st.astype(np.complex64).astype(np.complex128)
    g = orc.Grid.periodic(N)
    prm, nrm = (model.params.cpu().numpy().astype(np.float64), model.norm.cpu().numpy().astype(np.float64))
    Q1, _ = orc.advance_rk4(st32, lambda q: (mo.rhs_learned(g, q, NU, prm, nrm, 2 * np.pi / N,
                                                               act=model.act_name), None), DT)
    for tile in (4, 8):
        grid = C.gridclass.periodic(N)
        main = C.variables(0, "learned", 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, DT, NU, precision=32,
                           model=model)
        shapes = [None] * 5
        shapes[2] = {"tile": tile, "radices": [6, 16]}
        grid.ctx(32).set_tuned_shapes(main.closure_code(), shapes)
        advanceQ_RK4(main, grid, None, None)
        got = main.Q.cpu().numpy().astype(np.complex128)
        assert rel(got - st32, Q1 - st32) < 1e-3, tile
