"""GPU parity of the dynamic Smagorinsky closure (turb_model 7,
PySpectral/src/RHSfunctions.py:1663-1862) beyond the common cases: the
fractional test-filter cutoff, the coefficient against the oracle, the RK4
step through psb_step_rk4 in FP64 and FP32 (Kahan), and a 32^3 field."""
import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import DT, NU, T, golden, rel

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def np_(t):
    return t.detach().cpu().numpy()


def _main(N, state, kc=None, precision=64, **kw):
    from pyspectral_b200 import Classes as C
    grid = C.gridclass.periodic(N) if kc is None else C.gridclass.periodic(N, kc=kc)
    main = C.variables(0, 7, kw.pop("rotate", 0), 0.0, 0.0, 0.0, grid, state[0], state[1], state[2], T, DT, NU,
                       precision=precision, **kw)
    return grid, main


@pytest.mark.parametrize("N", [12, 16])
def test_fractional_cutoff_matches_reference(N):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(N, d["state"], kc=N // 2 - 1)
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), d["dsmag_kc_rhs"]) < TOL64
    assert rel(np_(main.W0), d["dsmag_kc_w0"]) < TOL64
    grid, main = _main(N, d["state"], kc=N // 2 - 1)
    advanceQ_RK4(main, grid, None, C.utilitiesClass())
    assert rel(np_(main.Q), d["dsmag_kc_step"]) < TOL64


@pytest.mark.parametrize("N,kc", [(16, 8), (16, 4), (32, 16), (32, 11)])
def test_coefficient_matches_oracle(N, kc):
    _torch()
    st = orc.isotropic_state(N, 3 + N, k0=3.0)
    g = orc.Grid.periodic(N, kc=kc)
    ref = orc.dsmag_cs2(g, *st)
    grid, main = _main(N, st, kc=kc)
    main.computeRHS(main, grid, None, None)
    assert main.Cs_sqr == pytest.approx(ref, rel=1e-11)
    r, w0, _ = orc.rhs_dsmag(g, st, orc.Params(nu=NU, t=T, dt=DT))
    assert rel(np_(main.Q), r) < TOL64
    assert rel(np_(main.W0), w0) < TOL64


def test_fp32_step_tracks_fp64():
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    _torch()
    N = 32
    st = orc.isotropic_state(N, 9, k0=3.0)
    util = C.utilitiesClass()
    grid, m64 = _main(N, st)
    grid32, m32 = _main(N, st, precision=32)
    for _ in range(5):
        advanceQ_RK4(m64, grid, None, util)
        advanceQ_RK4(m32, grid32, None, util)
    assert rel(np_(m32.Q).astype(np.complex128), np_(m64.Q)) < 5e-6
    g = orc.Grid.periodic(N)
    Q, _ = orc.advance_rk4(st, lambda q: (orc.rhs_dsmag(g, q, orc.Params(nu=NU, t=T, dt=DT))[0], q), DT)
    grid, m = _main(N, st)
    advanceQ_RK4(m, grid, None, util)
    assert rel(np_(m.Q), Q) < TOL64


def test_zero_field_gives_nan_coefficient_like_the_reference():
    """<M:M> = 0 for a state at rest: the reference's np.mean ratio is 0/0."""
    torch = _torch()
    N = 12
    st = np.zeros((3, N, N, N // 2 + 1), complex)
    grid, main = _main(N, st)
    main.computeRHS(main, grid, None, None)
    assert np.isnan(main.Cs_sqr)
    del torch


def test_not_tuned():
    """psb_autotune rejects the closure with an error, not a wrong shape."""
    torch = _torch()
    from pyspectral_b200 import _capi
    N = 16
    ctx = _capi.Context(N, N, N)
    st = torch.zeros((3, N, N, N // 2 + 1), dtype=torch.complex128, device="cuda")
    with pytest.raises(RuntimeError, match="not tunable"):
        ctx.autotune(_capi.DSMAG, st, _capi.make_params(nu=NU))
