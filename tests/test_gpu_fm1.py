"""GPU parity of the first-order finite memory model (turb_model 3,
PySpectral/src/RHSfunctions.py:882-1024) with three subintegrations from
non-zero memory variables; the fixtures were made with pad_2x standing in for
the reference's undefined pad_2x_var.  The fresh-state case runs in
test_gpu_parity.py."""
import numpy as np
import pytest

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


def _main(d, N, precision=64, rotate=0, nsub=3):
    torch = _torch()
    from pyspectral_b200 import Classes as C
    grid = C.gridclass.periodic(N)
    st = d["state"]
    main = C.variables(0, 3, rotate, 0.1, 0.2, 0.3, grid, st[0], st[1], st[2], T, DT, NU, dt0=0.08,
                       dt0_subintegrations=nsub, precision=precision)
    # as the reference's case setup would: fill main.w0_* then U2Q (src/Classes.py:253-259)
    init = torch.as_tensor(d["fm1w_init"][:nsub], device=main.Q.device).to(main.Q.dtype)
    for i in range(nsub):
        main.w0_u[..., i], main.w0_v[..., i], main.w0_w[..., i] = init[i]
    main.U2Q()
    return grid, main


@pytest.mark.parametrize("N", [12, 16])
def test_fm1_three_subintegrations_match_reference(N):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(d, N)
    assert main.Q.shape[0] == 12 and main.nvars == 12
    assert tuple(main.w0_u.shape) == (N, N, N // 2 + 1, 3)
    Q0 = np_(main.Q)
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), d["fm1w_rhs"]) < TOL64
    assert rel(np_(main.U), d["fm1w_uhat"]) < TOL64
    # main.w0_* hold the memory variables the RHS read
    assert rel(np_(main.w0_v.permute(3, 0, 1, 2)), Q0[4::3]) == 0
    grid, main = _main(d, N)
    advanceQ_RK4(main, grid, None, C.utilitiesClass())
    assert rel(np_(main.Q), d["fm1w_step"]) < TOL64


def test_fm1_fp32_tracks_fp64():
    d = golden("serial_N16.npz")
    grid, m64 = _main(d, 16)
    grid32, m32 = _main(d, 16, precision=32)
    m64.computeRHS(m64, grid, None, None)
    m32.computeRHS(m32, grid32, None, None)
    assert rel(np_(m32.Q).astype(np.complex128), np_(m64.Q)) < 2e-5


def test_fm1_rotating_with_memory_matches_oracle():
    """Rotating FM1 from non-zero memory variables (the fresh rotating case
    runs against the fixtures in test_gpu_parity.py)."""
    from oracle import spectral_oracle as orc
    d = golden("serial_N12.npz")
    grid, main = _main(d, 12, rotate=1)
    st = np_(main.Q)
    main.computeRHS(main, grid, None, None)
    p = orc.Params(nu=NU, t=T, dt=DT, rotate=1, Om=(0.1, 0.2, 0.3))
    r, _, _ = orc.rhs_fm1(orc.Grid.periodic(12), st, p, dt0=0.08, nsub=3)
    assert rel(np_(main.Q), r) < TOL64


def test_fm1_rejects_too_many_subintegrations():
    d = golden("serial_N12.npz")
    grid, _ = _main(d, 12)
    from pyspectral_b200 import Classes as C
    st = d["state"]
    main = C.variables(0, 3, 0, 0, 0, 0, grid, st[0], st[1], st[2], T, DT, NU, dt0=0.08, dt0_subintegrations=9)
    with pytest.raises(RuntimeError, match="fm_nsub"):
        main.computeRHS(main, grid, None, None)


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("case", ["fm2t", "fm2tw"])
def test_fm1_two_term_matches_reference(N, case):
    """turb_model 5 through PSB_FM1 (two subintegrations of 2 dt0), against the
    reference's own outputs (it runs as written)."""
    torch = _torch()
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    d = golden(f"serial_N{N}.npz")
    st = d["state"]
    for stage in ("rhs", "step"):
        grid = C.gridclass.periodic(N)
        main = C.variables(0, 5, 0, 0, 0, 0, grid, st[0], st[1], st[2], T, DT, NU, dt0=0.04)
        assert main.nvars == 9 and tuple(main.w01_u.shape) == (N, N, N // 2 + 1)
        if case == "fm2tw":
            init = torch.as_tensor(d["fm2t_init"], device=main.Q.device)
            main.w0_u[:], main.w0_v[:], main.w0_w[:] = init[0]
            main.w01_u[:], main.w01_v[:], main.w01_w[:] = init[1]
            main.U2Q()
        if stage == "rhs":
            main.computeRHS(main, grid, None, None)
            assert rel(np_(main.U), d[f"{case}_uhat"]) < TOL64
        else:
            advanceQ_RK4(main, grid, None, C.utilitiesClass())
        assert rel(np_(main.Q), d[f"{case}_{stage}"]) < TOL64
    main = C.variables(0, 5, 1, 0.1, 0.2, 0.3, grid, st[0], st[1], st[2], T, DT, NU, dt0=0.04)
    with pytest.raises(RuntimeError, match="no rotating form"):
        main.computeRHS(main, grid, None, None)
