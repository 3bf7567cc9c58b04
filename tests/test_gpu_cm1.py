"""GPU parity of the first-order complete memory model (turb_model 6,
PySpectral/src/RHSfunctions.py:1411-1542) from non-zero memory variables,
against the reference's own outputs; the common fresh-state cases run in
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


def _main(d, N, precision=64, rotate=0):
    torch = _torch()
    from pyspectral_b200 import Classes as C
    grid = C.gridclass.periodic(N)
    st = d["state"]
    main = C.variables(0, 6, rotate, 0.1, 0.2, 0.3, grid, st[0], st[1], st[2], T, DT, NU, precision=precision)
    main.Q[3:6].copy_(torch.as_tensor(d["cm1w_init"], device=main.Q.device).to(main.Q.dtype))
    return grid, main


@pytest.mark.parametrize("N", [12, 16])
def test_cm1_with_memory_matches_reference(N):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(d, N)
    assert main.Q.shape[0] == 6 and main.nvars == 6
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), d["cm1w_rhs"]) < TOL64
    assert rel(np_(main.W0), d["cm1w_w0"]) < TOL64
    assert rel(np_(main.U), d["cm1w_uhat"]) < TOL64
    grid, main = _main(d, N)
    advanceQ_RK4(main, grid, None, C.utilitiesClass())
    assert rel(np_(main.Q), d["cm1w_step"]) < TOL64


def test_cm1_fp32_tracks_fp64():
    """FP32 bars: 2e-5 for one RHS (as for every closure), 1e-4 after three
    RK4 steps (12 stages of rounding carried by the memory variables)."""
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    d = golden("serial_N16.npz")
    util = C.utilitiesClass()
    grid, m64 = _main(d, 16)
    grid32, m32 = _main(d, 16, precision=32)
    m64.computeRHS(m64, grid, None, None)
    m32.computeRHS(m32, grid32, None, None)
    assert rel(np_(m32.Q).astype(np.complex128), np_(m64.Q)) < 2e-5
    grid, m64 = _main(d, 16)
    grid32, m32 = _main(d, 16, precision=32)
    for _ in range(3):
        advanceQ_RK4(m64, grid, None, util)
        advanceQ_RK4(m32, grid32, None, util)
    assert rel(np_(m32.Q).astype(np.complex128), np_(m64.Q)) < 1e-4


def test_cm1_has_no_rotating_form():
    d = golden("serial_N12.npz")
    grid, main = _main(d, 12, rotate=1)
    with pytest.raises(RuntimeError, match="no rotating form"):
        main.computeRHS(main, grid, None, None)
