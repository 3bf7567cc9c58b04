"""GPU parity of the orthogonal dynamics ('Orthogonal Dynamics',
PySpectral/src/RHSfunctions.py:53-143) against the reference's own outputs
(kc = N/4, so that Gf u differs from u)."""
import numpy as np
import pytest

from tests.helpers import DT, NU, T, golden, rel

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,rot", [("ortho", (0, 0.0, 0.0, 0.0)), ("ortho_rot", (1, 0.3, 0.1, -0.2))])
def test_orthogonal_dynamics_matches_reference(N, name, rot):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    d = golden(f"serial_N{N}.npz")
    st = d["state"]
    grid = C.gridclass.periodic(N, kc=N // 4)
    main = C.variables(0, "Orthogonal Dynamics", *rot, grid, st[0], st[1], st[2], T, DT, NU)
    main.computeRHS(main, grid, None, None)
    assert rel(np_(main.Q), d[f"{name}_rhs"]) < TOL64
    assert rel(np_(main.U), d[f"{name}_uhat"]) < TOL64
    main = C.variables(0, "Orthogonal Dynamics", *rot, grid, st[0], st[1], st[2], T, DT, NU)
    advanceQ_RK4(main, grid, None, C.utilitiesClass())
    assert rel(np_(main.Q), d[f"{name}_step"]) < TOL64
    assert rel(np_(main.U), d[f"{name}_step_uhat"]) < TOL64
    m32 = C.variables(0, "Orthogonal Dynamics", *rot, grid, st[0], st[1], st[2], T, DT, NU, precision=32)
    m32.computeRHS(m32, grid, None, None)
    assert rel(np_(m32.Q).astype(np.complex128), d[f"{name}_rhs"]) < 2e-5
