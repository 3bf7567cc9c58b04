"""GPU parity of the MPI solver's Navier-Stokes (turb_model 0,
PySpectral/src_MPI/RHSfunctions.py:22-93) and orthogonal dynamics (:179-268):
2/3-rule dealiasing on the N grid, with and without rotation, against the
reference's own outputs."""
import numpy as np
import pytest

from tests.helpers import golden, rel

pytestmark = pytest.mark.gpu
CASES = [("dns", 0, (0, 0.0, 0.0, 0.0)), ("dns_rot", 0, (1, 0.2, -0.3, 0.4)),
         ("ortho", "Orthogonal Dynamics", (0, 0.0, 0.0, 0.0)),
         ("ortho_rot", "Orthogonal Dynamics", (1, 0.2, -0.3, 0.4))]


def np_(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,tm,rot", CASES)
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_mpi_navier_stokes_matches_reference(N, name, tm, rot, precision, tol):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import mpi as M
    d = golden(f"mpi_ns_N{N}.npz")
    nu, dt = float(d["nu"]), float(d["dt"])
    grid = M.gridclass.periodic(N, kc=int(d["kc"]))
    x = [np.fft.irfftn(d["state"][i], s=(N, N, N), axes=(0, 1, 2)) for i in range(3)]
    zero = np.zeros((N, N, N))

    def make():
        return M.variables(tm, *rot, grid, *x, zero, zero, zero, t=0.0, dt=dt, nu=nu, precision=precision)
    main = make()
    assert main.Q.shape[0] == 3
    assert rel(np_(main.Q).astype(np.complex128), d["state"]) < (1e-13 if precision == 64 else 1e-6)
    main.computeRHS(main, grid, None)
    assert rel(np_(main.Q).astype(np.complex128), d[f"{name}_rhs"]) < tol
    assert rel(np_(main.U).astype(np.complex128), d[f"{name}_uhat"]) < tol
    main = make()
    M.advanceQ_RK4(main, grid, None)
    assert rel(np_(main.Q).astype(np.complex128), d[f"{name}_step"]) < tol


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,rot", [("si", (0, 0.0, 0.0, 0.0)), ("si_rot", (1, 0.2, -0.3, 0.4))])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_mpi_semi_implicit_matches_reference(N, name, rot, precision, tol):
    """advanceQ_SI (src_MPI/time_schemes.py:9-11), two steps from H = 0."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import mpi as M
    d = golden(f"mpi_ns_N{N}.npz")
    nu, dt = float(d["nu"]), float(d["dt"])
    grid = M.gridclass.periodic(N, kc=int(d["kc"]))
    x = [np.fft.irfftn(d["state"][i], s=(N, N, N), axes=(0, 1, 2)) for i in range(3)]
    zero = np.zeros((N, N, N))
    main = M.variables(0, *rot, grid, *x, zero, zero, zero, t=0.0, dt=dt, nu=nu, precision=precision,
                       time_scheme="Semi-Implicit")
    for k in (1, 2):
        main.advanceQ(main, grid, None)
        assert rel(np_(main.Q).astype(np.complex128), d[f"{name}_step{k}"]) < tol
        assert rel(np_(main.H).astype(np.complex128), d[f"{name}_H{k}"]) < tol
    with pytest.raises(ValueError):
        M.variables("Orthogonal Dynamics", 0, 0, 0, 0, grid, *x, zero, zero, zero, dt=dt, nu=nu,
                    time_scheme="Semi-Implicit")
