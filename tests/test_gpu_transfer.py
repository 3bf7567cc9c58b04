"""Energy transfer spectrum (computeTransfer, src/Classes.py:988-1040) on the
GPU against the reference's own values (tests/golden) and the oracle."""
import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import golden, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_transfer_matches_reference(N, precision, tol):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    d = golden(f"serial_N{N}.npz")
    st = d["state"]
    grid = C.gridclass.periodic(N)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 1e-3, 0.01, precision=precision)
    Q0 = main.Q.clone()
    k, tr = C.utilitiesClass().computeTransfer(main, grid, None)
    np.testing.assert_array_equal(k, d["transfer_k"])
    assert rel(tr, d["transfer"]) < tol
    # the velocity views lose their Nyquist modes as in the reference; the state does not
    assert float(main.U[:, N // 2].abs().max()) == 0.0 and float(main.U[:, :, :, N // 2].abs().max()) == 0.0
    assert torch.equal(main.Q, Q0)


def test_transfer_conserves_energy_on_a_solenoidal_field():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    N = 32
    st = orc.isotropic_state(N, 4, k0=4.0)
    grid = C.gridclass.periodic(N)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 1e-3, 0.01)
    _, tr = C.utilitiesClass().computeTransfer(main, grid, None)
    _, ref = orc.transfer(orc.Grid.periodic(N), st)
    assert rel(tr, ref) < 1e-12
    assert abs(tr.real.sum()) < 1e-11 * np.abs(tr).sum()


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_resolved_and_sgs_transfer_match_reference(N, precision, tol):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    d = golden(f"serial_N{N}.npz")
    grid = C.gridclass.periodic(N, kc=N // 4)
    util = C.utilitiesClass()
    st = d["state"]
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 1e-3, 0.01, precision=precision)
    _, tr = util.computeTransfer_resolved(main, grid, None)
    assert rel(tr, d["transfer_res"]) < tol
    su = d["transfer_sgs_u"]
    main = C.variables(0, 1, 0, 0, 0, 0, grid, su[0], su[1], su[2], 0.0, 1e-3, 0.01, precision=precision)
    main.W0 = torch.as_tensor(d["transfer_sgs_w0"], device=main.Q.device).to(main.Q.dtype).contiguous()
    k, tr = util.computeTransfer_SGS(main, grid, None)
    np.testing.assert_array_equal(k, d["transfer_k"])
    assert rel(tr, d["transfer_sgs"]) < tol


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 2e-5)])
def test_2d_transfer_variants_match_reference(N, precision, tol):
    """computeTransfer_2D / _resolved_2D / _SGS_2D (src/Classes.py:1043-1092,
    1152-1205, 1241-1270): the k3 = 0 plane binned by |k_h|."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    d = golden(f"serial_N{N}.npz")
    util = C.utilitiesClass()
    st = d["state"]
    grid = C.gridclass.periodic(N)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 1e-3, 0.01, precision=precision)
    k, tr = util.computeTransfer_2D(main, grid, None)
    np.testing.assert_array_equal(k, d["transfer2d_k"])
    assert rel(tr, d["transfer2d"]) < tol
    grid = C.gridclass.periodic(N, kc=N // 4)
    main = C.variables(0, 0, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, 1e-3, 0.01, precision=precision)
    _, tr = util.computeTransfer_resolved_2D(main, grid, None)
    assert rel(tr, d["transfer2d_res"]) < tol
    su = d["transfer_sgs_u"]
    main = C.variables(0, 1, 0, 0, 0, 0, grid, su[0], su[1], su[2], 0.0, 1e-3, 0.01, precision=precision)
    main.W0 = torch.as_tensor(d["transfer_sgs_w0"], device=main.Q.device).to(main.Q.dtype).contiguous()
    k, tr = util.computeTransfer_SGS_2D(main, grid, None)
    np.testing.assert_array_equal(k, d["transfer2d_k"])
    assert rel(tr, d["transfer2d_sgs"]) < tol
