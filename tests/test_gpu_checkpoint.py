"""A run driven by the reference's loop writes its 3DSolution files; a restart
from a solution file continues it bit for bit (exact state and Kahan
compensation in the file)."""
import numpy as np
import pytest

from oracle import spectral_oracle as orc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,turb,kw", [(64, 1, {}), (32, 0, {}), (64, 2, {}), (64, 7, {}), (64, 6, {}),
                                               (32, 3, dict(dt0=0.02, dt0_subintegrations=2))])
def test_restart_continues_the_run_exactly(tmp_path, precision, turb, kw):
    """Memory models (turb_model 3, 6) carry their memory variables in Q; the
    file's Q restores them with the velocity."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyspectral_b200 import Classes as C
    from pyspectral_b200 import checkpoint as ck
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    N, dt, nu = 16, 1e-3, 0.02
    st = orc.isotropic_state(N, 3, k0=3.0)
    grid = C.gridclass.periodic(N)
    util = C.utilitiesClass()
    d = str(tmp_path / "3DSolution")
    a = C.variables(0, turb, 0, 0, 0, 0, grid, st[0], st[1], st[2], 0.0, dt, nu, precision=precision, **kw)
    stats = ck.run(a, grid, util, et=5.5e-3, save_freq=3, directory=d)
    assert len(stats["t"]) == 7 and np.isfinite(stats["Energy"]).all() and len(stats["Dissipation"]) == 6
    sol = ck.load_solution(f"{d}/npsol3.npz")
    assert sol["t"] == pytest.approx(3e-3)  # the start of the step that produced it
    if turb in (3, 6):
        assert sol["Q"].shape[0] == a.Q.shape[0] and np.abs(sol["Q"][3:]).max() > 0
        assert sol["w0_u"].shape[-1] == kw.get("dt0_subintegrations", 1)
    b = ck.restart(f"{d}/npsol3.npz", grid, turb, dt, nu, precision=precision, **kw)
    t = b.t
    for _ in range(2):
        b.t = t
        advanceQ_RK4(b, grid, None, util)
        t += dt
    assert t == pytest.approx(a.t)
    assert torch.equal(b.Q, a.Q)
    if precision == 32:
        assert torch.equal(b.comp, a.comp)
