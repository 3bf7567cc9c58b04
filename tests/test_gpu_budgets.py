"""GPU parity of the DNS-with-SGS-budgets run (turb_model 99,
PySpectral/src/RHSfunctions.py:1543-1661, hooks src/Classes.py:632-649):
PL and PLQL of one RHS, and the budget file written around a step at
iteration 20, against the reference's own outputs."""
import os

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


def _main(d, N, kc=None, rotate=0):
    from pyspectral_b200 import Classes as C
    grid = C.gridclass.periodic(N) if kc is None else C.gridclass.periodic(N, kc=kc)
    st = d["state"]
    return grid, C.variables(0, 99, rotate, 0.1, 0.2, 0.3, grid, st[0], st[1], st[2], T, DT, NU)


@pytest.mark.parametrize("N", [12, 16])
def test_budget_terms_match_reference(N):
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(d, N)
    main.computeRHS(main, grid, None, None)
    assert rel(np.stack([np_(main.PLu), np_(main.PLv), np_(main.PLw)]), d["budgets_plu"]) < TOL64
    assert rel(np.stack([np_(main.PLQLu), np_(main.PLQLv), np_(main.PLQLw)]), d["budgets_plql"]) < TOL64


@pytest.mark.parametrize("N", [12, 16])
def test_budget_file_matches_reference(N, tmp_path):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    _torch()
    d = golden(f"serial_N{N}.npz")
    grid, main = _main(d, N, kc=N // 4)
    main.iteration = 20
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        advanceQ_RK4(main, grid, None, C.utilitiesClass())
        with np.load(os.path.join("3DSolution", "budget20.npz")) as b:
            files = {k: b[k] for k in b.files}
    finally:
        os.chdir(cwd)
    assert rel(np_(main.Q), d["budgetfile_step"]) < TOL64
    keys = sorted(k[len("budgetfile_"):] for k in d.files if k.startswith("budgetfile_") and k != "budgetfile_step")
    assert sorted(files) == keys
    for k in keys:
        assert files[k].shape == d["budgetfile_" + k].shape
        assert files[k].dtype == d["budgetfile_" + k].dtype
        assert rel(files[k], d["budgetfile_" + k]) < 1e-11, k


def test_no_budget_file_off_the_20_step_cadence(tmp_path):
    from pyspectral_b200 import Classes as C
    from pyspectral_b200.RHSfunctions import advanceQ_RK4
    _torch()
    d = golden("serial_N12.npz")
    grid, main = _main(d, 12)
    main.iteration = 7
    cwd = os.getcwd()
    os.chdir(tmp_path)
    try:
        advanceQ_RK4(main, grid, None, C.utilitiesClass())
        assert not os.path.exists("3DSolution")
    finally:
        os.chdir(cwd)


def test_budgets_have_no_rotating_form():
    _torch()
    d = golden("serial_N12.npz")
    grid, main = _main(d, 12, rotate=1)
    with pytest.raises(RuntimeError, match="no rotating form"):
        main.computeRHS(main, grid, None, None)
