"""Checkpoint files in the reference's .npz layout: the keys, shapes and dtypes
that PySpectral/src/postProcessingFunctions.py:5-60 reads, and the
statistics file of PySpectral/src/PySpec_3d.py:145-148 (no GPU needed)."""
import types

import numpy as np

from pyspectral_b200 import checkpoint as ck
from pyspectral_b200.Classes import gridclass


def _main(N, turb_model, seed=0):
    rng = np.random.default_rng(seed)
    shape = (N, N, N // 2 + 1)
    f = [rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for _ in range(3)]
    Q = np.stack([x * 0.5 for x in f])
    m = types.SimpleNamespace(uhat=f[0], vhat=f[1], what=f[2], t=0.25, Q=Q, comp=None, W0=None, turb_model=turb_model)
    if turb_model != 0:
        m.W0 = np.stack([x * 2.0 for x in f])
        m.w0_u, m.w0_v, m.w0_w = (m.W0[i][..., None] for i in range(3))
    return m


def test_files_read_like_the_reference_post_processing(tmp_path):
    N = 8
    grid = gridclass.periodic(N)
    main = _main(N, 1)
    d = str(tmp_path / "3DSolution")
    ck.save_grid(grid, d)
    ck.save_runinfo(d, 1, 0.01, 5, 0.02)
    path = ck.savehook(main, grid, 5, d)
    assert path.endswith("npsol5.npz")
    gridFile, infoFile, sol = (np.load(f"{d}/{n}.npz") for n in ("grid", "runinfo", "npsol5"))
    # variablesFromFile (postProcessingFunctions.py:6-23)
    assert infoFile["turb_model"].mean() == 1
    uhat = np.zeros(np.shape(sol["uhat"]), dtype="complex")
    uhat[:, :, :] = sol["uhat"][:, :, :]
    assert np.array_equal(uhat, main.uhat)
    assert sol["uhat"].dtype == np.complex128 and sol["what"].shape == (N, N, N // 2 + 1)
    assert np.array_equal(sol["w0_v"][:, :, :, 0], main.W0[1])
    assert float(sol["t"]) == 0.25
    # gridFromFile (postProcessingFunctions.py:36-49)
    N1, N2, N3 = np.shape(sol["uhat"])
    N3 = (N3 - 1) * 2
    k1 = np.zeros((N1, N2, N3 // 2 + 1))
    k1[:, :, :] = gridFile["k1"]
    assert N3 == N and k1[1, 0, 0] == 1.0 and k1[N // 2, 0, 0] == -N // 2
    assert np.array_equal(gridFile["k3"][0, 0, :], np.arange(N // 2 + 1, dtype=float))
    # exact restart data
    assert np.array_equal(sol["Q"], main.Q)
    back = ck.load_solution(path)
    assert set(back) >= {"uhat", "vhat", "what", "t", "Q", "w0_u", "w0_v", "w0_w"}


def test_dns_solution_has_no_memory_fields(tmp_path):
    main = _main(8, 0)
    path = ck.savehook(main, gridclass.periodic(8), 0, str(tmp_path))
    assert "w0_u" not in ck.load_solution(path)


def test_stats_dissipation_is_the_reference_difference(tmp_path):
    t = np.array([0.0, 0.1, 0.2, 0.35])
    E = np.array([1.0, 0.9, 0.85, 0.8])
    Er = E * 0.5
    ck.save_stats(str(tmp_path), t, E, Er, E * 3)
    s = np.load(str(tmp_path / "stats.npz"))
    assert set(s.files) == {"Energy", "Dissipation", "Energy_resolved", "Dissipation_resolved", "t", "Enstrophy"}
    assert np.allclose(s["Dissipation"], 1.0 / (t[1:] - t[:-1]) * (E[1:] - E[:-1]), rtol=0, atol=0)
    assert np.allclose(s["Dissipation_resolved"], 1.0 / (t[1:] - t[:-1]) * (Er[1:] - Er[:-1]), rtol=0, atol=0)


def _fake_run(tmp_path, monkeypatch, reference_t0):
    """checkpoint.run with the step replaced by a host stand-in (energy decays
    by 10% a step), started at t = 0.25 as after a restart."""
    from pyspectral_b200 import RHSfunctions

    def step(main, grid, myFFT, utilities):
        main.e *= 0.9

    monkeypatch.setattr(RHSfunctions, "advanceQ_RK4", step)
    util = types.SimpleNamespace(
        computeEnergy=lambda m, g: m.e, computeEnstrophy=lambda m, g: 2 * m.e,
        computeEnergy_resolved=lambda m, g: 0.5 * m.e,
        computeAllStats=lambda m, g: (2 * m.e, m.e, 0.0, 0.0, 0.0, 0.0))
    main = _main(8, 0)
    main.e, main.dt, main.nu = 1.0, 0.05, 0.01
    return ck.run(main, gridclass.periodic(8), util, 0.39, 100, str(tmp_path / "3DSolution"),
                  turb_model=0, reference_t0=reference_t0)


def test_run_after_restart_starts_its_time_history_at_its_own_time(tmp_path, monkeypatch):
    s = _fake_run(tmp_path, monkeypatch, False)
    assert np.allclose(s["t"], [0.25, 0.30, 0.35, 0.40])
    assert np.allclose(s["Dissipation"][0], (0.9 - 1.0) / 0.05)


def test_run_reference_t0_writes_zero_first_as_the_reference(tmp_path, monkeypatch):
    s = _fake_run(tmp_path, monkeypatch, True)
    assert s["t"][0] == 0.0 and np.allclose(s["t"][1:], [0.30, 0.35, 0.40])
    assert np.allclose(s["Dissipation"][0], (0.9 - 1.0) / 0.30)
    on_disk = np.load(str(tmp_path / "3DSolution" / "stats.npz"))
    assert on_disk["t"][0] == 0.0
