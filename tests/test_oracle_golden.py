"""Pin the CPU oracle to the reference: fixtures produced by running the
unmodified PySpectral sources (tests/golden/make_golden.py) and the
reference's own known-answer TGV energy history."""
import numpy as np
import pytest

from oracle import spectral_oracle as orc
from tests.helpers import CASES, DT, NU, T, golden, rel

FN = {"dns": orc.rhs_nosgs, "smag": orc.rhs_smag, "tmodel": orc.rhs_tmodel, "stau": orc.rhs_staumodel,
      "dtau": orc.rhs_dtaumodel, "dsmag": orc.rhs_dsmag, "cm1": orc.rhs_cm1, "budgets": orc.rhs_budgets,
      "fm1": lambda g, st, p: orc.rhs_fm1(g, st, p, dt0=0.05)}


def _fn(name):
    return FN[name.split("_")[0]]


def _read(name, res, Q):
    base = name.split("_")[0]
    if base == "dns":
        return res[1]
    if base in ("smag", "dsmag"):
        return Q
    return res[2]


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name", list(CASES))
def test_rhs_and_step_match_reference(N, name):
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT, **CASES[name][2])
    st = d["state"]
    if CASES[name][0] in (3, 6):  # memory models: the memory variables start at zero
        st = np.concatenate([st, np.zeros_like(st)])
    res = _fn(name)(g, st, p)
    assert rel(res[0], d[f"{name}_rhs"]) < 1e-13
    if f"{name}_w0" in d:
        assert rel(res[1], d[f"{name}_w0"]) < 1e-13
    if f"{name}_tau" in d:
        assert abs(res[3] - float(d[f"{name}_tau"])) <= 1e-13 * max(1.0, abs(float(d[f"{name}_tau"])))
    Q, read = orc.advance_rk4(st, lambda q: (lambda r: (r[0], _read(name, r, q)))(_fn(name)(g, q, p)), DT)
    assert rel(Q, d[f"{name}_step"]) < 1e-13
    assert rel(read, d[f"{name}_step_uhat"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
def test_dsmag_fractional_cutoff_matches_reference(N):
    """Dynamic Smagorinsky with kc = N/2 - 1: the test filter kc/2 is
    fractional and myFilter truncates it (src/RHSfunctions.py:1697,
    src/Classes.py:1271-1279)."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N, kc=N // 2 - 1)
    p = orc.Params(nu=NU, t=T, dt=DT)
    st = d["state"]
    r, w0, cs2 = orc.rhs_dsmag(g, st, p)
    assert rel(r, d["dsmag_kc_rhs"]) < 1e-13
    assert rel(w0, d["dsmag_kc_w0"]) < 1e-13
    Q, _ = orc.advance_rk4(st, lambda q: (orc.rhs_dsmag(g, q, p)[0], q), DT)
    assert rel(Q, d["dsmag_kc_step"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
def test_cm1_with_memory_matches_reference(N):
    """CM1 from non-zero memory variables: the reference reads w0_v as zero
    (src/Classes.py:489) while its slot of the state still evolves."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT)
    st = np.concatenate([d["state"], d["cm1w_init"]])
    r, w0, ur = orc.rhs_cm1(g, st, p)
    assert rel(r, d["cm1w_rhs"]) < 1e-13
    assert rel(w0, d["cm1w_w0"]) < 1e-13
    assert rel(ur, d["cm1w_uhat"]) < 1e-13
    assert np.abs(d["cm1w_w0"][1]).max() == 0.0 and np.abs(d["cm1w_init"][1]).max() > 0
    Q, _ = orc.advance_rk4(st, lambda q: (orc.rhs_cm1(g, q, p)[0], q), DT)
    assert rel(Q, d["cm1w_step"]) < 1e-13
    with pytest.raises(ValueError):
        orc.rhs_cm1(g, st, orc.Params(nu=NU, rotate=1, Om=(0.1, 0.2, 0.3)))


@pytest.mark.parametrize("N", [12, 16])
def test_budgets_match_reference(N):
    """computeRHS_BUDGETS' PL and PLQL, and the budget file its hooks write
    around a step at iteration 20 (src/Classes.py:632-649)."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT)
    st = d["state"]
    r, plql, _ = orc.rhs_budgets(g, st, p)
    assert rel(r, d["budgets_plu"]) < 1e-13
    assert rel(plql, d["budgets_plql"]) < 1e-13
    # the file: last stage's PL/PLQL, rates of change over the step
    gk = orc.Grid.periodic(N, kc=N // 4)
    last = {}

    def f(q):
        r, plql, read = orc.rhs_budgets(gk, q, p)
        last.update(r=r, plql=plql, read=read)
        return r, read
    Q, read = orc.advance_rk4(st, f, DT)
    assert rel(Q, d["budgetfile_step"]) < 1e-13
    assert rel(last["plql"], np.stack([d[f"budgetfile_PLQL{c}"] for c in "uvw"])) < 1e-13
    assert rel(last["r"][0], d["budgetfile_PLu"]) < 1e-13
    assert rel((read[0] - st[0]) / DT, d["budgetfile_u_dot"]) < 1e-12
    w1, _ = orc.sgs_dns(gk, read)
    w0, _ = orc.sgs_dns(gk, st)
    for i, c in enumerate("uvw"):
        assert rel((w1[i] - w0[i]) / DT, d[f"budgetfile_w0_{c}dot"][..., 0]) < 1e-12
    with pytest.raises(ValueError):
        orc.rhs_budgets(g, st, orc.Params(nu=NU, rotate=1, Om=(0.1, 0.2, 0.3)))


@pytest.mark.parametrize("N", [12, 16])
def test_fm1_three_subintegrations_match_reference(N):
    """FM1 with dt0 = 0.08 in three subintegrations from non-zero memory
    variables (fixtures made with pad_2x for the reference's undefined
    pad_2x_var)."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT)
    st = np.concatenate([d["state"], d["fm1w_init"].reshape(9, *d["state"].shape[1:])])
    r, _, ur = orc.rhs_fm1(g, st, p, dt0=0.08, nsub=3)
    assert rel(r, d["fm1w_rhs"]) < 1e-13
    assert rel(ur, d["fm1w_uhat"]) < 1e-13
    Q, _ = orc.advance_rk4(st, lambda q: (orc.rhs_fm1(g, q, p, dt0=0.08, nsub=3)[0], q), DT)
    assert rel(Q, d["fm1w_step"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("case", ["fm2t", "fm2tw"])
def test_fm1_two_term_matches_reference(N, case):
    """turb_model 5 (no undefined names: the reference runs as written)."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT)
    mem = d["fm2t_init"].reshape(6, *d["state"].shape[1:]) if case == "fm2tw" else np.zeros((6,) + d["state"].shape[1:])
    st = np.concatenate([d["state"], mem])
    r, ur = orc.rhs_fm1_2term(g, st, p, dt0=0.04)
    assert rel(r, d[f"{case}_rhs"]) < 1e-13
    assert rel(ur, d[f"{case}_uhat"]) < 1e-13
    Q, _ = orc.advance_rk4(st, lambda q: (orc.rhs_fm1_2term(g, q, p, dt0=0.04)[0], q), DT)
    assert rel(Q, d[f"{case}_step"]) < 1e-13
    # the same as FM1 with two subintegrations of 2 dt0
    r1, _, _ = orc.rhs_fm1(g, st, p, dt0=0.08, nsub=2)
    assert rel(r1, r) < 1e-14


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,okw", [("ortho", {}), ("ortho_rot", dict(rotate=1, Om=(0.3, 0.1, -0.2)))])
def test_orthogonal_dynamics_matches_reference(N, name, okw):
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N, kc=N // 4)
    p = orc.Params(nu=NU, t=T, dt=DT, **okw)
    st = d["state"]
    r, ur = orc.rhs_orthogonal(g, st, p)
    assert rel(r, d[f"{name}_rhs"]) < 1e-13
    assert rel(ur, d[f"{name}_uhat"]) < 1e-13
    Q, read = orc.advance_rk4(st, lambda q: orc.rhs_orthogonal(g, q, p), DT)
    assert rel(Q, d[f"{name}_step"]) < 1e-13
    assert rel(read, d[f"{name}_step_uhat"]) < 1e-13


def test_myfilter_slice_semantics():
    """myFilter keeps rows [0:kc] and [-kc+1:]; kc = 1 makes the second slice
    [0:], the whole axis (Python slicing), and kc = 0 keeps nothing."""
    g = orc.Grid.periodic(8)
    m1, m2, m3 = orc.myfilter_axes(g, 3)
    np.testing.assert_array_equal(m1, [1, 1, 1, 0, 0, 0, 1, 1])
    np.testing.assert_array_equal(m3, [1, 1, 1, 0, 0])
    m1, _, m3 = orc.myfilter_axes(g, 1)
    np.testing.assert_array_equal(m1, np.ones(8))
    np.testing.assert_array_equal(m3, [1, 0, 0, 0, 0])
    m1, _, m3 = orc.myfilter_axes(g, 2.5)
    np.testing.assert_array_equal(m1, [1, 1, 0, 0, 0, 0, 0, 1])
    assert orc.myfilter_axes(g, 0)[2].sum() == 0


@pytest.mark.parametrize("N", [12, 16])
def test_diagnostics_match_reference(N):
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N, kc=int(d["diag_kc"]))
    st = d["state"]
    assert orc.energy(g, st) == pytest.approx(float(d["energy"]), rel=1e-14)
    assert orc.energy_resolved(g, st) == pytest.approx(float(d["energy_resolved"]), rel=1e-14)
    assert orc.enstrophy(g, st) == pytest.approx(float(d["enstrophy"]), rel=1e-14)
    np.testing.assert_allclose(np.array(orc.all_stats(g, st, NU)), d["allstats"], rtol=1e-13)
    k, s = orc.spectrum(g, st)
    np.testing.assert_array_equal(k, d["spectrum_k"])
    assert rel(s, d["spectrum"]) < 1e-14
    _, s = orc.spectrum(g, st, filtered=True)
    assert rel(s, d["spectrum_res"]) < 1e-14
    w0, _ = orc.sgs_dns(g, st)
    assert np.abs(d["sgs_dns_w0"]).max() > 1e-3
    assert rel(w0, d["sgs_dns_w0"]) < 1e-13
    assert orc.compute_dt(g, st, 0.4, NU, DT) == pytest.approx(float(d["cfl_dt"]), rel=1e-14)


@pytest.mark.parametrize("N", [12, 16])
def test_transfer_matches_reference(N):
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    k, tr = orc.transfer(g, d["state"])
    np.testing.assert_array_equal(k, d["transfer_k"])
    assert rel(tr, d["transfer"]) < 1e-13
    # on a solenoidal field the dealiased nonlinear term only moves energy
    # between shells (the fixture state is not solenoidal)
    _, tr = orc.transfer(g, orc.isotropic_state(N, 3, k0=3.0))
    assert abs(tr.real.sum()) < 1e-12 * np.abs(tr).sum()
    gq = orc.Grid.periodic(N, kc=N // 4)
    _, tr = orc.transfer(gq, d["state"], filtered=True)
    assert rel(tr, d["transfer_res"]) < 1e-13
    _, tr = orc.transfer(gq, d["transfer_sgs_u"], w0=d["transfer_sgs_w0"])
    assert np.abs(d["transfer_sgs"]).max() > 1e-4
    assert rel(tr, d["transfer_sgs"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
def test_transfer_2d_matches_reference(N):
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    k, tr = orc.transfer(g, d["state"], two_d=True)
    np.testing.assert_array_equal(k, d["transfer2d_k"])
    assert rel(tr, d["transfer2d"]) < 1e-13
    gq = orc.Grid.periodic(N, kc=N // 4)
    _, tr = orc.transfer(gq, d["state"], filtered=True, two_d=True)
    assert rel(tr, d["transfer2d_res"]) < 1e-13
    _, tr = orc.transfer(gq, d["transfer_sgs_u"], w0=d["transfer_sgs_w0"], two_d=True)
    assert np.abs(d["transfer2d_sgs"]).max() > 1e-5
    assert rel(tr, d["transfer2d_sgs"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
def test_mhd_matches_reference(N):
    d = golden(f"mhd_N{N}.npz")
    g = orc.MHDGrid(N, N, N, N // 2)
    nu, dt = float(d["nu"]), float(d["dt"])
    x, y, z = orc.periodic_coords(N)
    assert rel(orc.mhd_forcing(g, x, y, z), d["force"]) < 1e-13
    r, _ = orc.rhs_mhd(g, d["state"], nu, force=d["force"])
    assert rel(r, d["rhs"]) < 1e-13
    Q, _ = orc.advance_rk4(d["state"], lambda q: (orc.rhs_mhd(g, q, nu, force=d["force"])[0], None), dt)
    assert rel(Q, d["step"]) < 1e-13
    ds = d["diag_state"]
    assert orc.mhd_energy(g, ds[:3]) == pytest.approx(float(d["energy_u"]), rel=1e-14)
    assert orc.mhd_energy(g, ds[3:]) == pytest.approx(float(d["energy_B"]), rel=1e-14)
    assert rel(orc.mhd_spectrum(g, ds[:3])[1], d["spectrum_u"]) < 1e-13
    assert rel(orc.mhd_spectrum(g, ds[3:])[1], d["spectrum_B"]) < 1e-13


def test_tgv64_known_answer_start():
    """First 5 steps of the reference's TGV validation run (64^3, nu=1/100,
    dt=0.010005) against its shipped energy history.  The shipped history
    was produced with slightly different settings (its E agrees with the
    reference code itself only to ~2.5e-4), so the bound is 5e-4."""
    b = golden("tgv64_benchmark.npz")
    t, E = b["t"], b["Energy"]
    N = 64
    g = orc.Grid.periodic(N)
    orc.set_workers(4)
    try:
        st = orc.tgv_state(N)
        assert orc.energy(g, st) == pytest.approx(0.125, rel=1e-14)
        assert orc.enstrophy(g, st) == pytest.approx(3 * 0.125, rel=1e-14)
        p = orc.Params(nu=0.01)
        dt = t[2] - t[1]
        Q = st
        for n in range(1, 6):
            Q, read = orc.advance_rk4(Q, lambda q: orc.rhs_nosgs(g, q, p), dt)
            assert abs(orc.energy(g, read) - E[n]) / E[n] < 5e-4
    finally:
        orc.set_workers(1)


def test_analytic_properties_of_the_oracle():
    """Single-mode RHS = -nu k^2 uhat; divergence-free DNS RHS."""
    N = 12
    g = orc.Grid.periodic(N)
    st = np.zeros((3, N, N, N // 2 + 1), dtype=complex)
    st[1, 2, 0, 0] = 3.0 + 1.0j  # v(k=(2,0,0)) : transverse, k.u = 0
    st[1, N - 2, 0, 0] = 3.0 - 1.0j
    r, _ = orc.rhs_nosgs(g, st, orc.Params(nu=0.1))
    expect = -0.1 * g.ksqr * st
    assert rel(r, expect) < 1e-13
    d = orc.isotropic_state(N, 3)
    r, _ = orc.rhs_nosgs(g, d, orc.Params(nu=0.01))
    div = g.k1 * r[0] + g.k2 * r[1] + g.k3 * r[2]
    assert np.abs(div).max() < 1e-10 * np.abs(r).max()


@pytest.mark.parametrize("N,kc", [(12, 6), (16, 8), (16, 7), (12, 3)])
def test_dsmag_coefficient_by_parseval(N, kc):
    """The GPU forms Cs^2 as a spectral sum (k3 > 0 twice, the Hermitian part
    of the k3 = 0 plane, modes pad() drops excluded) instead of means over the
    3/2 grid; by Parseval the two agree."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N, kc=kc)
    u, v, w = d["state"]
    ref = orc.dsmag_cs2(g, u, v, w)
    kL = kc / 2.0
    k1, k2, k3 = g.k1, g.k2, g.k3
    s = orc.scale_32(g)
    P = orc._products_32(g, u, v, w)
    PF = orc._products_32(g, *(orc.myfilter(g, x, kL) for x in (u, v, w)))

    def ss(a, b, c):
        Sh = (1j * k1 * a, 1j * k2 * b, 1j * k3 * c, 0.5 * (1j * k2 * a + 1j * k1 * b),
              0.5 * (1j * k3 * a + 1j * k1 * c), 0.5 * (1j * k3 * b + 1j * k2 * c))
        S = [orc.ifft32(g, orc.pad(x) * s) for x in Sh]
        mag = np.sqrt(2.0 * (S[0] ** 2 + S[1] ** 2 + S[2] ** 2 + 2 * S[3] ** 2 + 2 * S[4] ** 2 + 2 * S[5] ** 2))
        return [orc.unpad(orc.fft32(mag * x)) for x in S]
    A6 = ss(u, v, w)
    B6 = ss(*(orc.myfilter(g, x, kL) for x in (u, v, w)))
    L = np.stack([orc.myfilter(g, P[m], kL) - PF[m] for m in range(6)])
    M = np.stack([-2 * g.Delta ** 2 * (4 * B6[m] - orc.myfilter(g, A6[m], kL)) for m in range(6)])
    keep = np.ones(L.shape[1:], bool)
    keep[N // 2] = keep[:, N // 2] = keep[:, :, N // 2] = False
    wgt = np.where(np.arange(N // 2 + 1) > 0, 2.0, 0.0)[None, None, :] * keep
    num = np.sum(wgt * np.real(L * np.conj(M)))
    den = np.sum(wgt * np.abs(M) ** 2)
    neg = (-np.arange(N)) % N
    Lm, Mm = L[:, :, :, 0], M[:, :, :, 0]
    Mp = M[:, neg][:, :, neg, 0]
    k0 = keep[:, :, 0]
    num += np.sum(k0 * (0.5 * np.real(Lm * np.conj(Mm)) + 0.5 * np.real(Lm * Mp)))
    den += np.sum(k0 * (0.5 * np.abs(Mm) ** 2 + 0.5 * np.real(Mm * Mp)))
    assert num / den == pytest.approx(ref, rel=1e-12)


MPI_NS = [("dns", 0, False), ("dns_rot", 1, False), ("ortho", 0, True), ("ortho_rot", 1, True)]


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,rot,ortho", MPI_NS)
def test_mpi_navier_stokes_matches_reference(N, name, rot, ortho):
    """The MPI solver's Navier-Stokes (turb_model 0) and orthogonal dynamics
    (src_MPI/RHSfunctions.py:22-93, 179-268), one RHS and one RK4 step."""
    d = golden(f"mpi_ns_N{N}.npz")
    g = orc.MHDGrid(N, N, N, int(d["kc"]))
    nu, dt = float(d["nu"]), float(d["dt"])
    Om = (0.2, -0.3, 0.4)
    r, s = orc.rhs_mpi_ns(g, d["state"], nu, rot, Om, ortho)
    assert rel(r, d[f"{name}_rhs"]) < 1e-13
    assert rel(s, d[f"{name}_uhat"]) < 1e-13
    Q, _ = orc.advance_rk4(d["state"], lambda q: orc.rhs_mpi_ns(g, q, nu, rot, Om, ortho), dt)
    assert rel(Q, d[f"{name}_step"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("name,rot", [("si", 0), ("si_rot", 1)])
def test_mpi_semi_implicit_matches_reference(N, name, rot):
    """Two AB2/Crank-Nicolson steps of the MPI solver (H zeroed first)."""
    d = golden(f"mpi_ns_N{N}.npz")
    g = orc.MHDGrid(N, N, N, int(d["kc"]))
    nu, dt = float(d["nu"]), float(d["dt"])
    Q, H = d["state"], np.zeros_like(d["state"])
    for k in (1, 2):
        Q, H = orc.step_mpi_si(g, Q, H, nu, dt, rot, (0.2, -0.3, 0.4))
        assert rel(Q, d[f"{name}_step{k}"]) < 1e-13
        assert rel(H, d[f"{name}_H{k}"]) < 1e-13


@pytest.mark.parametrize("N", [12, 16])
@pytest.mark.parametrize("case", ["fm2", "fm2w"])
def test_fm2_matches_reference(N, case):
    """turb_model 4 (second-order finite memory model; the oracle only, the
    GPU path is not built): fresh with one subintegration each, and from
    non-zero memory variables with two each (interleaved w0/w1 layout)."""
    d = golden(f"serial_N{N}.npz")
    g = orc.Grid.periodic(N)
    p = orc.Params(nu=NU, t=T, dt=DT)
    st = d["state"]
    if case == "fm2":
        nsub, full = 1, np.concatenate([st, np.zeros((6,) + st.shape[1:], complex)])
    else:
        nsub = 2
        full = np.zeros((15,) + st.shape[1:], complex)
        full[:3] = st
        o0, o1 = orc.fm2_layout(2)
        for i in range(2):
            full[o0[i]:o0[i] + 3] = d["fm2w_init"][i]
            full[o1[i]:o1[i] + 3] = d["fm2w_init"][2 + i]

    def f(q):
        return orc.rhs_fm2(g, q, p, dt0=0.05, dt1=0.03, nsub=nsub)
    r, ur = f(full)
    assert rel(r, d[f"{case}_rhs"]) < 1e-13
    assert rel(ur, d[f"{case}_uhat"]) < 1e-13
    Q, _ = orc.advance_rk4(full, f, DT)
    assert rel(Q, d[f"{case}_step"]) < 1e-13
