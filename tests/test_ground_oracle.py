"""Impedance ground (extension: the rigid south face as a 6-pole TDBC with
poles fitted to Miki's impedance) in the oracle and the fit, on the CPU:
the fit's accuracy, the rigid limit, the refusals, and the reflection
coefficient a plane wave meets at normal incidence against the scheme's own
discrete theory and against Miki's."""

import importlib

import numpy as np
import pytest

import cases
import oracle

casegen = importlib.import_module("3d_mpi_test_b200.casegen")
ground = importlib.import_module("3d_mpi_test_b200.ground")

SIGMA = 50e3  # Pa s/m^2, the long-range configuration's ground
DT_WINDOW = 0.5 * 0.05 / 343.0  # its time step (d = 0.05 m, CFL 0.5)
BANDS = np.array([50.0, 100.0, 200.0, 500.0, 1000.0, 2000.0])


def _rel(a, b):
    return np.abs(a - b) / np.abs(b)


def test_continuous_fit_matches_miki():
    fit = ground.fit_tdbc(SIGMA)
    assert fit.max_rel_err < 5e-3
    assert np.all(fit.a >= 0) and np.all(fit.r >= 0)


def test_discrete_fit_error_per_band():
    """The recursion's own response (time step of the long-range run)
    against Miki: within 2.5 % from 50 Hz to 1 kHz and 8 % at 2 kHz (a
    first-order recursion of real poles bends away from Miki's constant
    57-degree phase toward the Nyquist frequency, 6.9 kHz here)."""
    fit = ground.fit_tdbc(SIGMA, dt=DT_WINDOW)
    err = _rel(fit.impedance(BANDS), ground.miki_impedance(BANDS, SIGMA))
    assert np.all(err[:5] < 0.025), err
    assert err[5] < 0.08, err
    # passive: the real part of the impedance stays above zero everywhere
    f = np.linspace(1.0, 0.5 / DT_WINDOW, 4000)
    assert np.all(fit.impedance(f).real > 0)


def test_discrete_response_tends_to_continuous():
    a, r = np.array([0.8, 0.7, 0.5, 1.4, 3.8, 0.1]), np.array([1e-3, 0.07, 0.2, 0.6, 3.5, 20.0])
    f = np.array([100.0, 1000.0])
    zc = ground.tdbc_impedance(f, 411.6, 1e-3, a, r)
    zd = ground.tdbc_impedance(f, 411.6, 1e-3, a, r, dt=1e-8)
    assert np.all(_rel(zd, zc) < 1e-4)


def test_dat_round_trip(tmp_path):
    c, _ = cases.ground_box()
    d = c.write(str(tmp_path / "g"))
    tok = open(f"{d}/tdbc_ground.dat").read().split()
    assert len(tok) == 14
    Zinf, tau, a, r = c.ground_tdbc
    assert float(tok[0]) == Zinf and float(tok[1]) == tau
    assert [float(x) for x in tok[2:8]] == list(a) and [float(x) for x in tok[8:]] == list(r)


def test_rigid_limit(tmp_path):
    """A huge impedance without memory terms holds w(1) at p / Z ~ 0: the
    run equals the rigid ground's."""
    c, rec = cases.ground_box()
    c.ground_tdbc = None
    rigid = c.write(str(tmp_path / "rigid"))
    c.ground_tdbc = (1e15, 1e-3, (0.0,) * 6, (1.0,) * 6)
    stiff = c.write(str(tmp_path / "stiff"))
    a = oracle.run_case(rigid, rec, 40)
    b = oracle.run_case(stiff, rec, 40)
    for k in ["receivers", "p", "u", "v", "w"]:
        assert np.linalg.norm(a[k] - b[k]) <= 1e-9 * np.linalg.norm(a[k]), k


def test_ground_changes_the_field(tmp_path):
    c, rec = cases.ground_box()
    g = oracle.run_case(c.write(str(tmp_path / "g")), rec, 40)
    c.ground_tdbc = None
    r = oracle.run_case(c.write(str(tmp_path / "r")), rec, 40)
    assert np.linalg.norm(g["receivers"] - r["receivers"]) > 1e-3 * np.linalg.norm(r["receivers"])
    oc = oracle.OracleCase(str(tmp_path / "g"))
    oc.run(40)
    psi = oc.ground_psi()
    oc.close()
    assert psi.shape == (c.NI, c.NJ, 6) and np.abs(psi).max() > 0
    assert np.all(psi[0] == 0) and np.all(psi[:, 0] == 0)  # interior nodes only


@pytest.mark.parametrize("what", ["porous", "terrain", "fb_v_p", "pml_south"])
def test_refusals(what, tmp_path):
    if what == "porous":
        c, _ = cases.porous_ground()
    elif what == "terrain":
        c, _ = cases.hill_wind_pml6()
    elif what == "fb_v_p":
        c, _ = cases.fb_v_p()
    else:
        c, _ = cases.south_pml_all_faces()
    c.ground_tdbc = cases.miki_poles(SIGMA)
    with pytest.raises(RuntimeError, match="impedance ground"):
        oracle.OracleCase(c.write(str(tmp_path / what)))


def _column(tmp_path, d, poles, name):
    """A 3 x 5 x nk column, rigid sides, PML top: with a pressure pulse that
    is uniform across the column every interior node runs the same 1D
    scheme."""
    nk = int(round(3.0 / d)) + 40
    dt = 0.5 * d / 343.0
    rho0, gamma = 1.2, 1.4
    c = casegen.Case(
        X=casegen.uniform_axis(3, 0.0, d), Y=casegen.uniform_axis(5, 0.0, d), Z=casegen.uniform_axis(nk, 0.0, d),
        pml_nodes=(0, 0, 0, 0, 0, 40), gauss_width=6 * d, bc=(casegen.PML,) + (casegen.RIGID,) * 5,
        time_domain=10, gamma=gamma, P0=rho0 * 343.0 ** 2 / gamma, c0=343.0, source=(d, 2 * d, 2.0),
        receiver=(d, 2 * d, 1.0), dt=dt, ground_tdbc=poles)
    oc = oracle.OracleCase(c.write(str(tmp_path / name)))
    z = np.arange(nk) * d
    p0 = np.exp(-4 * np.log(2) / (6 * d) ** 2 * (z - 2.0) ** 2)
    oc.set_field("p", np.broadcast_to(p0, (3, 5, nk)).copy())
    oc.set_receivers([(d, 2 * d, 1.0)])
    steps = int(2.0 * 2.9 / 343.0 / dt)
    tr = oc.run(steps)[:, 0]
    oc.close()
    return tr, dt


def test_normal_incidence_reflection(tmp_path):
    """Pulse in a column at 2 m, receiver at 1 m: the rigid run's reflected
    pulse S (windowed) and the difference D of the impedance and rigid runs
    (no direct part) give R = 1 + D / S at the face. It matches the
    scheme's discrete theory (ground.normal_reflection) to 0.015 and
    Miki's plane-wave R to 0.02 from 200 Hz to 1 kHz (d = 1 cm)."""
    d = 0.01
    fit = ground.fit_tdbc(SIGMA, dt=0.5 * d / 343.0)
    poles = (fit.Zinf, fit.tau, tuple(fit.a), tuple(fit.r))
    rig, dt = _column(tmp_path, d, None, "rigid")
    imp, _ = _column(tmp_path, d, poles, "tdbc")
    t = np.arange(rig.size) * dt
    t2 = 3.0 / 343.0
    win = np.abs(t - t2) < 0.4 / 343.0
    n = 1 << 16
    S = np.fft.rfft(np.where(win, rig, 0.0), n)
    D = np.fft.rfft(imp - rig, n)
    f = np.fft.rfftfreq(n, dt)
    sel = [int(np.argmin(np.abs(f - fc))) for fc in (200.0, 500.0, 1000.0)]
    R = 1.0 + D[sel] / S[sel]
    Rth = ground.normal_reflection(fit.impedance(f[sel]), f[sel], dt, d)
    Rmiki = ground.reflection(ground.miki_impedance(f[sel], SIGMA))
    assert np.all(np.abs(R - Rth) < 0.015), (R, Rth)
    assert np.all(np.abs(R - Rmiki) < 0.02), (R, Rmiki)
