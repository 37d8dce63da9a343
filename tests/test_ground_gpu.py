"""Impedance ground (the rigid south face as a 6-pole TDBC with poles
fitted to Miki's impedance; extension of the reference, whose TDBC acts on
the east face only) on the B200 against the oracle's restatement, through
the C ABI: receivers, fields, both TDBC states and every PML slab."""

import importlib

import numpy as np
import pytest

import cases
import oracle

pkg = importlib.import_module("3d_mpi_test_b200")

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-10
TOL_F32 = 1e-4


def rel_l2(x, y):
    n = np.linalg.norm(y)
    return float(np.linalg.norm(x - y) / n) if n > 0 else float(np.linalg.norm(x - y))


@pytest.fixture(scope="module")
def ground_dirs(tmp_path_factory):
    root = tmp_path_factory.mktemp("ground")
    made = {}
    for name, fn in cases.GROUND_CASES.items():
        c, rec = fn()
        d = str(root / name)
        c.write(d)
        made[name] = (d, rec, c.time_domain)
    return made


def _oracle(d, rec, n):
    ref = oracle.run_case(d, rec, n)
    oc = oracle.OracleCase(d)
    oc.run(n)
    ref["ground_psi"] = oc.ground_psi()
    oc.close()
    return ref


def _errors(a, ref, r, slabs=True):
    errs = {"receivers": rel_l2(r, ref["receivers"])}
    for f in "puvw":
        errs[f] = rel_l2(a.field(f), ref[f])
    errs["ground_psi"] = rel_l2(a.ground_psi(), ref["ground_psi"])
    if slabs:
        errs["psi"] = rel_l2(a.psi(), ref["psi"])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel_l2(sl[s][c], q[c])
    return errs


@pytest.mark.parametrize("name", sorted(cases.GROUND_CASES))
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_ground_matches_oracle(name, precision, ground_dirs):
    d, rec, n = ground_dirs[name]
    ref = _oracle(d, rec, n)
    with pkg.Airpore(d, precision) as a:
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = _errors(a, ref, r, slabs=precision == "f64")
    assert max(errs.values()) <= (TOL_F64 if precision == "f64" else TOL_F32), errs


@pytest.mark.parametrize("shapes", [((2, 2, 1, 3), (3, 5, 2, 4), (2, 2, 3, 4)), ((8, 8, 9, 5), (8, 16, 7, 6),
                                                                                (4, 8, 64, 5))])
def test_ground_tile_shapes(shapes, ground_dirs):
    """The ground kernel runs after the step whatever the tiles were."""
    d, rec, n = ground_dirs["ground_loglaw_tdbc_east"]
    ref = _oracle(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        for kind in range(3):
            a.set_tile_shape(kind, *shapes[kind])
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = _errors(a, ref, r)
    assert max(errs.values()) <= TOL_F64, errs


def _per_step(d):
    with pkg.Airpore(d, "f64") as b:
        b.reset(40)
        b.advance(1)
        l0 = b.launch_count()
        b.advance(1)
        return b.launch_count() - l0


def test_ground_half_steps_and_launches(ground_dirs, tmp_path):
    """Cal_velocity applies the ground too; one extra launch per step."""
    d, rec, _ = ground_dirs["ground_box"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(10)
        for _ in range(6):
            a.Cal_pressure()
            a.Cal_velocity()
        half = {f: a.field(f) for f in "puvw"}
        gpsi = a.ground_psi()
    with pkg.Airpore(d, "f64") as c:
        c.get_output(6)
        for f in "puvw":
            assert rel_l2(half[f], c.field(f)) <= 1e-13, f
        assert rel_l2(gpsi, c.ground_psi()) <= 1e-13
    plain, _ = cases.ground_box()
    plain.ground_tdbc = None
    assert _per_step(d) == _per_step(plain.write(str(tmp_path / "plain"))) + 1


def test_ground_refusals(ground_dirs, tmp_path):
    d, rec, _ = ground_dirs["ground_box"]
    with pkg.Airpore(d, "f64") as a:
        with pytest.raises(pkg.FdtdError) as e:
            a.Save_restart(str(tmp_path / "r.txt"))
        assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
        with pytest.raises(pkg.FdtdError) as e:
            pkg.Ensemble([a])
        assert e.value.code == pkg.FDTD_ERR_ARG
    c, _ = cases.porous_ground()
    c.ground_tdbc = cases.miki_poles(50e3)
    p = c.write(str(tmp_path / "porous"))
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Airpore(p, "f64")
    assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
    c, _ = cases.pml_rigid()
    with pkg.Airpore(c.write(str(tmp_path / "plain")), "f64") as a:
        with pytest.raises(pkg.FdtdError) as e:
            a.ground_psi()
        assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED


def test_loglaw_over_ground_stays_bounded(tmp_path):
    """Config 3's physics (log wind u* = 0.4 m/s, z0 = 0.01 m, upwind
    advection, Miki ground at 50 kPa s/m^2) for 3000 steps at d = 0.05 m,
    both precisions: finite, bounded, FP32 within 1e-4 of FP64 on the
    receivers."""
    c, rec = cases.ground_loglaw_tdbc_east()
    c.time_domain = 3000
    d = c.write(str(tmp_path / "lw"))
    out = {}
    for prec in ("f64", "f32"):
        with pkg.Airpore(d, prec) as a:
            a.set_receivers(rec)
            r = a.get_output(3000)
            p = a.field("p")
        assert np.all(np.isfinite(p)) and np.abs(p).max() < 0.5, prec
        assert np.all(np.isfinite(r)) and np.abs(r).max() < 1.0, prec
        out[prec] = r
    assert rel_l2(out["f32"], out["f64"]) <= TOL_F32
