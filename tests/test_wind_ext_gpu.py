"""Log-law wind (method 7) and upwind velocity advection on the B200
against the oracle's restatement (extensions of the reference: checked
against the oracle only), through the C ABI."""

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
def ext_dirs(tmp_path_factory):
    root = tmp_path_factory.mktemp("ext")
    made = {}
    for name, fn in cases.EXT_CASES.items():
        c, rec = fn()
        d = str(root / name)
        c.write(d)
        made[name] = (d, rec, c.time_domain)
    return made


def _errors(a, ref, r, slabs=True):
    errs = {"receivers": rel_l2(r, ref["receivers"])}
    for f in "puvw":
        errs[f] = rel_l2(a.field(f), ref[f])
        if a.has_pore:
            errs["pore_" + f] = rel_l2(a.field(f, "pore"), ref["pore_" + f])
    if slabs:
        errs["psi"] = rel_l2(a.psi(), ref["psi"])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel_l2(sl[s][c], q[c])
    return errs


@pytest.mark.parametrize("name", sorted(cases.EXT_CASES))
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_wind_extensions_match_oracle(name, precision, ext_dirs):
    d, rec, n = ext_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, precision) as a:
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = _errors(a, ref, r, slabs=precision == "f64")
    assert max(errs.values()) <= (TOL_F64 if precision == "f64" else TOL_F32), errs


@pytest.mark.parametrize("shapes", [((2, 2, 1, 3), (3, 5, 2, 4), (2, 2, 3, 4)), ((8, 8, 9, 5), (8, 16, 7, 6),
                                                                                (4, 8, 64, 5))])
@pytest.mark.parametrize("name", ["wind_loglaw_upwind", "hill_loglaw_upwind", "wind_vortex_upwind"])
def test_upwind_tile_shapes(name, shapes, ext_dirs):
    """Upwind advection reads the backward neighbours from the staged boxes:
    exact for any tile shape (halo rows and vectors, warm-up planes)."""
    d, rec, n = ext_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        for kind in range(3):
            a.set_tile_shape(kind, *shapes[kind])
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = _errors(a, ref, r)
    assert max(errs.values()) <= TOL_F64, errs


def test_upwind_half_steps_and_refusals(ext_dirs):
    """The two-pass kernels (half steps) read the same backward neighbours;
    the row marching kernel has no upwind form and refuses."""
    d, rec, _ = ext_dirs["wind_loglaw_upwind"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(10)
        for _ in range(6):
            a.Cal_pressure()
            a.Cal_velocity()
        half = {f: a.field(f) for f in "puvw"}
        with pytest.raises(pkg.FdtdError) as e:
            a.set_tiling(4, 8, 256)
        assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
    with pkg.Airpore(d, "f64") as b:
        b.get_output(6)
        for f in "puvw":
            assert rel_l2(half[f], b.field(f)) <= 1e-13, f


def test_log_law_with_upwind_stays_bounded(tmp_path):
    """Config 3's log wind (u* = 0.4 m/s, z0 = 0.01 m) at d = 0.05 m over a
    porous ground with upwind advection: 3000 steps, both precisions,
    bounded and finite."""
    c, rec = cases.wind_loglaw_upwind()
    c.logwind = (0.41, 0.01)
    c.velocity_coef = 0.4
    c.time_domain = 3000
    d = str(tmp_path / "lw")
    c.write(d)
    for prec in ("f32", "f64"):
        with pkg.Airpore(d, prec) as a:
            a.set_receivers(rec)
            r = a.get_output(3000)
            p = a.field("p")
        assert np.all(np.isfinite(p)) and np.abs(p).max() < 0.5, prec
        assert np.all(np.isfinite(r)) and np.abs(r).max() < 1.0, prec
