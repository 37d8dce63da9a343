"""Terrain-following grid on the B200 (config 2's hill): the CUDA path
against the oracle's restatement (the reference itself pins its cross
metrics to zero, so this extension is checked against the oracle only),
through the C ABI. FP64: relative L2 <= 1e-10 for receivers, final fields
of both media, the TDBC state and every PML slab; FP32 <= 1e-4."""

import copy
import importlib

import numpy as np
import pytest

import cases
import oracle

pkg = importlib.import_module("3d_mpi_test_b200")
casegen = importlib.import_module("3d_mpi_test_b200.casegen")

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-10
TOL_F32 = 1e-4


def rel_l2(x, y):
    n = np.linalg.norm(y)
    return float(np.linalg.norm(x - y) / n) if n > 0 else float(np.linalg.norm(x - y))


@pytest.fixture(scope="module")
def terrain_dirs(tmp_path_factory):
    root = tmp_path_factory.mktemp("terrain")
    made = {}
    for name, fn in cases.TERRAIN_CASES.items():
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


@pytest.mark.parametrize("name", sorted(cases.TERRAIN_CASES))
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_terrain_matches_oracle(name, precision, terrain_dirs):
    d, rec, n = terrain_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, precision) as a:
        idx = a.set_receivers(rec)
        np.testing.assert_array_equal(idx, ref["rec_index"])
        r = a.get_output(n)
        errs = _errors(a, ref, r, slabs=precision == "f64")
    assert max(errs.values()) <= (TOL_F64 if precision == "f64" else TOL_F32), errs


@pytest.mark.parametrize("shapes", [((2, 2, 1, 3), (3, 5, 2, 4), (2, 2, 3, 3)), ((16, 8, 40, 5), (8, 32, 7, 6),
                                                                                (4, 16, 64, 5))])
@pytest.mark.parametrize("name", ["hill_porous", "hill_wind_pml6"])
def test_terrain_tile_shapes(name, shapes, terrain_dirs):
    """Any tile shape of the three tile kinds gives the oracle's solve on the
    terrain grid (halo rows and vectors, warm-up planes, faces)."""
    d, rec, n = terrain_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        for kind in range(3):
            a.set_tile_shape(kind, *shapes[kind])
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = _errors(a, ref, r)
    assert max(errs.values()) <= TOL_F64, errs


def test_terrain_half_steps(terrain_dirs):
    """Cal_pressure + Cal_velocity (two-pass kernels) on the terrain grid
    equal the fused time loop."""
    d, rec, _ = terrain_dirs["hill_porous"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(10)
        for _ in range(6):
            a.Cal_pressure()
            a.Cal_velocity()
        half = {f: a.field(f) for f in "puvw"}
    with pkg.Airpore(d, "f64") as b:
        b.get_output(6)
        for f in "puvw":
            assert rel_l2(half[f], b.field(f)) <= 1e-13, f


def test_terrain_refusals(terrain_dirs, tmp_path):
    """The row marching kernel, the contour writer and the moving frame have
    no terrain-following form: each is refused with FDTD_ERR_UNSUPPORTED."""
    d, rec, _ = terrain_dirs["hill_porous"]
    with pkg.Airpore(d, "f64") as a:
        with pytest.raises(pkg.FdtdError) as e:
            a.set_tiling(4, 8, 256)
        assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
        with pytest.raises(pkg.FdtdError) as e:
            a.get_data_contour(str(tmp_path / "c.dat"))
        assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
    c, _ = cases.moving_frame()
    c.terrain = [0.02] * c.NJ
    dm = str(tmp_path / "mf")
    c.write(dm)
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Airpore(dm, "f64")
    assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED


def test_hill_workload_stays_bounded(tmp_path):
    """The bench's hill workload (h = 0.5 m, w = 1 m, full height) on a
    quarter of its footprint runs 2000 steps in both precisions with a
    bounded, finite field: the stretched, sloped cells stay inside the
    scheme's stability limit."""
    c, rec = casegen.porous_hill(ni=64, nj=128, nk=96, layer=16, pml=20, seed=1, steps=2000)
    d = str(tmp_path / "hill")
    c.write(d)
    for prec in ("f32", "f64"):
        with pkg.Airpore(d, prec) as a:
            a.set_receivers(rec)
            r = a.get_output(2000)
            p = a.field("p")
        assert np.all(np.isfinite(p)) and np.abs(p).max() < 1.0, prec
        assert np.all(np.isfinite(r)) and np.abs(r[1000:]).max() < 0.5, prec
