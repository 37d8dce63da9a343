"""B200 parity: the CUDA path against the oracle, through the C ABI.

FP64: relative L2 <= 1e-10 for receiver p(t), final p/u/v/w of both media,
the TDBC state and every PML integral slab.
FP32: relative L2 <= 1e-4 for receivers and final pressure against the FP64
oracle (FP32 fields and stencil; FP64 TDBC state and receiver series)."""

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


def _gpu_run(case_dir, rec, nsteps, precision):
    with pkg.Airpore(case_dir, precision) as a:
        idx = a.set_receivers(rec)
        r = a.get_output(nsteps)
        out = {"receivers": r, "rec_index": idx}
        for f in "puvw":
            out[f] = a.field(f)
            if a.has_pore:
                out["pore_" + f] = a.field(f, "pore")
        out["psi"] = a.psi()
        out["slabs"] = a.slabs()
        out["launches"] = a.launch_count()
    return out


@pytest.fixture(scope="module")
def case_dirs(tmp_path_factory):
    root = tmp_path_factory.mktemp("cases")
    made = {}
    for name, fn in cases.CASES.items():
        c, rec = fn()
        d = str(root / name)
        c.write(d)
        made[name] = (d, rec, c.time_domain)
    return made


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_fp64_matches_oracle(name, case_dirs):
    d, rec, n = case_dirs[name]
    ref = oracle.run_case(d, rec, n)
    got = _gpu_run(d, rec, n, "f64")
    np.testing.assert_array_equal(got["rec_index"], ref["rec_index"])
    errs = {"receivers": rel_l2(got["receivers"], ref["receivers"])}
    for f in "puvw":
        errs[f] = rel_l2(got[f], ref[f])
        if "pore_" + f in ref:
            errs["pore_" + f] = rel_l2(got["pore_" + f], ref["pore_" + f])
    errs["psi"] = rel_l2(got["psi"], ref["psi"])
    assert set(got["slabs"]) == set(ref["slabs"])
    for s, q in ref["slabs"].items():
        for c in "uvwp":
            errs[f"Q{c}_{s}"] = rel_l2(got["slabs"][s][c], q[c])
    assert max(errs.values()) <= TOL_F64, errs
    assert got["launches"] >= n  # at least one kernel per step ran on the device


@pytest.mark.parametrize("name", ["pml_rigid", "porous_ground", "tdbc_east", "moving_frame", "wind_log", "hill1"])
def test_fp32_within_tolerance(name, case_dirs):
    d, rec, n = case_dirs[name]
    ref = oracle.run_case(d, rec, n)
    got = _gpu_run(d, rec, n, "f32")
    assert rel_l2(got["receivers"], ref["receivers"]) <= TOL_F32
    assert rel_l2(got["p"], ref["p"]) <= TOL_F32


def test_half_steps_match_full_step(case_dirs):
    """Cal_pressure + Cal_velocity (half steps) equal one time-loop step."""
    d, rec, _ = case_dirs["tdbc_east"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(10)
        for _ in range(5):
            a.Cal_pressure()
            a.Cal_velocity()
        p_half = a.field("p")
    with pkg.Airpore(d, "f64") as b:
        b.get_output(5)
        p_full = b.field("p")
    # half steps run the two-pass kernels, the time loop the fused pass
    assert rel_l2(p_half, p_full) <= 1e-13


def test_pressure_half_step_matches_oracle(case_dirs):
    """After one Cal_pressure, the new pressure level (p_nn) equals the
    oracle's p after one full step (the velocity half step does not touch p)."""
    d, rec, _ = case_dirs["porous_ground"]
    ref = oracle.run_case(d, rec, 1)
    with pkg.Airpore(d, "f64") as a:
        a.reset(1)
        a.Cal_pressure()
        assert rel_l2(a.field("p", level="nn"), ref["p"]) <= TOL_F64
        assert rel_l2(a.field("p", "pore", level="nn"), ref["pore_p"]) <= TOL_F64


def test_linearity_exact(case_dirs):
    """The update is linear and x2 is exact in binary floating point, so
    doubling the initial pressure doubles every output bit for bit."""
    d, rec, n = case_dirs["porous_tdbc_fine_pore"]
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(n)
        r1 = a.advance(n)
        p1 = a.field("p")
        a.reset(n)
        pa, pp = a.field("p"), a.field("p", "pore")  # read both before writing: they share two rows
        a.set_field("p", 2.0 * pa)
        a.set_field("p", 2.0 * pp, "pore")
        r2 = a.advance(n)
        p2 = a.field("p")
    assert np.array_equal(r2, 2.0 * r1)
    assert np.array_equal(p2, 2.0 * p1)


def test_errors_are_reported(tmp_path):
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Airpore(str(tmp_path / "missing"), "f64")
    assert e.value.code == pkg.FDTD_ERR_INPUT
    c, rec = cases.pml_rigid()
    c.scheme = 5  # RK4: the reference prints "wrong with scheme name" and never steps
    d = str(tmp_path / "rk4")
    c.write(d)
    with pytest.raises(pkg.FdtdError) as e:
        pkg.Airpore(d, "f64")
    assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED


def test_horizon_state_error(case_dirs):
    d, rec, _ = case_dirs["pml_rigid"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(3)
        a.advance(3)
        with pytest.raises(pkg.FdtdError) as e:
            a.advance(1)
        assert e.value.code == pkg.FDTD_ERR_STATE


def test_nonfinite_watchdog(case_dirs):
    """A non-finite pressure is reported with FDTD_ERR_NONFINITE (host-side
    check of a device flag; the context stays usable)."""
    d, rec, _ = case_dirs["pml_rigid"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(5)
        p = a.field("p")
        p[5, 10, 5] = np.inf
        a.set_field("p", p)
        with pytest.raises(pkg.FdtdError) as e:
            a.advance(2)
        assert e.value.code == pkg.FDTD_ERR_NONFINITE
        a.reset(5)
        a.advance(2)  # usable after the error


# (rows, planes, threads, vector width, ring stages): thread counts round
# down to whole thread rows of NJP / width column-vector threads; rings from
# the minimum to the maximum depth (planes in flight)
TILINGS = [(2, 1, 1, 0, 0), (3, 5, 32, 2, 5), (8, 7, 1000, 0, 0), (4, 16, 64, 2, 0), (5, 3, 48, 0, 7),
           (4, 4, 256, 0, 12)]


@pytest.mark.parametrize("tiling", TILINGS)
@pytest.mark.parametrize("name", ["porous_tdbc_fine_pore", "south_pml_all_faces", "wind_log", "moving_frame",
                                  "odd_columns_wind", "odd_columns_porous"])
def test_fused_tilings_match_oracle(name, tiling, case_dirs):
    """The fused FB_p_v pass is exact for any tile shape: halo rows,
    warm-up planes, odd row splits, single-plane chunks."""
    d, rec, n = case_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        a.set_tiling(*tiling)
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = {"receivers": rel_l2(r, ref["receivers"])}
        for f in "puvw":
            errs[f] = rel_l2(a.field(f), ref[f])
        errs["psi"] = rel_l2(a.psi(), ref["psi"])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel_l2(sl[s][c], q[c])
    assert max(errs.values()) <= TOL_F64, errs


def test_autotune_keeps_results_exact(case_dirs):
    d, rec, n = case_dirs["porous_ground"]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f32") as a:
        best = a.autotune(4)
        assert best[0] >= 2 and best[1] >= 1 and best[2] >= 1 and best[3] in (2, 4) and best[4] >= 3
        a.set_receivers(rec)
        r = a.get_output(n)
    assert rel_l2(r, ref["receivers"]) <= TOL_F32


def test_fused_and_two_pass_agree(case_dirs):
    """FB_v_p still runs the two-pass kernels; FB_p_v the fused pass. Both
    are pinned to the oracle above; here the FB_p_v half-step API (two-pass
    kernels) is checked against the fused time loop for the same state."""
    d, rec, _ = case_dirs["hill2"]
    with pkg.Airpore(d, "f64") as a:
        a.reset(8)
        for _ in range(4):
            a.Cal_pressure()
            a.Cal_velocity()
        p2 = a.field("p")
    with pkg.Airpore(d, "f64") as b:
        b.get_output(4)
        p1 = b.field("p")
    assert rel_l2(p1, p2) <= 1e-13


def test_half_step_past_horizon_is_state_error(case_dirs):
    """Cal_pressure samples receivers into a buffer of `horizon` steps, so a
    half step at the horizon is refused before any launch and the handle
    stays usable."""
    d, rec, _ = case_dirs["pml_rigid"]
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(2)
        for _ in range(2):
            a.Cal_pressure()
            a.Cal_velocity()
        launches = a.launch_count()
        with pytest.raises(pkg.FdtdError) as e:
            a.Cal_pressure()
        assert e.value.code == pkg.FDTD_ERR_STATE
        assert a.launch_count() == launches
        with pytest.raises(pkg.FdtdError) as e:
            a.receivers(1, 2)  # steps 1..2 are not all taken: only 0 and 1 are
        assert e.value.code == pkg.FDTD_ERR_ARG
        assert a.receivers(0, 2).shape == (2, len(rec))
        a.reset(2)
        a.Cal_pressure()  # usable again after a reset


# (rows, vectors, planes, ring stages) of the full, the lean and the
# single-layer PML tiles of the tiled kernel: single-row / single-vector /
# single-plane tiles at the minimum ring depth, odd splits, tiles larger
# than the domain, deep rings
TILE_SHAPES = [((2, 2, 1, 3), (2, 2, 1, 3), (2, 2, 1, 3)), ((3, 5, 2, 4), (5, 3, 3, 3), (3, 3, 5, 4)),
               ((16, 8, 40, 5), (8, 32, 7, 6), (4, 16, 64, 5)), ((4, 16, 5, 12), (16, 16, 64, 3), (16, 8, 3, 12))]


@pytest.mark.parametrize("shapes", TILE_SHAPES)
@pytest.mark.parametrize("name", ["porous_tdbc_fine_pore", "south_pml_all_faces", "wind_log", "moving_frame",
                                  "odd_columns_wind", "odd_columns_porous", "narrow_y", "hill5", "delayed_y1",
                                  "pml_box_all", "pml_box_wind_porous"])
def test_tile_shapes_match_oracle(name, shapes, case_dirs):
    """The tiled kernel is exact for any tile shape: full, lean and
    single-layer PML tiles, halo rows and column vectors, warm-up planes,
    face rows and columns."""
    d, rec, n = case_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, "f64") as a:
        for kind in range(3):
            a.set_tile_shape(kind, *shapes[kind])
        assert a.tile_shape()["tiled"]
        a.set_receivers(rec)
        r = a.get_output(n)
        errs = {"receivers": rel_l2(r, ref["receivers"])}
        for f in "puvw":
            errs[f] = rel_l2(a.field(f), ref[f])
            if a.has_pore:
                errs["pore_" + f] = rel_l2(a.field(f, "pore"), ref["pore_" + f])
        errs["psi"] = rel_l2(a.psi(), ref["psi"])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel_l2(sl[s][c], q[c])
    assert max(errs.values()) <= TOL_F64, errs


@pytest.mark.parametrize("name", ["pml_box_all", "pml_box_wind_porous"])
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_single_layer_tiles_match_oracle(name, precision, case_dirs):
    """Domains wide enough for tiles inside one PML layer: every field, slab
    and receiver against the oracle, with the single-layer launches
    present (one per layer axis)."""
    d, rec, n = case_dirs[name]
    ref = oracle.run_case(d, rec, n)
    with pkg.Airpore(d, precision) as a:
        ts = a.tile_shape()
        assert ts["tiled"] and ts["pml"]["tiles"] > 0
        a.set_receivers(rec)
        l0 = a.launch_count()
        r = a.get_output(n)
        assert (a.launch_count() - l0) >= 3 * n  # full, lean and at least one single-layer launch per step
        errs = {"receivers": rel_l2(r, ref["receivers"])}
        for f in "puvw":
            errs[f] = rel_l2(a.field(f), ref[f])
            if a.has_pore:
                errs["pore_" + f] = rel_l2(a.field(f, "pore"), ref["pore_" + f])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel_l2(sl[s][c], q[c])
    assert max(errs.values()) <= (TOL_F64 if precision == "f64" else TOL_F32), errs


def test_kernel_selection(case_dirs):
    """FB_p_v runs the tiled kernel by default (a lean launch and one per
    PML / face layer set present, besides the generic full tiles);
    set_tiling selects the row marching kernel (one launch per step) and
    set_tile_shape the tiled one again; all three agree to rounding."""
    d, rec, n = case_dirs["porous_ground"]
    with pkg.Airpore(d, "f64") as a:
        ts = a.tile_shape()
        assert ts["tiled"] and ts["pml"]["tiles"] > 0 and ts["lean"]["tiles"] > 0
        a.set_receivers(rec)
        l0 = a.launch_count()
        r1 = a.get_output(n)
        per_step = (a.launch_count() - l0) // n
        assert a.launch_count() - l0 == per_step * n and 2 <= per_step <= 10
        a.set_tiling(4, 8, 256)
        assert not a.tile_shape()["tiled"]
        l0 = a.launch_count()
        r2 = a.get_output(n)
        assert a.launch_count() - l0 == n
        a.set_tile_shape(0, 8, 16, 16, 4)
        assert a.tile_shape()["tiled"]
        r3 = a.get_output(n)
    assert rel_l2(r2, r1) <= 1e-13 and rel_l2(r3, r1) <= 1e-13


def test_rows_wider_than_row_marching_kernel(case_dirs):
    """1300 columns: only the tiled kernel runs this domain (the row marching
    kernel refuses its tiling), in both precisions."""
    d, rec, n = case_dirs["very_wide_2d"]
    ref = oracle.run_case(d, rec, n)
    for prec, tol in (("f64", TOL_F64), ("f32", TOL_F32)):
        with pkg.Airpore(d, prec) as a:
            assert a.tile_shape()["tiled"]
            with pytest.raises(pkg.FdtdError) as e:
                a.set_tiling(2, 8, 256)
            assert e.value.code == pkg.FDTD_ERR_UNSUPPORTED
            a.set_receivers(rec)
            r = a.get_output(n)
            errs = {"receivers": rel_l2(r, ref["receivers"]), "p": rel_l2(a.field("p"), ref["p"]),
                    "pore_p": rel_l2(a.field("p", "pore"), ref["pore_p"])}
        assert max(errs.values()) <= tol, (prec, errs)
