"""Batched ensembles: many independent solves stepped by one batched
marching launch per group per step (fdtd_ensemble_*), and the seeded member
generator (casegen.ensemble_member).

CPU: the generator's draws (ranges, 2D half, determinism, files the
reference parser accepts) and the C ABI's argument checks.
GPU: every member of a batched run agrees with its own single solve (same
marching code and tile; the batched kernel is a separate compilation, so
the compiler may fuse multiply-adds differently: FP64 within 1e-13, FP32
within 1e-5 relative L2) and with the oracle within the FP64 / FP32
tolerances; horizons, parity after single steps, unsupported members, the
ensemble autotuner, the bounded-wait timeout path, and narrow tiles with
more receivers than threads."""

from __future__ import annotations

import ctypes
import importlib
import os

import numpy as np
import pytest

import cases
import oracle

pkg = importlib.import_module("3d_mpi_test_b200")
casegen = importlib.import_module("3d_mpi_test_b200.casegen")

SMALL = cases.ENS_SMALL


def rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n else float(np.linalg.norm(a - b))


def _members(tmp_path, n, steps, seed=11, wind="loglaw"):
    out = []
    for i in range(n):
        c, rec, p = casegen.ensemble_member(seed, i, pml=4, layer=4, steps=steps, n_receivers=3, sizes=SMALL,
                                            wind=wind)
        d = str(tmp_path / f"m{i}")
        c.write(d)
        out.append((d, rec, p))
    return out


# ------------------------------------------------------------------ CPU
def test_generator_draws_follow_the_workload():
    ps = [casegen.ensemble_member(0, i)[2] for i in range(48)]
    assert [p["two_d"] for p in ps] == [i % 2 == 0 for i in range(48)]
    for p in ps:
        assert 64 <= p["NJ"] <= 512 and 32 <= p["NK"] <= 192
        assert p["NI"] == 3 if p["two_d"] else 32 <= p["NI"] <= 96
        assert 1e4 <= p["sigma"] <= 2e6 and 0.2 <= p["porosity"] <= 0.6 and 1 <= p["tortuosity"] <= 2.5
        assert 0.1 <= p["source_height"] <= 3.0 and 0 <= p["hill_height"] <= 2.0 and 0 <= p["ustar"] <= 0.6
    # uneven sizes: the draws spread over the ranges
    assert np.ptp([p["NJ"] for p in ps]) > 200 and np.ptp([p["NK"] for p in ps]) > 80
    assert casegen.ensemble_member(0, 7)[2] == ps[7]
    assert casegen.ensemble_member(1, 7)[2] != ps[7]


def test_generated_members_write_reference_files(tmp_path):
    for i in range(256):  # every member of the 256-solve workload has a well-formed input.txt
        casegen.ensemble_member(0, i)[0].input_text()
    for i in (0, 1, 2, 3):
        c, rec, p = casegen.ensemble_member(3, i)
        d = c.write(str(tmp_path / f"m{i}"))
        txt = open(os.path.join(d, "input.txt")).read().split("\n")
        assert txt[3].split()[:6] == (["2", "3", "2", "2", "1", "1"] if p["two_d"] else ["2", "3", "2", "2", "2", "2"])
        assert os.path.exists(os.path.join(d, "coordi_pore1.dat"))
        if p["hill_height"] > 0:
            # the hill box bounds are grid nodes (air::cal_hill_var matches them within d/8)
            box = c.hill_box
            assert min(abs(np.array(c.Y) - box[2])) < 1e-12 and min(abs(np.array(c.Z) - box[5])) < 1e-12
            assert c.curve[0] == 1 and c.curve[2] == pytest.approx(p["hill_height"])


def test_ensemble_argument_checks():
    L = pkg.load_library()
    out = ctypes.c_void_p()
    assert L.fdtd_ensemble_create(None, 0, ctypes.byref(out)) == pkg.FDTD_ERR_ARG
    arr = (ctypes.c_void_p * 1)(None)
    assert L.fdtd_ensemble_create(arr, 1, ctypes.byref(out)) == pkg.FDTD_ERR_ARG
    assert not out.value
    assert L.fdtd_ensemble_destroy(None) == pkg.FDTD_OK
    assert L.fdtd_ensemble_advance(None, 1, None) == pkg.FDTD_ERR_ARG
    with pytest.raises(pkg.FdtdError):
        pkg.Ensemble([])


# ------------------------------------------------------------------ GPU
def _launches_per_step(case_dir, precision, tile) -> int:
    """Kernels one FB step of this member launches on its own (tiled
    members: one per tile kind present)."""
    with pkg.Airpore(case_dir, precision) as b:
        if tile:
            b.set_tiling(*tile)
        b.reset(2)
        n0 = b.launch_count()
        b.advance(1)
        return b.launch_count() - n0


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tile,mode", [("f32", None, 0), ("f64", None, 0), ("f32", (2, 3, 48, 2, 5), 0),
                                                 ("f64", (8, 7, 1000, 0, 0), 0), ("f32", None, 1),
                                                 ("f64", (3, 5, 32, 2, 5), 1)])
def test_batch_equals_single_solves(precision, tile, mode, tmp_path):
    steps = 37  # a graph of 16 steps twice plus 5 single launches
    # the row marching kernels (mode 0, explicit tilings) run only the
    # reference's forward-difference advection
    ms = _members(tmp_path, 6, steps, wind="reference" if (mode == 0 or tile) else "loglaw")
    mem = []
    for d, rec, _ in ms:
        a = pkg.Airpore(d, precision)
        a.set_receivers(rec)
        a.reset(steps)
        if tile:
            a.set_tiling(*tile)
        mem.append(a)
    with pkg.Ensemble(mem, mode=mode) as e:
        assert e.advance(7) == 7
        assert e.advance(steps) == steps - 7  # capped at the members' horizon
        info = e.info()
        # mode 1: each member's own launches (tiled members: one for the
        # full tiles and one for the lean tiles where both exist)
        per_step = info["groups"] if mode == 0 else sum(_launches_per_step(d, precision, tile) for d, _, _ in ms)
        assert info["launches"] == steps * per_step and info["blocks_per_step"] >= 6
    tol = 1e-10 if precision == "f64" else 1e-4
    same = 1e-13 if precision == "f64" else 1e-5  # batch vs single: rounding only
    for (d, rec, _), a in zip(ms, mem):
        with pkg.Airpore(d, precision) as b:
            b.set_receivers(rec)
            if tile:
                b.set_tiling(*tile)
            r = b.get_output(steps)
            assert rel(a.receivers(0, steps), r) <= same
            for f in "puvw":
                assert rel(a.field(f), b.field(f)) <= same, f
                assert rel(a.field(f, "pore"), b.field(f, "pore")) <= same, f
            sa, sb = a.slabs(), b.slabs()
            for s in sb:
                for c in "uvwp":
                    assert rel(sa[s][c], sb[s][c]) <= same, (s, c)
        o = oracle.run_case(d, rec, steps)
        assert rel(a.receivers(0, steps), o["receivers"]) <= tol
        for f in "puvw":
            assert rel(a.field(f), o[f]) <= tol, f
            assert rel(a.field(f, "pore"), o["pore_" + f]) <= tol, f
        a.close()


@pytest.mark.gpu
def test_members_stepped_alone_keep_their_parity(tmp_path):
    steps = 24
    ms = _members(tmp_path, 3, steps, seed=4)
    mem = []
    for d, rec, _ in ms:
        a = pkg.Airpore(d, "f64")
        a.set_receivers(rec)
        a.reset(steps)
        mem.append(a)
    mem[1].advance(3)  # one member runs ahead by an odd count
    with pkg.Ensemble(mem) as e:
        assert e.advance(steps) == steps - 3  # the nearest horizon bounds the step
        with pytest.raises(pkg.FdtdError) as err:
            e.advance(1)
        assert err.value.code == pkg.FDTD_ERR_STATE
    for (d, rec, _), a, n in zip(ms, mem, (steps - 3, steps, steps - 3)):
        o = oracle.run_case(d, rec, n)
        assert rel(a.receivers(0, n), o["receivers"]) <= 1e-10
        assert rel(a.field("p"), o["p"]) <= 1e-10
        a.close()


@pytest.mark.gpu
def test_unsupported_members_are_rejected(tmp_path):
    for name in ("fb_v_p", "moving_frame"):
        c, rec = cases.CASES[name]()
        d = str(tmp_path / name)
        c.write(d)
        with pkg.Airpore(d, "f32") as a:
            with pkg.Ensemble([a]) as e:
                with pytest.raises(pkg.FdtdError) as err:
                    e.advance(2)
                assert err.value.code == pkg.FDTD_ERR_UNSUPPORTED
    ms = _members(tmp_path, 2, 10)
    with pkg.Airpore(ms[0][0], "f32") as a, pkg.Airpore(ms[1][0], "f64") as b:
        with pytest.raises(pkg.FdtdError) as err:
            pkg.Ensemble([a, b])
        assert err.value.code == pkg.FDTD_ERR_ARG
        with pytest.raises(pkg.FdtdError):
            pkg.Ensemble([a, a])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_ensemble_autotune_keeps_results(mode, tmp_path):
    """Mode 0 tunes the batched row marching kernel's rows and plane chunk;
    mode 1 picks one set of tile shapes for every member's tiled kernels
    (returning the lean tiles' rows and planes)."""
    steps = 20
    ms = _members(tmp_path, 4, steps, seed=2, wind="reference" if mode == 0 else "loglaw")
    mem = []
    for d, rec, _ in ms:
        a = pkg.Airpore(d, "f32")
        a.set_receivers(rec)
        a.reset(steps)
        mem.append(a)
    with pkg.Ensemble(mem, mode=mode) as e:
        TI, GC = e.autotune(3)
        if mode == 0:
            assert TI in (2, 4, 8) and GC in (4, 8, 16, 32)
        else:
            assert TI in (8, 16) and GC in (8, 16, 32)
        assert e.advance(steps) == steps  # members were reset to t = 0 with their horizon
    for (d, rec, _), a in zip(ms, mem):
        o = oracle.run_case(d, rec, steps)
        assert rel(a.receivers(0, steps), o["receivers"]) <= 1e-4
        a.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_wait_timeout_is_reported_and_recoverable(precision, tmp_path):
    """A staged-copy wait allowed no polls gives up at once: the kernel
    records it, lets its copies land, and the step returns FDTD_ERR_TIMEOUT;
    the context stays usable and a reset run is correct again."""
    c, rec = cases.CASES["porous_tdbc_fine_pore"]()
    d = str(tmp_path / "case")
    c.write(d)
    tol = 1e-10 if precision == "f64" else 1e-4
    with pkg.Airpore(d, precision) as a:
        a.set_receivers(rec)
        a.reset(30)
        a.set_wait_limit(0)
        with pytest.raises(pkg.FdtdError) as err:
            a.advance(3)
        assert err.value.code == pkg.FDTD_ERR_TIMEOUT
        a.set_wait_limit(-1)
        a.reset(30)
        r = a.advance(30)
    o = oracle.run_case(d, rec, 30)
    assert rel(r, o["receivers"]) <= tol


@pytest.mark.gpu
def test_narrow_blocks_record_every_receiver(tmp_path):
    """A 1-thread-row tile of 4-column vectors has fewer threads than
    receivers; every receiver is still sampled each step."""
    c, _ = cases.CASES["pml_rigid"]()
    d = str(tmp_path / "case")
    c.write(d)
    rec = [(0.2 + 0.01 * (r % 20), 0.4 + 0.02 * (r // 20), 0.3) for r in range(40)]
    with pkg.Airpore(d, "f32") as a:
        a.set_receivers(rec)
        a.set_tiling(2, 1, 1, 4, 0)
        r = a.get_output(25)
    o = oracle.run_case(d, rec, 25)
    assert np.all(np.abs(r).max(axis=0) > 0)
    assert rel(r, o["receivers"]) <= 1e-4
