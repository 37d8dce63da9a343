"""Restart files in the reference's format (airpore::Save_restart /
Read_restart).

GPU, against the compiled reference (oracle/_ref/ref_harness, which writes
its restart with the reference's save_restartfile and reads one with its
input_restartfile):
  - the file this library writes equals the reference's, line for line and
    token for token to the printed precision;
  - continuing from the reference's own restart file with reference
    semantics reproduces the reference's continuation (FP64 tolerance);
  - an exact save / load / continue round trip -- moving frame and TDBC
    included, through this library's extra block -- agrees with the
    uninterrupted run to the 11-digit precision of the text format."""

from __future__ import annotations

import importlib
import os
import subprocess

import numpy as np
import pytest

import cases
import refio

pkg = importlib.import_module("3d_mpi_test_b200")
pytestmark = pytest.mark.gpu


def rel(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / n) if n else float(np.linalg.norm(a - b))


def _write(tmp_path, name):
    c, rec = cases.CASES[name]()
    d = str(tmp_path / name)
    c.write(d)
    rf = os.path.join(d, "rec.txt")
    with open(rf, "w") as f:
        f.write("\n".join(" ".join(map(str, r)) for r in rec))
    return d, rec, rf


def _harness():
    if not os.path.exists(refio.REF_HARNESS):
        pytest.skip("oracle/_ref/ref_harness not built")
    return refio.REF_HARNESS


def _lines(path):
    return [ln.split() for ln in open(path).read().split("\n") if ln.strip()]


@pytest.mark.parametrize("name", ["porous_tdbc_fine_pore", "pml_rigid", "wind_log"])
def test_restart_file_matches_reference(name, tmp_path):
    h = _harness()
    d, rec, rf = _write(tmp_path, name)
    subprocess.run([h, d, "--steps", "12", "--out", d + "/a.bin", "--restart-out", d + "/ref.dat"], check=True)
    with pkg.Airpore(d, "f64") as a:
        a.reset(100)
        a.advance(12)
        a.Save_restart(d + "/mine.dat")
    ref, mine = _lines(d + "/ref.dat"), _lines(d + "/mine.dat")
    assert mine[0] == ref[0]  # "size rank index"
    assert mine[len(ref)][0] == "B200" and len(mine) == len(ref) + 2  # this library's extra block
    for lr, lm in zip(ref[1:], mine[1:]):
        assert len(lr) == len(lm)
        x, y = np.array(lr, float), np.array(lm, float)
        scale = np.max(np.abs(x))
        # 11 printed digits: the FP64 states agree far below the last digit
        assert np.all(np.abs(x - y) <= 1e-10 * np.abs(x) + 1e-12 * scale)


@pytest.mark.parametrize("name", ["porous_tdbc_fine_pore", "delayed_y1", "wind_log"])
def test_continue_from_reference_restart(name, tmp_path):
    h = _harness()
    d, rec, rf = _write(tmp_path, name)
    subprocess.run([h, d, "--steps", "12", "--out", d + "/a.bin", "--restart-out", d + "/ref.dat"], check=True)
    subprocess.run([h, d, "--steps", "9", "--restart-in", d + "/ref.dat", "--out", d + "/b.bin",
                    "--receivers", rf], check=True)
    ref = refio.read_dump(d + "/b.bin")
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(100)
        a.Read_restart(d + "/ref.dat", reference_semantics=True)
        r = a.advance(9)
        errs = {"receivers": rel(r, ref["receivers"])}
        for f in "puvw":
            errs[f] = rel(a.field(f), ref[f])
        sl = a.slabs()
        for s, q in ref["slabs"].items():
            for c in "uvwp":
                errs[f"Q{c}_{s}"] = rel(sl[s][c], q[c])
    assert max(errs.values()) <= 1e-10, errs


@pytest.mark.parametrize("name,save_at", [("moving_frame", 30), ("moving_frame", 47), ("porous_tdbc_fine_pore", 13),
                                          ("tdbc_east", 20)])
def test_exact_round_trip(name, save_at, tmp_path):
    d, rec, _ = _write(tmp_path, name)
    more = 10
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(save_at + more)
        r_full = a.advance(save_at + more)
        full = {f: a.field(f) for f in "puvw"}
        psi = a.psi()
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(save_at + more)
        a.advance(save_at)
        a.Save_restart(d + "/ct.dat")
    with pkg.Airpore(d, "f64") as a:
        a.set_receivers(rec)
        a.reset(save_at + more)
        a.Read_restart(d + "/ct.dat")
        r = a.advance(more)
        assert rel(r, r_full[save_at:]) <= 1e-9
        for f in "puvw":
            assert rel(a.field(f), full[f]) <= 1e-9, f
        assert rel(a.psi(), psi) <= 1e-9


def test_restart_errors(tmp_path):
    d, rec, _ = _write(tmp_path, "pml_rigid")
    with pkg.Airpore(d, "f64") as a:
        a.reset(20)
        with pytest.raises(pkg.FdtdError) as e:
            a.Read_restart(d + "/missing.dat")
        assert e.value.code == pkg.FDTD_ERR_INPUT
        a.advance(5)
        a.Save_restart(d + "/ct.dat")
        a.reset(4)  # horizon below the saved step
        with pytest.raises(pkg.FdtdError) as e:
            a.Read_restart(d + "/ct.dat")
        assert e.value.code == pkg.FDTD_ERR_STATE
