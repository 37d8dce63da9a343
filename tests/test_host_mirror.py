"""The C++ host classes (airpore / calculation_2D / air / porous over the C
ABI, 3d_mpi_test_b200/host/airpore_b200.hpp): a compiled driver in the shape
of the reference's main.cpp runs cases through them and matches the oracle."""

from __future__ import annotations

import importlib
import os
import shutil
import subprocess

import numpy as np
import pytest

import cases
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "3d_mpi_test_b200", "lib")
casegen = importlib.import_module("3d_mpi_test_b200.casegen")
build = importlib.import_module("3d_mpi_test_b200.build")


def _compile(tmp_path) -> str:
    build.build()
    exe = str(tmp_path / "mirror_driver")
    cmd = [shutil.which("g++") or "g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(ROOT, "3d_mpi_test_b200", "host"), os.path.join(ROOT, "tests", "cpp", "mirror_driver.cpp"),
           "-o", exe, "-L", LIBDIR, "-lairpore_b200", "-lfdtd_b200", f"-Wl,-rpath,{LIBDIR}"]
    subprocess.run(cmd, check=True)
    return exe


def _case(tmp_path, name, table):
    c, rec = table[name]()
    d = str(tmp_path / name)
    c.write(d)
    rf = casegen.write_receivers(os.path.join(d, "rec.txt"), rec)
    return d, rf, rec, c.time_domain


def test_mirror_builds_and_reports_errors(tmp_path):
    """The classes compile against the C ABI header and link against the
    library; a failing construction surfaces as b200::Error with the ABI's
    code (here: a missing case directory, FDTD_ERR_INPUT, or no sm_100
    device, FDTD_ERR_CUDA)."""
    exe = _compile(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "missing"), str(tmp_path / "none.txt"), "3", str(tmp_path / "o")],
                       capture_output=True, text=True)
    assert r.returncode == 3
    assert "fdtd error -1" in r.stderr or "fdtd error -3" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name,table", [("porous_ground", cases.CASES), ("tdbc_east", cases.CASES),
                                        ("hill_porous", cases.TERRAIN_CASES)])
def test_mirror_matches_oracle(name, table, tmp_path):
    exe = _compile(tmp_path)
    d, rf, rec, n = _case(tmp_path, name, table)
    out = str(tmp_path / "out")
    r = subprocess.run([exe, d, rf, str(n), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ref = oracle.run_case(d, rec, n)

    def load(suffix, shape):
        return np.fromfile(out + suffix, dtype=np.float64).reshape(shape)

    def rel(x, y):
        return float(np.linalg.norm(x - y) / np.linalg.norm(y))

    assert rel(load(".rec", ref["receivers"].shape), ref["receivers"]) <= 1e-10
    assert rel(load(".p", ref["p"].shape), ref["p"]) <= 1e-10
    if "pore_p" in ref:
        assert rel(load(".pore_p", ref["pore_p"].shape), ref["pore_p"]) <= 1e-10
    # the reference's member-call order (half steps) reaches the same state
    assert rel(load(".half_p", ref["p"].shape), load(".p", ref["p"].shape)) <= 1e-13
