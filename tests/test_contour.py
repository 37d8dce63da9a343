"""Pressure contour files (airpore::get_data_contour): the Tecplot file this
library writes against the one the compiled reference writes with its own
operator<< (oracle/_ref/ref_harness --contour-out), and the binary variant
against the field read-out."""

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


@pytest.mark.parametrize("name,steps", [("pml_rigid", 12), ("porous_tdbc_fine_pore", 12), ("moving_frame", 60)])
def test_contour_matches_reference(name, steps, tmp_path):
    if not os.path.exists(refio.REF_HARNESS):
        pytest.skip("oracle/_ref/ref_harness not built")
    c, rec = cases.CASES[name]()
    d = str(tmp_path / name)
    c.write(d)
    subprocess.run([refio.REF_HARNESS, d, "--steps", str(steps), "--out", d + "/a.bin", "--contour-out",
                    d + "/ref.dat"], check=True)
    with pkg.Airpore(d, "f64") as a:
        a.get_output(steps)
        a.get_data_contour(d + "/mine.dat")
        a.get_data_contour(d + "/mine.bin", binary=True)
        p = a.field("p")
    ref = open(d + "/ref.dat").read().splitlines()
    mine = open(d + "/mine.dat").read().splitlines()
    assert len(ref) == len(mine)
    for lr, lm in zip(ref, mine):
        if not lr[:1].isdigit() and not lr[:1] == "-":
            assert lr == lm  # VARIABLES / ZONE lines
            continue
        tr, tm = lr.split(), lm.split()
        assert tr[:3] == tm[:3]  # X Y Z of the frame, identical text
        assert float(tm[3]) == pytest.approx(float(tr[3]), rel=2e-6, abs=1e-12)
    # binary: the same nodes, full precision
    b = open(d + "/mine.bin", "rb").read()
    assert b[:8] == b"FDTDCNT1"
    I, J, K = np.frombuffer(b[12:24], dtype=np.int32)
    vals = np.frombuffer(b[24: 24 + 8 * (I + J + K + I * J * K)], dtype=np.float64)
    P = vals[I + J + K: I + J + K + I * J * K].reshape(K, J, I)
    keep = lambda n: [q for q in range(n) if q % 4 == 0 or q == n - 1]  # noqa: E731
    want = p[np.ix_(keep(p.shape[0]), keep(p.shape[1]), keep(p.shape[2]))].transpose(2, 1, 0)
    np.testing.assert_array_equal(P, want)
