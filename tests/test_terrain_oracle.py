"""Terrain-following grid in the oracle (CPU): the extension reduces to the
reference's flat grid exactly where the terrain is flat, and a uniformly
raised ground is the same solve as a flat grid whose air axis is the
stretched one. The GPU path is checked against this oracle in
test_terrain_gpu.py."""

from __future__ import annotations

import copy
import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cases  # noqa: E402
import oracle  # noqa: E402

casegen = importlib.import_module("3d_mpi_test_b200.casegen")


def _fields(d, rec, n):
    r = oracle.run_case(d, rec, n)
    out = {"receivers": r["receivers"]}
    for f in "puvw":
        out[f] = r[f]
        if "pore_" + f in r:
            out["pore_" + f] = r["pore_" + f]
    return out


@pytest.mark.parametrize("name", ["porous_ground", "wind_log", "south_pml_all_faces"])
def test_zero_terrain_is_the_flat_grid_bit_for_bit(name, tmp_path):
    c, rec = cases.CASES[name]()
    c.time_domain = 25
    d0 = str(tmp_path / "flat")
    c.write(d0)
    c1 = copy.deepcopy(c)
    c1.terrain = [0.0] * c1.NJ
    d1 = str(tmp_path / "zero")
    c1.write(d1)
    a, b = _fields(d0, rec, 25), _fields(d1, rec, 25)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


def test_uniform_terrain_is_a_stretched_flat_grid(tmp_path):
    """Ground raised by c everywhere: Z(j,k) = Z[k] + c (1 - Z[k]/H), the
    z_over_Y cross term vanishes, and the solve equals a flat grid whose air
    axis file holds those heights (porous axis shifted by c). Rigid north
    face and no wind keep the file-axis PML profile and the wind height out
    of the comparison."""
    layer = 5
    c = cases._base(ni=14, nj=30, nk=20, bc=(cases.RIGID, cases.POROUS, cases.PML, cases.PML, cases.PML, cases.PML),
                    pml_nodes=(4, 4, 4, 4, 0, 0), pore=(1.34, 0.3, 2.0e5))
    c.pore_Z = cases.uniform_axis(layer + 2, -layer * cases.D, cases.D)
    c.pore_dxyz = (cases.D, cases.D, cases.D)
    c.source = (0.35, 0.7, 0.4)
    rec = [(0.35, 1.0, 0.5), (0.3, 1.2, 0.6)]
    lift = 0.2
    ct = copy.deepcopy(c)
    ct.terrain = [lift] * c.NJ
    dt = str(tmp_path / "terrain")
    ct.write(dt)
    cf = copy.deepcopy(c)
    H = c.Z[-1]
    cf.Z = [z + lift * (1.0 - z / H) for z in c.Z]
    cf.pore_Z = [z + lift for z in c.pore_Z]
    cf.dxyz = c.spacing()  # input line 17 keeps the computational spacing
    df = str(tmp_path / "stretched")
    cf.write(df)
    a, b = _fields(dt, rec, 30), _fields(df, rec, 30)
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("name", sorted(cases.TERRAIN_CASES))
def test_terrain_cases_run_and_stay_bounded(name, tmp_path):
    """Every terrain case runs in the oracle for 240 steps (six times its
    parity length), its receivers record the pulse, and the field stays
    bounded by the initial pulse amplitude: the reference's forward /
    backward scheme is stable on these stretched and sloped cells."""
    c, rec = cases.TERRAIN_CASES[name]()
    c.time_domain = 240
    d = str(tmp_path / name)
    c.write(d)
    r = oracle.run_case(d, rec, c.time_domain)
    assert np.all(np.isfinite(r["p"])) and np.abs(r["p"]).max() < 1.5
    assert np.abs(r["receivers"]).max() > 1e-6


def test_hill_workload_geometry():
    """The hill workload's ground follows z_g = h exp(-(y - y0)^2 / 2w^2),
    its source and receivers sit at their heights above the local ground,
    and the stretched air grid keeps the flat top."""
    c, rec = casegen.porous_hill(ni=8, nj=64, nk=24, layer=4, pml=4, seed=3)
    assert len(c.terrain) == c.NJ and max(c.terrain) == pytest.approx(0.5)
    j0 = int(np.argmax(c.terrain))
    assert c.Y[j0] == pytest.approx(c.Y[c.NJ // 2])
    assert c.height(j0, 0) == pytest.approx(0.5) and c.height(j0, c.NK - 1) == c.Z[-1]
    y0 = c.Y[c.NJ // 2]
    for (_, y, z) in rec:
        assert z - 0.5 * np.exp(-((y - y0) ** 2) / 2.0) == pytest.approx(1.0)
