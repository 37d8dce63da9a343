"""Log-law wind and upwind velocity advection in the oracle (CPU). The log
law V = (u*/kappa) ln(z/z0) grows without bound under the reference's
forward-difference velocity advection, as the reference's own log profile
(method 5) does; backward (upwind) differences keep it bounded."""

from __future__ import annotations

import copy
import importlib
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import cases  # noqa: E402
import oracle  # noqa: E402


def _box(method, b, advection=None, d=0.05):
    R = cases.RIGID
    c = cases._base(ni=3, nj=160, nk=60, bc=(R,) * 6, pml_nodes=(0,) * 6, velocity_coef=b, velocity_method=method,
                    steps=3000)
    c.X = cases.uniform_axis(3, 0.0, d)
    c.Y = cases.uniform_axis(160, 0.0, d)
    c.Z = cases.uniform_axis(60, 0.0, d)
    c.dt = 0.5 * d / 343.0
    c.source = (d, 40 * d, 10 * d)
    c.gauss_width = 6 * d
    c.advection = advection
    return c


def _max_p(c, tmp_path, steps):
    d = str(tmp_path)
    c.write(d)
    oc = oracle.OracleCase(d)
    out, done = [], 0
    for n in steps:
        oc.run(n - done)
        done = n
        out.append(float(np.abs(oc.field("p")).max()))
    return out


def test_log_law_profile(tmp_path):
    """The wind arrays hold (u*/kappa) ln(z/z0) above z0 and calm below,
    with kappa and z0 from logwind.dat."""
    c, _ = cases.wind_loglaw_upwind()
    d = str(tmp_path / "w")
    c.write(d)
    oc = oracle.OracleCase(d)
    oc.run(1)  # the frame set-up (SetWindProfile) runs with the first step
    U, V, W = oc.wind()
    assert np.all(U == 0) and np.all(W == 0)
    for k, z in enumerate(c.Z):
        want = 0.5 / 0.41 * np.log(z / 0.05) if z > 0.05 else 0.0
        assert V[5, 7, k] == pytest.approx(want, rel=1e-15, abs=0)


def test_log_law_grows_under_reference_advection(tmp_path):
    p = _max_p(_box(7, 0.4), tmp_path, (500, 3000))
    assert p[0] < 0.5 and p[1] > 1e3  # bounded early, then unbounded growth


def test_log_law_bounded_with_upwind_advection(tmp_path):
    p = _max_p(_box(7, 0.6, "upwind"), tmp_path, (500, 3000))
    assert max(p) < 0.5


def test_reference_advection_file_is_the_default(tmp_path):
    """advection.dat 'reference' is the reference's scheme bit for bit."""
    c, rec = cases.CASES["wind_log"]()
    d0, d1 = str(tmp_path / "a"), str(tmp_path / "b")
    c.write(d0)
    c1 = copy.deepcopy(c)
    c1.advection = "reference"
    c1.write(d1)
    a, b = oracle.run_case(d0, rec, 20), oracle.run_case(d1, rec, 20)
    for k in ("receivers", "p", "u", "v", "w"):
        np.testing.assert_array_equal(a[k], b[k])
