"""Small generated cases that exercise every feature of the reference's
time-marching path.  Shared by the oracle pin tests (CPU) and the GPU parity
tests.  Each builder returns ``(Case, receivers)``; sizes keep the oracle
to well under a second per case."""

from __future__ import annotations

import functools
import importlib
import math
from typing import Callable, Dict, List, Tuple

casegen = importlib.import_module("3d_mpi_test_b200.casegen")
Case = casegen.Case
uniform_axis = casegen.uniform_axis
RIGID, PML, POROUS, TDBC = casegen.RIGID, casegen.PML, casegen.POROUS, casegen.TDBC

D = 0.05
C0 = 343.0


def _base(ni=20, nj=28, nk=18, steps=40, pml=5, bc=(PML, RIGID, PML, PML, PML, PML), **kw) -> Case:
    gamma, rho0 = 1.4, 1.2
    P0 = rho0 * C0 * C0 / gamma
    pml_nodes = kw.pop("pml_nodes", (pml, pml, pml, pml, pml if bc[1] == PML else 0, pml))
    c = Case(
        X=uniform_axis(ni, 0.0, D), Y=uniform_axis(nj, 0.0, D), Z=uniform_axis(nk, 0.0, D),
        pml_nodes=pml_nodes, gauss_width=6 * D, bc=bc, time_domain=steps, gamma=gamma, P0=P0, c0=C0,
        source=(0.5, 0.55, 0.3), receiver=(0.5, 0.9, 0.3), dt=0.5 * D / C0, **kw,
    )
    return c


REC = [(0.5, 0.9, 0.3), (0.45, 1.1, 0.4), (0.3, 0.6, 0.15)]


def pml_rigid():
    return _base(), REC


def tdbc_east():
    return _base(bc=(PML, RIGID, TDBC, PML, PML, PML), pore=(1.79, 0.877, 5.1e4)), REC


def porous_ground():
    layer = 6
    c = _base(bc=(PML, POROUS, PML, PML, PML, PML), pore=(math.sqrt(1.8), 0.3, 2.0e5))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.source = (0.5, 0.55, 0.15)
    return c, REC + [(0.5, 0.7, 0.05)]


def porous_tdbc_fine_pore():
    """Porous ground with a finer porous z spacing (ratio 2 < 5 keeps the
    two-plane coupling) plus the east TDBC."""
    layer = 8
    c = _base(bc=(PML, POROUS, TDBC, PML, RIGID, PML), pore=(1.5, 0.5, 3.0e4))
    c.pore_Z = uniform_axis(layer + 2, -layer * D / 2, D / 2)
    c.pore_dxyz = (D, D, D / 2)
    c.source = (0.5, 0.55, 0.1)
    return c, REC


def south_pml_all_faces():
    return _base(bc=(PML, PML, PML, PML, PML, PML)), REC


def front_only_pml():
    # Front alone selects the x2 slab (high-i side): airpore.cpp:93-95,199-212
    return _base(bc=(PML, RIGID, PML, PML, PML, RIGID)), REC


def back_only_pml():
    return _base(bc=(RIGID, RIGID, RIGID, PML, RIGID, PML)), REC


def all_rigid():
    return _base(bc=(RIGID,) * 6, pml_nodes=(0,) * 6), REC


def wind_linear():
    return _base(velocity_coef=3.0, velocity_method=1), REC


def wind_log():
    return _base(velocity_coef=1.5, velocity_method=5), REC


def wind_vortex():
    return _base(velocity_coef=0.0, velocity_method=2), REC


def hill(judge: int):
    def build():
        c = _base(nk=20)
        box = (0.2, 0.8, 0.7, 1.2, 0.0, 0.5)
        curves = {
            1: (1, 0.0, 0.2, 0.5, 0.95, 0.15, 0, 0, 0, 0, 0, 0, 0, 0),  # sphere r=0.2 at (0.5,0.95,0.15)
            2: (2, 0.35, 0.65, 0.8, 1.05, 0.0, 0.3, 0, 0, 0, 0, 0, 0, 0),  # box
            3: (3, 0.08, 0.2, 0.4, 0.8, 0.3, 0.6, 0.85, 0.25, 0.5, 0.9, 0.2, 0, 2),  # rows of cylinders
            4: (4, 0.07, 0.3, 0.8, 0.15, 0.2, 3, 2, 0, 0, 0, 0, 0, 0),  # cylinder array
        }
        if judge == 5:
            # tree centred at (0, 3) m in the reference's hard-coded geometry (air.cpp:1097-1114)
            c.X = uniform_axis(24, -0.6, D)
            c.Y = uniform_axis(30, 2.3, D)
            c.Z = uniform_axis(40, 0.0, D)
            c.source = (0.0, 2.6, 1.0)
            box = (-0.55, 0.5, 2.4, 3.6, 0.0, 1.85)
            c.curve = (5,) + (0.0,) * 12 + (0,)
            c.hill_box = box
            rec = [(0.0, 3.3, 1.0), (0.1, 2.9, 0.8)]
            return c, rec
        c.curve = curves[judge]
        c.hill_box = box
        return c, REC

    build.__name__ = f"hill{judge}"
    return build


def moving_frame():
    """Window of 24 j-nodes over a 44-node range, frames of trail_DJ-1 = 5
    cells (calculation_2D.cpp:405-496, air.cpp:2447-2730)."""
    c = _base(nj=24, steps=60, pml_nodes=(5, 5, 5, 5, 0, 5))
    c.Y = uniform_axis(44, 0.0, D)
    c.mf_jmax, c.mf_lead, c.mf_trail, c.mf_judge, c.mf_ratio = 24, 6, 6, 1, 0.75
    c.ijkmax = 44
    c.source = (0.5, 0.4, 0.3)
    return c, [(0.5, 0.8, 0.3), (0.5, 1.4, 0.3), (0.5, 1.9, 0.35)]


def fb_v_p():
    c = _base(scheme=1, bc=(PML, RIGID, TDBC, PML, PML, PML))
    return c, REC


def delayed_y1():
    return _base(pml_y=(2.0, 1000.0, 17)), REC


def stretched():
    """Non-uniform axes: the 1D metric terms X_over_x etc. vary per node."""
    c = _base()
    c.X = [0.05 * i + 0.002 * math.sin(0.7 * i) for i in range(20)]
    c.Y = [0.05 * j + 0.01 * (j / 27.0) ** 2 for j in range(28)]
    c.Z = [0.05 * k * (1.0 + 0.01 * k) for k in range(18)]
    return c, REC


def odd_columns_wind():
    """29 columns: the east face column (j = 28) starts a new 16-byte column
    vector in both precisions; with the east TDBC and a log wind profile."""
    c = _base(nj=29, bc=(PML, RIGID, TDBC, PML, PML, PML), pore=(1.79, 0.877, 5.1e4),
              velocity_coef=1.5, velocity_method=5)
    return c, REC


def odd_columns_porous():
    """29 columns over porous ground with the east TDBC."""
    layer = 6
    c = _base(nj=29, bc=(PML, POROUS, TDBC, PML, PML, PML), pore=(math.sqrt(1.8), 0.3, 2.0e5))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.source = (0.5, 0.55, 0.15)
    return c, REC


def pml_box_all():
    """PML on all six faces, wide enough that tiles lie inside one x, y or
    z layer (single-layer tile kernel) besides the edges, corners, faces
    and the lean interior."""
    c = _base(ni=34, nj=46, nk=30, steps=30, bc=(PML,) * 6, pml_nodes=(6, 6, 6, 6, 6, 6))
    c.source = (0.85, 1.1, 0.75)
    return c, [(0.85, 1.6, 0.75), (0.1, 1.1, 0.75), (0.85, 0.1, 0.5), (0.85, 1.1, 1.35), (0.2, 2.1, 1.3)]


def pml_box_wind_porous():
    """Porous ground, log wind, y1 PML switched on after 11 steps, layers of
    odd and unequal widths (5 / 7 rows, 7 / 5 columns, 6 planes): the
    single-layer tiles with wind, layer boundaries inside column vectors."""
    layer = 5
    c = _base(ni=32, nj=45, nk=28, steps=30, bc=(PML, POROUS, PML, PML, PML, PML), pml_nodes=(5, 7, 7, 5, 0, 6),
              pore=(math.sqrt(1.8), 0.3, 2.0e5), velocity_coef=1.5, velocity_method=5, pml_y=(2.0, 1000.0, 11))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.source = (0.8, 1.0, 0.3)
    return c, [(0.8, 1.5, 0.3), (0.1, 1.0, 0.5), (0.8, 0.15, 0.4), (0.8, 1.0, 1.2), (0.8, 2.1, 0.1)]


def narrow_y():
    """5 columns with 2-node y PML layers on both sides: one 16-byte column
    vector holds nodes of both y layers."""
    c = _base(ni=12, nj=5, nk=12, pml_nodes=(3, 3, 2, 2, 0, 3))
    c.source = (0.3, 0.1, 0.3)
    return c, [(0.3, 0.1, 0.25), (0.35, 0.15, 0.3)]


def wide_2d():
    """2D (NI = 3, Front/Back rigid) with 900 columns: the FP32 marching tile
    fits shared memory only with its stage sized to the rows it stages;
    porous ground, linear wind, PML."""
    layer = 4
    c = _base(ni=3, nj=900, nk=40, steps=30, bc=(PML, POROUS, PML, PML, RIGID, RIGID),
              pml_nodes=(0, 0, 10, 10, 0, 10), pore=(math.sqrt(1.5), 0.4, 1.0e5), velocity_coef=0.8,
              velocity_method=1)
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.source = (0.05, 20.0, 0.5)
    return c, [(0.05, 20.5, 0.5), (0.05, 25.0, 1.0), (0.05, 40.0, 0.3)]


def very_wide_2d():
    """2D (NI = 3) with 1300 columns: wider than the row marching kernel's
    limit (256 threads of one 16-byte column vector each), so only the
    tiled kernel runs it; porous ground and PML."""
    layer = 4
    c = _base(ni=3, nj=1300, nk=24, steps=24, bc=(PML, POROUS, PML, PML, RIGID, RIGID),
              pml_nodes=(0, 0, 10, 10, 0, 8), pore=(math.sqrt(1.5), 0.4, 1.0e5))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.source = (0.05, 32.0, 0.4)
    return c, [(0.05, 32.3, 0.4), (0.05, 33.0, 0.6), (0.05, 60.0, 0.3)]


ENS_SMALL = ((24, 36), (16, 20), (10, 13))  # NJ, NK, 3D NI ranges of the small ensemble members


def ensemble_member_2d():
    """A small member of the seeded batched-ensemble generator: 2D (NI = 3,
    Front/Back rigid), porous ground, porous hill, the reference's
    logarithmic wind (these cases are pinned to the compiled reference, which
    has neither the log law of method 7 nor upwind advection)."""
    c, rec, _ = casegen.ensemble_member(5, 0, pml=4, layer=4, steps=40, n_receivers=3, sizes=ENS_SMALL,
                                        wind="reference")
    return c, rec


def ensemble_member_3d():
    """A small 3D member of the same generator (x PML on both sides)."""
    c, rec, _ = casegen.ensemble_member(5, 3, pml=4, layer=4, steps=40, n_receivers=3, sizes=ENS_SMALL,
                                        wind="reference")
    return c, rec


# ------------------------------------------------ terrain-following grid
# Extension of the reference (its cross metrics are fixed at zero), so these
# cases are checked against the oracle's restatement only, not against the
# compiled reference.
def _hill(c: Case, h: float = 0.12, w: float = 0.3) -> Case:
    y0 = c.Y[len(c.Y) // 2]
    c.terrain = casegen.gaussian_hill(c.Y, h, w, y0)
    return c


def _above(c: Case, x: float, y: float, dz: float) -> Tuple[float, float, float]:
    j = min(range(len(c.Y)), key=lambda q: abs(c.Y[q] - y))
    return (x, y, c.terrain[j] + dz)


def hill_porous():
    """Porous ground under a Gaussian hill (h = 0.12 m, w = 0.3 m), PML on
    the five air faces."""
    layer = 5
    c = _base(ni=16, nj=40, nk=24, bc=(PML, POROUS, PML, PML, PML, PML), pore=(math.sqrt(1.8), 0.3, 2.0e5))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    _hill(c)
    c.source = _above(c, 0.4, 0.7, 0.2)
    return c, [_above(c, 0.4, 1.0, 0.3), _above(c, 0.4, 1.3, 0.2), _above(c, 0.3, 0.5, 0.5)]


def hill_wind_pml6():
    """Gaussian hill with PML on all six faces (the z1 layer follows the
    ground) and a log wind profile over the local ground."""
    c = _base(ni=16, nj=40, nk=26, bc=(PML,) * 6, pml_nodes=(5, 5, 5, 5, 4, 5), velocity_coef=1.5,
              velocity_method=5)
    _hill(c, h=0.12)
    c.source = _above(c, 0.4, 0.8, 0.35)
    return c, [_above(c, 0.4, 1.1, 0.3), _above(c, 0.45, 1.4, 0.25), _above(c, 0.4, 0.5, 0.5)]


def hill_fbvp_tdbc():
    """Gaussian hill with the FB_v_p scheme (two-pass kernels) and the east
    TDBC."""
    c = _base(ni=14, nj=36, nk=22, scheme=1, bc=(PML, RIGID, TDBC, PML, PML, PML), pore=(1.79, 0.877, 5.1e4))
    _hill(c, h=0.1, w=0.25)
    c.source = _above(c, 0.35, 0.7, 0.25)
    return c, [_above(c, 0.35, 1.2, 0.3), _above(c, 0.3, 1.6, 0.2)]


def hill_porous_tdbc():
    """Porous ground under a hill with the east TDBC (generic tile kernel on
    the terrain-following grid)."""
    layer = 4
    c = _base(ni=14, nj=37, nk=22, bc=(PML, POROUS, TDBC, PML, PML, PML), pore=(math.sqrt(1.5), 0.4, 1.0e5))
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    _hill(c, h=0.1, w=0.3)
    c.source = _above(c, 0.35, 0.8, 0.2)
    return c, [_above(c, 0.35, 1.1, 0.25), _above(c, 0.3, 1.5, 0.3)]


TERRAIN_CASES: Dict[str, Callable[[], Tuple[Case, List]]] = {
    f.__name__: f for f in [hill_porous, hill_wind_pml6, hill_fbvp_tdbc, hill_porous_tdbc]
}


# ------------------------------------------- log-law wind, upwind advection
# Extensions of the reference (its wind methods stop at 6 and its velocity
# advection is a forward difference), checked against the oracle only.
def wind_loglaw():
    """The surface-layer log law V = (u*/kappa) ln(z/z0) (method 7,
    kappa 0.41, z0 0.01 m) with the reference's forward-difference
    velocity advection."""
    return _base(velocity_coef=0.4, velocity_method=7), REC


def wind_loglaw_upwind():
    """The log law (kappa 0.41, z0 0.05 m from logwind.dat) with upwind
    (backward-difference) velocity advection, porous ground."""
    layer = 5
    c = _base(bc=(PML, POROUS, PML, PML, PML, PML), pore=(math.sqrt(1.8), 0.3, 2.0e5), velocity_coef=0.5,
              velocity_method=7)
    c.pore_Z = uniform_axis(layer + 2, -layer * D, D)
    c.pore_dxyz = (D, D, D)
    c.logwind = (0.41, 0.05)
    c.advection = "upwind"
    c.source = (0.5, 0.55, 0.15)
    return c, REC


def wind_vortex_upwind():
    """The reference's vortex profile (method 2, V and W components) with
    upwind velocity advection and the east TDBC."""
    c = _base(velocity_coef=0.0, velocity_method=2, bc=(PML, RIGID, TDBC, PML, PML, PML), pore=(1.79, 0.877, 5.1e4))
    c.advection = "upwind"
    return c, REC


def hill_loglaw_upwind():
    """Log-law wind over a hill (height above the local ground) with upwind
    advection, PML on all six faces."""
    c = _base(ni=16, nj=40, nk=26, bc=(PML,) * 6, pml_nodes=(5, 5, 5, 5, 4, 5), velocity_coef=0.4,
              velocity_method=7)
    _hill(c, h=0.12)
    c.advection = "upwind"
    c.source = _above(c, 0.4, 0.8, 0.35)
    return c, [_above(c, 0.4, 1.1, 0.3), _above(c, 0.45, 1.4, 0.25), _above(c, 0.4, 0.5, 0.5)]


EXT_CASES: Dict[str, Callable[[], Tuple[Case, List]]] = {
    f.__name__: f for f in [wind_loglaw, wind_loglaw_upwind, wind_vortex_upwind, hill_loglaw_upwind]
}


# ----------------------------------------------------- impedance ground
# Extension of the reference (its TDBC acts on the east face only): the
# rigid south face as a 6-pole TDBC with poles fitted to Miki's impedance,
# checked against the oracle only.
ground = importlib.import_module("3d_mpi_test_b200.ground")


@functools.lru_cache(maxsize=None)
def miki_poles(sigma: float, dt: float = 0.5 * D / C0):
    """(Zinf, tau, a, r) fitted to Miki at flow resistivity sigma on the
    discrete recursion of time step dt."""
    f = ground.fit_tdbc(sigma, dt=dt)
    return (f.Zinf, f.tau, tuple(f.a), tuple(f.r))


def ground_box():
    """Miki ground at 50 kPa s/m^2 under a PML box."""
    c = _base()
    c.ground_tdbc = miki_poles(50e3)
    c.source = (0.5, 0.55, 0.15)
    return c, REC + [(0.5, 0.7, 0.05)]


def ground_rigid_sides():
    """Miki ground at 200 kPa s/m^2 with rigid east/west/front/back faces
    (face copies of w at k = 1 on every side), PML top."""
    c = _base(bc=(PML, RIGID, RIGID, RIGID, RIGID, RIGID), pml_nodes=(0, 0, 0, 0, 0, 5))
    c.ground_tdbc = miki_poles(200e3)
    c.source = (0.3, 0.4, 0.1)
    return c, REC


def ground_loglaw_tdbc_east():
    """Config 3's physics on a small box: log-law wind with upwind
    advection over the Miki ground, the east TDBC too, y1 PML switched on
    late."""
    c = _base(bc=(PML, RIGID, TDBC, PML, PML, PML), pore=(1.79, 0.877, 5.1e4), velocity_coef=0.4,
              velocity_method=7, pml_y=(2.0, 1000.0, 13))
    c.ground_tdbc = miki_poles(50e3)
    c.logwind = (0.41, 0.01)
    c.advection = "upwind"
    c.source = (0.5, 0.55, 0.2)
    return c, REC


def ground_moving_frame():
    """The moving frame over the Miki ground: the ground state moves with
    the frame."""
    c, rec = moving_frame()
    c.ground_tdbc = miki_poles(50e3)
    c.source = (0.5, 0.4, 0.1)
    return c, rec


GROUND_CASES: Dict[str, Callable[[], Tuple[Case, List]]] = {
    f.__name__: f for f in [ground_box, ground_rigid_sides, ground_loglaw_tdbc_east, ground_moving_frame]
}


CASES: Dict[str, Callable[[], Tuple[Case, List]]] = {
    f.__name__: f
    for f in [pml_rigid, tdbc_east, porous_ground, porous_tdbc_fine_pore, south_pml_all_faces, front_only_pml,
              back_only_pml, all_rigid, wind_linear, wind_log, wind_vortex, hill(1), hill(2), hill(3), hill(4),
              hill(5), moving_frame, fb_v_p, delayed_y1, stretched, odd_columns_wind, odd_columns_porous, narrow_y,
              pml_box_all, pml_box_wind_porous,
              ensemble_member_2d, ensemble_member_3d, wide_2d, very_wide_2d]
}
