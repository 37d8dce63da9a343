"""Case generator: emits the reference solver's own setup files.

A case directory holds ``input.txt`` (the positional format parsed by
``airpore::airpore``, airpore.cpp:17-316) and the axis files
``coordi_air{1,2,3}.dat`` (header ``IMAX IMAX1 IMAX2 JMAX JMAX1 JMAX2 KMAX
KMAX1 KMAX2 IJKMAX`` in file 1, then one coordinate per node; read by
``calculation_2D::calculation_2D``, calculation_2D.cpp:44-204).  When the
south face is porous (input line 4, second code = 3) the porous grid gets
``coordi_pore{1,2,3}.dat`` in the same format; the reference repository
does not ship those files, so they are always generated here.

Axis convention is the reference's: X = i (transverse, Front/Back faces),
Y = j (range / propagation, West/East faces, moving-frame axis),
Z = k (height, South = ground, North = top).

The line layout written by :func:`Case.input_text` mirrors the shipped
``input.txt`` line for line, because the reference parser skips comment
lines positionally (``infile.ignore(100, '\\n')``).
"""

from __future__ import annotations

import dataclasses
import importlib
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

# Boundary codes of input line 4 (airpore.cpp:52-159).
RIGID, PML, POROUS, RADIATION, TDBC = 1, 2, 3, 4, 5


def _fmt(x: float) -> str:
    """Shortest text that parses back to exactly the same double."""
    if isinstance(x, int):
        return str(x)
    r = repr(float(x))
    return r


def uniform_axis(n: int, start: float, step: float) -> List[float]:
    return [start + i * step for i in range(n)]


@dataclass
class Case:
    """Every field of input.txt plus the three air axes (and porous axes)."""

    X: List[float]
    Y: List[float]
    Z: List[float]
    # PML node counts in the coordi header (IMAX1, IMAX2, JMAX1, JMAX2, KMAX1, KMAX2)
    pml_nodes: Tuple[int, int, int, int, int, int] = (0, 0, 0, 0, 0, 0)
    ijkmax: Optional[int] = None  # whole-domain JMAX for the moving frame; default = len(Y)
    gauss_width: float = 0.3  # line 1: Gaussian FWHM (m)
    # line 2: moving frame JMAX lead_DJ trail_DJ Judge ratio
    mf_jmax: Optional[int] = None
    mf_lead: int = 11
    mf_trail: int = 11
    mf_judge: int = 0
    mf_ratio: float = 0.75
    scheme: int = 2  # line 3: 1 FB_v_p, 2 FB_p_v
    # line 4: North South East West Front Back
    bc: Tuple[int, int, int, int, int, int] = (PML, RIGID, PML, PML, PML, PML)
    time_domain: int = 100  # line 6
    out_difft: int = 100000
    fft_m: int = 12
    frequency: float = 300.0
    velocity_coef: float = 0.0  # line 8
    velocity_method: int = 4  # 4 = no wind (air.cpp:102-105,170-174,231-235)
    gamma: float = 1.4  # line 9
    P0: float = 1.0e5
    c0: float = 340.0
    pml_x: Tuple[float, float] = (2.0, 1000.0)  # line 10: alpha, sigma_max
    pml_y: Tuple[float, float, int] = (2.0, 1000.0, 0)  # line 11: + y1 activation step
    pml_z: Tuple[float, float] = (2.0, 1000.0)  # line 12
    pore: Tuple[float, float, float] = (1.3416407864998738, 0.3, 2.0e5)  # line 13: q, porosity, sigma
    source: Tuple[float, float, float] = (0.0, 0.0, 0.0)  # line 14 (X, Y, Z)
    receiver: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    dt: float = 1e-5  # line 16
    dxyz: Optional[Tuple[float, float, float]] = None  # line 17; default from the axes
    restart: Tuple[int, int, str] = (0, 1000000, "ct003")  # line 22
    # line 24: curve_judge a..l curve_points ; lines 25-27 hill/canopy/trunk (q, porosity, sigma)
    curve: Tuple[float, ...] = (0,) + (0.0,) * 12 + (0,)
    hill: Tuple[float, float, float] = (1.79, 0.877, 5.0e4)
    canopy: Tuple[float, float, float] = (1.79, 0.877, 5.0e4)
    trunk: Tuple[float, float, float] = (0.52, 0.5712, 8.0e4)
    hill_box: Tuple[float, float, float, float, float, float] = (0.0,) * 6  # line 29
    # porous grid (only when the south code is POROUS)
    pore_Z: Optional[List[float]] = None
    pore_X: Optional[List[float]] = None
    pore_Y: Optional[List[float]] = None
    pore_dxyz: Optional[Tuple[float, float, float]] = None  # line 32
    # terrain-following grid (extension; terrain.dat): ground elevation at
    # every Y node. Air nodes are stretched between the ground and the flat
    # top, porous nodes follow the ground. None: flat ground.
    terrain: Optional[List[float]] = None
    # log-law wind (extension, velocity_method 7): (kappa, z0) written to
    # logwind.dat; None keeps kappa 0.41 and z0 0.01 m
    logwind: Optional[Tuple[float, float]] = None
    # velocity advection by the mean wind (extension, advection.dat): None or
    # "reference" (forward differences) or "upwind" (backward differences)
    advection: Optional[str] = None
    # impedance ground (extension, tdbc_ground.dat): the rigid south face
    # becomes a 6-pole TDBC, (Zinf, tau, a[6], r[6]); ground.fit_tdbc makes one
    ground_tdbc: Optional[Tuple[float, float, Sequence[float], Sequence[float]]] = None

    # ------------------------------------------------------------------ #
    @property
    def NI(self) -> int:
        return len(self.X)

    @property
    def NJ(self) -> int:
        return len(self.Y)

    @property
    def NK(self) -> int:
        return len(self.Z)

    @property
    def porous_south(self) -> bool:
        return self.bc[1] == POROUS

    def spacing(self) -> Tuple[float, float, float]:
        if self.dxyz is not None:
            return self.dxyz
        return (self.X[1] - self.X[0], self.Y[1] - self.Y[0], self.Z[1] - self.Z[0])

    def input_text(self) -> str:
        mf_jmax = self.mf_jmax if self.mf_jmax is not None else self.NJ
        dx, dy, dz = self.spacing()
        c = self.curve
        curve_txt = " ".join([str(int(c[0]))] + [_fmt(v) for v in c[1:13]] + [str(int(c[13]))])
        lines = [
            f"{_fmt(self.gauss_width)} //gaussian_width",
            f"{mf_jmax} {self.mf_lead} {self.mf_trail} {self.mf_judge} {_fmt(self.mf_ratio)} //moving frame",
            f"{self.scheme} //scheme",
            " ".join(str(b) for b in self.bc) + " //North South East West Front Back",
            "//B.C type: 1 rigid 2 PML 3 porous 4 radiation 5 TDBC",
            f"{self.time_domain} {self.out_difft} {self.fft_m} {_fmt(self.frequency)} //time_domain out_difft FFT_m frequency",
            "",
            f"{_fmt(self.velocity_coef)} {self.velocity_method} //wind b, method",
            f"{_fmt(self.gamma)} {_fmt(self.P0)} {_fmt(self.c0)} //gamma P0 c0",
            f"{_fmt(self.pml_x[0])} {_fmt(self.pml_x[1])} //PMLx",
            f"{_fmt(self.pml_y[0])} {_fmt(self.pml_y[1])} {int(self.pml_y[2])} //PMLy",
            f"{_fmt(self.pml_z[0])} {_fmt(self.pml_z[1])} //PMLz",
            " ".join(_fmt(v) for v in self.pore) + " //pore q porosity sigma",
            " ".join(_fmt(v) for v in (*self.source, *self.receiver)) + " //source receiver",
            "",
            f"{_fmt(self.dt)} //dt",
            f"{_fmt(dx)} {_fmt(dy)} {_fmt(dz)} //dx dy dz",
            "",
            "1 1 1 //mpi dims",
            "",
            "output.data;",
            f"{self.restart[0]} {self.restart[1]} {self.restart[2]}",
            "",
            curve_txt + " //curve",
            " ".join(_fmt(v) for v in self.hill) + " //hill",
            " ".join(_fmt(v) for v in self.canopy) + " //canopy",
            " ".join(_fmt(v) for v in self.trunk) + " //trunk",
            "",
            " ".join(_fmt(v) for v in self.hill_box) + " //box",
            "",
            "porous_media;",
        ]
        if self.porous_south:
            pd = self.pore_dxyz if self.pore_dxyz is not None else (dx, dy, dz)
            lines.append(" ".join(_fmt(v) for v in pd) + " //pore dx dy dz")
        else:
            lines.append("0 0 0")
        for ln in lines:
            # ignore(100, '\n') skips at most 100 characters past the last value
            assert len(ln) < 95, ln
        return "\n".join(lines) + "\n"

    def coordi_texts(self, prefix: str = "coordi_air") -> dict:
        I1, I2, J1, J2, K1, K2 = self.pml_nodes
        ijk = self.ijkmax if self.ijkmax is not None else self.NJ
        head = f"{self.NI} {I1} {I2} {self.NJ} {J1} {J2} {self.NK} {K1} {K2} {ijk}"
        return {
            f"{prefix}1.dat": head + "\n" + " ".join(_fmt(v) for v in self.X) + "\n",
            f"{prefix}2.dat": " ".join(_fmt(v) for v in self.Y) + "\n",
            f"{prefix}3.dat": " ".join(_fmt(v) for v in self.Z) + "\n",
        }

    def pore_coordi_texts(self) -> dict:
        Xp = self.pore_X if self.pore_X is not None else self.X
        Yp = self.pore_Y if self.pore_Y is not None else self.Y
        Zp = self.pore_Z
        ijk = self.ijkmax if self.ijkmax is not None else len(Yp)
        head = f"{len(Xp)} 0 0 {len(Yp)} 0 0 {len(Zp)} 0 0 {ijk}"
        return {
            "coordi_pore1.dat": head + "\n" + " ".join(_fmt(v) for v in Xp) + "\n",
            "coordi_pore2.dat": " ".join(_fmt(v) for v in Yp) + "\n",
            "coordi_pore3.dat": " ".join(_fmt(v) for v in Zp) + "\n",
        }

    def write(self, case_dir: str) -> str:
        os.makedirs(case_dir, exist_ok=True)
        files = {"input.txt": self.input_text()}
        files.update(self.coordi_texts())
        if self.porous_south:
            if self.pore_Z is None:
                raise ValueError("porous south face needs pore_Z")
            files.update(self.pore_coordi_texts())
        if self.terrain is not None:
            if len(self.terrain) != self.NJ:
                raise ValueError("terrain needs one elevation per Y node")
            files["terrain.dat"] = f"{self.NJ}\n" + " ".join(_fmt(float(v)) for v in self.terrain) + "\n"
        if self.advection is not None:
            if self.advection not in ("reference", "upwind"):
                raise ValueError("advection must be 'reference' or 'upwind'")
            files["advection.dat"] = self.advection + "\n"
        if self.ground_tdbc is not None:
            Zinf, tau, a, r = self.ground_tdbc
            if len(a) != 6 or len(r) != 6:
                raise ValueError("the ground TDBC has six poles")
            files["tdbc_ground.dat"] = (f"{_fmt(float(Zinf))} {_fmt(float(tau))}\n"
                                        + " ".join(_fmt(float(x)) for x in a) + "\n"
                                        + " ".join(_fmt(float(x)) for x in r) + "\n")
        if self.logwind is not None:
            files["logwind.dat"] = f"{_fmt(float(self.logwind[0]))} {_fmt(float(self.logwind[1]))}\n"
        for name, txt in files.items():
            with open(os.path.join(case_dir, name), "w") as f:
                f.write(txt)
        return case_dir

    def height(self, j: int, k: int) -> float:
        """Physical height of air node (j, k): the file axis Z[k] stretched
        between the ground elevation and the flat top (the same expression
        as the solver's and the oracle's)."""
        z = self.Z[k]
        if self.terrain is None:
            return z
        H = self.Z[-1]
        return z + self.terrain[j] * (1.0 - z / H)


def write_receivers(path: str, receivers: Sequence[Tuple[float, float, float]]) -> str:
    with open(path, "w") as f:
        for r in receivers:
            f.write(" ".join(_fmt(v) for v in r) + "\n")
    return path


# ---------------------------------------------------------------------- #
# Named workloads.  The range axis of a workload maps to the reference's
# Y/j, the transverse axis to X/i and the height to Z/k.
# ---------------------------------------------------------------------- #

def plain_box(ni=48, nj=96, nk=48, d=0.05, steps=500, pml=10):
    """Plain reference method on a Cartesian box: rigid ground, PML on the
    other five faces, Gaussian pulse (amplitude 1 Pa, FWHM 6 d) at
    (X, Y, Z) = (1.2, 0.6, 0.3) m, receivers at Z = 0.3 m, X = 1.2 m,
    Y = 1.5/2.5/3.5/4.2 m.  96 x 48 x 48 nodes, d = 0.05 m, c0 = 343 m/s,
    rho0 = 1.2 kg/m^3, CFL 0.5, 500 steps."""
    c0, rho0, gamma = 343.0, 1.2, 1.4
    P0 = rho0 * c0 * c0 / gamma
    case = Case(
        X=uniform_axis(ni, 0.0, d), Y=uniform_axis(nj, 0.0, d), Z=uniform_axis(nk, 0.0, d),
        pml_nodes=(pml, pml, pml, pml, 0, pml),
        gauss_width=6 * d, bc=(PML, RIGID, PML, PML, PML, PML), time_domain=steps,
        gamma=gamma, P0=P0, c0=c0, pml_y=(2.0, 1000.0, 0),
        source=(1.2, 0.6, 0.3), receiver=(1.2, 1.5, 0.3), dt=0.5 * d / c0,
    )
    receivers = [(1.2, y, 0.3) for y in (1.5, 2.5, 3.5, 4.2)]
    return case, receivers


def porous_ground(ni=128, nj=256, nk=96, layer=16, d=0.05, steps=4000, pml=20, seed=0,
                  sigma=2.0e5, porosity=0.3, tortuosity=1.8):
    """Air box over a Zwikker-Kosten porous layer coupled through the
    two-plane airpore interface (calculation_2D.cpp:865-985): 256 x 128 x 96
    air nodes, a 16-cell-deep porous grid with the same X/Y nodes and
    layer+2 Z nodes, 20-node PML on the five air faces, 8 receivers on a line
    at 1 m height.  The source position is drawn from ``seed`` (height
    uniform in 0.2-1 m)."""
    import random

    rng = random.Random(seed)
    c0, rho0, gamma = 343.0, 1.2, 1.4
    P0 = rho0 * c0 * c0 / gamma
    Y = uniform_axis(nj, 0.0, d)
    X = uniform_axis(ni, 0.0, d)
    Z = uniform_axis(nk, 0.0, d)
    pore_Z = uniform_axis(layer + 2, -layer * d, d)  # pore k=layer is Z=0 (= air k=0)
    Xc = X[ni // 2]
    src = (Xc, Y[pml] + 10 * d + rng.uniform(0.0, 1.0) * 10 * d, rng.uniform(0.2, 1.0))
    rec_y0 = src[1] + 1.0
    receivers = [(Xc, min(rec_y0 + r * (Y[nj - pml - 2] - rec_y0) / 7.0, Y[nj - pml - 2]), 1.0)
                 for r in range(8)]
    case = Case(
        X=X, Y=Y, Z=Z, pml_nodes=(pml, pml, pml, pml, 0, pml),
        gauss_width=6 * d, bc=(PML, POROUS, PML, PML, PML, PML), time_domain=steps,
        gamma=gamma, P0=P0, c0=c0, pml_y=(2.0, 1000.0, 0),
        pore=(math.sqrt(tortuosity), porosity, sigma),
        source=src, receiver=receivers[0], dt=0.5 * d / c0,
        pore_Z=pore_Z, pore_dxyz=(d, d, d),
    )
    return case, receivers


def gaussian_hill(Y: Sequence[float], h: float, w: float, y0: float) -> List[float]:
    """Ground elevation z_g(y) = h exp(-(y - y0)^2 / (2 w^2)) at the Y nodes."""
    return [h * math.exp(-((y - y0) ** 2) / (2.0 * w * w)) for y in Y]


def porous_hill(ni=128, nj=256, nk=96, layer=16, d=0.05, steps=4000, pml=20, seed=0, h=0.5, w=1.0,
                sigma=2.0e5, porosity=0.3, tortuosity=1.8):
    """The porous-ground domain of :func:`porous_ground` over an analytic
    hill z_g(y) = h exp(-(y - y0)^2 / 2w^2) at mid-range (h = 0.5 m, w =
    1 m): the air grid stretched vertically between the ground and the flat
    top, the porous layer following the ground (terrain.dat). The source
    height above the local ground is drawn from ``seed`` (uniform in
    0.2-1 m); 8 receivers on a line 1 m above the local ground."""
    import random

    case, _ = porous_ground(ni=ni, nj=nj, nk=nk, layer=layer, d=d, steps=steps, pml=pml, seed=seed,
                            sigma=sigma, porosity=porosity, tortuosity=tortuosity)
    rng = random.Random(seed)
    Y = case.Y
    y0 = Y[nj // 2]
    case.terrain = gaussian_hill(Y, h, w, y0)
    zg = lambda y: h * math.exp(-((y - y0) ** 2) / (2.0 * w * w))  # noqa: E731
    Xc = case.X[ni // 2]
    # coordinates rounded to 1 um: input.txt lines stay inside the
    # reference parser's 100-character comment skip
    ys = round(Y[pml] + 10 * d + rng.uniform(0.0, 1.0) * 10 * d, 6)
    case.source = (Xc, ys, round(zg(ys) + rng.uniform(0.2, 1.0), 6))
    rec_y0 = ys + 1.0
    ymax = Y[nj - pml - 2]
    receivers = []
    for r in range(8):
        yr = round(min(rec_y0 + r * (ymax - rec_y0) / 7.0, ymax), 6)
        receivers.append((Xc, yr, round(zg(yr) + 1.0, 6)))
    case.receiver = receivers[0]
    return case, receivers


ENSEMBLE_SIZES = ((64, 512), (32, 192), (32, 96))  # NJ, NK, 3D NI: inclusive ranges


def ensemble_member(seed: int, index: int, d: float = 0.1, pml: int = 10, layer: int = 8, steps: int = 100,
                    n_receivers: int = 8, sizes=ENSEMBLE_SIZES, wind: str = "loglaw"):
    """Member ``index`` of the seeded batched-ensemble workload: one
    independent outdoor-sound solve whose size and physics are drawn from
    ``numpy.random.default_rng([seed, index])``:

    - range NJ uniform in [64, 512] nodes, height NK uniform in [32, 192];
      the transverse axis is NI = 3 for even ``index`` -- a 2D (y-z) solve:
      Front/Back rigid and no x PML, so the single interior row i = 1 is
      exactly two-dimensional (calculation_2D.cpp:835-860) -- and uniform in
      [32, 96] with x PML otherwise;
    - porous Zwikker-Kosten ground ``layer`` cells deep: flow resistivity
      log-uniform in 1e4..2e6 Pa s/m^2, porosity uniform in 0.2..0.6,
      tortuosity uniform in 1..2.5 (input line 13 holds its square root);
    - source height uniform in 0.1..3 m (kept below the top PML), source
      10 cells past the west PML;
    - a porous hill: a half sphere of height uniform in 0..2 m on the
      ground half way down the range, made with the reference's sphere
      inclusion (curve_judge 1, air.cpp:1019-1031) and its canopy
      parameters; heights under two cells leave it out;
    - wind with u* uniform in 0..0.6 m/s: ``wind="loglaw"`` the log law
      V(z) = (u*/0.41) ln(z / 0.01 m) (method 7) with upwind velocity
      advection (advection.dat), which stays bounded over long runs;
      ``wind="reference"`` the reference's V(z) = b ln(z / 0.1 + 1)
      (velocity_method 5, air.cpp:175-177) with b = u* / 0.4 and its
      forward-difference advection, which grows without bound after a few
      thousand steps (the row marching kernels run only this one).

    Uniform spacing ``d``, PML of ``pml`` nodes on every air face but the
    ground, CFL 0.5. ``sizes`` replaces the three node-count ranges (small
    members for tests). Receivers: ``n_receivers`` on a line at 1.2 m height
    (lower in short domains) from 1 m past the source to the east PML.
    Returns (Case, receivers, params) with the drawn parameters."""
    import numpy as np

    rng = np.random.default_rng([seed, index])
    (j0, j1), (k0, k1), (i0, i1) = sizes
    nj = int(rng.integers(j0, j1 + 1))
    nk = int(rng.integers(k0, k1 + 1))
    two_d = index % 2 == 0
    ni = 3 if two_d else int(rng.integers(i0, i1 + 1))
    sigma = float(10.0 ** rng.uniform(4.0, math.log10(2.0e6)))
    porosity = float(rng.uniform(0.2, 0.6))
    tortuosity = float(rng.uniform(1.0, 2.5))
    src_h = float(rng.uniform(0.1, 3.0))
    hill_h = float(rng.uniform(0.0, 2.0))
    ustar = float(rng.uniform(0.0, 0.6))

    c0, rho0, gamma = 343.0, 1.2, 1.4
    P0 = rho0 * c0 * c0 / gamma
    X = uniform_axis(ni, 0.0, d)
    Y = uniform_axis(nj, 0.0, d)
    Z = uniform_axis(nk, 0.0, d)
    top = (nk - pml - 3) * d  # highest height clear of the top PML
    src_h = round(min(src_h, top), 6)
    xc = round(X[ni // 2], 9)  # short text: input.txt lines hold under 100 characters
    src = (xc, round(Y[pml + 10], 9), src_h)
    if two_d:
        bc = (PML, POROUS, PML, PML, RIGID, RIGID)
        pml_nodes = (0, 0, pml, pml, 0, pml)
    else:
        bc = (PML, POROUS, PML, PML, PML, PML)
        pml_nodes = (pml, pml, pml, pml, 0, pml)
    rec_h = round(min(1.2, top), 9)
    y0, y1 = src[1] + 1.0, Y[nj - pml - 2]
    y0 = min(y0, y1)
    receivers = [(xc, round(y0 + r * (y1 - y0) / max(n_receivers - 1, 1), 9), rec_h) for r in range(n_receivers)]
    case = Case(
        X=X, Y=Y, Z=Z, pml_nodes=pml_nodes, gauss_width=6 * d, bc=bc, time_domain=steps,
        gamma=gamma, P0=P0, c0=c0, pml_y=(2.0, 1000.0, 0),
        pore=(math.sqrt(tortuosity), porosity, sigma), source=src, receiver=receivers[0],
        dt=0.5 * d / c0, velocity_coef=ustar / 0.4, velocity_method=5,
        pore_Z=uniform_axis(layer + 2, -layer * d, d), pore_dxyz=(d, d, d),
    )
    if wind == "loglaw":
        case.velocity_method, case.velocity_coef, case.advection = 7, ustar, "upwind"
    elif wind != "reference":
        raise ValueError("wind must be 'loglaw' or 'reference'")
    # hill: nodes of its bounding box, snapped to the grid, below the top PML
    r_cells = int(round(hill_h / d))
    r_cells = min(r_cells, nk - pml - 4, (nj - 2 * pml) // 4)
    if r_cells >= 2:
        jc = (pml + 10 + nj - pml - 2) // 2
        r = r_cells * d
        i_lo, i_hi = max(ni // 2 - r_cells, 1), min(ni // 2 + r_cells, ni - 2)
        case.curve = (1, 0.0, round(r, 9), xc, round(Y[jc], 9), 0.0) + (0.0,) * 7 + (0,)
        case.hill_box = tuple(round(v, 9) for v in (X[i_lo], X[i_hi], Y[jc - r_cells], Y[jc + r_cells], Z[0],
                                                     Z[r_cells]))
    params = dict(index=index, NI=ni, NJ=nj, NK=nk, two_d=two_d, sigma=sigma, porosity=porosity,
                  tortuosity=tortuosity, source_height=src_h, hill_height=r_cells * d if r_cells >= 2 else 0.0,
                  ustar=ustar)
    return case, receivers, params


def moving_window(ni=256, window=1024, nk=192, total=11264, d=0.05, pml=20, trail=11, ratio=0.05, steps=20000,
                  ustar: Optional[float] = 0.4, sigma: Optional[float] = 50e3):
    """The long-range configuration: a window of `window` range nodes (Y/j)
    x `ni` transverse x `nk` height moving over `total` range nodes with the
    reference's moving frame (calculation_2D.cpp:405-496,
    air.cpp:2447-2730; lead = trail, frames of trail - 1 cells that follow
    the pulse at c0, the first frame shortened by `ratio`; 11264 nodes keep
    the window moving through 20000 steps), PML on the top, front and back
    faces, rigid leading and trailing faces, Gaussian pulse at 1.5 m,
    receivers every 5 m to 100 m at 1.5 m height. The frame moves at c0, so
    no wave reaches the leading face and the waves reflected at the
    trailing face leave the window at the next shifts; PML layers at those
    faces grow without bound under the reference's moving frame (it moves
    the x and z layers' integrals with the fields and leaves the y layers'
    in place, air.cpp:2522-2729). With `ustar` the log-law wind V = (u*/0.41) ln(z / 0.01 m)
    (method 7, logwind.dat) advects the velocity by backward differences
    (advection.dat: the reference's forward differences grow without bound
    under a log profile); with `sigma` the ground is the 6-pole TDBC fitted
    to Miki's impedance at that flow resistivity on this time step
    (tdbc_ground.dat), otherwise rigid."""
    c0, rho0, gamma = 343.0, 1.2, 1.4
    dt = 0.5 * d / c0
    case = Case(
        X=uniform_axis(ni, 0.0, d), Y=uniform_axis(total, 0.0, d), Z=uniform_axis(nk, 0.0, d),
        pml_nodes=(pml, pml, 0, 0, 0, pml), gauss_width=6 * d, bc=(PML, RIGID, RIGID, RIGID, PML, PML),
        time_domain=steps, gamma=gamma, P0=rho0 * c0 * c0 / gamma, c0=c0, pml_y=(2.0, 1000.0, 0),
        source=(round(ni // 2 * d, 9), round((pml + 20) * d, 9), 1.5),
        receiver=(round(ni // 2 * d, 9), 5.0, 1.5), dt=dt,
        mf_jmax=window, mf_lead=trail, mf_trail=trail, mf_judge=1, mf_ratio=ratio, ijkmax=total,
    )
    if ustar:
        case.velocity_method, case.velocity_coef = 7, ustar
        case.logwind = (0.41, 0.01)
        case.advection = "upwind"
    if sigma:
        ground = importlib.import_module(__package__ + ".ground")
        fit = ground.fit_tdbc(sigma, dt=dt)
        case.ground_tdbc = (fit.Zinf, fit.tau, tuple(fit.a), tuple(fit.r))
    xc = round(ni // 2 * d, 9)
    receivers = [(xc, float(r), 1.5) for r in range(5, int(total * d) - 5, 5)][:20]
    return case, receivers
