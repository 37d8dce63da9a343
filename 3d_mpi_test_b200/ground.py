"""Impedance ground for the south-face TDBC (tdbc_ground.dat): the Miki
model of a rigid-frame porous ground and a fit of the solver's 6-pole
recursive convolution to it.

The reference's TDBC (calculation_2D.cpp:986-1017, poles
calculation_2D.h:73-75) acts on the east face with fixed poles; the same
recursion on the ground face takes its poles from tdbc_ground.dat
("Zinf tau", six a, six r). With dt' = dt / tau the solver advances

    p / Zinf = v_n + sum_q psi_q,   psi_q <- exp(-r_q dt') psi_q + a_q dt' v_n

(v_n the velocity into the ground), whose impedance at angular frequency w
(time convention exp(+i w t)) is exactly

    Z_d(w) = Zinf (1 + sum_q a_q dt' / (1 - exp(-r_q dt') exp(-i w dt)))

and tends to the continuous Zinf (1 + sum_q a_q / (r_q + i w tau)) as
dt -> 0. `fit_tdbc` fits a_q, r_q >= 0 (a passive, hence stable, boundary)
to Miki's impedance over a band, on the discrete response when dt is
given."""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

RHO0 = 1.2
C0 = 343.0


def miki_impedance(f, sigma: float, rho0: float = RHO0, c0: float = C0) -> np.ndarray:
    """Characteristic impedance (Pa s/m) of a rigid-frame porous medium of
    flow resistivity `sigma` (Pa s/m^2) after Miki (1990):
    Z = rho0 c0 (1 + 5.50 X^-0.632 - i 8.43 X^-0.632), X = f / sigma with
    sigma in kPa s/m^2 (time convention exp(+i w t)). A semi-infinite
    ground of this medium has this surface impedance."""
    X = 1000.0 * np.asarray(f, dtype=np.float64) / sigma
    t = X ** -0.632
    return rho0 * c0 * (1.0 + 5.50 * t - 1j * 8.43 * t)


def tdbc_impedance(f, Zinf: float, tau: float, a: Sequence[float], r: Sequence[float],
                   dt: Optional[float] = None) -> np.ndarray:
    """Impedance (Pa s/m) of the 6-pole TDBC at frequencies f (Hz): the
    discrete recursion's exact response with dt, the continuous one
    without."""
    w = 2.0 * np.pi * np.atleast_1d(np.asarray(f, dtype=np.float64))
    a = np.asarray(a, dtype=np.float64)
    r = np.asarray(r, dtype=np.float64)
    if dt is None:
        phi = 1.0 / (r[None, :] + 1j * w[:, None] * tau)
    else:
        dtp = dt / tau
        phi = dtp / (1.0 - np.exp(-r * dtp)[None, :] * np.exp(-1j * w * dt)[:, None])
    return Zinf * (1.0 + phi @ a)


def reflection(Z, theta: float = 0.0, rho0: float = RHO0, c0: float = C0):
    """Plane-wave pressure reflection coefficient of a locally reacting
    surface of impedance Z at incidence angle theta (from the normal)."""
    zc = np.asarray(Z) * np.cos(theta) / (rho0 * c0)
    return (zc - 1.0) / (zc + 1.0)


def normal_reflection(Zd, f, dt: float, dz: float, rho0: float = RHO0, c0: float = C0):
    """Reflection coefficient at normal incidence, referred to the face,
    that the FB_p_v scheme (p on nodes, w half a cell below node k and half
    a step after p) produces with a ground-face operator of impedance Zd
    (`tdbc_impedance` with dt). A plane wave p_k = exp(i(w n dt +- kz k dz))
    obeys sin(w dt / 2) = nu sin(kz dz / 2), nu = c0 dt / dz, and w(k) =
    -+ exp(i w dt / 2) exp(+- i kz dz / 2) p / (rho0 c0); the boundary
    relation p(1) = -Zd w(1) then gives R = (zeta - e^{i phi}) /
    (zeta + e^{-i phi}) with zeta = Zd e^{i w dt / 2} / (rho0 c0) and
    phi = kz dz / 2, which tends to (Z - rho0 c0) / (Z + rho0 c0) as dz -> 0."""
    f = np.asarray(f, dtype=np.float64)
    th = 2.0 * np.pi * f * dt
    phi = np.arcsin(np.sin(th / 2.0) / (c0 * dt / dz))
    zeta = np.asarray(Zd) * np.exp(0.5j * th) / (rho0 * c0)
    return (zeta - np.exp(1j * phi)) / (zeta + np.exp(-1j * phi))


@dataclass
class GroundFit:
    Zinf: float
    tau: float
    a: np.ndarray
    r: np.ndarray
    dt: Optional[float]
    f: np.ndarray          # fit frequencies (Hz)
    rel_err: np.ndarray    # |Z_tdbc - Z_miki| / |Z_miki| at f

    @property
    def max_rel_err(self) -> float:
        return float(self.rel_err.max())

    def impedance(self, f, dt: Optional[float] = None) -> np.ndarray:
        return tdbc_impedance(f, self.Zinf, self.tau, self.a, self.r, self.dt if dt is None else dt)

    def dat(self) -> str:
        """tdbc_ground.dat contents: Zinf tau / a0..a5 / r0..r5."""
        return (f"{self.Zinf!r} {self.tau!r}\n" + " ".join(repr(float(x)) for x in self.a) + "\n"
                + " ".join(repr(float(x)) for x in self.r) + "\n")


def fit_tdbc(sigma: float, f_lo: float = 20.0, f_hi: float = 2500.0, dt: Optional[float] = None,
             npole: int = 6, tau: Optional[float] = None, rho0: float = RHO0, c0: float = C0,
             nfreq: int = 80, starts: int = 8, seed: int = 0) -> GroundFit:
    """Fits the TDBC poles to Miki's impedance at flow resistivity `sigma`
    over [f_lo, f_hi] (log-spaced frequencies, relative complex error), on
    the discrete recursion's response when dt is given. Zinf = rho0 c0
    (Miki's high-frequency limit); tau defaults to 1 / (2 pi sqrt(f_lo
    f_hi)). Each of `starts` seeded starts spreads the poles log-uniformly
    over the band, takes the a's by non-negative least squares, then
    refines log a and log r together (trust-region least squares, so a,
    r > 0); the lowest cost wins. The optimum often leaves a pole unused
    (a ~ 0); the recursion still carries six."""
    from scipy.optimize import least_squares, nnls

    if dt is not None and f_hi >= 0.5 / dt:
        raise ValueError("f_hi must stay below the Nyquist frequency 1 / (2 dt)")
    Zinf = rho0 * c0
    if tau is None:
        tau = 1.0 / (2.0 * np.pi * np.sqrt(f_lo * f_hi))
    f = np.geomspace(f_lo, f_hi, nfreq)
    w = 2.0 * np.pi * f
    target = miki_impedance(f, sigma, rho0, c0)
    y = target / Zinf - 1.0
    wgt = Zinf / np.abs(target)

    def basis(r):
        if dt is None:
            return 1.0 / (r[None, :] + 1j * w[:, None] * tau)
        dtp = dt / tau
        return dtp / (1.0 - np.exp(-r * dtp)[None, :] * np.exp(-1j * w * dt)[:, None])

    def resid(x):
        x = np.clip(x, -40.0, 40.0)
        e = (basis(np.exp(x[npole:])) @ np.exp(x[:npole]) - y) * wgt
        return np.concatenate([e.real, e.imag])

    rng = np.random.default_rng(seed)
    rhs = np.concatenate([(y * wgt).real, (y * wgt).imag])
    best = None
    for _ in range(starts):
        lo = f_lo / 4.0 * np.exp(rng.normal(0.0, 0.5))
        hi = f_hi * 2.0 * np.exp(rng.normal(0.0, 0.5))
        r0 = 2.0 * np.pi * tau * np.geomspace(lo, hi, npole) * np.exp(rng.normal(0.0, 0.2, npole))
        B = basis(r0) * wgt[:, None]
        a0, _ = nnls(np.vstack([B.real, B.imag]), rhs)
        a0 = np.maximum(a0, 1e-6 * max(a0.max(), 1e-30))
        with np.errstate(over="ignore", invalid="ignore"):
            sol = least_squares(resid, np.concatenate([np.log(a0), np.log(r0)]), method="trf",
                                x_scale="jac", max_nfev=3000)
        if np.isfinite(sol.cost) and (best is None or sol.cost < best.cost):
            best = sol
    x = np.clip(best.x, -40.0, 40.0)
    a = np.exp(x[:npole])
    r = np.exp(x[npole:])
    order = np.argsort(r)
    a, r = a[order], r[order]
    got = tdbc_impedance(f, Zinf, tau, a, r, dt)
    return GroundFit(Zinf=Zinf, tau=float(tau), a=a, r=r, dt=dt, f=f,
                     rel_err=np.abs(got - target) / np.abs(target))
