"""Colliding plasma jets (src/cases/jet.py): 1, 3 or 12 argon jets (case
names ``1jet``, ``3jet``, ``12jet``; axes in the x-z plane at 0, +-30 or every
30 degrees) fired at the origin of an open [-2, 2]^3 box, SI units.

Each jet is a close-packed cylinder of radius R between axial positions
inner_radius and outer_radius (spacing 2 R / nx), moving inward at
axial_speed with a swirl, and threaded by a helical field: an axial
component B_a (1 - s^2)^3 (1 - 5 s^2), a toroidal one peaking at B_t, and the
radial one that keeps div B = 0 under the tanh end tapers (s = r / R).  The
gas is uniform: rho = n m_Ar, p = rho (k T / m) from the temperature in eV.
The ``[jet]`` table of the TOML file holds the jet parameters.
"""

from __future__ import annotations

from dataclasses import dataclass
from math import cos, pi, sin

import numpy as np

from ..application import MHDApplication
from ..config import SimulationConfig, _check
from .lattice import close_packed_lattice

ARGON_MASS_NUMBER = 39.948
ARGON_MOLAR_MASS = 0.039948  # kg/mol
ATOMIC_MASS = 1.6726231e-27  # kg per mass number unit, as the reference takes it
EV_TO_K = 11604.505
GAS_CONSTANT = 8.31  # J/(mol K), as the reference rounds it

JET_ANGLES = {"1jet": (0.0,), "3jet": (0.0, 30.0, -30.0), "12jet": tuple(30.0 * k for k in range(12))}
# peak of s (1 - s^2)^3 over [0, 1] (at s = 1/sqrt7): normalises the swirl
# and the toroidal field to their stated peaks
_PEAK = 216.0 / (343.0 * np.sqrt(7.0))


@dataclass(frozen=True)
class JetConfig:
    inner_radius: float
    outer_radius: float
    radius: float
    end_taper_fraction: float
    axial_speed: float
    azimuthal_speed: float
    temperature_ev: float
    number_density: float
    axial_field: float
    toroidal_field: float


@dataclass(frozen=True)
class JetSimulationConfig(SimulationConfig):
    jet: JetConfig

    def validate(self):
        super().validate()
        j = self.jet
        _check(self.case.name in JET_ANGLES, "case.name (1jet, 3jet or 12jet)")
        for k in ("inner_radius", "outer_radius", "radius", "end_taper_fraction", "axial_speed", "azimuthal_speed",
                  "temperature_ev", "number_density", "axial_field", "toroidal_field"):
            _check(type(getattr(j, k)) is float, f"jet.{k}")
        _check(j.inner_radius >= 0.0 and j.outer_radius > j.inner_radius, "jet.inner_radius / outer_radius")
        _check(j.radius > 0.0, "jet.radius")
        _check(0.0 < j.end_taper_fraction <= 0.5, "jet.end_taper_fraction")
        _check(j.axial_speed > 0.0 and j.azimuthal_speed >= 0.0, "jet speeds")
        _check(j.temperature_ev > 0.0 and j.number_density > 0.0, "jet.temperature_ev / number_density")
        _check(j.axial_field >= 0.0 and j.toroidal_field >= 0.0, "jet fields")


def _jet_profiles(axial, cy, cz, jet):
    """Radius, 1/radius (0 on the axis), s = r / R, 1 - s^2, and the axial
    envelope with its derivative along -axial."""
    r = np.sqrt(cy * cy + cz * cz)
    inv_r = np.divide(1.0, r, out=np.zeros_like(r), where=r > 0.0)
    s = r / jet.radius
    rem = 1.0 - s * s
    length = jet.outer_radius - jet.inner_radius
    taper = jet.end_taper_fraction * length
    local = 0.5 * (jet.inner_radius + jet.outer_radius) - axial
    ap = (local + 0.5 * length) / taper
    am = (local - 0.5 * length) / taper
    env = 0.5 * (np.tanh(ap) - np.tanh(am))
    denv = 0.5 * (1.0 / np.cosh(ap) ** 2 - 1.0 / np.cosh(am) ** 2) / taper
    return r, inv_r, s, rem, env, denv


def _rotate(a, py, pz, c, s_):
    """A vector given as (axial, y, cross-z) components for a jet whose axis
    points along (cos, 0, sin), pointing inward: world (x, y, z)."""
    return -a * c - pz * s_, py, -a * s_ + pz * c


class JMXJets(MHDApplication):
    config_type = JetSimulationConfig

    @property
    def bounds(self):
        return -2.0, 2.0, -2.0, 2.0, -2.0, 2.0

    @property
    def dx(self):
        return 2.0 * self.config.jet.radius / self.nx

    def _one_jet(self):
        j = self.config.jet
        box = (j.inner_radius, j.outer_radius, -j.radius, j.radius, -j.radius, j.radius)
        a, cy, cz = close_packed_lattice(box, self.dx)
        keep = cy * cy + cz * cz < j.radius ** 2
        return a[keep], cy[keep], cz[keep]

    def create_mhd_particles(self):
        j = self.config.jet
        a, cy, cz = self._one_jet()
        r, inv_r, s, rem, env, denv = _jet_profiles(a, cy, cz, j)
        # helical field in the jet frame
        b_ax = j.axial_field * rem ** 3 * (1.0 - 5.0 * s ** 2) * env
        b_r = -0.5 * j.axial_field * r * rem ** 4 * denv
        b_t = j.toroidal_field * s * rem ** 3 / _PEAK * env
        b_y = (b_r * cy + b_t * cz) * inv_r
        b_z = (b_r * cz - b_t * cy) * inv_r
        # swirl in the jet frame
        v_t = j.azimuthal_speed * s * rem ** 3 / _PEAK * env
        v_y = v_t * cz * inv_r
        v_z = -v_t * cy * inv_r
        pos, vel, mag = [], [], []
        for deg in JET_ANGLES[self.config.case.name]:
            c, sn = cos(deg * pi / 180.0), sin(deg * pi / 180.0)
            pos.append((a * c - cz * sn, cy, a * sn + cz * c))
            vel.append(_rotate(j.axial_speed, v_y, v_z, c, sn))
            mag.append(_rotate(b_ax, b_y, b_z, c, sn))
        cat = lambda vs, k: np.concatenate([np.broadcast_to(v[k], a.shape) for v in vs])  # noqa: E731
        x, y, z = cat(pos, 0), cat(pos, 1), cat(pos, 2)
        n = len(x)
        rho = j.number_density * ARGON_MASS_NUMBER * ATOMIC_MASS
        pressure = rho * (j.temperature_ev * EV_TO_K) * GAS_CONSTANT / ARGON_MOLAR_MASS
        volume = pi * j.radius ** 2 * (j.outer_radius - j.inner_radius) / len(a)
        return dict(x=x, y=y, z=z, u=cat(vel, 0), v=cat(vel, 1), w=cat(vel, 2), rho=np.full(n, rho),
                    h=np.full(n, self.hfact * volume ** (1.0 / 3.0)), m=np.full(n, rho * volume),
                    e=np.full(n, pressure / ((self.gamma - 1.0) * rho)), gid=np.arange(n, dtype=np.float64),
                    Bx=cat(mag, 0), By=cat(mag, 1), Bz=cat(mag, 2), alpha1=np.zeros(n))
