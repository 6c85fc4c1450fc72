"""Advected MHD vortex (src/cases/mhdvortex.py): rho = 1 moving with
(1, 1, 1) plus a swirl and an equal magnetic swirl of strength
exp((1 - r^2) / 2) / (2 pi), in pressure balance
p = 1 + exp(1 - r^2) ((1 - r^2) - 1) / (8 pi^2), on a close-packed slab of
[-5, 5]^2 x [-4 sqrt6/nx, 4 sqrt6/nx].  The warm-up resets e from that p
with the summed density (``refresh_initial_thermodynamics``)."""

import numpy as np

from ..application import MHDApplication
from .mhdsine import slab_bounds, uniform_slab


def vortex_pressure(x, y):
    s = 1.0 - x * x - y * y
    return 1.0 + np.exp(s) * (s - 1.0) / (8.0 * np.pi ** 2)


class MHDVortex(MHDApplication):
    @property
    def bounds(self):
        return slab_bounds(-5.0, 5.0, -5.0, 5.0, self.nx)

    def refresh_initial_thermodynamics(self, particle):
        particle.e[:] = vortex_pressure(particle.x, particle.y) / ((self.gamma - 1.0) * particle.rho)

    def create_mhd_particles(self):
        rho = 1.0
        x, y, z, mass = uniform_slab(self.bounds, self.nx, rho)
        n = len(x)
        swirl = np.exp(0.5 * (1.0 - x * x - y * y)) / (2.0 * np.pi)
        return dict(x=x, y=y, z=z, u=1.0 - y * swirl, v=1.0 + x * swirl, w=np.ones(n), rho=np.full(n, rho),
                    h=np.full(n, self.hfact * (mass / rho) ** (1.0 / 3.0)), m=np.full(n, mass),
                    e=vortex_pressure(x, y) / (rho * (self.gamma - 1.0)), Bx=-y * swirl, By=x * swirl,
                    Bz=np.zeros(n), alpha1=np.zeros(n))
