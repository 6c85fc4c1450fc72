"""Magnetosonic pulse (src/cases/mhdwave.py): rho = 2, e = 0.75,
Bx = sqrt(2/3), and a Gaussian velocity pulse u = 0.01 exp(-(x / 3h)^2) on a
close-packed slab of [-2, 2] x [-1, 1] x [-4 sqrt6/nx, 4 sqrt6/nx]."""

import numpy as np

from ..application import MHDApplication
from .mhdsine import slab_bounds, uniform_slab


class MHDWave(MHDApplication):
    @property
    def bounds(self):
        return slab_bounds(-2.0, 2.0, -1.0, 1.0, self.nx)

    def create_mhd_particles(self):
        rho = 2.0
        x, y, z, mass = uniform_slab(self.bounds, self.nx, rho)
        n = len(x)
        h = self.hfact * (mass / rho) ** (1.0 / 3.0)
        zero = np.zeros(n)
        return dict(x=x, y=y, z=z, u=0.01 * np.exp(-((x / (3.0 * h)) ** 2)), v=zero.copy(), w=zero.copy(),
                    rho=np.full(n, rho), h=np.full(n, h), m=np.full(n, mass), e=np.full(n, 0.75),
                    Bx=np.full(n, np.sqrt(2.0 / 3.0)), By=zero.copy(), Bz=zero.copy(), alpha1=zero.copy())
