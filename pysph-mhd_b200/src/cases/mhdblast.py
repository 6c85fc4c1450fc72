"""MHD blast (src/cases/mhdblast.py) and the benchmark's 3-D blast.

``MHDBlast``: the reference case (close-packed lattice, p = 100 inside
r < 0.125 else 1, B = 10/sqrt2 along x and z).  ``MHDBlast3D``: nx^3 cubic
lattice in the periodic unit cube, rho = 1, p = 10 inside r < 0.1 else 0.1,
B = (1/sqrt2, 1/sqrt2, 0), alpha starting at alpha_min.
"""

import numpy as np

from ..application import MHDApplication, square_lattice
from .lattice import close_packed_lattice


class MHDBlast(MHDApplication):
    @property
    def bounds(self):
        return -0.5, 0.5, -0.5, 0.5, -0.5, 0.5

    def create_mhd_particles(self):
        xmin, xmax, ymin, ymax, zmin, zmax = self.bounds
        x, y, z = close_packed_lattice(self.bounds, (xmax - xmin) / self.nx)
        count = len(x)
        mass = 1.0 / count
        pressure = np.where(x * x + y * y + z * z < 0.125 ** 2, 100.0, 1.0)
        b = 10.0 / np.sqrt(2.0)
        return dict(x=x, y=y, z=z, u=np.zeros(count), v=np.zeros(count), w=np.zeros(count), rho=np.ones(count),
                    h=np.full(count, self.hfact * mass ** (1.0 / 3.0)), m=np.full(count, mass),
                    e=pressure / (self.gamma - 1.0), Bx=np.full(count, b), By=np.zeros(count), Bz=np.full(count, b),
                    alpha1=np.zeros(count))


class MHDBlast3D(MHDApplication):
    @property
    def bounds(self):
        return -0.5, 0.5, -0.5, 0.5, -0.5, 0.5

    def create_mhd_particles(self):
        n = self.nx
        x, y, z = square_lattice((n, n, n), (-0.5,) * 3, (0.5,) * 3)
        count = len(x)
        mass = 1.0 / count
        pressure = np.where(x * x + y * y + z * z < 0.1 ** 2, 10.0, 0.1)
        b = 1.0 / np.sqrt(2.0)
        a0 = self.config.physics.alpha_min or 0.0
        return dict(x=x, y=y, z=z, u=np.zeros(count), v=np.zeros(count), w=np.zeros(count), rho=np.ones(count),
                    h=np.full(count, self.hfact / n), m=np.full(count, mass), e=pressure / (self.gamma - 1.0),
                    Bx=np.full(count, b), By=np.full(count, b), Bz=np.zeros(count), alpha1=np.full(count, a0))
