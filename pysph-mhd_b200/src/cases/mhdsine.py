"""Magnetic sine wave (src/cases/mhdsine.py): a uniform gas at rest, rho = 2,
e = 7.5, with By = sin(2 pi (x - xmin)) on a close-packed slab of
[-0.5, 0.5]^2 x [-4 sqrt6/nx, 4 sqrt6/nx]."""

import numpy as np

from ..application import MHDApplication
from .lattice import close_packed_lattice


def slab_bounds(x0, x1, y0, y1, nx):
    """The reference's thin periodic slab: z spans +-4 sqrt6 / nx."""
    half = 4.0 * np.sqrt(6.0) / nx
    return x0, x1, y0, y1, -half, half


def uniform_slab(bounds, nx, rho):
    """Close-packed points of `bounds` at spacing (xmax - xmin) / nx and the
    equal particle mass of a uniform density `rho`."""
    x, y, z = close_packed_lattice(bounds, (bounds[1] - bounds[0]) / nx)
    volume = (bounds[1] - bounds[0]) * (bounds[3] - bounds[2]) * (bounds[5] - bounds[4])
    return x, y, z, rho * volume / len(x)


class MHDSine(MHDApplication):
    @property
    def bounds(self):
        return slab_bounds(-0.5, 0.5, -0.5, 0.5, self.nx)

    def create_mhd_particles(self):
        xmin = self.bounds[0]
        rho = 2.0
        x, y, z, mass = uniform_slab(self.bounds, self.nx, rho)
        n = len(x)
        zero = np.zeros(n)
        return dict(x=x, y=y, z=z, u=zero.copy(), v=zero.copy(), w=zero.copy(), rho=np.full(n, rho),
                    h=np.full(n, self.hfact * (mass / rho) ** (1.0 / 3.0)), m=np.full(n, mass), e=np.full(n, 7.5),
                    Bx=zero.copy(), By=np.sin(2.0 * np.pi * (x - xmin)), Bz=zero.copy(), alpha1=zero.copy())
