"""Current-loop advection (src/cases/jadvect.py): a weak azimuthal field
loop |B| = 1e-3 inside r < 0.3 carried by a uniform flow (2, 1, 0.1 sqrt5),
rho = 1, e = 1.5, on a close-packed slab of [-1, 1] x [-0.5, 0.5] x
[-4 sqrt6/nx, 4 sqrt6/nx]."""

import numpy as np

from ..application import MHDApplication
from .mhdsine import slab_bounds, uniform_slab


class CurrentLoopAdvection(MHDApplication):
    loop_radius = 0.3
    amplitude = 1.0e-3

    @property
    def bounds(self):
        return slab_bounds(-1.0, 1.0, -0.5, 0.5, self.nx)

    def create_mhd_particles(self):
        rho = 1.0
        x, y, z, mass = uniform_slab(self.bounds, self.nx, rho)
        n = len(x)
        r = np.sqrt(x * x + y * y)
        inside = r < self.loop_radius
        bx, by = np.zeros(n), np.zeros(n)
        bx[inside] = -self.amplitude * y[inside] / r[inside]
        by[inside] = self.amplitude * x[inside] / r[inside]
        return dict(x=x, y=y, z=z, u=np.full(n, 2.0), v=np.full(n, 1.0), w=np.full(n, 0.1 * np.sqrt(5.0)),
                    rho=np.full(n, rho), h=np.full(n, self.hfact * (mass / rho) ** (1.0 / 3.0)), m=np.full(n, mass),
                    e=np.full(n, 1.5), Bx=bx, By=by, Bz=np.zeros(n), alpha1=np.zeros(n))
