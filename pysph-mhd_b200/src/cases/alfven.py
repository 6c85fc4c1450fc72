"""Circularly polarised Alfven wave (src/cases/alfven.py) and its 2-D form.

``AlfvenWave``: the reference case (close-packed lattice, box 3 x 1.5 x 1.5,
B_perp amplitude 0.1, v_perp = B_perp).  ``AlfvenWave2D``: 2-D square lattice
of nx x 2nx particles in the periodic box [0, 1] x [0, 2], rho = 1,
p = 0.1, B_par = 1 along x, wavelength 1 along x, amplitude a (0.1):
B = (1, a sin phi, a cos phi), v = (0, a sin phi, a cos phi), phi = 2 pi x.
"""

import numpy as np

from ..application import MHDApplication, square_lattice
from .lattice import close_packed_lattice


class AlfvenWave(MHDApplication):
    @property
    def bounds(self):
        return -1.5, 1.5, -0.75, 0.75, -0.75, 0.75

    def create_mhd_particles(self):
        x, y, z = close_packed_lattice(self.bounds, 3.0 / self.nx)
        x, y, z = (a.astype(np.float32).astype(float) for a in (x, y, z))
        phase = 2.0 * np.pi * (x + 1.5)
        by, bz = 0.1 * np.sin(phase), 0.1 * np.cos(phase)
        count = len(x)
        mass = float(np.float32(6.75 / count))
        return dict(x=x, y=y, z=z, u=np.zeros(count), v=by, w=bz, rho=np.ones(count),
                    h=np.full(count, self.hfact * mass ** (1.0 / 3.0)), m=np.full(count, mass),
                    e=np.full(count, 0.15), Bx=np.ones(count), By=by, Bz=bz, alpha1=np.zeros(count))


class AlfvenWave2D(MHDApplication):
    amplitude = 0.1

    @property
    def bounds(self):
        return 0.0, 1.0, 0.0, 2.0, -0.5, 0.5

    def create_mhd_particles(self):
        n = self.nx
        x, y = square_lattice((n, 2 * n), (0.0, 0.0), (1.0, 2.0))
        count = len(x)
        a = self.amplitude
        phase = 2.0 * np.pi * x
        by, bz = a * np.sin(phase), a * np.cos(phase)
        mass = 2.0 / count
        return dict(x=x, y=y, z=np.zeros(count), u=np.zeros(count), v=by, w=bz, rho=np.ones(count),
                    h=np.full(count, self.hfact * np.sqrt(mass)), m=np.full(count, mass),
                    e=np.full(count, 0.1 / ((self.gamma - 1.0) * 1.0)), Bx=np.ones(count), By=by, Bz=bz,
                    alpha1=np.zeros(count))
