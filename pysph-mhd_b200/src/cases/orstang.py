"""Orszag-Tang vortex (src/cases/orstang.py) and its 2-D square-lattice form.

``OrszagTang``: the reference's 3-D close-packed slab (bounds
[-0.5, 0.5]^2 x [-4 sqrt6/nx, 4 sqrt6/nx]).  ``OrszagTang2D``: nx x nx
square lattice in the periodic unit box, dim 2 -- the benchmark's CPU
configuration (rho = 25/(36 pi), p = 5/(12 pi), B0 = 1/sqrt(4 pi)).
"""

import numpy as np

from ..application import MHDApplication, square_lattice
from .lattice import close_packed_lattice


def _fields(x, y, count, mass, rho, gamma, hfact, dim, xmin, ymin, b0scale=1.0):
    b0 = b0scale / np.sqrt(4.0 * np.pi)
    pressure = 0.5 * (1.0 / np.sqrt(4.0 * np.pi)) ** 2 * (10.0 / 3.0)
    return dict(
        u=-np.sin(2.0 * np.pi * (y - ymin)), v=np.sin(2.0 * np.pi * (x - xmin)), w=np.zeros(count),
        rho=np.full(count, rho), h=np.full(count, hfact * (mass / rho) ** (1.0 / dim)), m=np.full(count, mass),
        e=np.full(count, pressure / ((gamma - 1.0) * rho)), Bx=-b0 * np.sin(2.0 * np.pi * (y - ymin)),
        By=b0 * np.sin(4.0 * np.pi * (x - xmin)), Bz=np.zeros(count), alpha1=np.zeros(count))


class OrszagTang(MHDApplication):
    @property
    def bounds(self):
        zmax = 4.0 * np.sqrt(6.0) / self.nx
        return -0.5, 0.5, -0.5, 0.5, -zmax, zmax

    def create_mhd_particles(self):
        xmin, xmax, ymin, ymax, zmin, zmax = self.bounds
        x, y, z = close_packed_lattice(self.bounds, (xmax - xmin) / self.nx)
        count = len(x)
        pressure = 0.5 * (1.0 / np.sqrt(4.0 * np.pi)) ** 2 * (10.0 / 3.0)
        rho = self.gamma * pressure
        mass = rho * (xmax - xmin) * (ymax - ymin) * (zmax - zmin) / count
        return dict(x=x, y=y, z=z, **_fields(x, y, count, mass, rho, self.gamma, self.hfact, 3, xmin, ymin))


class OrszagTang2D(MHDApplication):
    @property
    def bounds(self):
        return -0.5, 0.5, -0.5, 0.5, -0.5, 0.5

    def create_mhd_particles(self, b0scale=1.0):
        n = self.nx
        x, y = square_lattice((n, n), (-0.5, -0.5), (0.5, 0.5))
        count = len(x)
        rho = 25.0 / (36.0 * np.pi)
        mass = rho / count
        return dict(x=x, y=y, z=np.zeros(count),
                    **_fields(x, y, count, mass, rho, self.gamma, self.hfact, 2, -0.5, -0.5, b0scale))


def orszag_tang_batch(config, n_inst=64, n_min=32, n_max=256, b0_range=(0.8, 1.2), seed=0):
    """The batched workload: ``n_inst`` independent 2-D Orszag-Tang
    instances (``OrszagTang2D`` with ``config``), instance k an N_k x N_k
    square lattice with N_k uniform in [n_min, n_max] and B0 scaled by a
    factor uniform in ``b0_range``, both drawn from ``seed``.  Returns the
    instance arrays, the shared kernel parameters, the sizes and the scales."""
    from dataclasses import replace

    rng = np.random.default_rng(seed)
    sizes = rng.integers(n_min, n_max + 1, n_inst)
    scales = rng.uniform(b0_range[0], b0_range[1], n_inst)
    instances, params = [], None
    for n, s in zip(sizes, scales):
        app = OrszagTang2D(replace(config, case=replace(config.case, nx=int(n))))
        instances.append(app.create_mhd_particles(b0scale=float(s)))
        if params is None:
            params = app.scheme.kernel_params(app.create_domain(), app.tf)
    return instances, params, sizes, scales
