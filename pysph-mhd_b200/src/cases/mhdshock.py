"""Brio-Wu shock tube (src/cases/mhdshock.py) and its 2-D lattice form.

``MHDShock``: the reference case (close-packed 3-D slab, frozen ends).
``MHDShock2D``: left 2 nx x nx/16 square lattice on [-0.5, 0) x [0, 1/32]
(nx = 2048 gives the benchmark's 4096 x 128 slab), right side at density
1/8 with equal masses (45 rows for 128 left rows), periodic in y; the box is
widened by 0.25 in x and particles within 6 spacings of the ends are frozen
(itype 3) as in the reference.
"""

import numpy as np

from ..application import MHDApplication
from .lattice import close_packed_lattice


class MHDShock(MHDApplication):
    @property
    def bounds(self):
        dx_left = 0.5 / self.nx
        dx_right = 2.0 * dx_left
        ymax = 6.0 * dx_right * np.sqrt(3.0 / 4.0)
        zmax = 6.0 * dx_right * np.sqrt(6.0) / 3.0
        return -0.5 - 1000.0 * dx_left, 0.5 + 1000.0 * dx_right, -ymax, ymax, -zmax, zmax

    def create_mhd_particles(self):
        assert self.nx % 2 == 0
        _, _, ymin, ymax, zmin, zmax = self.bounds
        dx_left = 0.5 / self.nx
        dx_right = 2.0 * dx_left
        left = close_packed_lattice((-0.5, 0.0, ymin, ymax, zmin, zmax), dx_left)
        right = close_packed_lattice((0.0, 0.5, ymin, ymax, zmin, zmax), dx_right)
        x, y, z = (np.concatenate((a, b)) for a, b in zip(left, right))
        count = len(x)
        is_left = x <= 0.0
        rho = np.where(is_left, 1.0, 0.125)
        pressure = np.where(is_left, 1.0, 0.1)
        mass = 0.5 * (ymax - ymin) * (zmax - zmin) / len(left[0])
        itype = np.where((x < -0.5 + 6.0 * dx_left) | (x > 0.5 - 6.0 * dx_right), 3, 1).astype(np.int32)
        return dict(x=x, y=y, z=z, u=np.zeros(count), v=np.zeros(count), w=np.zeros(count), rho=rho,
                    h=self.hfact * (mass / rho) ** (1.0 / 3.0), m=np.full(count, mass),
                    e=pressure / ((self.gamma - 1.0) * rho), Bx=np.full(count, 0.75), By=np.where(is_left, 1.0, -1.0),
                    Bz=np.zeros(count), alpha1=np.zeros(count), itype=itype)


class MHDShock2D(MHDApplication):
    @property
    def bounds(self):
        ly = (self.nx // 16) * (0.5 / self.nx)
        return -0.75, 0.75, 0.0, ly, -0.5, 0.5

    def create_mhd_particles(self):
        nl = self.nx  # left columns
        dx = 0.5 / nl
        rows = nl // 16
        ly = rows * dx
        i, j = np.meshgrid(np.arange(nl), np.arange(rows), indexing="ij")
        xl, yl = (-0.5 + (i + 0.5) * dx).ravel(), ((j + 0.5) * dx).ravel()
        rows_r = int(round(rows / np.sqrt(8.0)))
        dyr = ly / rows_r
        dxr = 8.0 * dx * dx / dyr
        cols_r = int(round(0.5 / dxr))
        dxr = 0.5 / cols_r
        i, j = np.meshgrid(np.arange(cols_r), np.arange(rows_r), indexing="ij")
        xr, yr = ((i + 0.5) * dxr).ravel(), ((j + 0.5) * dyr).ravel()
        x, y = np.concatenate((xl, xr)), np.concatenate((yl, yr))
        count = len(x)
        left = x < 0.0
        m = dx * dx
        rho = np.where(left, 1.0, 0.125)
        pressure = np.where(left, 1.0, 0.1)
        itype = np.where((x < -0.5 + 6 * dx) | (x > 0.5 - 6 * dxr), 3, 1).astype(np.int32)
        return dict(x=x, y=y, z=np.zeros(count), u=np.zeros(count), v=np.zeros(count), w=np.zeros(count), rho=rho,
                    h=self.hfact * np.sqrt(m / rho), m=np.full(count, m), e=pressure / ((self.gamma - 1.0) * rho),
                    Bx=np.full(count, 0.75), By=np.where(left, 1.0, -1.0), Bz=np.zeros(count), alpha1=np.zeros(count),
                    itype=itype)
