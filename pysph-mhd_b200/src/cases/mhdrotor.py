"""MHD rotor (src/cases/mhdrotor.py): a dense disk (rho = 10, r <= 0.1)
spinning with angular velocity 2 / 0.1 in a gas of rho = 1, p = 1 everywhere,
Bx = 5 / sqrt(4 pi).  The disk is a second close-packed lattice with the
spacing shrunk by 10^(1/3), so all particles have one mass."""

import numpy as np

from ..application import MHDApplication
from .lattice import close_packed_lattice


class MHDRotor(MHDApplication):
    disk_radius = 0.1

    @property
    def bounds(self):
        half = 2.0 * np.sqrt(6.0) / self.nx
        return -0.5, 0.5, -0.5, 0.5, -half, half

    def create_mhd_particles(self):
        xmin, xmax, ymin, ymax, zmin, zmax = self.bounds
        dx = (xmax - xmin) / self.nx
        r0 = self.disk_radius
        ox, oy, oz = close_packed_lattice(self.bounds, dx)
        keep_out = ox * ox + oy * oy >= r0 ** 2
        ix, iy, iz = close_packed_lattice(self.bounds, dx * 10.0 ** (-1.0 / 3.0))
        keep_in = ix * ix + iy * iy <= r0 ** 2
        x = np.concatenate((ox[keep_out], ix[keep_in]))
        y = np.concatenate((oy[keep_out], iy[keep_in]))
        z = np.concatenate((oz[keep_out], iz[keep_in]))
        n = len(x)
        disk = np.sqrt(x * x + y * y) <= r0
        rho = np.where(disk, 10.0, 1.0)
        # the box's area at rho = 1 plus the disk's area at rho = 10, over all particles
        mass = ((xmax - xmin) * (ymax - ymin) + 10.0 * np.pi * r0 ** 2) * (zmax - zmin) / n
        omega = np.where(disk, 2.0 / r0, 0.0)
        zero = np.zeros(n)
        return dict(x=x, y=y, z=z, u=-omega * y, v=omega * x, w=zero.copy(), rho=rho,
                    h=self.hfact * (mass / rho) ** (1.0 / 3.0), m=np.full(n, mass), e=1.0 / ((self.gamma - 1.0) * rho),
                    Bx=np.full(n, 5.0 / np.sqrt(4.0 * np.pi)), By=zero.copy(), Bz=zero.copy(), alpha1=zero.copy())
