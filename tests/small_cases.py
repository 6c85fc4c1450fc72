"""Seeded small initial conditions for the parity tests (test infrastructure).

Positions get a seeded jitter so that div v and curl v are resolved
quantities rather than roundoff, which keeps the Cullen-Dehnen limiter
well-conditioned and allows strict FP64 tolerances.
"""

import math

import numpy as np

BASE = dict(density="iterate", mu0=1.0, av=1.0, ac=1.0, ar=1.0, clean_speed=1.0, clean_damp=1.0,
            timestep_factor=1.0, tf=1e30, alpha_min=0.0, alpha_max=1.0)


def orszag_tang_2d(n=32, kernel="quintic", hfact=1.2, jitter=0.05, seed=0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x = (-0.5 + (i + 0.5) * dx).ravel() + jitter * dx * rng.uniform(-1, 1, n * n)
    y = (-0.5 + (j + 0.5) * dx).ravel() + jitter * dx * rng.uniform(-1, 1, n * n)
    cnt = len(x)
    g = 5.0 / 3.0
    rho, p, b0 = 25.0 / (36.0 * math.pi), 5.0 / (12.0 * math.pi), 1.0 / math.sqrt(4.0 * math.pi)
    m = rho * dx * dx
    ic = dict(x=x, y=y, z=np.zeros(cnt), u=-np.sin(2 * np.pi * (y + 0.5)), v=np.sin(2 * np.pi * (x + 0.5)),
              w=np.zeros(cnt), rho=np.full(cnt, rho), h=np.full(cnt, hfact * dx), m=np.full(cnt, m),
              e=np.full(cnt, p / ((g - 1.0) * rho)), Bx=-b0 * np.sin(2 * np.pi * (y + 0.5)),
              By=b0 * np.sin(4 * np.pi * (x + 0.5)), Bz=np.zeros(cnt), alpha1=np.zeros(cnt),
              gid=np.arange(cnt, dtype=np.float64))
    prm = dict(BASE, dim=2, kernel=kernel, hfact=hfact, gamma=g, lo=[-0.5, -0.5, -0.5], hi=[0.5, 0.5, 0.5],
               periodic=[True, True, False])
    return ic, prm


def blast_3d(n=12, kernel="cubic", hfact=1.2, jitter=0.05, seed=1, alpha=(0.1, 1.0)):
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    pos = [(-0.5 + (a + 0.5) * dx).ravel() + jitter * dx * rng.uniform(-1, 1, n ** 3) for a in (i, j, k)]
    x, y, z = pos
    cnt = len(x)
    g = 5.0 / 3.0
    p = np.where(x * x + y * y + z * z < 0.25 ** 2, 10.0, 0.1)
    b = 1.0 / math.sqrt(2.0)
    ic = dict(x=x, y=y, z=z, u=np.zeros(cnt), v=np.zeros(cnt), w=np.zeros(cnt), rho=np.ones(cnt),
              h=np.full(cnt, hfact * dx), m=np.full(cnt, dx ** 3), e=p / (g - 1.0), Bx=np.full(cnt, b),
              By=np.full(cnt, b), Bz=np.zeros(cnt), alpha1=np.full(cnt, alpha[0]), gid=np.arange(cnt, dtype=float))
    prm = dict(BASE, dim=3, kernel=kernel, hfact=hfact, gamma=g, lo=[-0.5] * 3, hi=[0.5] * 3, periodic=[True] * 3,
               alpha_min=alpha[0], alpha_max=alpha[1])
    return ic, prm


def open_blob_2d(n=20, kernel="wendland_c2", hfact=1.3, seed=2):
    """A non-periodic square of gas with a pressure bump (periodic_mode None)."""
    rng = np.random.default_rng(seed)
    dx = 1.0 / n
    i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    x = ((i + 0.5) * dx).ravel() + 0.05 * dx * rng.uniform(-1, 1, n * n)
    y = ((j + 0.5) * dx).ravel() + 0.05 * dx * rng.uniform(-1, 1, n * n)
    cnt = len(x)
    g = 1.4
    r2 = (x - 0.5) ** 2 + (y - 0.5) ** 2
    p = 1.0 + 2.0 * np.exp(-r2 / 0.02)
    ic = dict(x=x, y=y, z=np.zeros(cnt), u=0.1 * (y - 0.5), v=-0.1 * (x - 0.5), w=np.zeros(cnt), rho=np.ones(cnt),
              h=np.full(cnt, hfact * dx), m=np.full(cnt, dx * dx), e=p / (g - 1.0), Bx=np.full(cnt, 0.3),
              By=np.zeros(cnt), Bz=np.full(cnt, 0.2), alpha1=np.zeros(cnt), gid=np.arange(cnt, dtype=float))
    prm = dict(BASE, dim=2, kernel=kernel, hfact=hfact, gamma=g, lo=[0.0] * 3, hi=[1.0] * 3,
               periodic=[False, False, False])
    return ic, prm
