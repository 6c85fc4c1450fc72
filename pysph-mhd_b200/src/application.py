"""MHDApplication: the reference's application driver (src/application.py) on B200.

Same hooks and order: ``initialize`` reads the config, ``create_particles``
wraps the case's arrays in a CUDA ``ParticleArray``, ``create_domain`` the
periodic box (``periodic_mode`` ``minimum_image``, or ``ghost``, which gives
the same pairs and displacements as the minimum image in a box wider than
twice the kernel reach; ``None`` gives an open domain), ``configure_scheme``
builds the solver, and ``solve`` runs the
warm-up (src/application.py:110-132), the initial timestep (:134-147) and the
time loop.  ``run()`` does all of it.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from .config import SimulationConfig
from .engine import Engine, params_from_dict
from .particle_array import ParticleArray
from .particles import INITIAL_PREDICTOR_PAIRS
from .scheme import MHDScheme


@dataclass
class Domain:
    lo: tuple
    hi: tuple
    periodic: tuple


class MHDApplication:
    config_type = SimulationConfig
    detailed_output = False  # dumps hold every property (restart files)

    def __init__(self, config):
        self.config = config
        self.fname = config.case.name
        self.initialize()
        self.scheme = self.create_scheme()
        self.particles = None
        self.engine = None

    def initialize(self):
        c = self.config
        self.gamma = c.physics.gamma
        self.mu0 = c.physics.mu0
        self.kernel = c.numerics.kernel
        self.hfact = c.numerics.hfact
        self.density = c.numerics.density
        self.periodic_mode = c.numerics.periodic_mode
        self.tf = c.solver.tf
        self.pfreq = c.solver.pfreq
        self.adaptive_timestep = c.solver.adaptive_timestep
        self.timestep_factor = c.solver.timestep_factor
        self.nx = c.case.nx
        self.dim = c.numerics.dim or 3

    # --- case hooks ---
    def create_mhd_particles(self) -> dict:
        raise NotImplementedError

    def refresh_initial_thermodynamics(self, particle):
        pass

    @property
    def bounds(self):
        raise NotImplementedError

    # --- reference hooks ---
    # The reference evaluates every equation of its groups, diagnostics
    # included (StrainDiagnostics' dvdx_*, the Cullen-Dehnen moments, the
    # density pass's arho/grho/dwdh); so does this application unless a
    # caller sets this to False before setup() (the state is the same).
    diagnostics = True

    def create_particles(self, device="cuda"):
        arrays = self.create_mhd_particles()
        pa = ParticleArray("fluid", arrays, device=device, diagnostics=self.diagnostics)
        self.scheme.setup_properties(pa)
        return [pa]

    def create_domain(self):
        xmin, xmax, ymin, ymax, zmin, zmax = self.bounds
        per = self.periodic_mode is not None
        return Domain((xmin, ymin, zmin), (xmax, ymax, zmax), (per, per, per and self.dim == 3))

    def create_scheme(self):
        return MHDScheme(self.config)

    def configure_scheme(self):
        self.scheme.configure_solver(dt=1.0, tf=self.tf, adaptive_timestep=self.adaptive_timestep, pfreq=self.pfreq,
                                     detailed_output=self.detailed_output,
                                     max_steps=self.config.solver.max_steps,
                                     output_directory=self.config.execution.directory, fname=self.fname)

    def setup(self, device="cuda"):
        """create_particles, create_domain, configure_scheme, and the engine."""
        self.particles = self.create_particles(device)
        self.domain = self.create_domain()
        self.configure_scheme()
        self.solver = self.scheme.solver
        self.solver.particles = self.particles
        prm = self.scheme.kernel_params(self.domain, self.tf)
        # execution.fused: the reference asks PySPH for fused CUDA kernels;
        # here it selects the fused production loop -- captured runs of
        # corrector-predictor steps with the adaptive step size kept on the
        # device (the literal MHDStep stages otherwise)
        fused = bool(self.config.execution.fused) and self.adaptive_timestep
        if fused:
            from .batch import BatchEngine

            self.engine = BatchEngine.single(params_from_dict(prm), self.particles[0])
        else:
            self.engine = Engine(params_from_dict(prm), self.particles[0])
        self.solver.fused = fused
        self.solver.integrator.set_engine(self.engine)
        return self

    # --- warm-up and initial dt (src/application.py:94-147) ---
    @staticmethod
    def _sync_initial_mhd_state(particle):
        particle.Bevolx.copy_(particle.Bx / particle.rho)
        particle.Bevoly.copy_(particle.By / particle.rho)
        particle.Bevolz.copy_(particle.Bz / particle.rho)
        particle.psi.zero_()
        for predicted, current in INITIAL_PREDICTOR_PAIRS:
            particle[predicted].copy_(particle[current])

    def _warm_initial_derivatives(self, solver):
        self.engine.warmup(refresh=self.refresh_initial_thermodynamics)
        solver.initial_acceleration_is_current = True

    def _compute_initial_dt(self, solver):
        solver.dt = self.engine.initial_dt()

    def solve(self):
        self._warm_initial_derivatives(self.solver)
        self._compute_initial_dt(self.solver)
        self.solver.solve()

    def run(self, device="cuda"):
        if self.engine is None:
            self.setup(device)
        self.solve()
        torch.cuda.synchronize()
        return self.particles[0]

    def restart(self, path, device="cuda"):
        """Continue a run from a dump written with ``detailed_output`` (every
        property: the state, the integrator copies and the last rates): the
        steps after it equal those of the uninterrupted run."""
        from .solver import load_output

        arrays, solver_data = load_output(path)
        missing = [k for k in ("x0", "au", "dt_adapt", "Bevolxpred") if k not in arrays]
        if missing:
            raise ValueError(f"{path} is not a detailed dump (lacks {missing}); write it with detailed_output")
        self.create_mhd_particles = lambda: arrays
        self.setup(device)
        self.solver.restore(solver_data)
        self.solver.solve()
        torch.cuda.synchronize()
        return self.particles[0]


def square_lattice(n_per_axis, lo, hi):
    """Cell-centred square (2-D) or cubic (3-D) lattice, x varying slowest."""
    axes = [lo[a] + (np.arange(n) + 0.5) * (hi[a] - lo[a]) / n for a, n in enumerate(n_per_axis)]
    grid = np.meshgrid(*axes, indexing="ij")
    return [g.ravel() for g in grid]
