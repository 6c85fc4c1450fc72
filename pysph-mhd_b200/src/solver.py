"""MHDSolver: the reference's time loop (src/solver.py:22-77) on the B200 path.

The loop is the reference's: skip the start-up RHS when the application has
already warmed it, ``dt = _get_timestep()``, step while ``tf - t`` exceeds the
tolerance and ``count < max_steps``, dump every ``pfreq`` steps.  The step and
the timestep reduction run on the device (``src.engine.Engine``).

A dump is an ``.npz`` ordered by ``gid`` in PySPH's version-2 layout: a
pickled ``particles`` dict ({name: {"name", "arrays", "constants",
"output_property_arrays"}}) and a ``solver_data`` dict (t, dt, count), as
PySPH's ``dump``/``load`` write and read them (restated from PySPH's
documented format, not checked against PySPH, which is not installed), plus
the same arrays and t, dt, count as plain top-level keys.  It holds
``OUTPUT_PROPERTIES``, or every property with ``detailed_output``: such a
dump restarts the run exactly (``MHDApplication.restart``).
"""

from __future__ import annotations

import logging
import os

import numpy as np

from .particles import OUTPUT_PROPERTIES

logger = logging.getLogger(__name__)

EPSILON = 2.220446049250313e-16


class MHDSolver:
    def __init__(self, dim=3, integrator=None, kernel="cubic", dt=1.0, tf=1.0, adaptive_timestep=True, pfreq=1,
                 max_steps=None, output_directory=None, fname="mhd", detailed_output=False, **kw):
        self.detailed_output = detailed_output
        self.dim = dim
        self.integrator = integrator
        self.kernel = kernel
        self.dt = dt
        self.tf = tf
        self.adaptive_timestep = adaptive_timestep
        self.pfreq = pfreq
        self.max_steps = max_steps if max_steps is not None else (1 << 62)
        self.output_directory = output_directory
        self.fname = fname
        self.t = 0.0
        self.count = 0
        self.initial_acceleration_is_current = False
        self.pre_step_callbacks = []
        self.post_step_callbacks = []
        self.particles = None
        # the fused loop (set by MHDApplication from execution.fused): steps
        # run as captured chunks that end at every dump; callbacks then run
        # once per chunk
        self.fused = False
        self.chunk = 50

    def _get_timestep(self):
        if self.adaptive_timestep:
            return self.integrator.compute_time_step(self.dt, t=self.t)
        dt = self.dt
        if self.t + dt > self.tf:
            dt = self.tf - self.t
        return dt

    def dump_output(self):
        if self.output_directory is None or self.particles is None:
            return None
        os.makedirs(self.output_directory, exist_ok=True)
        pa = self.particles[0]
        names = tuple(pa.properties) if self.detailed_output else OUTPUT_PROPERTIES
        arrays = pa.pull(*names, order="gid")
        path = os.path.join(self.output_directory, f"{self.fname}_{self.count:06d}.npz")
        solver_data = {"t": self.t, "dt": self.dt, "count": self.count}
        particles = {pa.name: {"name": pa.name, "arrays": arrays, "constants": {},
                               "output_property_arrays": list(OUTPUT_PROPERTIES)}}
        blob = {"version": np.array(2), "particles": np.array(particles, dtype=object),
                "solver_data": np.array(solver_data, dtype=object)}
        np.savez(path, t=self.t, dt=self.dt, count=self.count, **blob, **arrays)
        return path

    def restore(self, solver_data):
        """Continue from a dump's clock: the state already holds the rates of
        the last right-hand side."""
        self.t = float(solver_data["t"])
        self.count = int(solver_data["count"])
        self.dt = float(solver_data["dt"])
        self.initial_acceleration_is_current = True

    def _solve_fused(self):
        """The same loop in captured chunks of at most ``chunk`` steps: each
        chunk is the predictor of its first step, then fused corrector-
        predictor steps with dt = min(dt_adapt) (clipped to tf) reduced on
        the device, the last step finished by its corrector; a chunk ends at
        every dump, at max_steps, and within two of its steps of tf (the
        steps there run one by one, so the last is the one clipped to tf)."""
        eng = self.integrator.engine
        while (self.tf - self.t) > self._epsilon and self.count < self.max_steps:
            k = min(self.pfreq - self.count % self.pfreq, self.max_steps - self.count, self.chunk)
            if (self.tf - self.t) <= 2.0 * k * self.dt:
                k = 1
            for cb in self.pre_step_callbacks:
                cb(self)
            eng.begin(self.dt, self.t)
            eng.advance(k, finish=True, capture=k > 1)
            t, dt = eng.clocks()
            self.t = float(t[0] + dt[0])
            self.count += k
            self._epsilon = EPSILON * self.tf * self.count
            for cb in self.post_step_callbacks:
                cb(self)
            self.dt = self._get_timestep()
            if self.count % self.pfreq == 0:
                self.dump_output()

    def solve(self, show_progress=False):
        self._epsilon = EPSILON * self.tf
        self.dump_output()
        if self.initial_acceleration_is_current:
            self.initial_acceleration_is_current = False
        else:
            self.integrator.initial_acceleration(self.t, self.dt)
        self.dt = self._get_timestep()
        if self.fused:
            self._solve_fused()
            self.dump_output()
            return
        while (self.tf - self.t) > self._epsilon and self.count < self.max_steps:
            for cb in self.pre_step_callbacks:
                cb(self)
            logger.debug("Iteration=%d, time=%f, timestep=%f", self.count, self.t, self.dt)
            self.integrator.step(self.t, self.dt)
            for cb in self.post_step_callbacks:
                cb(self)
            self.t += self.dt
            self.count += 1
            self._epsilon = EPSILON * self.tf * self.count
            self.dt = self._get_timestep()
            if self.count % self.pfreq == 0:
                self.dump_output()
        self.dump_output()


def load_output(path):
    """Arrays (by property name, in gid order) and solver data of a dump."""
    with np.load(path, allow_pickle=True) as d:
        if "particles" in d.files:
            particles = d["particles"].item()
            pa = next(iter(particles.values()))
            return dict(pa["arrays"]), dict(d["solver_data"].item())
        skip = {"t", "dt", "count"}
        return {k: d[k] for k in d.files if k not in skip}, {k: d[k].item() for k in skip}
