"""MHDStep and the predictor-evaluate-corrector integrator on the B200 path.

``MHDStep`` (src/integrator.py:6-82) carries gamma; its three stages run as
``k_stage_initialize``/``k_stage1``/``k_stage2`` in ``csrc/mhd_integrate.cu``.
``PECIntegrator`` keeps PySPH's integrator surface (``initial_acceleration``,
``step``, ``compute_time_step``) over an ``src.engine.Engine``.
"""

from __future__ import annotations


class MHDStep:
    def __init__(self, gamma):
        assert gamma > 1.0
        self.gamma1 = gamma - 1.0


class PECIntegrator:
    def __init__(self, **steppers):
        self.steppers = steppers
        self.engine = None

    def set_engine(self, engine):
        self.engine = engine

    def _eng(self):
        if self.engine is None:
            raise RuntimeError("PECIntegrator has no engine: call MHDApplication.setup() first")
        return self.engine

    def initial_acceleration(self, t, dt):
        self._eng().rhs()

    def step(self, t, dt):
        # initialize, stage1, wrap, RHS, stage2, wrap (PECIntegrator.one_timestep)
        self._eng().step(dt)

    def compute_time_step(self, dt, cfl=None, t=0.0):
        return self._eng().timestep(t)
