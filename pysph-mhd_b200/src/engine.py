"""Drives the sm_100a kernels through the C ABI for one particle array.

``Engine`` is what PySPH's generated acceleration evaluator and integrator
were for the reference: ``rhs()`` evaluates the ten equation groups of
``MHDScheme.get_equations`` (src/scheme.py:66-81), ``step(dt)`` runs one
``PECIntegrator.one_timestep`` with ``MHDStep`` (src/integrator.py), and
``timestep(t)`` applies the adaptive rule (min dt_adapt, clipped to tf).
``advance(k)`` is the fused production loop: the corrector of step n and the
predictor of step n+1 share one kernel, dt stays on the device.
"""

from __future__ import annotations

import ctypes

import torch

from . import _abi
from .particle_array import ParticleArray


def params_from_dict(p: dict, precision=None) -> _abi.MhdParams:
    """MhdParams from a flat dict (keys as in the fixture ``params`` record)."""
    return _abi.make_params(
        dim=p["dim"], kernel=p["kernel"], hfact=p["hfact"], gamma=p["gamma"], mu0=p["mu0"], av=p["av"], ac=p["ac"],
        ar=p["ar"], clean_speed=p["clean_speed"], clean_damp=p["clean_damp"], timestep_factor=p["timestep_factor"],
        tf=p.get("tf", 1e30), lo=p["lo"], hi=p["hi"], periodic=p["periodic"],
        iterate=p.get("density", "iterate") == "iterate", alpha_min=p.get("alpha_min", 0.0),
        alpha_max=p.get("alpha_max", 1.0), precision=precision or p.get("precision", "fp64"))


class Engine:
    def __init__(self, params: _abi.MhdParams, pa: ParticleArray):
        if not torch.cuda.is_available():
            raise RuntimeError("the SPMHD B200 engine needs a CUDA device (no CPU fallback)")
        self.lib = _abi.load()
        self.pa = pa
        self.params = params
        self.ctx = ctypes.c_void_p()
        _abi.check(self.lib.mhd_ctx_create(ctypes.byref(params), pa.n, ctypes.byref(self.ctx)), None)
        self.density_passes: list[int] = []
        self.grid_rebuilds = 0
        self.last_stats = _abi.MhdRhsStats()

    def close(self):
        if self.ctx:
            self.lib.mhd_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def _check(self, rc):
        _abi.check(rc, self.ctx)

    def launches(self) -> int:
        return int(self.lib.mhd_launch_count(self.ctx))

    def set_params(self, params: _abi.MhdParams):
        self.params = params
        self._check(self.lib.mhd_ctx_set_params(self.ctx, ctypes.byref(params)))

    # ------------------------------------------------------------ groups
    def _record(self, st):
        self.last_stats = st
        self.density_passes.append(int(st.density_passes))
        self.grid_rebuilds += int(st.grid_rebuilds)

    def rhs(self):
        """One right-hand side (Integrator.compute_accelerations)."""
        st = _abi.MhdRhsStats()
        src, dst = self.pa.state(), self.pa.state(spare=True)
        self._check(self.lib.mhd_rhs(self.ctx, ctypes.byref(src), ctypes.byref(dst), self.pa.n, ctypes.byref(st),
                                     self.stream))
        self.pa.swap()
        self._record(st)
        return st

    def step(self, dt: float):
        """PECIntegrator.one_timestep with MHDStep, every property written."""
        st = _abi.MhdRhsStats()
        src, dst = self.pa.state(), self.pa.state(spare=True)
        self._check(self.lib.mhd_step(self.ctx, ctypes.byref(src), ctypes.byref(dst), self.pa.n, float(dt),
                                      ctypes.byref(st), self.stream))
        self.pa.swap()
        self._record(st)
        return st

    def timestep(self, t: float) -> float:
        """min(dt_adapt) clipped so t + dt <= tf (synchronising)."""
        dt = ctypes.c_double()
        s = self.pa.state()
        self._check(self.lib.mhd_timestep(self.ctx, ctypes.byref(s), self.pa.n, float(t), ctypes.byref(dt),
                                          self.stream))
        return dt.value

    def cells_build(self):
        """Neighbour sort + lists (PySPH's NNPS update) without evaluating."""
        src, dst = self.pa.state(), self.pa.state(spare=True)
        self._check(self.lib.mhd_cells_build(self.ctx, ctypes.byref(src), ctypes.byref(dst), self.pa.n, self.stream))
        self.pa.swap()

    def neighbour_counts(self):
        """Per-particle neighbour counts under the exact rule (current order)."""
        out = torch.empty(self.pa.n, dtype=torch.int32, device=self.pa.device)
        s = self.pa.state()
        self._check(self.lib.mhd_neighbour_counts(self.ctx, ctypes.byref(s), self.pa.n, ctypes.c_void_p(out.data_ptr()),
                                                  self.stream))
        return out

    # --------------------------------------------------------- fused loop
    def begin(self, dt0: float, t0: float = 0.0):
        """Initialize + stage1 of the first step (after the warm-up)."""
        s = self.pa.state()
        self._check(self.lib.mhd_corrector_predictor(self.ctx, ctypes.byref(s), self.pa.n, 2, 0.0, float(dt0),
                                                     self.stream))
        self._check(self.lib.mhd_clock_set(self.ctx, float(t0), float(dt0), self.stream))

    def advance(self, n_steps: int, finish: bool = True):
        """n_steps fused steps; with ``finish`` the last applies only stage2."""
        for k in range(n_steps):
            self.rhs()
            s = self.pa.state()
            self._check(self.lib.mhd_timestep(self.ctx, ctypes.byref(s), self.pa.n, -1.0, None, self.stream))
            mode = 1 if (finish and k == n_steps - 1) else 3
            self._check(self.lib.mhd_corrector_predictor(self.ctx, ctypes.byref(s), self.pa.n, mode, -1.0, -1.0,
                                                         self.stream))

    def clock(self):
        t, dt = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mhd_clock_get(self.ctx, ctypes.byref(t), ctypes.byref(dt), self.stream))
        return t.value, dt.value

    # ------------------------------------------------ reference warm-up
    def sync_initial_mhd_state(self):
        """src/application.py:99-108 on the device."""
        pa = self.pa
        pa.Bevolx.copy_(pa.Bx / pa.rho)
        pa.Bevoly.copy_(pa.By / pa.rho)
        pa.Bevolz.copy_(pa.Bz / pa.rho)
        pa.psi.zero_()
        for pred, cur in (("Bevolxpred", "Bevolx"), ("Bevolypred", "Bevoly"), ("Bevolzpred", "Bevolz"),
                          ("psipred", "psi"), ("upred", "u"), ("vpred", "v"), ("wpred", "w"), ("epred", "e")):
            pa[pred].copy_(pa[cur])

    def warmup(self, refresh=None):
        """src/application.py:110-132: three RHS with the B restore and re-sync."""
        pa = self.pa
        gid0 = pa.gid.clone()
        b0 = {k: pa[k].clone() for k in ("Bx", "By", "Bz")}
        pa.h0.copy_(pa.h)
        self.sync_initial_mhd_state()
        self.rhs()
        if not bool(torch.all(pa.converged == 1)):
            raise RuntimeError("density iteration did not converge in the warm-up RHS")
        # B was overwritten by MagneticStateReconstruction; restore it in the
        # current (sorted) particle order.
        order = torch.argsort(gid0)
        idx = order[torch.searchsorted(gid0[order], pa.gid)]
        for k in ("Bx", "By", "Bz"):
            pa[k].copy_(b0[k][idx])
        if refresh is not None:
            refresh(pa)
        pa.h0.copy_(pa.h)
        self.sync_initial_mhd_state()
        for _ in range(2):
            self.rhs()
        if not bool(torch.all(pa.converged == 1)):
            raise RuntimeError("density iteration did not converge in the warm-up RHS")

    def initial_dt(self) -> float:
        """src/application.py:134-147."""
        pa = self.pa
        tf = self.params.timestep_factor
        force = torch.sqrt(pa.au * pa.au + pa.av * pa.av + pa.aw * pa.aw)
        if not bool(torch.all(pa.dt_cfl > 0.0)):
            raise RuntimeError("dt_cfl must be positive after the warm-up")
        cands = [float(torch.min(tf * 0.3 * pa.h / pa.dt_cfl))]
        mask = force > 0.0
        if bool(torch.any(mask)):
            cands.append(float(torch.min(tf * 0.25 * torch.sqrt(pa.h[mask] / force[mask]))))
        dt = min(cands)
        if not dt > 0.0:
            raise RuntimeError("initial dt must be positive")
        return dt
