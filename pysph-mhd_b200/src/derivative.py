"""Derivative form: gradients of a simulation output through the SPMHD step.

Forward mode (tangent-linear): the state is held as dual numbers -- every
particle property is an ``(n, 1 + DIRS)`` FP64 CUDA tensor whose column 0 is
the value and columns 1.. its derivatives with respect to up to ``DIRS``
parameters -- and the library's tangent kernels (``mhd_tangent_*``) run the
reference's literal PEC step (``MHDStep`` with the ten groups of
``MHDScheme.get_equations``, src/scheme.py:66-81) on it.  A parameter enters
through the initial state (a seed direction per property) or through
``alpha_max`` (the Cullen-Dehnen clip, src/equations.py:428).  The warm-up
(src/application.py:110-132) is differentiated too; the adaptive timestep
(src/solver.py:40,61) is evaluated on the values and frozen.  The density
step must be the single pass (``density = "single"``), which keeps the map
smooth.

``MagneticEnergy`` wraps a whole run as a ``torch.autograd.Function`` of
(amplitude, alpha_max) for the circularly polarised Alfven wave: the final
magnetic energy sum m |B|^2 / (2 mu0 rho) after ``steps`` steps.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _abi
from .particles import property_names

DIRS = 2


class TangentState:
    """Dual-number particle arrays on the device (no neighbour sort: the
    derivative form keeps the particle order)."""

    def __init__(self, arrays: dict, seeds: dict | None = None, device="cuda"):
        _abi.load()
        n = len(np.asarray(arrays["x"]))
        self.n = n
        self.device = torch.device(device)
        self._t: dict[str, torch.Tensor] = {}
        for k in property_names():
            if k == "itype":
                v = arrays.get("itype")
                a = np.ones(n, dtype=np.int32) if v is None else np.asarray(v, dtype=np.int32)
                self._t[k] = torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
                continue
            t = torch.zeros((n, 1 + DIRS), dtype=torch.float64)
            v = arrays.get(k)
            if k == "gid" and v is None:
                v = np.arange(n, dtype=np.float64)
            if v is not None:
                t[:, 0] = torch.from_numpy(np.asarray(v, dtype=np.float64))
            for d, seed in enumerate((seeds or {}).get(k, ())):
                if seed is not None:
                    t[:, 1 + d] = torch.from_numpy(np.asarray(seed, dtype=np.float64))
            self._t[k] = t.to(self.device)

    def __getitem__(self, k):
        return self._t[k]

    def value(self, k):
        return self._t[k][:, 0]

    def state(self):
        S = _abi.state_type()
        s = S()
        for f in _abi.STATE_FIELDS:
            t = self._t.get(f)
            if t is not None:
                setattr(s, f, ctypes.c_void_p(t.data_ptr()))
        return s


class TangentEngine:
    """The derivative form of ``Engine`` (src/engine.py) on a TangentState."""

    def __init__(self, params: _abi.MhdParams, ts: TangentState, alpha_max_seed=None):
        if not torch.cuda.is_available():
            raise RuntimeError("the derivative form needs a CUDA device (no CPU fallback)")
        if params.iterate:
            raise ValueError('the derivative form needs density = "single" (params.iterate = 0)')
        self.lib = _abi.load()
        self.params = params
        self.ts = ts
        self.ctx = ctypes.c_void_p()
        _abi.check(self.lib.mhd_ctx_create(ctypes.byref(params), ts.n, ctypes.byref(self.ctx)), None)
        amax = [params.alpha_max] + list(alpha_max_seed if alpha_max_seed is not None else [0.0] * DIRS)
        self._amax = (ctypes.c_double * (1 + DIRS))(*amax)
        self.dts: list[float] = []

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

    def rhs(self):
        s = self.ts.state()
        self._check(self.lib.mhd_tangent_rhs(self.ctx, ctypes.byref(s), self.ts.n, self._amax, self.stream))

    def step(self, dt: float):
        s = self.ts.state()
        self._check(self.lib.mhd_tangent_step(self.ctx, ctypes.byref(s), self.ts.n, float(dt), self._amax,
                                              self.stream))
        self.dts.append(float(dt))

    def sync_initial_mhd_state(self):
        s = self.ts.state()
        self._check(self.lib.mhd_tangent_sync(self.ctx, ctypes.byref(s), self.ts.n, self.stream))

    def warmup(self):
        """src/application.py:110-132: three RHS with the B restore."""
        ts = self.ts
        b0 = {k: ts[k].clone() for k in ("Bx", "By", "Bz")}
        ts["h0"].copy_(ts["h"])
        self.sync_initial_mhd_state()
        self.rhs()
        for k in ("Bx", "By", "Bz"):
            ts[k].copy_(b0[k])
        ts["h0"].copy_(ts["h"])
        self.sync_initial_mhd_state()
        self.rhs()
        self.rhs()

    def initial_dt(self) -> float:
        """src/application.py:134-147 on the values."""
        ts = self.ts
        tf = self.params.timestep_factor
        h, cfl = ts.value("h"), ts.value("dt_cfl")
        force = torch.sqrt(ts.value("au") ** 2 + ts.value("av") ** 2 + ts.value("aw") ** 2)
        cands = [float(torch.min(tf * 0.3 * h / cfl))]
        mask = force > 0.0
        if bool(torch.any(mask)):
            cands.append(float(torch.min(tf * 0.25 * torch.sqrt(h[mask] / force[mask]))))
        return min(cands)

    def next_dt(self, t: float) -> float:
        """min dt_adapt on the values, clipped so t + dt <= tf."""
        dt = float(torch.min(self.ts.value("dt_adapt")))
        return self.params.tf - t if t + dt > self.params.tf else dt

    def run(self, steps: int, dts=None):
        """`steps` PEC steps after warmup(): with ``dts`` the given step sizes
        (frozen), else the adaptive rule evaluated on the values."""
        t = 0.0
        dt = self.initial_dt() if dts is None else dts[0]
        for k in range(steps):
            self.step(dt)
            t += dt
            if k + 1 < steps:
                dt = self.next_dt(t) if dts is None else dts[k + 1]
        return t

    def magnetic_energy(self):
        """(value, derivatives) of sum m |B|^2 / (2 mu0 rho)."""
        out = (ctypes.c_double * (1 + DIRS))()
        s = self.ts.state()
        self._check(self.lib.mhd_tangent_magnetic_energy(self.ctx, ctypes.byref(s), self.ts.n, out, self.stream))
        return out[0], np.array(out[1:])


# ------------------------------------------------------ Alfven wave loss
def alfven_case(config, amplitude: float, alpha_max: float):
    """Initial state of ``AlfvenWave2D`` with ``config`` (single density
    pass), its derivative with respect to the amplitude (the perturbation is
    linear in it), and the kernel parameters with ``alpha_max``."""
    from dataclasses import replace

    from .cases.alfven import AlfvenWave2D

    cfg = replace(config, numerics=replace(config.numerics, density="single"),
                  physics=replace(config.physics, alpha_max=alpha_max))

    class _Case(AlfvenWave2D):
        pass

    _Case.amplitude = amplitude
    app = _Case(cfg)
    ic = app.create_mhd_particles()
    phase = 2.0 * np.pi * ic["x"]
    seed = {"v": [np.sin(phase), None], "w": [np.cos(phase), None], "By": [np.sin(phase), None],
            "Bz": [np.cos(phase), None]}
    prm = app.scheme.kernel_params(app.create_domain(), app.tf)
    return ic, seed, prm


def magnetic_energy_and_gradient(config, amplitude: float, alpha_max: float, steps: int, dts=None):
    """Final magnetic energy after `steps` steps and its gradient with respect
    to (amplitude, alpha_max), in one forward-mode sweep.  Returns
    (value, gradient[2], step sizes used)."""
    from .engine import params_from_dict

    ic, seed, prm = alfven_case(config, amplitude, alpha_max)
    params = params_from_dict(prm)
    eng = TangentEngine(params, TangentState(ic, seed), alpha_max_seed=[0.0, 1.0])
    try:
        eng.warmup()
        eng.run(steps, dts)
        value, grad = eng.magnetic_energy()
        return value, grad, list(eng.dts)
    finally:
        eng.close()


class MagneticEnergy(torch.autograd.Function):
    """Final magnetic energy of the 2-D Alfven wave as a differentiable
    function of (amplitude, alpha_max): ``MagneticEnergy.apply(a, am, config,
    steps)``.  The forward pass runs the dual-number simulation once and
    keeps the gradient; backward scales it by the incoming gradient."""

    @staticmethod
    def forward(ctx, amplitude, alpha_max, config, steps):
        value, grad, _ = magnetic_energy_and_gradient(config, float(amplitude), float(alpha_max), int(steps))
        ctx.save_for_backward(torch.as_tensor(grad, dtype=torch.float64))
        return torch.as_tensor(value, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return g * grad[0], g * grad[1], None, None
