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

Reverse mode (adjoint) over the step loop: ``AdjointEngine`` runs the steps
keeping the state every ``every`` steps and then the adjoint sweep
(``mhd_adjoint_*``), re-running each segment from its checkpoint.  The
warm-up before the first step is differentiated in forward mode and joined
to the adjoint at the first step's state.

``MagneticEnergy`` wraps a whole run as a ``torch.autograd.Function`` of
(amplitude, alpha_max) for the circularly polarised Alfven wave: the final
magnetic energy sum m |B|^2 / (2 mu0 rho) after ``steps`` steps, gradient by
the checkpointed adjoint.
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


class AdjointEngine:
    """Reverse mode over the step loop (``mhd_adjoint_*``): the forward sweep
    keeps the step state every ``every`` steps, the backward sweep re-runs
    each segment from its checkpoint with a tape and returns dL/dS_0 and
    dL/dalpha_max for L = sum m |B|^2 / (2 mu0 rho) after the last step."""

    def __init__(self, params: _abi.MhdParams, n: int):
        if params.iterate:
            raise ValueError('the adjoint needs density = "single" (params.iterate = 0)')
        self.lib = _abi.load()
        self.params = params
        self.n = n
        self.ctx = ctypes.c_void_p()
        _abi.check(self.lib.mhd_ctx_create(ctypes.byref(params), n, ctypes.byref(self.ctx)), None)
        self.fields = [self.lib.mhd_adjoint_field_name(k).decode() for k in range(self.lib.mhd_adjoint_field_count())]

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

    def _state(self, values: dict):
        S = _abi.state_type()
        s = S()
        for f, t in values.items():
            setattr(s, f, ctypes.c_void_p(t.data_ptr()))
        return s

    def forward(self, values: dict, steps: int, dts, every: int):
        """values: contiguous device tensors of the step-state fields, m and
        itype.  dts: step sizes, None or negative entries for the adaptive
        rule.  Returns (loss, step sizes used, checkpoints)."""
        s = self._state(values)
        d = [-1.0] * steps if dts is None else [float(x) for x in dts]
        if d[0] < 0:
            raise ValueError("the first step size must be given")
        arr = (ctypes.c_double * steps)(*d)
        nseg = (steps + every - 1) // every
        cps = torch.empty((nseg + 1, len(self.fields), self.n), dtype=torch.float64, device=values["x"].device)
        loss = ctypes.c_double()
        _abi.check(self.lib.mhd_adjoint_forward(self.ctx, ctypes.byref(s), self.n, steps, arr, every,
                                                ctypes.c_void_p(cps.data_ptr()), ctypes.byref(loss), self.stream),
                   self.ctx)
        return loss.value, list(arr), cps

    def backward(self, values: dict, steps: int, dts, every: int, checkpoints):
        s = self._state(values)
        arr = (ctypes.c_double * steps)(*[float(x) for x in dts])
        lam = torch.empty((len(self.fields), self.n), dtype=torch.float64, device=values["x"].device)
        dam = ctypes.c_double()
        _abi.check(self.lib.mhd_adjoint_backward(self.ctx, ctypes.byref(s), self.n, steps, arr, every,
                                                 ctypes.c_void_p(checkpoints.data_ptr()),
                                                 ctypes.c_void_p(lam.data_ptr()), ctypes.byref(dam), self.stream),
                   self.ctx)
        return lam, dam.value


def _warm_start(config, amplitude, alpha_max):
    """Warm-up in forward mode: the state at the first step (values) and its
    derivatives with respect to (amplitude, alpha_max)."""
    from .engine import params_from_dict

    ic, seed, prm = alfven_case(config, amplitude, alpha_max)
    params = params_from_dict(prm)
    te = TangentEngine(params, TangentState(ic, seed), alpha_max_seed=[0.0, 1.0])
    te.warmup()
    dt0 = te.initial_dt()
    return params, te, dt0


def magnetic_energy_adjoint(config, amplitude: float, alpha_max: float, steps: int, every: int = 16, dts=None):
    """The same loss and gradient as ``magnetic_energy_and_gradient``, by the
    checkpointed adjoint over the steps (the warm-up in forward mode)."""
    params, te, dt0 = _warm_start(config, amplitude, alpha_max)
    ae = AdjointEngine(params, te.ts.n)
    try:
        values = {f: te.ts[f][:, 0].contiguous() for f in ae.fields}
        values["m"] = te.ts["m"][:, 0].contiguous()
        values["itype"] = te.ts["itype"]
        loss, used, cps = ae.forward(values, steps, [dt0] + [-1.0] * (steps - 1) if dts is None else dts, every)
        lam, dam = ae.backward(values, steps, used, every, cps)
        tan = torch.stack([te.ts[f][:, 1:] for f in ae.fields])  # fields x n x DIRS
        grad = torch.einsum("fn,fnd->d", lam, tan).cpu().numpy()
        grad[1] += dam
        return loss, grad, used
    finally:
        ae.close()
        te.close()


class MagneticEnergy(torch.autograd.Function):
    """Final magnetic energy of the 2-D Alfven wave as a differentiable
    function of (amplitude, alpha_max): ``MagneticEnergy.apply(a, am, config,
    steps, every)``.  Forward: the warm-up in forward mode, then the steps
    with the state kept every ``every`` steps.  Backward: the adjoint sweep,
    re-running each segment from its checkpoint, contracted with the
    warm-up's derivatives."""

    @staticmethod
    def forward(ctx, amplitude, alpha_max, config, steps, every=16):
        params, te, dt0 = _warm_start(config, float(amplitude), float(alpha_max))
        ae = AdjointEngine(params, te.ts.n)
        values = {f: te.ts[f][:, 0].contiguous() for f in ae.fields}
        values["m"] = te.ts["m"][:, 0].contiguous()
        values["itype"] = te.ts["itype"]
        loss, used, cps = ae.forward(values, int(steps), [dt0] + [-1.0] * (int(steps) - 1), int(every))
        ctx.engines = (te, ae)
        ctx.values, ctx.used, ctx.cps, ctx.steps, ctx.every = values, used, cps, int(steps), int(every)
        return torch.as_tensor(loss, dtype=torch.float64)

    @staticmethod
    def backward(ctx, g):
        te, ae = ctx.engines
        try:
            lam, dam = ae.backward(ctx.values, ctx.steps, ctx.used, ctx.every, ctx.cps)
            tan = torch.stack([te.ts[f][:, 1:] for f in ae.fields])
            grad = torch.einsum("fn,fnd->d", lam, tan).cpu()
            grad[1] += dam
        finally:
            ae.close()
            te.close()
        return g * grad[0], g * grad[1], None, None, None
