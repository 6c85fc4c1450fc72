"""The batched form: many independent cases advanced together on one GPU.

Instances are particle sets of uneven size that share the scheme parameters
and the domain.  The reference runs one case per ``MHDApplication``
(src/application.py) and has no batch driver; here the instances are stored
one after another in one ``ParticleArray`` and each keeps its own neighbour
grid, clock and adaptive timestep (src/solver.py:40,61), so an instance's
result is the result of running it alone.  Every kernel launch covers all
instances; ``advance`` runs a whole multi-step run as one captured CUDA graph
(``mhd_advance``) and replays it step by step from a snapshot in the rare
case the captured run meets a neighbour-list rebuild.  ``tune`` is the
autotuner: it times the cell size (grid stencil) and the force pass's launch
shape on the instances themselves and keeps the fastest.
"""

from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _abi
from .engine import Engine
from .particle_array import ParticleArray
from .particles import property_names

STENCILS = (1, 2, 3)
FORCE_SHAPES = (0, 1, 2, 3)
_TUNE_CACHE: dict[str, dict] = {}


def concatenate(instances: list[dict]):
    """One array dict from instance dicts; gid becomes offset + local gid."""
    counts = [len(np.asarray(a["x"])) for a in instances]
    if min(counts) < 1:
        raise ValueError("every instance needs at least one particle")
    start = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    out = {}
    for k in property_names():
        parts = [a.get(k) for a in instances]
        if all(p is None for p in parts):
            continue
        if k == "gid":
            parts = [start[i] + (np.arange(c, dtype=np.float64) if p is None else np.asarray(p, dtype=np.float64))
                     for i, (p, c) in enumerate(zip(parts, counts))]
        elif k == "itype":
            parts = [np.ones(c, dtype=np.int32) if p is None else np.asarray(p, dtype=np.int32)
                     for p, c in zip(parts, counts)]
        else:
            parts = [np.zeros(c) if p is None else np.asarray(p, dtype=np.float64) for p, c in zip(parts, counts)]
        out[k] = np.concatenate(parts)
    return out, start


class BatchEngine(Engine):
    def __init__(self, params: _abi.MhdParams, instances: list[dict], cell_headroom: float = 1.25):
        arrays, start = concatenate(instances)
        self.start = start
        self.n_inst = len(instances)
        self.cell_headroom = float(cell_headroom)
        super().__init__(params, ParticleArray("batch", arrays))
        self.replays = 0
        self.tuned = None
        self.set_instances()

    @classmethod
    def single(cls, params: _abi.MhdParams, pa: ParticleArray, cell_headroom: float = 1.25):
        """One simulation on the device planner and captured runs: the fused
        production loop of ``MHDSolver`` (``execution.fused``)."""
        self = cls.__new__(cls)
        self.start = np.array([0, pa.n], dtype=np.int64)
        self.n_inst = 1
        self.cell_headroom = float(cell_headroom)
        Engine.__init__(self, params, pa)
        self.replays = 0
        self.tuned = None
        self.set_instances()
        return self

    # ------------------------------------------------------------ set-up
    def set_instances(self):
        """(Re)declare the instances; plans capacities, resets the clocks."""
        s = self.pa.state()
        start = (ctypes.c_int64 * (self.n_inst + 1))(*[int(v) for v in self.start])
        self._check(self.lib.mhd_ctx_set_instances(self.ctx, ctypes.byref(s), self.n_inst, start,
                                                   self.cell_headroom, self.stream))

    def instance(self, k: int) -> slice:
        return slice(int(self.start[k]), int(self.start[k + 1]))

    def pull_instance(self, k: int, *names):
        """numpy copies of instance k's properties in its own gid order."""
        sl = self.instance(k)
        names = names or tuple(self.pa.properties)
        gid = self.pa.gid[sl].cpu().numpy()
        perm = np.argsort(gid, kind="stable")
        out = {}
        for name in names:
            v = self.pa[name][sl].cpu().numpy()[perm]
            out[name] = v - self.start[k] if name == "gid" else v
        return out

    # ------------------------------------------------------------ clocks
    def clocks(self):
        t = (ctypes.c_double * self.n_inst)()
        dt = (ctypes.c_double * self.n_inst)()
        self._check(self.lib.mhd_clock_get_all(self.ctx, t, dt, self.stream))
        return np.array(t[:]), np.array(dt[:])

    def set_clocks(self, t, dt):
        tv = (ctypes.c_double * self.n_inst)(*np.broadcast_to(np.asarray(t, dtype=float), (self.n_inst,)))
        dv = (ctypes.c_double * self.n_inst)(*np.broadcast_to(np.asarray(dt, dtype=float), (self.n_inst,)))
        self._check(self.lib.mhd_clock_set_all(self.ctx, tv, dv, self.stream))

    # ------------------------------------------------- warm-up and start
    def initial_dt(self) -> np.ndarray:
        """src/application.py:134-147 for every instance."""
        pa = self.pa
        tf = self.params.timestep_factor
        out = np.empty(self.n_inst)
        for k in range(self.n_inst):
            sl = self.instance(k)
            h, dt_cfl = pa.h[sl], pa.dt_cfl[sl]
            force = torch.sqrt(pa.au[sl] ** 2 + pa.av[sl] ** 2 + pa.aw[sl] ** 2)
            if not bool(torch.all(dt_cfl > 0.0)):
                raise RuntimeError(f"instance {k}: dt_cfl must be positive after the warm-up")
            cands = [float(torch.min(tf * 0.3 * h / dt_cfl))]
            mask = force > 0.0
            if bool(torch.any(mask)):
                cands.append(float(torch.min(tf * 0.25 * torch.sqrt(h[mask] / force[mask]))))
            out[k] = min(cands)
            if not out[k] > 0.0:
                raise RuntimeError(f"instance {k}: initial dt must be positive")
        return out

    def begin(self, dt0, t0=0.0):
        """Initialize + stage1 of every instance's first step with its dt0."""
        self.set_clocks(t0, dt0)
        s = self.pa.state()
        self._check(self.lib.mhd_corrector_predictor(self.ctx, ctypes.byref(s), self.pa.n, 2, -1.0, -1.0,
                                                     self.stream))

    # ------------------------------------------------------------- runs
    def snapshot(self):
        return {k: v.clone() for k, v in self.pa.properties.items()}, self.clocks()

    def restore(self, snap):
        tensors, (t, dt) = snap
        for k, v in tensors.items():
            self.pa[k].copy_(v)
        self.set_clocks(t, dt)

    def advance(self, n_steps: int, finish: bool = True, capture: bool = True, snapshot=None):
        """n_steps fused steps of every instance (the last applies only the
        corrector when ``finish``).  Captured: one CUDA graph launch, replayed
        uncaptured from a snapshot if the run met a list rebuild."""
        if n_steps <= 0:
            return
        a, b = self.pa.state(), self.pa.state(spare=True)
        if capture:
            snap = snapshot if snapshot is not None else self.snapshot()
            rc = self.lib.mhd_advance(self.ctx, ctypes.byref(a), ctypes.byref(b), self.pa.n, n_steps, int(finish), 1,
                                      self.stream)
            if rc == _abi.MHD_ERR_RELIST:
                self.replays += 1
                self.restore(snap)
                rc = self.lib.mhd_advance(self.ctx, ctypes.byref(a), ctypes.byref(b), self.pa.n, n_steps,
                                          int(finish), 0, self.stream)
        else:
            rc = self.lib.mhd_advance(self.ctx, ctypes.byref(a), ctypes.byref(b), self.pa.n, n_steps, int(finish), 0,
                                      self.stream)
        self._check(rc)
        if n_steps % 2:
            self.pa.swap()

    # ---------------------------------------------------------- autotune
    def _signature(self):
        p = self.params
        return json.dumps(dict(dim=p.dim, kernel=p.kernel, precision=p.precision, n_inst=self.n_inst,
                               n=int(self.pa.n), hfact=round(p.hfact, 6),
                               device=torch.cuda.get_device_name()), sort_keys=True)

    def apply(self, stencil: int, force_shape: int):
        self._check(self.lib.mhd_ctx_tune(self.ctx, int(stencil), int(force_shape)))
        self.set_instances()

    def tune(self, steps: int = 4, stencils=STENCILS, shapes=FORCE_SHAPES, cache_path=None):
        """Time `steps` captured steps for every (stencil, force shape) on the
        current state (restored after each trial) and apply the fastest.
        Results are cached per workload signature in memory and, when
        ``cache_path`` (or $MHD_TUNE_CACHE) names a JSON file, on disk."""
        cache_path = cache_path or os.environ.get("MHD_TUNE_CACHE")
        key = self._signature()
        disk = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                disk = json.load(f)
        hit = _TUNE_CACHE.get(key) or disk.get(key)
        snap = self.snapshot()
        if hit is None:
            trials = []
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            for st in stencils:
                for sh in shapes:
                    self.apply(st, sh)
                    self.restore(snap)
                    self.advance(steps, finish=False, snapshot=snap)  # capture + first launch
                    self.restore(snap)
                    ev0.record()
                    self.advance(steps, finish=False, snapshot=snap)
                    ev1.record()
                    ev1.synchronize()
                    trials.append(dict(stencil=st, force_shape=sh, ms_per_step=ev0.elapsed_time(ev1) / steps))
                    self.restore(snap)
            best = min(trials, key=lambda r: r["ms_per_step"])
            hit = dict(best, trials=trials)
            _TUNE_CACHE[key] = hit
            if cache_path:
                disk[key] = hit
                with open(cache_path, "w") as f:
                    json.dump(disk, f, indent=1)
        self.apply(hit["stencil"], hit["force_shape"])
        self.restore(snap)
        self.tuned = hit
        return hit
