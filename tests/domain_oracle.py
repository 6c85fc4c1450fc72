"""The C oracle as the stepper of src.domain.DomainSolver (test helper).

The decomposition logic -- slabs, migration, the double-width halo, the
frozen outer ghosts, the collectives -- is host code; with this stepper it
runs on CPU ranks (gloo) and must reproduce a one-process oracle run bit for
bit: the local arrays are ordered by gid before each right-hand side, so the
oracle visits every particle's neighbours in the same (ascending gid) order
as on the whole case, and any ghost missing from a neighbourhood changes
the sums.
"""

from __future__ import annotations

import numpy as np
import torch

import oracle


class OracleStepper:
    def __init__(self, prm: dict, nthreads: int = 2):
        self.o = oracle.Oracle(prm, exact_order=True, nthreads=nthreads)

    @staticmethod
    def _state(a: dict) -> oracle.State:
        return oracle.State({k: v.cpu().numpy() for k, v in a.items()})

    @staticmethod
    def _write_back(s: oracle.State, a: dict):
        for k in s.names:
            if k in a:
                a[k] = torch.from_numpy(s[k].copy())

    def predict(self, a: dict, dt: float):
        if a["x"].numel() == 0:
            return
        s = self._state(a)
        self.o.predict(s, dt)
        self._write_back(s, a)

    def rhs(self, a: dict) -> dict:
        if a["x"].numel() == 0:
            return a
        order = torch.argsort(a["gid"])
        b = {k: v[order].contiguous() for k, v in a.items()}
        s = self._state(b)
        self.o.rhs(s)
        self._write_back(s, b)
        return b

    def correct(self, a: dict, dt: float):
        if a["x"].numel() == 0:
            return
        s = self._state(a)
        self.o.correct(s, dt)
        self._write_back(s, a)


def single_run(ic: dict, prm: dict, steps: int):
    """The same case in one process: warm-up, initial dt, `steps` PEC steps
    with the adaptive step; returns the state by gid."""
    s = oracle.State(ic)
    o = oracle.Oracle(prm, exact_order=True, nthreads=2)
    o.warmup(s)
    dt = o.initial_dt(s)
    for _ in range(steps):
        o.step(s, dt)
        dt = o.min_dt(s)
    out = {k: s[k].copy() for k in s.names}
    out["gid"] = s["gid"].copy()
    return out, dt


def as_tensors(ic: dict) -> dict:
    return {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in ic.items()}
