"""Particle arrays held as CUDA tensors, one FP64 tensor per property name.

Stands in for PySPH's ``ParticleArray`` + ``.gpu`` mirror for the hot path:
``pa.x`` is a ``torch.Tensor`` on the GPU, ``pa.pull(...)`` returns numpy
copies, ``pa.push(name, array)`` uploads.  The neighbour sort permutes the
particles (like PySPH's ``reorder_particles``), so every field the sort
carries has a second buffer; ``gid`` tracks particle identity.

Diagnostic outputs -- the Cullen-Dehnen moments ``cd_*``, ``xilimiter``,
``divvdt``, the strain rates ``dvdx_*`` and the density pass's ``arho``,
``grhox/y/z`` and ``dwdh`` -- are read by no equation.  With
``diagnostics=True`` the array hands them to the kernels, which then write
every one of them as the reference does (the density passes then also
re-sum converged particles, so ``rho_sum`` is the last pass's sum); by
default they are left out of the kernel state and not written.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _abi
from .particles import property_names


DIAGNOSTIC_FIELDS = frozenset(
    ("xilimiter", "divvdt", "arho", "grhox", "grhoy", "grhoz", "dwdh")
    + tuple(f"cd_{k}" for k in "rxx rxy rxz ryy ryz rzz".split())
    + tuple(f"cd_{q}{a}{b}" for q in "va" for a in "xyz" for b in "xyz")
    + tuple(f"dvdx_{a}{b}" for a in "xyz" for b in "xyz"))


class ParticleArray:
    def __init__(self, name: str, arrays: dict, device="cuda", diagnostics: bool = False):
        _abi.load()
        self.name = name
        self.diagnostics = bool(diagnostics)
        n = len(np.asarray(arrays["x"]))
        self.n = n
        self.device = torch.device(device)
        self._t: dict[str, torch.Tensor] = {}
        names = property_names()
        for k in names:
            if k == "itype":
                v = arrays.get("itype")
                a = np.ones(n, dtype=np.int32) if v is None else np.asarray(v, dtype=np.int32)
                self._t[k] = torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
            else:
                v = arrays.get(k)
                if k == "gid" and v is None:
                    v = np.arange(n, dtype=np.float64)
                a = np.zeros(n) if v is None else np.asarray(v, dtype=np.float64)
                if a.shape != (n,):
                    raise ValueError(f"property {k} has shape {a.shape}, expected ({n},)")
                self._t[k] = torch.from_numpy(np.ascontiguousarray(a)).to(self.device)
        self._spare = {k: torch.empty_like(self._t[k]) for k in _abi.SORTED_FIELDS}

    # --- attribute access like a PySPH ParticleArray ---
    def __getattr__(self, k):
        t = self.__dict__.get("_t")
        if t is not None and k in t:
            return t[k]
        raise AttributeError(k)

    def __getitem__(self, k):
        return self._t[k]

    def get_number_of_particles(self):
        return self.n

    @property
    def properties(self):
        return self._t

    def pull(self, *names, order="current"):
        """numpy copies; ``order="gid"`` returns them indexed by particle id."""
        names = names or tuple(self._t)
        out = {k: self._t[k].cpu().numpy() for k in names}
        if order == "gid":
            perm = np.argsort(self._t["gid"].cpu().numpy(), kind="stable")
            out = {k: v[perm] for k, v in out.items()}
        return out

    def push(self, name, values):
        self._t[name].copy_(torch.as_tensor(np.asarray(values), dtype=self._t[name].dtype))

    # --- C ABI views ---
    def state(self, spare=False):
        """An ``MhdState`` with this array's device pointers; with ``spare``
        the sorted fields point at the second buffers (a sort destination)."""
        S = _abi.state_type()
        s = S()
        for f in _abi.STATE_FIELDS:
            if not self.diagnostics and f in DIAGNOSTIC_FIELDS:
                continue
            src = self._spare if (spare and f in self._spare) else self._t
            t = src.get(f)
            if t is not None:
                setattr(s, f, ctypes.c_void_p(t.data_ptr()))
        return s

    def swap(self):
        """Make the sort destination current (after ``mhd_cells_build``)."""
        for k in self._spare:
            self._t[k], self._spare[k] = self._spare[k], self._t[k]

    def permutation_to_gid(self):
        return torch.argsort(self._t["gid"])
