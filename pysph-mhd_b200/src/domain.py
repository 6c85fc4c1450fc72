"""One simulation over several ranks: slab domain decomposition with halos.

The reference runs one case in one process; PySPH's MPI hooks in its solver
(src/solver.py:22,27: ``in_parallel``, ``barrier``) are inert there.  Here a
case can be split over ranks (one GPU each) along one axis of the box:

* Rank r owns the particles whose coordinate along ``axis`` lies in
  ``[cuts[r], cuts[r+1])``.  The cuts balance particle counts: they are
  quantiles of a global histogram (an all-reduce) taken when the
  decomposition is made.
* Before every right-hand side each rank receives, from every other rank,
  that rank's particles within ``2 W`` of its own slab (minimum image along
  periodic axes): its *ghosts*.  ``W = R (1 + margin) h_max safety`` covers
  every pair the scheme can form (``r < R max(h_i, h_j)``).  Ghosts within
  ``W`` of the slab (*inner*) then see their whole neighbourhood locally,
  so the density iteration (src/equations.py:14-94, src/scheme.py:71) gives
  them the h their owner gives them.  Ghosts beyond ``W`` (*outer*) are
  frozen for it (``converged = 1``): with compact kernels an owned or inner
  particle's density sums take only their positions and masses.  The force
  groups of every owned particle then read only owned and inner-ghost
  neighbours.  Doubling the halo costs work, not messages: one exchange per
  step, and the right-hand side runs unchanged on owned + ghost particles.
* After the right-hand side the ghosts are dropped; the step size is the
  minimum of ``dt_adapt`` over all ranks (``allreduce(min)``), the largest
  h over all ranks checks the halo (``allreduce(max)``; a step whose h
  outgrew it is redone from its start with a wider halo), and particles
  that the predictor moved into another rank's slab move there.

Every rank takes the same collectives in the same order.  Data moves with
``all_to_all_single`` of packed FP64 rows: NCCL over NVLink between GPUs,
gloo on CPU tensors for the tests.  No collective reads another GPU's memory
from a kernel.

``DomainSolver`` is the driver; the right-hand side and the two integrator
halves come from a *stepper*: ``EngineStepper`` runs them through the C ABI
on this rank's GPU (``mhd_rhs``, ``mhd_step_initialize/stage1/stage2``).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _abi
from .particle_array import DIAGNOSTIC_FIELDS
from .particles import property_names

# Radius scale R of each kernel (support R h), src/scheme.py:48-56.
RADIUS_SCALE = {"cubic": 2.0, "quintic": 3.0, "wendland_c2": 2.0, "wendland_c4": 2.0, "wendland_c6": 2.0,
                "gaussian": 3.0, "super_gaussian": 3.0}
COMPACT = frozenset(("cubic", "quintic", "wendland_c2", "wendland_c4", "wendland_c6"))

# Halo slack: W covers R (1 + LIST_MARGIN) h_max * HALO_SAFETY of the h at
# the start of the step, so h may grow by a quarter during the density
# iteration before a step is redone.
LIST_MARGIN = 0.02
HALO_SAFETY = 1.25


def _dist():
    import torch.distributed as tdist

    return tdist if tdist.is_available() and tdist.is_initialized() else None


def complete_arrays(arrays: dict) -> dict:
    """Every property name of the scheme as a contiguous tensor of the
    particle count (absent ones zero; ``itype`` 1, int32)."""
    x = arrays["x"]
    n, dev = x.numel(), x.device
    out = {}
    for k in property_names():
        v = arrays.get(k)
        if v is None:
            v = torch.ones(n, dtype=torch.int32, device=dev) if k == "itype" else torch.zeros(
                n, dtype=torch.float64, device=dev)
        elif k == "itype":
            v = v.to(torch.int32)
        else:
            v = v.to(torch.float64)
        if v.shape != (n,):
            raise ValueError(f"property {k} has shape {tuple(v.shape)}, expected ({n},)")
        out[k] = v.contiguous()
    return out


class Comm:
    """The collectives of the decomposition on the initialised process group
    (world 1 without one).  With the gloo backend tensors travel through host
    memory; with NCCL they stay on the device."""

    def __init__(self):
        tdist = _dist()
        self.tdist = tdist
        self.rank = tdist.get_rank() if tdist else 0
        self.world = tdist.get_world_size() if tdist else 1
        self.host = bool(tdist) and tdist.get_backend() == "gloo"

    def _to(self, t: torch.Tensor):
        return t.cpu() if self.host else t

    def allreduce(self, value: float, op: str, device) -> float:
        if self.tdist is None:
            return float(value)
        t = self._to(torch.tensor([float(value)], dtype=torch.float64, device=device))
        self.tdist.all_reduce(t, op=self.tdist.ReduceOp.MIN if op == "min" else
                              (self.tdist.ReduceOp.MAX if op == "max" else self.tdist.ReduceOp.SUM))
        return float(t.item())

    def allreduce_tensor(self, t: torch.Tensor) -> torch.Tensor:
        if self.tdist is None:
            return t
        h = self._to(t.clone())
        self.tdist.all_reduce(h)
        return h.to(t.device)

    def alltoall_rows(self, rows: torch.Tensor, counts: list[int]) -> torch.Tensor:
        """Rows ``rows[sum(counts[:q]) : sum(counts[:q+1])]`` go to rank q; the
        result holds the rows every rank sent here, in rank order."""
        if self.tdist is None:
            return rows[: counts[0]].clone()
        dev = rows.device
        send = torch.tensor(counts, dtype=torch.int64)
        recv = torch.empty_like(send)
        if self.host:
            self.tdist.all_to_all_single(recv, send)
        else:
            r = send.to(dev)
            o = torch.empty_like(r)
            self.tdist.all_to_all_single(o, r)
            recv = o.cpu()
        width = rows.shape[1]
        out = torch.empty((int(recv.sum()), width), dtype=rows.dtype, device="cpu" if self.host else dev)
        self.tdist.all_to_all_single(out, self._to(rows).contiguous(), output_split_sizes=recv.tolist(),
                                     input_split_sizes=list(counts))
        return out.to(dev)


class Slabs:
    """Slabs along ``axis`` of the box ``[lo, hi]``: rank r owns coordinates
    in ``[cuts[r], cuts[r+1])`` (the first and last slabs are open towards
    the box faces)."""

    def __init__(self, lo: float, hi: float, periodic: bool, cuts):
        self.lo, self.hi = float(lo), float(hi)
        self.L = self.hi - self.lo
        self.periodic = bool(periodic)
        self.cuts = [float(c) for c in cuts]
        if len(self.cuts) < 2 or any(b < a for a, b in zip(self.cuts, self.cuts[1:])):
            raise ValueError("slab cuts must be non-decreasing, one more than the ranks")

    @property
    def world(self):
        return len(self.cuts) - 1

    @classmethod
    def balanced(cls, coord: torch.Tensor, lo: float, hi: float, periodic: bool, comm: Comm, bins: int = 4096):
        """Cuts at the quantiles of the global particle distribution along the
        axis (a histogram summed over ranks), so every slab holds about the
        same number of particles."""
        world = comm.world
        lo_, hi_ = float(lo), float(hi)
        if not periodic:
            lo_ = -comm.allreduce(-float(coord.min()) if coord.numel() else -math.inf, "max", coord.device)
            hi_ = comm.allreduce(float(coord.max()) if coord.numel() else -math.inf, "max", coord.device)
            hi_ = hi_ + 1e-12 * max(1.0, abs(hi_ - lo_))
        edges = torch.linspace(lo_, hi_, bins + 1, dtype=torch.float64)
        idx = torch.clamp(((coord.double().cpu() - lo_) / (hi_ - lo_) * bins).floor().long(), 0, bins - 1)
        hist = torch.bincount(idx, minlength=bins).to(torch.float64)
        hist = comm.allreduce_tensor(hist.to(coord.device)).cpu()
        cum = torch.cumsum(hist, 0)
        total = float(cum[-1])
        cuts = [lo_]
        for r in range(1, world):
            b = int(torch.searchsorted(cum, torch.tensor(total * r / world, dtype=torch.float64)))
            cuts.append(float(edges[min(b + 1, bins)]))
        cuts.append(hi_)
        for r in range(1, len(cuts)):
            cuts[r] = max(cuts[r], cuts[r - 1])
        return cls(lo if periodic else lo_, hi if periodic else hi_, periodic, cuts)

    def owner(self, coord: torch.Tensor) -> torch.Tensor:
        inner = torch.tensor(self.cuts[1:-1], dtype=torch.float64, device=coord.device)
        return torch.bucketize(coord.double(), inner, right=True)

    def distance(self, coord: torch.Tensor, r: int) -> torch.Tensor:
        """Distance along the axis from each coordinate to slab r (0 inside),
        through the periodic images when the axis is periodic."""
        a, b = self.cuts[r], self.cuts[r + 1]
        c = coord.double()
        d = torch.clamp(a - c, min=0.0) + torch.clamp(c - b, min=0.0)
        if self.periodic:
            for s in (-self.L, self.L):
                cs = c + s
                d = torch.minimum(d, torch.clamp(a - cs, min=0.0) + torch.clamp(cs - b, min=0.0))
        return d

    def thickness(self, r: int) -> float:
        return self.cuts[r + 1] - self.cuts[r]


class DomainSolver:
    """The reference's time loop (src/solver.py:22-77) for one case whose
    particles are shared out over the ranks of the process group.

    ``arrays`` holds this rank's particles as tensors keyed by property name
    (all the same length; ``gid`` is the global particle id).  ``stepper``
    evaluates right-hand sides and the integrator halves on them.  With one
    rank the solver runs the whole case with no ghosts and no messages.
    """

    def __init__(self, stepper, arrays: dict, params: dict, axis: int = 0, comm: Comm | None = None,
                 slabs: Slabs | None = None):
        self.stepper = stepper
        self.comm = comm or Comm()
        self.p = dict(params)
        self.axis = int(axis)
        self.coord = "xyz"[self.axis]
        if self.p["kernel"] not in COMPACT and self.comm.world > 1:
            # a truncated Gaussian's density sums also take j's h (r < R h_j),
            # which the frozen outer ghosts do not carry exactly
            raise ValueError("the domain decomposition needs a compact kernel")
        self.R = RADIUS_SCALE[self.p["kernel"]]
        self.device = arrays["x"].device
        arrays = complete_arrays(arrays)
        self.names = list(arrays)
        lo, hi = self.p["lo"][self.axis], self.p["hi"][self.axis]
        periodic = bool(self.p["periodic"][self.axis])
        self.slabs = slabs or Slabs.balanced(arrays[self.coord], lo, hi, periodic, self.comm)
        self.owned = arrays
        self.halo_scale = HALO_SAFETY
        self.t = 0.0
        self.count = 0
        self.redone = 0
        self.ghost_counts: list[int] = []
        self.owned = self._migrate(self.owned)

    # ------------------------------------------------------------ plumbing
    def _pack(self, arrays, names):
        cols = [arrays[k].to(torch.float64) for k in names]
        return torch.stack(cols, 1) if cols else torch.empty((0, 0), dtype=torch.float64, device=self.device)

    def _unpack(self, rows, names, like):
        out = {}
        for c, k in enumerate(names):
            out[k] = rows[:, c].to(like[k].dtype).contiguous()
        return out

    def _cat(self, a, b):
        return {k: torch.cat([a[k], b[k]]) for k in a}

    def _take(self, arrays, idx):
        return {k: v[idx].contiguous() for k, v in arrays.items()}

    def _migrate(self, arrays):
        """Particles outside this rank's slab move to the rank that owns them."""
        if self.comm.world == 1:
            return arrays
        own = self.slabs.owner(arrays[self.coord])
        order = torch.argsort(own, stable=True)
        counts = torch.bincount(own, minlength=self.comm.world).tolist()
        rows = self._pack(self._take(arrays, order), self.names)
        got = self.comm.alltoall_rows(rows, counts)
        return self._unpack(got, self.names, arrays)

    def halo_width(self, h_max: float) -> float:
        return self.R * (1.0 + LIST_MARGIN) * h_max * self.halo_scale

    def _with_ghosts(self, owned, width):
        """Owned particles followed by the ghosts every other rank sends
        (within 2 width of this slab); outer ghosts (beyond width) frozen for
        the density iteration.  Returns (local arrays, number owned)."""
        comm = self.comm
        if comm.world == 1:
            return owned, owned["x"].numel()
        for r in range(comm.world):
            if self.slabs.thickness(r) < 2.0 * width:
                raise RuntimeError(f"slab {r} is thinner than twice the halo ({self.slabs.thickness(r):.3g} < "
                                   f"{2.0 * width:.3g}): use fewer ranks")
        c = owned[self.coord]
        parts, counts = [], []
        for q in range(comm.world):
            if q == comm.rank:
                counts.append(0)
                continue
            sel = torch.nonzero(self.slabs.distance(c, q) < 2.0 * width).flatten()
            parts.append(sel)
            counts.append(int(sel.numel()))
        idx = torch.cat(parts) if parts else torch.empty(0, dtype=torch.long, device=self.device)
        rows = self._pack(self._take(owned, idx), self.names)
        got = comm.alltoall_rows(rows, counts)
        ghosts = self._unpack(got, self.names, owned)
        outer = self.slabs.distance(ghosts[self.coord], comm.rank) >= width
        ghosts["converged"] = torch.where(outer, torch.ones_like(ghosts["converged"]), ghosts["converged"])
        self.ghost_counts.append(int(got.shape[0]))
        return self._cat(owned, ghosts), owned["x"].numel()

    def _owned_after(self, local):
        mask = self.slabs.owner(local[self.coord]) == self.comm.rank
        return self._take(local, torch.nonzero(mask).flatten())

    def _h_max(self, arrays):
        h = arrays["h"]
        return self.comm.allreduce(float(h.max()) if h.numel() else 0.0, "max", self.device)

    def _rhs(self, owned):
        """Right-hand side of the owned particles with ghosts; widens the halo
        and repeats while the resulting h outgrow it."""
        while True:
            width = self.halo_width(self._h_max(owned))
            # with several ranks the local arrays are new tensors: `owned`
            # stays as it was for a repeat
            local, _ = self._with_ghosts(owned, width)
            local = self.stepper.rhs(local)
            out = self._owned_after(local)
            h_new = self._h_max(out)
            if self.comm.world == 1 or self.R * (1.0 + LIST_MARGIN) * h_new <= width:
                return out
            self.halo_scale *= 1.5
            self.redone += 1

    # ------------------------------------------------------- time stepping
    def warmup(self):
        """src/application.py:110-132: three right-hand sides with the B restore."""
        owned = self.owned
        b0 = {k: owned[k].clone() for k in ("Bx", "By", "Bz")}
        gid0 = owned["gid"].clone()
        owned["h0"] = owned["h"].clone()
        self._sync_initial_mhd_state(owned)
        owned = self._rhs(owned)
        self._check_converged(owned)
        order = torch.argsort(gid0)
        idx = order[torch.searchsorted(gid0[order], owned["gid"])]
        for k in ("Bx", "By", "Bz"):
            owned[k] = b0[k][idx].clone()
        owned["h0"] = owned["h"].clone()
        self._sync_initial_mhd_state(owned)
        for _ in range(2):
            owned = self._rhs(owned)
        self._check_converged(owned)
        self.owned = owned

    def _check_converged(self, owned):
        bad = float((owned["converged"] != 1).sum()) if owned["converged"].numel() else 0.0
        if self.comm.allreduce(bad, "sum", self.device) > 0:
            raise RuntimeError("density iteration did not converge in the warm-up RHS")

    @staticmethod
    def _sync_initial_mhd_state(a):
        """src/application.py:99-108."""
        a["Bevolx"] = a["Bx"] / a["rho"]
        a["Bevoly"] = a["By"] / a["rho"]
        a["Bevolz"] = a["Bz"] / a["rho"]
        a["psi"] = torch.zeros_like(a["psi"])
        for pred, cur in (("Bevolxpred", "Bevolx"), ("Bevolypred", "Bevoly"), ("Bevolzpred", "Bevolz"),
                          ("psipred", "psi"), ("upred", "u"), ("vpred", "v"), ("wpred", "w"), ("epred", "e")):
            a[pred] = a[cur].clone()

    def initial_dt(self) -> float:
        """src/application.py:134-147 over all ranks."""
        a = self.owned
        tf = self.p["timestep_factor"]
        dev = self.device
        if a["h"].numel():
            if not bool(torch.all(a["dt_cfl"] > 0.0)):
                raise RuntimeError("dt_cfl must be positive after the warm-up")
            c = float(torch.min(tf * 0.3 * a["h"] / a["dt_cfl"]))
            force = torch.sqrt(a["au"] * a["au"] + a["av"] * a["av"] + a["aw"] * a["aw"])
            mask = force > 0.0
            f = float(torch.min(tf * 0.25 * torch.sqrt(a["h"][mask] / force[mask]))) if bool(mask.any()) else math.inf
        else:
            c = f = math.inf
        dt = min(self.comm.allreduce(c, "min", dev), self.comm.allreduce(f, "min", dev))
        if not dt > 0.0:
            raise RuntimeError("initial dt must be positive")
        return dt

    def min_dt(self) -> float:
        """The adaptive rule over all ranks: min dt_adapt."""
        d = self.owned["dt_adapt"]
        return self.comm.allreduce(float(d.min()) if d.numel() else math.inf, "min", self.device)

    def step(self, dt: float):
        """PECIntegrator.one_timestep: predictor, migration, RHS with ghosts,
        corrector."""
        owned = self.owned
        self.stepper.predict(owned, dt)
        owned = self._migrate(owned)
        owned = self._rhs(owned)
        self.stepper.correct(owned, dt)
        self.owned = owned
        self.t += dt
        self.count += 1

    def run(self, n_steps: int, tf: float = 1e30):
        """The solver loop with the adaptive step (min over ranks), clipped to tf."""
        dt = min(self.min_dt(), tf - self.t)
        done = 0
        while (tf - self.t) > 2.220446049250313e-16 * tf * max(self.count, 1) and done < n_steps:
            self.step(dt)
            done += 1
            dt = self.min_dt()
            if self.t + dt > tf:
                dt = tf - self.t
        return done

    def gather(self, names=None) -> dict:
        """Every rank's owned particles, in gid order, as numpy arrays (on every rank)."""
        names = list(names or self.names)
        part = {k: self.owned[k].cpu().numpy() for k in names}
        tdist = self.comm.tdist
        parts = [part]
        if tdist is not None:
            parts = [None] * self.comm.world
            tdist.all_gather_object(parts, part)
        out = {k: np.concatenate([p[k] for p in parts]) for k in names}
        if "gid" in out:
            order = np.argsort(out["gid"], kind="stable")
            out = {k: v[order] for k, v in out.items()}
        return out


class EngineStepper:
    """The right-hand side and the integrator halves on this rank's GPU
    through the C ABI: ``mhd_rhs`` (the neighbour sort, DensityIteration and
    the fused force groups), ``mhd_step_initialize`` + ``mhd_step_stage1``
    (with the periodic wrap) and ``mhd_step_stage2``.  The particle count
    changes every step (ghosts, migration); the context is sized with
    headroom and re-made when a step needs more."""

    def __init__(self, params: _abi.MhdParams, capacity: int):
        if not torch.cuda.is_available():
            raise RuntimeError("the SPMHD B200 engine needs a CUDA device (no CPU fallback)")
        self.lib = _abi.load()
        self.params = params
        self.ctx = ctypes.c_void_p()
        self.capacity = 0
        self._ensure(int(capacity))
        self.density_passes: list[int] = []

    def _ensure(self, n: int):
        if n <= self.capacity and self.ctx:
            return
        self.close()
        cap = max(int(n * 1.25) + 64, 64)
        _abi.check(self.lib.mhd_ctx_create(ctypes.byref(self.params), cap, ctypes.byref(self.ctx)), None)
        self.capacity = cap

    def close(self):
        if self.ctx:
            self.lib.mhd_ctx_destroy(self.ctx)
            self.ctx = ctypes.c_void_p()
            self.capacity = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def _state(a: dict, spare: dict | None = None):
        """MhdState over the tensors of `a` (the sorted fields from `spare`
        when given); diagnostic outputs are left out, as ParticleArray
        leaves them out by default."""
        s = _abi.state_type()()
        for f in _abi.STATE_FIELDS:
            if f in DIAGNOSTIC_FIELDS:
                continue
            t = (spare or {}).get(f, a.get(f))
            if t is not None:
                setattr(s, f, ctypes.c_void_p(t.data_ptr()))
        return s

    @staticmethod
    def _complete(a: dict):
        for f in a:
            if not a[f].is_contiguous():
                a[f] = a[f].contiguous()

    def predict(self, a: dict, dt: float):
        n = a["x"].numel()
        if n == 0:
            return
        self._ensure(n)
        self._complete(a)
        s = self._state(a)
        _abi.check(self.lib.mhd_step_initialize(self.ctx, ctypes.byref(s), n, self.stream), self.ctx)
        _abi.check(self.lib.mhd_step_stage1(self.ctx, ctypes.byref(s), n, float(dt), self.stream), self.ctx)

    def rhs(self, a: dict) -> dict:
        n = a["x"].numel()
        if n == 0:
            return a
        self._ensure(n)
        self._complete(a)
        spare = {k: torch.empty_like(a[k]) for k in _abi.SORTED_FIELDS if k in a}
        src, dst = self._state(a), self._state(a, spare)
        st = _abi.MhdRhsStats()
        _abi.check(self.lib.mhd_rhs(self.ctx, ctypes.byref(src), ctypes.byref(dst), n, ctypes.byref(st), self.stream),
                   self.ctx)
        self.density_passes.append(int(st.density_passes))
        out = dict(a)
        out.update(spare)
        return out

    def correct(self, a: dict, dt: float):
        n = a["x"].numel()
        if n == 0:
            return
        self._ensure(n)
        s = self._state(a)
        _abi.check(self.lib.mhd_step_stage2(self.ctx, ctypes.byref(s), n, float(dt), self.stream), self.ctx)
