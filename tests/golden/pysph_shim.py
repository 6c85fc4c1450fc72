"""Minimal PySPH-semantics shim, used only by ``make_golden.py``.

Test infrastructure: nothing in the product imports this file.

PySPH (the library the reference runs on) is not installed and cannot be
installed here.  The reference's physics, however, is plain Python: every
``Equation`` and ``IntegratorStep`` method in ``src/equations.py`` and
``src/integrator.py`` is a scalar function of ``d_idx``/``s_idx``, named
arrays and the pair symbols ``XIJ, RIJ, WI, DWI, DWJ, GHI, RHOIJ``.  This shim
installs small stand-ins for the ``pysph``/``compyle`` modules the reference
imports, so the reference's own equation, integrator, scheme, warm-up
(``src/application.py:94-147``) and solver-loop (``src/solver.py:22-77``) code
runs unchanged, in pure-Python loops, on tiny particle sets.

What the shim itself restates (PySPH semantics; unpinned, since PySPH's
source is not available) -- each item is a decision of this restatement:

* kernels: cubic spline (Monaghan M4, R=2), quintic spline (Morris, R=3),
  Wendland C2/C4/C6 (R=2), Gaussian and super-Gaussian (R=3), each with its
  d-dimensional normalisation and ``dW/dh = -(d*w + q*dw/dq) * sigma/h^(d+1)``;
* neighbours of i: every j (i included) with ``r2 < (R*h_i)^2`` or
  ``r2 < (R*h_j)^2``, ``r2 = (dx*dx + dy*dy) + dz*dz`` on the minimum-image
  displacement ``x_i - x_j``; summation in ascending j;
* ``Group`` execution: ``initialize`` for all particles, ``loop`` over every
  neighbour pair, ``post_loop``; an iterated group stops after a pass when
  ``passes >= min_iterations`` and ``converged() > 0``, or when
  ``passes == max_iterations``; neighbours are recomputed from the current h
  before every pass;
* ``PECIntegrator.one_timestep``: initialize, stage1, periodic wrap, RHS,
  stage2, periodic wrap;
* ``Solver._get_timestep``: ``min(dt_adapt)``, clipped so ``t + dt <= tf``.
"""

from __future__ import annotations

import contextlib
import inspect
import math
import sys
import types

import numpy as np

M_PI = math.pi


# --------------------------------------------------------------------------
# Kernels (PySPH ``pysph.base.kernels`` semantics, restated)
# --------------------------------------------------------------------------
class _Kernel:
    radius_scale = 2.0
    norms = {}

    def __init__(self, dim=3):
        self.dim = dim
        self.fac = self.norms[dim]

    def _fac(self, h1):
        if self.dim == 1:
            return self.fac * h1
        if self.dim == 2:
            return self.fac * h1 * h1
        return self.fac * h1 * h1 * h1

    def kernel(self, xij, rij, h):
        h1 = 1.0 / h
        q = rij * h1
        w, _ = self.w_dw(q)
        return w * self._fac(h1)

    def gradient(self, xij, rij, h, grad):
        h1 = 1.0 / h
        if rij > 1.0e-12:
            q = rij * h1
            _, dw = self.w_dw(q)
            tmp = self._fac(h1) * dw * h1 / rij
        else:
            tmp = 0.0
        grad[0] = tmp * xij[0]
        grad[1] = tmp * xij[1]
        grad[2] = tmp * xij[2]

    def gradient_h(self, xij, rij, h):
        h1 = 1.0 / h
        q = rij * h1
        w, dw = self.w_dw(q)
        return -self._fac(h1) * h1 * (dw * q + w * self.dim)


class CubicSpline(_Kernel):
    radius_scale = 2.0
    norms = {1: 2.0 / 3.0, 2: 10.0 / (7.0 * M_PI), 3: 1.0 / M_PI}

    @staticmethod
    def w_dw(q):
        if q > 2.0:
            return 0.0, 0.0
        if q > 1.0:
            t = 2.0 - q
            return 0.25 * t * t * t, -0.75 * t * t
        return 1.0 - 1.5 * q * q * (1.0 - 0.5 * q), -3.0 * q * (1.0 - 0.75 * q)


class QuinticSpline(_Kernel):
    radius_scale = 3.0
    norms = {1: 1.0 / 120.0, 2: 7.0 / (478.0 * M_PI), 3: 1.0 / (120.0 * M_PI)}

    @staticmethod
    def w_dw(q):
        if q > 3.0:
            return 0.0, 0.0
        t3 = 3.0 - q
        t2 = 2.0 - q
        t1 = 1.0 - q
        w = t3 * t3 * t3 * t3 * t3
        dw = -5.0 * t3 * t3 * t3 * t3
        if q > 2.0:
            return w, dw
        w -= 6.0 * t2 * t2 * t2 * t2 * t2
        dw += 30.0 * t2 * t2 * t2 * t2
        if q > 1.0:
            return w, dw
        w += 15.0 * t1 * t1 * t1 * t1 * t1
        dw -= 75.0 * t1 * t1 * t1 * t1
        return w, dw


class WendlandQuintic(_Kernel):
    radius_scale = 2.0
    norms = {1: 3.0 / 4.0, 2: 7.0 / (4.0 * M_PI), 3: 21.0 / (16.0 * M_PI)}

    @staticmethod
    def w_dw(q):
        if q >= 2.0:
            return 0.0, 0.0
        s = 1.0 - 0.5 * q
        s3 = s * s * s
        return s3 * s * (2.0 * q + 1.0), -5.0 * q * s3


class WendlandQuinticC4(_Kernel):
    radius_scale = 2.0
    norms = {1: 5.0 / 8.0, 2: 9.0 / (4.0 * M_PI), 3: 495.0 / (256.0 * M_PI)}

    @staticmethod
    def w_dw(q):
        if q >= 2.0:
            return 0.0, 0.0
        s = 1.0 - 0.5 * q
        s5 = s * s * s * s * s
        w = s5 * s * (35.0 / 12.0 * q * q + 3.0 * q + 1.0)
        dw = -14.0 / 3.0 * q * (1.0 + 2.5 * q) * s5
        return w, dw


class WendlandQuinticC6(_Kernel):
    radius_scale = 2.0
    norms = {1: 55.0 / 64.0, 2: 78.0 / (28.0 * M_PI), 3: 1365.0 / (512.0 * M_PI)}

    @staticmethod
    def w_dw(q):
        if q >= 2.0:
            return 0.0, 0.0
        s = 1.0 - 0.5 * q
        s7 = s * s * s * s * s * s * s
        w = s7 * s * (4.0 * q * q * q + 6.25 * q * q + 4.0 * q + 1.0)
        dw = -5.5 * q * (1.0 + 3.5 * q + 4.0 * q * q) * s7
        return w, dw


class Gaussian(_Kernel):
    radius_scale = 3.0
    norms = {1: 1.0 / math.sqrt(M_PI), 2: 1.0 / M_PI, 3: 1.0 / (M_PI * math.sqrt(M_PI))}

    @staticmethod
    def w_dw(q):
        if q >= 3.0:
            return 0.0, 0.0
        e = math.exp(-q * q)
        return e, -2.0 * q * e


class SuperGaussian(_Kernel):
    radius_scale = 3.0
    norms = Gaussian.norms

    def w_dw(self, q):
        if q >= 3.0:
            return 0.0, 0.0
        e = math.exp(-q * q)
        d2 = 0.5 * self.dim
        return e * (d2 + 1.0 - q * q), -2.0 * q * e * (d2 + 2.0 - q * q)


# --------------------------------------------------------------------------
# Particle array, domain, neighbours
# --------------------------------------------------------------------------
class ParticleArray:
    def __init__(self, name, **props):
        object.__setattr__(self, "name", name)
        object.__setattr__(self, "gpu", None)
        object.__setattr__(self, "properties", {})
        n = len(next(iter(props.values())))
        for k, v in props.items():
            a = np.asarray(v)
            if k == "itype":
                a = a.astype(np.int32)
            else:
                a = a.astype(np.float64)
            self.properties[k] = a.copy()
        for k in ("x", "y", "z", "u", "v", "w", "m", "h", "rho", "p", "au", "av", "aw"):
            self.properties.setdefault(k, np.zeros(n))
        self.properties.setdefault("gid", np.arange(n, dtype=np.float64))
        self.properties.setdefault("tag", np.zeros(n))

    def __getattr__(self, k):
        try:
            return self.properties[k]
        except KeyError as e:
            raise AttributeError(k) from e

    def __setattr__(self, k, v):
        self.properties[k][:] = v

    def get_number_of_particles(self):
        return len(self.properties["x"])

    def add_property(self, name, default=0.0, type="double"):
        if name not in self.properties:
            dt = np.int32 if type == "int" else np.float64
            self.properties[name] = np.full(self.get_number_of_particles(), default, dtype=dt)

    def set_output_arrays(self, names):
        pass


def get_particle_array(name="", **props):
    return ParticleArray(name, **props)


class DomainManager:
    def __init__(self, xmin=0.0, xmax=0.0, ymin=0.0, ymax=0.0, zmin=0.0, zmax=0.0,
                 periodic_in_x=False, periodic_in_y=False, periodic_in_z=False, periodic_mode=None, **kw):
        self.lo = (xmin, ymin, zmin)
        self.hi = (xmax, ymax, zmax)
        self.periodic = (periodic_in_x, periodic_in_y, periodic_in_z)
        self.mode = periodic_mode

    def min_image(self, d, axis):
        if not self.periodic[axis]:
            return d
        L = self.hi[axis] - self.lo[axis]
        half = 0.5 * L
        d = np.where(d > half, d - L, d)
        d = np.where(d < -half, d + L, d)
        return d

    def wrap(self, pa):
        for axis, name in enumerate(("x", "y", "z")):
            if not self.periodic[axis]:
                continue
            lo, hi = self.lo[axis], self.hi[axis]
            L = hi - lo
            a = pa.properties[name]
            a[:] = np.where(a < lo, a + L, a)
            a[:] = np.where(a > hi, a - L, a)


def neighbour_lists(pa, domain, radius_scale, dim):
    """Brute-force neighbour lists under the symmetric rule, ascending j."""
    x, y, z, h = pa.x, pa.y, pa.z, pa.h
    n = len(x)
    out = []
    rh = radius_scale * h
    rh2 = rh * rh
    for i in range(n):
        dx = domain.min_image(x[i] - x, 0)
        dy = domain.min_image(y[i] - y, 1)
        dz = domain.min_image(z[i] - z, 2) if dim == 3 else np.zeros(n)
        r2 = dx * dx + dy * dy + dz * dz
        sel = (r2 < rh2[i]) | (r2 < rh2)
        out.append(np.nonzero(sel)[0])
    return out


# --------------------------------------------------------------------------
# Equations, groups, integrator, solver
# --------------------------------------------------------------------------
class Equation:
    def __init__(self, dest, sources):
        self.dest = dest
        self.sources = sources

    def converged(self):
        return 1.0


class Group:
    def __init__(self, equations, real=True, update_nnps=False, iterate=False,
                 max_iterations=1, min_iterations=0, pre=None, post=None, condition=None, start_idx=0, stop_idx=None):
        self.equations = equations
        self.update_nnps = update_nnps
        self.iterate = iterate
        self.max_iterations = max_iterations
        self.min_iterations = min_iterations


class IntegratorStep:
    pass


_PAIR = ("XIJ", "RIJ", "WI", "DWI", "DWJ", "GHI", "RHOIJ")


def _own(obj, name):
    """The method ``name`` if the equation's class defines it (not the base)."""
    for cls in type(obj).__mro__:
        if cls in (Equation, IntegratorStep, object):
            return None
        if name in cls.__dict__:
            return getattr(obj, name)
    return None


class _Caller:
    def __init__(self, meth):
        self.meth = meth
        self.params = [p for p in inspect.signature(meth).parameters]

    def __call__(self, arrays, i, j=None, pair=None, dt=None, t=None):
        kw = {}
        for p in self.params:
            if p == "d_idx":
                kw[p] = i
            elif p == "s_idx":
                kw[p] = j
            elif p.startswith("d_") or p.startswith("s_"):
                kw[p] = arrays[p[2:]]
            elif p in _PAIR:
                kw[p] = pair[p]
            elif p == "dt":
                kw[p] = dt
            elif p == "t":
                kw[p] = t
            else:
                raise KeyError(p)
        return self.meth(**kw)


class Runtime:
    """Executes equation groups and integrator stages over a ParticleArray."""

    def __init__(self, pa, groups, kernel, domain, dim):
        self.pa = pa
        self.groups = groups
        self.kernel = kernel
        self.domain = domain
        self.dim = dim
        self.density_passes = []

    def _lists(self):
        return {k: v.tolist() for k, v in self.pa.properties.items()}

    def _store(self, arrays):
        for k, v in arrays.items():
            self.pa.properties[k][:] = v

    def _pair(self, arrays, i, j):
        d = self.domain
        x, y, z = arrays["x"], arrays["y"], arrays["z"]
        dx = float(d.min_image(np.float64(x[i] - x[j]), 0))
        dy = float(d.min_image(np.float64(y[i] - y[j]), 1))
        dz = float(d.min_image(np.float64(z[i] - z[j]), 2)) if self.dim == 3 else 0.0
        xij = [dx, dy, dz]
        rij = math.sqrt(dx * dx + dy * dy + dz * dz)
        hi, hj = arrays["h"][i], arrays["h"][j]
        k = self.kernel
        dwi = [0.0, 0.0, 0.0]
        dwj = [0.0, 0.0, 0.0]
        k.gradient(xij, rij, hi, dwi)
        k.gradient(xij, rij, hj, dwj)
        return {
            "XIJ": xij,
            "RIJ": rij,
            "WI": k.kernel(xij, rij, hi),
            "DWI": dwi,
            "DWJ": dwj,
            "GHI": k.gradient_h(xij, rij, hi),
            "RHOIJ": 0.5 * (arrays["rho"][i] + arrays["rho"][j]),
        }

    def _run_group(self, g):
        n = self.pa.get_number_of_particles()
        passes = 0
        while True:
            arrays = self._lists()
            for eq in g.equations:
                f = _own(eq, "initialize")
                if f is not None:
                    c = _Caller(f)
                    for i in range(n):
                        c(arrays, i)
            # An equation without sources runs its ``loop`` once per destination
            # particle (no neighbours), e.g. ``IdealGasEOS`` (src/equations.py:103-106).
            for eq in g.equations:
                f = _own(eq, "loop")
                if f is not None and not eq.sources:
                    c = _Caller(f)
                    for i in range(n):
                        c(arrays, i)
            loops = [(_Caller(_own(eq, "loop"))) for eq in g.equations if eq.sources and _own(eq, "loop")]
            if loops:
                self._store(arrays)
                nbrs = neighbour_lists(self.pa, self.domain, self.kernel.radius_scale, self.dim)
                for i in range(n):
                    for j in nbrs[i]:
                        j = int(j)
                        pair = self._pair(arrays, i, j)
                        for c in loops:
                            c(arrays, i, j, pair)
            for eq in g.equations:
                f = _own(eq, "post_loop")
                if f is not None:
                    c = _Caller(f)
                    for i in range(n):
                        c(arrays, i)
            self._store(arrays)
            passes += 1
            if not g.iterate:
                break
            conv = min(eq.converged() for eq in g.equations)
            if (passes >= g.min_iterations and conv > 0) or passes == g.max_iterations:
                break
        return passes

    def compute_accelerations(self):
        for k, g in enumerate(self.groups):
            p = self._run_group(g)
            if k == 0:
                self.density_passes.append(p)

    def stage(self, stepper, name, dt):
        f = _own(stepper, name)
        if f is None:
            return
        c = _Caller(f)
        arrays = self._lists()
        for i in range(self.pa.get_number_of_particles()):
            c(arrays, i, dt=dt)
        self._store(arrays)


class PECIntegrator:
    def __init__(self, **steppers):
        self.steppers = steppers
        self.rt = None

    def attach(self, runtime):
        self.rt = runtime

    def initial_acceleration(self, t, dt):
        self.rt.compute_accelerations()

    def step(self, t, dt):
        st = self.steppers["fluid"]
        self.rt.stage(st, "initialize", dt)
        self.rt.stage(st, "stage1", dt)
        self.rt.domain.wrap(self.rt.pa)
        self.rt.compute_accelerations()
        self.rt.stage(st, "stage2", dt)
        self.rt.domain.wrap(self.rt.pa)

    def compute_time_step(self):
        return float(np.min(self.rt.pa.dt_adapt))


EPSILON = 2.220446049250313e-16


class Solver:
    def __init__(self, dim=3, integrator=None, kernel=None, dt=1.0, tf=1.0, adaptive_timestep=True, pfreq=1, **kw):
        self.dim = dim
        self.integrator = integrator
        self.kernel = kernel
        self.dt = dt
        self.tf = tf
        self.adaptive_timestep = adaptive_timestep
        self.t = 0.0
        self.count = 0
        self.max_steps = 1 << 62
        self.in_parallel = False
        self.rank = 0
        self.reorder_freq = 0
        self.pre_step_callbacks = []
        self.post_step_callbacks = []
        self.execute_commands = None
        self.command_interval = 1

    def dump_output(self):
        pass

    def barrier(self):
        pass

    def reorder_particles(self):
        pass

    def _dump_output_if_needed(self):
        pass

    def update_particle_time(self):
        pass

    def _get_timestep(self):
        dt = self.integrator.compute_time_step() if self.adaptive_timestep else self.dt
        if self.t + dt > self.tf:
            dt = self.tf - self.t
        return dt


class ProgressBar:
    def __init__(self, *a, **k):
        pass

    def update(self, *a):
        pass

    def finish(self):
        pass


class Scheme:
    def _ensure_properties(self, pa, props, clean=True):
        for p in props:
            if isinstance(p, dict):
                pa.add_property(p["name"], default=p.get("default", 0), type=p.get("type", "double"))
            else:
                pa.add_property(p)


class Application:
    def __init__(self, fname=None, **kw):
        self.fname = fname
        self.initialize()
        self.scheme = self.create_scheme()

    def solve(self):
        self.solver.solve()


@contextlib.contextmanager
def profile_ctx(name):
    yield


def install():
    """Register the stand-in modules under the names the reference imports."""

    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        sys.modules[name] = m
        return m

    mod("pysph")
    mod("pysph.base")
    mod("pysph.base.kernels", CubicSpline=CubicSpline, QuinticSpline=QuinticSpline, Gaussian=Gaussian,
        SuperGaussian=SuperGaussian, WendlandQuintic=WendlandQuintic, WendlandQuinticC4=WendlandQuinticC4,
        WendlandQuinticC6=WendlandQuinticC6)
    mod("pysph.base.nnps", DomainManager=DomainManager)
    mod("pysph.base.utils", get_particle_array=get_particle_array)
    mod("pysph.sph")
    mod("pysph.sph.equation", Equation=Equation, Group=Group)
    mod("pysph.sph.integrator", PECIntegrator=PECIntegrator, Integrator=PECIntegrator)
    mod("pysph.sph.integrator_step", IntegratorStep=IntegratorStep)
    mod("pysph.sph.scheme", Scheme=Scheme)
    mod("pysph.solver")
    mod("pysph.solver.solver", Solver=Solver, EPSILON=EPSILON)
    mod("pysph.solver.utils", ProgressBar=ProgressBar)
    mod("pysph.solver.application", Application=Application)
    mod("compyle")
    mod("compyle.profile", profile_ctx=profile_ctx)
