"""Generate the golden fixtures in ``tests/golden/*.npz``.

Test infrastructure.  Run in the development container only (it imports the
read-only reference checkout, which does not exist on GPU machines):

    python tests/golden/make_golden.py /path/to/reference [case ...]
    MHD_REFERENCE_ROOT=/path/to/reference python tests/golden/make_golden.py

The physics executed here is the reference's own code, imported unchanged:
the 14 ``Equation`` classes of ``src/equations.py``, ``MHDStep`` of
``src/integrator.py``, the group list of ``MHDScheme.get_equations``
(``src/scheme.py:66-81``), the warm-up and initial-dt routines of
``src/application.py:99-147`` and the time loop ``MHDSolver.solve``
(``src/solver.py:22-77``).  ``pysph_shim`` supplies the PySPH layer the
reference runs on (kernels, neighbour rule, group iteration, PEC order,
timestep rule); those are restated, not pinned.

Cases (all tiny, pure-Python loops):

* ``ref_orstang3d`` -- the reference's own ``OrszagTang`` case at nx=8
  (close-packed 3-D slab, cubic kernel, ``configs/orstang.toml``), warm-up,
  initial dt and 2 adaptive steps;
* ``ot2d`` -- 2-D Orszag-Tang on a 16x16 square lattice, quintic kernel,
  hfact 1.2, dim=2 (the reference equations built with ``dim=2``), 3 steps;
* ``shock2d`` -- 2-D Brio-Wu tube, 16x24 left / 6x8 right lattice, frozen
  ``itype=3`` ends, quintic, hfact 1.0, gamma 2, 3 steps;
* ``blast3d`` -- 3-D MHD blast on an 8^3 cubic lattice, cubic kernel,
  hfact 1.2, gamma 5/3, 3 steps;
* ``ref_ics`` -- the initial particles the reference's sine, wave, rotor,
  vortex, current-loop and jet generators build from its own TOML files at a
  small nx (no stepping).
"""

from __future__ import annotations

import json
import math
import os
import sys
import time
from dataclasses import replace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import pysph_shim  # noqa: E402


def _import_reference(path):
    pysph_shim.install()
    sys.path.insert(0, path)
    import builtins

    # src/solver.py annotates a class attribute with a name it only imports
    # under TYPE_CHECKING; Python 3.12 evaluates class annotations eagerly.
    builtins.Integrator = object
    import src.application as application  # noqa: F401
    import src.cases.orstang as orstang
    import src.config as config
    import src.equations as equations
    import src.integrator as integrator
    import src.scheme as scheme
    import src.solver as solver

    return dict(application=application, orstang=orstang, config=config, equations=equations,
                integrator=integrator, scheme=scheme, solver=solver)


STORED = (
    "x y z gid itype u v w rho rho_sum h m cs p e au av aw ae ah h0 upred vpred wpred epred "
    "div dt_cfl dt_adapt omega converged alpha1 alpha10 alphaloc Bx By Bz Bevolx Bevoly Bevolz psi "
    "Bevolxpred Bevolypred Bevolzpred psipred Bxpred Bypred Bzpred aBevolx aBevoly aBevolz apsi "
    "divBsymm divBdiff div_for_psi xilimiter divvdt dwdh"
).split()


def _snap(pa, prefix, out):
    for k in STORED:
        out[f"{prefix}/{k}"] = np.array(pa.properties[k], copy=True)


def _case_config(ref, toml_name, **over):
    cfgmod = ref["config"]
    sim = cfgmod.load_config(os.path.join(REF, "configs", toml_name), {toml_name[:-5]: cfgmod.SimulationConfig})
    for section, kv in over.items():
        sim = replace(sim, **{section: replace(getattr(sim, section), **kv)})
    return sim


def _make_app(ref, cls, sim):
    app = cls(sim)
    app.particles = app.create_particles()
    domain = app.create_domain()
    app.configure_scheme()
    app.solver = app.scheme.solver
    return app, domain


def _run(app, domain, dim, steps, out):
    pa = app.particles[0]
    solver = app.solver
    if dim != 3:
        solver.kernel = type(solver.kernel)(dim=dim)
    groups = app.scheme.get_equations()
    if dim != 3:
        for g in groups:
            for eq in g.equations:
                if hasattr(eq, "dim"):
                    eq.dim = dim
                if hasattr(eq, "dim1"):
                    eq.dim1 = 1.0 / dim
    rt = pysph_shim.Runtime(pa, groups, solver.kernel, domain, dim)
    solver.integrator.attach(rt)
    solver.max_steps = steps
    _snap(pa, "ic", out)
    t0 = time.time()
    app._warm_initial_derivatives(solver)
    _snap(pa, "warm", out)
    app._compute_initial_dt(solver)
    out["dt0"] = np.array(solver.dt)
    records = []

    def after_step(s):
        k = s.count + 1
        _snap(pa, f"step{k}", out)
        records.append((s.t, s.dt))

    solver.post_step_callbacks.append(after_step)
    solver.solve()
    out["step_t"] = np.array([r[0] for r in records])
    out["step_dt"] = np.array([r[1] for r in records])
    out["density_passes"] = np.array(rt.density_passes)
    out["n_steps"] = np.array(steps)
    print(f"  {pa.get_number_of_particles()} particles, {steps} steps, {time.time() - t0:.1f}s, "
          f"density passes {rt.density_passes}", flush=True)


def _params(sim, dim, domain, alpha=(0.0, 1.0)):
    return dict(
        dim=dim, kernel=sim.numerics.kernel, hfact=sim.numerics.hfact, density=sim.numerics.density,
        gamma=sim.physics.gamma, mu0=sim.physics.mu0, av=sim.physics.artificial_viscosity,
        ac=sim.physics.artificial_thermal_conductivity, ar=sim.physics.artificial_magnetic_dissipation,
        clean_speed=sim.numerics.cleaning_speed_factor, clean_damp=sim.numerics.cleaning_damping_factor,
        timestep_factor=sim.solver.timestep_factor, tf=sim.solver.tf, adaptive=sim.solver.adaptive_timestep,
        lo=list(domain.lo), hi=list(domain.hi), periodic=[bool(p) for p in domain.periodic],
        alpha_min=alpha[0], alpha_max=alpha[1],
    )


def _square_app(ref, name, sim, bounds, make):
    """A case class over the reference's MHDApplication with our own initial condition."""
    base = ref["application"].MHDApplication

    class Case(base):
        @property
        def bounds(self):
            return bounds

        def create_mhd_particles(self):
            return [pysph_shim.get_particle_array(name="fluid", **make(self))]

    Case.__name__ = name
    return Case


def case_ref_orstang3d(ref, out):
    sim = _case_config(ref, "orstang.toml", case=dict(nx=8))
    app, domain = _make_app(ref, ref["orstang"].OrszagTang, sim)
    out["params"] = np.array(json.dumps(_params(sim, 3, domain)))
    _run(app, domain, 3, 2, out)


def case_ot2d(ref, out, n=16):
    sim = _case_config(ref, "orstang.toml", case=dict(nx=n), numerics=dict(kernel="quintic", hfact=1.2))
    lo, hi = -0.5, 0.5
    bounds = (lo, hi, lo, hi, -0.5, 0.5)

    def make(app):
        dx = (hi - lo) / n
        i, j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        x = (lo + (i + 0.5) * dx).ravel()
        y = (lo + (j + 0.5) * dx).ravel()
        cnt = len(x)
        b0 = 1.0 / math.sqrt(4.0 * math.pi)
        p = 5.0 / (12.0 * math.pi)
        rho = 25.0 / (36.0 * math.pi)
        m = rho * dx * dx
        return dict(x=x, y=y, z=np.zeros(cnt), u=-np.sin(2 * np.pi * (y - lo)), v=np.sin(2 * np.pi * (x - lo)),
                    w=np.zeros(cnt), rho=np.full(cnt, rho), h=np.full(cnt, app.hfact * math.sqrt(m / rho)),
                    m=np.full(cnt, m), e=np.full(cnt, p / ((app.gamma - 1.0) * rho)),
                    Bx=-b0 * np.sin(2 * np.pi * (y - lo)), By=b0 * np.sin(4 * np.pi * (x - lo)), Bz=np.zeros(cnt),
                    alpha1=np.zeros(cnt))

    cls = _square_app(ref, "OT2D", sim, bounds, make)
    app, domain = _make_app(ref, cls, sim)
    domain.periodic = (True, True, False)
    out["params"] = np.array(json.dumps(_params(sim, 2, domain)))
    _run(app, domain, 2, 3, out)


def case_shock2d(ref, out):
    sim = _case_config(ref, "mhdshock.toml", case=dict(nx=16))
    nxl, nyl = 16, 24
    dx = 0.5 / nxl
    ly = nyl * dx
    nxr = 6
    nyr = 8
    bounds = (-0.75, 0.75, 0.0, ly, -0.5, 0.5)

    def make(app):
        i, j = np.meshgrid(np.arange(nxl), np.arange(nyl), indexing="ij")
        xl = (-0.5 + (i + 0.5) * dx).ravel()
        yl = ((j + 0.5) * dx).ravel()
        dxr, dyr = 0.5 / nxr, ly / nyr
        i, j = np.meshgrid(np.arange(nxr), np.arange(nyr), indexing="ij")
        xr = ((i + 0.5) * dxr).ravel()
        yr = ((j + 0.5) * dyr).ravel()
        x = np.concatenate([xl, xr])
        y = np.concatenate([yl, yr])
        cnt = len(x)
        left = x < 0.0
        m = dx * dx
        rho = np.where(left, 1.0, 0.125)
        p = np.where(left, 1.0, 0.1)
        itype = np.where((x < -0.5 + 3 * dx) | (x > 0.5 - 3 * dxr), 3, 1).astype(np.int32)
        return dict(x=x, y=y, z=np.zeros(cnt), u=np.zeros(cnt), v=np.zeros(cnt), w=np.zeros(cnt), rho=rho,
                    h=app.hfact * np.sqrt(m / rho), m=np.full(cnt, m), e=p / ((app.gamma - 1.0) * rho),
                    Bx=np.full(cnt, 0.75), By=np.where(left, 1.0, -1.0), Bz=np.zeros(cnt), alpha1=np.zeros(cnt),
                    itype=itype)

    cls = _square_app(ref, "Shock2D", sim, bounds, make)
    app, domain = _make_app(ref, cls, sim)
    domain.periodic = (True, True, False)
    out["params"] = np.array(json.dumps(_params(sim, 2, domain)))
    _run(app, domain, 2, 3, out)


def case_blast3d(ref, out, n=8):
    sim = _case_config(ref, "mhdblast.toml", case=dict(nx=n), physics=dict(gamma=5.0 / 3.0))
    bounds = (-0.5, 0.5, -0.5, 0.5, -0.5, 0.5)

    def make(app):
        dx = 1.0 / n
        i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        x = (-0.5 + (i + 0.5) * dx).ravel()
        y = (-0.5 + (j + 0.5) * dx).ravel()
        z = (-0.5 + (k + 0.5) * dx).ravel()
        cnt = len(x)
        m = dx ** 3
        p = np.where(x * x + y * y + z * z < 0.3 ** 2, 10.0, 0.1)
        b = 1.0 / math.sqrt(2.0)
        return dict(x=x, y=y, z=z, u=np.zeros(cnt), v=np.zeros(cnt), w=np.zeros(cnt), rho=np.ones(cnt),
                    h=np.full(cnt, app.hfact * dx), m=np.full(cnt, m), e=p / (app.gamma - 1.0),
                    Bx=np.full(cnt, b), By=np.full(cnt, b), Bz=np.zeros(cnt), alpha1=np.zeros(cnt))

    cls = _square_app(ref, "Blast3D", sim, bounds, make)
    app, domain = _make_app(ref, cls, sim)
    out["params"] = np.array(json.dumps(_params(sim, 3, domain)))
    _run(app, domain, 3, 3, out)


def case_lattice(ref, out):
    """Points of the reference's close_packed_lattice (src/cases/lattice.py) for
    the bounds its case generators use."""
    import src.cases.lattice as lattice

    setups = [
        ((-0.5, 0.5, -0.5, 0.5, -4 * math.sqrt(6.0) / 16, 4 * math.sqrt(6.0) / 16), 1.0 / 16),  # orstang nx=16
        ((-0.5, 0.5, -0.5, 0.5, -0.5, 0.5), 1.0 / 12),  # mhdblast nx=12
        ((-1.5, 1.5, -0.75, 0.75, -0.75, 0.75), 3.0 / 24),  # alfven nx=24
        ((-0.5, 0.0, -0.65, 0.65, -0.61, 0.61), 0.0625),  # mhdshock left, nx=8
    ]
    for k, (b, s) in enumerate(setups):
        x, y, z = lattice.close_packed_lattice(b, s)
        out[f"set{k}/bounds"] = np.array(b)
        out[f"set{k}/spacing"] = np.array(s)
        out[f"set{k}/x"], out[f"set{k}/y"], out[f"set{k}/z"] = x, y, z
    out["n_sets"] = np.array(len(setups))


IC_FIELDS = "x y z u v w rho h m e Bx By Bz alpha1".split()
# the reference's remaining case generators at small nx: (config, module, class, nx)
IC_CASES = [
    ("mhdsine", "mhdsine", "MHDSine", 12),
    ("mhdwave", "mhdwave", "MHDWave", 16),
    ("mhdrotor", "mhdrotor", "MHDRotor", 16),
    ("mhdvortex", "mhdvortex", "MHDVortex", 12),
    ("jadvect", "jadvect", "CurrentLoopAdvection", 12),
    ("1jet", "jet", "JMXJets", 6),
    ("3jet", "jet", "JMXJets", 5),
    ("12jet", "jet", "JMXJets", 4),
]


def case_ref_ics(ref, out):
    """Initial particles of the reference's other case generators
    (src/cases/{mhdsine,mhdwave,mhdrotor,mhdvortex,jadvect,jet}.py), built by
    the reference's own classes from its own TOML files at a small nx."""
    import importlib

    cfgmod = ref["config"]
    for name, module, cls_name, nx in IC_CASES:
        mod = importlib.import_module(f"src.cases.{module}")
        cls = getattr(mod, cls_name)
        sim = cfgmod.load_config(os.path.join(REF, "configs", f"{name}.toml"), {name: cls.config_type})
        sim = replace(sim, case=replace(sim.case, nx=nx))
        app = cls(sim)
        pa = app.create_mhd_particles()[0]
        for k in IC_FIELDS:
            out[f"{name}/{k}"] = np.array(pa.properties[k], copy=True)
        out[f"{name}/nx"] = np.array(nx)
        print(f"  {name}: {pa.get_number_of_particles()} particles", flush=True)


CASES = {
    "ref_ics": case_ref_ics,
    "lattice": case_lattice,
    "ot2d": case_ot2d,
    "shock2d": case_shock2d,
    "blast3d": case_blast3d,
    "ref_orstang3d": case_ref_orstang3d,
}

if __name__ == "__main__":
    REF = sys.argv[1] if len(sys.argv) > 1 and sys.argv[1] not in CASES else os.environ.get("MHD_REFERENCE_ROOT")
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: make_golden.py /path/to/reference [case ...]  (or set MHD_REFERENCE_ROOT)")
    only = [a for a in sys.argv[1:] if a in CASES]
    ref = _import_reference(REF)
    for name, fn in CASES.items():
        if only and name not in only:
            continue
        print(name, flush=True)
        out = {}
        fn(ref, out)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
