"""MHDScheme: the reference scheme's configuration surface on the B200 path.

``get_equations`` returns the reference's ten groups (src/scheme.py:66-81)
built from ``src.equations``; ``compile_groups`` checks a group list against
that structure and extracts the kernel parameters -- the role PySPH's code
generator played.  A group list of any other shape is rejected: only this
scheme's fused kernels exist on the B200 path.
"""

from __future__ import annotations

from . import equations as E
from .integrator import MHDStep, PECIntegrator
from .particles import BASE_PROPERTIES, OUTPUT_PROPERTIES, PROPERTIES
from .solver import MHDSolver

MAX_DENSITY_ITERATIONS = 250  # src/scheme.py:28

KERNELS = ("cubic", "quintic", "wendland_c2", "wendland_c4", "wendland_c6", "gaussian", "super_gaussian")


class Group:
    """PySPH ``Group`` surface: equations plus iteration controls."""

    def __init__(self, equations, real=True, update_nnps=False, iterate=False, max_iterations=1, min_iterations=0,
                 **kw):
        self.equations = list(equations)
        self.real = real
        self.update_nnps = update_nnps
        self.iterate = iterate
        self.max_iterations = max_iterations
        self.min_iterations = min_iterations

    def __repr__(self):
        return f"Group({[type(e).__name__ for e in self.equations]}, iterate={self.iterate})"


# The group structure this build runs (class names per group, in order).
STRUCTURE = (
    ("DensityIteration",),
    ("SmoothingLengthRateFromDensityRelation", "DensityFromSmoothingLength"),
    ("IdealGasEOS",),
    ("CullenDehnenAlphaDiagnostics",),
    ("StrainDiagnostics", "MagneticStateReconstruction"),
    ("MHDAccelerations",),
    ("SmoothingLengthRateFromForceDivergence",),
    ("MagneticStressAccelerations",),
    ("MagneticStateRates",),
    ("EnergyLimiter", "DivBCorrection", "AdaptiveTimestep"),
)


def compile_groups(groups) -> dict:
    """Kernel parameters of a group list with the reference structure."""
    shape = tuple(tuple(type(e).__name__ for e in g.equations) for g in groups)
    if shape != STRUCTURE:
        raise NotImplementedError(
            f"the B200 path runs the reference MHD group list only; got {shape}")
    eq = {type(e).__name__: e for g in groups for e in g.equations}
    g1 = groups[0]
    d = eq["DensityIteration"]
    mu0s = {eq[n].mu0 for n in ("MHDAccelerations", "MagneticStressAccelerations", "MagneticStateRates",
                                "DivBCorrection")}
    if len(mu0s) != 1:
        raise ValueError("equations disagree on mu0")
    if eq["EnergyLimiter"].c_cour != eq["AdaptiveTimestep"].c_cour:
        raise ValueError("equations disagree on the timestep factor")
    return dict(
        hfact=d.k, dim=d.dim, iterate=not d.iterate_only_once and g1.iterate,
        min_iter=g1.min_iterations if g1.iterate else 0, max_iter=g1.max_iterations if g1.iterate else 1,
        gamma=eq["IdealGasEOS"].gamma, mu0=mu0s.pop(), av=eq["MHDAccelerations"].artificial_viscosity,
        ac=eq["MHDAccelerations"].artificial_thermal_conductivity,
        ar=eq["MagneticStateRates"].artificial_magnetic_dissipation,
        clean_speed=eq["MagneticStateRates"].cleaning_speed_factor,
        clean_damp=eq["MagneticStateRates"].cleaning_damping_factor,
        timestep_factor=eq["AdaptiveTimestep"].c_cour / E.COURANT_FACTOR,
    )


class MHDScheme:
    """src/scheme.py:31-81, with ``numerics.dim`` (default 3) as an extension."""

    def __init__(self, config):
        self.gamma = config.physics.gamma
        self.mu0 = config.physics.mu0
        self.kernel_name = config.numerics.kernel
        self.density = config.numerics.density
        self.hfact = config.numerics.hfact
        self.artificial_viscosity = config.physics.artificial_viscosity
        self.artificial_thermal_conductivity = config.physics.artificial_thermal_conductivity
        self.artificial_magnetic_dissipation = config.physics.artificial_magnetic_dissipation
        self.cleaning_speed_factor = config.numerics.cleaning_speed_factor
        self.cleaning_damping_factor = config.numerics.cleaning_damping_factor
        self.timestep_factor = config.solver.timestep_factor
        self.dim = getattr(config.numerics, "dim", None) or 3
        self.alpha_min = getattr(config.physics, "alpha_min", None)
        self.alpha_max = getattr(config.physics, "alpha_max", None)
        self.precision = getattr(config.execution, "precision", None) or "fp64"
        self.solver = None

    def configure_solver(self, **kw):
        if self.kernel_name not in KERNELS:
            raise KeyError(self.kernel_name)
        integrator = PECIntegrator(fluid=MHDStep(self.gamma))
        self.solver = MHDSolver(dim=self.dim, integrator=integrator, kernel=self.kernel_name, **kw)

    def setup_properties(self, particle):
        # Every reference property already exists on a src.particle_array.ParticleArray.
        names = set(particle.properties)
        for p in BASE_PROPERTIES + PROPERTIES:
            n = p["name"] if isinstance(p, dict) else p
            if n not in names:
                raise KeyError(f"particle array lacks property {n}")
        particle.output_arrays = list(OUTPUT_PROPERTIES)

    def get_equations(self):
        sources = ["fluid"]
        dim = self.dim
        iterate = self.density == "iterate"
        density = E.DensityIteration(dest="fluid", sources=sources, k=self.hfact, dim=dim,
                                     iterate_only_once=not iterate)
        return [
            Group([density], update_nnps=True, iterate=iterate, min_iterations=2 if iterate else 0,
                  max_iterations=MAX_DENSITY_ITERATIONS if iterate else 1),
            Group([E.SmoothingLengthRateFromDensityRelation(dest="fluid", sources=None, k=self.hfact, dim=dim),
                   E.DensityFromSmoothingLength(dest="fluid", sources=None, k=self.hfact, dim=dim)]),
            Group([E.IdealGasEOS(dest="fluid", sources=None, gamma=self.gamma)]),
            Group([E.CullenDehnenAlphaDiagnostics(dest="fluid", sources=sources)]),
            Group([E.StrainDiagnostics(dest="fluid", sources=None), E.MagneticStateReconstruction(dest="fluid",
                                                                                                 sources=None)]),
            Group([E.MHDAccelerations(dest="fluid", sources=sources, mu0=self.mu0,
                                      artificial_viscosity=self.artificial_viscosity,
                                      artificial_thermal_conductivity=self.artificial_thermal_conductivity)]),
            Group([E.SmoothingLengthRateFromForceDivergence(dest="fluid", sources=None, dim=dim)]),
            Group([E.MagneticStressAccelerations(dest="fluid", sources=sources, mu0=self.mu0)]),
            Group([E.MagneticStateRates(dest="fluid", sources=sources, mu0=self.mu0,
                                        artificial_magnetic_dissipation=self.artificial_magnetic_dissipation,
                                        cleaning_speed_factor=self.cleaning_speed_factor,
                                        cleaning_damping_factor=self.cleaning_damping_factor)]),
            Group([E.EnergyLimiter(dest="fluid", sources=None, timestep_factor=self.timestep_factor),
                   E.DivBCorrection(dest="fluid", sources=None, mu0=self.mu0),
                   E.AdaptiveTimestep(dest="fluid", sources=None, timestep_factor=self.timestep_factor)]),
        ]

    def kernel_params(self, domain, tf) -> dict:
        """Flat parameter dict for ``src.engine.params_from_dict``."""
        p = compile_groups(self.get_equations())
        p.update(kernel=self.kernel_name, tf=tf, lo=list(domain.lo), hi=list(domain.hi),
                 periodic=list(domain.periodic), density="iterate" if p.pop("iterate") else "single",
                 alpha_min=0.0 if self.alpha_min is None else self.alpha_min,
                 alpha_max=1.0 if self.alpha_max is None else self.alpha_max, precision=self.precision)
        p.pop("min_iter")
        p.pop("max_iter")
        return p
