"""The 14 equations of the reference scheme, as parameter carriers.

Class names, constructor arguments and module constants are those of the
reference's ``src/equations.py``; a group list built from them (by
``MHDScheme.get_equations``) is what ``src.scheme.compile_groups`` recognises
and runs as the fused sm_100a kernels.  The arithmetic of every class lives
in the CUDA sources: ``DensityIteration`` in ``csrc/mhd_pairs.cu``
(``k_density_pass``); ``DensityFromSmoothingLength``, ``IdealGasEOS`` and
``MagneticStateReconstruction`` in the force prologue and every other
equation of groups G4-G10 in the force pass (``csrc/mhd_force.cu``); the
integrator stages in ``csrc/mhd_integrate.cu``.  Each class below names the
kernel stage that executes it.
"""

DENSITY_TOLERANCE = 1.0e-4  # src/equations.py:6
COURANT_FACTOR = 0.3  # src/equations.py:7
FORCE_FACTOR = 0.25  # src/equations.py:8
PAIR_DISTANCE_EPSILON = 1.0e-12  # src/equations.py:9
INTERACTION_DISTANCE_EPSILON = 1.0e-8  # src/equations.py:10
FLOAT_TINY = 2.2250738585072014e-308  # src/equations.py:11


class Equation:
    """Destination/source names plus parameters (PySPH ``Equation`` surface)."""

    kernel_stage = None

    def __init__(self, dest, sources):
        self.dest = dest
        self.sources = sources

    def converged(self):
        return 1.0

    def __repr__(self):
        kw = {k: v for k, v in vars(self).items() if k not in ("dest", "sources")}
        return f"{type(self).__name__}(dest={self.dest!r}, sources={self.sources!r}, {kw})"


class DensityIteration(Equation):
    """src/equations.py:14-94 -> k_density_pass (pair sums + Newton on h)."""

    kernel_stage = "density_pass"

    def __init__(self, dest, sources, *, k, dim, iterate_only_once):
        self.density_iterations = True
        self.iterate_only_once = iterate_only_once
        self.dim = dim
        self.k = k
        self.htol = DENSITY_TOLERANCE
        self.equation_has_converged = 1
        super().__init__(dest, sources)


class IdealGasEOS(Equation):
    """src/equations.py:97-106 -> k_force_prologue."""

    kernel_stage = "force_prologue"

    def __init__(self, dest, sources, gamma):
        self.gamma = gamma
        self.gamma1 = gamma - 1.0
        super().__init__(dest, sources)


class DensityFromSmoothingLength(Equation):
    """src/equations.py:109-118 -> k_force_prologue."""

    kernel_stage = "force_prologue"

    def __init__(self, dest, sources, k, dim):
        self.k = k
        self.dim = dim
        super().__init__(dest, sources)


class SmoothingLengthRateFromDensityRelation(Equation):
    """src/equations.py:121-130; its ``ah`` is overwritten by
    SmoothingLengthRateFromForceDivergence, so no kernel writes it."""

    kernel_stage = "dead"

    def __init__(self, dest, sources, k, dim):
        self.k = k
        self.dim = dim
        super().__init__(dest, sources)


class SmoothingLengthRateFromForceDivergence(Equation):
    """src/equations.py:133-140 -> k_force_pass epilogue."""

    kernel_stage = "force_epilogue"

    def __init__(self, dest, sources, dim):
        self.dim1 = 1.0 / dim
        super().__init__(dest, sources)


class MagneticStressAccelerations(Equation):
    """src/equations.py:143-195 -> k_force_pass pair loop."""

    kernel_stage = "force_pass"

    def __init__(self, dest, sources, mu0):
        self.mu0 = mu0
        super().__init__(dest, sources)


class MHDAccelerations(Equation):
    """src/equations.py:198-280 -> k_force_pass pair loop + epilogue."""

    kernel_stage = "force_pass"

    def __init__(self, dest, sources, mu0, artificial_viscosity, artificial_thermal_conductivity):
        self.beta = 2.0
        self.mu0 = mu0
        self.artificial_viscosity = artificial_viscosity
        self.artificial_thermal_conductivity = artificial_thermal_conductivity
        super().__init__(dest, sources)


class CullenDehnenAlphaDiagnostics(Equation):
    """src/equations.py:283-429 -> k_force_pass (moments) + epilogue (alpha_loc)."""

    kernel_stage = "force_pass"

    def __init__(self, dest, sources):
        super().__init__(dest, sources)


class StrainDiagnostics(Equation):
    """src/equations.py:432-471 -> k_force_pass epilogue (written when the
    ``dvdx_*`` arrays are requested)."""

    kernel_stage = "force_epilogue"


class MagneticStateReconstruction(Equation):
    """src/equations.py:474-485 -> k_force_prologue."""

    kernel_stage = "force_prologue"


class MagneticStateRates(Equation):
    """src/equations.py:488-567 -> k_force_pass pair loop + epilogue."""

    kernel_stage = "force_pass"

    def __init__(self, dest, sources, mu0, artificial_magnetic_dissipation, cleaning_speed_factor,
                 cleaning_damping_factor):
        super().__init__(dest, sources)
        self.mu0 = mu0
        self.artificial_magnetic_dissipation = artificial_magnetic_dissipation
        self.cleaning_speed_factor = cleaning_speed_factor
        self.cleaning_damping_factor = cleaning_damping_factor
        self.cleaning_active = float(cleaning_speed_factor > 0.0)


class AdaptiveTimestep(Equation):
    """src/equations.py:570-585 -> k_force_pass epilogue."""

    kernel_stage = "force_epilogue"

    def __init__(self, dest, sources, timestep_factor):
        self.c_cour = timestep_factor * COURANT_FACTOR
        self.c_force = timestep_factor * FORCE_FACTOR
        self.bignumber = 1.0e29
        super().__init__(dest, sources)


class EnergyLimiter(Equation):
    """src/equations.py:588-598 -> k_force_pass epilogue."""

    kernel_stage = "force_epilogue"

    def __init__(self, dest, sources, timestep_factor):
        self.c_cour = timestep_factor * COURANT_FACTOR
        super().__init__(dest, sources)


class DivBCorrection(Equation):
    """src/equations.py:601-624 -> k_force_pass epilogue."""

    kernel_stage = "force_epilogue"

    def __init__(self, dest, sources, mu0):
        self.mu0 = mu0
        super().__init__(dest, sources)
