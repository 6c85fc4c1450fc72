"""CPU oracle for the SPMHD hot path -- test infrastructure only.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only as the checker or the timed
CPU baseline.  The product (``pysph-mhd_b200``) never imports it and has no
CPU fallback.

``mhd_oracle.c`` is an FP64 restatement of ``src/equations.py`` and
``src/integrator.py``; this module loads it through ctypes and mirrors, in
Python, the reference's warm-up (``src/application.py:99-132``), initial
timestep (``src/application.py:134-147``) and time loop
(``src/solver.py:22-77``).

Parity status: pinned against fixtures produced by executing the reference's
own equation, integrator, scheme, warm-up and solver code on small cases
(``tests/golden/make_golden.py``); the PySPH layer below that code (kernels,
neighbour rule, group iteration, PEC order, timestep rule) is a documented
restatement, since PySPH itself is not available.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "mhd_oracle.c")
LIB = os.path.join(HERE, "libmhd_oracle.so")

KERNELS = {"cubic": 0, "quintic": 1, "wendland_c2": 2, "wendland_c4": 3, "wendland_c6": 4, "gaussian": 5,
           "super_gaussian": 6}

COURANT_FACTOR = 0.3
FORCE_FACTOR = 0.25
MAX_DENSITY_ITERATIONS = 250


def build(force=False):
    """Compile the oracle (gcc, OpenMP, no FP contraction)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"]
    subprocess.check_call(cmd)
    return LIB


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("kernel", ctypes.c_int),
        ("iterate", ctypes.c_int),
        ("min_iter", ctypes.c_int),
        ("max_iter", ctypes.c_int),
        ("exact_order", ctypes.c_int),
        ("nthreads", ctypes.c_int),
        ("periodic", ctypes.c_int * 3),
        ("hfact", ctypes.c_double),
        ("gamma", ctypes.c_double),
        ("mu0", ctypes.c_double),
        ("av", ctypes.c_double),
        ("ac", ctypes.c_double),
        ("ar", ctypes.c_double),
        ("clean_speed", ctypes.c_double),
        ("clean_damp", ctypes.c_double),
        ("timestep_factor", ctypes.c_double),
        ("alpha_min", ctypes.c_double),
        ("alpha_max", ctypes.c_double),
        ("lo", ctypes.c_double * 3),
        ("hi", ctypes.c_double * 3),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build() if not os.path.exists(LIB) else LIB
        _lib = ctypes.CDLL(path)
        _lib.oracle_prop_name.restype = ctypes.c_char_p
        _lib.oracle_rhs.restype = ctypes.c_int
        _lib.oracle_step.restype = ctypes.c_int
        _lib.oracle_step.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p),
                                     ctypes.c_void_p, ctypes.c_double]
        _lib.oracle_rhs.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.c_void_p]
        _lib.oracle_neighbour_counts.restype = ctypes.c_int
        _lib.oracle_neighbour_counts.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int64,
                                                 ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]
        for fn in (_lib.oracle_predict, _lib.oracle_correct):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(OracleParams), ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p),
                           ctypes.c_void_p, ctypes.c_double]
        _lib.oracle_min_dt.restype = ctypes.c_double
        _lib.oracle_min_dt.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_void_p)]
    return _lib


def prop_names():
    L = lib()
    return [L.oracle_prop_name(i).decode() for i in range(L.oracle_nprops())]


def make_params(p: dict, exact_order=True, nthreads=0) -> OracleParams:
    """``p`` uses the keys of the fixture ``params`` record."""
    o = OracleParams()
    o.dim = int(p["dim"])
    o.kernel = KERNELS[p["kernel"]]
    o.iterate = 1 if p.get("density", "iterate") == "iterate" else 0
    o.min_iter = 2
    o.max_iter = MAX_DENSITY_ITERATIONS
    o.exact_order = 1 if exact_order else 0
    o.nthreads = nthreads
    for a in range(3):
        o.periodic[a] = 1 if p["periodic"][a] else 0
        o.lo[a] = p["lo"][a]
        o.hi[a] = p["hi"][a]
    o.hfact = p["hfact"]
    o.gamma = p["gamma"]
    o.mu0 = p["mu0"]
    o.av = p["av"]
    o.ac = p["ac"]
    o.ar = p["ar"]
    o.clean_speed = p["clean_speed"]
    o.clean_damp = p["clean_damp"]
    o.timestep_factor = p["timestep_factor"]
    o.alpha_min = p.get("alpha_min", 0.0)
    o.alpha_max = p.get("alpha_max", 1.0)
    return o


class State:
    """All reference property arrays (FP64, contiguous) plus int32 ``itype``."""

    def __init__(self, arrays: dict):
        n = len(arrays["x"])
        self.n = n
        self.names = prop_names()
        self.a = {}
        for k in self.names:
            v = arrays.get(k)
            self.a[k] = np.ascontiguousarray(v, dtype=np.float64).copy() if v is not None else np.zeros(n)
        self.itype = np.ascontiguousarray(arrays.get("itype", np.ones(n)), dtype=np.int32).copy()
        self.gid = np.asarray(arrays.get("gid", np.arange(n)), dtype=np.float64).copy()
        self._ptrs = (ctypes.c_void_p * len(self.names))(*[self.a[k].ctypes.data for k in self.names])

    def __getitem__(self, k):
        if k == "itype":
            return self.itype
        if k == "gid":
            return self.gid
        return self.a[k]


class Oracle:
    def __init__(self, params: dict, exact_order=True, nthreads=0):
        self.p = params
        self.cp = make_params(params, exact_order, nthreads)
        self.density_passes = []

    def rhs(self, s: State):
        k = lib().oracle_rhs(ctypes.byref(self.cp), s.n, s._ptrs, s.itype.ctypes.data)
        self.density_passes.append(k)
        return k

    def step(self, s: State, dt: float):
        k = lib().oracle_step(ctypes.byref(self.cp), s.n, s._ptrs, s.itype.ctypes.data, float(dt))
        self.density_passes.append(k)
        return k

    def predict(self, s: State, dt: float):
        """MHDStep.initialize + stage1 + wrap: the half of one_timestep before its RHS."""
        lib().oracle_predict(ctypes.byref(self.cp), s.n, s._ptrs, s.itype.ctypes.data, float(dt))

    def correct(self, s: State, dt: float):
        """MHDStep.stage2 + wrap: the half of one_timestep after its RHS."""
        lib().oracle_correct(ctypes.byref(self.cp), s.n, s._ptrs, s.itype.ctypes.data, float(dt))

    def min_dt(self, s: State):
        return lib().oracle_min_dt(s.n, s._ptrs)

    def neighbour_counts(self, s: State) -> np.ndarray:
        """Per-particle neighbour counts (exact rule, self included) from the
        oracle's own cell search with the current h."""
        out = np.zeros(s.n, dtype=np.int32)
        lib().oracle_neighbour_counts(ctypes.byref(self.cp), s.n, s._ptrs, out.ctypes.data_as(ctypes.c_void_p))
        return out

    # --- src/application.py:99-108 ---
    @staticmethod
    def sync_initial_mhd_state(s: State):
        s["Bevolx"][:] = s["Bx"] / s["rho"]
        s["Bevoly"][:] = s["By"] / s["rho"]
        s["Bevolz"][:] = s["Bz"] / s["rho"]
        s["psi"][:] = 0.0
        for pred, cur in (("Bevolxpred", "Bevolx"), ("Bevolypred", "Bevoly"), ("Bevolzpred", "Bevolz"),
                          ("psipred", "psi"), ("upred", "u"), ("vpred", "v"), ("wpred", "w"), ("epred", "e")):
            s[pred][:] = s[cur]

    # --- src/application.py:110-132 ---
    def warmup(self, s: State):
        b0 = (s["Bx"].copy(), s["By"].copy(), s["Bz"].copy())
        s["h0"][:] = s["h"]
        self.sync_initial_mhd_state(s)
        self.rhs(s)
        if not np.all(s["converged"] == 1):
            raise RuntimeError("density iteration did not converge in warm-up")
        s["Bx"][:], s["By"][:], s["Bz"][:] = b0
        s["h0"][:] = s["h"]
        self.sync_initial_mhd_state(s)
        for _ in range(2):
            self.rhs(s)
        if not np.all(s["converged"] == 1):
            raise RuntimeError("density iteration did not converge in warm-up")

    # --- src/application.py:134-147 ---
    def initial_dt(self, s: State):
        tf = self.p["timestep_factor"]
        force = np.sqrt(s["au"] * s["au"] + s["av"] * s["av"] + s["aw"] * s["aw"])
        if not np.all(s["dt_cfl"] > 0.0):
            raise RuntimeError("dt_cfl must be positive")
        cands = [float(np.min(tf * COURANT_FACTOR * s["h"] / s["dt_cfl"]))]
        mask = force > 0.0
        if np.any(mask):
            cands.append(float(np.min(tf * FORCE_FACTOR * np.sqrt(s["h"][mask] / force[mask]))))
        dt = min(cands)
        if not dt > 0.0:
            raise RuntimeError("dt must be positive")
        return dt

    # --- src/solver.py:22-77 with the adaptive rule min(dt_adapt), clipped to tf ---
    def run(self, s: State, n_steps: int, tf: float = 1e30, fixed_dt=None, callback=None):
        t = 0.0
        dt = self._timestep(s, t, tf, fixed_dt)
        count = 0
        record = []
        while (tf - t) > 2.220446049250313e-16 * tf * max(count, 1) and count < n_steps:
            self.step(s, dt)
            record.append((t, dt))
            if callback is not None:
                callback(count + 1, s, t, dt)
            t += dt
            count += 1
            dt = self._timestep(s, t, tf, fixed_dt)
        return record

    def _timestep(self, s, t, tf, fixed_dt):
        dt = fixed_dt if fixed_dt is not None else self.min_dt(s)
        if t + dt > tf:
            dt = tf - t
        return dt
