"""B200 (sm_100a) SPMHD particle update with the reference's Python surface.

Module names follow the reference package (``src.scheme``, ``src.equations``,
``src.integrator``, ``src.particles``, ``src.solver``, ``src.application``,
``src.config``, ``src.cases``, ``src.run``); the hot path runs in
``libmhd_b200.so`` through ``src._abi``.
"""
