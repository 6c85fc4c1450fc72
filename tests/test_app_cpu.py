"""Host-side layer on CPU: configs, lattice, cases, scheme compilation.

No GPU work: the case generators produce numpy arrays, the scheme's group
list is checked against the reference structure, and the TOML schema
accepts the reference's files and the benchmark configs.
"""

import glob
import os

import numpy as np
import pytest

from golden_io import GOLDEN

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")
# the reference checkout, when present (development machines only): its
# configs/*.toml must load unchanged
REFERENCE_CONFIGS = os.path.join(os.environ.get("MHD_REFERENCE_ROOT", ""), "configs")


def test_close_packed_lattice_matches_reference_function():
    from src.cases.lattice import close_packed_lattice

    d = np.load(os.path.join(GOLDEN, "lattice.npz"))
    for k in range(int(d["n_sets"])):
        x, y, z = close_packed_lattice(tuple(d[f"set{k}/bounds"]), float(d[f"set{k}/spacing"]))
        np.testing.assert_array_equal(x, d[f"set{k}/x"])
        np.testing.assert_array_equal(y, d[f"set{k}/y"])
        np.testing.assert_array_equal(z, d[f"set{k}/z"])


def test_benchmark_configs_load_and_build_cases():
    from src.run import CASES
    from src.config import load_config

    types = {n: a.config_type for n, a in CASES.items()}
    sizes = {}
    for path in sorted(glob.glob(os.path.join(PKG, "configs", "*.toml"))):
        cfg = load_config(path, types)
        app = CASES[cfg.case.name](cfg)
        arrays = app.create_mhd_particles()
        sizes[cfg.case.name] = len(arrays["x"])
        assert np.all(np.isfinite(arrays["e"])) and np.all(arrays["h"] > 0)
    assert sizes["orstang2d"] == 128 * 128
    assert sizes["mhdblast3d"] == 128 ** 3
    assert sizes["alfven2d"] == 64 * 128
    assert 294_000 < sizes["mhdshock2d"] < 296_000  # 4096 x 128 left + 8:1 right


@pytest.mark.skipif(not os.environ.get("MHD_REFERENCE_ROOT") or not os.path.isdir(REFERENCE_CONFIGS),
                    reason="MHD_REFERENCE_ROOT does not name a reference checkout")
def test_reference_toml_files_load_unchanged():
    from src.config import load_config
    from src.run import CASES

    types = {n: a.config_type for n, a in CASES.items()}
    for path in sorted(glob.glob(os.path.join(REFERENCE_CONFIGS, "*.toml"))):
        cfg = load_config(path, types)
        assert cfg.numerics.dim is None and cfg.execution.precision is None


IC_FIELDS = "x y z u v w rho h m e Bx By Bz alpha1".split()


@pytest.mark.parametrize("name", ["mhdsine", "mhdwave", "mhdrotor", "mhdvortex", "jadvect", "1jet", "3jet", "12jet"])
def test_case_generators_match_reference_fixtures(name):
    # the fixtures hold what the reference's own generators build from its
    # own TOML files at a small nx (tests/golden/make_golden.py, ref_ics)
    from dataclasses import replace

    from src.config import load_config
    from src.run import CASES

    d = np.load(os.path.join(GOLDEN, "ref_ics.npz"))
    cfg = load_config(os.path.join(PKG, "configs", f"{name}.toml"), {k: v.config_type for k, v in CASES.items()})
    cfg = replace(cfg, case=replace(cfg.case, nx=int(d[f"{name}/nx"])))
    got = CASES[name](cfg).create_mhd_particles()
    for k in IC_FIELDS:
        ref = d[f"{name}/{k}"]
        assert got[k].shape == ref.shape, f"{name} {k}"
        scale = max(float(np.abs(ref).max()), 1e-300)
        np.testing.assert_allclose(got[k], ref, rtol=1e-13, atol=1e-13 * scale, err_msg=f"{name} {k}")


def test_scheme_groups_compile_to_kernel_parameters():
    from src.config import load_config
    from src.run import CASES
    from src.scheme import MHDScheme, compile_groups

    types = {n: a.config_type for n, a in CASES.items()}
    cfg = load_config(os.path.join(PKG, "configs", "mhdblast3d.toml"), types)
    scheme = MHDScheme(cfg)
    groups = scheme.get_equations()
    assert [type(e).__name__ for g in groups for e in g.equations][:3] == [
        "DensityIteration", "SmoothingLengthRateFromDensityRelation", "DensityFromSmoothingLength"]
    p = compile_groups(groups)
    assert p["hfact"] == 1.2 and p["dim"] == 3 and p["iterate"] and p["min_iter"] == 2 and p["max_iter"] == 250
    assert p["gamma"] == cfg.physics.gamma and abs(p["timestep_factor"] - 1.0) < 1e-15
    with pytest.raises(NotImplementedError):
        compile_groups(groups[:5] + groups[6:])


def test_config_rejects_unknown_keys_and_bad_types(tmp_path):
    from src.config import SimulationConfig, load_config

    good = open(os.path.join(PKG, "configs", "orstang2d.toml")).read()
    bad1 = good.replace("nx = 128", "nx = 128\nbogus = 1")
    bad2 = good.replace("gamma = 1.6666666666666667", "gamma = 2")
    for k, text in enumerate((bad1, bad2)):
        p = tmp_path / f"c{k}.toml"
        p.write_text(text)
        with pytest.raises(ValueError):
            load_config(p, {"orstang2d": SimulationConfig})


def test_dump_layout_and_load_round_trip(tmp_path):
    # PySPH's version-2 npz layout (pickled particles / solver_data dicts)
    # plus plain top-level arrays; a detailed dump holds every property
    from src.particle_array import ParticleArray
    from src.particles import OUTPUT_PROPERTIES
    from src.solver import MHDSolver, load_output

    rng = np.random.default_rng(3)
    n = 50
    arrays = {k: rng.random(n) for k in ("x", "y", "z", "u", "rho", "h", "m", "e", "Bx", "au", "x0")}
    arrays["gid"] = rng.permutation(n).astype(np.float64)
    pa = ParticleArray("fluid", arrays, device="cpu")
    for detailed in (False, True):
        s = MHDSolver(output_directory=str(tmp_path / str(detailed)), fname="t", detailed_output=detailed)
        s.particles = [pa]
        s.t, s.dt, s.count = 0.25, 1e-3, 7
        path = s.dump_output()
        with np.load(path, allow_pickle=True) as d:
            assert int(d["version"]) == 2
            parts = d["particles"].item()
            assert list(parts) == ["fluid"] and parts["fluid"]["output_property_arrays"] == list(OUTPUT_PROPERTIES)
            assert d["solver_data"].item() == {"t": 0.25, "dt": 1e-3, "count": 7}
        got, sd = load_output(path)
        assert sd == {"t": 0.25, "dt": 1e-3, "count": 7}
        order = np.argsort(arrays["gid"])
        np.testing.assert_array_equal(got["x"], arrays["x"][order])
        assert ("au" in got) == detailed and ("x0" in got) == detailed
        assert set(OUTPUT_PROPERTIES) <= set(got)
