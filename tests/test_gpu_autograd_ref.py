"""The derivative forms against an FP64 autograd-traced step.

``oracle/autograd_step.py`` restates the warm-up and the literal PEC step in
PyTorch (CPU, float64, dense all-pairs) and lets torch.autograd take the
gradient; the library's forward-mode and adjoint gradients must match it.
"""

import math
import os
from dataclasses import replace

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import small_cases as sc_  # noqa: E402
from oracle.autograd_step import Step  # noqa: E402

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")


def _alfven_config(nx):
    from src.config import load_config
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "alfven2d.toml"), {k: v.config_type for k, v in CASES.items()})
    return replace(cfg, case=replace(cfg.case, nx=nx))


def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


def test_alfven_gradient_matches_autograd():
    from src.derivative import alfven_case, magnetic_energy_adjoint, magnetic_energy_and_gradient

    cfg = _alfven_config(12)
    steps = 2
    value, grad, dts = magnetic_energy_and_gradient(cfg, 0.1, 1.0, steps)
    ic, _, prm = alfven_case(cfg, 0.1, 1.0)
    amp = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    amax = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    phase = 2.0 * math.pi * _t(ic["x"])
    tic = {k: _t(v) for k, v in ic.items()}
    tic.update(v=amp * torch.sin(phase), w=amp * torch.cos(phase), By=amp * torch.sin(phase),
               Bz=amp * torch.cos(phase))
    loss = Step(dict(prm, density="single")).run(tic, amax, dts)
    ga, gm = torch.autograd.grad(loss, (amp, amax), allow_unused=True)
    assert abs(float(loss.detach()) - value) <= 1e-12 * abs(value)
    assert abs(float(ga) - grad[0]) <= 1e-9 * abs(grad[0]), (float(ga), grad[0])
    assert (gm is None or float(gm) == 0.0) and grad[1] == 0.0
    adj_value, adj_grad, _ = magnetic_energy_adjoint(cfg, 0.1, 1.0, steps, every=1, dts=dts)
    assert abs(adj_grad[0] - float(ga)) <= 1e-9 * abs(float(ga))


def test_blast_gradient_matches_autograd():
    from src.derivative import TangentEngine, TangentState
    from src.engine import params_from_dict

    ic, prm = sc_.blast_3d(6, "cubic", seed=5, alpha=(0.1, 0.6))
    prm = dict(prm, density="single")
    steps = 2
    te = TangentEngine(params_from_dict(prm), TangentState(dict(ic), {"e": [0.01 * ic["e"], None]}),
                       alpha_max_seed=[0.0, 1.0])
    te.warmup()
    te.run(steps)
    value, grad = te.magnetic_energy()
    dts = list(te.dts)
    te.close()
    th = torch.tensor(0.0, dtype=torch.float64, requires_grad=True)
    amax = torch.tensor(0.6, dtype=torch.float64, requires_grad=True)
    tic = {k: _t(v) for k, v in ic.items()}
    tic["e"] = tic["e"] * (1.0 + 0.01 * th)
    loss = Step(prm).run(tic, amax, dts)
    ge, gm = torch.autograd.grad(loss, (th, amax))
    assert abs(float(loss.detach()) - value) <= 1e-12 * abs(value)
    assert abs(float(ge) - grad[0]) <= 1e-9 * abs(grad[0]), (float(ge), grad[0])
    assert float(gm) != 0.0
    assert abs(float(gm) - grad[1]) <= 1e-8 * abs(float(gm)), (float(gm), grad[1])
