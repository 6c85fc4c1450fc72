"""Reverse mode (checkpointed adjoint) against forward mode.

Both differentiate the same map -- the warm-up (forward mode in both) and
`steps` literal PEC steps with frozen step sizes -- so the adjoint's
gradient must equal the tangent's to roundoff, for any checkpoint interval.
Forward mode is itself checked against central differences of the drop-in
path (test_gpu_tangent.py).
"""

import os
from dataclasses import replace

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import small_cases as sc_  # noqa: E402

pytestmark = pytest.mark.gpu

PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pysph-mhd_b200")


def _alfven_config(nx):
    from src.config import load_config
    from src.run import CASES

    cfg = load_config(os.path.join(PKG, "configs", "alfven2d.toml"), {k: v.config_type for k, v in CASES.items()})
    return replace(cfg, case=replace(cfg.case, nx=nx))


def _both(ic, prm, seeds, steps, every):
    """(loss, grad) by forward mode and by the adjoint on the same warm-up."""
    from src.derivative import AdjointEngine, TangentEngine, TangentState
    from src.engine import params_from_dict

    params = params_from_dict(dict(prm, density="single"))
    te = TangentEngine(params, TangentState(dict(ic), seeds), alpha_max_seed=[0.0, 1.0])
    te.warmup()
    ae = AdjointEngine(params, te.ts.n)
    values = {f: te.ts[f][:, 0].contiguous() for f in ae.fields}
    values["m"] = te.ts["m"][:, 0].contiguous()
    values["itype"] = te.ts["itype"]
    tan0 = torch.stack([te.ts[f][:, 1:].clone() for f in ae.fields])
    loss_a, used, cps = ae.forward(values, steps, [te.initial_dt()] + [-1.0] * (steps - 1), every)
    lam, dam = ae.backward(values, steps, used, every, cps)
    grad_a = torch.einsum("fn,fnd->d", lam, tan0).cpu().numpy()
    grad_a[1] += dam
    te.run(steps, used)
    loss_t, grad_t = te.magnetic_energy()
    ae.close()
    te.close()
    return (loss_a, grad_a), (loss_t, grad_t), used


def test_adjoint_equals_forward_mode_alfven():
    from src.derivative import alfven_case

    ic, seed, prm = alfven_case(_alfven_config(16), 0.1, 1.0)
    (la, ga), (lt, gt), _ = _both(ic, prm, seed, 12, 4)
    assert abs(la - lt) <= 1e-12 * abs(lt)
    assert abs(ga[0] - gt[0]) <= 1e-9 * abs(gt[0]), (ga, gt)
    assert ga[1] == 0.0 and gt[1] == 0.0


@pytest.mark.parametrize("every", [1, 5])
def test_adjoint_equals_forward_mode_blast(every):
    ic, prm = sc_.blast_3d(8, "cubic", seed=3, alpha=(0.1, 0.6))
    seeds = {"e": [0.01 * ic["e"], None], "x": [None, None]}
    (la, ga), (lt, gt), _ = _both(ic, prm, seeds, 7, every)
    assert abs(la - lt) <= 1e-12 * abs(lt)
    for d in range(2):
        assert gt[d] != 0.0
        assert abs(ga[d] - gt[d]) <= 1e-8 * abs(gt[d]), (d, ga, gt)


def test_autograd_function_gradient():
    from src.derivative import MagneticEnergy, magnetic_energy_and_gradient

    cfg = _alfven_config(16)
    a = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    am = torch.tensor(1.0, dtype=torch.float64, requires_grad=True)
    loss = MagneticEnergy.apply(a, am, cfg, 10, 4)
    loss.backward()
    value, grad, _ = magnetic_energy_and_gradient(cfg, 0.1, 1.0, 10)
    assert abs(float(loss.detach()) - value) <= 1e-12 * abs(value)
    assert abs(float(a.grad) - grad[0]) <= 1e-9 * abs(grad[0])
    assert float(am.grad) == grad[1] == 0.0


def test_hand_written_pair_vjp_equals_dual_jacobian(monkeypatch):
    # the reverse force-pair and Cullen-Dehnen pair passes by the
    # hand-written VJPs (default) and by contracting dual-number Jacobians
    # (MHD_ADJOINT_DUAL=1): every lambda of the initial state agrees to
    # roundoff
    from src.derivative import AdjointEngine, TangentEngine, TangentState
    from src.engine import params_from_dict

    ic, prm = sc_.blast_3d(8, "cubic", seed=5, alpha=(0.1, 0.6))
    params = params_from_dict(dict(prm, density="single"))
    te = TangentEngine(params, TangentState(dict(ic), {"e": [0.01 * ic["e"], None]}), alpha_max_seed=[0.0, 1.0])
    te.warmup()
    ae = AdjointEngine(params, te.ts.n)
    values = {f: te.ts[f][:, 0].contiguous() for f in ae.fields}
    values["m"] = te.ts["m"][:, 0].contiguous()
    values["itype"] = te.ts["itype"]
    steps, every = 5, 2
    _, used, cps = ae.forward(values, steps, [te.initial_dt()] + [-1.0] * (steps - 1), every)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("MHD_ADJOINT_DUAL", mode)
        lam, dam = ae.backward(values, steps, used, every, cps)
        out[mode] = (lam.clone(), dam)
    ae.close()
    te.close()
    a, b = out["0"][0], out["1"][0]
    assert float(torch.linalg.norm(b)) > 0.0
    for f in range(a.shape[0]):
        scale = max(float(torch.linalg.norm(b[f])), 1e-300)
        assert float(torch.linalg.norm(a[f] - b[f])) <= 1e-11 * max(scale, 1e-12 * float(torch.linalg.norm(b))), f
    assert abs(out["0"][1] - out["1"][1]) <= 1e-11 * max(abs(out["1"][1]), 1e-300)


def test_adjoint_beyond_small_cases():
    # 256 x 512 = 131,072 particles: the grid search has no size limit, and
    # above 65,536 particles the pair passes run as one slice
    from src.derivative import alfven_case

    ic, seed, prm = alfven_case(_alfven_config(256), 0.1, 1.0)
    assert len(ic["x"]) == 131072
    (la, ga), (lt, gt), _ = _both(ic, prm, seed, 4, 2)
    assert abs(la - lt) <= 1e-12 * abs(lt)
    assert abs(ga[0] - gt[0]) <= 1e-9 * abs(gt[0]), (ga, gt)
