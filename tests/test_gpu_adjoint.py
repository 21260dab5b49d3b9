"""Adjoint differentiation on the GPU: A^H identity, gradients against central
finite differences of this solver and of the oracle (cfg3), batched sums,
mixed precision.  Gradient convention: dL/dRe V + i dL/dIm V."""

from __future__ import annotations

import json
import pathlib

import numpy as np
import pytest
import torch

from multiscat_b200 import ScatteringPlan
from multiscat_b200.adjoint import scattering_intensities
from multiscat_b200.workloads import cfg0_case, cfg2_batch, cfg3_problem

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
GRAD_RTOL = 1e-5          # adjoint vs central finite differences (relative)


def _cdot(a: torch.Tensor, b: torch.Tensor) -> complex:
    return complex((a.conj() * b).sum().item())


def _loss(v, case, systems, weights, **kw) -> float:
    plan = ScatteringPlan(v, case.t, systems, **kw)
    res = plan.solve()
    out = float((torch.as_tensor(weights, device="cuda") * res.intensities).sum())
    plan.close()
    return out


def test_adjoint_operator_identity():
    """<y, A x> = <A^H y, x> on a non-Hermitian potential (complex, asymmetric taps)."""
    case = cfg0_case(nz=40)
    rng = np.random.default_rng(5)
    v = case.v.copy()
    v[1, 2] = (rng.normal(size=40) + 1j * rng.normal(size=40)) * 0.05   # no partner at (-1, -2)
    v[3, 0] += 1j * 0.02 * rng.normal(size=40)
    plan = ScatteringPlan(v, case.t, [case.system()])
    c, n = plan.total_rows, plan.nz
    x = torch.randn(c, n, dtype=torch.complex128, device="cuda")
    y = torch.randn(c, n, dtype=torch.complex128, device="cuda")
    ax = plan.apply_operator(x)
    plan.set_adjoint(True)
    ahy = plan.apply_operator(y)
    plan.set_adjoint(False)
    lhs, rhs = _cdot(y, ax), _cdot(ahy, x)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)
    # back in forward mode the operator is A again
    assert torch.allclose(plan.apply_operator(x), ax, rtol=0, atol=1e-13)
    plan.close()


def test_gradient_directional_fd_cfg0():
    """Re<grad, E> against (L(V + eps E) - L(V - eps E)) / 2 eps, E random on the taps."""
    case = cfg0_case(nz=60)
    system = case.system()
    rng = np.random.default_rng(1)
    weights = np.where(case.pkd.ravel() < 0, rng.uniform(0, 1, case.pkd.size), 0.0)
    vt = torch.tensor(case.v, dtype=torch.complex128, device="cuda", requires_grad=True)
    inten = scattering_intensities(vt, case.t, [system], rtol=1e-13)
    loss = (torch.as_tensor(weights, device="cuda") * inten).sum()
    loss.backward()
    grad = vt.grad.detach()
    # relative step 1e-5 on every nonzero element, in a random complex direction
    e = (rng.normal(size=case.v.shape) + 1j * rng.normal(size=case.v.shape)) * np.abs(case.v)
    e[0, 0] = e[0, 0].real                       # only Re V_0 enters
    eps = 1e-5
    lp = _loss(case.v + eps * e, case, [system], weights, rtol=1e-13)
    lm = _loss(case.v - eps * e, case, [system], weights, rtol=1e-13)
    fd = (lp - lm) / (2 * eps)
    ad = float(torch.real((grad.conj() * torch.as_tensor(e, device="cuda")).sum()))
    assert abs(ad - fd) <= GRAD_RTOL * abs(fd), (ad, fd)


@pytest.fixture(scope="module")
def cfg3():
    return cfg3_problem()


@pytest.fixture(scope="module")
def cfg3_grads(cfg3):
    """Adjoint gradients of L w.r.t. (D, alpha, h) and V (FP64, rtol 1e-13)."""
    p = {k: torch.tensor(v, dtype=torch.float64, device="cuda", requires_grad=True)
         for k, v in cfg3.params.items()}
    v = cfg3.potential(p["depth"], p["alpha"], p["h"], device="cuda")
    v.retain_grad()
    inten = scattering_intensities(v, cfg3.case.t, [cfg3.case.system()], rtol=1e-13)
    loss = (torch.as_tensor(cfg3.weights, device="cuda") * inten).sum()
    loss.backward()
    return {"loss": loss.item(), "depth": float(p["depth"].grad), "alpha": float(p["alpha"].grad),
            "h": float(p["h"].grad), "v": v.grad.detach().cpu().numpy()}


def test_cfg3_parameter_gradients_vs_own_fd(cfg3, cfg3_grads):
    sysm = [cfg3.case.system()]
    for k in ("depth", "alpha", "h"):
        step = 1e-5 * cfg3.params[k]
        vals = []
        for sgn in (1, -1):
            q = dict(cfg3.params)
            q[k] = q[k] + sgn * step
            v = cfg3.potential(q["depth"], q["alpha"], q["h"]).numpy()
            vals.append(_loss(v, cfg3.case, sysm, cfg3.weights, rtol=1e-13))
        fd = (vals[0] - vals[1]) / (2 * step)
        assert abs(cfg3_grads[k] - fd) <= GRAD_RTOL * abs(fd), (k, cfg3_grads[k], fd)


def _oracle_fd():
    path = GOLDEN / "oracle_cfg3_fd.json"
    if not path.exists():
        pytest.skip("oracle_cfg3_fd.json not generated")
    return json.loads(path.read_text())


def test_cfg3_parameter_gradients_vs_oracle_fd(cfg3_grads):
    ref = _oracle_fd()
    assert ref["all_converged"]
    assert abs(cfg3_grads["loss"] - ref["loss"]) <= 1e-9
    for k, rec in ref["params"].items():
        assert abs(cfg3_grads[k] - rec["dL"]) <= GRAD_RTOL * abs(rec["dL"]), (k, cfg3_grads[k], rec)


def test_cfg3_component_gradients_vs_oracle_fd(cfg3_grads):
    ref = _oracle_fd()
    g = cfg3_grads["v"]
    for rec in ref["components"]:
        val = g[rec["ix"], rec["iy"], rec["z"]]
        ad = val.real if rec["part"] == "re" else val.imag
        assert abs(ad - rec["dL"]) <= GRAD_RTOL * abs(rec["dL"]) + 1e-12, (rec, ad)


def test_mixed_precision_gradient_matches_fp64(cfg3, cfg3_grads):
    v = torch.tensor(cfg3.case.v, dtype=torch.complex128, device="cuda", requires_grad=True)
    inten = scattering_intensities(v, cfg3.case.t, [cfg3.case.system()], rtol=1e-12,
                                   precision="mixed")
    (torch.as_tensor(cfg3.weights, device="cuda") * inten).sum().backward()
    g = v.grad.detach().cpu().numpy()
    ref = cfg3_grads["v"]
    assert np.abs(g - ref).max() <= 1e-6 * np.abs(ref).max()


def test_batched_gradient_is_sum_of_single_system_gradients():
    case, systems = cfg2_batch(n_solves=3, seed=2)
    rng = np.random.default_rng(3)
    weights = [np.where(s.pkd < 0, rng.uniform(0, 1, s.pkd.size), 0.0) for s in systems]
    weights[1][:] = 0.0            # a system with a zero adjoint right-hand side
    v = torch.tensor(case.v, dtype=torch.complex128, device="cuda", requires_grad=True)
    inten = scattering_intensities(v, case.t, systems, rtol=1e-12)
    (torch.as_tensor(np.concatenate(weights), device="cuda") * inten).sum().backward()
    total = v.grad.detach().clone()
    acc = torch.zeros_like(total)
    for s, w in zip(systems, weights):
        vs = torch.tensor(case.v, dtype=torch.complex128, device="cuda", requires_grad=True)
        (torch.as_tensor(w, device="cuda") * scattering_intensities(vs, case.t, [s], rtol=1e-12)
         ).sum().backward()
        acc += vs.grad
    assert float((total - acc).abs().max()) <= 1e-9 * float(acc.abs().max())


def test_gradient_window_matches_full_torus():
    case = cfg0_case(nz=40)
    plan = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-12)
    res = plan.solve()
    w = torch.rand(plan.total_rows, dtype=torch.float64, device="cuda")
    lam = plan.solve_adjoint(res.psi, dl_dintensity=w).psi
    full = plan.potential_gradient(res.psi, lam)
    win = plan.potential_gradient(res.psi, lam, window=(2, 3))
    idx_x = [i % 11 for i in range(-2, 3)]
    idx_y = [i % 11 for i in range(-3, 4)]
    sub = full[idx_x][:, idx_y]
    assert torch.equal(win[idx_x][:, idx_y], sub)
    mask = torch.ones(11, 11, dtype=torch.bool, device="cuda")
    mask[np.ix_(idx_x, idx_y)] = False
    assert float(win[mask].abs().max()) == 0.0
    assert not plan.adjoint
    plan.close()
