"""The reference's block Gauss-Seidel splitting A = L + U on the GPU.

- the lower block L = D + V^lower and its inverse (the forward sweep of
  ``solve_lower_block``, ``multiscat_gmres.f90:641-687``;
  ``_apply_lower_block`` / ``_apply_inverse_lower_block``,
  ``_scipy.py:262-297, 357-380``) against the oracle's sweep and a numpy
  restatement of L;
- the reference's state convention L psi (``_gmres.py:127``,
  ``_multiscat.py:63-99``) on the He-LiF golden case;
- the Gauss-Seidel preconditioner (and its Neumann order 1, the reference's
  default ``use_neumann_preconditioner=True``) in the solver, FP64 and mixed,
  against the oracle, and on the beam that stalls the block-diagonal FP32
  inner solve.

Tolerances: operators within 1e-10 relative of the CPU restatements (the
sweep runs through C channels in sequence); solves at the FP64 bar
max |Delta |S|^2| <= 1e-8 against the oracle, mixed vs FP64 <= 1e-8.
"""

from __future__ import annotations

import json
import pathlib

import numpy as np
import pytest
import torch

from multiscat_b200 import (OptimizationConfig, ScatteringPlan, full_grid_system,
                            get_scattering_matrix, get_scattering_matrix_from_state,
                            get_scattering_state)
from multiscat_b200.api import _reference_order_system, natural_arrays
from multiscat_b200.workloads import cfg0_case, cfg2_batch

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def _rand(shape, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def _numpy_lower(v, t, pkd, wc, ix, iy, x):
    """L x = D x + sum_{j < i} V[(G_i - G_j) mod] x_j in the given channel order
    (the reference's _apply_lower_block, _scipy.py:357-380)."""
    nkx, nky, _ = v.shape
    vv = v.copy()
    v00 = vv[0, 0].real.copy()
    vv[0, 0] = 0.0
    y = x @ t.T + (v00[None, :] + pkd[:, None]) * x
    y[:, -1] -= wc * x[:, -1]
    for i in range(len(ix)):
        for j in range(i):
            y[i] += vv[(ix[i] - ix[j]) % nkx, (iy[i] - iy[j]) % nky] * x[j]
    return y


def test_lower_block_sweep_matches_the_oracle_sweep():
    from oracle import solver as osol
    case = cfg0_case(nz=40)
    plan = ScatteringPlan(case.v, case.t, [case.system()])
    x = _rand((121, 40), 3)
    got = plan.solve_lower_block(torch.as_tensor(x, device="cuda")).cpu().numpy()
    want = osol.solve_lower(case.v, case.pkd, case.wc, case.t, x)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-10 * np.abs(want).max())
    back = plan.apply_lower_block(torch.as_tensor(got, device="cuda")).cpu().numpy()
    np.testing.assert_allclose(back, x, rtol=0, atol=1e-10 * np.abs(x).max())
    plan.close()


def test_apply_lower_block_in_the_reference_channel_order():
    case = cfg0_case(nz=30)
    sp = _reference_order_system(case_arrays(case), None)
    plan = ScatteringPlan(case.v, case.t, [sp])
    x = _rand((121, 30), 4)
    got = plan.apply_lower_block(torch.as_tensor(x, device="cuda")).cpu().numpy()
    want = _numpy_lower(case.v, case.t, sp.pkd, sp.wave_c, sp.channel_ix, sp.channel_iy, x)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.abs(want).max())
    plan.close()


def case_arrays(case):
    class A:
        pass
    a = A()
    a.pkd, a.wave_a, a.wave_b, a.wave_c = case.pkd, case.wa, case.wb, case.wc
    return a


def _wolken():
    from tests.test_gpu_solver import _read_wolken_golden, _wolken_condition
    return _wolken_condition(0.0), _read_wolken_golden()


def test_reference_state_is_lower_block_times_psi():
    cond, golden = _wolken()
    cfg = OptimizationConfig(precision=1e-7, max_iterations=1000)
    psi = get_scattering_state(cond, cfg, convention="psi")
    ref_state = get_scattering_state(cond, cfg)          # the reference's convention
    arr = natural_arrays(cond)
    sp = _reference_order_system(arr, None)
    rows = psi[sp.channel_ix, sp.channel_iy]
    want = _numpy_lower(arr.potential_values, arr.kinetic, sp.pkd, sp.wave_c, sp.channel_ix,
                        sp.channel_iy, rows)
    got = ref_state[sp.channel_ix, sp.channel_iy]
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-9 * np.abs(want).max())
    s_ref = get_scattering_matrix_from_state(ref_state, cond)
    np.testing.assert_allclose(s_ref.real, golden, rtol=0, atol=1e-5)
    np.testing.assert_allclose(s_ref.real, get_scattering_matrix(cond, cfg).real, rtol=0,
                               atol=1e-9)


@pytest.mark.parametrize("order", [0, 1])
def test_gauss_seidel_preconditioner_matches_oracle(order):
    golden = json.loads((GOLDEN / "oracle_cfg0.json").read_text())
    case = cfg0_case()
    plan = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-10, gauss_seidel=True,
                          preconditioner_order=order)
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    plan.close()
    assert res.status[0] == 0 and res.residual[0] <= 1e-10
    np.testing.assert_allclose(inten, golden["intensities"], rtol=0.0, atol=1e-8)
    assert abs(inten.sum() - 1.0) <= 1e-8
    # the reference's own operator: Gauss-Seidel with the Neumann factor takes
    # about the oracle's iteration count (restarts and the stop rule differ)
    if order == 1:
        assert res.iterations[0] <= golden["iterations"] + 6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gauss_seidel_batch_matches_block_jacobi(precision):
    case, systems = cfg2_batch(n_solves=12, seed=2)
    ref = ScatteringPlan(case.v, case.t, systems, rtol=1e-10)
    want = ref.solve().intensities.cpu().numpy()
    ref.close()
    plan = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision=precision,
                          gauss_seidel=True)
    res = plan.solve()
    plan.close()
    assert (res.status == 0).all()
    assert np.abs(res.intensities.cpu().numpy() - want).max() <= 1e-8


def test_gauss_seidel_converges_the_stalled_beam():
    want = json.loads((GOLDEN / "oracle_cfg2_stall.json").read_text())
    case, systems = cfg2_batch(n_solves=3, seed=1, nz=41)
    plan = ScatteringPlan(case.v, case.t, [systems[1]], rtol=1e-10, gauss_seidel=True)
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    plan.close()
    assert res.status[0] == 0 and res.iterations[0] <= 200, res.iterations
    assert np.abs(inten - np.array(want["intensities"])).max() <= 1e-8
