"""GPU test of the allocation-free operator entry point (collected last).

``msc_apply_operator_noalloc`` serves callers that cannot call cudaMalloc
(code inside another framework's memory pool, fixed device-memory budgets,
plug-ins that may only touch the buffers they are given): it computes
y = A x for one full-grid system with its working storage in a fixed
__device__ array of the library.  Here it is called straight through the
C-ABI, twice in a row, and checked against the plan-based entry point
``msc_debug_apply_operator`` at the tolerance the operator tests use.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from multiscat_b200 import ScatteringPlan, full_grid_system
from multiscat_b200 import _native as nat
from multiscat_b200.workloads import Case, cfg0_case

pytestmark = pytest.mark.gpu


def _call_noalloc(lib, case, x, y, stream):
    nkx, nky, nz = case.v.shape
    dev = x.device
    v = torch.as_tensor(np.ascontiguousarray(case.v), device=dev)
    t = torch.as_tensor(np.ascontiguousarray(case.t), device=dev)
    pkd = torch.as_tensor(np.ascontiguousarray(case.pkd.ravel()), device=dev)
    wc = torch.as_tensor(np.ascontiguousarray(np.asarray(case.wc).ravel()), device=dev)
    st = lib.msc_apply_operator_noalloc(nkx, nky, nz, ctypes.c_void_p(v.data_ptr()),
                                        ctypes.c_void_p(t.data_ptr()),
                                        ctypes.c_void_p(pkd.data_ptr()),
                                        ctypes.c_void_p(wc.data_ptr()),
                                        ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return st


def test_noalloc_operator_matches_plan_operator_twice():
    lib = nat.load()
    case = cfg0_case()
    rng = np.random.default_rng(21)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    plan = ScatteringPlan(case.v, case.t, [case.system()])
    for call in range(2):
        x_np = rng.standard_normal((121, 100)) + 1j * rng.standard_normal((121, 100))
        x = torch.as_tensor(x_np, device=dev)
        want = plan.apply_operator(x).cpu().numpy()
        y = torch.full_like(x, complex(float("nan"), float("nan")))
        st = _call_noalloc(lib, case, x, y, stream)
        assert st == nat.MSC_OK, nat.last_error()
        got = y.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-11, atol=1e-11 * np.abs(want).max(),
                                   err_msg=f"call {call}")
    plan.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = nat.load()
    dev = torch.device("cuda", 0)
    x = torch.zeros(8, dtype=torch.complex128, device=dev)
    # 45 x 45 channels x 1000 nodes needs far more than the fixed scratch
    st = lib.msc_apply_operator_noalloc(45, 45, 1000, ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(0))
    assert st == nat.MSC_ERR_DIMS
    assert "scratch" in nat.last_error()


def _asymmetric_case(nkx=5, nky=7, nz=12, seed=5):
    """A random complex potential on a 5 x 7 torus: no x <-> y or d <-> -d
    symmetry, so a swapped axis or a tap applied with the wrong sign in the
    neighbour table would change y."""
    rng = np.random.default_rng(seed)
    v = 0.3 * (rng.standard_normal((nkx, nky, nz)) + 1j * rng.standard_normal((nkx, nky, nz)))
    a = rng.standard_normal((nz, nz))
    t = a @ a.T + nz * np.eye(nz)
    pkd = rng.uniform(-2.0, 5.0, (nkx, nky))
    c = nkx * nky
    wa, wb, wc = (rng.standard_normal(c) + 1j * rng.standard_normal(c) for _ in range(3))
    return Case("asymmetric 5x7", v, t, pkd, wa, wb, wc, np.arange(nz, dtype=float),
                np.ones(nz))


def test_noalloc_operator_matches_plan_on_an_asymmetric_torus():
    lib = nat.load()
    case = _asymmetric_case()
    rng = np.random.default_rng(22)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    plan = ScatteringPlan(case.v, case.t, [full_grid_system(case.pkd, case.wa, case.wb, case.wc)])
    for call in range(2):
        x_np = rng.standard_normal((35, 12)) + 1j * rng.standard_normal((35, 12))
        x = torch.as_tensor(x_np, device=dev)
        want = plan.apply_operator(x).cpu().numpy()
        y = torch.full_like(x, complex(float("nan"), float("nan")))
        st = _call_noalloc(lib, case, x, y, stream)
        assert st == nat.MSC_OK, nat.last_error()
        np.testing.assert_allclose(y.cpu().numpy(), want, rtol=1e-11,
                                   atol=1e-11 * np.abs(want).max(), err_msg=f"call {call}")
    plan.close()


def test_noalloc_rejects_a_nonfinite_potential():
    lib = nat.load()
    case = _asymmetric_case()
    case.v[2, 3, 4] = complex(float("nan"), 0.0)
    dev = torch.device("cuda", 0)
    x = torch.zeros((35, 12), dtype=torch.complex128, device=dev)
    y = torch.zeros_like(x)
    st = _call_noalloc(lib, case, x, y, torch.cuda.current_stream(dev).cuda_stream)
    assert st == nat.MSC_ERR_NONFINITE
    assert "non-finite" in nat.last_error()
