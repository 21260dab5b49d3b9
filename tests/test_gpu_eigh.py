"""The preconditioner's FP64 eigen-decomposition on the device
(``msc_debug_symmetric_eigh``, the routine ``msc_plan_set_potential`` runs
for H0 = T + diag Re V_00) against LAPACK (numpy ``eigh``).

The reference diagonalises H0 with EISPACK rs (tred2 + tql2,
``diagsub.f90:5-262``) and its tests accept eigenvalues at rtol 3e-9
(``tests/test_fixed_example.py:449-454``); the bar here is FP64 round-off:
eigenvalues within 1e-12 ||H||, ||E^T E - I|| and ||H E - E diag(w)|| / ||H||
within 1e-12 (times a small multiple of n where noted).
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from multiscat_b200 import _native as nat
from multiscat_b200 import setup_arrays as sa
from multiscat_b200.workloads import cfg0_case, cfg1_case

pytestmark = pytest.mark.gpu


def _device_eigh(h: np.ndarray):
    lib = nat.load()
    h = np.ascontiguousarray(h, np.float64)
    n = h.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n))
    dp = ctypes.POINTER(ctypes.c_double)
    st = lib.msc_debug_symmetric_eigh(n, h.ctypes.data_as(dp), w.ctypes.data_as(dp),
                                      v.ctypes.data_as(dp))
    assert st == nat.MSC_OK, nat.last_error()
    return w, v


def _check(h, tol=1e-12):
    n = h.shape[0]
    w, v = _device_eigh(h)
    scale = max(np.abs(np.linalg.eigvalsh(h)).max(), 1e-300)
    want = np.linalg.eigvalsh(h)
    assert np.all(np.diff(w) >= 0.0)
    assert np.abs(w - want).max() <= tol * scale * max(1.0, n / 50)
    assert np.abs(v.T @ v - np.eye(n)).max() <= tol * max(1.0, n / 50)
    assert np.abs(h @ v - v * w[None, :]).max() <= tol * scale * max(1.0, n / 50)


@pytest.mark.parametrize("n", [2, 3, 17, 100, 150, 160, 161, 300, 550])
def test_random_symmetric_matches_lapack(n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    _check(a + a.T)


def test_structured_matrices():
    rng = np.random.default_rng(5)
    # diagonal: nothing to reduce, no rotations
    _check(np.diag(rng.standard_normal(40)))
    # two decoupled blocks: columns with nothing below the sub-diagonal
    a = rng.standard_normal((30, 30))
    a = a + a.T
    a[:15, 15:] = 0.0
    a[15:, :15] = 0.0
    _check(a)
    # repeated eigenvalues
    q, _ = np.linalg.qr(rng.standard_normal((24, 24)))
    _check(q @ np.diag(np.repeat([1.0, -2.0, 3.0], 8)) @ q.T)


@pytest.mark.parametrize("which", ["cfg0", "cfg1", "cfg4"])
def test_preconditioner_hamiltonians(which):
    """H0 = T + diag Re V_00 of the benchmark grids (n = 100, 200, 300)."""
    if which == "cfg0":
        case = cfg0_case()
        t, v00 = case.t, case.v[0, 0].real
    elif which == "cfg1":
        case = cfg1_case(nk=9)
        t, v00 = case.t, case.v[0, 0].real
    else:
        nodes, w = sa.lobatto_rule(-2.0, 14.0, 300)
        t = sa.kinetic_matrix(nodes, w)
        v00 = np.zeros(300)
    _check(t + np.diag(v00))
