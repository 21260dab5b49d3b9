"""CPU tests: the package's input builders against the oracle's restatement."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from multiscat_b200 import setup_arrays as sa
from oracle import inputs


@pytest.mark.parametrize("n", [2, 3, 10, 57, 100, 200, 550])
def test_lobatto_rule_matches_oracle(n):
    x, w = sa.lobatto_rule(-0.4, 1.7, n)
    xo, wo = inputs.lobatto_rule(-0.4, 1.7, n)
    np.testing.assert_allclose(x, xo, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(w, wo, rtol=1e-11, atol=1e-14)
    assert math.isclose(w.sum(), 2.1, rel_tol=1e-12)


@pytest.mark.parametrize("n", [5, 40, 120])
def test_kinetic_matrix_matches_oracle_and_is_exact_on_polynomials(n):
    x, w = sa.lobatto_rule(-1.0, 2.0, n)
    t = sa.kinetic_matrix(x, w)
    np.testing.assert_allclose(t, inputs.kinetic_matrix(x, w), rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(t, t.T, atol=1e-12 * np.abs(t).max())
    # <f|T|g> = int f' g' for polynomials of low degree (f = z, g = z^2)
    f = x * np.sqrt(w)
    g = x**2 * np.sqrt(w)
    exact = 2.0 ** 2 - (-1.0) ** 2   # int_{-1}^{2} 1 * 2z dz = z^2 |
    assert math.isclose(f @ t @ g, exact, rel_tol=1e-9)


def test_pkd_and_waves_match_oracle():
    fac = sa.natural_units_factor(sa.HE4_MASS)
    k = sa.momentum_from_angles(40.0, math.radians(25.0), math.radians(10.0), fac)
    a1 = np.array([3.16, 0.0])
    a2 = np.array([1.58, 3.16 * math.sqrt(3) / 2])
    pkd = sa.perpendicular_kinetic_difference(k, a1, a2, 9, 7)
    np.testing.assert_allclose(pkd, inputs.perpendicular_kinetic_difference(k, a1, a2, 9, 7),
                               rtol=1e-12, atol=1e-12)
    x, w = sa.lobatto_rule(-1.5, 10.0, 80)
    got = sa.waves(pkd, w, -1.5, 11.5)
    want = inputs.waves(pkd, w, -1.5, 11.5)
    for g, o in zip(got, want):
        np.testing.assert_allclose(g, o, rtol=1e-12, atol=1e-12)


def test_units_factor_he4():
    assert math.isclose(sa.natural_units_factor(sa.HE4_MASS), 1.91505, rel_tol=2e-5)
    assert math.isclose(sa.natural_units_factor(sa.HE4_MASS),
                        inputs.natural_units_factor(inputs.HE4_MASS_AMU * inputs.AMU), rel_tol=1e-8)


@pytest.mark.parametrize("hexagonal", [False, True])
def test_corrugated_morse_matches_oracle(hexagonal):
    x, _ = sa.lobatto_rule(-1.5, 10.0, 20)
    if hexagonal:
        a1 = np.array([3.16, 0.0])
        a2 = np.array([1.58, 3.16 * math.sqrt(3) / 2])
        xi = sa.hexagonal_xi(a1, a2, 0.2)
        b1, b2 = inputs.reciprocal_vectors(a1, a2)
        b3 = b1 + b2

        def xi_np(px, py):
            return (0.2 / 3) * (np.cos(b1[0] * px + b1[1] * py) + np.cos(b2[0] * px + b2[1] * py) +
                                np.cos(b3[0] * px + b3[1] * py))
    else:
        a1 = np.array([2.54, 0.0])
        a2 = np.array([0.0, 2.54])
        xi = sa.square_xi(2.54, 0.1)

        def xi_np(px, py):
            return 0.05 * (np.cos(2 * np.pi * px / 2.54) + np.cos(2 * np.pi * py / 2.54))
    got = sa.corrugated_morse_fourier(x, a1, a2, xi, 7.63, 1.1, 64, 4, 11, 11).numpy()
    want = inputs.corrugated_morse_fourier(x, a1, a2, xi_np, 7.63, 1.1, 64, 4, 11, 11)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)


def test_corrugated_morse_is_differentiable():
    x, _ = sa.lobatto_rule(-1.0, 6.0, 8)
    h = torch.tensor(0.1, dtype=torch.float64, requires_grad=True)
    d = torch.tensor(7.63, dtype=torch.float64, requires_grad=True)
    v = sa.corrugated_morse_fourier(x, [2.54, 0.0], [0.0, 2.54], sa.square_xi(2.54, h), d, 1.1,
                                    32, 2, 5, 5)
    v.real.sum().backward()
    assert h.grad is not None and torch.isfinite(h.grad)
    assert d.grad is not None and torch.isfinite(d.grad)
