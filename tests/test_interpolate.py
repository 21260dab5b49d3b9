"""interpolate_potential (the reference's interpolate.py:38-116) against a
numpy restatement, and against the analytic builder on a fine z grid."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from multiscat_b200 import setup_arrays as sa


def _numpy_interp(vals, zg, nodes, nkx, nky):
    nx, ny, _ = vals.shape
    c = np.fft.fft2(vals, axes=(0, 1)) / (nx * ny)
    out = np.zeros((nkx, nky, nodes.size), complex)
    for ix, m in enumerate(sa.fft_modes(nkx)):
        if not -(nx // 2) <= m <= (nx - 1) // 2:
            continue
        for iy, k in enumerate(sa.fft_modes(nky)):
            if not -(ny // 2) <= k <= (ny - 1) // 2:
                continue
            src = c[m % nx, k % ny]
            out[ix, iy] = np.interp(nodes, zg, src.real) + 1j * np.interp(nodes, zg, src.imag)
    return out


@pytest.mark.parametrize("shape", [(16, 12, 9, 7), (10, 10, 12, 12), (8, 6, 5, 5)])
def test_interpolate_potential_matches_numpy(shape):
    nx, ny, nkx, nky = shape
    rng = np.random.default_rng(nx + nkx)
    vals = rng.normal(size=(nx, ny, 30)) + 1j * rng.normal(size=(nx, ny, 30))
    zg = np.sort(rng.uniform(-2.0, 10.0, 30))
    nodes = np.linspace(-3.0, 11.0, 41)           # both ends outside the samples
    got = sa.interpolate_potential(vals, zg, nodes, nkx, nky).numpy()
    np.testing.assert_allclose(got, _numpy_interp(vals, zg, nodes, nkx, nky), rtol=0, atol=1e-13)


def test_interpolated_morse_approaches_the_analytic_components():
    """A corrugated Morse potential sampled on 64 x 64 x 2000 points and
    interpolated onto Lobatto nodes agrees with the builder that evaluates the
    same potential at the nodes directly (linear interpolation error only)."""
    a = 2.54
    a1, a2 = np.array([a, 0.0]), np.array([0.0, a])
    nodes, _ = sa.lobatto_rule(-1.5, 10.0, 60)
    xi = sa.square_xi(a, 0.1)
    direct = sa.corrugated_morse_fourier(nodes, a1, a2, xi, 7.63, 1.1, 64, 4, 11, 11).numpy()
    zg = np.linspace(-1.5, 10.0, 2000)
    f = np.arange(64) / 64
    fx, fy = np.meshgrid(f, f, indexing="ij")
    xiv = xi(torch.as_tensor(fx * a), torch.as_tensor(fy * a)).numpy()
    samples = 7.63 * (np.exp(-2.2 * (zg[None, None, :] - xiv[:, :, None]))
                      - 2.0 * np.exp(-1.1 * zg)[None, None, :])
    got = sa.interpolate_potential(samples, zg, nodes, 11, 11).numpy()
    # keep the |m|,|n| <= 4 modes the builder keeps; the others must be tiny
    mask = np.zeros((11, 11), bool)
    keep = [i for i, m in enumerate(sa.fft_modes(11)) if abs(m) <= 4]
    mask[np.ix_(keep, keep)] = True
    scale = np.abs(direct).max()
    assert np.abs(got[mask] - direct[mask]).max() <= 2e-4 * scale
    assert np.abs(got[~mask]).max() <= 1e-6 * scale
