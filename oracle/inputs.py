"""Numpy restatement of the reference's solver inputs.

TEST INFRASTRUCTURE ONLY: the oracle's own input builders.  The product
(`multiscat_b200`) builds the same arrays with its own code; tests compare the
two.  Each function cites the reference routine it restates (paths relative to
the multiscat project):

- ``lobatto_rule``: ``lib/multiscat_fortran/fortran/scatsub.f90:293-369``
  (Newton iteration on P'_{n-1} from a Tricomi-type start, 7 steps, end nodes
  fixed, weights (b-a)/(n(n-1)P_{n-1}^2)).
- ``kinetic_matrix``: ``multiscat/polynomial.py:54-127`` (barycentric
  derivative matrix, T_ij = sum_k w_k u_i'(z_k) u_j'(z_k)) with the sign flip of
  ``multiscat/multiscat/_fortran.py:127`` already applied (T is positive).
- ``perpendicular_kinetic_difference``: ``scatsub.f90:102-150`` and
  ``multiscat/multiscat/_util.py:58-75``.
- ``waves``: ``multiscat/multiscat/_util.py:78-147`` (a, b, c arrays).
- ``intensities``: ``multiscat/multiscat/_multiscat.py:40-60``.
- ``natural_units_factor``: the unit change of ``multiscat/config.py:61-84,
  230-296`` (hbar = 1, m = 1/2, lengths in Angstrom, so energies become
  (2m/hbar^2) E in 1/Angstrom^2).
"""

from __future__ import annotations

import numpy as np
from scipy import constants as sc

AMU = sc.atomic_mass
MEV = sc.electron_volt * 1e-3
HE4_MASS_AMU = 4.0026
ALPHA_PARTICLE_MASS_KG = sc.physical_constants["alpha particle mass"][0]


def natural_units_factor(mass_kg: float) -> float:
    """2m/hbar^2 in 1/(Angstrom^2 meV): multiply an energy in meV by this."""
    return 2.0 * mass_kg / sc.hbar**2 * MEV * 1e-20


def fft_mode(i: int, n: int) -> int:
    """FFT-order mode index of storage index i (scatsub.f90:137-144)."""
    return i if i <= (n - 1) // 2 else i - n


def lobatto_rule(z_min: float, z_max: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Nodes (ascending) and quadrature weights of the n-point Lobatto rule."""
    x = np.zeros(n)
    w = np.zeros(n)
    shift = 0.5 * (z_max + z_min)
    scale = 0.5 * (z_max - z_min)
    weight = (z_max - z_min) / (n * (n - 1))
    x[0] = z_min
    w[0] = weight
    half = (n + 1) // 2
    for k in range(2, half + 1):
        z = np.cos(np.pi * (4 * k - 3) / (4 * n - 2))
        for _ in range(7):
            p2, p1 = 0.0, 1.0
            for j in range(1, n):
                p3 = p2
                p2 = p1
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j
            dp = (n - 1) * (p2 - z * p1) / (1.0 - z * z)
            d2p = (2.0 * z * dp - n * (n - 1) * p1) / (1.0 - z * z)
            z = z - dp / d2p
        x[k - 1] = shift - scale * z
        x[n - k] = shift + scale * z
        w[k - 1] = weight / (p1 * p1)
        w[n - k] = w[k - 1]
    x[n - 1] = z_max
    w[n - 1] = weight
    return x, w


def kinetic_matrix(nodes: np.ndarray, weights: np.ndarray) -> np.ndarray:
    """Positive Lobatto DVR kinetic matrix T_ij = sum_k w_k u_i'(z_k) u_j'(z_k)."""
    n = nodes.size
    scale = 1.0 / (nodes[-1] - nodes[0])
    s = (nodes - nodes[0]) * scale
    diff = s[:, None] - s[None, :]
    np.fill_diagonal(diff, 1.0)
    logw = np.sum(np.log(np.abs(diff)), axis=1)
    sgn = np.prod(np.sign(diff), axis=1)
    ratio = (sgn[:, None] * sgn[None, :]) * np.exp(logw[:, None] - logw[None, :])
    d = ratio / diff                       # d[i, j] = l_j'(s_i)
    inv = 1.0 / diff
    np.fill_diagonal(inv, 0.0)
    d[np.diag_indices(n)] = np.sum(inv, axis=1)
    d *= scale
    bw = 1.0 / np.sqrt(weights)
    deriv = d.T * bw[:, None]              # deriv[i, k] = u_i'(z_k)
    return np.einsum("k,ik,jk->ij", weights, deriv, deriv)


def reciprocal_vectors(a1: np.ndarray, a2: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """b_i . a_j = 2 pi delta_ij (scatsub.f90:102-116)."""
    auc = abs(a1[0] * a2[1] - a1[1] * a2[0])
    rec = 2.0 * np.pi / auc
    b1 = np.array([a2[1] * rec, -a2[0] * rec])
    b2 = np.array([-a1[1] * rec, a1[0] * rec])
    return b1, b2


def perpendicular_kinetic_difference(incident_k, a1, a2, nkx: int, nky: int) -> np.ndarray:
    """pkd[ix, iy] = |K + G|^2 - |k|^2 on the FFT-ordered channel grid."""
    b1, b2 = reciprocal_vectors(np.asarray(a1, float), np.asarray(a2, float))
    k = np.asarray(incident_k, float)
    out = np.zeros((nkx, nky))
    for ix in range(nkx):
        mx = fft_mode(ix, nkx)
        for iy in range(nky):
            my = fft_mode(iy, nky)
            g = mx * b1 + my * b2
            out[ix, iy] = (k[0] + g[0]) ** 2 + (k[1] + g[1]) ** 2 - float(np.sum(k**2))
    return out


def waves(pkd: np.ndarray, weights: np.ndarray, z_start: float, z_delta: float):
    """(a, b, c) per channel, flattened in C order (_util.py:78-147).

    theta uses (delta - start) exactly as _util.py:108 does; |S|^2 does not
    depend on it.
    """
    e = np.asarray(pkd, float).ravel()
    dk = np.sqrt(np.abs(e))
    a = np.zeros(e.shape, complex)
    b = np.zeros(e.shape, complex)
    open_ = e < 0.0
    theta = dk[open_] * (z_delta - z_start)
    a[open_] = np.exp(-2.0j * theta)
    b[open_] = np.sqrt(dk[open_]) * np.exp(-1.0j * theta)
    bw_last = 1.0 / np.sqrt(weights[-1])
    b = b * bw_last
    c = 1j * np.emath.sqrt(-e) * bw_last**2
    return a, b, np.asarray(c, complex)


def intensities(psi: np.ndarray, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """|S_G0|^2 from the last z row of psi[C, nz] (_multiscat.py:40-60)."""
    s = 2.0j * b * psi[:, -1]
    s = s.copy()
    s[0] += a[0]
    return np.abs(s) ** 2


# ---------------------------------------------------------------------------
# Potentials
# ---------------------------------------------------------------------------

def wolken_potential(nodes: np.ndarray, nkx: int, nky: int) -> np.ndarray:
    """He-LiF Wolken corrugated Morse potential in meV on the channel grid.

    V00 = D[e^{2a(z0-z)} - 2 e^{a(z0-z)}], V(+-1,0) = V(0,+-1) = -D b e^{-2a(z-z0)}
    with D = 7.63 meV, a = 1.1 /A, z0 = 3 A, b = 0.10: the convention that the
    reference's own fixture tests/data/expected_potential.npy holds.
    """
    depth, alpha, z0, beta = 7.63, 1.1, 3.0, 0.10
    v = np.zeros((nkx, nky, nodes.size), complex)
    v[0, 0] = depth * (np.exp(2 * alpha * (z0 - nodes)) - 2 * np.exp(alpha * (z0 - nodes)))
    corr = -depth * beta * np.exp(-2 * alpha * (nodes - z0))
    for ix, iy in ((1, 0), (nkx - 1, 0), (0, 1), (0, nky - 1)):
        v[ix, iy] = corr
    return v


def corrugated_morse_fourier(nodes, a1, a2, xi_fn, depth, alpha, n_cell, k_max, nkx, nky):
    """Fourier components (meV) of V = D[e^{-2a(z - xi)} - 2 e^{-a z}].

    V is sampled on an n_cell x n_cell grid of fractional cell coordinates at
    each node; coefficients are fft2 / n_cell^2; modes with |m|,|n| <= k_max
    are placed in FFT order on the nkx x nky channel grid.
    """
    f = np.arange(n_cell) / n_cell
    fx, fy = np.meshgrid(f, f, indexing="ij")
    rx = fx * a1[0] + fy * a2[0]
    ry = fx * a1[1] + fy * a2[1]
    xi = xi_fn(rx, ry)
    out = np.zeros((nkx, nky, nodes.size), complex)
    modes = [(m, n) for m in range(-k_max, k_max + 1) for n in range(-k_max, k_max + 1)]
    for k, z in enumerate(nodes):
        v = depth * (np.exp(-2 * alpha * (z - xi)) - 2 * np.exp(-alpha * z))
        c = np.fft.fft2(v) / n_cell**2
        for m, n in modes:
            out[m % nkx, n % nky, k] = c[m % n_cell, n % n_cell]
    return out
