"""Solver inputs: Lobatto grid, kinetic matrix, channel energies, waves, potentials.

These build exactly the arrays the reference passes to its Fortran solve
(``multiscat/multiscat/_fortran.py:105-156``), in natural units (hbar = 1,
m = 1/2, lengths in Angstrom, energies in 1/Angstrom^2):

- ``lobatto_rule``: Gauss-Lobatto nodes/weights on [z_min, z_max]
  (``lib/multiscat_fortran/fortran/scatsub.f90:293-369``; here Newton's
  method on P'_{n-1} is iterated to convergence, vectorised over nodes).
- ``kinetic_matrix``: positive Lobatto DVR kinetic matrix
  T_ij = sum_k w_k u_i'(z_k) u_j'(z_k) with u_i = l_i / sqrt(w_i)
  (``multiscat/polynomial.py:54-127`` negated as ``_fortran.py:127`` does).
- ``perpendicular_kinetic_difference``: |K + G|^2 - |k|^2 on the FFT-ordered
  channel grid (``scatsub.f90:118-150``, ``_util.py:58-75``).
- ``waves``: a, b, c boundary arrays (``_util.py:78-147``).
- ``corrugated_morse_fourier``: mean-normalised Fourier components of a
  corrugated Morse potential on the channel grid, written with torch so that
  gradients flow to (D, alpha, h).

Everything here is setup (O(n^3 + C n) once per potential or beam); the hot
path is the CUDA solve.
"""

from __future__ import annotations

import math

import numpy as np
import torch

HBAR = 1.054571817e-34
ATOMIC_MASS = 1.66053906660e-27
ELECTRON_VOLT = 1.602176634e-19
MEV = ELECTRON_VOLT * 1e-3
ANGSTROM = 1e-10
ALPHA_PARTICLE_MASS = 6.6446573450e-27
HE4_MASS = 4.0026 * ATOMIC_MASS


def natural_units_factor(mass_kg: float) -> float:
    """2m/hbar^2 in 1/(Angstrom^2 meV): energy in meV times this is in 1/A^2."""
    return 2.0 * mass_kg / HBAR**2 * MEV * ANGSTROM**2


def fft_modes(n: int) -> np.ndarray:
    """Mode index of each storage index in FFT order (0, 1, ..., -1)."""
    i = np.arange(n)
    return np.where(i <= (n - 1) // 2, i, i - n)


def lobatto_rule(z_min: float, z_max: float, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Nodes (ascending, both end points included) and weights of the n-point rule."""
    if n < 2:
        raise ValueError("a Lobatto rule needs at least 2 nodes")
    k = np.arange(2, (n + 1) // 2 + 1)
    z = np.cos(np.pi * (4 * k - 3) / (4 * n - 2))
    for _ in range(100):
        p_prev = np.zeros_like(z)
        p = np.ones_like(z)
        for j in range(1, n):
            p_prev, p = p, ((2 * j - 1) * z * p - (j - 1) * p_prev) / j
        dp = (n - 1) * (p_prev - z * p) / (1.0 - z * z)
        d2p = (2.0 * z * dp - n * (n - 1) * p) / (1.0 - z * z)
        step = dp / d2p
        z = z - step
        if np.max(np.abs(step), initial=0.0) < 1e-16:
            break
    # final Legendre value at the converged roots for the weights
    p_prev = np.zeros_like(z)
    p = np.ones_like(z)
    for j in range(1, n):
        p_prev, p = p, ((2 * j - 1) * z * p - (j - 1) * p_prev) / j
    shift = 0.5 * (z_max + z_min)
    scale = 0.5 * (z_max - z_min)
    base = (z_max - z_min) / (n * (n - 1))
    x = np.empty(n)
    w = np.empty(n)
    x[0], x[-1] = z_min, z_max
    w[0] = w[-1] = base
    idx = k - 1
    x[idx] = shift - scale * z
    x[n - k] = shift + scale * z
    w[idx] = base / (p * p)
    w[n - k] = w[idx]
    return x, w


def kinetic_matrix(nodes: np.ndarray, weights: np.ndarray) -> np.ndarray:
    """Positive Lobatto kinetic matrix (n x n, symmetric)."""
    nodes = np.asarray(nodes, float)
    weights = np.asarray(weights, float)
    n = nodes.size
    scale = 1.0 / (nodes[-1] - nodes[0])
    s = (nodes - nodes[0]) * scale
    diff = s[:, None] - s[None, :]
    np.fill_diagonal(diff, 1.0)
    log_prod = np.log(np.abs(diff)).sum(axis=1)
    sign = np.prod(np.sign(diff), axis=1)
    # l_j'(s_i) = (prod_i / prod_j) / (s_i - s_j) off the diagonal
    deriv = (sign[:, None] * sign[None, :]) * np.exp(log_prod[:, None] - log_prod[None, :]) / diff
    inv = 1.0 / diff
    np.fill_diagonal(inv, 0.0)
    deriv[np.diag_indices(n)] = inv.sum(axis=1)
    deriv *= scale
    # u_j'(z_i) = l_j'(z_i) / sqrt(w_j);  T = U^T W U with U[i, j] = u_j'(z_i)
    u = deriv / np.sqrt(weights)[None, :]
    t = u.T @ (weights[:, None] * u)
    return 0.5 * (t + t.T)


def reciprocal_vectors(a1, a2) -> tuple[np.ndarray, np.ndarray]:
    """Reciprocal lattice vectors with b_i . a_j = 2 pi delta_ij."""
    a1 = np.asarray(a1, float)[:2]
    a2 = np.asarray(a2, float)[:2]
    area = abs(a1[0] * a2[1] - a1[1] * a2[0])
    if area <= 0.0:
        raise ValueError("unit cell area must be positive")
    f = 2.0 * np.pi / area
    return np.array([a2[1] * f, -a2[0] * f]), np.array([-a1[1] * f, a1[0] * f])


def perpendicular_kinetic_difference(incident_k, a1, a2, nkx: int, nky: int) -> np.ndarray:
    """pkd[ix, iy] = |K + G(ix, iy)|^2 - |k|^2 (negative = open channel)."""
    b1, b2 = reciprocal_vectors(a1, a2)
    k = np.asarray(incident_k, float)
    mx = fft_modes(nkx)[:, None]
    my = fft_modes(nky)[None, :]
    gx = k[0] + mx * b1[0] + my * b2[0]
    gy = k[1] + mx * b1[1] + my * b2[1]
    return gx * gx + gy * gy - float(k @ k)


def waves(pkd: np.ndarray, weights: np.ndarray, z_start: float, z_delta: float):
    """Boundary arrays (a, b, c), flattened in C order.

    theta = sqrt(-pkd) * (z_delta - z_start) as in ``_util.py:108``; |S|^2
    does not depend on theta.
    """
    e = np.asarray(pkd, float).ravel()
    bw_last = 1.0 / math.sqrt(float(weights[-1]))
    dk = np.sqrt(np.abs(e))
    opened = e < 0.0
    theta = dk * (z_delta - z_start)
    a = np.where(opened, np.exp(-2.0j * theta), 0.0).astype(np.complex128)
    b = np.where(opened, np.sqrt(dk) * np.exp(-1.0j * theta), 0.0).astype(np.complex128) * bw_last
    c = np.where(opened, 1.0j * dk, -dk).astype(np.complex128) * bw_last**2
    return a, b, c


def perpendicular_kinetic_difference_batch(incident_ks, a1, a2, nkx: int, nky: int) -> np.ndarray:
    """pkd of many beams at once, [B, nkx, nky]: element for element the same
    arithmetic as ``perpendicular_kinetic_difference`` (identical results)."""
    b1, b2 = reciprocal_vectors(a1, a2)
    ks = np.asarray(incident_ks, float).reshape(-1, 3)
    mx = fft_modes(nkx)[None, :, None]
    my = fft_modes(nky)[None, None, :]
    gx = ks[:, 0, None, None] + mx * b1[0] + my * b2[0]
    gy = ks[:, 1, None, None] + mx * b1[1] + my * b2[1]
    kk = np.array([float(k @ k) for k in ks])
    return gx * gx + gy * gy - kk[:, None, None]


def momentum_from_angles(energy_mev: float, theta: float, phi: float, factor: float):
    """Incident k (1/A) for an energy in meV and angles in radians."""
    k = math.sqrt(factor * energy_mev)
    return (k * math.sin(theta) * math.cos(phi), k * math.sin(theta) * math.sin(phi),
            k * math.cos(theta))


def corrugated_morse_fourier(nodes, a1, a2, xi_fn, depth, alpha, n_cell: int, k_max: int,
                             nkx: int, nky: int, *, device=None) -> torch.Tensor:
    """Fourier components V_G(z_k) (same unit as ``depth``) on the channel grid.

    V(R, z) = D [exp(-2 alpha (z - xi(R))) - 2 exp(-alpha z)] is sampled on an
    n_cell x n_cell grid of fractional cell coordinates at every node;
    V_G = fft2 / n_cell^2; modes |m|, |n| <= k_max are placed in FFT order on
    the nkx x nky grid (the reference's potential_values convention,
    ``_util.py:150-163``).  ``depth``, ``alpha`` and whatever ``xi_fn``
    closes over may be tensors with requires_grad.
    """
    if 2 * k_max + 1 > min(nkx, nky):
        raise ValueError("channel grid too small for the requested Fourier modes")
    dev = device if device is not None else "cpu"
    z = torch.as_tensor(np.asarray(nodes, float), dtype=torch.float64, device=dev)
    f = torch.arange(n_cell, dtype=torch.float64, device=dev) / n_cell
    fx, fy = torch.meshgrid(f, f, indexing="ij")
    rx = fx * float(a1[0]) + fy * float(a2[0])
    ry = fx * float(a1[1]) + fy * float(a2[1])
    xi = xi_fn(rx, ry)
    depth = torch.as_tensor(depth, dtype=torch.float64, device=dev)
    alpha = torch.as_tensor(alpha, dtype=torch.float64, device=dev)
    v = depth * (torch.exp(-2.0 * alpha * (z[:, None, None] - xi[None])) -
                 2.0 * torch.exp(-alpha * z)[:, None, None])
    coef = torch.fft.fft2(v) / (n_cell * n_cell)          # [nz, n_cell, n_cell]
    modes = torch.arange(-k_max, k_max + 1, device=dev)
    src_x = torch.remainder(modes, n_cell)
    src_y = torch.remainder(modes, n_cell)
    dst_x = torch.remainder(modes, nkx)
    dst_y = torch.remainder(modes, nky)
    sub = coef[:, src_x][:, :, src_y]                      # [nz, 2K+1, 2K+1]
    out = torch.zeros((nkx, nky, z.numel()), dtype=torch.complex128, device=dev)
    out = out.index_put((dst_x[:, None].expand(-1, dst_y.numel()),
                         dst_y[None, :].expand(dst_x.numel(), -1)),
                        sub.permute(1, 2, 0))
    return out


def square_xi(a: float, h):
    """xi = (h/2)(cos 2 pi x/a + cos 2 pi y/a)."""
    def fn(x, y):
        return 0.5 * h * (torch.cos(2 * math.pi * x / a) + torch.cos(2 * math.pi * y / a))
    return fn


def hexagonal_xi(a1, a2, h):
    """xi = (h/3) sum_j cos(b_j . R) over b1, b2, b1 + b2 (first shell)."""
    b1, b2 = reciprocal_vectors(a1, a2)
    b3 = b1 + b2

    def fn(x, y):
        return (h / 3.0) * (torch.cos(b1[0] * x + b1[1] * y) + torch.cos(b2[0] * x + b2[1] * y) +
                            torch.cos(b3[0] * x + b3[1] * y))
    return fn


def interpolate_potential(values, z_grid, nodes, nkx: int, nky: int, *, device=None) -> torch.Tensor:
    """Potential samples on an evenly spaced (x, y, z) grid -> V_G(z_k) on the
    channel grid at the Lobatto nodes (``interpolate.py:38-116``).

    values   [nx, ny, nz_grid] real or complex samples V(x_i, y_j, z_l) over
             one unit cell (fractional coordinates i/nx, j/ny);
    z_grid   [nz_grid] increasing sample heights; nodes [n] target heights.

    The parallel directions go to momentum space (fft2 / (nx ny), the
    solver's convention) and the modes are placed in FFT order on the
    nkx x nky grid (modes beyond the sample grid's Nyquist range are zero;
    modes beyond the channel grid are dropped).  Along z each V_G is linearly
    interpolated with the end values held outside the sampled range
    (``np.interp`` behaviour).  The result holds plain values V_G(z_k), the
    solver's ``potential_values`` (the reference multiplies by the Lobatto
    weights only because it stores an operator in a weighted basis).
    """
    dev = device if device is not None else (values.device if torch.is_tensor(values) else "cpu")
    v = torch.as_tensor(values, device=dev)
    v = v.to(torch.complex128) if not torch.is_complex(v) else v.to(torch.complex128)
    nx, ny, ng = v.shape
    zg = torch.as_tensor(np.asarray(z_grid, float) if not torch.is_tensor(z_grid) else z_grid,
                         dtype=torch.float64, device=dev)
    zn = torch.as_tensor(np.asarray(nodes, float) if not torch.is_tensor(nodes) else nodes,
                         dtype=torch.float64, device=dev)
    if zg.numel() != ng or ng < 2 or bool((zg[1:] <= zg[:-1]).any()):
        raise ValueError("z_grid must be increasing and match the last axis of values")
    coef = torch.fft.fft2(v, dim=(0, 1)) / (nx * ny)                    # [nx, ny, ng]

    def mode_map(nk: int, ns: int):
        # FFT-order index on the channel grid -> index on the sample grid (or -1);
        # both grids use numpy's FFT mode order (0, 1, ..., -1)
        m = fft_modes(nk)
        ok = (m <= (ns - 1) // 2) & (m >= -(ns // 2))
        return np.where(ok, np.mod(m, ns), -1)

    mx, my = mode_map(nkx, nx), mode_map(nky, ny)
    out_modes = torch.zeros((nkx, nky, ng), dtype=torch.complex128, device=dev)
    ix = torch.as_tensor(np.nonzero(mx >= 0)[0], device=dev)
    iy = torch.as_tensor(np.nonzero(my >= 0)[0], device=dev)
    sx = torch.as_tensor(mx[mx >= 0], device=dev)
    sy = torch.as_tensor(my[my >= 0], device=dev)
    out_modes[ix[:, None], iy[None, :]] = coef[sx[:, None], sy[None, :]]
    # linear interpolation along z, clamped at the ends
    zc = zn.clamp(zg[0], zg[-1])
    hi = torch.searchsorted(zg, zc).clamp(1, ng - 1)
    lo = hi - 1
    t = ((zc - zg[lo]) / (zg[hi] - zg[lo])).to(torch.complex128)
    return out_modes[:, :, lo] * (1 - t) + out_modes[:, :, hi] * t
