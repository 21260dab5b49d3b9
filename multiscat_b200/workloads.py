"""The benchmark and test workloads, built with this package's own setup code.

All in natural units (1/Angstrom^2, Angstrom), He-4 (4.0026 u) unless stated:

- ``cfg0_case``: square lattice a = 2.54 A, corrugated Morse
  V = D[exp(-2 alpha (z - xi)) - 2 exp(-alpha z)], D = 7.63 meV,
  alpha = 1.1 /A, xi = (h/2)(cos 2pi x/a + cos 2pi y/a), h = 0.1 A;
  Fourier modes |m|,|n| <= 4 from a 64 x 64 cell grid; 11 x 11 channels;
  100 Lobatto nodes on [-1.5, 10] A; E = 20 meV at normal incidence.
- ``cfg1_case``: hexagonal a = 3.16 A, xi = (h/3) sum_j cos(b_j . R) over the
  first shell (b1, b2, b1 + b2), h = 0.2 A; E = 64 meV, theta = 30 deg,
  phi = 0; 41 x 41 channels; 200 nodes on [-1.5, 12] A.
- ``cfg2_batch``: 512 seeded beams over cfg0's square potential with
  h = 0.15 A and 150 nodes; E ~ U(8, 64) meV, theta ~ U(0, 60) deg,
  phi ~ U(0, 45) deg; each beam keeps the channels with
  pkd <= (2m/hbar^2) * 200 meV (the ``n_channels``-style truncation by pkd)
  out of a 32 x 32 coupling torus, giving uneven channel counts.
- ``cfg3_problem``: cfg1's system with the loss L = sum_open w_G |S_G|^2,
  w_G ~ U(0, 1) (seeded) on the open channels, and the potential as a
  differentiable function of (D, alpha, h) for adjoint gradients.
- ``cfg4_batch``: square a = 2.54 A, h = 0.25 A, modes |m|,|n| <= 8 from a
  128 x 128 cell grid; 81 x 81 channels; 300 nodes on [-2, 14] A;
  E = 100 meV, theta = 45 deg, 16 azimuths phi = 3k deg.
- ``wolken_case``: the reference's He-LiF golden case
  (``tests/test_fixed_example.py:135-170``): alpha-particle mass, square
  a = 2.84 A (optionally rotated), 10 x 10 x 550 on [0, 8] A, E = 20 meV,
  theta = 30 deg, closed-form potential of ``tests/data/expected_potential.npy``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import setup_arrays as sa
from .solver import SystemSpec, channel_subset_system, full_grid_system

D_MORSE = 7.63
ALPHA_MORSE = 1.1


@dataclass
class Case:
    name: str
    v: np.ndarray          # complex [nkx, nky, nz]  (1/A^2)
    t: np.ndarray          # [nz, nz]
    pkd: np.ndarray        # [nkx, nky]
    wa: np.ndarray         # complex [C]
    wb: np.ndarray
    wc: np.ndarray
    nodes: np.ndarray
    weights: np.ndarray
    extra: dict = field(default_factory=dict)

    def system(self) -> SystemSpec:
        return full_grid_system(self.pkd, self.wa, self.wb, self.wc)


def _beam(factor, energy, theta, phi, a1, a2, nkx, nky, weights, z0, dz):
    k = sa.momentum_from_angles(energy, theta, phi, factor)
    pkd = sa.perpendicular_kinetic_difference(k, a1, a2, nkx, nky)
    wa, wb, wc = sa.waves(pkd, weights, z0, dz)
    return pkd, wa, wb, wc


def square_potential(nodes, a, h, k_max, n_cell, nk, factor, depth=D_MORSE, alpha=ALPHA_MORSE):
    a1, a2 = np.array([a, 0.0]), np.array([0.0, a])
    v = sa.corrugated_morse_fourier(nodes, a1, a2, sa.square_xi(a, h), depth, alpha, n_cell,
                                    k_max, nk, nk)
    return (v * factor).numpy(), a1, a2


def hex_potential(nodes, a, h, k_max, n_cell, nk, factor, depth=D_MORSE, alpha=ALPHA_MORSE):
    a1, a2 = np.array([a, 0.0]), np.array([0.5 * a, 0.5 * math.sqrt(3.0) * a])
    v = sa.corrugated_morse_fourier(nodes, a1, a2, sa.hexagonal_xi(a1, a2, h), depth, alpha,
                                    n_cell, k_max, nk, nk)
    return (v * factor).numpy(), a1, a2


def cfg0_case(nz: int = 100) -> Case:
    factor = sa.natural_units_factor(sa.HE4_MASS)
    z0, z1 = -1.5, 10.0
    nodes, w = sa.lobatto_rule(z0, z1, nz)
    v, a1, a2 = square_potential(nodes, 2.54, 0.1, 4, 64, 11, factor)
    pkd, wa, wb, wc = _beam(factor, 20.0, 0.0, 0.0, a1, a2, 11, 11, w, z0, z1 - z0)
    return Case("cfg0: square 11x11x100", v, sa.kinetic_matrix(nodes, w), pkd, wa, wb, wc,
                nodes, w)


def cfg1_case(nz: int = 200, nk: int = 41) -> Case:
    factor = sa.natural_units_factor(sa.HE4_MASS)
    z0, z1 = -1.5, 12.0
    nodes, w = sa.lobatto_rule(z0, z1, nz)
    v, a1, a2 = hex_potential(nodes, 3.16, 0.2, 4, 64, nk, factor)
    pkd, wa, wb, wc = _beam(factor, 64.0, math.radians(30.0), 0.0, a1, a2, nk, nk, w, z0, z1 - z0)
    return Case(f"cfg1: hexagonal {nk}x{nk}x{nz}", v, sa.kinetic_matrix(nodes, w), pkd, wa, wb,
                wc, nodes, w)


@dataclass
class AdjointProblem:
    """Loss L = sum_G w_G |S_G|^2 over one system and its potential builder."""
    case: Case
    weights: np.ndarray          # [C] (0 on closed channels)
    a1: np.ndarray
    a2: np.ndarray
    h: float
    k_max: int
    n_cell: int
    factor: float
    params: dict = field(default_factory=dict)

    def potential(self, depth=D_MORSE, alpha=ALPHA_MORSE, h=None, device=None) -> torch.Tensor:
        """V (complex128 [nk, nk, nz], 1/A^2) as a torch function of (D meV, alpha 1/A, h A)."""
        h = self.h if h is None else h
        nk = self.case.pkd.shape[0]
        v = sa.corrugated_morse_fourier(self.case.nodes, self.a1, self.a2,
                                        sa.hexagonal_xi(self.a1, self.a2, h), depth, alpha,
                                        self.n_cell, self.k_max, nk, nk, device=device)
        return v * self.factor


def cfg3_problem(nz: int = 200, nk: int = 41, seed: int = 0) -> AdjointProblem:
    """cfg1's hexagonal system; w_G ~ U(0, 1) from default_rng(seed) on the
    open channels (pkd < 0) in the row-major channel order, 0 elsewhere."""
    factor = sa.natural_units_factor(sa.HE4_MASS)
    z0, z1 = -1.5, 12.0
    nodes, w = sa.lobatto_rule(z0, z1, nz)
    a = 3.16
    a1, a2 = np.array([a, 0.0]), np.array([0.5 * a, 0.5 * math.sqrt(3.0) * a])
    h = 0.2
    v = (sa.corrugated_morse_fourier(nodes, a1, a2, sa.hexagonal_xi(a1, a2, h), D_MORSE,
                                     ALPHA_MORSE, 64, 4, nk, nk) * factor).numpy()
    pkd, wa, wb, wc = _beam(factor, 64.0, math.radians(30.0), 0.0, a1, a2, nk, nk, w, z0, z1 - z0)
    case = Case(f"cfg3: hexagonal {nk}x{nk}x{nz}, weighted-intensity loss", v,
                sa.kinetic_matrix(nodes, w), pkd, wa, wb, wc, nodes, w)
    rng = np.random.default_rng(seed)
    draws = rng.uniform(0.0, 1.0, pkd.size)
    weights = np.where(pkd.ravel() < 0.0, draws, 0.0)
    return AdjointProblem(case, weights, a1, a2, h, 4, 64, factor,
                          {"depth": D_MORSE, "alpha": ALPHA_MORSE, "h": h})


def cfg2_batch(n_solves: int = 512, seed: int = 0, nz: int = 150, torus: int = 32,
               cutoff_mev: float = 200.0):
    """(Case holding the shared potential, list of SystemSpec, draws)."""
    factor = sa.natural_units_factor(sa.HE4_MASS)
    z0, z1 = -1.5, 10.0
    nodes, w = sa.lobatto_rule(z0, z1, nz)
    v, a1, a2 = square_potential(nodes, 2.54, 0.15, 4, 64, torus, factor)
    rng = np.random.default_rng(seed)
    energy = rng.uniform(8.0, 64.0, n_solves)
    theta = np.radians(rng.uniform(0.0, 60.0, n_solves))
    phi = np.radians(rng.uniform(0.0, 45.0, n_solves))
    systems = []
    for e, th, ph in zip(energy, theta, phi):
        pkd, wa, wb, wc = _beam(factor, e, th, ph, a1, a2, torus, torus, w, z0, z1 - z0)
        systems.append(channel_subset_system(pkd, wa, wb, wc, max_pkd=factor * cutoff_mev))
    case = Case(f"cfg2: {n_solves} beams, square h=0.15, nz={nz}", v,
                sa.kinetic_matrix(nodes, w), np.zeros((torus, torus)), np.zeros(0), np.zeros(0),
                np.zeros(0), nodes, w, extra={"energy": energy, "theta": theta, "phi": phi})
    return case, systems


def cfg4_batch(n_azimuths: int = 16, nz: int = 300, nk: int = 81):
    factor = sa.natural_units_factor(sa.HE4_MASS)
    z0, z1 = -2.0, 14.0
    nodes, w = sa.lobatto_rule(z0, z1, nz)
    v, a1, a2 = square_potential(nodes, 2.54, 0.25, 8, 128, nk, factor)
    systems = []
    for k in range(n_azimuths):
        pkd, wa, wb, wc = _beam(factor, 100.0, math.radians(45.0), math.radians(3.0 * k), a1, a2,
                                nk, nk, w, z0, z1 - z0)
        systems.append(full_grid_system(pkd, wa, wb, wc))
    case = Case(f"cfg4: square {nk}x{nk}x{nz}, {n_azimuths} azimuths", v,
                sa.kinetic_matrix(nodes, w), np.zeros((nk, nk)), np.zeros(0), np.zeros(0),
                np.zeros(0), nodes, w)
    return case, systems


def wolken_potential(nodes, nkx: int, nky: int) -> np.ndarray:
    """Closed form of the He-LiF potential's Fourier components (meV)."""
    depth, alpha, z0, beta = 7.63, 1.1, 3.0, 0.10
    v = np.zeros((nkx, nky, nodes.size), np.complex128)
    v[0, 0] = depth * (np.exp(2 * alpha * (z0 - nodes)) - 2 * np.exp(alpha * (z0 - nodes)))
    corr = -depth * beta * np.exp(-2 * alpha * (nodes - z0))
    for ix, iy in ((1, 0), (nkx - 1, 0), (0, 1), (0, nky - 1)):
        v[ix, iy] = corr
    return v


def wolken_case(rotation_deg: float = 0.0, nz: int = 550) -> Case:
    factor = sa.natural_units_factor(sa.ALPHA_PARTICLE_MASS)
    nodes, w = sa.lobatto_rule(0.0, 8.0, nz)
    rot = math.radians(rotation_deg)
    rm = np.array([[math.cos(rot), -math.sin(rot)], [math.sin(rot), math.cos(rot)]])
    a1 = rm @ np.array([2.84, 0.0])
    a2 = rm @ np.array([0.0, 2.84])
    v = wolken_potential(nodes, 10, 10) * factor
    pkd, wa, wb, wc = _beam(factor, 20.0, math.radians(30.0), 0.0, a1, a2, 10, 10, w, 0.0, 8.0)
    return Case(f"wolken He-LiF rot={rotation_deg}", v, sa.kinetic_matrix(nodes, w), pkd, wa, wb,
                wc, nodes, w)


def intensities_host(psi: np.ndarray, system: SystemSpec) -> np.ndarray:
    """|S|^2 from psi[C, nz] on the host (tests and the CPU oracle path)."""
    s = 2.0j * system.wave_b * psi[:, -1]
    s = s.copy()
    s[system.specular] += system.wave_a[system.specular]
    return np.abs(s) ** 2


def to_torch(case: Case, device) -> dict:
    return {"v": torch.as_tensor(case.v, device=device), "t": torch.as_tensor(case.t, device=device)}
