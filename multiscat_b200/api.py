"""Reference-shaped public API: conditions and configs in, intensities out.

Mirrors ``multiscat/multiscat/_multiscat.py:131-175`` (``get_scattering_matrix``)
and ``multiscat/config.py:41-227`` (``OptimizationConfig``, ``UnitSystem``,
``ScatteringCondition.from_angles``, ``momentum_from_angles``) with the same
field names, without the slate basis objects: a condition carries its lattice
vectors, grid shape, z domain and the potential's Fourier components on the
Lobatto nodes (what ``potential_as_array`` returns, ``_util.py:150-163``).

``get_scattering_matrix`` returns |S_G0|^2 on the (nkx, nky) channel grid as
complex128, exactly as the reference's array does (``_multiscat.py:166-175``).
"""

from __future__ import annotations

import math
from collections import OrderedDict
from dataclasses import dataclass, field
from typing import Literal, Sequence

import numpy as np
import torch

from . import setup_arrays as sa
from .solver import (ScatteringPlan, SolveResult, SystemSpec, beam_systems,
                     channel_subset_system, full_grid_system)


@dataclass(frozen=True, kw_only=True)
class OptimizationConfig:
    """Solver options (``config.py:41-58``) plus the GPU solver's own."""

    precision: float = 1e-5
    max_iterations: int = 1000
    use_neumann_preconditioner: bool = True
    n_channels: int | None = None
    restart: int = 30
    precision_mode: Literal["fp64", "mixed"] = "fp64"

    @property
    def residual_tolerance(self) -> float:
        """Stop rule ||b - A psi|| <= 1e-3 precision ||b||.

        The reference stops on its left-preconditioned residual
        (multiscat_gmres.f90:590-597); this solver stops on the true residual,
        which is larger by the conditioning of A.  The 1e-3 factor keeps
        |sum |S|^2 - 1| below ``precision`` on the golden He-LiF case.
        """
        if self.precision <= 0:
            raise ValueError("Optimization precision must be greater than zero")
        return self.precision * 1e-3


@dataclass(frozen=True, kw_only=True)
class UnitSystem:
    """Units of a condition (``config.py:61-84``); SI by default."""

    hbar: float = sa.HBAR
    atomic_mass: float = sa.ATOMIC_MASS
    angstrom: float = sa.ANGSTROM

    @classmethod
    def si(cls) -> "UnitSystem":
        """The SI units (``config.py:69-72``)."""
        return cls()

    @property
    def kinetic_energy_unit(self) -> float:
        return self.hbar**2 / (2 * self.atomic_mass * self.angstrom**2)

    @property
    def electron_volt(self) -> float:
        """The reference's definition (``config.py:79-84``):
        eV_SI * (kinetic_energy_unit of SI / kinetic_energy_unit of this system),
        kept as is for drop-in parity.  It is 1.602e-19 for SI; for other
        systems it is the inverse of the factor `with_units` applies to
        energies, and the reference itself never reads it."""
        return sa.ELECTRON_VOLT * (UnitSystem().kinetic_energy_unit / self.kinetic_energy_unit)


SI_UNITS = UnitSystem.si()


@dataclass
class ScatteringMetadata:
    """Grid of a scattering problem: lattice vectors, channel grid and z domain.

    ``vectors`` are the two lattice vectors (SI lengths, 2 or 3 components);
    ``shape`` = (nkx, nky, nz); the z domain is [z_start, z_start + z_delta].
    """

    vectors: tuple[Sequence[float], Sequence[float]]
    shape: tuple[int, int, int]
    z_delta: float
    z_start: float = 0.0


def momentum_from_angles(theta: float, phi: float, energy: float, mass: float, *,
                         units: UnitSystem = SI_UNITS) -> tuple[float, float, float]:
    """Incident momentum from angles (``config.py:213-227``)."""
    abs_k = math.sqrt(2 * mass * energy) / units.hbar
    return (abs_k * math.sin(theta) * math.cos(phi), abs_k * math.sin(theta) * math.sin(phi),
            abs_k * math.cos(theta))


@dataclass
class ScatteringCondition:
    """Mass (kg), incident k (1/m), potential V_G(z_k) (J) and grid."""

    mass: float
    incident_k: tuple[float, float, float]
    potential_values: np.ndarray
    metadata: ScatteringMetadata
    units: UnitSystem = field(default_factory=UnitSystem)

    @staticmethod
    def from_angles(*, mass: float, theta: float = 0.0, phi: float = 0.0, energy: float,
                    potential_values, metadata: ScatteringMetadata,
                    units: UnitSystem = SI_UNITS) -> "ScatteringCondition":
        return ScatteringCondition(mass, momentum_from_angles(theta, phi, energy, mass, units=units),
                                   np.asarray(potential_values), metadata, units)

    @property
    def incident_energy(self) -> float:
        k2 = sum(k * k for k in self.incident_k)
        return self.units.hbar**2 * k2 / (2 * self.mass)

    @property
    def theta(self) -> float:
        """Polar angle of the incident wavevector (radians, ``config.py:186-190``)."""
        kx, ky, kz = self.incident_k
        return float(np.arccos(kz / np.sqrt(kx * kx + ky * ky + kz * kz)))

    @property
    def phi(self) -> float:
        """Azimuth of the incident wavevector (radians, ``config.py:192-196``)."""
        kx, ky, _ = self.incident_k
        return float(np.arctan2(ky, kx))

    def with_units(self, units: UnitSystem) -> "ScatteringCondition":
        """The same condition expressed in another unit system
        (``config.py:198-200, 230-296``): masses scale with the atomic mass
        unit, lengths with the angstrom, wavevectors inversely, and the
        potential values with the kinetic-energy unit."""
        mass_factor = units.atomic_mass / self.units.atomic_mass
        length_factor = units.angstrom / self.units.angstrom
        energy_factor = units.kinetic_energy_unit / self.units.kinetic_energy_unit
        md = self.metadata
        metadata = ScatteringMetadata(
            vectors=tuple(np.asarray(v, float) * length_factor for v in md.vectors),
            shape=tuple(md.shape), z_delta=md.z_delta * length_factor,
            z_start=md.z_start * length_factor)
        return ScatteringCondition(self.mass * mass_factor,
                                   tuple(float(k) / length_factor for k in self.incident_k),
                                   np.asarray(self.potential_values) * energy_factor, metadata,
                                   units)

    def __eq__(self, other: object) -> bool:
        """Same mass, incident k, potential, grid and units (``config.py:202-210``)."""
        if not isinstance(other, ScatteringCondition):
            return False
        m, o = self.metadata, other.metadata
        return (self.mass == other.mass and tuple(self.incident_k) == tuple(other.incident_k)
                and self.units == other.units and tuple(m.shape) == tuple(o.shape)
                and m.z_start == o.z_start and m.z_delta == o.z_delta
                and all(np.array_equal(np.asarray(a, float), np.asarray(b, float))
                        for a, b in zip(m.vectors, o.vectors))
                and np.array_equal(np.asarray(self.potential_values),
                                   np.asarray(other.potential_values)))

    __hash__ = None


@dataclass
class NaturalArrays:
    """The solver's inputs in natural units (1/A^2, A)."""

    potential_values: np.ndarray
    kinetic: np.ndarray
    pkd: np.ndarray
    wave_a: np.ndarray
    wave_b: np.ndarray
    wave_c: np.ndarray
    nodes: np.ndarray
    weights: np.ndarray


def _lattice_frame(condition: ScatteringCondition):
    """Lattice vectors (a1 along x) and z domain of a condition, in Angstrom.

    Incident k is read in the lattice frame: rotating both lattice vectors
    leaves the result unchanged, as the reference's
    tests/test_fixed_example.py:259-330 requires."""
    to_ang = 1.0 / condition.units.angstrom                     # length unit -> Angstrom
    md = condition.metadata
    a1 = np.asarray(md.vectors[0], float)[:2] * to_ang
    a2 = np.asarray(md.vectors[1], float)[:2] * to_ang
    rot = math.atan2(a1[1], a1[0])
    cr, sr = math.cos(rot), math.sin(rot)
    unrot = np.array([[cr, sr], [-sr, cr]])
    return unrot @ a1, unrot @ a2, md.z_start * to_ang, md.z_delta * to_ang


def _beam_arrays(condition: ScatteringCondition, a1, a2, weights, z0: float, dz: float):
    """pkd and the boundary waves (a, b, c) of one beam on a built grid."""
    nkx, nky, _ = condition.metadata.shape
    k = tuple(float(c) * condition.units.angstrom for c in condition.incident_k)
    pkd = sa.perpendicular_kinetic_difference(k, a1, a2, nkx, nky)
    wa, wb, wc = sa.waves(pkd, weights, z0, dz)
    return pkd, wa, wb, wc


_GRID_CACHE: "OrderedDict[tuple, tuple]" = OrderedDict()
_GRID_CACHE_SIZE = 8


def _lobatto_grid(z_min: float, z_max: float, n: int):
    """(nodes, weights, kinetic matrix) of the n-point Lobatto grid, cached by
    (z_min, z_max, n): one condition after another on the same grid (the
    reference's usual loop) rebuilds nothing (n = 550: ~30 ms saved per call).
    Returns copies, so callers may modify them."""
    key = (float(z_min), float(z_max), int(n))
    hit = _GRID_CACHE.get(key)
    if hit is None:
        nodes, weights = sa.lobatto_rule(z_min, z_max, n)
        hit = (nodes, weights, sa.kinetic_matrix(nodes, weights))
        _GRID_CACHE[key] = hit
        while len(_GRID_CACHE) > _GRID_CACHE_SIZE:
            _GRID_CACHE.popitem(last=False)
    else:
        _GRID_CACHE.move_to_end(key)
    return tuple(a.copy() for a in hit)


def natural_arrays(condition: ScatteringCondition) -> NaturalArrays:
    """Convert to hbar = 1, m = 1/2, Angstrom (``_multiscat.py:102-128``) and build arrays."""
    u = condition.units
    energy_to_nat = 2.0 * condition.mass / u.hbar**2 * u.angstrom**2   # energy -> 1/A^2
    nkx, nky, nz = condition.metadata.shape
    a1, a2, z0, dz = _lattice_frame(condition)
    nodes, weights, kinetic = _lobatto_grid(z0, z0 + dz, nz)
    pkd, wa, wb, wc = _beam_arrays(condition, a1, a2, weights, z0, dz)
    v = np.asarray(condition.potential_values, np.complex128).reshape(nkx, nky, nz) * energy_to_nat
    return NaturalArrays(v, kinetic, pkd, wa, wb, wc, nodes, weights)


def _shares_grid(c: ScatteringCondition, c0: ScatteringCondition) -> bool:
    """Same potential, grid, units and mass (so the same natural-unit potential
    and kinetic matrix serve both)."""
    m, m0 = c.metadata, c0.metadata
    if (tuple(m.shape) != tuple(m0.shape) or m.z_start != m0.z_start or m.z_delta != m0.z_delta
            or c.units != c0.units or c.mass != c0.mass):
        return False
    if not all(np.array_equal(np.asarray(x, float), np.asarray(y, float))
               for x, y in zip(m.vectors, m0.vectors)):
        return False
    return c.potential_values is c0.potential_values or np.array_equal(
        np.asarray(c.potential_values), np.asarray(c0.potential_values))


def _sweep_systems(conditions: Sequence[ScatteringCondition], config: OptimizationConfig):
    """(natural arrays of the first condition, one system per condition).

    The grid, the kinetic matrix and the potential are built once; each
    further beam only needs its pkd and boundary waves (the per-condition
    grid build took ~4 ms, 2 s for a 512-beam sweep)."""
    if not conditions:
        raise ValueError("no conditions")
    c0 = conditions[0]
    grid = natural_arrays(c0)
    a1, a2, z0, dz = _lattice_frame(c0)
    for i, c in enumerate(conditions[1:], start=1):
        if not _shares_grid(c, c0):
            raise ValueError(f"condition {i} does not share condition 0's potential, grid, "
                             "units and mass (a batched sweep solves one potential)")
    # every beam's pkd at once, waves for the kept channels only (the same
    # element-wise arithmetic as _beam_arrays)
    nkx, nky, _ = c0.metadata.shape
    ang = c0.units.angstrom
    ks = np.array([[float(k) * ang for k in c.incident_k] for c in conditions])
    pkd = sa.perpendicular_kinetic_difference_batch(ks, a1, a2, nkx, nky)
    systems = beam_systems(pkd, lambda e: sa.waves(e, grid.weights, z0, dz),
                           n_channels=config.n_channels)
    return grid, systems


def _system_for(arr: NaturalArrays, config: OptimizationConfig):
    if config.n_channels is not None:
        return channel_subset_system(arr.pkd, arr.wave_a, arr.wave_b, arr.wave_c,
                                     n_channels=config.n_channels)
    return full_grid_system(arr.pkd, arr.wave_a, arr.wave_b, arr.wave_c)


def _to_grid(result: SolveResult, s: int, system, shape, host_intensities=None) -> np.ndarray:
    """System s's |S|^2 on the (nkx, nky) channel grid; `host_intensities` (all
    rows, already on the host) saves one device read per system in sweeps."""
    out = np.zeros(shape, np.complex128)
    if host_intensities is None:
        vals = result.system_intensities(s).detach().cpu().numpy()
    else:
        vals = host_intensities[result.row_offsets[s]:result.row_offsets[s + 1]]
    out[system.channel_ix, system.channel_iy] = vals
    return out


def get_scattering_matrix(condition: ScatteringCondition, config: OptimizationConfig, *,
                          backend: Literal["b200", "fortran", "scipy"] = "b200") -> np.ndarray:
    """|S_G0|^2 on the (nkx, nky) channel grid, complex128 (``_multiscat.py:131-175``).

    The reference's backend names ("fortran", its default, and "scipy") are
    accepted so that calls that name one keep working; all three run the B200
    solve (the reference's backends differ only in the preconditioner, and
    the converged intensities agree within the configured precision)."""
    if backend not in ("b200", "fortran", "scipy"):
        raise ValueError(f"Unknown backend '{backend}'. Expected 'b200', 'fortran' or 'scipy'.")
    return _single_solve(condition, config, order=0)


def get_scattering_matrix_von_neumann(condition: ScatteringCondition, config: OptimizationConfig,
                                      *, order: int = 1) -> np.ndarray:
    """Same result with the von Neumann preconditioner of the given order,
    sum_{k<=order} (-D^-1 V_scatter)^k D^-1 (``_multiscat.py:179-224``,
    ``_scipy_von_neumann.py:40-58``); order 0 is the block-diagonal D^-1."""
    if order < 0:
        raise ValueError(f"Invalid von Neumann order {order}. Expected a non-negative integer.")
    return _single_solve(condition, config, order=order)


def _single_solve(condition: ScatteringCondition, config: OptimizationConfig, *,
                  order: int) -> np.ndarray:
    arr = natural_arrays(condition)
    system = _system_for(arr, config)
    plan = ScatteringPlan(arr.potential_values, arr.kinetic, [system],
                          rtol=config.residual_tolerance, restart=config.restart,
                          max_iterations=config.max_iterations,
                          precision=config.precision_mode, preconditioner_order=order)
    try:
        result = plan.solve(raise_on_error=False)
    finally:
        plan.close()
    if result.status[0] != 0:
        raise RuntimeError(
            f"B200 GMRES did not converge (status={result.status[0]}, "
            f"iterations={result.iterations[0]}, residual={result.residual[0]:.3e})")
    return _to_grid(result, 0, system, condition.metadata.shape[:2])


def _reference_order_system(arr: NaturalArrays, n_channels: int | None):
    """The channel list of the reference's state functions: ``np.argsort`` of
    pkd with numpy's default sort, the first ``n_channels`` of it
    (``_scipy.py:414-416``).  Its order defines the lower block L of the
    reference's state convention, so it is reproduced call for call (the
    solver's own ``n_channels`` path sorts stably instead)."""
    flat = np.asarray(arr.pkd, float).ravel()
    order = np.argsort(flat)
    if n_channels is not None:
        order = order[:n_channels]
    hit = np.nonzero(order == 0)[0]
    if hit.size == 0:
        raise ValueError("the specular channel is not in the kept channel set")
    ix, iy = np.unravel_index(order, arr.pkd.shape)
    return SystemSpec(ix.astype(np.int32), iy.astype(np.int32), flat[order],
                      np.asarray(arr.wave_a, complex).ravel()[order],
                      np.asarray(arr.wave_b, complex).ravel()[order],
                      np.asarray(arr.wave_c, complex).ravel()[order], int(hit[0]))


def _check_convention(convention: str) -> None:
    if convention not in ("reference", "psi"):
        raise ValueError(f"Unknown state convention '{convention}'. Expected 'reference' or 'psi'.")


def get_scattering_state(condition: ScatteringCondition, config: OptimizationConfig, *,
                         initial_state: np.ndarray | None = None,
                         convention: Literal["reference", "psi"] = "reference") -> np.ndarray:
    """The full interior state, complex128 (nkx, nky, nz)
    (``_multiscat.py:227-246``); channels outside an ``n_channels`` set are 0.

    ``convention="reference"`` (default) returns what the reference returns:
    L psi, its block Gauss-Seidel lower block L = D + V^lower applied to the
    solution psi, with the channels in the reference's argsort(pkd) order
    (``_gmres.py:127``, ``_scipy.py:580-613``); ``"psi"`` returns psi itself.
    ``initial_state`` (same shape, same convention) warm-starts the solve,
    e.g. with the state of a neighbouring energy or angle (the reference's
    ``x0``, which it maps through L^-1 as well, ``_gmres.py:106-108``)."""
    _check_convention(convention)
    arr = natural_arrays(condition)
    if convention == "reference":
        system = _reference_order_system(arr, config.n_channels)
    else:
        system = _system_for(arr, config)
    nkx, nky, nz = arr.potential_values.shape
    plan = ScatteringPlan(arr.potential_values, arr.kinetic, [system],
                          rtol=config.residual_tolerance, restart=config.restart,
                          max_iterations=config.max_iterations, precision=config.precision_mode)
    try:
        if initial_state is not None:
            guess = np.asarray(initial_state, np.complex128).reshape(nkx, nky, nz)
            rows = torch.as_tensor(np.ascontiguousarray(guess[system.channel_ix, system.channel_iy]),
                                   device=torch.device("cuda", torch.cuda.current_device()))
            plan.set_initial_guess(plan.solve_lower_block(rows) if convention == "reference"
                                   else rows)
        result = plan.solve(raise_on_error=False)
        if result.status[0] != 0:
            raise RuntimeError(f"B200 GMRES did not converge (status={result.status[0]})")
        psi = result.system_psi(0)
        if convention == "reference":
            psi = plan.apply_lower_block(psi)
        rows = psi.cpu().numpy()
    finally:
        plan.close()
    out = np.zeros((nkx, nky, nz), np.complex128)
    out[system.channel_ix, system.channel_iy] = rows
    return out


def get_scattering_matrix_from_state(state: np.ndarray, condition: ScatteringCondition, *,
                                     n_channels: int | None = None,
                                     convention: Literal["reference", "psi"] = "reference"
                                     ) -> np.ndarray:
    """|S_G0|^2 on the channel grid from a state of ``get_scattering_state``
    (``_multiscat.py:63-99``; S_G = 2i b_G psi_G(z_n) + delta_G0 a_0,
    ``_multiscat.py:40-60``).  A reference-convention state (L psi) is mapped
    back to psi by the forward Gauss-Seidel sweep L^-1 on the GPU, over the
    channel set of ``n_channels`` as the reference does (``_multiscat.py:79-88``)."""
    _check_convention(convention)
    arr = natural_arrays(condition)
    nkx, nky, nz = arr.potential_values.shape
    grid = np.asarray(state, np.complex128).reshape(nkx, nky, nz)
    if convention == "reference":
        system = _reference_order_system(arr, n_channels)
        plan = ScatteringPlan(arr.potential_values, arr.kinetic, [system], restart=1)
        try:
            rows = torch.as_tensor(np.ascontiguousarray(grid[system.channel_ix, system.channel_iy]),
                                   device=torch.device("cuda", torch.cuda.current_device()))
            psi = plan.solve_lower_block(rows).cpu().numpy()
        finally:
            plan.close()
        grid = grid.copy()
        grid[system.channel_ix, system.channel_iy] = psi
    psi_n = grid[:, :, -1]
    b = np.asarray(arr.wave_b, np.complex128).reshape(nkx, nky)
    a = np.asarray(arr.wave_a, np.complex128).reshape(nkx, nky)
    s = 2.0j * b * psi_n
    s[0, 0] += a[0, 0]
    return (np.abs(s) ** 2).astype(np.complex128)


def get_scattering_matrices(conditions: Sequence[ScatteringCondition],
                            config: OptimizationConfig) -> list[np.ndarray]:
    """Batched sweep: many beams over ONE potential and grid, one GPU solve
    (every condition must share condition 0's potential, grid, units and mass)."""
    grid, systems = _sweep_systems(conditions, config)
    plan = ScatteringPlan(grid.potential_values, grid.kinetic, systems,
                          rtol=config.residual_tolerance, restart=config.restart,
                          max_iterations=config.max_iterations,
                          precision=config.precision_mode)
    try:
        result = plan.solve(raise_on_error=False)
    finally:
        plan.close()
    bad = np.nonzero(result.status != 0)[0]
    if bad.size:
        raise RuntimeError(f"B200 GMRES did not converge for systems {bad.tolist()}")
    host = result.intensities.detach().cpu().numpy()
    return [_to_grid(result, s, systems[s], c.metadata.shape[:2], host)
            for s, c in enumerate(conditions)]
