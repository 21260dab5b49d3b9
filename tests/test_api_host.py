"""Host side of the reference-shaped API and the plan inputs (no GPU): the
state-to-intensity formula, units and condition helpers, sweeps built once
per grid, the batched channel arrays handed to the library."""

from __future__ import annotations

import math

import numpy as np
import pytest

from multiscat_b200 import setup_arrays as sa
from oracle import inputs


def test_scattering_matrix_from_state_is_the_boundary_formula():
    """get_scattering_matrix_from_state (_multiscat.py:63-99) against the oracle's
    S_G = 2i b_G psi_G(z_n) + delta_G0 a_0 on a random state of a 10x10x40 grid."""
    from multiscat_b200.api import (ScatteringCondition, ScatteringMetadata,
                                    get_scattering_matrix_from_state, natural_arrays)
    nkx, nky, nz = 10, 10, 40
    nodes, _ = inputs.lobatto_rule(0.0, 8.0, nz)
    md = ScatteringMetadata(vectors=(np.array([2.84e-10, 0.0]), np.array([0.0, 2.84e-10])),
                            shape=(nkx, nky, nz), z_delta=8e-10)
    cond = ScatteringCondition.from_angles(
        mass=sa.ALPHA_PARTICLE_MASS, theta=math.radians(30.0), phi=math.radians(15.0),
        energy=20e-3 * sa.ELECTRON_VOLT,
        potential_values=inputs.wolken_potential(nodes, nkx, nky) * sa.MEV, metadata=md)
    rng = np.random.default_rng(11)
    state = rng.normal(size=(nkx, nky, nz)) + 1j * rng.normal(size=(nkx, nky, nz))
    got = get_scattering_matrix_from_state(state, cond, convention="psi")
    assert got.dtype == np.complex128 and got.shape == (nkx, nky)
    arr = natural_arrays(cond)
    wa, wb, _ = inputs.waves(arr.pkd.ravel(), arr.weights, 0.0, 8.0)
    want = inputs.intensities(state.reshape(nkx * nky, nz), np.asarray(wa).ravel(),
                              np.asarray(wb).ravel()).reshape(nkx, nky)
    np.testing.assert_allclose(got.real, want, rtol=1e-12, atol=0)
    assert float(np.abs(got.imag).max()) == 0.0


def test_stacked_systems_match_the_per_system_arrays():
    """The batched msc_plan_set_systems input: system k's channels at
    offsets[k]..offsets[k + 1] of every concatenated array, C-ABI dtypes."""
    from multiscat_b200.solver import _stack_systems
    from multiscat_b200.workloads import cfg0_case, cfg2_batch
    systems = cfg2_batch(n_solves=3, seed=5)[1] + [cfg0_case(nz=20).system()]
    sa = _stack_systems(systems)
    off = sa["offsets"]
    assert off.dtype == np.int64 and off[0] == 0 and off.size == len(systems) + 1
    assert sa["ix"].dtype == np.int32 and sa["iy"].dtype == np.int32
    assert sa["specular"].dtype == np.int32 and sa["wb"].dtype == np.complex128
    for k, sp in enumerate(systems):
        sl = slice(off[k], off[k + 1])
        np.testing.assert_array_equal(sa["ix"][sl], sp.channel_ix)
        np.testing.assert_array_equal(sa["iy"][sl], sp.channel_iy)
        np.testing.assert_array_equal(sa["pkd"][sl], sp.pkd)
        np.testing.assert_array_equal(sa["wb"][sl], sp.wave_b)
        np.testing.assert_array_equal(sa["wc"][sl], sp.wave_c)
        assert sa["specular"][k] == sp.specular
        assert sa["a_spec"][k] == sp.wave_a[sp.specular]
    with pytest.raises(ValueError):
        _stack_systems([])


def _sweep_conditions(n: int, nz: int = 40):
    from multiscat_b200.api import ScatteringCondition, ScatteringMetadata
    nodes, _ = inputs.lobatto_rule(0.0, 8.0, nz)
    v = inputs.wolken_potential(nodes, 10, 10) * sa.MEV
    md = ScatteringMetadata(vectors=(np.array([2.84e-10, 0.0]), np.array([0.0, 2.84e-10])),
                            shape=(10, 10, nz), z_delta=8e-10)
    return [ScatteringCondition.from_angles(
        mass=sa.ALPHA_PARTICLE_MASS, theta=math.radians(5.0 + 7.0 * i),
        phi=math.radians(3.0 * i), energy=(20.0 + i) * 1e-3 * sa.ELECTRON_VOLT,
        potential_values=v, metadata=md) for i in range(n)]


@pytest.mark.parametrize("n_channels", [None, 37])
def test_sweep_systems_match_per_condition_build(n_channels):
    """get_scattering_matrices builds the grid once: every beam's system must
    equal the one the per-condition path (natural_arrays) gives."""
    from multiscat_b200.api import (OptimizationConfig, _sweep_systems, _system_for,
                                    natural_arrays)
    conds = _sweep_conditions(6)
    cfg = OptimizationConfig(n_channels=n_channels)
    grid, systems = _sweep_systems(conds, cfg)
    ref0 = natural_arrays(conds[0])
    np.testing.assert_array_equal(grid.kinetic, ref0.kinetic)
    np.testing.assert_array_equal(grid.potential_values, ref0.potential_values)
    for c, got in zip(conds, systems):
        want = _system_for(natural_arrays(c), cfg)
        for name in ("channel_ix", "channel_iy", "pkd", "wave_a", "wave_b", "wave_c"):
            np.testing.assert_array_equal(getattr(got, name), getattr(want, name))
        assert got.specular == want.specular


def test_sweep_rejects_conditions_on_another_grid():
    import dataclasses

    from multiscat_b200.api import OptimizationConfig, _sweep_systems
    conds = _sweep_conditions(3)
    other = dataclasses.replace(conds[2], mass=conds[2].mass * 2.0)
    with pytest.raises(ValueError):
        _sweep_systems([conds[0], conds[1], other], OptimizationConfig())
    shifted = dataclasses.replace(conds[1], potential_values=conds[1].potential_values * 1.5)
    with pytest.raises(ValueError):
        _sweep_systems([conds[0], shifted], OptimizationConfig())


def test_to_grid_from_host_intensities_matches_per_system_read():
    """Sweeps read all intensities once and slice them per system."""
    import torch

    from multiscat_b200.api import OptimizationConfig, _sweep_systems, _to_grid
    from multiscat_b200.solver import SolveResult
    conds = _sweep_conditions(3)
    _, systems = _sweep_systems(conds, OptimizationConfig(n_channels=30))
    offsets = np.concatenate([[0], np.cumsum([len(sp.pkd) for sp in systems])])
    inten = torch.rand(int(offsets[-1]), dtype=torch.float64)
    res = SolveResult(psi=torch.zeros(0), intensities=inten, row_offsets=offsets,
                      iterations=np.zeros(3), cycles=np.zeros(3), status=np.zeros(3),
                      residual=np.zeros(3))
    host = inten.numpy()
    for s, sp in enumerate(systems):
        a = _to_grid(res, s, sp, (10, 10))
        b = _to_grid(res, s, sp, (10, 10), host)
        np.testing.assert_array_equal(a, b)
        assert np.count_nonzero(a) == len(sp.pkd)


def test_lobatto_grid_cache_returns_fresh_copies_of_the_same_grid():
    from multiscat_b200 import api
    a = api._lobatto_grid(-1.5, 10.0, 33)
    b = api._lobatto_grid(-1.5, 10.0, 33)
    x, w = sa.lobatto_rule(-1.5, 10.0, 33)
    np.testing.assert_array_equal(a[0], x)
    np.testing.assert_array_equal(a[1], w)
    np.testing.assert_array_equal(a[2], sa.kinetic_matrix(x, w))
    for p, q in zip(a, b):
        np.testing.assert_array_equal(p, q)
        assert p is not q
    a[2][0, 0] = 1e9                      # a caller's change does not reach the cache
    assert api._lobatto_grid(-1.5, 10.0, 33)[2][0, 0] == b[2][0, 0]
    for n in range(2, 2 + api._GRID_CACHE_SIZE + 3):
        api._lobatto_grid(0.0, 1.0, n)
    assert len(api._GRID_CACHE) <= api._GRID_CACHE_SIZE


def test_unknown_backend_is_rejected_before_any_solve():
    from multiscat_b200.api import OptimizationConfig, get_scattering_matrix
    with pytest.raises(ValueError, match="Unknown backend"):
        get_scattering_matrix(_sweep_conditions(1)[0], OptimizationConfig(), backend="cuda")


def test_unit_system_and_condition_helpers():
    """UnitSystem.si / electron_volt and ScatteringCondition.theta / phi /
    with_units / == (config.py:61-84, 180-296)."""
    from multiscat_b200.api import UnitSystem, natural_arrays
    si = UnitSystem.si()
    assert si == UnitSystem() and math.isclose(si.electron_volt, sa.ELECTRON_VOLT, rel_tol=1e-15)
    nat_units = UnitSystem(hbar=1.0, atomic_mass=1.0, angstrom=1.0)
    # the reference's definition, eV_SI * keu_SI / keu
    assert math.isclose(nat_units.electron_volt,
                        sa.ELECTRON_VOLT * si.kinetic_energy_unit / 0.5, rel_tol=1e-12)
    energy_factor = nat_units.kinetic_energy_unit / si.kinetic_energy_unit
    c = _sweep_conditions(4)[3]
    assert math.isclose(c.theta, math.radians(26.0), rel_tol=1e-12)
    assert math.isclose(c.phi, math.radians(9.0), rel_tol=1e-12)
    other = c.with_units(nat_units)
    assert other.units == nat_units and other != c
    assert math.isclose(other.theta, c.theta, rel_tol=1e-12)
    assert math.isclose(other.incident_energy, c.incident_energy * energy_factor, rel_tol=1e-12)
    a, b = natural_arrays(c), natural_arrays(other)
    for name in ("potential_values", "kinetic", "pkd", "wave_a", "wave_b", "wave_c", "nodes"):
        np.testing.assert_allclose(getattr(b, name), getattr(a, name), rtol=1e-9,
                                   atol=1e-12 * np.abs(getattr(a, name)).max())
    back = other.with_units(si)
    assert math.isclose(back.mass, c.mass, rel_tol=1e-15)
    assert c == _sweep_conditions(4)[3]


@pytest.mark.parametrize("mode", ["max_pkd", "n_channels", "full"])
def test_beam_systems_match_per_beam_builders(mode):
    """solver.beam_systems (all beams at once, waves for kept channels only)
    against channel_subset_system / full_grid_system beam by beam."""
    from multiscat_b200.solver import beam_systems, channel_subset_system, full_grid_system
    fac = sa.natural_units_factor(sa.HE4_MASS)
    a1, a2 = np.array([2.54, 0.0]), np.array([0.0, 2.54])
    x, w = sa.lobatto_rule(-1.5, 10.0, 50)
    rng = np.random.default_rng(9)
    ks = [sa.momentum_from_angles(e, th, ph, fac) for e, th, ph in
          zip(rng.uniform(8, 64, 12), np.radians(rng.uniform(0, 60, 12)),
              np.radians(rng.uniform(0, 45, 12)))]
    pkd = sa.perpendicular_kinetic_difference_batch(ks, a1, a2, 16, 16)
    kw = {"max_pkd": {"max_pkd": fac * 120.0}, "n_channels": {"n_channels": 57}, "full": {}}[mode]
    got = beam_systems(pkd, lambda e: sa.waves(e, w, -1.5, 11.5), **kw)
    for k, sp in zip(ks, got):
        p1 = sa.perpendicular_kinetic_difference(k, a1, a2, 16, 16)
        wa, wb, wc = sa.waves(p1, w, -1.5, 11.5)
        want = (full_grid_system(p1, wa, wb, wc) if mode == "full"
                else channel_subset_system(p1, wa, wb, wc, **kw))
        for name in ("channel_ix", "channel_iy", "pkd", "wave_a", "wave_b", "wave_c"):
            np.testing.assert_array_equal(getattr(sp, name), getattr(want, name))
        assert sp.specular == want.specular
    with pytest.raises(ValueError):
        beam_systems(pkd, lambda e: sa.waves(e, w, -1.5, 11.5), max_pkd=-1e9)


def test_reference_order_system_is_the_reference_channel_list():
    """The state convention's channel list: numpy's default argsort of pkd, the
    first n_channels of it (_scipy.py:414-416), specular located in it."""
    from multiscat_b200.api import _reference_order_system
    from multiscat_b200.workloads import cfg0_case
    case = cfg0_case(nz=20)

    class Arr:
        pkd, wave_a, wave_b, wave_c = case.pkd, case.wa, case.wb, case.wc
    for n_channels in (None, 40):
        sp = _reference_order_system(Arr, n_channels)
        order = np.argsort(case.pkd.ravel())
        if n_channels:
            order = order[:n_channels]
        assert np.array_equal(sp.channel_ix * 11 + sp.channel_iy, order)
        assert np.array_equal(sp.pkd, case.pkd.ravel()[order])
        assert sp.channel_ix[sp.specular] == 0 and sp.channel_iy[sp.specular] == 0
        assert np.array_equal(sp.wave_c, np.asarray(case.wc).ravel()[order])
    with pytest.raises(ValueError):
        from multiscat_b200.api import _check_convention
        _check_convention("lpsi")


def test_bench_kernel_records_classify_each_kernel_by_its_bound():
    """bench.py's roofline arithmetic on a synthetic result: the coupling and
    the SIMT block inverse are FMA-bound, the tcgen05 block inverse tensor-bound,
    the Arnoldi passes HBM-bound with one pass per Krylov vector row touched."""
    import importlib.util
    import pathlib
    spec = importlib.util.spec_from_file_location(
        "bench", pathlib.Path(__file__).resolve().parents[1] / "bench.py")
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)

    class Res:
        row_offsets = np.array([0, 100, 300])
        iterations = np.array([10, 20])
        basis_vectors = np.array([55, 150])
        cycles = np.array([2, 3])
    kt = {k: {"ms": 1.0, "launches": 10} for k in
          ("block_inverse", "coupling", "arnoldi_project", "arnoldi_update_project")}
    peaks = {"hbm_gbs": 6000.0, "bf16_tflops": 1600.0, "bf16_tflops_sustained": 1400.0}
    fma = {"fp32": 70.0, "fp64": 35.0}
    n, taps = 150, 80
    rec = bench.kernel_records(kt, Res, n, taps, True, True, True, peaks, fma, "cfg2")
    steps_rows = 100 * 10 + 200 * 20
    vec_rows = 100 * 55 + 200 * 150
    assert rec["coupling"]["bound"] == "fma" and rec["coupling"]["peak"] == 70.0
    assert rec["coupling"]["achieved"] == pytest.approx(8 * taps * n * steps_rows / 1e-3 / 1e12)
    bi = rec["block_inverse"]
    assert bi["bound"] == "tensor" and bi["peak"] == 1400.0
    assert bi["achieved"] == pytest.approx(24 * n * n * (steps_rows + 100 * 2 + 200 * 3) / 1e-3 / 1e12)
    red = rec["arnoldi_project"]
    assert red["bound"] == "hbm"
    assert red["achieved"] == pytest.approx((vec_rows + steps_rows) * n * 8 / 1e-3 / 1e9)
    upd = rec["arnoldi_update_project"]
    assert upd["achieved"] == pytest.approx((vec_rows + 3 * steps_rows) * n * 8 / 1e-3 / 1e9)
    for r in rec.values():
        assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    simt = bench.kernel_records(kt, Res, n, taps, False, False, False, peaks, fma, "cfg2")
    assert simt["block_inverse"]["bound"] == "fma" and simt["block_inverse"]["peak"] == 35.0
    sep = bench.kernel_records(kt, Res, n, taps, True, True, True, peaks, fma, "cfg2", (4, 4))
    per_row = 8 * (9 * 16 / 8 + 10) * n                       # 28 complex MACs per output
    fl, nb = per_row * steps_rows, 3 * 8 * n * steps_rows
    c = sep["coupling"]
    assert c["bound"] == ("fma" if fl / 70e12 >= nb / 6000e9 else "hbm")
    want = fl / 1e-3 / 1e12 if c["bound"] == "fma" else nb / 1e-3 / 1e9
    assert c["achieved"] == pytest.approx(want)
