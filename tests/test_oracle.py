"""CPU tests of the oracle itself: pinned to the reference's golden vectors.

The oracle (oracle/msc_oracle.c + oracle/inputs.py) restates the reference's
Fortran solve.  Before it is trusted as the checker it must reproduce:
- the reference's golden intensities for the He-LiF Wolken case
  (tests/test_fixed_example.py:233-256: flux 1 within 1e-6, intensities
  within 1e-5 absolute).  The 20-degree rotated-lattice variant (:307-330)
  is an API-level property (incident k is taken in the lattice frame) and is
  tested on the package's own API;
- the potential convention of tests/data/expected_potential.npy (:599-607);
- its own internal identities (eigenpairs, L L^-1 = I as :610-635).
"""

from __future__ import annotations

import json
import math
import pathlib

import numpy as np
import pytest

from oracle import inputs, solver

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def read_wolken_golden(shape=(10, 10)) -> np.ndarray:
    out = np.zeros(shape)
    for line in (GOLDEN / "wolken_expected_intensities.txt").read_text().splitlines():
        if not line.strip() or line.lstrip().startswith("#"):
            continue
        hx, ky, val = line.split()[:3]
        out[int(hx) % shape[0], int(ky) % shape[1]] = float(val)
    return out


def wolken_inputs(rotation_deg: float = 0.0):
    mass = inputs.ALPHA_PARTICLE_MASS_KG
    fac = inputs.natural_units_factor(mass)
    k = math.sqrt(fac * 20.0)
    th = math.radians(30.0)
    kin = (k * math.sin(th), 0.0, k * math.cos(th))
    nodes, w = inputs.lobatto_rule(0.0, 8.0, 550)
    t = inputs.kinetic_matrix(nodes, w)
    v = inputs.wolken_potential(nodes, 10, 10) * fac
    rot = math.radians(rotation_deg)
    rm = np.array([[math.cos(rot), -math.sin(rot)], [math.sin(rot), math.cos(rot)]])
    a1 = rm @ np.array([2.84, 0.0])
    a2 = rm @ np.array([0.0, 2.84])
    pkd = inputs.perpendicular_kinetic_difference(kin, a1, a2, 10, 10)
    a, b, c = inputs.waves(pkd, w, 0.0, 8.0)
    return v, pkd, a, b, c, t


def test_potential_convention_matches_reference_fixture():
    samples = json.loads((GOLDEN / "wolken_potential_samples.json").read_text())
    nodes, _ = inputs.lobatto_rule(0.0, 8.0, 550)
    model = inputs.wolken_potential(nodes, 10, 10)
    idx = samples["nodes_index"]
    np.testing.assert_allclose(model[0, 0, idx].real, samples["v00"], rtol=1e-12)
    np.testing.assert_allclose(model[1, 0, idx].real, samples["v10"], rtol=1e-12)
    np.testing.assert_allclose(model[0, 1, idx].real, samples["v01"], rtol=1e-12)
    np.testing.assert_allclose(model[9, 0, idx].real, samples["v90"], rtol=1e-12)
    assert samples["max_abs_other_modes"] < 1e-11
    assert samples["closed_form_max_rel_dev"] < 1e-12


def test_oracle_reproduces_reference_golden_intensities():
    v, pkd, a, b, c, t = wolken_inputs()
    psi = solver.run_multiscat_fortran(1, 5, v, pkd, a, b, c, t)
    inten = inputs.intensities(psi.reshape(-1, 550), a, b).reshape(10, 10)
    assert math.isclose(inten.sum(), 1.0, abs_tol=1e-6)
    np.testing.assert_allclose(inten, read_wolken_golden(), rtol=0.0, atol=1e-5)


def test_oracle_without_neumann_flag_agrees():
    v, pkd, a, b, c, t = wolken_inputs()
    psi1 = solver.run_multiscat_fortran(1, 8, v, pkd, a, b, c, t)
    psi0 = solver.run_multiscat_fortran(0, 8, v, pkd, a, b, c, t)
    i1 = inputs.intensities(psi1.reshape(-1, 550), a, b)
    i0 = inputs.intensities(psi0.reshape(-1, 550), a, b)
    np.testing.assert_allclose(i0, i1, atol=1e-8)


def test_oracle_bad_dims_raise_code_1():
    with pytest.raises(RuntimeError, match="error code 1"):
        solver.run_multiscat_fortran(1, 5, np.zeros((0, 1, 4), complex), np.zeros((0, 1)),
                                     np.zeros(0), np.zeros(0), np.zeros(0), np.eye(4))


def test_oracle_eigh_matches_lapack():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((60, 60))
    a = a + a.T
    w, z = solver.eigh(a)
    w_ref = np.linalg.eigvalsh(a)
    np.testing.assert_allclose(w, w_ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(z @ np.diag(w) @ z.T, a, atol=1e-11)
    np.testing.assert_allclose(z.T @ z, np.eye(60), atol=1e-12)


def test_oracle_upper_block_matches_definition():
    rng = np.random.default_rng(5)
    nkx, nky, nz = 4, 3, 6
    v = rng.standard_normal((nkx, nky, nz)) + 1j * rng.standard_normal((nkx, nky, nz))
    x = rng.standard_normal((nkx * nky, nz)) + 1j * rng.standard_normal((nkx * nky, nz))
    got = solver.apply_upper(v, x)
    ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
    ix, iy = ix.ravel(), iy.ravel()
    want = np.zeros_like(x)
    for j in range(nkx * nky):
        for i in range(j + 1, nkx * nky):
            want[j] += v[(ix[j] - ix[i]) % nkx, (iy[j] - iy[i]) % nky] * x[i]
    np.testing.assert_allclose(got, want, rtol=1e-13, atol=1e-13)


def test_oracle_lower_solve_inverts_lower_operator():
    """L (L^-1 x) = x with L = D + V_lower (reference test :610-635, at 1e-10 here)."""
    rng = np.random.default_rng(7)
    nkx, nky, nz = 3, 3, 12
    nodes, w = inputs.lobatto_rule(0.0, 6.0, nz)
    t = inputs.kinetic_matrix(nodes, w)
    v = 0.05 * (rng.standard_normal((nkx, nky, nz)) + 1j * rng.standard_normal((nkx, nky, nz)))
    v[0, 0] = 2.0 + 0.1 * rng.standard_normal(nz)
    pkd = rng.uniform(-3.0, 8.0, (nkx, nky))
    _, _, c = inputs.waves(pkd, w, 0.0, 6.0)
    x = rng.standard_normal((nkx * nky, nz)) + 1j * rng.standard_normal((nkx * nky, nz))
    y = solver.solve_lower(v, pkd, c, t, x)
    ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
    ix, iy = ix.ravel(), iy.ravel()
    lx = np.zeros_like(x)
    pk = pkd.ravel()
    for j in range(nkx * nky):
        d = t @ y[j] + (v[0, 0].real + pk[j]) * y[j]
        d[-1] -= c[j] * y[j, -1]
        lx[j] = d
        for i in range(j):
            lx[j] += v[(ix[j] - ix[i]) % nkx, (iy[j] - iy[i]) % nky] * y[i]
    np.testing.assert_allclose(lx, x, rtol=1e-10, atol=1e-10)


def test_golden_oracle_fixtures_are_converged():
    cfg0 = json.loads((GOLDEN / "oracle_cfg0.json").read_text())
    assert cfg0["info"] == 0
    assert abs(cfg0["flux"] - 1.0) < 1e-11
    for rec in json.loads((GOLDEN / "oracle_subsets.json").read_text()):
        assert rec["info"] == 0
        assert abs(rec["flux"] - 1.0) < 1e-11


def test_cfg3_fd_fixture_consistent_with_cfg1_fixture():
    """The oracle FD fixture's base loss is sum_G w_G I_G of the cfg1 oracle
    intensities (same system, independent runs at 1e-10 and 5e-14)."""
    path = GOLDEN / "oracle_cfg3_fd.json"
    if not path.exists():
        pytest.skip("oracle_cfg3_fd.json not generated")
    from multiscat_b200.workloads import cfg3_problem
    fd = json.loads(path.read_text())
    cfg1 = json.loads((GOLDEN / "oracle_cfg1.json").read_text())
    w = cfg3_problem().weights
    assert fd["all_converged"]
    assert abs(float(np.dot(w, cfg1["intensities"])) - fd["loss"]) < 1e-8
    for rec in list(fd["params"].values()) + fd["components"]:
        assert math.isfinite(rec["dL"])
