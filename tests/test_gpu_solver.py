"""GPU parity tests: the CUDA solver against the oracle (CPU restatement of the
reference solve) and the reference's own golden vectors.

Tolerances (plain FP64 form): max |Delta |S_G0|^2| <= 1e-8 against the oracle
run at precision <= 1e-10, and |sum |S|^2 - 1| <= 1e-8; operator kernels match
a numpy FP64 restatement to 1e-12 relative.
"""

from __future__ import annotations

import json
import math
import pathlib

import numpy as np
import pytest
import torch

from multiscat_b200 import (OptimizationConfig, ScatteringCondition, ScatteringMetadata,
                            ScatteringPlan, full_grid_system, get_scattering_matrix,
                            run_multiscat_fortran)
from multiscat_b200 import setup_arrays as sa
from multiscat_b200.workloads import cfg0_case, cfg1_case, cfg2_batch, wolken_case, wolken_potential

pytestmark = pytest.mark.gpu

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
INTENSITY_TOL = 1e-8
FLUX_TOL = 1e-8


def _numpy_operators(case):
    """FP64 numpy restatement of coupling, D and D^-1 for a full-grid system."""
    nkx, nky, nz = case.v.shape
    ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
    ix, iy = ix.ravel(), iy.ravel()
    pk = case.pkd.ravel()
    c = case.wc

    def coupling(x):
        y = np.zeros_like(x)
        for j in range(nkx * nky):
            dx = (ix[j] - ix) % nkx
            dy = (iy[j] - iy) % nky
            taps = case.v[dx, dy]                 # [C, nz]
            taps[j] = 0.0
            y[j] = (taps * x).sum(axis=0)
        return y

    def diag(x):
        y = x @ case.t.T + (case.v[0, 0].real[None, :] + pk[:, None]) * x
        y[:, -1] -= c * x[:, -1]
        return y

    def block_inverse(x):
        out = np.empty_like(x)
        for j in range(nkx * nky):
            m = case.t + np.diag(case.v[0, 0].real + pk[j])
            m = m.astype(complex)
            m[-1, -1] -= c[j]
            out[j] = np.linalg.solve(m, x[j])
        return out

    return coupling, diag, block_inverse


@pytest.fixture(scope="module")
def cfg0():
    return cfg0_case()


def test_operator_kernels_match_numpy(cfg0):
    coupling, diag, block_inverse = _numpy_operators(cfg0)
    plan = ScatteringPlan(cfg0.v, cfg0.t, [cfg0.system()])
    rng = np.random.default_rng(11)
    x = rng.standard_normal((121, 100)) + 1j * rng.standard_normal((121, 100))
    xt = torch.as_tensor(x, device="cuda")
    y_c = plan.apply_coupling(xt).cpu().numpy()
    want_c = coupling(x)
    np.testing.assert_allclose(y_c, want_c, rtol=1e-12, atol=1e-12 * np.abs(want_c).max())
    y_a = plan.apply_operator(xt).cpu().numpy()
    want_a = diag(x) + want_c
    np.testing.assert_allclose(y_a, want_a, rtol=1e-11, atol=1e-11 * np.abs(want_a).max())
    y_i = plan.apply_block_inverse(xt).cpu().numpy()
    want_i = block_inverse(x)
    np.testing.assert_allclose(y_i, want_i, rtol=1e-9, atol=1e-11 * np.abs(want_i).max())
    plan.close()


def test_cfg0_solve_matches_oracle(cfg0):
    golden = json.loads((GOLDEN / "oracle_cfg0.json").read_text())
    plan = ScatteringPlan(cfg0.v, cfg0.t, [cfg0.system()], rtol=1e-10)
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    assert res.status[0] == 0
    assert res.residual[0] <= 1e-10
    np.testing.assert_allclose(inten, golden["intensities"], rtol=0.0, atol=INTENSITY_TOL)
    assert abs(inten.sum() - 1.0) <= FLUX_TOL
    plan.close()


def test_drop_in_run_multiscat_fortran_matches_oracle(cfg0):
    from oracle import inputs as oin
    from oracle import solver as osol
    psi = run_multiscat_fortran(1, 10, cfg0.v, cfg0.pkd, cfg0.wa, cfg0.wb, cfg0.wc, cfg0.t)
    assert psi.shape == (11, 11, 100) and psi.dtype == np.complex128
    psi_o = osol.run_multiscat_fortran(1, 12, cfg0.v, cfg0.pkd, cfg0.wa, cfg0.wb, cfg0.wc, cfg0.t)
    i = oin.intensities(psi.reshape(121, 100), cfg0.wa, cfg0.wb)
    io = oin.intensities(psi_o.reshape(121, 100), cfg0.wa, cfg0.wb)
    np.testing.assert_allclose(i, io, rtol=0.0, atol=INTENSITY_TOL)
    # psi itself (interior wave function) agrees with the reference solve too
    np.testing.assert_allclose(psi, psi_o, rtol=0.0, atol=1e-7 * np.abs(psi_o).max())


def test_drop_in_not_converged_raises_code_2(cfg0):
    """A limit that cannot be met maps to the reference's ierr = 2."""
    lib_plan = ScatteringPlan(cfg0.v, cfg0.t, [cfg0.system()], rtol=1e-10, max_iterations=2)
    res = lib_plan.solve(raise_on_error=False)
    assert res.status[0] == 2
    with pytest.raises(RuntimeError):
        lib_plan.solve(raise_on_error=True)
    lib_plan.close()


def _wolken_condition(rotation_deg: float):
    nodes, _ = sa.lobatto_rule(0.0, 8.0, 550)
    v_joule = wolken_potential(nodes, 10, 10) * sa.MEV
    rot = math.radians(rotation_deg)
    rm = np.array([[math.cos(rot), -math.sin(rot)], [math.sin(rot), math.cos(rot)]])
    md = ScatteringMetadata(vectors=(rm @ np.array([2.84e-10, 0.0]), rm @ np.array([0.0, 2.84e-10])),
                            shape=(10, 10, 550), z_delta=8e-10)
    return ScatteringCondition.from_angles(mass=sa.ALPHA_PARTICLE_MASS, theta=math.radians(30.0),
                                           phi=0.0, energy=20e-3 * sa.ELECTRON_VOLT,
                                           potential_values=v_joule, metadata=md)


def _read_wolken_golden():
    out = np.zeros((10, 10))
    for line in (GOLDEN / "wolken_expected_intensities.txt").read_text().splitlines():
        if line.strip() and not line.lstrip().startswith("#"):
            hx, ky, val = line.split()[:3]
            out[int(hx) % 10, int(ky) % 10] = float(val)
    return out


def test_batched_sweep_matches_single_beam_calls():
    """get_scattering_matrices (one plan, grid built once) against
    get_scattering_matrix per beam, three incidence angles of the He-LiF case."""
    from multiscat_b200 import get_scattering_matrices
    base = _wolken_condition(0.0)
    conds = [ScatteringCondition.from_angles(
        mass=sa.ALPHA_PARTICLE_MASS, theta=math.radians(th), phi=math.radians(ph),
        energy=20e-3 * sa.ELECTRON_VOLT, potential_values=base.potential_values,
        metadata=base.metadata) for th, ph in ((30.0, 0.0), (20.0, 10.0), (40.0, 5.0))]
    cfg = OptimizationConfig(precision=1e-7, max_iterations=1000)
    batch = get_scattering_matrices(conds, cfg)
    for c, got in zip(conds, batch):
        want = get_scattering_matrix(c, cfg)
        np.testing.assert_allclose(got.real, want.real, rtol=0.0, atol=1e-9)


@pytest.mark.parametrize("rotation,backend", [(0.0, "b200"), (20.0, "b200"), (0.0, "fortran"),
                                              (0.0, "scipy")])
def test_api_reproduces_reference_golden(rotation, backend):
    """tests/test_fixed_example.py:233-256 and :307-330 on the B200 API (the
    reference's backend names run the same solve)."""
    s = get_scattering_matrix(_wolken_condition(rotation),
                              OptimizationConfig(precision=1e-5, max_iterations=1000),
                              backend=backend)
    assert s.dtype == np.complex128 and s.shape == (10, 10)
    inten = np.real_if_close(s)
    assert math.isclose(float(np.sum(inten).real), 1.0, abs_tol=1e-6)
    np.testing.assert_allclose(inten.real, _read_wolken_golden(), rtol=0.0, atol=1e-5)


def test_wolken_matches_oracle_tightly():
    from oracle import inputs as oin
    from oracle import solver as osol
    case = wolken_case()
    plan = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-11)
    inten = plan.solve().intensities.cpu().numpy()
    plan.close()
    psi_o = osol.run_multiscat_fortran(1, 12, case.v, case.pkd, case.wa, case.wb, case.wc, case.t)
    io = oin.intensities(psi_o.reshape(100, 550), case.wa, case.wb)
    np.testing.assert_allclose(inten, io, rtol=0.0, atol=INTENSITY_TOL)
    assert abs(inten.sum() - 1.0) <= FLUX_TOL


def test_batched_channel_subsets_match_oracle():
    golden = json.loads((GOLDEN / "oracle_subsets.json").read_text())
    systems = []
    case = None
    for rec in golden:
        case, sys_list = cfg2_batch(n_solves=2, seed=rec["seed"])
        systems.append(sys_list[0])
    # uneven batch: both beams plus a repeat of the first
    plan = ScatteringPlan(case.v, case.t, systems + [systems[0]], rtol=1e-10)
    res = plan.solve()
    assert (res.status == 0).all()
    for s, rec in enumerate(golden):
        got = res.system_intensities(s).cpu().numpy()
        assert got.size == rec["n_channels"]
        np.testing.assert_allclose(got, rec["intensities"], rtol=0.0, atol=INTENSITY_TOL)
        assert abs(got.sum() - 1.0) <= FLUX_TOL
    # a system's answer does not depend on its batch neighbours
    assert torch.equal(res.system_intensities(0), res.system_intensities(2))
    plan.close()


def test_cfg1_matches_oracle_golden():
    path = GOLDEN / "oracle_cfg1.json"
    if not path.exists():
        pytest.skip("oracle_cfg1.json not generated")
    golden = json.loads(path.read_text())
    case = cfg1_case()
    plan = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-10)
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    np.testing.assert_allclose(inten, golden["intensities"], rtol=0.0, atol=INTENSITY_TOL)
    assert abs(inten.sum() - 1.0) <= FLUX_TOL
    plan.close()


def test_nonfinite_potential_is_rejected(cfg0):
    v = cfg0.v.copy()
    v[1, 0, 5] = np.nan
    with pytest.raises(RuntimeError, match="status 4"):
        ScatteringPlan(v, cfg0.t, [cfg0.system()])


# ---------------------------------------------------------------------------
# Mixed form: FP32 inner GMRES inside FP64 iterative refinement.  Bar:
# max |Delta |S|^2| <= 1e-6 against the FP64 oracle (and flux within 1e-6);
# the refinement drives the FP64 true residual to the same rtol as the plain
# form, so in practice the error is far smaller.
# ---------------------------------------------------------------------------
MIXED_TOL = 1e-6


def test_mixed_cfg0_matches_oracle(cfg0):
    golden = json.loads((GOLDEN / "oracle_cfg0.json").read_text())
    plan = ScatteringPlan(cfg0.v, cfg0.t, [cfg0.system()], rtol=1e-10, precision="mixed")
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    assert res.status[0] == 0
    assert res.residual[0] <= 1e-10
    np.testing.assert_allclose(inten, golden["intensities"], rtol=0.0, atol=MIXED_TOL)
    assert abs(inten.sum() - 1.0) <= MIXED_TOL
    plan.close()


@pytest.mark.parametrize("passes", [1, 2])
def test_mixed_cfg1_matches_oracle(passes):
    path = GOLDEN / "oracle_cfg1.json"
    if not path.exists():
        pytest.skip("oracle_cfg1.json not generated")
    golden = json.loads(path.read_text())
    case = cfg1_case()
    plan = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-10, precision="mixed",
                          inner_gram_schmidt_passes=passes)
    res = plan.solve()
    inten = res.intensities.cpu().numpy()
    assert res.status[0] == 0
    np.testing.assert_allclose(inten, golden["intensities"], rtol=0.0, atol=MIXED_TOL)
    assert abs(inten.sum() - 1.0) <= MIXED_TOL
    plan.close()


@pytest.mark.parametrize("passes", [1, 2])
def test_mixed_batched_subsets_match_oracle_and_fp64(passes):
    golden = json.loads((GOLDEN / "oracle_subsets.json").read_text())
    systems = []
    case = None
    for rec in golden:
        case, sys_list = cfg2_batch(n_solves=2, seed=rec["seed"])
        systems.append(sys_list[0])
    mixed = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed",
                           inner_gram_schmidt_passes=passes)
    fp64 = ScatteringPlan(case.v, case.t, systems, rtol=1e-10)
    rm = mixed.solve()
    rf = fp64.solve()
    for s, rec in enumerate(golden):
        got = rm.system_intensities(s).cpu().numpy()
        np.testing.assert_allclose(got, rec["intensities"], rtol=0.0, atol=MIXED_TOL)
        np.testing.assert_allclose(got, rf.system_intensities(s).cpu().numpy(), rtol=0.0,
                                   atol=MIXED_TOL)
    mixed.close()
    fp64.close()


# ---------------------------------------------------------------------------
# tcgen05 BF16x3 block inverse (mixed form) against the FP64 kernel.  BF16x3
# keeps ~16 bits per operand, so the tolerance is 2e-4 relative to the
# largest entry of the output row set.
# ---------------------------------------------------------------------------
TC_TOL = 2e-4


@pytest.mark.parametrize("which", ["cfg0", "cfg1", "cfg2"])
def test_tensor_core_block_inverse_matches_fp64(which):
    if which == "cfg0":
        case = cfg0_case()
        systems = [case.system()]
    elif which == "cfg1":
        case = cfg1_case()
        systems = [case.system()]
    else:
        case, systems = cfg2_batch(n_solves=5, seed=3)
    mixed = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=True)
    simt = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=False)
    rows = mixed.total_rows
    rng = np.random.default_rng(17)
    x = rng.standard_normal((rows, case.v.shape[2])) + 1j * rng.standard_normal((rows, case.v.shape[2]))
    x32 = torch.as_tensor(x.astype(np.complex64), device="cuda")
    y_tc = mixed.apply_block_inverse_f32(x32).cpu().numpy()
    assert mixed.tensor_core_tile > 0, "tcgen05 path not selected"
    y_simt = simt.apply_block_inverse_f32(x32).cpu().numpy()
    assert simt.tensor_core_tile == 0
    scale = np.abs(y_simt).max()
    np.testing.assert_allclose(y_tc, y_simt, rtol=0, atol=TC_TOL * scale)
    if len(systems) == 1:
        fp64 = ScatteringPlan(case.v, case.t, systems)
        y64 = fp64.apply_block_inverse(torch.as_tensor(x32.cpu().numpy().astype(np.complex128),
                                                       device="cuda")).cpu().numpy()
        np.testing.assert_allclose(y_tc, y64, rtol=0, atol=TC_TOL * scale)
        fp64.close()
    mixed.close()
    simt.close()


def test_mixed_odd_node_count_matches_fp64():
    """nz = 41 with an odd row total (11 x 11 channels): the FP32 basis vectors
    then start on odd elements (8-byte aligned only), so the paired 16-byte
    load paths of the Arnoldi and update kernels must step aside."""
    case = cfg0_case(nz=41)
    systems = [case.system()]
    assert len(systems[0].pkd) * 41 % 2 == 1
    ref = ScatteringPlan(case.v, case.t, systems).solve().intensities
    for tc in (True, False):
        res = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=tc).solve()
        assert (res.status == 0).all(), (tc, res.status)
        assert float((res.intensities - ref).abs().max()) <= MIXED_TOL


@pytest.mark.parametrize("groups,width", [(1, 16), (1, 32), (1, 64), (1, 128),
                                          (2, 16), (2, 32), (2, 64), (3, 128)])
def test_tensor_core_width_and_warp_groups_match_simt(groups, width, monkeypatch):
    """Every tcgen05 variant the autotuner can pick (tile width N; one tile
    loop per CTA, two warp groups with their own, or the channel-major
    kernel, bg=3), forced through MSC_TUNE, on a 24-beam batch with enough
    rows for every width."""
    case, systems = cfg2_batch(n_solves=24, seed=3)
    rng = np.random.default_rng(19)
    # a plan reads MSC_TUNE when its first call sets it up
    monkeypatch.setenv("MSC_TUNE", f"c64=2,c32=2,bi={width},bg={groups}")
    mixed = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=True)
    shape = (mixed.total_rows, case.v.shape[2])
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    x32 = torch.as_tensor(x.astype(np.complex64), device="cuda")
    y_tc = mixed.apply_block_inverse_f32(x32).cpu().numpy()
    monkeypatch.setenv("MSC_TUNE", "c64=2,c32=2,bi=0")
    simt = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=False)
    y_simt = simt.apply_block_inverse_f32(x32).cpu().numpy()
    assert mixed.tensor_core_tile == width
    tag = "tcc" if groups == 3 else ("tc2_N" if groups == 2 else "tc_N") + str(width)
    assert f"block_inverse32={tag}" in mixed.tuning_report()["chosen"]
    scale = np.abs(y_simt).max()
    np.testing.assert_allclose(y_tc, y_simt, rtol=0, atol=TC_TOL * scale)
    # a whole mixed solve on this variant against FP64
    ref = ScatteringPlan(case.v, case.t, systems).solve().intensities
    res = mixed.solve()
    assert (res.status == 0).all()
    assert float((res.intensities - ref).abs().max()) <= MIXED_TOL
    mixed.close()
    simt.close()


# ---------------------------------------------------------------------------
# cfg4 shape: 81 x 81 channels, 300 nodes, |m|,|n| <= 8 (288 taps, halo 8),
# several azimuths batched.  No oracle here (the CPU restatement would need
# tens of GB); the check is mixed vs the plain FP64 form, plus flux.
# ---------------------------------------------------------------------------
def test_cfg4_batch_mixed_matches_fp64():
    from multiscat_b200.workloads import cfg4_batch
    case, systems = cfg4_batch(n_azimuths=4)
    fp64 = ScatteringPlan(case.v, case.t, systems, rtol=1e-10)
    r64 = fp64.solve()
    assert (r64.status == 0).all()
    fp64.close()
    mixed = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed")
    rm = mixed.solve()
    assert (rm.status == 0).all()
    d = (rm.intensities - r64.intensities).abs().max().item()
    assert d <= MIXED_TOL, d
    for s in range(len(systems)):
        inten = r64.system_intensities(s).cpu().numpy()
        assert abs(inten.sum() - 1.0) <= 1e-8
    mixed.close()


# ---------------------------------------------------------------------------
# Every coupling kernel the autotuner can pick (forced through MSC_TUNE):
# FP64 operators against the neighbour-table kernel, and mixed solves of a
# small uneven batch against the FP64 solve.
# ---------------------------------------------------------------------------
COUPLING_KINDS = {0: "neighbour", 1: "halo_y8", 2: "halo_y4", 3: "separable", 4: "separable_z2",
                  5: "separable_rows"}


@pytest.mark.parametrize("kind", sorted(COUPLING_KINDS))
def test_every_coupling_kernel_agrees(kind, monkeypatch):
    case, systems = cfg2_batch(n_solves=5, seed=4)
    monkeypatch.setenv("MSC_TUNE", f"c64={kind},c32={kind},bi=128")
    plan = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed")
    res = plan.solve()
    assert plan.tuning_report()["chosen"].startswith(f"coupling64={COUPLING_KINDS[kind]},"
                                                     f"coupling32={COUPLING_KINDS[kind]}")
    monkeypatch.setenv("MSC_TUNE", "c64=0,c32=0,bi=128")
    ref = ScatteringPlan(case.v, case.t, systems, rtol=1e-10).solve()
    assert (res.status == 0).all()
    d = (res.intensities - ref.intensities).abs().max().item()
    assert d <= MIXED_TOL, d
    plan.close()
    # FP64 operator of one full-grid system with this kind vs the neighbour
    # table (a plan reads MSC_TUNE when its first call sets it up)
    c0 = cfg0_case(nz=48)
    x = torch.randn(c0.pkd.size, 48, dtype=torch.complex128, device="cuda")
    monkeypatch.setenv("MSC_TUNE", f"c64={kind},c32={kind},bi=0")
    pk = ScatteringPlan(c0.v, c0.t, [c0.system()])
    yk = pk.apply_coupling(x)
    monkeypatch.setenv("MSC_TUNE", "c64=0,c32=0,bi=0")
    p0 = ScatteringPlan(c0.v, c0.t, [c0.system()])
    y0 = p0.apply_coupling(x)
    # (the separable form sums in another order: 1e-12)
    assert float((yk - y0).abs().max()) <= (1e-12 if kind >= 3 else 1e-13) * float(y0.abs().max())
    pk.close()
    p0.close()


def test_separable_coupling_is_found_only_where_the_taps_factorise(monkeypatch):
    """The square-lattice Morse potentials (cfg0/cfg2/cfg4) factorise, the
    hexagonal one (cfg1) and the He-LiF cross of four taps do not; a
    factorised plan is exact in both operators it solves with (A and A^H)."""
    monkeypatch.setenv("MSC_TUNE", "c64=3,c32=3,bi=0")
    c0 = cfg0_case(nz=40)
    pk = ScatteringPlan(c0.v, c0.t, [c0.system()])
    x = torch.randn(c0.pkd.size, 40, dtype=torch.complex128, device="cuda")
    yk = pk.apply_coupling(x)
    assert "coupling64=separable" in pk.tuning_report()["chosen"]
    pk.set_adjoint(True)
    ya = pk.apply_coupling(x)
    pk.close()
    monkeypatch.setenv("MSC_TUNE", "c64=0,c32=0,bi=0")
    p0 = ScatteringPlan(c0.v, c0.t, [c0.system()])
    y0 = p0.apply_coupling(x)
    p0.set_adjoint(True)
    y0a = p0.apply_coupling(x)
    p0.close()
    assert float((yk - y0).abs().max()) <= 1e-12 * float(y0.abs().max())
    assert float((ya - y0a).abs().max()) <= 1e-12 * float(y0a.abs().max())
    monkeypatch.setenv("MSC_TUNE", "c64=3,c32=3,bi=0")
    for case in (cfg1_case(nz=30, nk=11), wolken_case(nz=40)):
        p1 = ScatteringPlan(case.v, case.t, [case.system()])
        p1.apply_coupling(torch.zeros(case.pkd.size, case.v.shape[2], dtype=torch.complex128,
                                      device="cuda"))
        assert "separable" not in p1.tuning_report()["chosen"]
        p1.close()


# ---------------------------------------------------------------------------
# von Neumann preconditioner of order k (the reference's
# _scipy_von_neumann.py; its tests ask orders 0-2 to agree with the scipy
# solve at 1e-5, tests/test_fixed_example.py:387-408).  Here: the API at
# orders 0-2 against the He-LiF golden file, and orders 1-2 of the plan
# against order 0 on a batch, in both precisions.
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("order", [0, 1, 2])
def test_von_neumann_api_reproduces_reference_golden(order):
    from multiscat_b200 import get_scattering_matrix_von_neumann
    s = get_scattering_matrix_von_neumann(_wolken_condition(0.0),
                                          OptimizationConfig(precision=1e-5, max_iterations=1000),
                                          order=order)
    inten = np.real_if_close(s)
    assert math.isclose(float(np.sum(inten).real), 1.0, abs_tol=1e-6)
    np.testing.assert_allclose(inten.real, _read_wolken_golden(), rtol=0.0, atol=1e-5)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_von_neumann_orders_agree_on_a_batch(precision):
    case, systems = cfg2_batch(n_solves=6, seed=7)
    res, iters = {}, {}
    for order in (0, 1, 2):
        plan = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision=precision,
                              preconditioner_order=order)
        r = plan.solve()
        assert (r.status == 0).all()
        res[order] = r.intensities
        iters[order] = int(r.iterations.sum())
        plan.close()
    tol = 1e-8 if precision == "fp64" else MIXED_TOL
    for order in (1, 2):
        assert float((res[order] - res[0]).abs().max()) <= tol
    assert iters[1] < iters[0] and iters[2] < iters[1], iters


def test_von_neumann_order_is_validated(cfg0):
    with pytest.raises(Exception):
        ScatteringPlan(cfg0.v, cfg0.t, [cfg0.system()], preconditioner_order=9)


POISON_SCRIPT = r"""
import sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from multiscat_b200 import ScatteringPlan
from multiscat_b200.workloads import cfg2_batch
case, systems = cfg2_batch(n_solves=6, seed=7)
ref = ScatteringPlan(case.v, case.t, systems, rtol=1e-10).solve().intensities
worst = 0.0
for tc in (True, False):
    for order in (0, 1):
        r = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed",
                           tensor_cores=tc, preconditioner_order=order).solve()
        assert (r.status == 0).all(), (tc, order, r.status)
        worst = max(worst, float((r.intensities - ref).abs().max()))
import os
for bg in (1, 2, 3):       # every tcgen05 kernel form, forced
    os.environ["MSC_TUNE"] = f"c64=2,c32=2,bi=16,bg={bg}"
    r = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed",
                       tensor_cores=True).solve()
    assert (r.status == 0).all(), (bg, r.status)
    worst = max(worst, float((r.intensities - ref).abs().max()))
print(worst)
"""


def test_no_kernel_reads_unwritten_memory():
    """Every plan buffer starts as NaN bytes (MSC_POISON_ALLOC=1, read once per
    process, hence the subprocess): mixed solves on tensor cores and SIMT, with
    and without the von Neumann preconditioner, still match FP64."""
    import os
    import subprocess
    import sys
    root = str(pathlib.Path(__file__).resolve().parents[1])
    env = dict(os.environ, MSC_POISON_ALLOC="1")
    out = subprocess.run([sys.executable, "-c", POISON_SCRIPT, root], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert float(out.stdout.strip().splitlines()[-1]) <= MIXED_TOL


# ---------------------------------------------------------------------------
# Full-state API and warm start (the reference's get_scattering_state /
# get_scattering_matrix_from_state, _multiscat.py:63-99, 227-246, and x0).
# ---------------------------------------------------------------------------
def ref_of(psi, cond):
    """L psi of a psi-convention state, through the library's lower block."""
    from multiscat_b200.api import _reference_order_system, natural_arrays
    from multiscat_b200 import ScatteringPlan
    arr = natural_arrays(cond)
    sp = _reference_order_system(arr, None)
    plan = ScatteringPlan(arr.potential_values, arr.kinetic, [sp], restart=1)
    rows = torch.as_tensor(np.ascontiguousarray(psi[sp.channel_ix, sp.channel_iy]), device="cuda")
    out = psi.copy()
    out[sp.channel_ix, sp.channel_iy] = plan.apply_lower_block(rows).cpu().numpy()
    plan.close()
    return out


def test_state_api_round_trip_matches_scattering_matrix():
    from multiscat_b200 import get_scattering_matrix_from_state, get_scattering_state
    cond = _wolken_condition(0.0)
    cfg = OptimizationConfig(precision=1e-7, max_iterations=1000)
    state = get_scattering_state(cond, cfg)
    assert state.shape == (10, 10, 550) and state.dtype == np.complex128
    s_state = get_scattering_matrix_from_state(state, cond)
    s_direct = get_scattering_matrix(cond, cfg)
    # two separate solves (the reference-convention state orders the channels
    # by pkd), each converged to a relative residual of 1e-10
    np.testing.assert_allclose(s_state.real, s_direct.real, rtol=0.0, atol=1e-9)
    np.testing.assert_allclose(s_state.real, _read_wolken_golden(), rtol=0.0, atol=1e-5)
    # warm start from the converged state: already below the tolerance
    again = get_scattering_state(cond, cfg, initial_state=state)
    np.testing.assert_allclose(again, state, rtol=0.0, atol=1e-10 * np.abs(state).max())
    # the psi convention round-trips the same way
    psi = get_scattering_state(cond, cfg, convention="psi")
    s_psi = get_scattering_matrix_from_state(psi, cond, convention="psi")
    np.testing.assert_allclose(s_psi.real, s_direct.real, rtol=0.0, atol=1e-12)
    # the reference convention's L^-1 (L psi) returns psi itself (to the
    # round-off of a forward sweep through 100 channels)
    np.testing.assert_allclose(get_scattering_matrix_from_state(ref_of(psi, cond), cond).real,
                               s_psi.real, rtol=0.0, atol=1e-9)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_warm_start_from_a_neighbouring_beam(precision):
    """Beams 0 and 1 of a seeded batch differ; warm-starting beam 0's plan from
    its own solution needs no iterations, and the answer does not depend on
    the guess."""
    case, systems = cfg2_batch(n_solves=2, seed=11)
    plan = ScatteringPlan(case.v, case.t, [systems[0]], rtol=1e-10, precision=precision)
    cold = plan.solve()
    plan.set_initial_guess(cold.psi)
    warm = plan.solve()
    assert warm.iterations[0] == 0 and warm.status[0] == 0
    assert float((warm.intensities - cold.intensities).abs().max()) <= 1e-12
    # a poor guess (a random state) still converges to the same answer
    plan.set_initial_guess(torch.randn_like(cold.psi))
    noisy = plan.solve()
    tol = 1e-8 if precision == "fp64" else MIXED_TOL
    assert float((noisy.intensities - cold.intensities).abs().max()) <= tol
    plan.set_initial_guess(None)
    assert plan.solve().iterations[0] == cold.iterations[0]
    plan.close()


def test_interpolated_potential_on_device_gives_the_same_intensities():
    """A sampled potential interpolated on the GPU (interpolate_potential, the
    reference's interpolate.py) scatters like the analytic components."""
    case = cfg0_case()
    a = 2.54
    zg = torch.linspace(-1.5, 10.0, 4000, dtype=torch.float64, device="cuda")
    f = torch.arange(64, dtype=torch.float64, device="cuda") / 64
    fx, fy = torch.meshgrid(f, f, indexing="ij")
    xiv = sa.square_xi(a, 0.1)(fx * a, fy * a)
    factor = sa.natural_units_factor(sa.HE4_MASS)
    samples = factor * 7.63 * (torch.exp(-2.2 * (zg[None, None, :] - xiv[:, :, None]))
                               - 2.0 * torch.exp(-1.1 * zg)[None, None, :])
    v = sa.interpolate_potential(samples, zg, case.nodes, 11, 11)
    assert v.is_cuda
    keep = torch.zeros(11, 11, dtype=torch.bool)
    idx = [i for i, m in enumerate(sa.fft_modes(11)) if abs(m) <= 4]
    keep[np.ix_(idx, idx)] = True
    v = v * keep.to(v.device)[:, :, None]        # the |m|,|n| <= 4 modes of the workload
    r_int = ScatteringPlan(v.cpu().numpy(), case.t, [case.system()], rtol=1e-12).solve()
    r_dir = ScatteringPlan(case.v, case.t, [case.system()], rtol=1e-12).solve()
    assert float((r_int.intensities - r_dir.intensities).abs().max()) <= 1e-4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dcgs2_and_cgs2_arnoldi_agree(precision):
    """The default Arnoldi step (delayed re-orthogonalisation, two passes over
    the basis) and classical Gram-Schmidt with two full passes give the same
    converged intensities and about the same iteration counts."""
    case, systems = cfg2_batch(n_solves=24, seed=3)
    out = {}
    for gs in ("dcgs2", "cgs2"):
        plan = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision=precision,
                              gram_schmidt=gs)
        res = plan.solve()
        plan.close()
        assert (res.status == 0).all() and (res.residual <= 1e-10).all()
        out[gs] = res
    d = np.abs(out["dcgs2"].intensities.cpu().numpy() - out["cgs2"].intensities.cpu().numpy())
    assert d.max() <= (1e-9 if precision == "fp64" else 1e-8)
    it_d, it_c = out["dcgs2"].iterations, out["cgs2"].iterations
    assert np.abs(it_d - it_c).max() <= 2 + 0.1 * it_c.max(), (it_d, it_c)


def test_streamed_arnoldi_passes_agree_with_register_form(monkeypatch):
    """The FP32 DCGS2 reduction and update that stream the basis through
    shared memory by bulk copies (the default for chunks of 2048-4096
    elements; the reduction alone, or both) and the register-streamed passes compute the
    same sums in another grouping: the same converged intensities and about
    the same iteration counts."""
    case, systems = cfg2_batch(n_solves=24, seed=3)
    out = {}
    # (24 beams make chunks of ~1300 elements, below the default threshold of
    # the streamed passes: "bulk" forces them)
    for mode, name in (("registers", "registers"), ("reduce", "bulk_reduce"), ("bulk", "bulk")):
        monkeypatch.setenv("MSC_ARNOLDI_STREAM", mode)
        plan = ScatteringPlan(case.v, case.t, systems, rtol=1e-10, precision="mixed")
        res = plan.solve()
        assert plan.tuning_report()["arnoldi_stream"] == name
        plan.close()
        assert (res.status == 0).all() and (res.residual <= 1e-10).all()
        out[name] = res
    ref = out["registers"]
    for name in ("bulk_reduce", "bulk"):
        d = np.abs(out[name].intensities.cpu().numpy() - ref.intensities.cpu().numpy())
        assert d.max() <= 1e-8, (name, d.max())
        assert np.abs(out[name].iterations - ref.iterations).max() <= 2 + 0.1 * ref.iterations.max()


@pytest.mark.parametrize("nz", [41, 150])
def test_channel_major_tensor_core_kernel_matches_simt(nz, monkeypatch):
    """The channel-major tcgen05 block inverse (bg=3) on odd and even node
    counts (odd: no bulk prefetch, 8-byte stores) and a row total that leaves
    a partial last tile, against the SIMT FP32 kernel and a mixed solve
    against FP64."""
    case, systems = cfg2_batch(n_solves=7, seed=5, nz=nz)
    monkeypatch.setenv("MSC_TUNE", "c64=2,c32=2,bi=128,bg=3")
    mixed = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=True)
    rows = mixed.total_rows
    rng = np.random.default_rng(nz)
    x = rng.standard_normal((rows, nz)) + 1j * rng.standard_normal((rows, nz))
    x32 = torch.as_tensor(x.astype(np.complex64), device="cuda")
    y_tc = mixed.apply_block_inverse_f32(x32).cpu().numpy()
    # (the plan read MSC_TUNE at its first call)
    assert "block_inverse32=tcc" in mixed.tuning_report()["chosen"]
    monkeypatch.setenv("MSC_TUNE", "c64=2,c32=2,bi=0")
    simt = ScatteringPlan(case.v, case.t, systems, precision="mixed", tensor_cores=False)
    y_simt = simt.apply_block_inverse_f32(x32).cpu().numpy()
    scale = np.abs(y_simt).max()
    np.testing.assert_allclose(y_tc, y_simt, rtol=0, atol=TC_TOL * scale)
    ref = ScatteringPlan(case.v, case.t, systems).solve().intensities
    res = mixed.solve()
    assert (res.status == 0).all()
    assert float((res.intensities - ref).abs().max()) <= MIXED_TOL
    mixed.close()
    simt.close()
