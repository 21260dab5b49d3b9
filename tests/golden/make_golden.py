"""Generate the golden fixtures in this folder (run here, where the reference is mounted).

    python tests/golden/make_golden.py [--reference PATH] [--cfg1] [--cfg3] [--cfg2-batch]

``--reference PATH`` (or the environment variable MULTISCAT_REFERENCE) names
the checkout of the reference project whose golden files are copied; without
it the two ``wolken_*`` files are left as they are.

Writes
- ``wolken_expected_intensities.txt``: copy of the reference's golden file
  ``tests/data/expected_intensities.txt`` (He-LiF Wolken case, 26 open
  channels, ``tests/test_fixed_example.py:233-256``).
- ``wolken_potential_samples.json``: samples of the reference fixture
  ``tests/data/expected_potential.npy`` (the potential convention), with the
  maximum relative deviation of the closed form over the whole fixture.
- ``oracle_cfg0.json``: oracle (CPU restatement of the reference solve)
  intensities for the 11x11-channel square Morse case at precision 1e-12.
- ``oracle_subsets.json``: oracle intensities for channel subsets (the
  ``n_channels`` truncation) of two seeded beams over the same potential.
- ``oracle_cfg2_stall.json``: oracle intensities of beam 1 of
  ``cfg2_batch(n_solves=3, seed=1, nz=41)``, a beam on which the
  block-diagonal FP32 inner solve stalls near a residual of 1e-5.
- ``oracle_cfg2_batch.npz`` (with --cfg2-batch, about a minute on 8 cores):
  the oracle on every beam of the benchmarked batch ``cfg2_batch(512,
  seed=0)`` at eps 0.5e-12; the intensities of 64 of them are kept: the 8
  largest-theta, the 8 lowest-energy and the 8 most-iterations beams plus 40
  more drawn with ``default_rng(2024)`` from the rest; the iteration counts
  of all 512 are kept too.
- ``oracle_cfg1.json`` (with --cfg1, minutes of CPU): oracle intensities of
  the 41x41-channel hexagonal case at precision 1e-10.
- ``oracle_cfg3_fd.json`` (with --cfg3, minutes of CPU on all cores): central
  finite differences, through the oracle, of L = sum_open w_G |S_G|^2 on the
  cfg1 system (w_G ~ U(0,1), seed 0) with respect to D, alpha, h (relative
  step 1e-5, potential from the oracle's own numpy builder) and to Re/Im of a
  few single Fourier components V_G(z_k) (step 1e-3 max(|V_G(z_k)|, 1)).

The GPU box has no reference tree; the tests read only these files.
"""

from __future__ import annotations

import json
import pathlib
import shutil
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from oracle import inputs, solver  # noqa: E402
from tests.cases import cfg0_case, cfg1_case, subset_case  # noqa: E402


def reference_root() -> pathlib.Path | None:
    """The reference checkout named by --reference PATH or MULTISCAT_REFERENCE."""
    import os
    if "--reference" in sys.argv:
        return pathlib.Path(sys.argv[sys.argv.index("--reference") + 1])
    env = os.environ.get("MULTISCAT_REFERENCE")
    return pathlib.Path(env) if env else None


def wolken_files(ref: pathlib.Path) -> None:
    src = ref / "tests" / "data" / "expected_intensities.txt"
    shutil.copyfile(src, HERE / "wolken_expected_intensities.txt")
    fixture = np.load(ref / "tests" / "data" / "expected_potential.npy").reshape(10, 10, 550)
    nodes, _ = inputs.lobatto_rule(0.0, 8.0, 550)
    model = inputs.wolken_potential(nodes, 10, 10)
    rel = float(np.abs(model - fixture).max() / np.abs(fixture).max())
    picks = [0, 1, 100, 275, 549]
    samples = {
        "nodes_index": picks,
        "v00": [float(fixture[0, 0, k].real) for k in picks],
        "v10": [float(fixture[1, 0, k].real) for k in picks],
        "v01": [float(fixture[0, 1, k].real) for k in picks],
        "v90": [float(fixture[9, 0, k].real) for k in picks],
        "max_abs_other_modes": float(np.abs(fixture[2:9]).max()),
        "closed_form_max_rel_dev": rel,
    }
    (HERE / "wolken_potential_samples.json").write_text(json.dumps(samples, indent=1))
    print("wolken potential closed form max rel dev", rel)


def oracle_case(case, sig: int, name: str) -> None:
    t0 = time.time()
    sx, sy = solver.full_grid_channels(*case.v.shape[:2])
    psi, info, iters, ratio = solver.solve_channels(
        case.v, sx, sy, case.pkd.ravel(), case.wc.ravel(), 0, case.wb.ravel()[0], case.t,
        eps=0.5 * 10.0 ** (-sig))
    inten = inputs.intensities(psi, case.wa.ravel(), case.wb.ravel())
    out = {"case": case.name, "precision": 10.0 ** (-sig), "info": info, "iterations": iters,
           "final_ratio": ratio, "seconds": time.time() - t0,
           "intensities": inten.tolist(), "flux": float(inten.sum())}
    (HERE / name).write_text(json.dumps(out))
    print(name, "info", info, "iters", iters, "flux-1", inten.sum() - 1, "s", time.time() - t0)


def oracle_subsets() -> None:
    res = []
    for seed in (0, 1):
        case, system = subset_case(seed)
        psi, info, iters, ratio = solver.solve_channels(
            case.v, system["ix"], system["iy"], system["pkd"], system["wc"], system["spec"],
            system["wb"][system["spec"]], case.t, eps=0.5e-12)
        s = 2.0j * system["wb"] * psi[:, -1]
        s[system["spec"]] += system["wa"][system["spec"]]
        inten = np.abs(s) ** 2
        res.append({"seed": seed, "info": info, "iterations": iters, "n_channels": int(len(inten)),
                    "intensities": inten.tolist(), "flux": float(inten.sum())})
        print("subset seed", seed, "C", len(inten), "info", info, "iters", iters,
              "flux-1", inten.sum() - 1)
    (HERE / "oracle_subsets.json").write_text(json.dumps(res))


# ---------------------------------------------------------------------------
# cfg3: finite differences of the weighted-intensity loss through the oracle
# ---------------------------------------------------------------------------
CFG3_COMPONENTS = [  # (ix, iy, z index, "re" | "im"); z nodes 40-55 lie at -0.2..0.9 A
    (1, 0, 45, "re"), (1, 0, 45, "im"), (40, 1, 40, "re"), (2, 39, 40, "im"),
    (0, 0, 55, "re"),
]


def _component_step(v, ix, iy, k) -> float:
    """1e-3 of max(|V_G(z_k)|, 1/A^2): one node's component moves L by only
    ~1e-4 per unit, so a 1e-5 step would leave the loss difference near the
    solver's own error; the central-difference truncation error at 1e-3 is
    ~1e-7 relative."""
    return 1e-3 * max(abs(v[ix, iy, k]), 1.0)
CFG3_EPS = 0.5e-13


def _cfg3_setup():
    from multiscat_b200.workloads import cfg3_problem
    pr = cfg3_problem()
    c = pr.case
    hex_xi = _hex_xi_numpy(pr.a1, pr.a2)
    return pr, c, hex_xi


def _hex_xi_numpy(a1, a2):
    b1, b2 = inputs.reciprocal_vectors(np.asarray(a1), np.asarray(a2))
    b3 = b1 + b2

    def make(h):
        def fn(x, y):
            return (h / 3.0) * (np.cos(b1[0] * x + b1[1] * y) + np.cos(b2[0] * x + b2[1] * y) +
                                np.cos(b3[0] * x + b3[1] * y))
        return fn
    return make


def _cfg3_potential(pr, hex_xi, depth, alpha, h):
    nk = pr.case.pkd.shape[0]
    v = inputs.corrugated_morse_fourier(pr.case.nodes, pr.a1, pr.a2, hex_xi(h), depth, alpha,
                                        pr.n_cell, pr.k_max, nk, nk)
    return v * pr.factor


def _cfg3_loss(v):
    pr, c, _ = _cfg3_setup()
    sx, sy = solver.full_grid_channels(*v.shape[:2])
    psi, info, iters, _ = solver.solve_channels(
        v, sx, sy, c.pkd.ravel(), c.wc.ravel(), 0, c.wb.ravel()[0], c.t, eps=CFG3_EPS)
    inten = inputs.intensities(psi, c.wa.ravel(), c.wb.ravel())
    return float(np.dot(pr.weights, inten)), int(info), int(iters)


def _cfg3_job(job):
    sys.path.insert(0, str(ROOT))
    pr, c, hex_xi = _cfg3_setup()
    kind, key, sign = job
    p = dict(pr.params)
    if kind == "param":
        p[key] = p[key] * (1.0 + sign * 1e-5)
        v = _cfg3_potential(pr, hex_xi, p["depth"], p["alpha"], p["h"])
    elif kind == "base":
        v = _cfg3_potential(pr, hex_xi, p["depth"], p["alpha"], p["h"])
    else:
        v = _cfg3_potential(pr, hex_xi, p["depth"], p["alpha"], p["h"])
        ix, iy, k, part = key
        step = _component_step(v, ix, iy, k)
        v[ix, iy, k] += sign * step * (1.0 if part == "re" else 1.0j)
    return job, _cfg3_loss(v)


def oracle_cfg3_fd() -> None:
    import multiprocessing as mp
    t0 = time.time()
    pr, c, hex_xi = _cfg3_setup()
    v0 = _cfg3_potential(pr, hex_xi, pr.params["depth"], pr.params["alpha"], pr.params["h"])
    jobs = [("base", None, 0)]
    for k in ("depth", "alpha", "h"):
        jobs += [("param", k, +1), ("param", k, -1)]
    for comp in CFG3_COMPONENTS:
        jobs += [("comp", comp, +1), ("comp", comp, -1)]
    with mp.get_context("spawn").Pool(min(len(jobs), 8)) as pool:
        res = dict(((j[0], j[1], j[2]), r) for j, r in pool.map(_cfg3_job, jobs))
    out = {"case": c.name, "oracle_eps": CFG3_EPS, "relative_step": 1e-5,
           "loss": res[("base", None, 0)][0], "params": {}, "components": [],
           "max_iterations": max(r[2] for r in res.values()),
           "all_converged": all(r[1] == 0 for r in res.values())}
    for k in ("depth", "alpha", "h"):
        step = 1e-5 * pr.params[k]
        out["params"][k] = {"value": pr.params[k], "step": step,
                            "dL": (res[("param", k, 1)][0] - res[("param", k, -1)][0]) / (2 * step)}
    for comp in CFG3_COMPONENTS:
        ix, iy, k, part = comp
        step = _component_step(v0, ix, iy, k)
        out["components"].append({"ix": ix, "iy": iy, "z": k, "part": part, "step": step,
                                  "dL": (res[("comp", comp, 1)][0] - res[("comp", comp, -1)][0]) /
                                        (2 * step)})
    out["seconds"] = time.time() - t0
    (HERE / "oracle_cfg3_fd.json").write_text(json.dumps(out, indent=1))
    print("cfg3 fd", json.dumps(out))


# ---------------------------------------------------------------------------
# cfg2: the benchmarked 512-beam batch itself, and the beam that stalls the
# FP32 inner solve
# ---------------------------------------------------------------------------
CFG2_EPS = 0.5e-12


def _subset_oracle(case, sp):
    psi, info, iters, _ = solver.solve_channels(
        case.v, sp.channel_ix, sp.channel_iy, sp.pkd, sp.wave_c, sp.specular,
        sp.wave_b[sp.specular], case.t, eps=CFG2_EPS)
    s = 2.0j * sp.wave_b * psi[:, -1]
    s[sp.specular] += sp.wave_a[sp.specular]
    return np.abs(s) ** 2, int(info), int(iters)


def _cfg2_beam_job(b):
    sys.path.insert(0, str(ROOT))
    from multiscat_b200.workloads import cfg2_batch
    case, systems = cfg2_batch(512, seed=0)
    inten, info, iters = _subset_oracle(case, systems[b])
    return b, inten, info, iters


def oracle_cfg2_batch() -> None:
    import multiprocessing as mp
    from multiscat_b200.workloads import cfg2_batch
    t0 = time.time()
    case, systems = cfg2_batch(512, seed=0)
    with mp.get_context("spawn").Pool(8) as pool:
        res = sorted(pool.map(_cfg2_beam_job, range(512), chunksize=4), key=lambda r: r[0])
    iters = np.array([r[3] for r in res], np.int32)
    info = np.array([r[2] for r in res], np.int32)
    theta, energy = case.extra["theta"], case.extra["energy"]
    picks: list[int] = []
    for order in (np.argsort(-theta, kind="stable"), np.argsort(energy, kind="stable"),
                  np.argsort(-iters, kind="stable")):
        picks += [int(b) for b in order if int(b) not in picks][:8]
    rest = np.array([b for b in range(512) if b not in picks])
    picks += sorted(np.random.default_rng(2024).choice(rest, 64 - len(picks), replace=False).tolist())
    picks = np.array(picks, np.int32)
    counts = np.array([len(res[b][1]) for b in picks], np.int64)
    offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    inten = np.concatenate([res[b][1] for b in picks])
    np.savez_compressed(HERE / "oracle_cfg2_batch.npz", beams=picks, offsets=offsets,
                        intensities=inten, iterations_all=iters, info_all=info,
                        eps=np.float64(CFG2_EPS))
    print("cfg2 batch: all converged", bool((info == 0).all()), "iterations", int(iters.min()),
          "-", int(iters.max()), "flux-1 max", max(abs(res[b][1].sum() - 1) for b in picks),
          "s", time.time() - t0)


def oracle_cfg2_stall() -> None:
    from multiscat_b200.workloads import cfg2_batch
    case, systems = cfg2_batch(n_solves=3, seed=1, nz=41)
    inten, info, iters = _subset_oracle(case, systems[1])
    out = {"case": "beam 1 of cfg2_batch(n_solves=3, seed=1, nz=41)", "oracle_eps": CFG2_EPS,
           "info": info, "iterations": iters, "n_channels": int(len(inten)),
           "intensities": inten.tolist(), "flux": float(inten.sum())}
    (HERE / "oracle_cfg2_stall.json").write_text(json.dumps(out))
    print("cfg2 stall beam: info", info, "iters", iters, "flux-1", inten.sum() - 1)


if __name__ == "__main__":
    ref = reference_root()
    if ref is not None:
        wolken_files(ref)
    oracle_case(cfg0_case(), 12, "oracle_cfg0.json")
    oracle_subsets()
    oracle_cfg2_stall()
    if "--cfg2-batch" in sys.argv:
        oracle_cfg2_batch()
    if "--cfg1" in sys.argv:
        oracle_case(cfg1_case(), 10, "oracle_cfg1.json")
    if "--cfg3" in sys.argv:
        oracle_cfg3_fd()
