"""Generate the golden fixtures in this folder (run here, where the reference is mounted).

    python tests/golden/make_golden.py [--cfg1]

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
- ``oracle_cfg1.json`` (with --cfg1, minutes of CPU): oracle intensities of
  the 41x41-channel hexagonal case at precision 1e-10.

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

REF = pathlib.Path("/root/reference")


def wolken_files() -> None:
    src = REF / "tests" / "data" / "expected_intensities.txt"
    shutil.copyfile(src, HERE / "wolken_expected_intensities.txt")
    fixture = np.load(REF / "tests" / "data" / "expected_potential.npy").reshape(10, 10, 550)
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


if __name__ == "__main__":
    wolken_files()
    oracle_case(cfg0_case(), 12, "oracle_cfg0.json")
    oracle_subsets()
    if "--cfg1" in sys.argv:
        oracle_case(cfg1_case(), 10, "oracle_cfg1.json")
