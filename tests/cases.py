"""Workloads shared by the tests and the golden-fixture script."""

from __future__ import annotations

import numpy as np

from multiscat_b200.workloads import cfg0_case, cfg1_case, cfg2_batch, wolken_case  # noqa: F401


def subset_case(seed: int):
    """Two-beam slice of the cfg2 batch: (case, oracle-ready channel list of beam 0)."""
    case, systems = cfg2_batch(n_solves=2, seed=seed)
    sp = systems[0]
    system = {"ix": sp.channel_ix, "iy": sp.channel_iy, "pkd": sp.pkd, "wa": sp.wave_a,
              "wb": sp.wave_b, "wc": sp.wave_c, "spec": sp.specular}
    return case, system
