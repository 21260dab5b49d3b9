"""CPU tests of the C-ABI library: it loads, exports the header's symbols, and
rejects bad arguments before touching the GPU."""

from __future__ import annotations

import ctypes
import pathlib
import re

import numpy as np
import pytest

from multiscat_b200 import _native as nat

ROOT = pathlib.Path(__file__).resolve().parents[1]


def header_functions() -> list[str]:
    names = []
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(msc_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_header_function():
    lib = nat.load()
    declared = header_functions()
    assert declared, "no functions found in include/*.h"
    for name in declared:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(declared) == set(nat.EXPORTED)


def test_version_string():
    assert b"sm_100a" in nat.load().msc_version()


def test_plan_create_rejects_bad_dims_without_gpu():
    lib = nat.load()
    plan = ctypes.c_void_p()
    d = nat.PlanDesc(n_z=0, nkx=3, nky=3, n_systems=1, restart=30, max_iterations=100,
                     rtol=1e-8, precision=0)
    assert lib.msc_plan_create(ctypes.byref(plan), ctypes.byref(d)) == nat.MSC_ERR_DIMS
    assert not plan.value
    d = nat.PlanDesc(n_z=10, nkx=3, nky=3, n_systems=1, restart=0, max_iterations=100,
                     rtol=1e-8, precision=0)
    assert lib.msc_plan_create(ctypes.byref(plan), ctypes.byref(d)) == nat.MSC_ERR_ARG
    d = nat.PlanDesc(n_z=10000, nkx=3, nky=3, n_systems=1, restart=30, max_iterations=100,
                     rtol=1e-8, precision=0)
    assert lib.msc_plan_create(ctypes.byref(plan), ctypes.byref(d)) == nat.MSC_ERR_DIMS
    assert "dimension" in nat.last_error()


def test_run_multiscat_bad_dims_is_code_1():
    from multiscat_b200 import run_multiscat_fortran
    with pytest.raises(RuntimeError, match="error code 1"):
        run_multiscat_fortran(1, 5, np.zeros((0, 2, 4), complex), np.zeros((0, 2)), np.zeros(0),
                              np.zeros(0), np.zeros(0), np.eye(4))


def test_product_does_not_import_oracle():
    for py in (ROOT / "multiscat_b200").rglob("*.py"):
        text = py.read_text()
        assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", text, flags=re.M), py
    for src in (ROOT / "multiscat_b200" / "csrc").iterdir():
        assert "msc_oracle" not in src.read_text(), src
