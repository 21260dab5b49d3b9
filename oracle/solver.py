"""ctypes wrapper of the CPU oracle (``msc_oracle.c``).

TEST INFRASTRUCTURE ONLY (see ``msc_oracle.c``).  ``run_multiscat_fortran``
here has the argument list and return of the reference's f2py export
``multiscat_fortran.run_multiscat_fortran``
(``lib/multiscat_fortran/src/multiscat_fortran/__init__.py:39-60``) and
raises the same ``RuntimeError`` codes (``bindings.f90:42-45, 58-60``).
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB_PATH = _HERE / "libmsc_oracle.so"
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build() -> pathlib.Path:
    """Compile the oracle with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        lib = ctypes.CDLL(str(_LIB_PATH))
        lib.msc_oracle_solve.restype = ctypes.c_int
        lib.msc_oracle_solve.argtypes = [
            ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
            _ip, _ip, ctypes.c_int,
            _dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp,
        ]
        lib.msc_oracle_eigh.restype = ctypes.c_int
        lib.msc_oracle_eigh.argtypes = [ctypes.c_int, _dp, _dp, _dp]
        lib.msc_oracle_build_preconditioner.restype = ctypes.c_int
        lib.msc_oracle_build_preconditioner.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp]
        lib.msc_oracle_apply_upper.restype = ctypes.c_int
        lib.msc_oracle_apply_upper.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _dp]
        lib.msc_oracle_solve_lower.restype = ctypes.c_int
        lib.msc_oracle_solve_lower.argtypes = [
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp]
        _lib = lib
    return _lib


def _d(a: np.ndarray):
    return a.ctypes.data_as(_dp)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_ip)


def full_grid_channels(nkx: int, nky: int) -> tuple[np.ndarray, np.ndarray]:
    """Row-major (ix, iy) storage positions: the Fortran channel order."""
    ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
    return ix.ravel().astype(np.int32), iy.ravel().astype(np.int32)


def solve_channels(potential_values, channel_ix, channel_iy, pkd_ch, wave_c_ch, spec, b_spec,
                   kinetic, *, flag=1, eps=5e-9, maxiter=2000, window=3):
    """Reference GMRES on an explicit channel list; returns (psi[C, nz], info, iters, ratio)."""
    lib = _load()
    v = np.ascontiguousarray(potential_values, dtype=np.complex128)
    nkx, nky, nz = v.shape
    sx = np.ascontiguousarray(channel_ix, dtype=np.int32)
    sy = np.ascontiguousarray(channel_iy, dtype=np.int32)
    c = sx.size
    pkd = np.ascontiguousarray(pkd_ch, dtype=np.float64)
    wc = np.ascontiguousarray(wave_c_ch, dtype=np.complex128)
    t = np.ascontiguousarray(kinetic, dtype=np.float64)
    b = np.array([complex(b_spec).real, complex(b_spec).imag])
    psi = np.zeros((c, nz), np.complex128)
    iters = np.zeros(1, np.int32)
    ratio = np.zeros(1, np.float64)
    info = lib.msc_oracle_solve(int(flag), float(eps), int(maxiter), int(window), nz, c, nkx, nky,
                                _i(sx), _i(sy), int(spec), _d(v.view(np.float64)), _d(pkd),
                                _d(wc.view(np.float64)), _d(b), _d(t),
                                _d(psi.view(np.float64)), _i(iters), _d(ratio))
    return psi, int(info), int(iters[0]), float(ratio[0])


def run_multiscat_fortran(gmres_preconditioner_flag, convergence_significant_figures,
                          potential_values, perpendicular_kinetic_difference,
                          wave_a, wave_b, wave_c, parallel_kinetic_energy):
    """Oracle twin of the reference f2py export; returns psi[nkx, nky, nz]."""
    v = np.asarray(potential_values, np.complex128)
    nkx, nky, nz = v.shape
    if nkx <= 0 or nky <= 0 or nz <= 0:
        raise RuntimeError("Fortran run_multiscat_fortran failed with error code 1")
    eps = 0.5 * 10.0 ** (-int(convergence_significant_figures))
    sx, sy = full_grid_channels(nkx, nky)
    psi, info, _, _ = solve_channels(
        v, sx, sy, np.asarray(perpendicular_kinetic_difference, float).ravel(),
        np.asarray(wave_c, complex).ravel(), 0, np.asarray(wave_b, complex).ravel()[0],
        parallel_kinetic_energy, flag=int(gmres_preconditioner_flag), eps=eps)
    if info < 0:
        raise RuntimeError(f"oracle internal failure {info}")
    if info != 0:
        raise RuntimeError("Fortran run_multiscat_fortran failed with error code 2")
    return psi.reshape(nkx, nky, nz)


def eigh(a: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    lib = _load()
    a = np.ascontiguousarray(a, np.float64)
    n = a.shape[0]
    w = np.zeros(n)
    z = np.zeros((n, n))
    st = lib.msc_oracle_eigh(n, _d(a), _d(w), _d(z))
    if st != 0:
        raise RuntimeError(f"eigensolver failed ({st})")
    return w, z


def build_preconditioner(potential_values, pkd, kinetic):
    lib = _load()
    v = np.ascontiguousarray(potential_values, np.complex128)
    nkx, nky, nz = v.shape
    pkd = np.ascontiguousarray(np.asarray(pkd, float).ravel())
    lam = np.zeros(nz)
    e = np.zeros((nz, nz))
    f = np.zeros((pkd.size, nz))
    st = lib.msc_oracle_build_preconditioner(nz, pkd.size, nkx, nky, _d(v.view(np.float64)), _d(pkd),
                                             _d(np.ascontiguousarray(kinetic, np.float64)),
                                             _d(lam), _d(e), _d(f))
    if st != 0:
        raise RuntimeError(f"preconditioner failed ({st})")
    return lam, e, f


def apply_upper(potential_values, state):
    """Reference debug_apply_upper_block on state[C, nz] (full channel grid)."""
    lib = _load()
    v = np.ascontiguousarray(potential_values, np.complex128)
    nkx, nky, nz = v.shape
    sx, sy = full_grid_channels(nkx, nky)
    x = np.ascontiguousarray(state, np.complex128).copy()
    lib.msc_oracle_apply_upper(nz, sx.size, nkx, nky, _i(sx), _i(sy), _d(v.view(np.float64)),
                               _d(x.view(np.float64)))
    return x


def solve_lower(potential_values, pkd, wave_c, kinetic, state):
    """Reference debug_solve_lower_block on state[C, nz] (full channel grid)."""
    lib = _load()
    v = np.ascontiguousarray(potential_values, np.complex128)
    nkx, nky, nz = v.shape
    sx, sy = full_grid_channels(nkx, nky)
    x = np.ascontiguousarray(state, np.complex128).copy()
    pkd = np.ascontiguousarray(np.asarray(pkd, float).ravel())
    wc = np.ascontiguousarray(np.asarray(wave_c, complex).ravel())
    st = lib.msc_oracle_solve_lower(nz, sx.size, nkx, nky, _i(sx), _i(sy), _d(v.view(np.float64)),
                                    _d(pkd), _d(wc.view(np.float64)),
                                    _d(np.ascontiguousarray(kinetic, np.float64)),
                                    _d(x.view(np.float64)))
    if st != 0:
        raise RuntimeError(f"lower solve failed ({st})")
    return x
