"""Host side of the solver: plans on torch device memory, and the drop-in call.

``run_multiscat_fortran`` has the argument list, return value and errors of
the reference's f2py export (``lib/multiscat_fortran/src/multiscat_fortran/
__init__.py:39-60``): it returns psi[nkx, nky, nz] and raises
``RuntimeError("... failed with error code N")`` with N = 1 for bad
dimensions and N = 2 when GMRES does not converge
(``multiscat_python_bindings.f90:42-45, 58-60``).

``ScatteringPlan`` is the batched, device-resident form: one potential,
many beams, all solved in one go on the current CUDA device.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as nat


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _stack_systems(systems: list) -> dict:
    """The systems' channel arrays concatenated in system order, as the batched
    msc_plan_set_systems takes them (offsets[k]..offsets[k + 1] is system k)."""
    if not systems:
        raise ValueError("a plan needs at least one system")
    counts = np.fromiter((len(sp.channel_ix) for sp in systems), dtype=np.int64, count=len(systems))
    offsets = np.zeros(len(systems) + 1, dtype=np.int64)
    np.cumsum(counts, out=offsets[1:])

    def cat(name, dtype):
        return np.ascontiguousarray(np.concatenate([getattr(sp, name) for sp in systems], axis=None),
                                    dtype=dtype)

    return {
        "offsets": offsets,
        "ix": cat("channel_ix", np.int32),
        "iy": cat("channel_iy", np.int32),
        "pkd": cat("pkd", np.float64),
        "wb": cat("wave_b", np.complex128),
        "wc": cat("wave_c", np.complex128),
        "specular": np.fromiter((int(sp.specular) for sp in systems), dtype=np.int32,
                                count=len(systems)),
        "a_spec": np.array([complex(sp.wave_a[sp.specular]) for sp in systems],
                           dtype=np.complex128),
    }


def run_multiscat_fortran(gmres_preconditioner_flag: int, convergence_significant_figures: int,
                          potential_values, perpendicular_kinetic_difference, wave_a, wave_b,
                          wave_c, parallel_kinetic_energy) -> np.ndarray:
    """Drop-in for ``multiscat_fortran.run_multiscat_fortran`` on the GPU (FP64)."""
    lib = nat.load()
    v = np.ascontiguousarray(potential_values, dtype=np.complex128)
    if v.ndim != 3:
        raise RuntimeError("B200 run_multiscat_fortran failed with error code 1")
    nkx, nky, nz = v.shape
    pkd = np.ascontiguousarray(perpendicular_kinetic_difference, dtype=np.float64)
    wa = np.ascontiguousarray(np.asarray(wave_a, np.complex128).ravel())
    wb = np.ascontiguousarray(np.asarray(wave_b, np.complex128).ravel())
    wc = np.ascontiguousarray(np.asarray(wave_c, np.complex128).ravel())
    t = np.ascontiguousarray(parallel_kinetic_energy, dtype=np.float64)
    c = nkx * nky
    if pkd.size != c or wa.size != c or wb.size != c or wc.size != c or t.shape != (nz, nz):
        raise RuntimeError("B200 run_multiscat_fortran failed with error code 1")
    out = np.zeros((nkx, nky, nz), np.complex128)
    iters = ctypes.c_int(0)
    ierr = lib.msc_run_multiscat(int(gmres_preconditioner_flag),
                                 int(convergence_significant_figures), nkx, nky, nz,
                                 _dptr(v.view(np.float64)), _dptr(pkd),
                                 _dptr(wa.view(np.float64)), _dptr(wb.view(np.float64)),
                                 _dptr(wc.view(np.float64)), _dptr(t),
                                 _dptr(out.view(np.float64)), ctypes.byref(iters))
    if ierr != 0:
        raise RuntimeError(f"B200 run_multiscat_fortran failed with error code {ierr}"
                           f" ({nat.last_error()})")
    return out


@dataclass
class SystemSpec:
    """One beam: channel list on the torus plus its boundary arrays."""

    channel_ix: np.ndarray      # int32 [C] storage positions
    channel_iy: np.ndarray
    pkd: np.ndarray             # float64 [C]
    wave_a: np.ndarray          # complex128 [C]
    wave_b: np.ndarray          # complex128 [C]
    wave_c: np.ndarray          # complex128 [C]
    specular: int = 0


@dataclass
class SolveResult:
    psi: torch.Tensor           # complex128 [R, nz] on the device
    intensities: torch.Tensor   # float64 [R] on the device
    row_offsets: np.ndarray     # [B + 1]
    iterations: np.ndarray
    cycles: np.ndarray
    status: np.ndarray
    residual: np.ndarray
    fp64_fallback: np.ndarray | None = None   # mixed: systems re-solved in FP64
    basis_vectors: np.ndarray | None = None   # sum over Arnoldi steps of j + 1

    def system_intensities(self, s: int) -> torch.Tensor:
        return self.intensities[self.row_offsets[s]:self.row_offsets[s + 1]]

    def system_psi(self, s: int) -> torch.Tensor:
        return self.psi[self.row_offsets[s]:self.row_offsets[s + 1]]


class ScatteringPlan:
    """A batch of beams sharing one potential, solved together on the GPU."""

    def __init__(self, potential_values, kinetic, systems: list[SystemSpec], *,
                 rtol: float = 1e-10, restart: int = 30, max_iterations: int = 2000,
                 precision: str = "fp64", inner_rtol: float = 0.0, inner_restart: int = 0,
                 max_refinements: int = 0, tensor_cores: bool | None = None,
                 inner_gram_schmidt_passes: int = 2, preconditioner_order: int = 0,
                 fp64_recovery: bool = True, gram_schmidt: str = "dcgs2",
                 gauss_seidel: bool = False):
        self._lib = nat.load()
        v = np.ascontiguousarray(np.asarray(potential_values), dtype=np.complex128)
        nkx, nky, nz = v.shape
        t = np.ascontiguousarray(np.asarray(kinetic), dtype=np.float64)
        self.nkx, self.nky, self.nz = nkx, nky, nz
        self.systems = systems
        desc = nat.PlanDesc()
        desc.n_z = nz
        desc.nkx = nkx
        desc.nky = nky
        desc.n_systems = len(systems)
        desc.restart = restart
        desc.max_iterations = max_iterations
        desc.rtol = rtol
        desc.precision = {"fp64": nat.PRECISION_FP64, "mixed": nat.PRECISION_MIXED}[precision]
        desc.inner_restart = inner_restart
        desc.inner_rtol = inner_rtol
        desc.max_refinements = max_refinements
        # tensor_cores: None = autotuned, True = always tcgen05, False = never
        desc.flags = {None: 0, True: 2, False: 1}[tensor_cores]
        # mixed form: Gram-Schmidt passes of the FP32 inner Arnoldi step (1 or 2)
        if inner_gram_schmidt_passes not in (1, 2):
            raise ValueError("inner_gram_schmidt_passes must be 1 or 2")
        if inner_gram_schmidt_passes == 1:
            desc.flags |= 4
        # mixed form: re-solve in FP64 the systems the refinement leaves unconverged
        if not fp64_recovery:
            desc.flags |= 8
        # Arnoldi orthogonalisation: "dcgs2" (delayed re-orthogonalisation, two
        # passes over the basis per step) or "cgs2" (two full CGS passes, three)
        if gram_schmidt not in ("dcgs2", "cgs2"):
            raise ValueError("gram_schmidt must be 'dcgs2' or 'cgs2'")
        if gram_schmidt == "cgs2":
            desc.flags |= 16
        # the reference's block Gauss-Seidel preconditioner M = L^-1 (with
        # preconditioner_order = 1: its Neumann flag on top) instead of the
        # block-diagonal D^-1 series
        if gauss_seidel:
            desc.flags |= 32
        # von Neumann order k: M = sum_{i<=k} (-D^-1 V)^i D^-1 (0 = block-diagonal D^-1)
        desc.precond_order = int(preconditioner_order)
        self._plan = ctypes.c_void_p()
        nat.check("msc_plan_create", self._lib.msc_plan_create(ctypes.byref(self._plan),
                                                              ctypes.byref(desc)))
        nat.check("msc_plan_set_potential", self._lib.msc_plan_set_potential(
            self._plan, _dptr(v.view(np.float64)), _dptr(t)))
        # every system in one call: per-channel arrays concatenated in system
        # order (converting pointers system by system costs ~25 us per beam)
        sa = _stack_systems(systems)
        nat.check("msc_plan_set_systems", self._lib.msc_plan_set_systems(
            self._plan, 0, len(systems), sa["offsets"].ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            _iptr(sa["ix"]), _iptr(sa["iy"]), _dptr(sa["pkd"]), _dptr(sa["wb"].view(np.float64)),
            _dptr(sa["wc"].view(np.float64)), _iptr(sa["specular"]),
            _dptr(sa["a_spec"].view(np.float64))))
        self.row_offsets = sa["offsets"].copy()
        self.total_rows = int(sa["offsets"][-1])

    def close(self) -> None:
        if getattr(self, "_plan", None) and self._plan.value:
            self._lib.msc_plan_destroy(self._plan)
            self._plan = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_initial_guess(self, psi0: torch.Tensor | None) -> None:
        """Warm start for the following solves: psi0 complex128 [total_rows, nz]
        (plan row order), or None for the zero guess."""
        stream = torch.cuda.current_stream().cuda_stream
        if psi0 is None:
            st = self._lib.msc_plan_set_initial_guess(self._plan, None, 0, ctypes.c_void_p(stream))
        else:
            dev = torch.device("cuda", torch.cuda.current_device())
            psi0 = torch.as_tensor(psi0).to(device=dev, dtype=torch.complex128).contiguous()
            if psi0.shape != (self.total_rows, self.nz):
                raise ValueError(f"expected [{self.total_rows}, {self.nz}], got {tuple(psi0.shape)}")
            self._x0_keepalive = psi0
            st = self._lib.msc_plan_set_initial_guess(self._plan, ctypes.c_void_p(psi0.data_ptr()), 1,
                                                      ctypes.c_void_p(stream))
        nat.check("msc_plan_set_initial_guess", st)

    def solve(self, *, raise_on_error: bool = True) -> SolveResult:
        dev = torch.device("cuda", torch.cuda.current_device())
        psi = torch.empty((self.total_rows, self.nz), dtype=torch.complex128, device=dev)
        inten = torch.empty((self.total_rows,), dtype=torch.float64, device=dev)
        res = (nat.Result * len(self.systems))()
        stream = torch.cuda.current_stream(dev).cuda_stream
        st = self._lib.msc_solve(self._plan, ctypes.c_void_p(psi.data_ptr()),
                                 ctypes.c_void_p(inten.data_ptr()), res, ctypes.c_void_p(stream))
        if st not in (nat.MSC_OK, nat.MSC_ERR_NOT_CONVERGED, nat.MSC_ERR_NONFINITE) or (
                raise_on_error and st != nat.MSC_OK):
            nat.check("msc_solve", st)
        return SolveResult(
            psi=psi, intensities=inten, row_offsets=self.row_offsets,
            iterations=np.array([r.iterations for r in res]),
            cycles=np.array([r.refinements for r in res]),
            status=np.array([r.status for r in res]),
            residual=np.array([r.residual for r in res]),
            fp64_fallback=np.array([r.fp64_fallback for r in res]),
            basis_vectors=np.array([r.basis_vectors for r in res]))

    # ---- adjoint differentiation -------------------------------------------------
    def set_adjoint(self, on: bool) -> None:
        """Solve with A^H (True) or A (False); eigenbasis, tuning and graphs are kept."""
        nat.check("msc_plan_set_adjoint", self._lib.msc_plan_set_adjoint(self._plan, 1 if on else 0))

    @property
    def adjoint(self) -> bool:
        return bool(self._lib.msc_plan_is_adjoint(self._plan))

    def set_boundary_rhs(self, rhs: torch.Tensor | None) -> None:
        """Outer-boundary right-hand side per row (complex128 [total_rows], cuda),
        or None for the scattering source b_spec at each specular row."""
        stream = torch.cuda.current_stream().cuda_stream
        if rhs is None:
            st = self._lib.msc_plan_set_boundary_rhs(self._plan, None, 0, ctypes.c_void_p(stream))
        else:
            rhs = _device_rows(rhs, torch.complex128, self.total_rows)
            st = self._lib.msc_plan_set_boundary_rhs(self._plan, ctypes.c_void_p(rhs.data_ptr()), 1,
                                                     ctypes.c_void_p(stream))
            self._rhs_keepalive = rhs
        nat.check("msc_plan_set_boundary_rhs", st)

    def solve_adjoint(self, psi: torch.Tensor, dl_dintensity: torch.Tensor | None = None,
                      dl_damplitude: torch.Tensor | None = None, *,
                      raise_on_error: bool = True) -> SolveResult:
        """lambda with A^H lambda = u, u_G(z_n) = -i gamma_G conj(b_G),
        gamma = 2 dL/dI_G S_G + dL/dS_G (S from psi).  lambda is in ``.psi``.
        The plan returns to the forward operator and source afterwards."""
        stream = torch.cuda.current_stream().cuda_stream
        psi = psi.contiguous()
        di = None if dl_dintensity is None else _device_rows(dl_dintensity, torch.float64,
                                                             self.total_rows)
        ds = None if dl_damplitude is None else _device_rows(dl_damplitude, torch.complex128,
                                                             self.total_rows)
        self.set_adjoint(True)
        try:
            nat.check("msc_plan_set_adjoint_rhs", self._lib.msc_plan_set_adjoint_rhs(
                self._plan, ctypes.c_void_p(psi.data_ptr()),
                None if di is None else ctypes.c_void_p(di.data_ptr()),
                None if ds is None else ctypes.c_void_p(ds.data_ptr()), ctypes.c_void_p(stream)))
            res = self.solve(raise_on_error=raise_on_error)
        finally:
            self.set_adjoint(False)
            self.set_boundary_rhs(None)
        res.intensities = None
        return res

    def potential_gradient(self, psi: torch.Tensor, lam: torch.Tensor,
                           window: tuple[int, int] | None = None) -> torch.Tensor:
        """dL/dV (complex128 [nkx, nky, nz], dL/dRe + i dL/dIm) from the forward
        solution psi and the adjoint solution lam; window = (half_x, half_y)
        restricts the offsets computed (others are 0)."""
        psi = psi.contiguous()
        lam = lam.contiguous()
        grad = torch.empty((self.nkx, self.nky, self.nz), dtype=torch.complex128, device=psi.device)
        hx, hy = (-1, -1) if window is None else window
        stream = torch.cuda.current_stream().cuda_stream
        nat.check("msc_potential_gradient", self._lib.msc_potential_gradient(
            self._plan, ctypes.c_void_p(psi.data_ptr()), ctypes.c_void_p(lam.data_ptr()), hx, hy,
            ctypes.c_void_p(grad.data_ptr()), ctypes.c_void_p(stream)))
        return grad

    def info(self) -> "nat.PlanInfo":
        inf = nat.PlanInfo()
        nat.check("msc_plan_get_info", self._lib.msc_plan_get_info(self._plan, ctypes.byref(inf)))
        return inf

    @property
    def n_taps(self) -> int:
        return int(self.info().n_taps)

    def launches_per_solve(self, _result=None) -> int:
        """Kernel launches issued by the last solve (graph kernel nodes, all cycles)."""
        return int(self.info().launches_last)

    def enable_kernel_timing(self, on: bool = True) -> None:
        nat.check("msc_plan_set_kernel_timing",
                  self._lib.msc_plan_set_kernel_timing(self._plan, 1 if on else 0))

    def kernel_timing(self) -> dict:
        ms = (ctypes.c_double * 5)()
        cnt = (ctypes.c_int64 * 5)()
        nat.check("msc_plan_kernel_timing", self._lib.msc_plan_kernel_timing(self._plan, ms, cnt))
        names = ("block_inverse", "coupling", "arnoldi_project", "arnoldi_update_project",
                 "arnoldi_normalize")
        return {k: {"ms": ms[i], "launches": cnt[i]} for i, k in enumerate(names)}

    # debug operators on one full-grid system (x, y: complex128 [C, nz] cuda tensors)
    def _debug(self, name: str, x: torch.Tensor) -> torch.Tensor:
        x = x.contiguous()
        y = torch.empty_like(x)
        stream = torch.cuda.current_stream(x.device).cuda_stream
        nat.check(name, getattr(self._lib, name)(self._plan, ctypes.c_void_p(x.data_ptr()),
                                                 ctypes.c_void_p(y.data_ptr()),
                                                 ctypes.c_void_p(stream)))
        return y

    def apply_coupling(self, x: torch.Tensor) -> torch.Tensor:
        return self._debug("msc_debug_apply_coupling", x)

    def apply_block_inverse(self, x: torch.Tensor) -> torch.Tensor:
        return self._debug("msc_debug_apply_block_inverse", x)

    def apply_operator(self, x: torch.Tensor) -> torch.Tensor:
        return self._debug("msc_debug_apply_operator", x)

    def apply_lower_block(self, x: torch.Tensor) -> torch.Tensor:
        """L x, L = D + V^lower of the block Gauss-Seidel splitting in plan row order."""
        return self._debug("msc_apply_lower_block", x)

    def solve_lower_block(self, x: torch.Tensor) -> torch.Tensor:
        """L^-1 x (the reference's forward sweep, solve_lower_block)."""
        return self._debug("msc_solve_lower_block", x)

    def apply_block_inverse_f32(self, x: torch.Tensor) -> torch.Tensor:
        """D^-1 x with the mixed form's FP32 kernel (x: complex64 [R, nz])."""
        return self._debug("msc_debug_apply_block_inverse_f32", x)

    def tuning_report(self) -> dict:
        """Autotuner timings (us) and the kernel variants it chose."""
        import json
        return json.loads(self._lib.msc_plan_tuning_report(self._plan).decode())

    @property
    def tensor_core_tile(self) -> int:
        """Tile width N of the tcgen05 block inverse (0 when it is not used)."""
        return int(self._lib.msc_plan_uses_tensor_cores(self._plan))


def release_cached_memory() -> None:
    """Give the library's unused plan memory on the current device back to the driver."""
    lib = nat.load()
    nat.check("msc_release_cached_memory", lib.msc_release_cached_memory())


def _device_rows(t, dtype, rows: int) -> torch.Tensor:
    t = torch.as_tensor(t).to(device=torch.device("cuda", torch.cuda.current_device()),
                              dtype=dtype).contiguous()
    if t.numel() != rows:
        raise ValueError(f"expected {rows} rows, got {t.numel()}")
    return t


def beam_systems(pkd, waves, n_channels: int | None = None,
                 max_pkd: float | None = None) -> list[SystemSpec]:
    """One system per beam from batched pkd [B, nkx, nky]: ``full_grid_system``
    when neither ``n_channels`` nor ``max_pkd`` is given, else
    ``channel_subset_system``, beam by beam, with the sort and gathers done for
    all beams at once.  ``waves(e) -> (a, b, c)`` maps pkd values (1-D) to the
    boundary waves element by element (``setup_arrays.waves``); it runs on the
    kept channels only, so the results equal the per-beam builders'."""
    pkd = np.asarray(pkd, float)
    nb, nkx, nky = pkd.shape
    flat = pkd.reshape(nb, -1)
    if n_channels is None and max_pkd is None:
        ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
        ix = ix.ravel().astype(np.int32)
        iy = iy.ravel().astype(np.int32)
        wa, wb, wc = (np.asarray(w, complex).reshape(nb, -1) for w in waves(flat.ravel()))
        return [SystemSpec(ix.copy(), iy.copy(), flat[b], wa[b], wb[b], wc[b], 0) for b in range(nb)]
    order = np.argsort(flat, axis=1, kind="stable")
    if n_channels is not None:
        order = order[:, :n_channels]
    spd = np.take_along_axis(flat, order, axis=1)
    keep = np.full(nb, order.shape[1]) if max_pkd is None else (spd <= max_pkd).sum(axis=1)
    mask = np.arange(order.shape[1])[None, :] < keep[:, None]
    kept = spd[mask]                                  # kept channels, beam after beam
    wa, wb, wc = (np.asarray(w, complex) for w in waves(kept))
    ix, iy = np.unravel_index(order, (nkx, nky))
    out = []
    pos = 0
    for b in range(nb):
        k = int(keep[b])
        spec = np.nonzero(order[b, :k] == 0)[0]
        if spec.size == 0:
            raise ValueError(f"beam {b}: the specular channel is not in the kept channel set")
        sl = slice(pos, pos + k)
        out.append(SystemSpec(ix[b, :k].astype(np.int32), iy[b, :k].astype(np.int32), kept[sl],
                              wa[sl], wb[sl], wc[sl], int(spec[0])))
        pos += k
    return out


def full_grid_system(pkd, wave_a, wave_b, wave_c) -> SystemSpec:
    """All nkx*nky channels in the reference's row-major (ix, iy) order."""
    pkd = np.asarray(pkd, float)
    nkx, nky = pkd.shape
    ix, iy = np.meshgrid(np.arange(nkx), np.arange(nky), indexing="ij")
    return SystemSpec(ix.ravel().astype(np.int32), iy.ravel().astype(np.int32), pkd.ravel(),
                      np.asarray(wave_a, complex).ravel(), np.asarray(wave_b, complex).ravel(),
                      np.asarray(wave_c, complex).ravel(), 0)


def channel_subset_system(pkd, wave_a, wave_b, wave_c, n_channels: int | None = None,
                          max_pkd: float | None = None) -> SystemSpec:
    """Lowest-pkd channels, as the reference's ``n_channels`` truncation.

    Channels are sorted by pkd (``_scipy.py:414-416``) and the first
    ``n_channels`` are kept, or all with pkd <= ``max_pkd``.  The specular
    channel (storage (0, 0)) always has the lowest pkd of a beam whose
    parallel momentum lies in the first Brillouin zone; it is located
    explicitly either way.
    """
    pkd = np.asarray(pkd, float)
    nkx, nky = pkd.shape
    flat = pkd.ravel()
    order = np.argsort(flat, kind="stable")
    if n_channels is not None:
        order = order[:n_channels]
    if max_pkd is not None:
        order = order[flat[order] <= max_pkd]
    if 0 not in set(order.tolist()):
        raise ValueError("the specular channel is not in the kept channel set")
    ix, iy = np.unravel_index(order, (nkx, nky))
    spec = int(np.nonzero(order == 0)[0][0])
    return SystemSpec(ix.astype(np.int32), iy.astype(np.int32), flat[order],
                      np.asarray(wave_a, complex).ravel()[order],
                      np.asarray(wave_b, complex).ravel()[order],
                      np.asarray(wave_c, complex).ravel()[order], spec)
