/*
 * multiscat_b200.h -- C-ABI of the B200 close-coupling scattering solver.
 *
 * Plain C types only (no torch, no C++).  Complex numbers are interleaved
 * (re, im) pairs of double or float.  Every function returns an msc_status
 * and never aborts the process.
 *
 * Reference interfaces replaced (paths relative to the multiscat project):
 *   msc_run_multiscat   <- run_multiscat_fortran
 *        lib/multiscat_fortran/fortran/multiscat_python_bindings.f90:1-61
 *        lib/multiscat_fortran/fortran/multiscat_python_bindings.pyf:3-17
 *        lib/multiscat_fortran/src/multiscat_fortran/__init__.py:39-60
 *   msc_plan_* / msc_solve  <- solve_scattering_gmres + run_preconditioned_gmres
 *        lib/multiscat_fortran/fortran/multiscat_gmres.f90:105-202
 *        (batched, device-resident form; no reference counterpart for the
 *        batching itself)
 *   msc_debug_apply_coupling     <- debug_apply_upper_block
 *        multiscat_gmres.f90:338-382 (full off-diagonal coupling here)
 *   msc_debug_apply_block_inverse <- the block-diagonal inverse D^-1 of
 *        multiscat/multiscat/_scipy.py:249-259 (apply_inverse_diagonal)
 *   msc_intensities          <- _get_scattered_intensity_data
 *        multiscat/multiscat/_multiscat.py:40-60
 */
#ifndef MULTISCAT_B200_H
#define MULTISCAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  1 and 2 keep the meaning of the reference's ierr
 * (bindings.f90:42-45 bad dimensions, :58-60 GMRES not converged). */
typedef enum {
    MSC_OK = 0,
    MSC_ERR_DIMS = 1,          /* non-positive or inconsistent sizes        */
    MSC_ERR_NOT_CONVERGED = 2, /* iteration limit reached                   */
    MSC_ERR_CUDA = 3,          /* CUDA runtime error or allocation failure  */
    MSC_ERR_NONFINITE = 4,     /* NaN/Inf met in a residual                 */
    MSC_ERR_EIGEN = 5,         /* preconditioner eigensolver failed         */
    MSC_ERR_ARG = 6,           /* null pointer or unsupported option        */
    MSC_ERR_NOT_BUILT = 7      /* solver compiled without a needed feature  */
} msc_status;

/* Arithmetic of the inner Krylov solve. */
typedef enum {
    MSC_PRECISION_FP64 = 0,   /* plain FP64 restarted GMRES                  */
    MSC_PRECISION_MIXED = 1   /* FP32 inner GMRES, FP64 iterative refinement */
} msc_precision;

/* Sizes and options of one plan.  A plan holds one potential (one z grid,
 * one coupling torus nkx x nky) and a batch of n_systems beams, each with
 * its own channel list. */
typedef struct {
    int32_t n_z;            /* Lobatto nodes per channel (2..1024)              */
    int32_t nkx, nky;       /* coupling torus (the potential's Fourier grid)    */
    int32_t n_systems;      /* batch size                                       */
    int32_t restart;        /* GMRES restart length m (1..64)                   */
    int32_t max_iterations; /* total Krylov iterations per system               */
    double rtol;            /* stop when ||b - A psi|| <= rtol ||b|| (per system)*/
    int32_t precision;      /* msc_precision                                    */
    int32_t inner_restart;  /* mixed: inner FP32 restart (0 = min(restart, 20)) */
    double inner_rtol;      /* mixed: inner relative tolerance (0 = 3e-6)       */
    int32_t max_refinements;/* mixed: outer FP64 refinement steps (0 = 30)      */
    int32_t flags;          /* bit 0: mixed form without the tcgen05 kernel;
                               bit 1: keep the tcgen05 kernel even when the
                               autotuner times the SIMT kernel faster;
                               bit 2: mixed form with ONE Gram-Schmidt pass
                               (Pythagorean norm) in the inner solve instead
                               of two; fewer bytes per iteration, but on
                               ill-conditioned batches more iterations;
                               bit 3: mixed form without the FP64 recovery of
                               systems left unconverged (see msc_solve);
                               bit 4: Arnoldi step by classical Gram-Schmidt
                               with two full passes (CGS2, three passes over
                               the basis per step) instead of the default
                               delayed re-orthogonalisation (DCGS2, two);
                               bit 5: block Gauss-Seidel preconditioner, the
                               reference's: L = D + V^lower in each system's
                               channel order, M = L^-1 by a forward sweep
                               (multiscat_gmres.f90:641-687)                  */
    int32_t precond_order;  /* order k of the preconditioner series
                               M = sum_{i<=k} (-B^-1 N)^i B^-1 with B = D,
                               N = V (von Neumann, the reference's
                               _scipy_von_neumann.py:40-58; 0 = block-diagonal
                               D^-1) or, with flag bit 5, B = L, N = V^upper
                               (k = 1 is the reference's Neumann flag on top
                               of Gauss-Seidel, _gmres.py:55-71); 0..8       */
} msc_plan_desc;

typedef struct msc_plan msc_plan;

/* Per-system result written by msc_solve. */
typedef struct {
    int32_t iterations;     /* Krylov iterations (inner iterations for mixed) */
    int32_t refinements;    /* FP64 outer steps (mixed), restart cycles (FP64)*/
    int32_t status;         /* msc_status of this system                      */
    int32_t fp64_fallback;  /* mixed: 1 if the FP64 recovery re-solved it     */
    double residual;        /* final true relative residual ||b-A psi||/||b|| */
    int32_t basis_vectors;  /* Krylov basis vectors the Arnoldi steps projected
                               against, summed over the steps (j + 1 at step
                               j): the per-step basis traffic for rooflines  */
    int32_t reserved;
} msc_result;

/* Create a plan on the current CUDA device.  Allocates all device memory
 * the solve needs; *plan is NULL on failure. */
msc_status msc_plan_create(msc_plan **plan, const msc_plan_desc *desc);

/* Destroy a plan (synchronises the device).  Its device memory goes back to
 * a memory pool the library keeps per device, so that the next plan (a new
 * batch of beams, a new potential) gets its buffers without cudaMalloc; up
 * to 32 GiB of unused pool memory stays reserved. */
msc_status msc_plan_destroy(msc_plan *plan);

/* Return the current device's unused pool memory to the driver (for callers
 * that share the GPU with another allocator, e.g. between phases). */
msc_status msc_release_cached_memory(void);

/* Set the potential (host arrays, C order):
 *   potential_values  complex [nkx][nky][n_z]  V_G(z_k) in 1/Angstrom^2
 *   kinetic           double  [n_z][n_z]       positive Lobatto kinetic T
 * Builds H0 = T + diag Re V_00, its FP64 eigen-decomposition (on the
 * device; see msc_debug_symmetric_eigh) and the coupling taps (every offset
 * G != 0 with V_G or V_-G nonzero).
 * Replaces build_preconditioner, multiscat_gmres.f90:226-273. */
msc_status msc_plan_set_potential(msc_plan *plan, const double *potential_values,
                                  const double *kinetic);

/* Set system s's channels (host arrays):
 *   n_channels        C_s (<= nkx*nky)
 *   channel_ix/iy     storage position of each channel on the torus [C_s]
 *   pkd               perpendicular kinetic difference per channel [C_s]
 *   wave_b, wave_c    complex per channel [C_s]
 *   specular          index of the specular channel in this list
 *   wave_a_spec       complex a of the specular channel (for S extraction)
 * All systems must be set before msc_solve. */
msc_status msc_plan_set_system(msc_plan *plan, int32_t s, int32_t n_channels,
                               const int32_t *channel_ix, const int32_t *channel_iy,
                               const double *pkd, const double *wave_b,
                               const double *wave_c, int32_t specular,
                               const double *wave_a_spec);

/* Set systems first .. first + count - 1 in one call (the batched form of
 * msc_plan_set_system, for sweeps of many beams): the per-channel host arrays
 * hold the systems one after another, system k's channels at
 * [offsets[k], offsets[k + 1]) (offsets: count + 1 entries, offsets[0] = 0;
 * wave_b / wave_c: complex, 2 doubles per channel); specular[k] indexes
 * within system k; wave_a_spec: count complex values (may be NULL).  Same
 * checks and error codes as msc_plan_set_system, applied system by system. */
msc_status msc_plan_set_systems(msc_plan *plan, int32_t first, int32_t count,
                                const int64_t *offsets, const int32_t *channel_ix,
                                const int32_t *channel_iy, const double *pkd,
                                const double *wave_b, const double *wave_c,
                                const int32_t *specular, const double *wave_a_spec);

/* Solve all systems.  psi_out (device, may be NULL): complex FP64 packed
 * rows [sum_s C_s][n_z] in system order.  intensities_out (device, may be
 * NULL): double [sum_s C_s] = |S_G0|^2.  results (host, may be NULL):
 * msc_result [n_systems].  stream is a cudaStream_t (NULL = legacy).
 * Mixed plans: a system still unconverged (or non-finite) after
 * max_refinements FP64 refinement steps is solved again in plain FP64 on the
 * same operator and right-hand side, starting from its mixed-precision
 * state (from zero if that went non-finite), before the results are
 * returned; its msc_result has fp64_fallback = 1 and counts both solves'
 * iterations.  Only a system the FP64 solve cannot converge either is
 * reported as MSC_ERR_NOT_CONVERGED, the reference's ierr 2
 * (multiscat_python_bindings.f90:58-60).  Flag bit 3 turns this off. */
msc_status msc_solve(msc_plan *plan, double *psi_out, double *intensities_out,
                     msc_result *results, void *stream);

/* Warm start: psi0 complex [total_rows][n_z] (plan row order) becomes the
 * initial guess of every following msc_solve (the reference's x0,
 * _gmres.py:106-108), e.g. the solution of a neighbouring beam in a sweep.
 * on_device != 0: device pointer read in order on `stream`; psi0 = NULL
 * returns to the zero guess.  The stop rule is unchanged (relative to ||u||). */
msc_status msc_plan_set_initial_guess(msc_plan *plan, const double *psi0, int32_t on_device,
                                      void *stream);

/* Total channel rows of the plan (sum of C_s) once all systems are set. */
int64_t msc_plan_total_rows(const msc_plan *plan);

/* Drop-in twin of the reference's run_multiscat_fortran (host buffers,
 * synchronous).  potential_values complex [nkx][nky][nz], perpendicular_
 * kinetic_difference [nkx][nky], waves complex [nkx*nky] (wave_a unused, as
 * in the reference), parallel_kinetic_energy [nz][nz]; scattered_state_out
 * complex [nkx][nky][nz].  gmres_preconditioner_flag is accepted for
 * signature parity (this solver always uses its block-diagonal
 * preconditioner); the stop rule is ||b - A psi|| <= 5e-4 * 10^-sig ||b||.
 * iterations_out may be NULL.  Returns 0, 1 (bad dims), 2 (not converged)
 * or another msc_status. */
int msc_run_multiscat(int gmres_preconditioner_flag, int convergence_significant_figures,
                      int nkx, int nky, int nz, const double *potential_values,
                      const double *perpendicular_kinetic_difference,
                      const double *wave_a, const double *wave_b, const double *wave_c,
                      const double *parallel_kinetic_energy, double *scattered_state_out,
                      int *iterations_out);

/* Debug / test entry points on device buffers of one full-grid system
 * (plan with n_systems == 1):
 *   msc_debug_apply_coupling:       y = sum_{G' != G} V_{G-G'} x_{G'}
 *   msc_debug_apply_block_inverse:  y = D^-1 x
 *   msc_debug_apply_operator:       y = A x = D x + V_off x
 * x, y: complex FP64 [C][n_z] device pointers. */
msc_status msc_debug_apply_coupling(msc_plan *plan, const double *x, double *y, void *stream);
msc_status msc_debug_apply_block_inverse(msc_plan *plan, const double *x, double *y, void *stream);
msc_status msc_debug_apply_operator(msc_plan *plan, const double *x, double *y, void *stream);

/* The reference's block Gauss-Seidel splitting A = L + U on device buffers
 * x, y (complex FP64 [total_rows][n_z], plan row order, x != y), system by
 * system, with "lower" meaning an earlier row of the same system (the
 * channel order the system was given in):
 *   msc_apply_lower_block: y = L x,    L = D + V^lower
 *   msc_solve_lower_block: y = L^-1 x  (forward sweep, one CTA per system,
 *                          rows in level sets)
 * Replace debug_solve_lower_block / _apply_lower_block /
 * _apply_inverse_lower_block (multiscat_gmres.f90:641-687,
 * multiscat/multiscat/_scipy.py:262-297, 357-380).  The reference's
 * interior state convention is L psi (_gmres.py:127, _multiscat.py:86-88). */
msc_status msc_apply_lower_block(msc_plan *plan, const double *x, double *y, void *stream);
msc_status msc_solve_lower_block(msc_plan *plan, const double *x, double *y, void *stream);

/* Allocation-free twin of msc_debug_apply_operator (no counterpart in the
 * reference): y = A x = D x + V_off x for ONE full-grid system, without a
 * plan and without allocating anything.  For callers that cannot call
 * cudaMalloc -- code running inside another framework's memory pool or
 * under a fixed device-memory budget, and plug-ins that may only use the
 * buffers they are handed.  Every argument is a device pointer:
 *   potential_values complex [nkx][nky][n_z], kinetic [n_z][n_z],
 *   pkd [nkx*nky], wave_c complex [nkx*nky], x and y complex [nkx*nky][n_z].
 * Working storage is a 32 MiB __device__ array inside the library, held by
 * every GPU that loads the library until the process exits; sizes whose tap
 * table, neighbour table and intermediate do not fit are rejected with
 * MSC_ERR_DIMS (nkx*nky <= 2049 channels, and about
 * 32 (nkx*nky) n_z + 4 (nkx*nky)^2 bytes in total).  The first call on each
 * device looks up the array's device address and sets kernel limits; make
 * it before any stream capture.  Every call waits on `stream` once: it
 * reads the number of nonzero taps and a non-finite-input flag back to the
 * host, and returns MSC_ERR_NONFINITE (as msc_plan_set_potential and
 * msc_plan_set_system do) when V, the kinetic matrix, pkd or wave_c holds a
 * NaN or infinity.  All calls share the array and keep the last call's
 * contents: calls that overlap on the GPU race. */
msc_status msc_apply_operator_noalloc(int32_t nkx, int32_t nky, int32_t n_z,
                                      const double *potential_values, const double *kinetic,
                                      const double *pkd, const double *wave_c, const double *x,
                                      double *y, void *stream);

/* Mixed-precision plans: y = D^-1 x with the FP32 kernel the inner solve
 * uses (tcgen05 BF16x3 when available), x and y complex FP32 packed rows. */
msc_status msc_debug_apply_block_inverse_f32(msc_plan *plan, const float *x, float *y, void *stream);

/* The FP64 eigen-decomposition msc_plan_set_potential uses for H0, on any
 * symmetric n x n host matrix a (row-major, 2 <= n <= 1024): w[n] ascending
 * eigenvalues, v[n*n] row-major with eigenvector k in column k.  Householder
 * tridiagonalisation and the eigenvector accumulations run on the current
 * device; the tridiagonal QR iteration (O(n^2)) on the host.  Replaces the
 * reference's rs (tred2 + tql2), diagsub.f90:5-262. */
msc_status msc_debug_symmetric_eigh(int32_t n, const double *a, double *w, double *v);

/* Tile width N of the tcgen05 block inverse the plan uses (0 = not used).
 * Valid after the first msc_solve or debug call. */
int msc_plan_uses_tensor_cores(const msc_plan *plan);

/* JSON text of the autotuner's timings (microseconds per candidate kernel)
 * and choices for this plan; owned by the plan, valid until the next call. */
const char *msc_plan_tuning_report(msc_plan *plan);

/* |S_G0|^2 per channel from psi[C][n_z] (device pointers), for one system. */
msc_status msc_intensities(msc_plan *plan, int32_t s, const double *psi, double *intensities,
                           void *stream);

/* Plan facts for callers and benchmarks. */
typedef struct {
    int64_t total_rows;        /* sum over systems of C_s                          */
    int32_t n_taps;            /* nonzero off-diagonal coupling taps               */
    int32_t n_tiles;           /* row tiles (kernel grid size)                     */
    int64_t launches_last;     /* kernel launches issued by the last msc_solve     */
    int32_t cycles_last;       /* restart cycles run by the last msc_solve         */
    int32_t fallbacks_last;    /* systems the last msc_solve re-solved in FP64     */
} msc_plan_info;

msc_status msc_plan_get_info(const msc_plan *plan, msc_plan_info *info);

/* Kernel timing (measurement only).  When enabled, the solve graphs carry
 * CUDA event pairs around every Arnoldi-step launch of kernel kind k
 * (0 = block-diagonal inverse, 1 = channel coupling, 2 = first projection,
 * 3 = update + second projection + Givens, 4 = normalisation) and msc_solve
 * adds the device time of the launches that did work.
 * msc_plan_kernel_timing copies ms[5] and launches[5] accumulated since the
 * previous call and resets them. */
msc_status msc_plan_set_kernel_timing(msc_plan *plan, int enable);
msc_status msc_plan_kernel_timing(msc_plan *plan, double *ms, int64_t *launches);

/* CUDA-core FMA throughput of the current GPU (measurement only; the
 * roofline denominator of the kernels that run on the FMA pipes, such as the
 * channel coupling).  Runs a kernel of independent fused multiply-adds on
 * every SM, FP32 for precision = MSC_PRECISION_MIXED and FP64 for
 * MSC_PRECISION_FP64, `iterations` FMAs per chain, timed with CUDA events on
 * `stream`; *flops = its floating-point operations (2 per FMA), *ms = its
 * device time.  No counterpart in the reference. */
msc_status msc_measure_fma_peak(int32_t precision, int32_t iterations, double *flops, float *ms,
                                void *stream);

/* ---- Adjoint differentiation (no counterpart in the reference, which has
 * no derivatives; the operator transposed is the one of
 * multiscat_gmres.f90:452-687 / _scipy.py:336-354).
 *
 * Forward:  A psi = u,  S_G = 2i b_G psi_G(z_n) + delta_{G,spec} a_spec.
 * For a real loss L(S) with gamma_G = dL/dRe S_G + i dL/dIm S_G:
 *   1. msc_plan_set_adjoint(plan, 1)                     operator -> A^H
 *   2. msc_plan_set_adjoint_rhs(plan, psi, dL/dI, dL/dS)  u_G = -i gamma_G conj(b_G)
 *   3. msc_solve(plan, lambda, NULL, ...)                 A^H lambda = u
 *   4. msc_potential_gradient(plan, psi, lambda, ...)     dL/dV
 *   5. msc_plan_set_adjoint(plan, 0); msc_plan_set_boundary_rhs(plan, NULL, ...)
 * The plan keeps its eigenbasis, tuning and graphs throughout. */

/* Select the operator the plan solves with: 0 = A, 1 = A^H (coupling taps
 * conj(V_{-d}) at offset d and c_G -> conj(c_G); D's eigenbasis is real and
 * unchanged).  Synchronises the device; no work of the plan may be in
 * flight.  msc_debug_apply_operator follows the selection. */
msc_status msc_plan_set_adjoint(msc_plan *plan, int32_t adjoint);
int msc_plan_is_adjoint(const msc_plan *plan);

/* Right-hand side on the outer boundary: rhs complex [total_rows] (plan row
 * order) is the source at z_n of each channel row; every other entry of the
 * right-hand side is zero.  rhs = NULL restores the scattering source
 * (b_spec at each system's specular row).  on_device != 0: rhs is a device
 * pointer read in order on `stream`.  Per-system norms are recomputed; a
 * system whose right-hand side is zero solves to psi = 0 at once. */
msc_status msc_plan_set_boundary_rhs(msc_plan *plan, const double *rhs, int32_t on_device,
                                     void *stream);

/* Adjoint right-hand side u_G = -i gamma_G conj(b_G) at z_n with
 * gamma = 2 dl_dintensity[G] S_G + dl_damplitude[G], S from psi (the
 * forward solution, complex [total_rows][n_z]).  Device pointers, in order on
 * `stream`; dl_dintensity (double [total_rows]) or dl_damplitude (complex
 * [total_rows]) may be NULL. */
msc_status msc_plan_set_adjoint_rhs(msc_plan *plan, const double *psi, const double *dl_dintensity,
                                    const double *dl_damplitude, void *stream);

/* dL/dV for the potential layout [nkx][nky][n_z] (complex, device), from
 * psi and lambda (device, complex [total_rows][n_z]), summed over the plan's
 * systems: grad[d][z] = -2 conj(K_d(z)) for d != 0 and -2 Re K_0(z) for
 * d = 0 (only Re V_0 enters), K_d(z) = sum_G conj(lambda_G(z)) psi_{G-d}(z),
 * in the (dL/dRe + i dL/dIm) convention.  half_x/half_y >= 0 restrict d to
 * |dx| <= half_x, |dy| <= half_y (signed torus offsets; entries outside are
 * written as 0); -1 = every offset of the torus. */
msc_status msc_potential_gradient(msc_plan *plan, const double *psi, const double *lambda,
                                  int32_t half_x, int32_t half_y, double *grad, void *stream);

/* Human-readable text of the last error on this thread. */
const char *msc_last_error(void);

/* Library version string. */
const char *msc_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MULTISCAT_B200_H */
