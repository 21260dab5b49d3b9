// msc_kernels.cuh -- kernels of the close-coupling GMRES solve.
//
// State layout in HBM: packed channel rows, psi[row][z] complex interleaved
// (double2 / float2), z contiguous.  A row is one diffraction channel of one
// system; the rows of a system are contiguous.  This is the reference's
// scattered_state(nz, C) column-major layout (multiscat_gmres.f90:144),
// extended with a batch of systems.
//
// Operator (per system):  A = D + V_off
//   (D psi)_G     = T psi_G + (Re V_00 + pkd_G) psi_G - c_G psi_G(z_n) e_n
//   (V_off psi)_G = sum_{G' != G} V_{(G-G') mod torus}(z) psi_{G'}(z)
// D_G^-1 uses the eigenbasis of H0 = T + diag Re V_00 (H0 = E diag(lam) E^T)
// and the Sherman-Morrison boundary term, as the reference's
// solve_lower_block does per channel (multiscat_gmres.f90:662-685) and
// apply_inverse_diagonal does for all channels (_scipy.py:249-259).
//
// The Krylov kernels are templated on the vector precision R: double for the
// plain FP64 solve, float for the inner solve of the mixed form.  Reductions
// (dot products, norms) always accumulate in FP64 and the GMRES scalars
// (Hessenberg, Givens, g) are FP64.
#pragma once

#include "msc_common.cuh"

namespace msc {

template <typename R> struct CT;
template <> struct CT<double> { using t = double2; };
template <> struct CT<float> { using t = float2; };

template <typename R>
__host__ __device__ __forceinline__ typename CT<R>::t mk2(R a, R b)
{
    typename CT<R>::t v;
    v.x = a;
    v.y = b;
    return v;
}

// ---------------------------------------------------------------------------
// Block-diagonal inverse:  out (=|+=) D^-1 x   on every row of a tile.
//   xt = E^T x ; s = sum_k en_k xt_k / (pkd + lam_k) ; beta = c s / (1 - c f_n)
//   yt = (xt + beta en) / (pkd + lam) ; u = E yt
// Two GEMMs along z with the tile's 2*TR real columns staged in shared
// memory; E and E^T stream from L2 (each is n*n values).  TR rows are
// processed per pass (8 for n <= 512, 4 above, so the two [n][2 TR] staging
// buffers fit in shared memory).  The diagonal scaling 1/(pkd + lam_k) and
// the Sherman-Morrison scalar are formed in FP64 for both precisions: near a
// channel resonance pkd + lam_k cancels, and an FP32 sum would make the FP32
// preconditioner inconsistent with D.
// ---------------------------------------------------------------------------
template <int TR, typename R>
__global__ void __launch_bounds__(256)
k_block_inverse(Tiles tiles, const int *__restrict__ gate, int n, const R *__restrict__ E,
                const R *__restrict__ ET, const double *__restrict__ lam,
                const double *__restrict__ en, const double *__restrict__ row_pkd,
                const double2 *__restrict__ row_c, const double *__restrict__ row_fn,
                const typename CT<R>::t *__restrict__ x, typename CT<R>::t *__restrict__ out,
                int accumulate)
{
    using C2 = typename CT<R>::t;
    constexpr int LD = 2 * TR;       // real columns per z row
    constexpr int HC = TR;           // columns handled per work item (half of LD)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *Xs = reinterpret_cast<R *>(smem_raw);   // [n][LD]
    R *Ys = Xs + (size_t)n * LD;
    __shared__ double2 beta_s[TR];

    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const int tile_row0 = tiles.row0[tile];
    const int tile_nrow = tiles.nrow[tile];

    for (int pass = 0; pass < tile_nrow; pass += TR) {
        const int row0 = tile_row0 + pass;
        const int nrow = min(TR, tile_nrow - pass);
        if (pass > 0) __syncthreads();

        for (int idx = threadIdx.x; idx < TR * n; idx += blockDim.x) {
            int r = idx / n, z = idx - r * n;
            C2 v = mk2<R>(0, 0);
            if (r < nrow) v = x[(size_t)(row0 + r) * n + z];
            Xs[z * LD + 2 * r] = v.x;
            Xs[z * LD + 2 * r + 1] = v.y;
        }
        __syncthreads();

        // GEMM 1: Ys[k][c] = sum_z E[z][k] Xs[z][c]
        for (int item = threadIdx.x; item < 2 * n; item += blockDim.x) {
            const int k = item >> 1, h = item & 1;
            R acc[HC];
#pragma unroll
            for (int c = 0; c < HC; ++c) acc[c] = 0;
            const R *xs = Xs + h * HC;
            const R *ek = E + k;
#pragma unroll 4
            for (int z = 0; z < n; ++z) {
                const R e = __ldg(ek + (size_t)z * n);
                const R *xr = xs + z * LD;
#pragma unroll
                for (int c = 0; c < HC; ++c) acc[c] = fma(e, xr[c], acc[c]);
            }
#pragma unroll
            for (int c = 0; c < HC; ++c) Ys[k * LD + h * HC + c] = acc[c];
        }
        __syncthreads();

        // Sherman-Morrison scalar of each row.
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        for (int r = warp; r < TR; r += (blockDim.x >> 5)) {
            double sr = 0.0, si = 0.0;
            if (r < nrow) {
                const double pk = row_pkd[row0 + r];
                for (int k = lane; k < n; k += 32) {
                    const double w = en[k] / (pk + lam[k]);
                    sr = fma(w, (double)Ys[k * LD + 2 * r], sr);
                    si = fma(w, (double)Ys[k * LD + 2 * r + 1], si);
                }
            }
            sr = warp_sum(sr);
            si = warp_sum(si);
            if (lane == 0) {
                double2 b = make_double2(0.0, 0.0);
                if (r < nrow) {
                    const double2 c = row_c[row0 + r];
                    const double fn = row_fn[row0 + r];
                    // beta = c s / (1 - c fn)
                    b = cdiv(cmul(c, make_double2(sr, si)), make_double2(1.0 - c.x * fn, -c.y * fn));
                }
                beta_s[r] = b;
            }
        }
        __syncthreads();

        for (int idx = threadIdx.x; idx < n * TR; idx += blockDim.x) {
            const int k = idx / TR, r = idx - k * TR;
            double inv = 0.0;
            if (r < nrow) inv = 1.0 / (row_pkd[row0 + r] + lam[k]);
            const double2 b = beta_s[r];
            const double ek = en[k];
            R *y = Ys + k * LD + 2 * r;
            y[0] = (R)(((double)y[0] + b.x * ek) * inv);
            y[1] = (R)(((double)y[1] + b.y * ek) * inv);
        }
        __syncthreads();

        // GEMM 2: out[z][c] = sum_k ET[k][z] Ys[k][c]
        for (int item = threadIdx.x; item < 2 * n; item += blockDim.x) {
            const int z = item >> 1, h = item & 1;
            R acc[HC];
#pragma unroll
            for (int c = 0; c < HC; ++c) acc[c] = 0;
            const R *ys = Ys + h * HC;
            const R *ez = ET + z;
#pragma unroll 4
            for (int k = 0; k < n; ++k) {
                const R e = __ldg(ez + (size_t)k * n);
                const R *yr = ys + k * LD;
#pragma unroll
                for (int c = 0; c < HC; ++c) acc[c] = fma(e, yr[c], acc[c]);
            }
#pragma unroll
            for (int rr = 0; rr < HC / 2; ++rr) {
                const int r = h * (HC / 2) + rr;
                if (r < nrow) {
                    C2 *o = out + (size_t)(row0 + r) * n + z;
                    C2 v = mk2<R>(acc[2 * rr], acc[2 * rr + 1]);
                    if (accumulate) {
                        const C2 prev = *o;
                        v.x += prev.x;
                        v.y += prev.y;
                    }
                    *o = v;
                }
            }
        }
    }  // pass
}

// ---------------------------------------------------------------------------
// Residual diagonal part (FP64):  out = b - D x  on every row of a tile.
//   D x = T x + (Re V00 + pkd) x - c x(z_n) e_n ; b = b_spec e_n on the
// specular row.  One FP64 GEMM with the symmetric T.  One item per
// (z, half of the tile's rows); the plan launches 2 n threads (rounded up to
// a warp) when that is at most 512, so that a block takes one round.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512)
k_residual_diag(Tiles tiles, const int *__restrict__ gate, int n,
                const double *__restrict__ Tm, const double *__restrict__ v00,
                const double *__restrict__ row_pkd, const double2 *__restrict__ row_c,
                const double2 *__restrict__ row_rhs,
                const double2 *__restrict__ x, double2 *__restrict__ out, int with_b)
{
    constexpr int TR = kTileRows;
    constexpr int LD = 2 * TR;
    constexpr int HC = TR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Xs = reinterpret_cast<double *>(smem_raw);  // [n][LD]

    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const int row0 = tiles.row0[tile];
    const int nrow = tiles.nrow[tile];

    for (int idx = threadIdx.x; idx < TR * n; idx += blockDim.x) {
        int r = idx / n, z = idx - r * n;
        double2 v = make_double2(0.0, 0.0);
        if (r < nrow) v = x[(size_t)(row0 + r) * n + z];
        Xs[z * LD + 2 * r] = v.x;
        Xs[z * LD + 2 * r + 1] = v.y;
    }
    __syncthreads();

    for (int item = threadIdx.x; item < 2 * n; item += blockDim.x) {
        const int z = item >> 1, h = item & 1;
        double acc[HC];
#pragma unroll
        for (int c = 0; c < HC; ++c) acc[c] = 0.0;
        const double *xs = Xs + h * HC;
        const double *tz = Tm + z;
#pragma unroll 4
        for (int k = 0; k < n; ++k) {
            const double t = __ldg(tz + (size_t)k * n);
            const double2 *xr = reinterpret_cast<const double2 *>(xs + k * LD);
#pragma unroll
            for (int c = 0; c < HC / 2; ++c) {
                double2 xv = xr[c];
                acc[2 * c] = fma(t, xv.x, acc[2 * c]);
                acc[2 * c + 1] = fma(t, xv.y, acc[2 * c + 1]);
            }
        }
        const double vz = v00[z];
#pragma unroll
        for (int rr = 0; rr < HC / 2; ++rr) {
            const int r = h * (HC / 2) + rr;
            if (r < nrow) {
                const int row = row0 + r;
                const double diag = vz + row_pkd[row];
                double2 xz = make_double2(Xs[z * LD + 2 * r], Xs[z * LD + 2 * r + 1]);
                double2 d = make_double2(acc[2 * rr] + diag * xz.x, acc[2 * rr + 1] + diag * xz.y);
                if (z == n - 1) d = csub(d, cmul(row_c[row], xz));
                double2 o = make_double2(-d.x, -d.y);
                if (with_b && z == n - 1) o = cadd(o, row_rhs[row]);
                out[(size_t)row * n + z] = o;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Channel coupling:  out = in0 + sgn * sum_t V_t(z) src[nbr[row][t]](z)
// The coupling sum is the reference's apply_upper_block + the coupling half
// of solve_lower_block (multiscat_gmres.f90:620-660) restricted to nonzero
// taps: a circular 2-D convolution over the channel torus at every z.
// Grid: (tiles, z-chunks of 32); block (32 z, kTileRows rows).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
k_coupling(Tiles tiles, const int *__restrict__ gate, int n, int K,
           const typename CT<R>::t *__restrict__ Vt, const int *__restrict__ nbr,
           const typename CT<R>::t *__restrict__ src, const typename CT<R>::t *__restrict__ in0,
           R sgn, typename CT<R>::t *__restrict__ out)
{
    using C2 = typename CT<R>::t;
    extern __shared__ int nb_s[];   // [kTileRows][K]
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const int row0 = tiles.row0[tile];
    const int nrow = tiles.nrow[tile];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < nrow * K; i += blockDim.x * blockDim.y)
        nb_s[i] = nbr[(size_t)row0 * K + i];
    __syncthreads();
    const int r = threadIdx.y;
    const int z = blockIdx.y * blockDim.x + threadIdx.x;
    if (r >= nrow || z >= n) return;
    const int *nb = nb_s + r * K;
    R ar = 0, ai = 0, br = 0, bi = 0;
    int t = 0;
    for (; t + 1 < K; t += 2) {
        const int j0 = nb[t], j1 = nb[t + 1];
        const C2 v0 = Vt[(size_t)t * n + z];
        const C2 v1 = Vt[(size_t)(t + 1) * n + z];
        if (j0 >= 0) {
            const C2 s0 = src[(size_t)j0 * n + z];
            ar = fma(v0.x, s0.x, ar); ar = fma(-v0.y, s0.y, ar);
            ai = fma(v0.x, s0.y, ai); ai = fma(v0.y, s0.x, ai);
        }
        if (j1 >= 0) {
            const C2 s1 = src[(size_t)j1 * n + z];
            br = fma(v1.x, s1.x, br); br = fma(-v1.y, s1.y, br);
            bi = fma(v1.x, s1.y, bi); bi = fma(v1.y, s1.x, bi);
        }
    }
    if (t < K) {
        const int j0 = nb[t];
        const C2 v0 = Vt[(size_t)t * n + z];
        if (j0 >= 0) {
            const C2 s0 = src[(size_t)j0 * n + z];
            ar = fma(v0.x, s0.x, ar); ar = fma(-v0.y, s0.y, ar);
            ai = fma(v0.x, s0.y, ai); ai = fma(v0.y, s0.x, ai);
        }
    }
    const size_t o = (size_t)(row0 + r) * n + z;
    C2 base = in0 ? in0[o] : mk2<R>(0, 0);
    out[o] = mk2<R>(base.x + sgn * (ar + br), base.y + sgn * (ai + bi));
}

// ---------------------------------------------------------------------------
// Triangular parts of the channel coupling in plan row order (the row order
// of a system is its channel order):
//   mask 1 (lower): out = in0 + sgn * sum_{t: nbr < row} V_t src[nbr]
//   mask 2 (upper): out = in0 + sgn * sum_{t: nbr > row} V_t src[nbr]
// the reference's V^lower and V^upper of its block Gauss-Seidel splitting
// A = L + U, L = D + V^lower (multiscat_gmres.f90:620-660, _scipy.py:81-102,
// 262-297).  Same layout as k_coupling.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
k_coupling_masked(Tiles tiles, const int *__restrict__ gate, int n, int K,
                  const typename CT<R>::t *__restrict__ Vt, const int *__restrict__ nbr,
                  const typename CT<R>::t *__restrict__ src,
                  const typename CT<R>::t *__restrict__ in0, R sgn, int mask,
                  typename CT<R>::t *__restrict__ out)
{
    using C2 = typename CT<R>::t;
    extern __shared__ int nbm_s[];   // [kTileRows][K]
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const int row0 = tiles.row0[tile];
    const int nrow = tiles.nrow[tile];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < nrow * K; i += blockDim.x * blockDim.y) {
        const int row = row0 + i / K;
        const int j = nbr[(size_t)row0 * K + i];
        const bool keep = j >= 0 && (mask == 1 ? j < row : j > row);
        nbm_s[i] = keep ? j : -1;
    }
    __syncthreads();
    const int r = threadIdx.y;
    const int z = blockIdx.y * blockDim.x + threadIdx.x;
    if (r >= nrow || z >= n) return;
    const int *nb = nbm_s + r * K;
    R ar = 0, ai = 0;
    for (int t = 0; t < K; ++t) {
        const int j = nb[t];
        if (j < 0) continue;
        const C2 v = Vt[(size_t)t * n + z];
        const C2 sv = src[(size_t)j * n + z];
        ar = fma(v.x, sv.x, ar); ar = fma(-v.y, sv.y, ar);
        ai = fma(v.x, sv.y, ai); ai = fma(v.y, sv.x, ai);
    }
    const size_t o = (size_t)(row0 + r) * n + z;
    C2 base = in0 ? in0[o] : mk2<R>(0, 0);
    out[o] = mk2<R>(base.x + sgn * ar, base.y + sgn * ai);
}

// ---------------------------------------------------------------------------
// Block Gauss-Seidel forward sweep y = L^-1 x, L = D + V^lower: the
// reference's solve_lower_block / _apply_inverse_lower_block
// (multiscat_gmres.f90:641-687, _scipy.py:262-297), channel after channel
//   y_r = D_r^-1 (x_r - sum_{r' < r} V_{r r'} y_{r'}).
// One CTA per system.  Rows are taken level by level (a row's level is one
// more than the highest level among its lower neighbours, so the rows of a
// level do not depend on each other), up to kGsRows rows of a level at a
// time, each phase spread over all threads of the CTA:
//   A  s_b(z) = x_b(z) - sum_{lower taps} V_t(z) y_{nbr}(z)     (b, z) per thread
//   B  xt_b(k) = sum_z E(z, k) s_b(z)                           (b, k) per thread
//   C  beta_b = c sigma / (1 - c f_n), sigma = sum_k en_k xt_b(k) / (pkd_b + lam_k)
//   D  yt_b(k) = (xt_b(k) + beta_b en_k) / (pkd_b + lam_k)
//   E  y_b(z) = sum_k E(z, k) yt_b(k)                           (b, z) per thread
// with D_r^-1 in the eigenbasis of H0 and the Sherman-Morrison boundary
// term, as k_block_inverse.  E (FP64, or FP32 in the mixed form's inner
// solve) sits in shared memory with a row stride of n + 1 (both the k-major
// and the z-major walk are free of bank conflicts) when it fits, else it is
// read from L2.  pkd + lam is formed in FP64 for both precisions.
// ---------------------------------------------------------------------------
struct GsLevels {
    const int *sys_lvl;     // [B + 1]  first level of each system
    const int *lvl_start;   // [levels + 1]  first entry of each level in lvl_rows
    const int *lvl_rows;    // [R]  rows, system by system, level by level
    const int *low_ptr;     // [R + 1]  each row's lower neighbours at low_ptr[r] .. low_ptr[r + 1]
    const int *low_tap;     //          their coupling tap
    const int *low_row;     //          and their row
};

constexpr int kGsRows = 8;

template <typename R>
__global__ void __launch_bounds__(256)
k_gs_sweep(int nsys, const int *__restrict__ gate, int n, int K,
           const typename CT<R>::t *__restrict__ Vt, const int *__restrict__ nbr, GsLevels lv,
           const R *__restrict__ E, int e_in_smem, const double *__restrict__ lam,
           const double *__restrict__ en, const double *__restrict__ row_pkd,
           const double2 *__restrict__ row_c, const double *__restrict__ row_fn,
           const typename CT<R>::t *__restrict__ x, typename CT<R>::t *__restrict__ y)
{
    using C2 = typename CT<R>::t;
    extern __shared__ __align__(16) unsigned char gs_raw[];
    const int s = blockIdx.x;
    if (s >= nsys || (gate && gate[s] == 0)) return;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int ld = e_in_smem ? n + 1 : n;
    R *Es = reinterpret_cast<R *>(gs_raw);
    C2 *sv = reinterpret_cast<C2 *>(gs_raw + (e_in_smem ? ((size_t)n * ld * sizeof(R) + 15) / 16 * 16 : 0));
    C2 *tv = sv + (size_t)kGsRows * n;
    __shared__ double2 beta_s[kGsRows];
    __shared__ int row_s[kGsRows];
    if (e_in_smem) {
        for (int i = tid; i < n * n; i += nt) {
            const int z = i / n, k = i - z * n;
            Es[z * ld + k] = E[i];
        }
    }
    const R *Em = e_in_smem ? Es : E;
    __syncthreads();
    for (int L = lv.sys_lvl[s]; L < lv.sys_lvl[s + 1]; ++L) {
        for (int i0 = lv.lvl_start[L]; i0 < lv.lvl_start[L + 1]; i0 += kGsRows) {
            const int nb = min(kGsRows, lv.lvl_start[L + 1] - i0);
            if (tid < nb) row_s[tid] = lv.lvl_rows[i0 + tid];
            __syncthreads();
            // A: right-hand side minus the lower coupling
            for (int idx = tid; idx < nb * n; idx += nt) {
                const int b = idx / n, z = idx - b * n;
                const int r = row_s[b];
                const C2 xv = x[(size_t)r * n + z];
                R ar = xv.x, ai = xv.y;
                const int e1 = __ldg(lv.low_ptr + r + 1);
#pragma unroll 8
                for (int e = __ldg(lv.low_ptr + r); e < e1; ++e) {
                    const int t = __ldg(lv.low_tap + e), j = __ldg(lv.low_row + e);
                    const C2 v = Vt[(size_t)t * n + z];
                    const C2 u = y[(size_t)j * n + z];
                    ar -= v.x * u.x - v.y * u.y;
                    ai -= v.x * u.y + v.y * u.x;
                }
                sv[(size_t)b * n + z] = mk2<R>(ar, ai);
            }
            __syncthreads();
            // B: xt = E^T s
            for (int idx = tid; idx < nb * n; idx += nt) {
                const int b = idx / n, k = idx - b * n;
                const C2 *sb = sv + (size_t)b * n;
                R ar = 0, ai = 0;
#pragma unroll 4
                for (int z = 0; z < n; ++z) {
                    const R e = Em[(size_t)z * ld + k];
                    const C2 q = sb[z];
                    ar = fma(e, q.x, ar);
                    ai = fma(e, q.y, ai);
                }
                tv[(size_t)b * n + k] = mk2<R>(ar, ai);
            }
            __syncthreads();
            // C: the Sherman-Morrison scalar of each row, one warp per row
            for (int b = warp; b < nb; b += nt >> 5) {
                const int r = row_s[b];
                const double pk = row_pkd[r];
                double sr = 0.0, si = 0.0;
                for (int k = lane; k < n; k += 32) {
                    const double w = en[k] / (pk + lam[k]);
                    const C2 q = tv[(size_t)b * n + k];
                    sr = fma(w, (double)q.x, sr);
                    si = fma(w, (double)q.y, si);
                }
                sr = warp_sum(sr);
                si = warp_sum(si);
                if (lane == 0) {
                    const double2 c = row_c[r];
                    const double fn = row_fn[r];
                    beta_s[b] = cdiv(cmul(c, make_double2(sr, si)), make_double2(1.0 - c.x * fn, -c.y * fn));
                }
            }
            __syncthreads();
            // D: yt = (xt + beta en) / (pkd + lam)
            for (int idx = tid; idx < nb * n; idx += nt) {
                const int b = idx / n, k = idx - b * n;
                const double inv = 1.0 / (row_pkd[row_s[b]] + lam[k]);
                const double2 bb = beta_s[b];
                const C2 q = tv[idx];
                tv[idx] = mk2<R>((R)(((double)q.x + bb.x * en[k]) * inv),
                                 (R)(((double)q.y + bb.y * en[k]) * inv));
            }
            __syncthreads();
            // E: y = E yt
            for (int idx = tid; idx < nb * n; idx += nt) {
                const int b = idx / n, z = idx - b * n;
                const C2 *tb = tv + (size_t)b * n;
                const R *ez = Em + (size_t)z * ld;
                R ar = 0, ai = 0;
#pragma unroll 4
                for (int k = 0; k < n; ++k) {
                    const R e = ez[k];
                    const C2 q = tb[k];
                    ar = fma(e, q.x, ar);
                    ai = fma(e, q.y, ai);
                }
                y[(size_t)row_s[b] * n + z] = mk2<R>(ar, ai);
            }
            __syncthreads();    // these rows are written before the next rows read them
        }
    }
}

// ---------------------------------------------------------------------------
// Channel coupling with shared-memory halo tiles (the hot form of k_coupling).
//
// A block owns an 8 x BX patch of torus positions of ONE system and ZC
// consecutive z.  It stages the patch plus a halo of HX (x) and HY (y)
// positions -- the reach of the coupling taps -- for its z range in shared
// memory (absent channels, i.e. positions outside a truncated channel set,
// read as zero; positions wrap around the torus exactly as the reference's
// modulo(G_j - G_i, n) does).  Each thread keeps one column of YS + 2 HY halo
// values in registers and produces YS outputs along y for one (x, z):
// for every tap (sdx, sdy) in the window it issues YS complex FMAs from
// registers, so a halo value loaded once serves up to 2 HY + 1 taps.
//   out[r] = in0[r] + sgn * sum_t V_t(z) src[pos(r) - delta_t](z)
// ---------------------------------------------------------------------------
struct CouplingTiles {
    const int *work;          // [nwork][3]: system, x0, y0
    const int *pos_row;       // [B][nkx * nky]: row of each torus position, -1 if absent
    const int *tap_window;    // [(2 HX + 1) * (2 HY + 1)]: tap index per signed offset, -1 if none
    int nwork, nkx, nky, hx;  // hx = HX (runtime); HY is the template parameter
    int ntaps;                // K
};

// MASK 1 / 2: only the source channels with a smaller / larger row index
// than the output's (V^lower / V^upper of the block Gauss-Seidel splitting,
// as k_coupling_masked); 0: the full coupling.
template <int HY, int BX, int ZC, int YS, typename R, int MASK = 0>
__global__ void __launch_bounds__(BX * ZC * (8 / YS))
k_coupling_halo(CouplingTiles ct, const int *__restrict__ gate, int n,
                const typename CT<R>::t *__restrict__ Vt, const typename CT<R>::t *__restrict__ src,
                const typename CT<R>::t *__restrict__ in0, R sgn, typename CT<R>::t *__restrict__ out)
{
    // YS outputs along y per thread; 8 / YS threads share one (x, z) column.
    using C2 = typename CT<R>::t;
    constexpr int BY = 8;
    constexpr int HYW = BY + 2 * HY;
    constexpr int WY = 2 * HY + 1;
    constexpr int NT = BX * ZC * (BY / YS);
    constexpr int CW = YS + 2 * HY;              // halo values one thread keeps per column
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int HX = ct.hx;
    const int HXW = BX + 2 * HX;
    const int nwin = (2 * HX + 1) * WY;
    C2 *halo = reinterpret_cast<C2 *>(smem_raw);                              // [HXW][HYW][ZC]
    C2 *vw = halo + (size_t)HXW * HYW * ZC;                                   // [window cell][ZC]
    int *rows = reinterpret_cast<int *>(vw + (size_t)nwin * ZC);              // [HXW][HYW]
    // Threads whose y segment (YS positions) of their patch column holds no
    // channel skip the tap loop (truncated channel sets leave many near the
    // edge of the channel disk); the test reads the staged rows table.

    const int w = blockIdx.x;
    const int s = ct.work[3 * w];
    if (gate && gate[s] == 0) return;
    const int x0 = ct.work[3 * w + 1], y0 = ct.work[3 * w + 2];
    const int z0 = blockIdx.y * ZC;
    const int nkx = ct.nkx, nky = ct.nky;
    const int *pr = ct.pos_row + (size_t)s * nkx * nky;
    // tap values of this z range, one row per window cell (zero where no tap)
    for (int i = threadIdx.x; i < nwin * ZC; i += NT) {
        const int cell = i / ZC, z = z0 + (i % ZC);
        const int t = ct.tap_window[cell];
        vw[i] = (t >= 0 && z < n) ? Vt[(size_t)t * n + z] : mk2<R>(0, 0);
    }
    // source row of every halo position (absent channels: -1)
    const int npos = HXW * HYW;
    for (int pidx = threadIdx.x; pidx < npos; pidx += NT) {
        const int hy = pidx % HYW, hx = pidx / HYW;
        int gx = (x0 + hx - HX) % nkx;
        if (gx < 0) gx += nkx;
        int gy = (y0 + hy - HY) % nky;
        if (gy < 0) gy += nky;
        rows[pidx] = pr[gx * nky + gy];
    }
    __syncthreads();
    constexpr int kU = 8;
    const int total = npos * ZC;
    if (std::is_same<R, float>::value && (n % 2) == 0) {
        // FP32, n even: two consecutive z per 16-byte load (z0 and ZC are even)
        const int total2 = total / 2;
        float4 *halo4 = reinterpret_cast<float4 *>(halo);
        for (int base = threadIdx.x; base < total2; base += NT * kU) {
            float4 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (idx < total2) {
                    const int row = rows[(2 * idx) / ZC];
                    const int z = z0 + ((2 * idx) % ZC);
                    if (row >= 0 && z < n)    // z < n implies z + 1 < n (both even)
                        v[u] = *reinterpret_cast<const float4 *>(src + (size_t)row * n + z);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total2) halo4[idx] = v[u];
            }
        }
    } else {
        for (int base = threadIdx.x; base < total; base += NT * kU) {
            C2 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = mk2<R>(0, 0);
                if (idx < total) {
                    const int row = rows[idx / ZC];
                    const int z = z0 + (idx % ZC);
                    if (row >= 0 && z < n) v[u] = src[(size_t)row * n + z];
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total) halo[idx] = v[u];
            }
        }
    }
    __syncthreads();

    const int zl = threadIdx.x % ZC;
    const int tx = (threadIdx.x / ZC) % BX;
    const int ysub = threadIdx.x / (ZC * BX);      // which YS-slice of the 8 y outputs
    const int z = z0 + zl;
    bool any = false;
#pragma unroll
    for (int y = ysub * YS; y < (ysub + 1) * YS; ++y)
        any |= (y0 + y < nky) && rows[(tx + HX) * HYW + y + HY] >= 0;
    if (x0 + tx >= nkx || z >= n || !any) return;
    R ar[YS], ai[YS];
#pragma unroll
    for (int y = 0; y < YS; ++y) {
        ar[y] = 0;
        ai[y] = 0;
    }
    int orow[MASK ? YS : 1];
    if (MASK) {
#pragma unroll
        for (int y = 0; y < YS; ++y) orow[y] = rows[(tx + HX) * HYW + ysub * YS + y + HY];
    }
    for (int sdx = -HX; sdx <= HX; ++sdx) {
        const int hx = tx - sdx + HX;
        const C2 *colp = halo + ((size_t)hx * HYW + ysub * YS) * ZC + zl;
        C2 col[CW];
#pragma unroll
        for (int i = 0; i < CW; ++i) col[i] = colp[(size_t)i * ZC];
        int crow[MASK ? CW : 1];
        if (MASK) {
#pragma unroll
            for (int i = 0; i < CW; ++i) crow[i] = rows[hx * HYW + ysub * YS + i];
        }
        const C2 *vrow = vw + (size_t)(sdx + HX) * WY * ZC + zl;
#pragma unroll
        for (int sdy = -HY; sdy <= HY; ++sdy) {
            const C2 v = vrow[(sdy + HY) * ZC];
#pragma unroll
            for (int y = 0; y < YS; ++y) {
                C2 q = col[y - sdy + HY];
                if (MASK) {
                    const int sr = crow[MASK ? y - sdy + HY : 0], orr = orow[MASK ? y : 0];
                    const bool keep = MASK == 1 ? sr < orr : sr > orr;
                    if (!keep) q = mk2<R>(0, 0);
                }
                ar[y] = fma(v.x, q.x, fma(-v.y, q.y, ar[y]));
                ai[y] = fma(v.x, q.y, fma(v.y, q.x, ai[y]));
            }
        }
    }
    // output rows from the staged rows table; the in0 loads of all YS
    // outputs go out before the stores
    int rowv[YS];
    C2 base[YS];
#pragma unroll
    for (int y = 0; y < YS; ++y)
        rowv[y] = (y0 + ysub * YS + y < nky) ? rows[(tx + HX) * HYW + ysub * YS + y + HY] : -1;
#pragma unroll
    for (int y = 0; y < YS; ++y)
        base[y] = (in0 && rowv[y] >= 0) ? in0[(size_t)rowv[y] * n + z] : mk2<R>(0, 0);
#pragma unroll
    for (int y = 0; y < YS; ++y)
        if (rowv[y] >= 0)
            out[(size_t)rowv[y] * n + z] = mk2<R>(base[y].x + sgn * ar[y], base[y].y + sgn * ai[y]);
}

// ---------------------------------------------------------------------------
// Channel coupling of a separable potential: when every z's tap window
// factorises as V_(sdx, sdy)(z) = p_sdx(z) q_sdy(z) off the centre (the
// corrugated Morse potential of a square lattice, xi = (h/2)(cos X + cos Y),
// gives exactly that: the FFT of e^{2 alpha xi} is a product of two 1-D
// transforms), the 2-D convolution is a pass along x and a pass along y:
//   t(x, y')  = sum_sdx p_sdx src(x - sdx, y')            (y' over the halo)
//   out(x, y) = in0 + sgn [sum_sdy q_sdy t(x, y - sdy) - kappa src(x, y)]
// with kappa = p_0 q_0 the product's value at the centre, which is no tap.
// (2 HX + 1) (8 + 2 HY) + 8 (2 HY + 2) complex MACs per thread for 8
// outputs instead of 8 K: 28 instead of 80 per output for |m|,|n| <= 4, 43
// instead of 288 for |m|,|n| <= 8.  A thread owns one (x, z) column of the
// 8 x 8 patch: pass 1 keeps the column's 8 + 2 HY values of t in registers,
// pass 2 reads nothing but its own registers and the q row.  The halo of the
// patch is staged as in k_coupling_halo.
// ---------------------------------------------------------------------------
struct SepTaps {
    const void *p;       // [2 HX + 1][n] complex (R), p_sdx at sdx + HX
    const void *q;       // [2 HY + 1][n] complex (R), q_sdy at sdy + HY
    const void *kappa;   // [n] complex (R)
};

// (Staging the halo by one bulk copy per halo position instead, on an
// mbarrier, measured the same: 283 against 280 us on the 512-beam batch.)
// HXT > 0 fixes the x reach at compile time (square windows: HXT = HY), so
// the x pass over the 2 HX + 1 halo columns unrolls; 0 takes it from ct.hx.
template <int HY, int BX, int ZC, typename R, int HXT = 0>
__global__ void __launch_bounds__(BX * ZC, HY <= 4 ? 3 : 1)
k_coupling_sep(CouplingTiles ct, const int *__restrict__ gate, int n, SepTaps sep,
               const typename CT<R>::t *__restrict__ src, const typename CT<R>::t *__restrict__ in0,
               R sgn, typename CT<R>::t *__restrict__ out)
{
    using C2 = typename CT<R>::t;
    constexpr int BY = 8;
    constexpr int HYW = BY + 2 * HY;
    constexpr int WY = 2 * HY + 1;
    constexpr int NT = BX * ZC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int HX = HXT > 0 ? HXT : ct.hx;
    const int HXW = BX + 2 * HX;
    const int WX = 2 * HX + 1;
    C2 *halo = reinterpret_cast<C2 *>(smem_raw);                       // [HXW][HYW][ZC]
    C2 *pw = halo + (size_t)HXW * HYW * ZC;                            // [WX][ZC]
    C2 *qw = pw + (size_t)WX * ZC;                                     // [WY][ZC]
    C2 *kw = qw + (size_t)WY * ZC;                                     // [ZC]
    int *rows = reinterpret_cast<int *>(kw + ZC);                      // [HXW][HYW]

    const int w = blockIdx.x;
    const int s = ct.work[3 * w];
    if (gate && gate[s] == 0) return;
    const int x0 = ct.work[3 * w + 1], y0 = ct.work[3 * w + 2];
    const int z0 = blockIdx.y * ZC;
    const int nkx = ct.nkx, nky = ct.nky;
    const int *pr = ct.pos_row + (size_t)s * nkx * nky;
    const C2 *P = reinterpret_cast<const C2 *>(sep.p);
    const C2 *Qv = reinterpret_cast<const C2 *>(sep.q);
    const C2 *Kp = reinterpret_cast<const C2 *>(sep.kappa);
    for (int i = threadIdx.x; i < (WX + WY + 1) * ZC; i += NT) {
        const int row = i / ZC, z = z0 + (i % ZC);
        C2 v = mk2<R>(0, 0);
        if (z < n) v = row < WX ? P[(size_t)row * n + z]
                     : row < WX + WY ? Qv[(size_t)(row - WX) * n + z] : Kp[z];
        pw[i] = v;          // pw, qw and kw are consecutive
    }
    const int npos = HXW * HYW;
    for (int pidx = threadIdx.x; pidx < npos; pidx += NT) {
        const int hy = pidx % HYW, hx = pidx / HYW;
        int gx = (x0 + hx - HX) % nkx;
        if (gx < 0) gx += nkx;
        int gy = (y0 + hy - HY) % nky;
        if (gy < 0) gy += nky;
        rows[pidx] = pr[gx * nky + gy];
    }
    __syncthreads();
    const int total = npos * ZC;
    constexpr int kU = 8;
    if (std::is_same<R, float>::value && (n % 2) == 0) {
        const int total2 = total / 2;
        float4 *halo4 = reinterpret_cast<float4 *>(halo);
        for (int base = threadIdx.x; base < total2; base += NT * kU) {
            float4 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (idx < total2) {
                    const int row = rows[(2 * idx) / ZC];
                    const int z = z0 + ((2 * idx) % ZC);
                    if (row >= 0 && z < n)
                        v[u] = *reinterpret_cast<const float4 *>(src + (size_t)row * n + z);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total2) halo4[idx] = v[u];
            }
        }
    } else {
        for (int base = threadIdx.x; base < total; base += NT * kU) {
            C2 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = mk2<R>(0, 0);
                if (idx < total) {
                    const int row = rows[idx / ZC];
                    const int z = z0 + (idx % ZC);
                    if (row >= 0 && z < n) v[u] = src[(size_t)row * n + z];
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total) halo[idx] = v[u];
            }
        }
    }
    __syncthreads();

    const int zl = threadIdx.x % ZC;
    const int tx = threadIdx.x / ZC;
    const int z = z0 + zl;
    bool any = false;       // a channel in this patch column (staged rows table)
#pragma unroll
    for (int y = 0; y < BY; ++y) any |= (y0 + y < nky) && rows[(tx + HX) * HYW + y + HY] >= 0;
    if (x0 + tx >= nkx || z >= n || !any) return;
    // pass 1: t(hy) = sum_sdx p_sdx halo(tx - sdx + HX, hy) over the halo column
    R tr[HYW], ti[HYW];
#pragma unroll
    for (int i = 0; i < HYW; ++i) {
        tr[i] = 0;
        ti[i] = 0;
    }
#pragma unroll
    for (int sdx = -HX; sdx <= HX; ++sdx) {
        const C2 pv = pw[(sdx + HX) * ZC + zl];
        const C2 *colp = halo + (size_t)(tx - sdx + HX) * HYW * ZC + zl;
#pragma unroll
        for (int i = 0; i < HYW; ++i) {
            const C2 v = colp[(size_t)i * ZC];
            tr[i] = fma(pv.x, v.x, fma(-pv.y, v.y, tr[i]));
            ti[i] = fma(pv.x, v.y, fma(pv.y, v.x, ti[i]));
        }
    }
    // pass 2: out(y) = sum_sdy q_sdy t(y - sdy + HY) - kappa src(x, y)
    C2 qv[WY];
#pragma unroll
    for (int i = 0; i < WY; ++i) qv[i] = qw[i * ZC + zl];
    const C2 kap = kw[zl];
    const C2 *own = halo + (size_t)(tx + HX) * HYW * ZC + zl;
    // the patch column's rows come from the staged rows table (its interior
    // positions), and the in0 values of all BY outputs are loaded before the
    // arithmetic: no global load waits on another inside the output loop
    int rowv[BY];
    C2 base[BY];
#pragma unroll
    for (int y = 0; y < BY; ++y)
        rowv[y] = (y0 + y < nky) ? rows[(tx + HX) * HYW + y + HY] : -1;
#pragma unroll
    for (int y = 0; y < BY; ++y)
        base[y] = (in0 && rowv[y] >= 0) ? in0[(size_t)rowv[y] * n + z] : mk2<R>(0, 0);
#pragma unroll
    for (int y = 0; y < BY; ++y) {
        if (rowv[y] < 0) continue;
        const C2 c = own[(size_t)(y + HY) * ZC];
        R ar = -(kap.x * c.x - kap.y * c.y), ai = -(kap.x * c.y + kap.y * c.x);
#pragma unroll
        for (int sdy = -HY; sdy <= HY; ++sdy) {
            const C2 q = qv[sdy + HY];
            const R xr = tr[y - sdy + HY], xi = ti[y - sdy + HY];
            ar = fma(q.x, xr, fma(-q.y, xi, ar));
            ai = fma(q.x, xi, fma(q.y, xr, ai));
        }
        out[(size_t)rowv[y] * n + z] = mk2<R>(base[y].x + sgn * ar, base[y].y + sgn * ai);
    }
}

// The separable coupling with the x pass run along the halo rows: one
// thread per (halo row, z) holds the row's BX + 2 HX values in registers
// and writes the BX values of t over the row's middle columns; the y pass
// then runs per (x, z) column as in k_coupling_sep.  Each halo value is read
// from shared memory once by the x pass instead of by up to 2 HX + 1
// threads: about half the shared-memory operations of k_coupling_sep, whose
// x pass is bound by them.  With 2 HX >= BX the row's t values go to its
// 2 HX outer columns (already read), so the patch's own values stay for
// the kappa term; narrower windows write t over the patch columns and keep
// the own values in registers.  The x reach HXT is a template parameter
// (the row lives in registers); the plan runs this form only for windows
// with hx = HXT.
template <int HY, int BX, int ZC, typename R, int HXT>
__global__ void __launch_bounds__(BX * ZC, HY <= 4 ? 3 : 1)
k_coupling_sep_rows(CouplingTiles ct, const int *__restrict__ gate, int n, SepTaps sep,
                    const typename CT<R>::t *__restrict__ src,
                    const typename CT<R>::t *__restrict__ in0, R sgn,
                    typename CT<R>::t *__restrict__ out)
{
    using C2 = typename CT<R>::t;
    constexpr int BY = 8;
    constexpr int HYW = BY + 2 * HY;
    constexpr int WY = 2 * HY + 1;
    constexpr int NT = BX * ZC;
    constexpr int HX = HXT;
    constexpr int HXW = BX + 2 * HX;
    constexpr int WX = 2 * HX + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2 *halo = reinterpret_cast<C2 *>(smem_raw);                       // [HXW][HYW][ZC]
    C2 *pw = halo + (size_t)HXW * HYW * ZC;                            // [WX][ZC]
    C2 *qw = pw + (size_t)WX * ZC;                                     // [WY][ZC]
    C2 *kw = qw + (size_t)WY * ZC;                                     // [ZC]
    int *rows = reinterpret_cast<int *>(kw + ZC);                      // [HXW][HYW]

    const int w = blockIdx.x;
    const int s = ct.work[3 * w];
    if (gate && gate[s] == 0) return;
    const int x0 = ct.work[3 * w + 1], y0 = ct.work[3 * w + 2];
    const int z0 = blockIdx.y * ZC;
    const int nkx = ct.nkx, nky = ct.nky;
    const int *pr = ct.pos_row + (size_t)s * nkx * nky;
    const C2 *P = reinterpret_cast<const C2 *>(sep.p);
    const C2 *Qv = reinterpret_cast<const C2 *>(sep.q);
    const C2 *Kp = reinterpret_cast<const C2 *>(sep.kappa);
    for (int i = threadIdx.x; i < (WX + WY + 1) * ZC; i += NT) {
        const int row = i / ZC, z = z0 + (i % ZC);
        C2 v = mk2<R>(0, 0);
        if (z < n) v = row < WX ? P[(size_t)row * n + z]
                     : row < WX + WY ? Qv[(size_t)(row - WX) * n + z] : Kp[z];
        pw[i] = v;          // pw, qw and kw are consecutive
    }
    constexpr int npos = HXW * HYW;
    for (int pidx = threadIdx.x; pidx < npos; pidx += NT) {
        const int hy = pidx % HYW, hx = pidx / HYW;
        int gx = (x0 + hx - HX) % nkx;
        if (gx < 0) gx += nkx;
        int gy = (y0 + hy - HY) % nky;
        if (gy < 0) gy += nky;
        rows[pidx] = pr[gx * nky + gy];
    }
    __syncthreads();
    constexpr int kU = 8;
    constexpr int total = npos * ZC;
    if (std::is_same<R, float>::value && (n % 2) == 0) {
        constexpr int total2 = total / 2;
        float4 *halo4 = reinterpret_cast<float4 *>(halo);
        for (int base = threadIdx.x; base < total2; base += NT * kU) {
            float4 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (idx < total2) {
                    const int row = rows[(2 * idx) / ZC];
                    const int z = z0 + ((2 * idx) % ZC);
                    if (row >= 0 && z < n)
                        v[u] = *reinterpret_cast<const float4 *>(src + (size_t)row * n + z);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total2) halo4[idx] = v[u];
            }
        }
    } else {
        for (int base = threadIdx.x; base < total; base += NT * kU) {
            C2 v[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                v[u] = mk2<R>(0, 0);
                if (idx < total) {
                    const int row = rows[idx / ZC];
                    const int z = z0 + (idx % ZC);
                    if (row >= 0 && z < n) v[u] = src[(size_t)row * n + z];
                }
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int idx = base + u * NT;
                if (idx < total) halo[idx] = v[u];
            }
        }
    }
    __syncthreads();

    // t(x) goes to column tcol(x): the outer columns x < HX and
    // HX + BX .. HX + BX + (BX - HX) - 1 when they are enough, else over
    // the patch columns HX + x
    constexpr bool kOuter = 2 * HX >= BX;
    auto tcol = [](int x) { return kOuter ? (x < HX ? x : x + BX) : x + HX; };
    const int zl = threadIdx.x % ZC;
    const int tx = threadIdx.x / ZC;
    const C2 *own = halo + (size_t)(tx + HX) * HYW * ZC + zl;
    C2 cen[kOuter ? 1 : BY];
    if constexpr (!kOuter) {
        // the column's own values (kappa term), before the x pass overwrites them
#pragma unroll
        for (int y = 0; y < BY; ++y) cen[y] = own[(size_t)(y + HY) * ZC];
        __syncthreads();
    }

    // x pass, one thread per halo row (hy, z): t(x, hy) = sum_sdx p_sdx
    // src(x - sdx, hy) for the patch's BX columns, written to columns
    // tcol(x) of the same row (no other thread touches that row)
    for (int item = threadIdx.x; item < HYW * ZC; item += NT) {
        const int hy = item / ZC, zr = item - hy * ZC;
        C2 *rowp = halo + (size_t)hy * ZC + zr;          // element hx at rowp[hx * HYW * ZC]
        C2 pv[WX], rv[HXW];
#pragma unroll
        for (int i = 0; i < WX; ++i) pv[i] = pw[i * ZC + zr];
#pragma unroll
        for (int i = 0; i < HXW; ++i) rv[i] = rowp[(size_t)i * HYW * ZC];
#pragma unroll
        for (int x = 0; x < BX; ++x) {
            R ar = 0, ai = 0;
#pragma unroll
            for (int sdx = -HX; sdx <= HX; ++sdx) {
                const C2 v = rv[x - sdx + HX];
                const C2 q = pv[sdx + HX];
                ar = fma(q.x, v.x, fma(-q.y, v.y, ar));
                ai = fma(q.x, v.y, fma(q.y, v.x, ai));
            }
            rowp[(size_t)tcol(x) * HYW * ZC] = mk2<R>(ar, ai);
        }
    }
    __syncthreads();

    // y pass, one thread per patch column (x, z): out(y) = in0 + sgn
    // [sum_sdy q_sdy t(x, y - sdy) - kappa src(x, y)]
    const int z = z0 + zl;
    bool any = false;       // a channel in this patch column (staged rows table)
#pragma unroll
    for (int y = 0; y < BY; ++y) any |= (y0 + y < nky) && rows[(tx + HX) * HYW + y + HY] >= 0;
    if (x0 + tx >= nkx || z >= n || !any) return;
    const C2 *tcolp = halo + (size_t)tcol(tx) * HYW * ZC + zl;
    R tr[HYW], ti[HYW];
#pragma unroll
    for (int i = 0; i < HYW; ++i) {
        const C2 v = tcolp[(size_t)i * ZC];
        tr[i] = v.x;
        ti[i] = v.y;
    }
    C2 qv[WY];
#pragma unroll
    for (int i = 0; i < WY; ++i) qv[i] = qw[i * ZC + zl];
    const C2 kap = kw[zl];
    int rowv[BY];
    C2 base[BY];
#pragma unroll
    for (int y = 0; y < BY; ++y)
        rowv[y] = (y0 + y < nky) ? rows[(tx + HX) * HYW + y + HY] : -1;
#pragma unroll
    for (int y = 0; y < BY; ++y)
        base[y] = (in0 && rowv[y] >= 0) ? in0[(size_t)rowv[y] * n + z] : mk2<R>(0, 0);
#pragma unroll
    for (int y = 0; y < BY; ++y) {
        if (rowv[y] < 0) continue;
        const C2 c = kOuter ? own[(size_t)(y + HY) * ZC] : cen[kOuter ? 0 : y];
        R ar = -(kap.x * c.x - kap.y * c.y), ai = -(kap.x * c.y + kap.y * c.x);
#pragma unroll
        for (int sdy = -HY; sdy <= HY; ++sdy) {
            const C2 q = qv[sdy + HY];
            const R xr = tr[y - sdy + HY], xi = ti[y - sdy + HY];
            ar = fma(q.x, xr, fma(-q.y, xi, ar));
            ai = fma(q.x, xi, fma(q.y, xr, ai));
        }
        out[(size_t)rowv[y] * n + z] = mk2<R>(base[y].x + sgn * ar, base[y].y + sgn * ai);
    }
}

// ---------------------------------------------------------------------------
// Arnoldi reductions.  partial[tile][i] = sum conj(Q_i) W over the tile for
// i < nvec; slot nvec holds ||W||^2 when with_norm.  One warp per vector;
// FP64 accumulation for both precisions.
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(256)
k_dots(Tiles tiles, const int *__restrict__ gate, int n, const typename CT<R>::t *__restrict__ Q,
       size_t qstride, int nvec, const typename CT<R>::t *__restrict__ W, int with_norm,
       double2 *__restrict__ partial, int pstride)
{
    using C2 = typename CT<R>::t;
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const size_t e0 = (size_t)tiles.row0[tile] * n;
    const int ne = tiles.nrow[tile] * n;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntask = nvec + (with_norm ? 1 : 0);
    for (int task = warp; task < ntask; task += (blockDim.x >> 5)) {
        double sr = 0.0, si = 0.0;
        if (task < nvec) {
            const C2 *q = Q + (size_t)task * qstride + e0;
            const C2 *w = W + e0;
            for (int e = lane; e < ne; e += 32) {
                const C2 a = q[e], b = w[e];
                sr = fma((double)a.x, (double)b.x, sr); sr = fma((double)a.y, (double)b.y, sr);
                si = fma((double)a.x, (double)b.y, si); si = fma(-(double)a.y, (double)b.x, si);
            }
        } else {
            const C2 *w = W + e0;
            for (int e = lane; e < ne; e += 32) {
                const C2 b = w[e];
                sr = fma((double)b.x, (double)b.x, sr); sr = fma((double)b.y, (double)b.y, sr);
            }
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) partial[(size_t)tile * pstride + task] = make_double2(sr, si);
    }
}

// out[s][i] = sum over the tiles of system s of partial[tile][i], i < nslot.
__global__ void __launch_bounds__(256)
k_reduce_partials(const int *__restrict__ sys_tile0, int nsys, const int *__restrict__ gate,
                  const double2 *__restrict__ partial, int pstride, int nslot,
                  double2 *__restrict__ out, int ostride)
{
    const int s = blockIdx.x;
    if (s >= nsys) return;
    if (gate && gate[s] == 0) return;
    const int t0 = sys_tile0[s], t1 = sys_tile0[s + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < nslot; i += (blockDim.x >> 5)) {
        double sr = 0.0, si = 0.0;
        for (int t = t0 + lane; t < t1; t += 32) {
            const double2 p = partial[(size_t)t * pstride + i];
            sr += p.x;
            si += p.y;
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) out[(size_t)s * ostride + i] = make_double2(sr, si);
    }
}

// dst = (W - sum_{i<nvec} Q_i coef[s][i]) * (scale ? scale[s] : 1)      (sum_only = 0)
// dst = sum_{i<nvec} Q_i coef[s][i]                                     (sum_only = 1)
// (dst may alias W).  coef and scale are FP64; the arithmetic is in R.
// Grid: (tiles, chunks); 256 threads.
template <typename R>
__global__ void __launch_bounds__(256)
k_update(Tiles tiles, const int *__restrict__ gate, int n, const typename CT<R>::t *__restrict__ Q,
         size_t qstride, int nvec, const int *__restrict__ nvec_sys,
         const double2 *__restrict__ coef, int cstride, const typename CT<R>::t *W,
         const double *__restrict__ scale, typename CT<R>::t *dst, int sum_only)
{
    using C2 = typename CT<R>::t;
    __shared__ C2 cf[kMaxRestart + 1];
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    int nv = nvec_sys ? nvec_sys[sys] : nvec;
    for (int i = threadIdx.x; i < nv; i += blockDim.x) {
        const double2 c = coef[(size_t)sys * cstride + i];
        cf[i] = mk2<R>((R)c.x, (R)c.y);
    }
    __syncthreads();
    const size_t e0 = (size_t)tiles.row0[tile] * n;
    const int ne = tiles.nrow[tile] * n;
    const R sc = scale ? (R)scale[sys] : R(1);
    const R sg = sum_only ? R(1) : R(-1);     // dst = sc (W - Q c)  or  sc (Q c)
    // Two consecutive elements per step: one 16-byte load per basis vector for
    // FP32 when every vector's chunk starts on an even element (chunk start
    // and vector stride even; otherwise an odd vector would be misaligned).
    const bool pairs = std::is_same<R, float>::value && (e0 % 2 == 0) && (qstride % 2 == 0);
    const int step = pairs ? 2 : 1;
    for (int e = (blockIdx.y * blockDim.x + threadIdx.x) * step; e < ne;
         e += gridDim.y * blockDim.x * step) {
        const bool two = pairs && e + 1 < ne;
        C2 a0 = mk2<R>(0, 0), a1 = mk2<R>(0, 0);
        if (W && !sum_only) {
            a0 = W[e0 + e];
            if (two) a1 = W[e0 + e + 1];
        }
        for (int i = 0; i < nv; ++i) {
            const C2 *qp = Q + (size_t)i * qstride + e0 + e;
            C2 q0, q1 = mk2<R>(0, 0);
            if (two) {
                const float4 v = *reinterpret_cast<const float4 *>(qp);
                q0 = mk2<R>((R)v.x, (R)v.y);
                q1 = mk2<R>((R)v.z, (R)v.w);
            } else {
                q0 = *qp;
            }
            const C2 c = cf[i];
            a0.x = fma(sg * q0.x, c.x, a0.x); a0.x = fma(-sg * q0.y, c.y, a0.x);
            a0.y = fma(sg * q0.x, c.y, a0.y); a0.y = fma(sg * q0.y, c.x, a0.y);
            a1.x = fma(sg * q1.x, c.x, a1.x); a1.x = fma(-sg * q1.y, c.y, a1.x);
            a1.y = fma(sg * q1.x, c.y, a1.y); a1.y = fma(sg * q1.y, c.x, a1.y);
        }
        dst[e0 + e] = mk2<R>(a0.x * sc, a0.y * sc);
        if (two) dst[e0 + e + 1] = mk2<R>(a1.x * sc, a1.y * sc);
    }
}

// Residual of the zero guess: out = b (b_spec e_n on the specular row, the
// boundary source of an adjoint solve otherwise).  Replaces the T GEMM and
// the FP64 coupling of the first refinement step when x = 0.
__global__ void __launch_bounds__(256)
k_rhs_residual(Tiles tiles, const int *__restrict__ gate, int n,
               const double2 *__restrict__ row_rhs, double2 *__restrict__ out)
{
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const int row0 = tiles.row0[tile];
    const size_t e0 = (size_t)row0 * n;
    const int ne = tiles.nrow[tile] * n;
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < ne; e += gridDim.y * blockDim.x) {
        const int r = e / n;
        const int z = e - r * n;
        out[e0 + e] = (z == n - 1) ? row_rhs[row0 + r] : make_double2(0.0, 0.0);
    }
}

// Mixed form: dst32 = src64 * scale[s]  (the normalised FP64 residual as the
// first FP32 Krylov vector).
__global__ void __launch_bounds__(256)
k_convert_scaled(Tiles tiles, const int *__restrict__ gate, int n, const double2 *__restrict__ src,
                 const double *__restrict__ scale, float2 *__restrict__ dst)
{
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const size_t e0 = (size_t)tiles.row0[tile] * n;
    const int ne = tiles.nrow[tile] * n;
    const double sc = scale[sys];
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < ne; e += gridDim.y * blockDim.x) {
        const double2 v = src[e0 + e];
        dst[e0 + e] = make_float2((float)(v.x * sc), (float)(v.y * sc));
    }
}

// Mixed form: x64 += u32 (the FP32 correction of one refinement step).
__global__ void __launch_bounds__(256)
k_accumulate_f32(Tiles tiles, const int *__restrict__ gate, int n, const float2 *__restrict__ u,
                 double2 *__restrict__ x)
{
    const int tile = blockIdx.x;
    const int sys = tiles.sys[tile];
    if (gate && gate[sys] == 0) return;
    const size_t e0 = (size_t)tiles.row0[tile] * n;
    const int ne = tiles.nrow[tile] * n;
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < ne; e += gridDim.y * blockDim.x) {
        const float2 d = u[e0 + e];
        double2 v = x[e0 + e];
        v.x += (double)d.x;
        v.y += (double)d.y;
        x[e0 + e] = v;
    }
}

// ---------------------------------------------------------------------------
// Per-system GMRES control (one thread per system; the work is O(m)).
// ---------------------------------------------------------------------------
struct GmresState {
    double2 *H;       // [B][(m+1)*m]  column j at j*(m+1)
    double2 *cs;      // [B][m]  Givens c (real stored in .x)
    double2 *sn;      // [B][m]  Givens s
    double2 *g;       // [B][m+1]
    double2 *h1;      // [B][m+2]  first-pass projections
    double2 *h2;      // [B][m+2]  second-pass projections (+ norm^2 slot)
    double2 *y;       // [B][m]
    double *scale;    // [B]  1/beta for the next basis vector
    double *bnorm;    // [B]  ||b||
    double *resid;    // [B]  last true relative residual
    double *est;      // [B]  GMRES residual estimate (absolute)
    double *beta0;    // [B]  residual norm at the start of the cycle
    int *active;      // [B]  iterating in this cycle
    int *kcyc;        // [B]  iterations done in this cycle
    int *iters;       // [B]  total iterations
    int *projv;       // [B]  basis vectors projected against, summed over steps (j + 1 at step j)
    int *cycles;      // [B]  restart cycles started
    int *unfinished;  // [B]  1 until converged or failed
    int *status;      // [B]  msc_status
    int *counter;     // [1]  systems still unfinished (host reads it)
};

// Cycle start: norm of r = b - A x from the reduced partials (slot 0).
__global__ void k_cycle_start(GmresState st, int nsys, int m, const double2 *__restrict__ nrm,
                              int nstride, double rtol, int max_iter, int max_cycles)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    st.active[s] = 0;
    st.kcyc[s] = 0;
    if (!st.unfinished[s]) return;
    const double nrm2 = nrm[(size_t)s * nstride].x;
    if (!isfinite(nrm2)) {              // (fmax would turn a NaN norm into 0)
        st.resid[s] = nrm2;
        st.unfinished[s] = 0;
        st.status[s] = 4;
        return;
    }
    const double beta = sqrt(fmax(nrm2, 0.0));
    if (beta == 0.0) {                  // exact (also: zero right-hand side)
        st.resid[s] = 0.0;
        st.unfinished[s] = 0;
        st.status[s] = 0;
        return;
    }
    const double rel = beta / st.bnorm[s];
    st.resid[s] = rel;
    if (!isfinite(beta)) {
        st.unfinished[s] = 0;
        st.status[s] = 4;
        return;
    }
    if (rel <= rtol) {
        st.unfinished[s] = 0;
        st.status[s] = 0;
        return;
    }
    if (st.iters[s] >= max_iter || (max_cycles > 0 && st.cycles[s] >= max_cycles)) {
        st.unfinished[s] = 0;
        st.status[s] = 2;
        return;
    }
    st.active[s] = 1;
    st.cycles[s] += 1;
    double2 *g = st.g + (size_t)s * (m + 1);
    g[0] = make_double2(beta, 0.0);
    for (int i = 1; i <= m; ++i) g[i] = make_double2(0.0, 0.0);
    st.scale[s] = 1.0 / beta;
    st.beta0[s] = beta;
    atomicAdd(st.counter, 1);
}

// Arnoldi step j: combine the two CGS passes, append column j of H, apply
// the previous Givens rotations, make rotation j, update g.  A system stops
// iterating in this cycle when its residual estimate reaches
// max(rtol ||b||, inner_rtol beta0) (inner_rtol > 0 only for the mixed
// form, whose FP32 inner solve cannot go below its own rounding level).
__device__ void arnoldi_givens(GmresState &st, int s, int m, int j, double rtol, int max_iter,
                               double inner_rtol, bool use_h1 = true)
{
    // use_h1 = false: one Gram-Schmidt pass (h2 holds the projections and
    // h2[j+1] the squared norm of w before projection; beta by Pythagoras).
    if (!st.active[s]) return;
    const int hs = m + 2;
    const double2 *h1 = st.h1 + (size_t)s * hs;
    const double2 *h2 = st.h2 + (size_t)s * hs;
    double2 *H = st.H + (size_t)s * (m + 1) * m + (size_t)j * (m + 1);
    double2 *cs = st.cs + (size_t)s * m;
    double2 *sn = st.sn + (size_t)s * m;
    double2 *g = st.g + (size_t)s * (m + 1);
    double proj2 = 0.0;
    for (int i = 0; i <= j; ++i) {
        H[i] = use_h1 ? cadd(h1[i], h2[i]) : h2[i];
        proj2 += cabs2(h2[i]);
    }
    const double w2 = h2[j + 1].x;          // ||W'||^2 after the first pass
    const double beta = sqrt(fmax(w2 - proj2, 0.0));
    for (int i = 0; i < j; ++i) {
        const double c = cs[i].x;
        const double2 sv = sn[i];
        const double2 a = H[i], b = H[i + 1];
        // [c, s; -conj(s), c] [a; b]
        H[i] = cadd(cscale(a, c), cmul(sv, b));
        H[i + 1] = csub(cscale(b, c), cmul(cconj(sv), a));
    }
    const double2 a = H[j];
    const double aa = sqrt(cabs2(a));
    const double r = hypot(aa, beta);
    double c;
    double2 sv;
    if (r == 0.0) {
        c = 1.0;
        sv = make_double2(0.0, 0.0);
    } else if (aa == 0.0) {
        c = 0.0;
        sv = make_double2(1.0, 0.0);
    } else {
        c = aa / r;
        sv = cscale(cscale(a, 1.0 / aa), beta / r);   // (a/|a|) * beta / r, beta real
    }
    cs[j] = make_double2(c, 0.0);
    sn[j] = sv;
    H[j] = (aa == 0.0) ? make_double2(beta, 0.0) : cscale(a, r / aa);
    H[j + 1] = make_double2(0.0, 0.0);
    const double2 gj = g[j];
    g[j] = cscale(gj, c);
    g[j + 1] = make_double2(-(sv.x * gj.x + sv.y * gj.y), -(sv.x * gj.y - sv.y * gj.x));  // -conj(s) g_j
    const double est = sqrt(cabs2(g[j + 1]));
    st.est[s] = est;
    st.kcyc[s] = j + 1;
    st.iters[s] += 1;
    st.projv[s] += j + 1;
    st.scale[s] = (beta > 0.0) ? 1.0 / beta : 0.0;
    bool stop = false;
    if (!isfinite(est) || !isfinite(beta)) stop = true;
    if (est <= fmax(rtol * st.bnorm[s], inner_rtol * st.beta0[s])) stop = true;
    if (j + 1 >= m) stop = true;
    if (st.iters[s] >= max_iter) stop = true;
    if (beta <= 1e-300) stop = true;
    if (stop) st.active[s] = 0;
}

// y = R^-1 g over the kcyc columns of this cycle.
__global__ void k_trisolve(GmresState st, int nsys, int m)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsys) return;
    const int k = st.kcyc[s];
    if (k == 0) return;
    const double2 *H = st.H + (size_t)s * (m + 1) * m;
    const double2 *g = st.g + (size_t)s * (m + 1);
    double2 *y = st.y + (size_t)s * m;
    for (int i = k - 1; i >= 0; --i) {
        double2 acc = g[i];
        for (int l = i + 1; l < k; ++l) acc = csub(acc, cmul(H[(size_t)l * (m + 1) + i], y[l]));
        y[i] = cdiv(acc, H[(size_t)i * (m + 1) + i]);
    }
}

// ---------------------------------------------------------------------------
// Fused Arnoldi step (CGS2), three launches per step:
//   P1  h1 = Q^H w                                  (partials + last-block reduce)
//   P2  w <- w - Q h1 ; h2 = Q^H w ; |w|^2 ; Givens  (partials + last-block reduce)
//   P3  q_{j+1} = (w - Q h2) / beta                  (k_update)
// Each block handles 1/split of a row tile; the block that finishes last for
// a system (per-system arrival counter) sums that system's partials in a
// fixed order, so results do not depend on scheduling.
// ---------------------------------------------------------------------------
struct ArnoldiArgs {
    Tiles tiles;
    const int *sys_tile0;   // [B + 1] first tile of each system
    const int *gate;        // [B] active flags
    int n;
    int split;              // blocks per tile
    size_t qstride;         // elements between basis vectors
    double2 *partial;       // [ntiles * split][pstride]
    int pstride;
    int *counter;           // [B] arrival counters (left at 0)
};

template <typename R>
__device__ __forceinline__ void elem_range(const ArnoldiArgs &a, int tile, int sub, size_t &e0, int &ne)
{
    const int tot = a.tiles.nrow[tile] * a.n;
    const int per = (tot + a.split - 1) / a.split;
    const int lo = min(tot, sub * per);
    e0 = (size_t)a.tiles.row0[tile] * a.n + lo;
    ne = min(tot, lo + per) - lo;
}

// Last-arriving block of system s sums the system's partials into dst[0..nslot).
__device__ __forceinline__ bool last_block_reduce(const ArnoldiArgs &a, int s, int nslot, double2 *dst)
{
    __shared__ int is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nblocks = (a.sys_tile0[s + 1] - a.sys_tile0[s]) * a.split;
        const int prev = atomicAdd(&a.counter[s], 1);
        is_last = (prev == nblocks - 1);
        if (is_last) a.counter[s] = 0;
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    const int b0 = a.sys_tile0[s] * a.split, b1 = a.sys_tile0[s + 1] * a.split;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < nslot; i += (blockDim.x >> 5)) {
        double sr = 0.0, si = 0.0;
        for (int b = b0 + lane; b < b1; b += 32) {
            const double2 v = __ldcg(a.partial + (size_t)b * a.pstride + i);
            sr += v.x;
            si += v.y;
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) dst[i] = make_double2(sr, si);
    }
    __syncthreads();
    return true;
}

// P1: h1 = Q^H w.  Warps take (basis vector, sub-range) tasks: each vector's
// slice of the block's row chunk is cut into S sub-ranges, S in {1, 2, 4, 8}
// chosen so that the 8 warps get the most even share (9 vectors on 8 warps
// would otherwise leave 7 warps idle while one reads a second vector).  A
// warp streams its sub-range of the vector and of w (w re-read from L1 by
// the other warps) with U loads in flight per thread, two FP64 accumulators
// per thread, then a warp sum; the sub-range sums add up in a fixed order
// (deterministic) before the per-system last-block reduction.  Few registers
// per thread, so the SM holds enough warps to keep DRAM busy.
template <typename R> struct P1Unroll { static constexpr int value = 8; };
template <> struct P1Unroll<double> { static constexpr int value = 4; };

template <typename R>
__global__ void __launch_bounds__(256)
k_arnoldi_p1(ArnoldiArgs a, const typename CT<R>::t *__restrict__ Q, int nvec,
             const typename CT<R>::t *__restrict__ W, double2 *__restrict__ h1, int hstride)
{
    using C2 = typename CT<R>::t;
    constexpr int U = P1Unroll<R>::value;
    constexpr int kSub = 8;
    __shared__ double2 red[kMaxRestart + 1][kSub];
    const int tile = blockIdx.x / a.split, sub0 = blockIdx.x - tile * a.split;
    const int s = a.tiles.sys[tile];
    if (a.gate && a.gate[s] == 0) return;
    size_t e0;
    int ne;
    elem_range<R>(a, tile, sub0, e0, ne);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    // S minimises the busiest warp's work, ceil(nvec S / nw) / S vector
    // passes, among the splits that leave every sub-range at least one full
    // unrolled warp pass (32 U elements; small chunks keep S = 1)
    int S = 1;
    {
        int best = (nvec + nw - 1) / nw * kSub;
        for (int c = 2; c <= kSub && ne >= c * 32 * U; c *= 2) {
            const int cost = (nvec * c + nw - 1) / nw * (kSub / c);
            if (cost < best) {
                best = cost;
                S = c;
            }
        }
    }
    const int per = (ne + S - 1) / S;
    const C2 *w = W + e0;
    for (int t = warp; t < nvec * S; t += nw) {
        const int i = t / S, sub = t - i * S;
        const int lo = min(ne, sub * per), hi = min(ne, lo + per);
        const C2 *q = Q + (size_t)i * a.qstride + e0;
        double sr = 0.0, si = 0.0;
        for (int base = lo + lane; base < hi; base += 32 * U) {
            C2 qv[U], wv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = base + u * 32;
                qv[u] = (e < hi) ? q[e] : mk2<R>(0, 0);
                wv[u] = (e < hi) ? w[e] : mk2<R>(0, 0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const double qx = (double)qv[u].x, qy = (double)qv[u].y;
                const double wx = (double)wv[u].x, wy = (double)wv[u].y;
                sr = fma(qx, wx, fma(qy, wy, sr));
                si = fma(qx, wy, fma(-qy, wx, si));
            }
        }
        sr = warp_sum(sr);
        si = warp_sum(si);
        if (lane == 0) red[i][sub] = make_double2(sr, si);
    }
    __syncthreads();
    double2 *out = a.partial + (size_t)blockIdx.x * a.pstride;
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
        double2 acc = red[i][0];
        for (int sub = 1; sub < S; ++sub) {
            acc.x += red[i][sub].x;
            acc.y += red[i][sub].y;
        }
        out[i] = acc;
    }
    last_block_reduce(a, s, nvec, h1 + (size_t)s * hstride);
}

__device__ void arnoldi_givens(GmresState &st, int s, int m, int j, double rtol, int max_iter,
                               double inner_rtol);

// P2: w <- w - Q h1 ; h2 = Q^H w, |w|^2 ; then the Givens step of the system.
// With cgs2 = 0 (single Gram-Schmidt pass) there is no h1 and no update:
// h2 = Q^H w and |w|^2 come from the unprojected w and the Givens step takes
// beta^2 = |w|^2 - |h2|^2.
template <typename R>
__global__ void __launch_bounds__(256)
k_arnoldi_p2(ArnoldiArgs a, const typename CT<R>::t *__restrict__ Q, int nvec,
             typename CT<R>::t *__restrict__ W, GmresState st, int m, int j, double rtol,
             int max_iter, double inner_rtol, int cgs2)
{
    using C2 = typename CT<R>::t;
    __shared__ C2 cf[kMaxRestart + 1];
    const int tile = blockIdx.x / a.split, sub = blockIdx.x - tile * a.split;
    const int s = a.tiles.sys[tile];
    if (a.gate && a.gate[s] == 0) return;
    const int hs = m + 2;
    size_t e0;
    int ne;
    elem_range<R>(a, tile, sub, e0, ne);
    if (cgs2) {
    for (int i = threadIdx.x; i < nvec; i += blockDim.x) {
        const double2 c = st.h1[(size_t)s * hs + i];
        cf[i] = mk2<R>((R)c.x, (R)c.y);
    }
    __syncthreads();
    // w <- w - Q h1, two consecutive elements per step (one 16-byte load per
    // basis vector for FP32 when the range start and the vector stride are
    // even, so that every vector's range is 16-byte aligned)
    const bool pairs = std::is_same<R, float>::value && (e0 % 2 == 0) && (a.qstride % 2 == 0);
    const int step = pairs ? 2 : 1;
    for (int e = threadIdx.x * step; e < ne; e += blockDim.x * step) {
        const bool two = pairs && e + 1 < ne;
        C2 w0 = W[e0 + e], w1 = two ? W[e0 + e + 1] : mk2<R>(0, 0);
        for (int i = 0; i < nvec; ++i) {
            const C2 *qp = Q + (size_t)i * a.qstride + e0 + e;
            C2 q0, q1 = mk2<R>(0, 0);
            if (two) {
                const float4 v = *reinterpret_cast<const float4 *>(qp);
                q0 = mk2<R>((R)v.x, (R)v.y);
                q1 = mk2<R>((R)v.z, (R)v.w);
            } else {
                q0 = *qp;
            }
            const C2 c = cf[i];
            w0.x = fma(-q0.x, c.x, fma(q0.y, c.y, w0.x));
            w0.y = fma(-q0.x, c.y, fma(-q0.y, c.x, w0.y));
            w1.x = fma(-q1.x, c.x, fma(q1.y, c.y, w1.x));
            w1.y = fma(-q1.x, c.y, fma(-q1.y, c.x, w1.y));
        }
        W[e0 + e] = w0;
        if (two) W[e0 + e + 1] = w1;
    }
    __syncthreads();            // the block's updated w is visible to all its warps
    }   // cgs2
    // Second projection and |w|^2: one warp per basis vector (the last task is
    // the norm), reading w and Q back from L1/L2.
    {
        constexpr int U = 4;
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
        double2 *out = a.partial + (size_t)blockIdx.x * a.pstride;
        const C2 *w = W + e0;
        for (int task = warp; task <= nvec; task += nw) {
            const C2 *q = Q + (size_t)min(task, nvec - 1) * a.qstride + e0;
            const bool norm = task == nvec;
            double sr = 0.0, si = 0.0;
            for (int base = lane; base < ne; base += 32 * U) {
                C2 qv[U], wv[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = base + u * 32;
                    wv[u] = (e < ne) ? w[e] : mk2<R>(0, 0);
                    qv[u] = (e < ne && !norm) ? q[e] : mk2<R>(0, 0);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const double wx = (double)wv[u].x, wy = (double)wv[u].y;
                    if (norm) {
                        sr = fma(wx, wx, fma(wy, wy, sr));
                    } else {
                        const double qx = (double)qv[u].x, qy = (double)qv[u].y;
                        sr = fma(qx, wx, fma(qy, wy, sr));
                        si = fma(qx, wy, fma(-qy, wx, si));
                    }
                }
            }
            sr = warp_sum(sr);
            si = warp_sum(si);
            if (lane == 0) out[task] = make_double2(sr, norm ? 0.0 : si);
        }
    }
    if (last_block_reduce(a, s, nvec + 1, st.h2 + (size_t)s * hs)) {
        if (threadIdx.x == 0) arnoldi_givens(st, s, m, j, rtol, max_iter, inner_rtol, cgs2 != 0);
    }
}

// ---------------------------------------------------------------------------
// Arnoldi step with delayed re-orthogonalisation (DCGS2): two passes over the
// basis per step instead of the three of CGS2.  Gram-Schmidt with the
// second projection of q_j delayed to step j + 1 (Bielich, Langou, Thomas,
// Swirydowicz, Yamazaki, Boman, "Low-synch Gram-Schmidt with delayed
// reorthogonalization for Krylov solvers", Parallel Computing 112, 2022).
//
// At step j the basis slots hold q_0 .. q_{j-1} (final) and, in slot j, the
// candidate v: the next vector projected once and not normalised; w = A M v.
//   reduction  s = Q_{j-1}^H v, t = Q_{j-1}^H w, ||v||^2, v^H w
//              nu = sqrt(||v||^2 - ||s||^2)   (q_j = (v - Q_{j-1} s) / nu)
//              column j-1 of H is final: H[:j, j-1] += s, H[j, j-1] = nu
//              Hs = Hbar s (unrotated Hessenberg, A M Q_{j-1} = Q_j Hbar)
//              h_j[:j] = (t - Hs[:j]) / nu
//              h_j[j]  = ((v^H w - s^H t) / nu - Hs[j]) / nu
//   update     q_j     = v / nu - Q_{j-1} s / nu
//              v_{j+1} = w / nu - (d / nu) v - Q_{j-1} (c - s d / nu),
//              e = Hs / nu + h_j, c = e[:j], d = e[j]
//              ||v_{j+1}||^2 -> provisional column j (H[j+1, j] = ||v_{j+1}||),
//              its Givens rotation and the GMRES residual estimate.
// The provisional column is made final (and its rotation redone) by the next
// step's reduction, so the stop test runs on the step it belongs to: a
// system that stops at step j never pays for the matvec of step j + 1.  The
// column a cycle ends on stays provisional: its only difference from the
// final one is the second projection of v_{j+1}, the loss-of-orthogonality
// level that the FP64 true residual of the next cycle absorbs.
// ---------------------------------------------------------------------------
struct DcgsState {
    double2 *Hraw;    // [B][(m+1)*m]  unrotated Hessenberg (column j at j*(m+1))
    double2 *dsum;    // [B][2(m+1)]   per-system reduction results of the step
    double2 *coef;    // [B][cstride]  update coefficients (see dcgs_coefficients_p)
    double2 *gsave;   // [B]           g[j] before the provisional rotation j
    int cstride;      // 2 m + 4
};

// Column j of H from its unrotated entries: apply rotations 0..j-1, make
// rotation j from (H[j], H[j+1]) and update g (g[j] is taken from gj, the
// value saved before the provisional rotation j; g[j+1] starts at 0).
// Returns the new residual estimate |g[j+1]|.  The arrays are one system's
// (raw: its unrotated column j; H: its column j; cs, sn, g), in global or
// shared memory.
__device__ double dcgs_rotate_column_p(const double2 *raw, double2 *H, double2 *cs, double2 *sn,
                                       double2 *g, double2 gj, int j)
{
    for (int i = 0; i <= j + 1; ++i) H[i] = raw[i];
    for (int i = 0; i < j; ++i) {
        const double c = cs[i].x;
        const double2 sv = sn[i];
        const double2 a = H[i], b = H[i + 1];
        H[i] = cadd(cscale(a, c), cmul(sv, b));
        H[i + 1] = csub(cscale(b, c), cmul(cconj(sv), a));
    }
    const double2 a = H[j];
    const double beta = H[j + 1].x;            // real, >= 0 (a norm)
    const double aa = sqrt(cabs2(a));
    const double r = hypot(aa, beta);
    double c;
    double2 sv;
    if (r == 0.0) {
        c = 1.0;
        sv = make_double2(0.0, 0.0);
    } else if (aa == 0.0) {
        c = 0.0;
        sv = make_double2(1.0, 0.0);
    } else {
        c = aa / r;
        sv = cscale(cscale(a, 1.0 / aa), beta / r);
    }
    cs[j] = make_double2(c, 0.0);
    sn[j] = sv;
    H[j] = (aa == 0.0) ? make_double2(beta, 0.0) : cscale(a, r / aa);
    H[j + 1] = make_double2(0.0, 0.0);
    g[j] = cscale(gj, c);
    g[j + 1] = make_double2(-(sv.x * gj.x + sv.y * gj.y), -(sv.x * gj.y - sv.y * gj.x));
    return sqrt(cabs2(g[j + 1]));
}

__device__ __forceinline__ double dcgs_rotate_column(GmresState &st, const DcgsState &ds, int s, int m, int j)
{
    return dcgs_rotate_column_p(ds.Hraw + (size_t)s * (m + 1) * m + (size_t)j * (m + 1),
                                st.H + (size_t)s * (m + 1) * m + (size_t)j * (m + 1),
                                st.cs + (size_t)s * m, st.sn + (size_t)s * m,
                                st.g + (size_t)s * (m + 1), ds.gsave[s], j);
}

__device__ __forceinline__ bool dcgs_stop(const GmresState &st, int s, double est, double rtol,
                                          double inner_rtol)
{
    return !isfinite(est) || est <= fmax(rtol * st.bnorm[s], inner_rtol * st.beta0[s]);
}

// Per-system scalar work of the reduction (one thread): finalise column j-1,
// redo its rotation, form h_j and the update coefficients:
//   coef[0..j)        a_i = -s_i / nu            (q_j = v / nu + sum a_i Q_i)
//   coef[j+1 .. 2j+1) b_i = -(c_i - s_i d / nu)  (v_{j+1} = w / nu - (d / nu) v + sum b_i Q_i)
//   coef[2m+2] = (1 / nu, 0), coef[2m+3] = -d / nu
// on one system's arrays (global or shared memory): raw = its unrotated
// Hessenberg columns, sum = its reduction results, Hj1 = its column j - 1 of
// H, hs = scratch of j + 1 entries.  Returns 1 when the system stops
// (converged, or no new direction), with *est set when j > 0.
__device__ int dcgs_coefficients_p(double2 *raw, const double2 *sum, double2 *Hj1, double2 *cs,
                                   double2 *sn, double2 *g, double2 gsave, double2 *cf, double2 *hs,
                                   int m, int j, double bnorm, double beta0, double rtol,
                                   double inner_rtol, double *est)
{
    const double2 *sv = sum;               // s_i = q_i^H v, i < j;  sum[j] = ||v||^2
    const double2 *tv = sum + (j + 1);     // t_i = q_i^H w, i < j;  tv[j] = v^H w
    double ss = 0.0;
    for (int i = 0; i < j; ++i) ss += cabs2(sv[i]);
    const double nu2 = sum[j].x - ss;
    const double nu = sqrt(fmax(nu2, 0.0));
    if (j == 0) {
        // v = q_0 up to rounding; g[0] = beta follows q_0 = v / nu
        g[0] = cscale(g[0], nu);
    } else {
        double2 *col = raw + (size_t)(j - 1) * (m + 1);
        for (int i = 0; i < j; ++i) col[i] = cadd(col[i], sv[i]);
        col[j] = make_double2(nu, 0.0);
        *est = dcgs_rotate_column_p(col, Hj1, cs, sn, g, gsave, j - 1);
        if (!isfinite(*est) || *est <= fmax(rtol * bnorm, inner_rtol * beta0))
            return 1;                      // q_0 .. q_{j-1} are final; kcyc = j
    }
    if (!(nu > 1e-300) || !isfinite(nu)) return 1;
    const double inu = 1.0 / nu;
    // Hs = Hbar[:j+1, :j] s (column k has entries 0..k+1)
    for (int i = 0; i <= j; ++i) hs[i] = make_double2(0.0, 0.0);
    for (int k = 0; k < j; ++k) {
        const double2 *colk = raw + (size_t)k * (m + 1);
        for (int i = 0; i <= k + 1; ++i) hs[i] = cadd(hs[i], cmul(colk[i], sv[k]));
    }
    double2 sht = make_double2(0.0, 0.0);   // s^H t
    for (int i = 0; i < j; ++i) sht = cadd(sht, cmul(cconj(sv[i]), tv[i]));
    double2 *colj = raw + (size_t)j * (m + 1);
    for (int i = 0; i < j; ++i) colj[i] = cscale(csub(tv[i], hs[i]), inu);
    colj[j] = cscale(csub(cscale(csub(tv[j], sht), inu), hs[j]), inu);
    const double2 d = cadd(cscale(hs[j], inu), colj[j]);
    const double2 dn = cscale(d, inu);
    for (int i = 0; i < j; ++i) {
        const double2 ci = cadd(cscale(hs[i], inu), colj[i]);
        cf[i] = cscale(sv[i], -inu);
        cf[j + 1 + i] = make_double2(-(ci.x - (sv[i].x * dn.x - sv[i].y * dn.y)),
                                     -(ci.y - (sv[i].x * dn.y + sv[i].y * dn.x)));
    }
    cf[2 * m + 2] = make_double2(inu, 0.0);
    cf[2 * m + 3] = make_double2(-dn.x, -dn.y);
    return 0;
}

// Double2 entries of the shared scratch dcgs_coefficients_block needs.
__host__ __device__ constexpr int dcgs_block_scratch(int m)
{
    return (m + 1) * (m + 1) + 5 * (m + 1) + 4 * m + 4;
}

// dcgs_coefficients_p for the last block of a system: the whole block copies
// the system's Hessenberg columns 0..j, reduction results, rotations and g
// into shared memory (one round of parallel loads), thread 0 runs the
// serial algebra there, and the block writes back what changed.  The
// serial part then waits on shared memory instead of an L2 round trip per
// element (the tail of the reduction kernel).  sc: dcgs_block_scratch(m)
// entries of shared memory.
__device__ void dcgs_coefficients_block(GmresState &st, const DcgsState &ds, int s, int m, int j,
                                        double rtol, double inner_rtol, double2 *sc)
{
    const int M1 = m + 1, ncol = j + 1;
    double2 *raw = sc;                           // [ncol][M1] unrotated columns 0..j
    double2 *sum = raw + (size_t)ncol * M1;      // [2 M1]
    double2 *cs = sum + 2 * M1;                  // [m]
    double2 *sn = cs + m;                        // [m]
    double2 *g = sn + m;                         // [M1]
    double2 *Hj1 = g + M1;                       // [M1] column j - 1 of H
    double2 *cf = Hj1 + M1;                      // [2 m + 4]
    double2 *hs = cf + 2 * m + 4;                // [M1]
    __shared__ int res;
    const size_t hb = (size_t)s * M1 * m;
    const int nt = blockDim.x;
    for (int i = threadIdx.x; i < ncol * M1; i += nt) raw[i] = ds.Hraw[hb + i];
    for (int i = threadIdx.x; i < 2 * M1; i += nt) sum[i] = ds.dsum[(size_t)s * 2 * M1 + i];
    for (int i = threadIdx.x; i < m; i += nt) {
        cs[i] = st.cs[(size_t)s * m + i];
        sn[i] = st.sn[(size_t)s * m + i];
    }
    for (int i = threadIdx.x; i < M1; i += nt) g[i] = st.g[(size_t)s * M1 + i];
    __syncthreads();
    if (threadIdx.x == 0) {
        double est = 0.0;
        res = dcgs_coefficients_p(raw, sum, Hj1, cs, sn, g, ds.gsave[s], cf, hs, m, j, st.bnorm[s],
                                  st.beta0[s], rtol, inner_rtol, &est);
        if (j > 0) st.est[s] = est;
        if (res) st.active[s] = 0;
    }
    __syncthreads();
    if (j == 0) {
        if (threadIdx.x == 0) st.g[(size_t)s * M1] = g[0];
    } else {
        // column j - 1: its final entries 0..j, its rotated form, rotation j - 1, g
        for (int i = threadIdx.x; i <= j; i += nt) {
            ds.Hraw[hb + (size_t)(j - 1) * M1 + i] = raw[(size_t)(j - 1) * M1 + i];
            st.H[hb + (size_t)(j - 1) * M1 + i] = Hj1[i];
        }
        if (threadIdx.x == 0) {
            st.cs[(size_t)s * m + j - 1] = cs[j - 1];
            st.sn[(size_t)s * m + j - 1] = sn[j - 1];
            st.g[(size_t)s * M1 + j - 1] = g[j - 1];
            st.g[(size_t)s * M1 + j] = g[j];
        }
    }
    if (res == 0) {
        double2 *cfg = ds.coef + (size_t)s * ds.cstride;
        for (int i = threadIdx.x; i <= j; i += nt) ds.Hraw[hb + (size_t)j * M1 + i] = raw[(size_t)j * M1 + i];
        for (int i = threadIdx.x; i < j; i += nt) {
            cfg[i] = cf[i];
            cfg[j + 1 + i] = cf[j + 1 + i];
        }
        if (threadIdx.x == 0) {
            cfg[2 * m + 2] = cf[2 * m + 2];
            cfg[2 * m + 3] = cf[2 * m + 3];
        }
    }
}

template <typename R> struct DcgsUnroll { static constexpr int value = 8; };
template <> struct DcgsUnroll<double> { static constexpr int value = 4; };

// Reduction pass of step j over row chunks.  Each warp takes sub-ranges of
// 32 U elements of the block's chunk, holds v and w there in registers and
// streams q_0 .. q_{j-1} and v itself (the basis slots 0 .. j), two dots per
// vector (q_i^H v, q_i^H w), reduced across the warp per vector and added in
// a fixed order (deterministic).  The last block of a system reduces the
// per-block partials and runs dcgs_coefficients_block.
// Precision: a lane's products and its partial sum of U terms are formed in
// the vectors' own type (FP32 for the inner solve of the mixed form: FP64
// products there made the FP64 pipe, not memory, the limit), the sums across
// lanes, warps and blocks in FP64.  The FP32 partials err by ~U ulp of the
// terms, the level of the FP32 basis itself; the quantities DCGS2 forms from
// them do not cancel: s = Q^H v is the small second-pass correction of an
// already projected v (nu^2 = ||v||^2 - ||s||^2 keeps ||v||^2), and the
// first-pass error of t = Q^H w is what the next step's s removes.
template <typename R>
__global__ void __launch_bounds__(256, 2)
k_dcgs_reduce(ArnoldiArgs a, const typename CT<R>::t *__restrict__ Q, int j,
              const typename CT<R>::t *__restrict__ W, GmresState st, DcgsState ds, int m,
              double rtol, double inner_rtol)
{
    using C2 = typename CT<R>::t;
    constexpr int U = DcgsUnroll<R>::value;
    constexpr int NW = 8;
    __shared__ double2 red[2 * (kMaxRestart + 1)][NW];
    const int blk = blockIdx.x;
    const int s = a.tiles.sys[blk];
    if (a.gate && a.gate[s] == 0) return;
    size_t e0;
    int ne;
    elem_range<R>(a, blk, 0, e0, ne);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nv = j + 1;                        // basis slots 0..j (slot j holds v)
    for (int i = threadIdx.x; i < 2 * nv * NW; i += blockDim.x)
        red[i / NW][i % NW] = make_double2(0.0, 0.0);
    __syncthreads();
    const C2 *vp = Q + (size_t)j * a.qstride + e0;
    const C2 *wp = W + e0;
    for (int base = warp * 32 * U; base < ne; base += NW * 32 * U) {
        C2 vv[U], ww[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = base + u * 32 + lane;
            vv[u] = (e < ne) ? vp[e] : mk2<R>(0, 0);
            ww[u] = (e < ne) ? wp[e] : mk2<R>(0, 0);
        }
        // q_i is loaded one vector ahead, so its loads are in flight while
        // the previous vector's products and warp sums run
        C2 qn[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = base + u * 32 + lane;
            qn[u] = (e < ne) ? Q[e0 + e] : mk2<R>(0, 0);
        }
        for (int i = 0; i < nv; ++i) {
            C2 qv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) qv[u] = qn[u];
            if (i + 1 < nv) {
                const C2 *q = Q + (size_t)(i + 1) * a.qstride + e0;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int e = base + u * 32 + lane;
                    qn[u] = (e < ne) ? q[e] : mk2<R>(0, 0);
                }
            }
            // products and the lane's partial sum of U terms in the vectors'
            // own precision, the sums across lanes, warps and blocks in FP64
            R ar = 0, ai = 0, br = 0, bi = 0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const R qx = qv[u].x, qy = qv[u].y;
                ar = fma(qx, vv[u].x, fma(qy, vv[u].y, ar));
                ai = fma(qx, vv[u].y, fma(-qy, vv[u].x, ai));
                br = fma(qx, ww[u].x, fma(qy, ww[u].y, br));
                bi = fma(qx, ww[u].y, fma(-qy, ww[u].x, bi));
            }
            const double sar = warp_sum((double)ar), sai = warp_sum((double)ai);
            const double sbr = warp_sum((double)br), sbi = warp_sum((double)bi);
            if (lane == 0) {
                double2 &x = red[i][warp];
                double2 &y = red[nv + i][warp];
                x.x += sar; x.y += sai;
                y.x += sbr; y.y += sbi;
            }
        }
    }
    __syncthreads();
    double2 *out = a.partial + (size_t)blk * a.pstride;
    for (int i = threadIdx.x; i < 2 * nv; i += blockDim.x) {
        double2 acc = red[i][0];
        for (int w = 1; w < NW; ++w) {
            acc.x += red[i][w].x;
            acc.y += red[i][w].y;
        }
        out[i] = acc;
    }
    if (last_block_reduce(a, s, 2 * nv, ds.dsum + (size_t)s * 2 * (m + 1))) {
        extern __shared__ __align__(16) unsigned char dcgs_scratch[];   // dcgs_block_scratch(m) entries
        dcgs_coefficients_block(st, ds, s, m, j, rtol, inner_rtol, reinterpret_cast<double2 *>(dcgs_scratch));
    }
}

// Reduction pass of step j with the basis streamed through shared memory
// (FP32 Krylov vectors).  The block's chunk of each vector is one contiguous
// range, so it arrives by a single cp.async.bulk into a ring of kBulkStages
// stages, each completing on its own mbarrier: up to kBulkStages vectors are
// in flight while one is reduced (the register form above keeps one).  The
// stream is v, w, q_0 .. q_{j-1}: v and w land in registers (thread t holds
// element pairs t, t + 256, ...), slot j (v itself) is reduced from them,
// so v is read once and no thread waits on a global load.  Two blocks per
// SM (3 stages of 32 KB each and 128 registers); one block with 6 stages was
// slower (239 against 186 us per launch on the 512-beam cfg2 batch: 8 warps
// cannot keep up the FP32 work).  Sums and their fixed order across warps
// are those of k_dcgs_reduce; the last block of a system runs
// dcgs_coefficients_block with the ring as its scratch.  Needs chunks of at
// most kBulkChunk elements, an even count, starting on an even element
// (16-byte aligned copies).  A wait that times out sets *err; the block then
// stops reducing, waits (bounded) for its copies in flight and still takes
// part in the per-system arrival count.
constexpr int kBulkChunk = 4096;
constexpr int kBulkStages = 3;

__host__ __device__ constexpr size_t dcgs_bulk_smem() { return (size_t)kBulkStages * kBulkChunk * 8; }
// the last block's scalar work reuses the ring as its scratch
static_assert((size_t)dcgs_block_scratch(kMaxRestart) * sizeof(double2) <= dcgs_bulk_smem(),
              "the DCGS2 scalar scratch must fit in the streaming ring");

__global__ void __launch_bounds__(256, 2)
k_dcgs_reduce_bulk(ArnoldiArgs a, const float2 *__restrict__ Q, int j, const float2 *__restrict__ W,
                   GmresState st, DcgsState ds, int m, double rtol, double inner_rtol, int *err)
{
    constexpr int NW = 8, NT = 256;
    constexpr int UP = kBulkChunk / (2 * NT);          // element pairs per thread
    constexpr int SP = kBulkChunk / 2;                 // float4 per stage
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4 *ring = reinterpret_cast<float4 *>(smem_raw);
    __shared__ __align__(8) uint64_t full[kBulkStages];
    __shared__ double2 red[2 * (kMaxRestart + 1)][NW];
    const int blk = blockIdx.x;
    const int s = a.tiles.sys[blk];
    if (a.gate && a.gate[s] == 0) return;
    size_t e0;
    int ne;
    elem_range<float>(a, blk, 0, e0, ne);
    const int np = ne >> 1;
    const uint32_t bytes = (uint32_t)ne * 8u;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nv = j + 1;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kBulkStages; ++q) mbar_init(&full[q], 1);
        mbar_fence_init();
    }
    for (int i = threadIdx.x; i < 2 * nv * NW; i += NT) red[i / NW][i % NW] = make_double2(0.0, 0.0);
    __syncthreads();
    // the stream: item 0 = v (slot j), item 1 = w, item 2 + i = q_i; v and
    // w come through the ring too, so no thread waits on a global load
    const int NI = j + 2;
    auto src_of = [&](int it) {
        return it == 0 ? Q + (size_t)j * a.qstride + e0
             : it == 1 ? W + e0 : Q + (size_t)(it - 2) * a.qstride + e0;
    };
    int issued = 0;                                    // thread 0: items whose copy was issued
    if (threadIdx.x == 0) {
        for (; issued < min(kBulkStages, NI); ++issued) {
            mbar_expect_tx(&full[issued], bytes);
            bulk_g2s(ring + (size_t)issued * SP, src_of(issued), bytes, &full[issued]);
        }
    }
    float4 vv[UP], ww[UP];
    // dots of one vector's pairs with v and w (FP32 products and lane
    // partial sums, as k_dcgs_reduce<float>); pair u comes from load(u)
    auto dots = [&](auto load, float &ar, float &ai, float &br, float &bi) {
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            const float4 qu = load(u);
            const float qe[4] = {qu.x, qu.y, qu.z, qu.w};
            const float ve[4] = {vv[u].x, vv[u].y, vv[u].z, vv[u].w};
            const float we[4] = {ww[u].x, ww[u].y, ww[u].z, ww[u].w};
#pragma unroll
            for (int h = 0; h < 4; h += 2) {
                const float qx = qe[h], qy = qe[h + 1];
                ar = fmaf(qx, ve[h], fmaf(qy, ve[h + 1], ar));
                ai = fmaf(qx, ve[h + 1], fmaf(-qy, ve[h], ai));
                br = fmaf(qx, we[h], fmaf(qy, we[h + 1], br));
                bi = fmaf(qx, we[h + 1], fmaf(-qy, we[h], bi));
            }
        }
    };
    auto add_sums = [&](int i, float ar, float ai, float br, float bi) {
        const double sar = warp_sum((double)ar), sai = warp_sum((double)ai);
        const double sbr = warp_sum((double)br), sbi = warp_sum((double)bi);
        if (lane == 0) {
            red[i][warp] = make_double2(sar, sai);
            red[nv + i][warp] = make_double2(sbr, sbi);
        }
    };
    bool ok = true;
    int i = 0;
    for (; i < NI; ++i) {
        const int stg = i % kBulkStages;
        const bool got = mbar_wait(&full[stg], (uint32_t)(i / kBulkStages) & 1u);
        const float4 *qs = ring + (size_t)stg * SP;
        auto ld = [&](int u) {
            const int p = threadIdx.x + u * NT;
            return (got && p < np) ? qs[p] : make_float4(0.f, 0.f, 0.f, 0.f);
        };
        if (i == 0) {
#pragma unroll
            for (int u = 0; u < UP; ++u) vv[u] = ld(u);
        } else if (i == 1) {
#pragma unroll
            for (int u = 0; u < UP; ++u) ww[u] = ld(u);
        } else {
            float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;
            dots(ld, ar, ai, br, bi);
            add_sums(i - 2, ar, ai, br, bi);
        }
        // every thread is done with this stage before it is refilled
        if (!__syncthreads_and(got)) {
            ok = false;
            break;
        }
        if (threadIdx.x == 0 && issued < NI) {
            fence_proxy_async();
            mbar_expect_tx(&full[stg], bytes);
            bulk_g2s(ring + (size_t)stg * SP, src_of(issued), bytes, &full[stg]);
            ++issued;
        }
    }
    if (ok) {
        float ar = 0.f, ai = 0.f, br = 0.f, bi = 0.f;   // slot j: v^H v and v^H w
        dots([&](int u) { return vv[u]; }, ar, ai, br, bi);
        add_sums(j, ar, ai, br, bi);
    } else if (threadIdx.x == 0) {
        if (err) atomicExch(err, 1);
        for (int q = i; q < issued; ++q)
            (void)mbar_wait(&full[q % kBulkStages], (uint32_t)(q / kBulkStages) & 1u);
    }
    __syncthreads();
    double2 *out = a.partial + (size_t)blk * a.pstride;
    for (int k = threadIdx.x; k < 2 * nv; k += NT) {
        double2 acc = red[k][0];
        for (int w = 1; w < NW; ++w) {
            acc.x += red[k][w].x;
            acc.y += red[k][w].y;
        }
        out[k] = acc;
    }
    if (last_block_reduce(a, s, 2 * nv, ds.dsum + (size_t)s * 2 * (m + 1))) {
        dcgs_coefficients_block(st, ds, s, m, j, rtol, inner_rtol, reinterpret_cast<double2 *>(smem_raw));
    }
}


// Per-system scalar work at the end of the update, for the last block of a
// system: the provisional column j from ||v_{j+1}||, its rotation, the
// iteration count and the stop rules.  Column j, the rotations and g are
// staged in shared memory by the whole block (sc: 3 (m + 1) + 2 m entries);
// thread 0 runs the serial part there.
__device__ void dcgs_update_finish_block(GmresState &st, const DcgsState &ds, int s, int m, int j,
                                         double rtol, int max_iter, double inner_rtol, double2 *sc)
{
    const int M1 = m + 1;
    double2 *rawj = sc;                          // [M1] unrotated column j
    double2 *Hj = rawj + M1;                     // [M1] its rotated form
    double2 *cs = Hj + M1;                       // [m]
    double2 *sn = cs + m;                        // [m]
    double2 *g = sn + m;                         // [M1]
    const size_t hb = (size_t)s * M1 * m + (size_t)j * M1;
    const int nt = blockDim.x;
    for (int i = threadIdx.x; i <= j; i += nt) rawj[i] = ds.Hraw[hb + i];
    for (int i = threadIdx.x; i < m; i += nt) {
        cs[i] = st.cs[(size_t)s * m + i];
        sn[i] = st.sn[(size_t)s * m + i];
    }
    for (int i = threadIdx.x; i < M1; i += nt) g[i] = st.g[(size_t)s * M1 + i];
    __syncthreads();
    if (threadIdx.x == 0) {
        const double vn2 = st.h2[(size_t)s * (m + 2)].x;
        const double beta = sqrt(fmax(vn2, 0.0));
        rawj[j + 1] = make_double2(beta, 0.0);
        ds.Hraw[hb + j + 1] = rawj[j + 1];
        const double2 gj = g[j];
        ds.gsave[s] = gj;
        const double est = dcgs_rotate_column_p(rawj, Hj, cs, sn, g, gj, j);
        st.cs[(size_t)s * m + j] = cs[j];
        st.sn[(size_t)s * m + j] = sn[j];
        st.g[(size_t)s * M1 + j] = g[j];
        st.g[(size_t)s * M1 + j + 1] = g[j + 1];
        st.est[s] = est;
        st.kcyc[s] = j + 1;
        st.iters[s] += 1;
        st.projv[s] += j + 1;
        bool stop = dcgs_stop(st, s, est, rtol, inner_rtol) || !isfinite(beta);
        if (j + 1 >= m) stop = true;
        if (st.iters[s] >= max_iter) stop = true;
        if (beta <= 1e-300) stop = true;
        if (stop) st.active[s] = 0;
    }
    __syncthreads();
    for (int i = threadIdx.x; i <= j + 1; i += nt) st.H[hb + i] = Hj[i];
}

// Update pass of step j over row chunks: slot j <- q_j, slot j + 1 <- v_{j+1}
// (one read of q_0 .. q_{j-1}, v, w; two writes), ||v_{j+1}||^2 reduced per
// system; the last block forms the provisional column j and its rotation,
// counts the iteration and applies the stop rules.
template <typename R>
__global__ void __launch_bounds__(256)
k_dcgs_update(ArnoldiArgs a, typename CT<R>::t *__restrict__ Q, int j,
              const typename CT<R>::t *__restrict__ W, GmresState st, DcgsState ds, int m,
              double rtol, int max_iter, double inner_rtol)
{
    using C2 = typename CT<R>::t;
    constexpr int UQ = 4;                        // basis vectors loaded per batch
    __shared__ C2 ca[kMaxRestart], cb[kMaxRestart];
    __shared__ double wsum[8];
    const int blk = blockIdx.x;
    const int s = a.tiles.sys[blk];
    if (a.gate && a.gate[s] == 0) return;
    const double2 *cf = ds.coef + (size_t)s * ds.cstride;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
        ca[i] = mk2<R>((R)cf[i].x, (R)cf[i].y);
        cb[i] = mk2<R>((R)cf[j + 1 + i].x, (R)cf[j + 1 + i].y);
    }
    const R inu = (R)cf[2 * m + 2].x;
    const C2 dv = mk2<R>((R)cf[2 * m + 3].x, (R)cf[2 * m + 3].y);
    __syncthreads();
    size_t e0;
    int ne;
    elem_range<R>(a, blk, 0, e0, ne);
    C2 *vq = Q + (size_t)j * a.qstride + e0;           // v in, q_j out
    C2 *vn = Q + (size_t)(j + 1) * a.qstride + e0;     // v_{j+1} out
    const C2 *wp = W + e0;
    // FP32: two consecutive elements per thread (16-byte loads) when every
    // vector's chunk starts on an even element
    const bool pairs = std::is_same<R, float>::value && (e0 % 2 == 0) && (a.qstride % 2 == 0);
    const int step = pairs ? 2 : 1;
    double nrm = 0.0;
    for (int e = threadIdx.x * step; e < ne; e += blockDim.x * step) {
        const bool two = pairs && e + 1 < ne;
        C2 v0 = vq[e], v1 = two ? vq[e + 1] : mk2<R>(0, 0);
        C2 w0 = wp[e], w1 = two ? wp[e + 1] : mk2<R>(0, 0);
        // q = v / nu ; n = w / nu + dv v
        C2 q0 = mk2<R>(v0.x * inu, v0.y * inu), q1 = mk2<R>(v1.x * inu, v1.y * inu);
        C2 n0 = mk2<R>(w0.x * inu + (dv.x * v0.x - dv.y * v0.y), w0.y * inu + (dv.x * v0.y + dv.y * v0.x));
        C2 n1 = mk2<R>(w1.x * inu + (dv.x * v1.x - dv.y * v1.y), w1.y * inu + (dv.x * v1.y + dv.y * v1.x));
        for (int i0 = 0; i0 < j; i0 += UQ) {
            C2 b0[UQ], b1[UQ];
#pragma unroll
            for (int u = 0; u < UQ; ++u) {
                const int i = i0 + u;
                b0[u] = mk2<R>(0, 0);
                b1[u] = mk2<R>(0, 0);
                if (i < j) {
                    const C2 *qp = Q + (size_t)i * a.qstride + e0 + e;
                    if (two) {
                        const float4 t = *reinterpret_cast<const float4 *>(qp);
                        b0[u] = mk2<R>((R)t.x, (R)t.y);
                        b1[u] = mk2<R>((R)t.z, (R)t.w);
                    } else {
                        b0[u] = *qp;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < UQ; ++u) {
                // past the last vector b0 = b1 = 0, so any coefficient works
                const int i = min(i0 + u, j - 1);
                const C2 x = ca[i], y = cb[i];
                const C2 p0 = b0[u], p1 = b1[u];
                q0.x = fma(p0.x, x.x, fma(-p0.y, x.y, q0.x));
                q0.y = fma(p0.x, x.y, fma(p0.y, x.x, q0.y));
                q1.x = fma(p1.x, x.x, fma(-p1.y, x.y, q1.x));
                q1.y = fma(p1.x, x.y, fma(p1.y, x.x, q1.y));
                n0.x = fma(p0.x, y.x, fma(-p0.y, y.y, n0.x));
                n0.y = fma(p0.x, y.y, fma(p0.y, y.x, n0.y));
                n1.x = fma(p1.x, y.x, fma(-p1.y, y.y, n1.x));
                n1.y = fma(p1.x, y.y, fma(p1.y, y.x, n1.y));
            }
        }
        vq[e] = q0;
        vn[e] = n0;
        nrm += (double)n0.x * n0.x + (double)n0.y * n0.y;
        if (two) {
            vq[e + 1] = q1;
            vn[e + 1] = n1;
            nrm += (double)n1.x * n1.x + (double)n1.y * n1.y;
        }
    }
    nrm = warp_sum(nrm);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = nrm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
        a.partial[(size_t)blk * a.pstride] = make_double2(t, 0.0);
    }
    if (last_block_reduce(a, s, 1, st.h2 + (size_t)s * (m + 2))) {
        extern __shared__ __align__(16) unsigned char dcgs_scratch[];   // 3 (m + 1) + 2 m entries
        dcgs_update_finish_block(st, ds, s, m, j, rtol, max_iter, inner_rtol,
                                 reinterpret_cast<double2 *>(dcgs_scratch));
    }
}

// Update pass of step j with the basis streamed through shared memory
// (FP32 Krylov vectors; the chunks and stages of k_dcgs_reduce_bulk).
// The stream is v, w, q_0 .. q_{j-1}: thread t forms q_j and v_{j+1} of its
// element pairs t, t + 256, ... in registers from v and w, then adds a_i q_i
// and b_i q_i as the basis arrives; the arithmetic and ||v_{j+1}||^2 are
// those of k_dcgs_update, the last block runs dcgs_update_finish_block with
// the ring as its scratch.  A wait that times out sets *err; the block then writes
// nothing, waits (bounded) for its copies in flight and still takes part
// in the per-system arrival count.
__global__ void __launch_bounds__(256, 2)
k_dcgs_update_bulk(ArnoldiArgs a, float2 *__restrict__ Q, int j, const float2 *__restrict__ W,
                   GmresState st, DcgsState ds, int m, double rtol, int max_iter,
                   double inner_rtol, int *err)
{
    constexpr int NT = 256;
    constexpr int UP = kBulkChunk / (2 * NT);
    constexpr int SP = kBulkChunk / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float4 *ring = reinterpret_cast<float4 *>(smem_raw);
    __shared__ __align__(8) uint64_t full[kBulkStages];
    __shared__ float2 ca[kMaxRestart], cb[kMaxRestart];
    __shared__ double wsum[NT / 32];
    const int blk = blockIdx.x;
    const int s = a.tiles.sys[blk];
    if (a.gate && a.gate[s] == 0) return;
    const double2 *cf = ds.coef + (size_t)s * ds.cstride;
    for (int i = threadIdx.x; i < j; i += NT) {
        ca[i] = make_float2((float)cf[i].x, (float)cf[i].y);
        cb[i] = make_float2((float)cf[j + 1 + i].x, (float)cf[j + 1 + i].y);
    }
    const float inu = (float)cf[2 * m + 2].x;
    const float2 dv = make_float2((float)cf[2 * m + 3].x, (float)cf[2 * m + 3].y);
    size_t e0;
    int ne;
    elem_range<float>(a, blk, 0, e0, ne);
    const int np = ne >> 1;
    const uint32_t bytes = (uint32_t)ne * 8u;
    if (threadIdx.x == 0) {
        for (int q = 0; q < kBulkStages; ++q) mbar_init(&full[q], 1);
        mbar_fence_init();
    }
    __syncthreads();
    // the stream: item 0 = v (slot j), item 1 = w, item 2 + i = q_i
    const int NI = j + 2;
    auto src_of = [&](int it) {
        return it == 0 ? Q + (size_t)j * a.qstride + e0
             : it == 1 ? W + e0 : Q + (size_t)(it - 2) * a.qstride + e0;
    };
    int issued = 0;
    if (threadIdx.x == 0) {
        for (; issued < min(kBulkStages, NI); ++issued) {
            mbar_expect_tx(&full[issued], bytes);
            bulk_g2s(ring + (size_t)issued * SP, src_of(issued), bytes, &full[issued]);
        }
    }
    float4 *vq = reinterpret_cast<float4 *>(Q + (size_t)j * a.qstride + e0);        // v in, q_j out
    float4 *vn = reinterpret_cast<float4 *>(Q + (size_t)(j + 1) * a.qstride + e0);  // v_{j+1} out
    float4 qa[UP], na[UP];
    bool ok = true;
    int i = 0;
    for (; i < NI; ++i) {
        const int stg = i % kBulkStages;
        const bool got = mbar_wait(&full[stg], (uint32_t)(i / kBulkStages) & 1u);
        const float4 *qs = ring + (size_t)stg * SP;
        if (i < 2) {
#pragma unroll
            for (int u = 0; u < UP; ++u) {
                const int p = threadIdx.x + u * NT;
                const float4 t = (got && p < np) ? qs[p] : make_float4(0.f, 0.f, 0.f, 0.f);
                if (i == 0) {
                    qa[u] = t;                          // v, until w arrives
                } else {
                    // q = v / nu ; n = w / nu + dv v   (two elements per float4)
                    const float4 v = qa[u], w = t;
                    qa[u] = make_float4(v.x * inu, v.y * inu, v.z * inu, v.w * inu);
                    na[u] = make_float4(w.x * inu + (dv.x * v.x - dv.y * v.y),
                                        w.y * inu + (dv.x * v.y + dv.y * v.x),
                                        w.z * inu + (dv.x * v.z - dv.y * v.w),
                                        w.w * inu + (dv.x * v.w + dv.y * v.z));
                }
            }
        } else {
        const float2 x = ca[i - 2], y = cb[i - 2];
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            const int p = threadIdx.x + u * NT;
            const float4 b = (got && p < np) ? qs[p] : make_float4(0.f, 0.f, 0.f, 0.f);
            float4 &q = qa[u];
            float4 &nn = na[u];
            q.x = fmaf(b.x, x.x, fmaf(-b.y, x.y, q.x));
            q.y = fmaf(b.x, x.y, fmaf(b.y, x.x, q.y));
            q.z = fmaf(b.z, x.x, fmaf(-b.w, x.y, q.z));
            q.w = fmaf(b.z, x.y, fmaf(b.w, x.x, q.w));
            nn.x = fmaf(b.x, y.x, fmaf(-b.y, y.y, nn.x));
            nn.y = fmaf(b.x, y.y, fmaf(b.y, y.x, nn.y));
            nn.z = fmaf(b.z, y.x, fmaf(-b.w, y.y, nn.z));
            nn.w = fmaf(b.z, y.y, fmaf(b.w, y.x, nn.w));
        }
        }
        if (!__syncthreads_and(got)) {
            ok = false;
            break;
        }
        if (threadIdx.x == 0 && issued < NI) {
            fence_proxy_async();
            mbar_expect_tx(&full[stg], bytes);
            bulk_g2s(ring + (size_t)stg * SP, src_of(issued), bytes, &full[stg]);
            ++issued;
        }
    }
    double nrm = 0.0;
    if (ok) {
#pragma unroll
        for (int u = 0; u < UP; ++u) {
            const int p = threadIdx.x + u * NT;
            if (p < np) {
                vq[p] = qa[u];
                vn[p] = na[u];
                const float4 nn = na[u];
                nrm += (double)nn.x * nn.x + (double)nn.y * nn.y + (double)nn.z * nn.z +
                       (double)nn.w * nn.w;
            }
        }
    } else if (threadIdx.x == 0) {
        if (err) atomicExch(err, 1);
        for (int q = i; q < issued; ++q)
            (void)mbar_wait(&full[q % kBulkStages], (uint32_t)(q / kBulkStages) & 1u);
    }
    nrm = warp_sum(nrm);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = nrm;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; ++w) t += wsum[w];
        a.partial[(size_t)blk * a.pstride] = make_double2(t, 0.0);
    }
    if (last_block_reduce(a, s, 1, st.h2 + (size_t)s * (m + 2))) {
        dcgs_update_finish_block(st, ds, s, m, j, rtol, max_iter, inner_rtol,
                                 reinterpret_cast<double2 *>(smem_raw));
    }
}

// I_G = |2i b_G psi_G(z_n) + delta_{G,spec} a_spec|^2
__global__ void k_intensities(int nrows, int row_offset, int n, const int *__restrict__ row_sys,
                              const int *__restrict__ sys_spec_row,
                              const double2 *__restrict__ sys_aspec,
                              const double2 *__restrict__ row_b, const double2 *__restrict__ psi,
                              double *__restrict__ out)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const int s = row_sys[row];
    const double2 p = psi[(size_t)row * n + (n - 1)];
    const double2 b = row_b[row];
    double2 amp = cmul(make_double2(0.0, 2.0), cmul(b, p));
    if (row + row_offset == sys_spec_row[s]) amp = cadd(amp, sys_aspec[s]);
    out[row] = cabs2(amp);
}

// ---------------------------------------------------------------------------
// Adjoint (no counterpart in the reference, which has no derivatives).
//
// Forward:  A psi = u_fwd,  S_G = 2i b_G psi_G(z_n) + delta_{G,spec} a_spec.
// For a real loss L with gamma_G = dL/dS_G in the (Re + i Im) convention,
// dL = Re sum conj(gamma_G) dS_G = 2 Re <u, d psi> with the outer-boundary
// vector u_G(z_n) = -i gamma_G conj(b_G).  With A^H lambda = u and
// d psi = -A^{-1} (dA) psi:  dL = -2 Re <lambda, (dA) psi>.
// ---------------------------------------------------------------------------

// u_G = -i gamma_G conj(b_G),  gamma_G = 2 dl_di[G] S_G + dl_ds[G]
// (either input may be null).
__global__ void k_adjoint_rhs(int nrows, int n, const int *__restrict__ row_sys,
                              const int *__restrict__ sys_spec_row,
                              const double2 *__restrict__ sys_aspec,
                              const double2 *__restrict__ row_b, const double2 *__restrict__ psi,
                              const double *__restrict__ dl_di, const double2 *__restrict__ dl_ds,
                              double2 *__restrict__ rhs)
{
    const int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= nrows) return;
    const double2 b = row_b[row];
    double2 gamma = make_double2(0.0, 0.0);
    if (dl_di) {
        const int s = row_sys[row];
        const double2 p = psi[(size_t)row * n + (n - 1)];
        double2 amp = cmul(make_double2(0.0, 2.0), cmul(b, p));
        if (row == sys_spec_row[s]) amp = cadd(amp, sys_aspec[s]);
        gamma = cscale(amp, 2.0 * dl_di[row]);
    }
    if (dl_ds) gamma = cadd(gamma, dl_ds[row]);
    rhs[row] = cmul(make_double2(0.0, -1.0), cmul(gamma, cconj(b)));
}

// bnorm[s] = || rhs restricted to system s ||  (one block per system, fixed
// summation order).
__global__ void __launch_bounds__(256)
k_system_norms(const int *__restrict__ sys_row0, const double2 *__restrict__ rhs,
               double *__restrict__ bnorm)
{
    __shared__ double ws[8];
    const int s = blockIdx.x;
    double acc = 0.0;
    for (int r = sys_row0[s] + threadIdx.x; r < sys_row0[s + 1]; r += blockDim.x)
        acc += cabs2(rhs[r]);
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
        bnorm[s] = sqrt(t);
    }
}

// dL/dV_D(z) for every torus offset D = (dx, dy) in a window, summed over the
// systems of the plan (they share V):
//   K_D(z) = sum_s sum_{G in s, G - D in s} conj(lambda_G(z)) psi_{G-D}(z)
//   grad[D][z] = -2 conj(K_D(z))   (D != 0: the coupling uses V_D, complex)
//   grad[0][z] = -2 Re K_0(z)       (only Re V_0 enters the diagonal)
// in the (dL/dRe + i dL/dIm) convention.  A per-z correlation of lambda with
// psi over the channel torus ("outer product" restricted to its diagonals).
// Layout: grad [nkx][nky][n], the potential's own layout.
// Grid: x = window offsets / (8 warps * kGradPerWarp), y = z / 32.  Lane = z,
// so psi / lambda rows ([row][z]) are read coalesced; each (D, z) is summed by
// one thread in a fixed order.
constexpr int kGradPerWarp = 4;

__global__ void __launch_bounds__(256)
k_potential_gradient(int nkx, int nky, int n, int nsys, const int *__restrict__ sys_row0,
                     const int *__restrict__ row_pos, const int *__restrict__ pos_map,
                     int wx, int wy, int hx, int hy, const double2 *__restrict__ psi,
                     const double2 *__restrict__ lam, double2 *__restrict__ grad)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.y * 32 + lane;
    const int nwin = wx * wy;
    const int d0 = (blockIdx.x * 8 + warp) * kGradPerWarp;
    if (d0 >= nwin) return;
    int dx[kGradPerWarp], dy[kGradPerWarp];
    double2 acc[kGradPerWarp];
#pragma unroll
    for (int k = 0; k < kGradPerWarp; ++k) {
        const int d = min(d0 + k, nwin - 1);
        const int ux = d / wy, uy = d - ux * wy;
        dx[k] = ((ux - hx) % nkx + nkx) % nkx;
        dy[k] = ((uy - hy) % nky + nky) % nky;
        acc[k] = make_double2(0.0, 0.0);
    }
    const int ntor = nkx * nky;
    const bool zok = z < n;
    for (int s = 0; s < nsys; ++s) {
        const int *map = pos_map + (size_t)s * ntor;
        for (int r = sys_row0[s]; r < sys_row0[s + 1]; ++r) {
            const double2 l = zok ? lam[(size_t)r * n + z] : make_double2(0.0, 0.0);
            const int pos = row_pos[r];
            const int ix = pos / nky, iy = pos - ix * nky;
#pragma unroll
            for (int k = 0; k < kGradPerWarp; ++k) {
                int sx = ix - dx[k];
                sx += (sx < 0) ? nkx : 0;
                int sy = iy - dy[k];
                sy += (sy < 0) ? nky : 0;
                const int r2 = __ldg(map + sx * nky + sy);
                if (r2 >= 0 && zok) {
                    const double2 q = psi[(size_t)r2 * n + z];
                    // conj(l) * q
                    acc[k].x = fma(l.x, q.x, fma(l.y, q.y, acc[k].x));
                    acc[k].y = fma(l.x, q.y, fma(-l.y, q.x, acc[k].y));
                }
            }
        }
    }
    if (!zok) return;
#pragma unroll
    for (int k = 0; k < kGradPerWarp; ++k) {
        if (d0 + k >= nwin) break;
        const size_t o = ((size_t)dx[k] * nky + dy[k]) * n + z;
        grad[o] = (dx[k] == 0 && dy[k] == 0) ? make_double2(-2.0 * acc[k].x, 0.0)
                                             : make_double2(-2.0 * acc[k].x, 2.0 * acc[k].y);
    }
}

// Plan set-up on the device, one thread per channel row:
//   fn[row]  = sum_k E[n-1,k]^2 / (pkd_row + lam_k)   (Sherman-Morrison factor
//              of the block inverse, multiscat_gmres.f90:226-273)
//   nbr[row][t] = row of the same system at position G - d_t, or -1
// pos_map [B][nkx*nky] gives the row of each torus position per system.
__global__ void k_row_tables(int nrows, int n, int ntaps, int nkx, int nky,
                             const int *__restrict__ row_pos, const int *__restrict__ row_sys,
                             const int *__restrict__ pos_map, const int2 *__restrict__ taps,
                             const double *__restrict__ row_pkd, const double *__restrict__ en,
                             const double *__restrict__ lam, double *__restrict__ fn,
                             float *__restrict__ fn32, int *__restrict__ nbr)
{
    const int ntor = nkx * nky;
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nrows;
         row += gridDim.x * blockDim.x) {
        const double pkd = row_pkd[row];
        double f = 0.0;
        for (int k = 0; k < n; ++k) {
            const double e = en[k];
            f += e * e / (pkd + lam[k]);
        }
        fn[row] = f;
        if (fn32) fn32[row] = (float)f;
        if (!nbr) continue;
        const int pos = row_pos[row];
        const int ix = pos / nky, iy = pos - ix * nky;
        const int *map = pos_map + (size_t)row_sys[row] * ntor;
        for (int t = 0; t < ntaps; ++t) {
            int sx = ix - taps[t].x;
            sx += (sx < 0) ? nkx : 0;
            int sy = iy - taps[t].y;
            sy += (sy < 0) ? nky : 0;
            nbr[(size_t)row * ntaps + t] = map[sx * nky + sy];
        }
    }
}

// The Sherman-Morrison factor of each row, c / (1 - c f_n), for the tcgen05
// block inverse (its per-channel complex division, formed once per plan and
// operator instead of in every tile).
__global__ void k_row_cfac(int nrows, const double2 *__restrict__ row_c,
                           const double *__restrict__ fn, double2 *__restrict__ cf)
{
    for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nrows;
         row += gridDim.x * blockDim.x) {
        const double2 c = row_c[row];
        const double f = fn[row];
        cf[row] = cdiv(c, make_double2(1.0 - c.x * f, -c.y * f));
    }
}

// dst = src (add = 0) or dst += src (add = 1) on the rows of the gated tiles.
template <typename R>
__global__ void __launch_bounds__(256)
k_copy_add(Tiles tiles, const int *__restrict__ gate, int n, const typename CT<R>::t *__restrict__ src,
           typename CT<R>::t *__restrict__ dst, int add)
{
    const int tile = blockIdx.x;
    if (gate && gate[tiles.sys[tile]] == 0) return;
    const size_t e0 = (size_t)tiles.row0[tile] * n;
    const int ne = tiles.nrow[tile] * n;
    for (int e = blockIdx.y * blockDim.x + threadIdx.x; e < ne; e += gridDim.y * blockDim.x) {
        typename CT<R>::t v = src[e0 + e];
        if (add) {
            const typename CT<R>::t d = dst[e0 + e];
            v.x += d.x;
            v.y += d.y;
        }
        dst[e0 + e] = v;
    }
}

__global__ void k_scale(double2 *p, size_t count, double sc)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count;
         i += (size_t)gridDim.x * blockDim.x)
        p[i] = make_double2(p[i].x * sc, p[i].y * sc);
}

}  // namespace msc
