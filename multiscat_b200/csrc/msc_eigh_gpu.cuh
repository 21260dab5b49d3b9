// msc_eigh_gpu.cuh -- FP64 symmetric eigen-decomposition of H0 on the GPU.
//
// The preconditioner needs H0 = T + diag Re V_00 = E diag(lam) E^T once per
// potential (the reference: build_preconditioner, multiscat_gmres.f90:226-273,
// with EISPACK rs = tred2 + tql2, diagsub.f90:5-262).  Here the O(n^3) parts
// run on the device and the host does O(n^2) scalar work only:
//
//   1. k_tridiagonalize (one CTA): Householder reduction A = Q_H T Q_H^T,
//      Q_H = H_0 H_1 ... H_{n-3}, H_k = I - 2 v_k v_k^T (unit v_k supported on
//      k+1 .. n-1).  The matrix lives in shared memory when it fits (n <= 160),
//      else in global memory (L2-resident for every n of this solver).
//   2. host: implicit symmetric QR with Wilkinson shifts on the tridiagonal
//      (d, e), recording every Givens rotation (k, c, s) it applies
//      (tridiagonal_qr_rotations in msc_eigh.hpp).  O(n) per sweep.
//   3. k_apply_rotations: Z = G_1 G_2 ... from the identity, one thread per
//      row of Z; a rotation acts on columns k, k+1 of every row, so rows are
//      independent and each CTA keeps its rows in shared memory.
//   4. k_back_transform: E = Q_H Z, the reflectors applied from the left in
//      reverse order; a reflector acts on rows, so columns are independent
//      and each CTA keeps its columns in shared memory.  Columns are written
//      in ascending eigenvalue order.
#pragma once

#include "msc_common.cuh"

namespace msc {
namespace eig {

constexpr int kTriThreads = 1024;
constexpr int kTriSmemMaxN = 160;          // n^2 doubles in shared memory up to here

__device__ __forceinline__ double block_sum(double v, double *red)
{
    v = warp_sum(v);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();                        // red may still be read by a previous call
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];   // same order in every thread
    return t;
}

// A: n x n symmetric, row-major, full storage (destroyed).  R: row k holds
// v_k at columns k+1 .. n-1 (unit vector); applied[k] = 0 when column k
// needed no reflection.  d[n], e[n-1].  Dynamic shared memory: n*n doubles
// when n <= kTriSmemMaxN (the matrix is worked on there), else none.
__global__ void __launch_bounds__(kTriThreads)
k_tridiagonalize(int n, double *__restrict__ A, double *__restrict__ R, double *__restrict__ d,
                 double *__restrict__ e, int *__restrict__ applied)
{
    extern __shared__ double sm_a[];
    __shared__ double v[kMaxNz], p[kMaxNz], red[32];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    const bool in_smem = n <= kTriSmemMaxN;
    double *M = A;
    if (in_smem) {
        for (int i = tid; i < n * n; i += nt) sm_a[i] = A[i];
        M = sm_a;
        __syncthreads();
    }
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        const double *rowk = M + (size_t)k * n + (k + 1);    // = column k below the diagonal
        double part = 0.0;
        for (int i = tid; i < m; i += nt) {
            const double x = rowk[i];
            v[i] = x;
            part += x * x;
        }
        const double nrm2 = block_sum(part, red);
        if (nrm2 == 0.0) {
            if (tid == 0) {
                d[k] = M[(size_t)k * n + k];
                e[k] = 0.0;
                applied[k] = 0;
            }
            __syncthreads();
            continue;
        }
        const double x0 = v[0];
        const double alpha = (x0 >= 0.0) ? -sqrt(nrm2) : sqrt(nrm2);
        const double vn2 = nrm2 - x0 * x0 + (x0 - alpha) * (x0 - alpha);
        const double inv = 1.0 / sqrt(vn2);
        __syncthreads();                                       // every thread has read v[0]
        for (int i = tid; i < m; i += nt) v[i] = (i == 0 ? x0 - alpha : v[i]) * inv;
        __syncthreads();
        // p = S v over the trailing block S = M[k+1.., k+1..]
        for (int i = warp; i < m; i += nw) {
            const double *row = M + (size_t)(k + 1 + i) * n + (k + 1);
            double s = 0.0;
            for (int j = lane; j < m; j += 32) s = fma(row[j], v[j], s);
            s = warp_sum(s);
            if (lane == 0) p[i] = s;
        }
        __syncthreads();
        part = 0.0;
        for (int i = tid; i < m; i += nt) part += v[i] * p[i];
        const double vp = block_sum(part, red);
        for (int i = tid; i < m; i += nt) p[i] -= vp * v[i];
        __syncthreads();
        // S <- (I - 2 v v^T) S (I - 2 v v^T) = S - 2 v p^T - 2 p v^T
        for (int i = warp; i < m; i += nw) {
            double *row = M + (size_t)(k + 1 + i) * n + (k + 1);
            const double vi2 = 2.0 * v[i], pi2 = 2.0 * p[i];
            for (int j = lane; j < m; j += 32) row[j] -= vi2 * p[j] + pi2 * v[j];
        }
        for (int i = tid; i < m; i += nt) R[(size_t)k * n + (k + 1) + i] = v[i];
        if (tid == 0) {
            d[k] = M[(size_t)k * n + k];
            e[k] = alpha;
            applied[k] = 1;
        }
        __syncthreads();
    }
    if (tid == 0) {
        if (n >= 2) {
            d[n - 2] = M[(size_t)(n - 2) * n + (n - 2)];
            e[n - 2] = M[(size_t)(n - 1) * n + (n - 2)];
            applied[n - 2] = 0;
        }
        d[n - 1] = M[(size_t)(n - 1) * n + (n - 1)];
        applied[n - 1] = 0;
    }
}

// Z = G_1 G_2 ... G_r (from the identity): rotation i acts on columns
// k = rk[i], k + 1 of every row: (z_k, z_{k+1}) <- (c z_k + s z_{k+1},
// c z_{k+1} - s z_k).  One thread per row, RB rows per CTA kept in shared
// memory as zs[col][row]; within a QR sweep k rises by one per rotation, so
// the updated z_{k+1} is carried to the next rotation in a register.
// Output Zt[col][row] (column-major Z).
template <int RB>
__global__ void __launch_bounds__(RB)
k_apply_rotations(int n, int nrot, const int *__restrict__ rk, const double *__restrict__ rc,
                  const double *__restrict__ rs, double *__restrict__ Zt)
{
    extern __shared__ double zs[];                 // [n][RB]
    const int t = threadIdx.x;
    const int row = blockIdx.x * RB + t;
    for (int c = 0; c < n; ++c) zs[c * RB + t] = (c == row) ? 1.0 : 0.0;
    int carry_k = -1;
    double carry = 0.0;
    for (int i = 0; i < nrot; ++i) {
        const int k = __ldg(rk + i);
        const double c = __ldg(rc + i), s = __ldg(rs + i);
        const double qa = (carry_k == k) ? carry : zs[k * RB + t];
        const double qb = zs[(k + 1) * RB + t];
        zs[k * RB + t] = c * qa + s * qb;
        carry = c * qb - s * qa;
        carry_k = k + 1;
        zs[(k + 1) * RB + t] = carry;
    }
    if (row < n)
        for (int c = 0; c < n; ++c) Zt[(size_t)c * n + row] = zs[c * RB + t];
}

// E = Q_H Z: CB columns of Z per CTA in shared memory (zc[col][row]),
// reflectors H_{n-3} .. H_0 applied in turn (z <- z - 2 v (v^T z) on rows
// k+1 .. n-1).  Column j of the result is written to column dest[j] of the
// row-major output E[row * n + col] (ascending eigenvalue order).
template <int CB>
__global__ void __launch_bounds__(256)
k_back_transform(int n, const double *__restrict__ R, const int *__restrict__ applied,
                 const double *__restrict__ Zt, const int *__restrict__ dest, double *__restrict__ E)
{
    extern __shared__ double zc[];                 // [CB][n]
    __shared__ double v[kMaxNz];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, nw = blockDim.x >> 5;
    const int c0 = blockIdx.x * CB;
    const int ncol = min(CB, n - c0);
    for (int i = tid; i < ncol * n; i += blockDim.x) zc[i] = Zt[(size_t)c0 * n + i];
    __syncthreads();
    for (int k = n - 3; k >= 0; --k) {
        if (!applied[k]) continue;
        const int m = n - k - 1;
        for (int i = tid; i < m; i += blockDim.x) v[i] = R[(size_t)k * n + (k + 1) + i];
        __syncthreads();
        for (int c = warp; c < ncol; c += nw) {
            double *z = zc + (size_t)c * n + (k + 1);
            double s = 0.0;
            for (int i = lane; i < m; i += 32) s = fma(v[i], z[i], s);
            s = 2.0 * warp_sum(s);
            for (int i = lane; i < m; i += 32) z[i] -= s * v[i];
        }
        __syncthreads();
    }
    for (int i = tid; i < ncol * n; i += blockDim.x) {
        const int c = i / n, r = i - c * n;
        E[(size_t)r * n + dest[c0 + c]] = zc[i];
    }
}

}  // namespace eig
}  // namespace msc
