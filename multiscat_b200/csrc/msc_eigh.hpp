// msc_eigh.hpp -- FP64 symmetric eigen-decomposition for the preconditioner.
//
// H0 = T + diag Re V_00 is diagonalised once per potential (the reference
// does the same with EISPACK rs = tred2 + tql2, diagsub.f90:5-262, inside
// build_preconditioner, multiscat_gmres.f90:251-253).  Method: Householder
// reduction to tridiagonal form (reflectors accumulated into Q), then
// implicit symmetric QR steps with a Wilkinson shift and explicit bulge
// chasing, rotations accumulated into Q.  Eigenvalues ascending; eigenvector
// k is column k of V (V[i*n + k]).
//
// Only the preconditioner depends on these eigenpairs: the true residual of
// the solve uses T itself, so eigenvector round-off changes the iteration
// count, never the converged answer.
#pragma once

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

namespace msc {

inline int symmetric_eigh(int n, const double *A, double *w, double *V)
{
    std::vector<double> a(A, A + (size_t)n * n);
    std::vector<double> q((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) q[(size_t)i * n + i] = 1.0;
    std::vector<double> v(n), p(n);

    // Tridiagonalise column by column: zero a[k+2.., k].
    for (int k = 0; k + 2 < n; ++k) {
        const int m = n - k - 1;
        double nrm2 = 0.0;
        for (int i = 0; i < m; ++i) {
            const double t = a[(size_t)(k + 1 + i) * n + k];
            nrm2 += t * t;
        }
        if (nrm2 == 0.0) continue;
        const double nrm = std::sqrt(nrm2);
        const double x0 = a[(size_t)(k + 1) * n + k];
        const double alpha = (x0 >= 0.0) ? -nrm : nrm;
        for (int i = 0; i < m; ++i) v[i] = a[(size_t)(k + 1 + i) * n + k];
        v[0] -= alpha;
        double vn2 = 0.0;
        for (int i = 0; i < m; ++i) vn2 += v[i] * v[i];
        if (vn2 == 0.0) continue;
        const double inv = 1.0 / std::sqrt(vn2);
        for (int i = 0; i < m; ++i) v[i] *= inv;
        // S <- (I - 2vv^T) S (I - 2vv^T) on the trailing block
        double vp = 0.0;
        for (int i = 0; i < m; ++i) {
            const double *row = &a[(size_t)(k + 1 + i) * n + (k + 1)];
            double s = 0.0;
            for (int j = 0; j < m; ++j) s += row[j] * v[j];
            p[i] = s;
            vp += v[i] * s;
        }
        for (int i = 0; i < m; ++i) p[i] -= vp * v[i];
        for (int i = 0; i < m; ++i) {
            double *row = &a[(size_t)(k + 1 + i) * n + (k + 1)];
            const double vi2 = 2.0 * v[i], pi2 = 2.0 * p[i];
            for (int j = 0; j < m; ++j) row[j] -= vi2 * p[j] + pi2 * v[j];
        }
        a[(size_t)(k + 1) * n + k] = alpha;
        a[(size_t)k * n + (k + 1)] = alpha;
        for (int i = 1; i < m; ++i) {
            a[(size_t)(k + 1 + i) * n + k] = 0.0;
            a[(size_t)k * n + (k + 1 + i)] = 0.0;
        }
        for (int r = 0; r < n; ++r) {
            double *row = &q[(size_t)r * n + (k + 1)];
            double s = 0.0;
            for (int j = 0; j < m; ++j) s += row[j] * v[j];
            s *= 2.0;
            for (int j = 0; j < m; ++j) row[j] -= s * v[j];
        }
    }
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = a[(size_t)i * n + i];
    for (int i = 0; i + 1 < n; ++i) e[i] = a[(size_t)(i + 1) * n + i];

    // Implicit QR on the tridiagonal (d, e).
    const double eps = std::numeric_limits<double>::epsilon();
    long steps = 0;
    const long max_steps = 60L * n + 100;
    for (;;) {
        for (int i = 0; i + 1 < n; ++i)
            if (std::fabs(e[i]) <= eps * (std::fabs(d[i]) + std::fabs(d[i + 1]))) e[i] = 0.0;
        int hi = n - 1;
        while (hi > 0 && e[hi - 1] == 0.0) --hi;
        if (hi == 0) break;
        int lo = hi - 1;
        while (lo > 0 && e[lo - 1] != 0.0) --lo;
        if (++steps > max_steps) return 1;
        const double half = 0.5 * (d[hi - 1] - d[hi]);
        const double eh = e[hi - 1];
        const double shift = d[hi] - eh * eh / (half + std::copysign(std::hypot(half, eh), half));
        double x = d[lo] - shift, y = e[lo];
        for (int k = lo; k < hi; ++k) {
            const double r = std::hypot(x, y);
            const double c = (r == 0.0) ? 1.0 : x / r;
            const double s = (r == 0.0) ? 0.0 : y / r;
            if (k > lo) e[k - 1] = r;
            const double dk = d[k], dk1 = d[k + 1], ek = e[k];
            const double cc = c * c, ss = s * s, cs2 = 2.0 * c * s;
            d[k] = cc * dk + cs2 * ek + ss * dk1;
            d[k + 1] = ss * dk - cs2 * ek + cc * dk1;
            e[k] = c * s * (dk1 - dk) + (cc - ss) * ek;
            if (k + 1 < hi) {
                x = e[k];
                y = s * e[k + 1];
                e[k + 1] *= c;
            }
            for (int r2 = 0; r2 < n; ++r2) {
                double *qr = &q[(size_t)r2 * n];
                const double qa = qr[k], qb = qr[k + 1];
                qr[k] = c * qa + s * qb;
                qr[k + 1] = c * qb - s * qa;
            }
        }
    }
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int i, int j) { return d[i] < d[j]; });
    for (int k = 0; k < n; ++k) {
        w[k] = d[order[k]];
        for (int r = 0; r < n; ++r) V[(size_t)r * n + k] = q[(size_t)r * n + order[k]];
    }
    return 0;
}

}  // namespace msc
