// msc_eigh.hpp -- host part of the FP64 symmetric eigen-decomposition of H0.
//
// H0 = T + diag Re V_00 is diagonalised once per potential (the reference
// does the same with EISPACK rs = tred2 + tql2, diagsub.f90:5-262, inside
// build_preconditioner, multiscat_gmres.f90:251-253).  The O(n^3) steps --
// Householder tridiagonalisation, accumulation of the rotations into the
// eigenvectors and the back-transformation -- run on the GPU
// (msc_eigh_gpu.cuh).  What stays here is the O(n^2) scalar iteration on the
// tridiagonal matrix: implicit symmetric QR steps with a Wilkinson shift and
// explicit bulge chasing, every Givens rotation recorded as (k, c, s) so the
// device can apply them to all rows of Z at once.  Eigenvalues come back in
// d (unsorted, as the iteration leaves them).
//
// Only the preconditioner depends on these eigenpairs: the true residual of
// the solve uses T itself, so eigenvector round-off changes the iteration
// count, never the converged answer.
#pragma once

#include <cmath>
#include <limits>
#include <vector>

namespace msc {

// d[n] diagonal, e[n] sub-diagonal (e[i] couples i and i+1; e[n-1] unused).
// Appends the rotations (k, c, s), in the order they act on the columns
// (k, k+1) of Z: (z_k, z_{k+1}) <- (c z_k + s z_{k+1}, c z_{k+1} - s z_k).
// Returns 0 on success, 1 if the iteration did not converge.
inline int tridiagonal_qr_rotations(int n, std::vector<double> &d, std::vector<double> &e,
                                    std::vector<int> &rk, std::vector<double> &rc,
                                    std::vector<double> &rs)
{
    const double eps = std::numeric_limits<double>::epsilon();
    long steps = 0;
    const long max_steps = 60L * n + 100;
    for (;;) {
        for (int i = 0; i + 1 < n; ++i)
            if (std::fabs(e[i]) <= eps * (std::fabs(d[i]) + std::fabs(d[i + 1]))) e[i] = 0.0;
        int hi = n - 1;
        while (hi > 0 && e[hi - 1] == 0.0) --hi;
        if (hi == 0) return 0;
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
            rk.push_back(k);
            rc.push_back(c);
            rs.push_back(s);
        }
    }
}

}  // namespace msc
