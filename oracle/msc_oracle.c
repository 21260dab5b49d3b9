/*
 * msc_oracle.c -- CPU restatement of the reference close-coupling solve.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product (the multiscat_b200
 * package, its CUDA library or its C-ABI) links, loads or calls this file.
 * It is the checker that the GPU solver is compared against, and the timed
 * CPU baseline in bench.py.  It is serial on purpose: the reference solve is
 * single-threaded Fortran.
 *
 * What it restates (reference paths are relative to the multiscat project):
 *   - lib/multiscat_fortran/fortran/multiscat_gmres.f90
 *       build_preconditioner      :226-273  (H0 = T + diag Re V00, eig, factors)
 *       apply_upper_block         :620-639  (strict upper channel coupling)
 *       solve_lower_block         :641-687  (block Gauss-Seidel forward solve
 *                                            + Sherman-Morrison boundary term)
 *       apply_scattering_operator :452-475  (I + L^-1 U, optional Neumann)
 *       solve_gmres_system        :477-618  (unrestarted MGS GMRES, complex
 *                                            Givens, back-solve every step,
 *                                            3-step convergence window)
 *       compute_complex_givens_rotation :689-716
 *   - lib/multiscat_fortran/fortran/multiscat.f90:35 (eps from sig. figures)
 *   - lib/multiscat_fortran/fortran/diagsub.f90 (rs = tred2 + tql2): the
 *     symmetric eigensolver is restated here as Householder tridiagonalisation
 *     followed by implicit symmetric QR with Wilkinson shifts (the same
 *     mathematical decomposition; eigenvalues ascending, eigenvectors as
 *     columns).
 *
 * One generalisation: the channel list is explicit (storage position of each
 * channel in the nkx x nky coupling torus, in solve order).  With every grid
 * point listed in row-major (ix, iy) order this is exactly the Fortran
 * channel order (multiscat_gmres.f90:58-80); a shorter list sorted by
 * perpendicular kinetic difference restates the `n_channels` truncation of
 * multiscat/multiscat/_scipy.py:414-443.
 *
 * Layouts (C order): V[(ix*nky + iy)*nz + k] complex interleaved; state
 * psi[j*nz + k] complex interleaved (channel-major, z contiguous) which is the
 * Fortran scattered_state(nz, C) column-major layout.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double complex cplx;

/* ------------------------------------------------------------------------ */
/* Symmetric eigensolver: Householder tridiagonalisation + implicit QR.       */
/* A is n x n row-major symmetric (only read).  On return w[k] ascending and  */
/* Z[i*n + k] = component i of eigenvector k.  Returns 0 on success.          */
/* ------------------------------------------------------------------------ */
int msc_oracle_eigh(int n, const double *A, double *w, double *Z)
{
    double *a = (double *)malloc(sizeof(double) * (size_t)n * n);
    double *q = Z;
    double *v = (double *)malloc(sizeof(double) * n);
    double *p = (double *)malloc(sizeof(double) * n);
    double *e = (double *)calloc((size_t)n, sizeof(double));
    if (!a || !v || !p || !e) { free(a); free(v); free(p); free(e); return -1; }
    memcpy(a, A, sizeof(double) * (size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) q[i * n + j] = (i == j) ? 1.0 : 0.0;

    /* Reduce to tridiagonal: annihilate column k below the subdiagonal. */
    for (int k = 0; k + 2 < n; ++k) {
        int m = n - k - 1;            /* length of x = a[k+1.., k] */
        double xnorm = 0.0;
        for (int i = 0; i < m; ++i) { double t = a[(k + 1 + i) * n + k]; xnorm += t * t; }
        xnorm = sqrt(xnorm);
        if (xnorm == 0.0) continue;
        double x0 = a[(k + 1) * n + k];
        double alpha = (x0 >= 0.0) ? -xnorm : xnorm;
        for (int i = 0; i < m; ++i) v[i] = a[(k + 1 + i) * n + k];
        v[0] -= alpha;
        double vnorm = 0.0;
        for (int i = 0; i < m; ++i) vnorm += v[i] * v[i];
        vnorm = sqrt(vnorm);
        if (vnorm == 0.0) continue;
        for (int i = 0; i < m; ++i) v[i] /= vnorm;
        /* trailing block S = a[k+1.., k+1..]; S <- H S H with H = I - 2 v v^T */
        double K = 0.0;
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            const double *row = a + (size_t)(k + 1 + i) * n + (k + 1);
            for (int j = 0; j < m; ++j) s += row[j] * v[j];
            p[i] = s;
            K += v[i] * s;
        }
        for (int i = 0; i < m; ++i) p[i] -= K * v[i];      /* q = p - (v.p) v */
        for (int i = 0; i < m; ++i) {
            double *row = a + (size_t)(k + 1 + i) * n + (k + 1);
            for (int j = 0; j < m; ++j) row[j] -= 2.0 * (v[i] * p[j] + p[i] * v[j]);
        }
        a[(k + 1) * n + k] = alpha;
        a[k * n + (k + 1)] = alpha;
        for (int i = 1; i < m; ++i) { a[(k + 1 + i) * n + k] = 0.0; a[k * n + (k + 1 + i)] = 0.0; }
        /* Q <- Q H on columns k+1.. */
        for (int r = 0; r < n; ++r) {
            double *row = q + (size_t)r * n + (k + 1);
            double s = 0.0;
            for (int j = 0; j < m; ++j) s += row[j] * v[j];
            for (int j = 0; j < m; ++j) row[j] -= 2.0 * s * v[j];
        }
    }
    for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
    for (int i = 0; i + 1 < n; ++i) e[i] = a[(i + 1) * n + i];

    /* Implicit symmetric QR with Wilkinson shift on (w, e). */
    const double eps = 2.220446049250313e-16;
    int status = 0;
    long steps = 0, max_steps = 60L * n + 100;
    for (;;) {
        for (int i = 0; i + 1 < n; ++i)
            if (fabs(e[i]) <= eps * (fabs(w[i]) + fabs(w[i + 1]))) e[i] = 0.0;
        int hi = n - 1;
        while (hi > 0 && e[hi - 1] == 0.0) --hi;
        if (hi == 0) break;
        int lo = hi - 1;
        while (lo > 0 && e[lo - 1] != 0.0) --lo;
        if (++steps > max_steps) { status = 1; break; }
        double dd = 0.5 * (w[hi - 1] - w[hi]);
        double eh = e[hi - 1];
        double den = dd + (dd >= 0.0 ? 1.0 : -1.0) * hypot(dd, eh);
        double mu = w[hi] - eh * eh / den;
        double x = w[lo] - mu, z = e[lo];
        for (int k = lo; k < hi; ++k) {
            double r = hypot(x, z);
            double c = 1.0, s = 0.0;
            if (r != 0.0) { c = x / r; s = z / r; }
            if (k > lo) e[k - 1] = r;
            double dk = w[k], dk1 = w[k + 1], ek = e[k];
            w[k] = c * c * dk + 2.0 * c * s * ek + s * s * dk1;
            w[k + 1] = s * s * dk - 2.0 * c * s * ek + c * c * dk1;
            e[k] = c * s * (dk1 - dk) + (c * c - s * s) * ek;
            if (k + 1 < hi) {
                x = e[k];
                z = s * e[k + 1];
                e[k + 1] = c * e[k + 1];
            }
            for (int rr = 0; rr < n; ++rr) {
                double qa = q[rr * n + k], qb = q[rr * n + k + 1];
                q[rr * n + k] = c * qa + s * qb;
                q[rr * n + k + 1] = -s * qa + c * qb;
            }
        }
    }
    /* sort ascending (selection sort keeps it simple; n is a few hundred) */
    for (int i = 0; i < n - 1; ++i) {
        int kmin = i;
        for (int j = i + 1; j < n; ++j) if (w[j] < w[kmin]) kmin = j;
        if (kmin != i) {
            double t = w[i]; w[i] = w[kmin]; w[kmin] = t;
            for (int r = 0; r < n; ++r) { double u = q[r * n + i]; q[r * n + i] = q[r * n + kmin]; q[r * n + kmin] = u; }
        }
    }
    free(a); free(v); free(p); free(e);
    return status;
}

/* ------------------------------------------------------------------------ */
/* Operator data                                                             */
/* ------------------------------------------------------------------------ */
typedef struct {
    int nz, C, nkx, nky;
    const int *sx, *sy;        /* storage position of each channel */
    const cplx *V;             /* [nkx*nky][nz] */
    const double *pkd;         /* [C] */
    const cplx *wc;            /* [C] */
    double *lam;               /* [nz] eigenvalues of H0 */
    double *E;                 /* [nz*nz] E[k*nz + i] = comp k of eigvec i */
    double *f;                 /* [C][nz] preconditioner factors */
    cplx *ytmp;                /* [nz] */
} op_t;

static inline const cplx *tap(const op_t *op, int j, int i)
{
    int dx = ((op->sx[j] - op->sx[i]) % op->nkx + op->nkx) % op->nkx;
    int dy = ((op->sy[j] - op->sy[i]) % op->nky + op->nky) % op->nky;
    return op->V + (size_t)(dx * op->nky + dy) * op->nz;
}

/* multiscat_gmres.f90:226-273 */
static int build_preconditioner(op_t *op, const double *T)
{
    int n = op->nz;
    double *H = (double *)malloc(sizeof(double) * (size_t)n * n);
    if (!H) return -1;
    memcpy(H, T, sizeof(double) * (size_t)n * n);
    for (int k = 0; k < n; ++k) H[k * n + k] += creal(op->V[k]);   /* V(1,1,k): storage (0,0) */
    int st = msc_oracle_eigh(n, H, op->lam, op->E);
    free(H);
    if (st != 0) return -2;
    double *g = (double *)malloc(sizeof(double) * n);
    for (int j = 0; j < op->C; ++j) {
        double ce = op->pkd[j];
        for (int k = 0; k < n; ++k) g[k] = op->E[(n - 1) * n + k] / (ce + op->lam[k]);
        double *fj = op->f + (size_t)j * n;
        for (int k = 0; k < n; ++k) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += op->E[k * n + i] * g[i];
            fj[k] = s;
        }
    }
    free(g);
    return 0;
}

/* multiscat_gmres.f90:620-639: x_j <- sum_{i>j} V[(G_j - G_i) mod] x_i */
static void apply_upper_block(const op_t *op, cplx *x)
{
    int n = op->nz;
    for (int j = 0; j < op->C; ++j) {
        cplx *xj = x + (size_t)j * n;
        for (int k = 0; k < n; ++k) xj[k] = 0.0;
        for (int i = j + 1; i < op->C; ++i) {
            const cplx *v = tap(op, j, i);
            const cplx *xi = x + (size_t)i * n;
            for (int k = 0; k < n; ++k) xj[k] += v[k] * xi[k];
        }
    }
}

/* multiscat_gmres.f90:641-687 */
static void solve_lower_block(const op_t *op, cplx *x)
{
    int n = op->nz;
    cplx *y = op->ytmp;
    for (int j = 0; j < op->C; ++j) {
        cplx *xj = x + (size_t)j * n;
        for (int i = 0; i < j; ++i) {
            const cplx *v = tap(op, j, i);
            const cplx *xi = x + (size_t)i * n;
            for (int k = 0; k < n; ++k) xj[k] -= v[k] * xi[k];
        }
        double ce = op->pkd[j];
        for (int k = 0; k < n; ++k) {
            cplx s = 0.0;
            for (int l = 0; l < n; ++l) s += xj[l] * op->E[l * n + k];
            y[k] = s / (ce + op->lam[k]);
        }
        for (int k = 0; k < n; ++k) xj[k] = 0.0;
        for (int l = 0; l < n; ++l) {
            cplx yl = y[l];
            for (int k = 0; k < n; ++k) xj[k] += op->E[k * n + l] * yl;
        }
        const double *fj = op->f + (size_t)j * n;
        cplx fac = xj[n - 1] * op->wc[j] / (1.0 - fj[n - 1] * op->wc[j]);
        for (int k = 0; k < n; ++k) xj[k] += fac * fj[k];
    }
}

/* multiscat_gmres.f90:452-475 */
static void apply_scattering_operator(const op_t *op, int flag, cplx *x, cplx *y, size_t mn)
{
    memcpy(y, x, sizeof(cplx) * mn);
    apply_upper_block(op, x);
    solve_lower_block(op, x);
    for (size_t i = 0; i < mn; ++i) x[i] = y[i] + x[i];
    if (flag == 1) {
        memcpy(y, x, sizeof(cplx) * mn);
        apply_upper_block(op, x);
        solve_lower_block(op, x);
        for (size_t i = 0; i < mn; ++i) x[i] = y[i] - x[i];
    }
}

/* multiscat_gmres.f90:689-716 */
static void complex_givens(cplx *a, cplx *b, cplx *c, cplx *s)
{
    cplx rho = *b;
    double aa = cabs(*a), ab = cabs(*b);
    if (aa > ab) rho = *a;
    double scale = aa + ab;
    double r;
    if (scale == 0.0) {
        *c = 1.0; *s = 0.0; r = 0.0;
    } else {
        cplx as = *a / scale, bs = *b / scale;
        r = creal(as * conj(as) + bs * conj(bs));
        r = scale * sqrt(r);
        if (creal(rho) < 0.0) r = -r;
        *c = conj(*a / r);
        *s = *b / r;
    }
    cplx z = 1.0;
    if (aa > ab) z = *s;
    if (ab >= aa && cabs(*c) != 0.0) z = 1.0 / *c;
    *a = r;
    *b = z;
}

/*
 * Solve with the reference's GMRES (multiscat_gmres.f90:477-618).
 * Returns info: 0 converged, 1 not converged, <0 internal failure.
 */
int msc_oracle_solve(int flag, double eps, int maxiter, int window,
                     int nz, int C, int nkx, int nky,
                     const int *sx, const int *sy, int spec,
                     const double *V, const double *pkd, const double *wc,
                     const double *b_spec, const double *T,
                     double *psi_out, int *iterations, double *final_ratio)
{
    if (nz <= 0 || C <= 0 || nkx <= 0 || nky <= 0) return -10;
    if (spec < 0 || spec >= C) return -11;
    op_t op;
    op.nz = nz; op.C = C; op.nkx = nkx; op.nky = nky;
    op.sx = sx; op.sy = sy;
    op.V = (const cplx *)V; op.pkd = pkd; op.wc = (const cplx *)wc;
    size_t mn = (size_t)nz * C;
    op.lam = (double *)malloc(sizeof(double) * nz);
    op.E = (double *)malloc(sizeof(double) * (size_t)nz * nz);
    op.f = (double *)malloc(sizeof(double) * mn);
    op.ytmp = (cplx *)malloc(sizeof(cplx) * nz);
    cplx *x = (cplx *)malloc(sizeof(cplx) * mn);
    cplx *y = (cplx *)malloc(sizeof(cplx) * mn);
    int cap = 64;
    cplx *xx = (cplx *)malloc(sizeof(cplx) * mn * cap);
    int L = maxiter;
    cplx *h = (cplx *)calloc((size_t)(L + 2) * (L + 2), sizeof(cplx));
    cplx *g = (cplx *)calloc((size_t)L + 1, sizeof(cplx));
    cplx *zc = (cplx *)calloc((size_t)L + 1, sizeof(cplx));
    cplx *co = (cplx *)calloc((size_t)L + 1, sizeof(cplx));
    cplx *si = (cplx *)calloc((size_t)L + 1, sizeof(cplx));
    int info = 0;
    if (!op.lam || !op.E || !op.f || !op.ytmp || !x || !y || !xx || !h || !g || !zc || !co || !si) {
        info = -1; goto done;
    }
    if (build_preconditioner(&op, T) != 0) { info = -2; goto done; }
#define H(i, j) h[(size_t)(i) * (L + 2) + (j)]

    /* initial residual, :519-545 */
    for (size_t i = 0; i < mn; ++i) x[i] = 0.0;
    memcpy(xx, x, sizeof(cplx) * mn);
    memcpy(y, x, sizeof(cplx) * mn);
    apply_upper_block(&op, x);
    for (size_t i = 0; i < mn; ++i) x[i] = -x[i];
    x[(size_t)spec * nz + (nz - 1)] += b_spec[0] + I * b_spec[1];
    solve_lower_block(&op, x);
    for (size_t i = 0; i < mn; ++i) x[i] = x[i] - y[i];
    if (flag == 1) {
        memcpy(y, x, sizeof(cplx) * mn);
        apply_upper_block(&op, x);
        solve_lower_block(&op, x);
        for (size_t i = 0; i < mn; ++i) x[i] = y[i] - x[i];
    }
    double xnorm = 0.0;
    for (size_t i = 0; i < mn; ++i) xnorm += creal(conj(x[i]) * x[i]);
    xnorm = sqrt(xnorm);
    g[0] = xnorm;
    double r0 = xnorm > 2.2250738585072014e-308 ? xnorm : 2.2250738585072014e-308;

    int kconv = 0, kk = 0;
    double resid = xnorm;
    for (int k = 1; k <= L; ++k) {
        for (size_t i = 0; i < mn; ++i) x[i] = x[i] / xnorm;
        if (k + 1 > cap) {
            int ncap = cap * 2;
            if (ncap > L + 1) ncap = L + 1;
            cplx *nx = (cplx *)realloc(xx, sizeof(cplx) * mn * ncap);
            if (!nx) { info = -1; goto done; }
            xx = nx; cap = ncap;
        }
        memcpy(xx + (size_t)k * mn, x, sizeof(cplx) * mn);
        apply_scattering_operator(&op, flag, x, y, mn);
        for (int j = 1; j <= k; ++j) {
            const cplx *vj = xx + (size_t)j * mn;
            cplx hj = 0.0;
            for (size_t i = 0; i < mn; ++i) hj += conj(vj[i]) * x[i];
            H(j, k) = hj;
            for (size_t i = 0; i < mn; ++i) x[i] -= vj[i] * hj;
        }
        xnorm = 0.0;
        for (size_t i = 0; i < mn; ++i) xnorm += creal(conj(x[i]) * x[i]);
        xnorm = sqrt(xnorm);
        H(k + 1, k) = xnorm;
        for (int j = 1; j <= k - 1; ++j) {
            cplx temp = co[j] * H(j, k) + conj(si[j]) * H(j + 1, k);
            H(j + 1, k) = conj(co[j]) * H(j + 1, k) - si[j] * H(j, k);
            H(j, k) = temp;
        }
        complex_givens(&H(k, k), &H(k + 1, k), &co[k], &si[k]);
        g[k] = -si[k] * g[k - 1];
        g[k - 1] = co[k] * g[k - 1];
        for (int j = 1; j <= k; ++j) zc[j] = g[j - 1];
        for (int j = k; j >= 1; --j) {
            zc[j] = zc[j] / H(j, j);
            for (int i = 1; i <= j - 1; ++i) zc[i] -= H(i, j) * zc[j];
        }
        resid = cabs(g[k]);
        if (resid < eps * r0) ++kconv; else kconv = 0;
        kk = k;
        if (kconv == window || xnorm == 0.0) break;
    }
    /* solution, :600-606 (x0 = 0) */
    memcpy(x, xx, sizeof(cplx) * mn);
    for (int j = 1; j <= kk; ++j) {
        const cplx *vj = xx + (size_t)j * mn;
        cplx zj = zc[j];
        for (size_t i = 0; i < mn; ++i) x[i] += vj[i] * zj;
    }
    memcpy(psi_out, x, sizeof(cplx) * mn);
    if (iterations) *iterations = kk;
    if (final_ratio) *final_ratio = resid / r0;
    if (kconv < window && xnorm > 0.0) info = 1;
#undef H
done:
    free(op.lam); free(op.E); free(op.f); free(op.ytmp);
    free(x); free(y); free(xx); free(h); free(g); free(zc); free(co); free(si);
    return info;
}

/* Debug entry points mirroring the reference's debug_* routines. */
int msc_oracle_build_preconditioner(int nz, int C, int nkx, int nky, const double *V,
                                    const double *pkd, const double *T,
                                    double *lam, double *E, double *f)
{
    op_t op;
    memset(&op, 0, sizeof(op));
    op.nz = nz; op.C = C; op.nkx = nkx; op.nky = nky;
    op.V = (const cplx *)V; op.pkd = pkd;
    op.lam = lam; op.E = E; op.f = f;
    return build_preconditioner(&op, T);
}

int msc_oracle_apply_upper(int nz, int C, int nkx, int nky, const int *sx, const int *sy,
                           const double *V, double *x)
{
    op_t op;
    memset(&op, 0, sizeof(op));
    op.nz = nz; op.C = C; op.nkx = nkx; op.nky = nky; op.sx = sx; op.sy = sy;
    op.V = (const cplx *)V;
    apply_upper_block(&op, (cplx *)x);
    return 0;
}

int msc_oracle_solve_lower(int nz, int C, int nkx, int nky, const int *sx, const int *sy,
                           const double *V, const double *pkd, const double *wc,
                           const double *T, double *x)
{
    op_t op;
    op.nz = nz; op.C = C; op.nkx = nkx; op.nky = nky; op.sx = sx; op.sy = sy;
    op.V = (const cplx *)V; op.pkd = pkd; op.wc = (const cplx *)wc;
    op.lam = (double *)malloc(sizeof(double) * nz);
    op.E = (double *)malloc(sizeof(double) * (size_t)nz * nz);
    op.f = (double *)malloc(sizeof(double) * (size_t)nz * C);
    op.ytmp = (cplx *)malloc(sizeof(cplx) * nz);
    int st = build_preconditioner(&op, T);
    if (st == 0) solve_lower_block(&op, (cplx *)x);
    free(op.lam); free(op.E); free(op.f); free(op.ytmp);
    return st;
}
