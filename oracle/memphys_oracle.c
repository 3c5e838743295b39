/*
 * memphys_oracle.c -- CPU FP64 restatement of the MeMPhyS hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is what the tests compare the CUDA
 * product path (memphys_b200/csrc) against, and the CPU baseline that
 * bench.py times beside the GPU.  Nothing in the product links or calls it.
 *
 * Reference paths below are relative to "MeMPhyS Latest Version/" of
 * aakashvshah/MemPhys.  The reference needs Eigen 3.3.7, Spectra and HYPRE,
 * none of which are available, so the pieces it delegates to them are
 * restated from their published algorithms:
 *   - Eigen PartialPivLU: LU with partial (row) pivoting, first max |a| wins.
 *   - Eigen PartialPivLU::rcond: Hager (1984) / Higham (1988) 1-norm estimator
 *     of ||A^-1||_1, with Higham's alternating-sign safeguard.
 *   - Eigen BiCGSTAB: van der Vorst (1992) right-preconditioned BiCGSTAB with
 *     the stop test ||r||^2 <= tol^2 ||b||^2 and one restart when rho collapses.
 *   - Eigen IncompleteLUT: Saad (1994) ILUT(tau, p) dual-threshold ILU,
 *     without Eigen's AMD pre-permutation (iteration counts may differ; the
 *     converged solution to the same residual does not).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* ------------------------------------------------------------------ */
/* parameters.cpp:122-130 -- number of appended monomials and cloud size */
int mo_num_poly_terms(int dim, int poly_deg)
{
    if (dim == 2)
        return (int)(0.5 * (poly_deg + 1) * (poly_deg + 2));
    return (poly_deg + 1) * (poly_deg + 2) * (poly_deg + 3) / 6;
}

int mo_cloud_size(int dim, int poly_deg, double multiplier)
{
    return (int)ceil(multiplier * mo_num_poly_terms(dim, poly_deg));
}

/* parameters.cpp:217-267 -- monomial exponent table, row-major m x dim.
 * 2D order: 1, x, y, x^2, xy, y^2, x^3, x^2y, xy^2, y^3, ...
 * 3D order: 1, x, y, z, then each degree block is x*(previous block),
 * y*(the previous block's y/z-only tail), z^deg. */
void mo_poly_exponents(int dim, int poly_deg, int *e)
{
    int m = mo_num_poly_terms(dim, poly_deg);
    memset(e, 0, sizeof(int) * m * dim);
    for (int d = 0; d < dim; d++)
        e[(1 + d) * dim + d] = 1;
    int prev = 1;
    for (int deg = 2; deg <= poly_deg; deg++) {
        int nprev = (dim == 2) ? deg : deg * (deg + 1) / 2; /* size of block deg-1 */
        int base = prev + nprev;
        for (int i = prev; i < prev + nprev; i++) {
            int r = base + i - prev;
            for (int d = 0; d < dim; d++)
                e[r * dim + d] = e[i * dim + d];
            e[r * dim + 0] += 1;
        }
        if (dim == 2) {
            e[(base + deg) * 2 + 0] = 0;
            e[(base + deg) * 2 + 1] = deg;
        } else {
            for (int i = prev + deg * (deg - 1) / 2; i < prev + nprev; i++) {
                int r = base + i - prev + deg;
                for (int d = 0; d < 3; d++)
                    e[r * 3 + d] = e[i * 3 + d];
                e[r * 3 + 1] += 1;
            }
            int last = base + (deg + 1) * (deg + 2) / 2 - 1;
            e[last * 3 + 0] = 0;
            e[last * 3 + 1] = 0;
            e[last * 3 + 2] = deg;
        }
        prev = base;
    }
}

/* ------------------------------------------------------------------ */
/* Dense LU with partial pivoting (Eigen PartialPivLU semantics), row-major */
static int lu_factor(double *a, int n, int *perm)
{
    int info = 0;
    for (int i = 0; i < n; i++)
        perm[i] = i;
    for (int k = 0; k < n; k++) {
        int p = k;
        double best = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++) {
            double v = fabs(a[i * n + k]);
            if (v > best) {
                best = v;
                p = i;
            }
        }
        if (p != k) {
            for (int j = 0; j < n; j++) {
                double t = a[k * n + j];
                a[k * n + j] = a[p * n + j];
                a[p * n + j] = t;
            }
            int t = perm[k];
            perm[k] = perm[p];
            perm[p] = t;
        }
        double piv = a[k * n + k];
        if (piv == 0.0) {
            info = k + 1;
            continue;
        }
        for (int i = k + 1; i < n; i++) {
            double l = a[i * n + k] / piv;
            a[i * n + k] = l;
            if (l != 0.0)
                for (int j = k + 1; j < n; j++)
                    a[i * n + j] -= l * a[k * n + j];
        }
    }
    return info;
}

/* solve A x = b in place (b has nrhs columns, column-major n x nrhs) */
static void lu_solve(const double *lu, const int *perm, int n, double *b, int nrhs, double *tmp)
{
    for (int c = 0; c < nrhs; c++) {
        double *x = b + (size_t)c * n;
        for (int i = 0; i < n; i++)
            tmp[i] = x[perm[i]];
        for (int i = 0; i < n; i++) {
            double s = tmp[i];
            for (int j = 0; j < i; j++)
                s -= lu[i * n + j] * tmp[j];
            tmp[i] = s;
        }
        for (int i = n - 1; i >= 0; i--) {
            double s = tmp[i];
            for (int j = i + 1; j < n; j++)
                s -= lu[i * n + j] * tmp[j];
            tmp[i] = s / lu[i * n + i];
        }
        memcpy(x, tmp, sizeof(double) * n);
    }
}

/* solve A^T x = b in place: P A = L U  ->  A^T = U^T L^T P */
static void lu_solve_t(const double *lu, const int *perm, int n, double *x, double *tmp)
{
    for (int i = 0; i < n; i++) { /* U^T w = b */
        double s = x[i];
        for (int j = 0; j < i; j++)
            s -= lu[j * n + i] * tmp[j];
        tmp[i] = s / lu[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) { /* L^T q = w */
        double s = tmp[i];
        for (int j = i + 1; j < n; j++)
            s -= lu[j * n + i] * tmp[j];
        tmp[i] = s;
    }
    for (int i = 0; i < n; i++)
        x[perm[i]] = tmp[i];
}

static double norm1_vec(const double *v, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += fabs(v[i]);
    return s;
}

/* Hager/Higham estimate of ||A^-1||_1 from an LU factorisation. */
static double inv_norm1_estimate(const double *lu, const int *perm, int n)
{
    double *v = (double *)malloc(sizeof(double) * n);
    double *sg = (double *)malloc(sizeof(double) * n);
    double *sg_old = (double *)malloc(sizeof(double) * n);
    double *tmp = (double *)malloc(sizeof(double) * n);
    for (int i = 0; i < n; i++)
        v[i] = 1.0 / n;
    lu_solve(lu, perm, n, v, 1, tmp);
    double est = norm1_vec(v, n);
    if (n > 1) {
        for (int i = 0; i < n; i++)
            sg[i] = (v[i] >= 0.0) ? 1.0 : -1.0;
        int jold = -1;
        double est_old = est;
        for (int it = 0; it < 5; it++) {
            memcpy(v, sg, sizeof(double) * n);
            lu_solve_t(lu, perm, n, v, tmp);
            int j = 0;
            for (int i = 1; i < n; i++)
                if (fabs(v[i]) > fabs(v[j]))
                    j = i;
            if (j == jold)
                break;
            memset(v, 0, sizeof(double) * n);
            v[j] = 1.0;
            lu_solve(lu, perm, n, v, 1, tmp);
            double e = norm1_vec(v, n);
            if (e <= est_old)
                break;
            est = e;
            memcpy(sg_old, sg, sizeof(double) * n);
            int same = 1;
            for (int i = 0; i < n; i++) {
                sg[i] = (v[i] >= 0.0) ? 1.0 : -1.0;
                if (sg[i] != sg_old[i])
                    same = 0;
            }
            if (same)
                break;
            jold = j;
            est_old = est;
        }
        double alt = 1.0;
        for (int i = 0; i < n; i++) {
            v[i] = alt * (1.0 + (double)i / (double)(n - 1));
            alt = -alt;
        }
        lu_solve(lu, perm, n, v, 1, tmp);
        double ae = 2.0 * norm1_vec(v, n) / (3.0 * n);
        if (ae > est)
            est = ae;
    }
    free(v);
    free(sg);
    free(sg_old);
    free(tmp);
    return est;
}

/* ------------------------------------------------------------------ */
/* coefficient_computations.cpp:33-68 -- anisotropic shift/scale to [0,1] */
static void shifting_scaling(double *vert, int nv, int dim, double *scale)
{
    double mn[3], mx[3];
    for (int i = 0; i < dim; i++)
        mn[i] = mx[i] = vert[i];
    for (int iv = 0; iv < nv; iv++)
        for (int i = 0; i < dim; i++) {
            double v = vert[dim * iv + i];
            if (mn[i] > v)
                mn[i] = v;
            if (mx[i] < v)
                mx[i] = v;
        }
    for (int i = 0; i < dim; i++)
        scale[i] = mx[i] - mn[i];
    for (int iv = 0; iv < nv; iv++)
        for (int i = 0; i < dim; i++)
            vert[dim * iv + i] = (vert[dim * iv + i] - mn[i]) / scale[i];
}

/*
 * coefficient_computations.cpp:70-328 -- PHS-RBF-FD weights of one stencil.
 * vert_in: n x dim coordinates (row 0 = the centre node), unscaled.
 * w: (dim+1) x n output: grad_x, grad_y, [grad_z], laplacian weights.
 * cond_est: 1/rcond as Eigen's PartialPivLU::rcond reports it (estimate).
 * cond_exact (nullable): exact ||A||_1 ||A^-1||_1.
 * Returns 0, or k+1 if pivot k was exactly zero (singular system).
 */
int mo_stencil_single(const double *vert_in, int n, int dim, int phs, int m, const int *e,
                      double *w, double *cond_est, double *cond_exact)
{
    int s = n + m, R = dim + 1;
    double scale[3];
    double *vert = (double *)malloc(sizeof(double) * n * dim);
    memcpy(vert, vert_in, sizeof(double) * n * dim);
    shifting_scaling(vert, n, dim, scale);
    double *A = (double *)calloc((size_t)s * s, sizeof(double));
    double *rhs = (double *)calloc((size_t)s * R, sizeof(double)); /* column-major */
    /* :75-89 RBF block, symmetric, zero diagonal */
    for (int ir = 0; ir < n; ir++)
        for (int ic = ir + 1; ic < n; ic++) {
            double r2 = 0.0;
            for (int i = 0; i < dim; i++) {
                double d = vert[dim * ir + i] - vert[dim * ic + i];
                r2 = r2 + d * d;
            }
            double rp = pow(r2, (double)(phs / 2.0));
            A[ir * s + ic] = rp;
            A[ic * s + ir] = rp;
        }
    /* :90-102 polynomial blocks */
    for (int ir = 0; ir < n; ir++)
        for (int j = 0; j < m; j++) {
            double t = pow(vert[dim * ir], e[j * dim + 0]);
            for (int i = 1; i < dim; i++)
                t = t * pow(vert[dim * ir + i], e[j * dim + i]);
            A[ir * s + n + j] = t;
            A[(n + j) * s + ir] = t;
        }
    const double *c = vert; /* centre node = local node 0 */
    /* :108-211 first-derivative right-hand sides */
    for (int k = 0; k < dim; k++) {
        double *col = rhs + (size_t)k * s;
        for (int ir = 0; ir < n; ir++) {
            double r2 = 0.0;
            for (int i = 0; i < dim; i++) {
                double d = vert[dim * ir + i] - c[i];
                r2 = r2 + d * d;
            }
            double rp = -phs * (vert[dim * ir + k] - c[k]) * pow(r2, (double)((phs - 2.0) / 2.0));
            col[ir] = rp / scale[k];
        }
        for (int j = 0; j < m; j++) {
            const int *ej = e + j * dim;
            if (ej[k] > 0) {
                double t;
                if (k == 0) {
                    t = ej[0] * pow(c[0], ej[0] - 1.0);
                    t = t * pow(c[1], ej[1]);
                    if (dim == 3)
                        t = t * pow(c[2], ej[2]);
                } else if (k == 1) {
                    t = pow(c[0], ej[0]);
                    t = t * ej[1] * pow(c[1], ej[1] - 1.0);
                    if (dim == 3)
                        t = t * pow(c[2], ej[2]);
                } else {
                    t = ej[2] * pow(c[2], ej[2] - 1.0);
                    t = t * pow(c[0], ej[0]);
                    t = t * pow(c[1], ej[1]);
                }
                col[n + j] = t / scale[k];
            }
        }
    }
    /* :213-292 Laplacian right-hand side */
    {
        double *col = rhs + (size_t)dim * s;
        for (int ir = 0; ir < n; ir++) {
            double r2 = 0.0;
            for (int i = 0; i < dim; i++) {
                double d = vert[dim * ir + i] - c[i];
                r2 = r2 + d * d;
            }
            if (fabs(r2) > 1E-14) {
                double acc = 0.0;
                for (int k = 0; k < dim; k++) {
                    double dk = vert[dim * ir + k] - c[k];
                    double g = phs * phs * pow(dk, 2.0) * pow(r2, (double)((phs - 4.0) / 2.0));
                    g = g - 2.0 * phs * pow(dk, 2.0) * pow(r2, (double)((phs - 4.0) / 2.0));
                    g = g + phs * pow(r2, (double)((phs - 2.0) / 2.0));
                    g = g / (scale[k] * scale[k]);
                    acc = (k == 0) ? g : acc + g;
                }
                col[ir] = acc;
            }
        }
        for (int j = 0; j < m; j++) {
            const int *ej = e + j * dim;
            double gxx = 0.0, gyy = 0.0, gzz = 0.0;
            if (ej[0] > 1) {
                gxx = ej[0] * (ej[0] - 1.0) * pow(c[0], ej[0] - 2.0);
                gxx = gxx * pow(c[1], ej[1]);
                if (dim == 3)
                    gxx = gxx * pow(c[2], ej[2]);
                gxx = gxx / (scale[0] * scale[0]);
            }
            if (ej[1] > 1) {
                gyy = ej[1] * (ej[1] - 1.0) * pow(c[1], ej[1] - 2.0);
                gyy = gyy * pow(c[0], ej[0]);
                if (dim == 3)
                    gyy = gyy * pow(c[2], ej[2]);
                gyy = gyy / (scale[1] * scale[1]);
            }
            if (dim == 3 && ej[2] > 1) {
                gzz = ej[2] * (ej[2] - 1.0) * pow(c[2], ej[2] - 2.0);
                gzz = gzz * pow(c[0], ej[0]);
                gzz = gzz * pow(c[1], ej[1]);
                gzz = gzz / (scale[2] * scale[2]);
            }
            col[n + j] = gxx + gyy + gzz;
        }
    }
    /* :311-312 answer = A.partialPivLu().solve(rhs); cond = 1/rcond */
    double anorm = 0.0;
    for (int j = 0; j < s; j++) {
        double cs = 0.0;
        for (int i = 0; i < s; i++)
            cs += fabs(A[i * s + j]);
        if (cs > anorm)
            anorm = cs;
    }
    int *perm = (int *)malloc(sizeof(int) * s);
    double *tmp = (double *)malloc(sizeof(double) * s);
    int info = lu_factor(A, s, perm);
    if (info == 0) {
        lu_solve(A, perm, s, rhs, R, tmp);
        /* :313-323 weights = first n rows of each solution column */
        for (int k = 0; k < R; k++)
            for (int i = 0; i < n; i++)
                w[k * n + i] = rhs[(size_t)k * s + i];
        if (cond_est)
            *cond_est = anorm * inv_norm1_estimate(A, perm, s);
        if (cond_exact) {
            double *inv = (double *)calloc((size_t)s * s, sizeof(double));
            for (int i = 0; i < s; i++)
                inv[(size_t)i * s + i] = 1.0;
            lu_solve(A, perm, s, inv, s, tmp);
            double in1 = 0.0;
            for (int j = 0; j < s; j++) {
                double cs = norm1_vec(inv + (size_t)j * s, s);
                if (cs > in1)
                    in1 = cs;
            }
            *cond_exact = anorm * in1;
            free(inv);
        }
    } else {
        for (int k = 0; k < R * n; k++)
            w[k] = NAN;
        if (cond_est)
            *cond_est = INFINITY;
        if (cond_exact)
            *cond_exact = INFINITY;
    }
    free(perm);
    free(tmp);
    free(A);
    free(rhs);
    free(vert);
    return info;
}

/*
 * cloud.cpp:207-279 -- CLOUD::calc_grad_laplace_coeffs, non-periodic branch.
 * Weights are written in CSR order aligned with nb_col (cloud.cpp:251-258).
 * gz may be NULL in 2D; cond_est / cond_exact may be NULL.
 * Returns the number of singular stencils.
 */
int mo_cloud_weights(const double *xyz, int nv, int dim, const int *nb_row, const int *nb_col,
                     int phs, int poly_deg, double *gx, double *gy, double *gz, double *lap,
                     double *cond_est, double *cond_exact)
{
    int m = mo_num_poly_terms(dim, poly_deg);
    int *e = (int *)malloc(sizeof(int) * m * dim);
    mo_poly_exponents(dim, poly_deg, e);
    int bad = 0, nmax = 0;
    for (int iv = 0; iv < nv; iv++)
        if (nb_row[iv + 1] - nb_row[iv] > nmax)
            nmax = nb_row[iv + 1] - nb_row[iv];
    double *vert = (double *)malloc(sizeof(double) * nmax * dim);
    double *w = (double *)malloc(sizeof(double) * nmax * (dim + 1));
    for (int iv = 0; iv < nv; iv++) {
        int b = nb_row[iv], n = nb_row[iv + 1] - b;
        for (int k = 0; k < n; k++)
            for (int i = 0; i < dim; i++)
                vert[k * dim + i] = xyz[(size_t)nb_col[b + k] * dim + i];
        double ce = 0.0, cx = 0.0;
        int info = mo_stencil_single(vert, n, dim, phs, m, e, w, &ce, cond_exact ? &cx : NULL);
        if (info)
            bad++;
        for (int k = 0; k < n; k++) {
            gx[b + k] = w[0 * n + k];
            gy[b + k] = w[1 * n + k];
            if (dim == 3 && gz)
                gz[b + k] = w[2 * n + k];
            lap[b + k] = w[dim * n + k];
        }
        if (cond_est)
            cond_est[iv] = ce;
        if (cond_exact)
            cond_exact[iv] = cx;
    }
    free(vert);
    free(w);
    free(e);
    return bad;
}

/*
 * Independent stencils of uneven size (batched benchmark workload).
 * pts: concatenated n_i x dim coordinates, offsets[i] = first point of system i.
 * w: concatenated (dim+1) x n_i weights at woff[i] = (dim+1) * offsets[i].
 */
int mo_batched_weights(int nsys, const int *sizes, const long long *offsets, const double *pts,
                       int dim, int phs, int poly_deg, double *w, double *cond_exact)
{
    int m = mo_num_poly_terms(dim, poly_deg);
    int *e = (int *)malloc(sizeof(int) * m * dim);
    mo_poly_exponents(dim, poly_deg, e);
    int bad = 0;
    for (int i = 0; i < nsys; i++) {
        double cx = 0.0;
        int info = mo_stencil_single(pts + offsets[i] * dim, sizes[i], dim, phs, m, e,
                                     w + (dim + 1) * offsets[i], NULL, cond_exact ? &cx : NULL);
        if (info)
            bad++;
        if (cond_exact)
            cond_exact[i] = cx;
    }
    free(e);
    return bad;
}

/* ------------------------------------------------------------------ */
/*
 * cloud.cpp:570-648 -- CLOUD::calc_cloud_points_fast stencil rule.
 * Interior node: its n nearest nodes of the whole cloud (itself first).
 * Boundary node: itself, then its n-1 nearest INTERIOR nodes (boundary nodes
 * are placed at infinity in the second KD-tree, cloud.cpp:596-601).
 * Neighbours are sorted by distance, ties by node index.  Exact search on a
 * uniform bucket grid (nanoflann's KD-tree returns the same sets).
 */
typedef struct {
    double d;
    int i;
} knn_item;

int mo_knn_stencils(const double *xyz, const unsigned char *bflag, int nv, int dim, int n,
                    int *nb_col)
{
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++)
        lo[d] = hi[d] = xyz[d];
    for (int i = 0; i < nv; i++)
        for (int d = 0; d < dim; d++) {
            double v = xyz[(size_t)i * dim + d];
            if (v < lo[d])
                lo[d] = v;
            if (v > hi[d])
                hi[d] = v;
        }
    double vol = 1.0;
    for (int d = 0; d < dim; d++)
        vol *= (hi[d] - lo[d]) > 0 ? (hi[d] - lo[d]) : 1.0;
    double cell = pow(vol * 2.0 / nv, 1.0 / dim); /* ~2 points per cell */
    int g[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) {
        g[d] = (int)((hi[d] - lo[d]) / cell) + 1;
        if (g[d] < 1)
            g[d] = 1;
    }
    long long ncell = (long long)g[0] * g[1] * g[2];
    int *head = (int *)malloc(sizeof(int) * (ncell + 1));
    int *cnt = (int *)calloc(ncell + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * nv);
    long long *cid = (long long *)malloc(sizeof(long long) * nv);
    for (int i = 0; i < nv; i++) {
        long long c = 0;
        for (int d = dim - 1; d >= 0; d--) {
            int k = (int)((xyz[(size_t)i * dim + d] - lo[d]) / cell);
            if (k >= g[d])
                k = g[d] - 1;
            c = c * g[d] + k;
        }
        cid[i] = c;
        cnt[c]++;
    }
    head[0] = 0;
    for (long long c = 0; c < ncell; c++)
        head[c + 1] = head[c] + cnt[c];
    memset(cnt, 0, sizeof(int) * (ncell + 1));
    for (int i = 0; i < nv; i++)
        order[head[cid[i]] + cnt[cid[i]]++] = i;
    knn_item *best = (knn_item *)malloc(sizeof(knn_item) * (n + 1));
    int fail = 0;
    for (int q = 0; q < nv; q++) {
        const double *xq = xyz + (size_t)q * dim;
        int isb = bflag[q] != 0;
        int want = isb ? n - 1 : n;
        int qc[3] = {0, 0, 0};
        for (int d = 0; d < dim; d++) {
            qc[d] = (int)((xq[d] - lo[d]) / cell);
            if (qc[d] >= g[d])
                qc[d] = g[d] - 1;
        }
        int cnt_b = 0;
        for (int R = 0;; R++) {
            int lo3[3] = {0, 0, 0}, hi3[3] = {0, 0, 0};
            for (int d = 0; d < dim; d++) {
                lo3[d] = qc[d] - R;
                hi3[d] = qc[d] + R;
            }
            for (int cz = lo3[2]; cz <= hi3[2]; cz++)
                for (int cy = lo3[1]; cy <= hi3[1]; cy++)
                    for (int cx = lo3[0]; cx <= hi3[0]; cx++) {
                        /* only the shell of ring R */
                        int on = (cx == lo3[0] || cx == hi3[0] || cy == lo3[1] || cy == hi3[1] ||
                                  (dim == 3 && (cz == lo3[2] || cz == hi3[2])));
                        if (!on)
                            continue;
                        if (cx < 0 || cx >= g[0] || cy < 0 || cy >= g[1] || cz < 0 || cz >= g[2])
                            continue;
                        long long c = ((long long)cz * g[1] + cy) * g[0] + cx;
                        for (int t = head[c]; t < head[c + 1]; t++) {
                            int j = order[t];
                            if (isb && bflag[j])
                                continue;
                            double dd = 0.0;
                            for (int d = 0; d < dim; d++) {
                                double df = xyz[(size_t)j * dim + d] - xq[d];
                                dd += df * df;
                            }
                            if (cnt_b == want && (dd > best[want - 1].d ||
                                                  (dd == best[want - 1].d && j > best[want - 1].i)))
                                continue;
                            int pos = cnt_b < want ? cnt_b++ : want - 1;
                            while (pos > 0 && (best[pos - 1].d > dd ||
                                               (best[pos - 1].d == dd && best[pos - 1].i > j))) {
                                best[pos] = best[pos - 1];
                                pos--;
                            }
                            best[pos].d = dd;
                            best[pos].i = j;
                        }
                    }
            double reach = R * cell;
            int covered = 1;
            for (int d = 0; d < dim; d++)
                if (qc[d] - R > 0 || qc[d] + R < g[d] - 1)
                    covered = 0;
            if (cnt_b == want && best[want - 1].d <= reach * reach)
                break;
            if (covered)
                break;
        }
        if (cnt_b < want) {
            fail++;
            continue;
        }
        int *out = nb_col + (size_t)q * n;
        if (isb) {
            out[0] = q;
            for (int k = 0; k < n - 1; k++)
                out[k + 1] = best[k].i;
        } else {
            for (int k = 0; k < n; k++)
                out[k] = best[k].i;
        }
    }
    free(best);
    free(head);
    free(cnt);
    free(order);
    free(cid);
    return fail;
}

/* ------------------------------------------------------------------ */
/* Row-parallel loops on host threads (pthreads): the rows [0, n) are split into
 * one contiguous range per thread; every row is computed exactly as in the
 * serial loop, so results do not depend on the thread count.  Dot products and
 * the ILUT triangular solves stay serial, as in Eigen. */
static int g_threads = 1;
#define MO_MAX_THREADS 128

typedef void (*mo_rows_fn)(void *ctx, int lo, int hi);
typedef struct {
    mo_rows_fn fn;
    void *ctx;
    int lo, hi;
} mo_rows_job;

static void *mo_rows_worker(void *a)
{
    mo_rows_job *j = (mo_rows_job *)a;
    j->fn(j->ctx, j->lo, j->hi);
    return NULL;
}

static void par_rows(int n, mo_rows_fn fn, void *ctx)
{
    int T = g_threads;
    if (T > n / 2048)
        T = n / 2048;
    if (T <= 1) {
        fn(ctx, 0, n);
        return;
    }
    pthread_t th[MO_MAX_THREADS];
    int started[MO_MAX_THREADS];
    mo_rows_job job[MO_MAX_THREADS];
    const int chunk = (n + T - 1) / T;
    for (int t = 0; t < T; t++) {
        job[t].fn = fn;
        job[t].ctx = ctx;
        job[t].lo = t * chunk < n ? t * chunk : n;
        job[t].hi = (t + 1) * chunk < n ? (t + 1) * chunk : n;
        started[t] = t > 0 && pthread_create(&th[t], NULL, mo_rows_worker, &job[t]) == 0;
    }
    fn(ctx, job[0].lo, job[0].hi);
    for (int t = 1; t < T; t++) {
        if (started[t])
            pthread_join(th[t], NULL);
        else
            fn(ctx, job[t].lo, job[t].hi); /* no thread: run the range here */
    }
}

/* Threads of the row-parallel loops (SpMV rows, fractional-step row loops);
 * returns the previous count. */
int mo_set_threads(int n)
{
    const int old = g_threads;
    if (n > 0)
        g_threads = n < MO_MAX_THREADS ? n : MO_MAX_THREADS;
    return old;
}

/* ------------------------------------------------------------------ */
/* CSR helpers */
typedef struct {
    const int *rp, *ci;
    const double *val, *x;
    double *y;
} mo_spmv_ctx;

static void spmv_rows(void *c, int lo, int hi)
{
    const mo_spmv_ctx *a = (const mo_spmv_ctx *)c;
    for (int i = lo; i < hi; i++) {
        double s = 0.0;
        for (int k = a->rp[i]; k < a->rp[i + 1]; k++)
            s += a->val[k] * a->x[a->ci[k]];
        a->y[i] = s;
    }
}

void mo_spmv_csr(int nrows, const int *rp, const int *ci, const double *val, const double *x,
                 double *y)
{
    mo_spmv_ctx c = {rp, ci, val, x, y};
    par_rows(nrows, spmv_rows, &c);
}

/*
 * solver.cpp:165-214 -- SOLVER::calc_coeff_matrix.  Fixed-width stencils
 * (n per row, nb_col row-major).  Interior rows: diff*L + conv*(Gx+Gy[+Gz])
 * + unsteady on the diagonal; Dirichlet boundary rows: identity; Neumann
 * boundary rows: normal . grad.  If bordered, column nv and row nv are all
 * ones with (nv,nv)=0 (the regularisation of solver.cpp:205-213).
 * Output CSR with columns in stencil order then the border; the caller
 * allocates rp[nv+2], ci and val of size nv*n + 2*nv + 1.
 * Returns the number of rows (nv or nv+1).
 */
int mo_ppe_assemble(int nv, int dim, int n, const int *nb_col, const double *gx,
                    const double *gy, const double *gz, const double *lap,
                    const unsigned char *bflag, const unsigned char *dirichlet,
                    const double *normal, double unsteady, double conv, double diff,
                    int bordered, int *rp, int *ci, double *val)
{
    int nnz = 0;
    rp[0] = 0;
    for (int iv = 0; iv < nv; iv++) {
        const int *cols = nb_col + (size_t)iv * n;
        size_t b = (size_t)iv * n;
        if (bflag[iv]) {
            if (dirichlet[iv]) {
                ci[nnz] = iv;
                val[nnz++] = 1.0;
            } else {
                for (int k = 0; k < n; k++) {
                    double v = normal[dim * iv] * gx[b + k] + normal[dim * iv + 1] * gy[b + k];
                    if (dim == 3)
                        v += normal[dim * iv + 2] * gz[b + k];
                    ci[nnz] = cols[k];
                    val[nnz++] = v;
                }
            }
        } else {
            for (int k = 0; k < n; k++) {
                double v = diff * lap[b + k];
                v += conv * gx[b + k];
                v += conv * gy[b + k];
                if (dim == 3)
                    v += conv * gz[b + k];
                if (cols[k] == iv)
                    v += unsteady;
                ci[nnz] = cols[k];
                val[nnz++] = v;
            }
        }
        if (bordered) {
            ci[nnz] = nv;
            val[nnz++] = 1.0;
        }
        rp[iv + 1] = nnz;
    }
    if (bordered) {
        for (int iv = 0; iv < nv; iv++) {
            ci[nnz] = iv;
            val[nnz++] = 1.0;
        }
        ci[nnz] = nv;
        val[nnz++] = 0.0;
        rp[nv + 1] = nnz;
        return nv + 1;
    }
    return nv;
}

/* ------------------------------------------------------------------ */
/* ILUT(tau, p) -- Saad, "ILUT: a dual threshold incomplete LU factorization"
 * (1994).  Row-wise IKJ elimination with a dense work row.  Rows of L (unit
 * diagonal, stored strictly lower) and U (diagonal first). */
typedef struct {
    int n;
    int *lp, *li;
    double *lv;
    int *up, *ui;
    double *uv;
} mo_ilut;

static int cmp_abs_desc(const void *a, const void *b)
{
    double x = fabs(((const knn_item *)a)->d), y = fabs(((const knn_item *)b)->d);
    return (x < y) - (x > y);
}

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

mo_ilut *mo_ilut_create(int n, const int *rp, const int *ci, const double *val, double tau, int p)
{
    mo_ilut *f = (mo_ilut *)calloc(1, sizeof(mo_ilut));
    f->n = n;
    size_t capL = (size_t)n * (p + 1) + 16, capU = (size_t)n * (p + 2) + 16;
    f->lp = (int *)malloc(sizeof(int) * (n + 1));
    f->up = (int *)malloc(sizeof(int) * (n + 1));
    f->li = (int *)malloc(sizeof(int) * capL);
    f->lv = (double *)malloc(sizeof(double) * capL);
    f->ui = (int *)malloc(sizeof(int) * capU);
    f->uv = (double *)malloc(sizeof(double) * capU);
    double *w = (double *)calloc(n, sizeof(double));
    char *nzf = (char *)calloc(n, 1);
    int *nzl = (int *)malloc(sizeof(int) * n);
    knn_item *buf = (knn_item *)malloc(sizeof(knn_item) * n);
    int *heap = (int *)malloc(sizeof(int) * n);
    f->lp[0] = f->up[0] = 0;
    size_t nl = 0, nu = 0;
    for (int i = 0; i < n; i++) {
        int cntnz = 0;
        double rn = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; k++) {
            int j = ci[k];
            if (!nzf[j]) {
                nzf[j] = 1;
                nzl[cntnz++] = j;
            }
            w[j] += val[k];
            rn += val[k] * val[k];
        }
        rn = sqrt(rn / (rp[i + 1] - rp[i] > 0 ? rp[i + 1] - rp[i] : 1));
        double thr = tau * rn;
        /* process lower entries in increasing column order (min-heap by sort) */
        int nh = 0;
        for (int t = 0; t < cntnz; t++)
            if (nzl[t] < i)
                heap[nh++] = nzl[t];
        qsort(heap, nh, sizeof(int), cmp_int);
        int hp = 0;
        while (hp < nh) {
            int k = heap[hp++];
            double wk = w[k] / f->uv[f->up[k]];
            if (fabs(wk) < thr) {
                w[k] = 0.0;
                continue;
            }
            w[k] = wk;
            for (int t = f->up[k] + 1; t < f->up[k + 1]; t++) {
                int j = f->ui[t];
                if (!nzf[j]) {
                    nzf[j] = 1;
                    nzl[cntnz++] = j;
                    if (j < i) { /* keep heap sorted: insert */
                        int pos = nh++;
                        while (pos > hp && heap[pos - 1] > j) {
                            heap[pos] = heap[pos - 1];
                            pos--;
                        }
                        heap[pos] = j;
                    }
                }
                w[j] -= wk * f->uv[t];
            }
        }
        /* gather L part: keep p largest */
        int cl = 0, cu = 0;
        double diag = w[i];
        for (int t = 0; t < cntnz; t++) {
            int j = nzl[t];
            if (j < i && w[j] != 0.0 && fabs(w[j]) >= thr) {
                buf[cl].d = w[j];
                buf[cl].i = j;
                cl++;
            }
        }
        if (cl > p) {
            qsort(buf, cl, sizeof(knn_item), cmp_abs_desc);
            cl = p;
        }
        for (int t = 0; t < cl; t++) {
            f->li[nl] = buf[t].i;
            f->lv[nl++] = buf[t].d;
        }
        f->lp[i + 1] = (int)nl;
        for (int t = 0; t < cntnz; t++) {
            int j = nzl[t];
            if (j > i && fabs(w[j]) >= thr && w[j] != 0.0) {
                buf[cu].d = w[j];
                buf[cu].i = j;
                cu++;
            }
        }
        if (cu > p) {
            qsort(buf, cu, sizeof(knn_item), cmp_abs_desc);
            cu = p;
        }
        if (diag == 0.0)
            diag = (tau > 0 ? tau : 1e-4) * (rn > 0 ? rn : 1.0);
        f->ui[nu] = i;
        f->uv[nu++] = diag;
        for (int t = 0; t < cu; t++) {
            f->ui[nu] = buf[t].i;
            f->uv[nu++] = buf[t].d;
        }
        f->up[i + 1] = (int)nu;
        for (int t = 0; t < cntnz; t++) {
            w[nzl[t]] = 0.0;
            nzf[nzl[t]] = 0;
        }
    }
    free(w);
    free(nzf);
    free(nzl);
    free(buf);
    free(heap);
    return f;
}

void mo_ilut_apply(const mo_ilut *f, const double *b, double *x)
{
    int n = f->n;
    for (int i = 0; i < n; i++) {
        double s = b[i];
        for (int t = f->lp[i]; t < f->lp[i + 1]; t++)
            s -= f->lv[t] * x[f->li[t]];
        x[i] = s;
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int t = f->up[i] + 1; t < f->up[i + 1]; t++)
            s -= f->uv[t] * x[f->ui[t]];
        x[i] = s / f->uv[f->up[i]];
    }
}

long long mo_ilut_nnz(const mo_ilut *f) { return (long long)f->lp[f->n] + f->up[f->n]; }

void mo_ilut_destroy(mo_ilut *f)
{
    if (!f)
        return;
    free(f->lp);
    free(f->li);
    free(f->lv);
    free(f->up);
    free(f->ui);
    free(f->uv);
    free(f);
}

/* ------------------------------------------------------------------ */
static double dot(const double *a, const double *b, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++)
        s += a[i] * b[i];
    return s;
}

/*
 * solver.cpp:337-350 -- Eigen BiCGSTAB<RowMajor, IncompleteLUT>::solveWithGuess,
 * restated from van der Vorst (1992), right-preconditioned.  precond may be
 * NULL (identity).  Returns iterations; *relres = ||b - A x|| / ||b||
 * recomputed from scratch as solver.cpp:342-343 logs it.
 */
int mo_bicgstab(int n, const int *rp, const int *ci, const double *val, const mo_ilut *precond,
                const double *b, double *x, double tol, int maxit, double *relres,
                double *recursive_relres)
{
    double *r = (double *)malloc(sizeof(double) * n), *r0 = (double *)malloc(sizeof(double) * n);
    double *p = (double *)calloc(n, sizeof(double)), *v = (double *)calloc(n, sizeof(double));
    double *y = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n);
    double *s = (double *)malloc(sizeof(double) * n), *t = (double *)malloc(sizeof(double) * n);
    mo_spmv_csr(n, rp, ci, val, x, r);
    for (int i = 0; i < n; i++)
        r[i] = b[i] - r[i];
    memcpy(r0, r, sizeof(double) * n);
    double r0_sq = dot(r0, r0, n), b_sq = dot(b, b, n);
    int it = 0;
    if (b_sq == 0.0) {
        memset(x, 0, sizeof(double) * n);
        if (relres)
            *relres = 0.0;
        if (recursive_relres)
            *recursive_relres = 0.0;
        free(r); free(r0); free(p); free(v); free(y); free(z); free(s); free(t);
        return 0;
    }
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    double tol2 = tol * tol * b_sq, eps = 2.220446049250313e-16, eps2 = eps * eps;
    int restarts = 0;
    while (dot(r, r, n) > tol2 && it < maxit) {
        double rho_old = rho;
        rho = dot(r0, r, n);
        if (fabs(rho) < eps2 * r0_sq) {
            mo_spmv_csr(n, rp, ci, val, x, r);
            for (int i = 0; i < n; i++)
                r[i] = b[i] - r[i];
            memcpy(r0, r, sizeof(double) * n);
            rho = r0_sq = dot(r, r, n);
            if (restarts++ == 0)
                it = 0;
        }
        double beta = (rho / rho_old) * (alpha / omega);
        for (int i = 0; i < n; i++)
            p[i] = r[i] + beta * (p[i] - omega * v[i]);
        if (precond)
            mo_ilut_apply(precond, p, y);
        else
            memcpy(y, p, sizeof(double) * n);
        mo_spmv_csr(n, rp, ci, val, y, v);
        alpha = rho / dot(r0, v, n);
        for (int i = 0; i < n; i++)
            s[i] = r[i] - alpha * v[i];
        if (precond)
            mo_ilut_apply(precond, s, z);
        else
            memcpy(z, s, sizeof(double) * n);
        mo_spmv_csr(n, rp, ci, val, z, t);
        double tt = dot(t, t, n);
        omega = tt > 0.0 ? dot(t, s, n) / tt : 0.0;
        for (int i = 0; i < n; i++) {
            x[i] += alpha * y[i] + omega * z[i];
            r[i] = s[i] - omega * t[i];
        }
        it++;
    }
    if (recursive_relres)
        *recursive_relres = sqrt(dot(r, r, n) / b_sq);
    if (relres) {
        mo_spmv_csr(n, rp, ci, val, x, r);
        double rr = 0.0;
        for (int i = 0; i < n; i++) {
            double d = r[i] - b[i];
            rr += d * d;
        }
        *relres = sqrt(rr / b_sq);
    }
    free(r); free(r0); free(p); free(v); free(y); free(z); free(s); free(t);
    return it;
}

/* ------------------------------------------------------------------ */
/*
 * fractional_step_1.cpp -- FRACTIONAL_STEP_1, hat-velocity projection.
 * The reference integrates 2D only (single_timestep_2d); dim==3 adds the w
 * component with the same steps (calc_vel_hat/calc_pressure/calc_vel_corr
 * extended by the z terms).
 */
typedef struct {
    int nv, dim, n, nsys, temporal_order, maxit, full_neumann;
    const int *nb_col;
    const double *g[3], *lap;
    const unsigned char *bflag, *vdir[3], *pdir;
    const double *normal;
    double rho, mu, dt, tol;
    int *rp, *ci;
    double *val;
    mo_ilut *ilu;
    double *hat[3], *src_old[3], *src_oldold[3], *psrc, *tmp;
} mo_fs1;

/* fractional_step_1.cpp:22-50 (ctor) + solver.cpp:14-79 (SOLVER::init for p) */
mo_fs1 *mo_fs1_create(int nv, int dim, int n, const int *nb_col, const double *gx,
                      const double *gy, const double *gz, const double *lap,
                      const unsigned char *bflag, const double *normal,
                      const unsigned char *u_dir, const unsigned char *v_dir,
                      const unsigned char *w_dir, const unsigned char *p_dir, double rho,
                      double mu, double dt, int temporal_order, double tol, int maxit,
                      double droptol, int fill, int use_ilut)
{
    mo_fs1 *f = (mo_fs1 *)calloc(1, sizeof(mo_fs1));
    f->nv = nv;
    f->dim = dim;
    f->n = n;
    f->nb_col = nb_col;
    f->g[0] = gx;
    f->g[1] = gy;
    f->g[2] = gz;
    f->lap = lap;
    f->bflag = bflag;
    f->normal = normal;
    f->vdir[0] = u_dir;
    f->vdir[1] = v_dir;
    f->vdir[2] = w_dir;
    f->pdir = p_dir;
    f->rho = rho;
    f->mu = mu;
    f->dt = dt;
    f->temporal_order = temporal_order;
    f->tol = tol;
    f->maxit = maxit;
    f->full_neumann = 1;
    for (int i = 0; i < nv; i++)
        if (bflag[i] && p_dir[i]) {
            f->full_neumann = 0;
            break;
        }
    size_t cap = (size_t)nv * n + 2 * (size_t)nv + 1;
    f->rp = (int *)malloc(sizeof(int) * (nv + 2));
    f->ci = (int *)malloc(sizeof(int) * cap);
    f->val = (double *)malloc(sizeof(double) * cap);
    f->nsys = mo_ppe_assemble(nv, dim, n, nb_col, gx, gy, gz, lap, bflag, p_dir, normal, 0.0, 0.0,
                              1.0, f->full_neumann, f->rp, f->ci, f->val);
    f->ilu = use_ilut ? mo_ilut_create(f->nsys, f->rp, f->ci, f->val, droptol, fill) : NULL;
    for (int d = 0; d < dim; d++) {
        f->hat[d] = (double *)calloc(nv, sizeof(double));
        f->src_old[d] = (double *)calloc(nv, sizeof(double));
        f->src_oldold[d] = (double *)calloc(nv, sizeof(double));
    }
    f->psrc = (double *)calloc(nv + 1, sizeof(double));
    f->tmp = (double *)calloc(nv + 1, sizeof(double));
    return f;
}

int mo_fs1_system_size(const mo_fs1 *f) { return f->nsys; }

static double row_dot(const mo_fs1 *f, const double *w, int iv, const double *x)
{
    const int *c = f->nb_col + (size_t)iv * f->n;
    const double *ww = w + (size_t)iv * f->n;
    double s = 0.0;
    for (int k = 0; k < f->n; k++)
        s += ww[k] * x[c[k]];
    return s;
}

/*
 * One step: vel (dim arrays of nv) and p (nsys entries) are advanced in place
 * from time level n to n+1.  it = timestep index (Euler at it == 0).
 * Returns BiCGSTAB iterations; relres = recomputed ||A p - b|| / ||b||.
 */
/* the row loops of one step, split over threads by par_rows */
typedef struct {
    const mo_fs1 *f;
    double **vel;
    double *p;
    int d;
} mo_step_ctx;

static void vel_src_rows(void *c, int lo, int hi)
{
    const mo_step_ctx *a = (const mo_step_ctx *)c;
    const mo_fs1 *f = a->f;
    const double *q = a->vel[a->d];
    for (int i = lo; i < hi; i++) {
        double conv = 0.0;
        for (int k = 0; k < f->dim; k++)
            conv += a->vel[k][i] * row_dot(f, f->g[k], i, q);
        double src = f->rho * (-conv) + f->mu * row_dot(f, f->lap, i, q);
        f->src_old[a->d][i] = src;
    }
}

static void p_rhs_rows(void *c, int lo, int hi)
{
    const mo_step_ctx *a = (const mo_step_ctx *)c;
    const mo_fs1 *f = a->f;
    const int dim = f->dim;
    for (int i = lo; i < hi; i++) {
        if (!f->bflag[i]) {
            double s = 0.0;
            for (int d = 0; d < dim; d++)
                s += row_dot(f, f->g[d], i, f->hat[d]);
            f->psrc[i] = s * f->rho / f->dt;
        } else if (f->pdir[i]) {
            f->psrc[i] = a->p[i];
        } else {
            double s = 0.0;
            for (int d = 0; d < dim; d++)
                s += (a->vel[d][i] - f->hat[d][i]) * f->normal[dim * i + d];
            f->psrc[i] = -f->rho * s / f->dt;
        }
    }
}

static void vel_corr_rows(void *c, int lo, int hi)
{
    const mo_step_ctx *a = (const mo_step_ctx *)c;
    const mo_fs1 *f = a->f;
    double *q = a->vel[a->d];
    for (int i = lo; i < hi; i++)
        q[i] = f->hat[a->d][i] - f->dt * row_dot(f, f->g[a->d], i, a->p) / f->rho;
}

int mo_fs1_step(mo_fs1 *f, double **vel, double *p, int it, double *relres)
{
    int nv = f->nv, dim = f->dim;
    double rho = f->rho, dt = f->dt;
    mo_step_ctx ctx = {f, vel, p, 0};
    /* calc_vel_hat :120-134 */
    for (int d = 0; d < dim; d++) {
        const double *q = vel[d];
        ctx.d = d;
        par_rows(nv, vel_src_rows, &ctx);
        for (int i = 0; i < nv; i++) {
            if (f->temporal_order == 1 || it == 0)
                f->hat[d][i] = q[i] + (dt / rho) * f->src_old[d][i];
            else
                f->hat[d][i] = q[i] + (dt / rho) * (1.5 * f->src_old[d][i] - 0.5 * f->src_oldold[d][i]);
        }
    }
    /* calc_pressure :136-151 */
    par_rows(nv, p_rhs_rows, &ctx);
    if (f->nsys == nv + 1)
        f->psrc[nv] = 0.0;
    int iters = mo_bicgstab(f->nsys, f->rp, f->ci, f->val, f->ilu, f->psrc, p, f->tol, f->maxit,
                            relres, NULL);
    /* calc_vel_corr :153-209 */
    for (int d = 0; d < dim; d++) {
        double *q = vel[d];
        for (int i = 0; i < nv; i++)
            f->tmp[i] = q[i]; /* u_old for Dirichlet copies */
        ctx.d = d;
        par_rows(nv, vel_corr_rows, &ctx);
        for (int i = 0; i < nv; i++) {
            if (!f->bflag[i] || f->pdir[i])
                continue;
            if (f->vdir[d][i]) {
                q[i] = f->tmp[i];
            } else {
                const int *c = f->nb_col + (size_t)i * f->n;
                double rhs = 0.0, diag = 0.0;
                for (int k = 0; k < f->n; k++) {
                    double cf = 0.0;
                    for (int e = 0; e < dim; e++)
                        cf += f->g[e][(size_t)i * f->n + k] * f->normal[dim * i + e];
                    if (c[k] == i)
                        diag = cf;
                    else
                        rhs -= cf * q[c[k]];
                }
                q[i] = rhs / diag;
            }
        }
    }
    /* extras :211-222 */
    if (f->temporal_order == 2)
        for (int d = 0; d < dim; d++)
            memcpy(f->src_oldold[d], f->src_old[d], sizeof(double) * nv);
    return iters;
}

void mo_fs1_destroy(mo_fs1 *f)
{
    if (!f)
        return;
    mo_ilut_destroy(f->ilu);
    free(f->rp);
    free(f->ci);
    free(f->val);
    for (int d = 0; d < f->dim; d++) {
        free(f->hat[d]);
        free(f->src_old[d]);
        free(f->src_oldold[d]);
    }
    free(f->psrc);
    free(f->tmp);
    free(f);
}
