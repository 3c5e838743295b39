// mp_stencil.cu -- batched PHS-RBF-FD stencil weights on sm_100a.
//
// Each stencil system is the saddle matrix of
// calc_PHS_RBF_grad_laplace_single_vert_A (coefficient_computations.cpp:70-106)
//     A = [[Phi, P], [P^T, 0]],  Phi_ij = r_ij^phs (0 on the diagonal),
//     P_ij = prod_d x_id^e_jd   (anisotropically scaled coordinates, :33-68)
// with the dim+1 right-hand sides of :108-292 (d/dx, d/dy, [d/dz], Laplacian of
// the basis at the centre node 0).  The weights are the first n rows of the
// solution (:311-323).  Interpolation mode (calc_interp_matrix, :456-518) has one
// right-hand side instead: the basis evaluated at a probe point that is shifted
// and scaled with its stencil (calc_PHS_RBF_interp_single_vert_rhs, :430-454).
//
// Weights kernel: one thread per matrix row, the augmented row [A_i | B_i]
// held in registers; Gauss-Jordan with partial pivoting.  At step k every
// row's column-k entry sits in register a[0] (rows shift left by one each
// step), so no register is ever indexed dynamically.  The pivot row is
// broadcast through shared memory; pivot rows are not normalised, so their
// diagonal value is kept and divided out at the end.  Rows are not swapped:
// the thread that pivoted at step k ends up holding solution row k.
//
// Condition kernel: the reference reports 1/rcond of Eigen's PartialPivLU
// (:312), i.e. the Hager/Higham estimate of ||A^-1||_1 from an LU with
// partial pivoting.  To reproduce those numbers the estimator needs the LU
// factors, so this kernel factorises A in shared memory (one warp per system,
// row swaps as in the reference, first max |a| wins) and runs the estimator.
#include <cmath>
#include "mp_common.cuh"

namespace mp {

constexpr int MAX_DIM = 3;
constexpr int MAX_M = 20;     // monomials (3D degree 3)
constexpr int MAX_S = 96;     // n + m

struct StencilJob {
    // point source: cloud mode (xyz + nb_col, fixed n) or batch mode (pts + offsets + sizes)
    const double *xyz;
    const int *nb_col;
    int n_fixed;
    const double *pts;
    const int64_t *offsets;
    const int *sizes;
    const int *list;  // systems of this size class (batch mode); nullptr = identity
    int count;        // systems to process
    int dim, m, phs;
    // outputs
    double *w0, *w1, *w2, *w3;  // cloud mode: per-operator arrays (nv*n)
    double *wb;                  // batch mode: (dim+1)*offsets[i]
    double *cond;
    int *singular;               // count of singular systems
    unsigned int *queue;         // persistent work counter
    const double *probe;         // interpolation mode: probe point of each system (count x dim)
};

__constant__ int c_exps[MAX_M * MAX_DIM];

__device__ __forceinline__ int sys_id(const StencilJob &J, int t) { return J.list ? J.list[t] : t; }
__device__ __forceinline__ int sys_n(const StencilJob &J, int id) {
    return J.nb_col ? J.n_fixed : J.sizes[id];
}
__device__ __forceinline__ const double *sys_point(const StencilJob &J, int id, int n, int k) {
    if (J.nb_col)
        return J.xyz + (size_t)J.nb_col[(size_t)id * n + k] * J.dim;
    return J.pts + (size_t)(J.offsets[id] + k) * J.dim;
}

// r^q for odd q from r^2
__device__ __forceinline__ double rpow_odd(double r2, int q) {
    double r = sqrt(r2);
    if (q == -1)
        return 1.0 / r;
    double v = r;
    for (int i = 1; i < q; i += 2)
        v *= r2;
    return v;
}

__device__ __forceinline__ double ipow(double x, int e) {
    double v = 1.0;
    for (int i = 0; i < e; i++)
        v *= x;
    return v;
}

__device__ __forceinline__ double monomial(const double *x, int j, int dim) {
    double t = ipow(x[0], c_exps[j * dim]);
    for (int d = 1; d < dim; d++)
        t *= ipow(x[d], c_exps[j * dim + d]);
    return t;
}

// Entry (r, j) of the augmented system [A | B] for a stencil with n nodes whose
// scaled coordinates are in sp (n x dim) and per-axis scales in sc.
__device__ double aug_entry(int r, int j, int n, int m, int dim, int phs, const double *sp,
                            const double *sc, const double *xp = nullptr) {
    const int S = n + m;
    if (j < S) {
        if (r < n && j < n) {
            if (r == j)
                return 0.0;
            double r2 = 0.0;
            for (int d = 0; d < dim; d++) {
                double t = sp[r * dim + d] - sp[j * dim + d];
                r2 += t * t;
            }
            return rpow_odd(r2, phs);
        }
        if (r < n)
            return monomial(sp + r * dim, j - n, dim);
        if (j < n)
            return monomial(sp + j * dim, r - n, dim);
        return 0.0;
    }
    if (xp) {  // interpolation: r^phs to the scaled probe, monomials at it (:430-454)
        if (r < n) {
            double r2 = 0.0;
            for (int d = 0; d < dim; d++) {
                double t = sp[r * dim + d] - xp[d];
                r2 += t * t;
            }
            return rpow_odd(r2, phs);
        }
        return monomial(xp, r - n, dim);
    }
    const int c = j - S;  // rhs column: 0..dim-1 gradient, dim Laplacian
    const double *x0 = sp;  // centre = local node 0
    if (r < n) {
        double r2 = 0.0;
        for (int d = 0; d < dim; d++) {
            double t = sp[r * dim + d] - x0[d];
            r2 += t * t;
        }
        if (c < dim)  // :124-125
            return -phs * (sp[r * dim + c] - x0[c]) * rpow_odd(r2, phs - 2) / sc[c];
        if (!(fabs(r2) > 1e-14))  // :229
            return 0.0;
        double acc = 0.0, rq4 = rpow_odd(r2, phs - 4), rq2 = rpow_odd(r2, phs - 2);
        for (int d = 0; d < dim; d++) {  // :231-248
            double dk = sp[r * dim + d] - x0[d];
            double g = phs * phs * (dk * dk) * rq4;
            g = g - 2.0 * phs * (dk * dk) * rq4;
            g = g + phs * rq2;
            acc += g / (sc[d] * sc[d]);
        }
        return acc;
    }
    const int p = r - n;
    const int *e = c_exps + p * dim;
    if (c < dim) {  // :128-140 and siblings
        if (e[c] <= 0)
            return 0.0;
        double t = e[c] * ipow(x0[c], e[c] - 1);
        for (int d = 0; d < dim; d++)
            if (d != c)
                t *= ipow(x0[d], e[d]);
        return t / sc[c];
    }
    double acc = 0.0;  // :252-289
    for (int k = 0; k < dim; k++) {
        if (e[k] > 1) {
            double t = e[k] * (e[k] - 1.0) * ipow(x0[k], e[k] - 2);
            for (int d = 0; d < dim; d++)
                if (d != k)
                    t *= ipow(x0[d], e[d]);
            acc += t / (sc[k] * sc[k]);
        }
    }
    return acc;
}

// Load a stencil's points into shared memory and apply shifting_scaling
// (coefficient_computations.cpp:33-68).  Executed by one group of `nt`
// threads (tid = thread index in the group); `sync` synchronises the group.
template <class Sync>
__device__ void load_scaled_points(const StencilJob &J, int id, int n, double *sp, double *sc,
                                   int tid, int nt, Sync sync) {
    const int dim = J.dim;
    for (int k = tid; k < n; k += nt) {
        const double *p = sys_point(J, id, n, k);
        for (int d = 0; d < dim; d++)
            sp[k * dim + d] = p[d];
    }
    sync();
    if (tid < 32) {
        double lo[MAX_DIM], hi[MAX_DIM];
        for (int d = 0; d < dim; d++) {
            lo[d] = sp[d];
            hi[d] = sp[d];
        }
        for (int k = tid; k < n; k += 32)
            for (int d = 0; d < dim; d++) {
                lo[d] = fmin(lo[d], sp[k * dim + d]);
                hi[d] = fmax(hi[d], sp[k * dim + d]);
            }
        for (int d = 0; d < dim; d++) {
            for (int o = 16; o > 0; o >>= 1) {
                lo[d] = fmin(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
                hi[d] = fmax(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
            }
        }
        if (tid == 0)
            for (int d = 0; d < dim; d++) {
                sc[d] = hi[d] - lo[d];
                sc[MAX_DIM + d] = lo[d];
            }
    }
    sync();
    for (int k = tid; k < n * dim; k += nt) {
        int d = k % dim;
        sp[k] = (sp[k] - sc[MAX_DIM + d]) / sc[d];
    }
    sync();
}

// -------------------------------------------------------------- weights
// Shared memory per group: points (MAX_S*3) + scales (6) + pivot row (W)
// + argmax slots (2*G) + matrix staging (S*(LD)).
template <int G, int W> struct GJShape {
    static constexpr int NT = 32 * G;
    static constexpr int GROUPS = (G == 1) ? 4 : 1;  // independent groups per CTA
    static constexpr int CTA = NT * GROUPS;
    static constexpr int SMAX = W - 3;               // rows available (R >= 3)
    static constexpr int LD = (W % 2) ? W : W + 1;   // odd leading dim: conflict-free row loads
    static constexpr int PTS = SMAX * MAX_DIM;
    static constexpr int DOUBLES = PTS + 3 * MAX_DIM + W + 2 * G + SMAX * LD;
};

template <int G, int W>
__global__ void __launch_bounds__(GJShape<G, W>::CTA)
    stencil_gj_kernel(StencilJob J) {
    using Sh = GJShape<G, W>;
    extern __shared__ double smem_raw[];
    const int grp = threadIdx.x / Sh::NT, tid = threadIdx.x % Sh::NT;
    const int lane = threadIdx.x & 31, warp_in_grp = tid >> 5;
    double *base = smem_raw + grp * Sh::DOUBLES;
    // sc: scales, minima, scaled probe (interpolation mode)
    double *sp = base, *sc = sp + Sh::PTS, *prow = sc + 3 * MAX_DIM;
    double *amax = prow + W;
    double *mat = amax + 2 * G;
    auto sync = [&]() {
        if (G == 1)
            __syncwarp();
        else
            __syncthreads();
    };
    const int dim = J.dim, m = J.m, R = J.probe ? 1 : dim + 1;
    double *xp = J.probe ? sc + 2 * MAX_DIM : nullptr;
    __shared__ int s_item[Sh::GROUPS];
    for (;;) {
        if (tid == 0)
            s_item[grp] = (int)atomicAdd(J.queue, 1u);
        sync();
        const int t = s_item[grp];
        sync();
        if (t >= J.count)
            break;
        const int id = sys_id(J, t);
        const int n = sys_n(J, id), S = n + m, SR = S + R;
        load_scaled_points(J, id, n, sp, sc, tid, Sh::NT, sync);
        if (xp) {  // the probe shifted and scaled with its stencil (:23-30)
            if (tid < dim)
                xp[tid] = (J.probe[(size_t)id * dim + tid] - sc[MAX_DIM + tid]) / sc[tid];
            sync();
        }
        for (int q = tid; q < S * SR; q += Sh::NT) {
            int r = q / SR, j = q - r * SR;
            mat[r * Sh::LD + j] = aug_entry(r, j, n, m, dim, J.phs, sp, sc, xp);
        }
        sync();
        double a[W];
        const bool live = tid < S;
#pragma unroll
        for (int j = 0; j < W; j++)
            a[j] = (live && j < SR) ? mat[tid * Sh::LD + j] : 0.0;
        bool eligible = live;
        int my_step = -1;
        double my_diag = 1.0;
        bool singular = false;
        for (int k = 0; k < S; k++) {
            // ---- pivot: largest |a[0]| among rows not yet used, lowest row on ties
            double cand = eligible ? fabs(a[0]) : -1.0;
            double mx = cand;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            unsigned ball = __ballot_sync(0xffffffffu, cand == mx);
            int p;
            if (G == 1) {
                p = __ffs(ball) - 1;
            } else {
                if (lane == 0) {
                    amax[warp_in_grp] = mx;
                    amax[G + warp_in_grp] = (double)(warp_in_grp * 32 + __ffs(ball) - 1);
                }
                __syncthreads();
                double best = amax[0];
                p = (int)amax[G];
#pragma unroll
                for (int g = 1; g < G; g++)
                    if (amax[g] > best) {
                        best = amax[g];
                        p = (int)amax[G + g];
                    }
                mx = best;
            }
            if (tid == p) {
#pragma unroll
                for (int j = 0; j < W; j++)
                    prow[j] = a[j];
                eligible = false;
                my_step = k;
                my_diag = a[0];
            }
            sync();
            const double piv = prow[0];
            if (!(mx > 0.0))
                singular = true;
            const double l = (tid == p) ? 0.0 : a[0] / piv;
#pragma unroll
            for (int j = 0; j < W - 1; j++)
                a[j] = fma(-l, prow[j + 1], a[j + 1]);
            a[W - 1] = 0.0;
            sync();
        }
        // ---- results: thread that pivoted at step k holds solution row k
        if (my_step >= 0 && my_step < n) {
            const double inv = 1.0 / my_diag;
            if (J.probe) {
                J.w0[(size_t)id * n + my_step] = a[0] * inv;
            } else if (J.nb_col) {
                size_t o = (size_t)id * n + my_step;
                J.w0[o] = a[0] * inv;
                J.w1[o] = a[1] * inv;
                if (dim == 3) {
                    J.w2[o] = a[2] * inv;
                    J.w3[o] = a[3] * inv;
                } else {
                    J.w3[o] = a[2] * inv;
                }
            } else {
                double *wo = J.wb + (size_t)R * J.offsets[id];
#pragma unroll
                for (int c = 0; c < 4; c++)
                    if (c < R)
                        wo[c * n + my_step] = a[c] * inv;
            }
        }
        if (tid == 0 && singular)
            atomicAdd(J.singular, 1);
        sync();
    }
}

// ------------------------------------------------------- condition numbers
// One warp per system; A (S x S, leading dim LDA odd) in dynamic shared memory.
struct CondSmem {
    int lda, s_max;
    __host__ __device__ int doubles() const { return MAX_S * MAX_DIM + 2 * MAX_DIM + s_max * lda + 4 * s_max; }
};

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// x <- A^-1 x using the in-place LU (row-major, unit L) and row permutation.
__device__ void lu_solve_warp(const double *lu, int lda, const int *perm, int s, double *x,
                              double *t, int lane) {
    for (int i = lane; i < s; i += 32)
        t[i] = x[perm[i]];
    __syncwarp();
    for (int j = 0; j < s; j++) {  // L y = Pb, column oriented
        const double yj = t[j];
        for (int i = j + 1 + lane; i < s; i += 32)
            t[i] -= lu[i * lda + j] * yj;
        __syncwarp();
    }
    for (int j = s - 1; j >= 0; j--) {  // U x = y
        if (lane == 0)
            t[j] = t[j] / lu[j * lda + j];
        __syncwarp();
        const double xj = t[j];
        for (int i = lane; i < j; i += 32)
            t[i] -= lu[i * lda + j] * xj;
        __syncwarp();
    }
    for (int i = lane; i < s; i += 32)
        x[i] = t[i];
    __syncwarp();
}

// x <- A^-T x:  A^T = U^T L^T P
__device__ void lu_solve_t_warp(const double *lu, int lda, const int *perm, int s, double *x,
                                double *t, int lane) {
    for (int i = lane; i < s; i += 32)
        t[i] = x[i];
    __syncwarp();
    for (int j = 0; j < s; j++) {  // U^T w = b
        if (lane == 0)
            t[j] = t[j] / lu[j * lda + j];
        __syncwarp();
        const double wj = t[j];
        for (int i = j + 1 + lane; i < s; i += 32)
            t[i] -= lu[j * lda + i] * wj;
        __syncwarp();
    }
    for (int j = s - 1; j >= 0; j--) {  // L^T q = w
        const double qj = t[j];
        for (int i = lane; i < j; i += 32)
            t[i] -= lu[j * lda + i] * qj;
        __syncwarp();
    }
    for (int i = lane; i < s; i += 32)
        x[perm[i]] = t[i];
    __syncwarp();
}

__device__ double norm1_warp(const double *v, int s, int lane) {
    double a = 0.0;
    for (int i = lane; i < s; i += 32)
        a += fabs(v[i]);
    return warp_sum(a);
}

__global__ void __launch_bounds__(32) stencil_cond_kernel(StencilJob J, CondSmem L) {
    extern __shared__ double sm[];
    double *sp = sm, *sc = sp + MAX_S * MAX_DIM, *A = sc + 2 * MAX_DIM;
    double *v = A + L.s_max * L.lda, *t = v + L.s_max, *sg = t + L.s_max;
    int *perm = (int *)(sg + L.s_max);
    const int lane = threadIdx.x;
    auto sync = [] { __syncwarp(); };
    const int dim = J.dim, m = J.m, lda = L.lda;
    for (;;) {
        int tt = 0;
        if (lane == 0)
            tt = (int)atomicAdd(J.queue, 1u);
        tt = __shfl_sync(0xffffffffu, tt, 0);
        if (tt >= J.count)
            break;
        const int id = sys_id(J, tt);
        const int n = sys_n(J, id), s = n + m;
        load_scaled_points(J, id, n, sp, sc, lane, 32, sync);
        for (int q = lane; q < s * s; q += 32) {
            int r = q / s, j = q - r * s;
            A[r * lda + j] = aug_entry(r, j, n, m, dim, J.phs, sp, sc);
        }
        for (int i = lane; i < s; i += 32)
            perm[i] = i;
        __syncwarp();
        // ||A||_1 (max column sum)
        double anorm = 0.0;
        for (int j = lane; j < s; j += 32) {
            double cs = 0.0;
            for (int i = 0; i < s; i++)
                cs += fabs(A[i * lda + j]);
            anorm = fmax(anorm, cs);
        }
        anorm = warp_max(anorm);
        // LU with partial pivoting, first max |a| wins (row swaps as in the reference)
        bool sing = false;
        for (int k = 0; k < s; k++) {
            double best = -1.0;
            int bi = k;
            for (int i = k + lane; i < s; i += 32) {
                double a = fabs(A[i * lda + k]);
                if (a > best) {
                    best = a;
                    bi = i;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (bi != k) {
                for (int j = lane; j < s; j += 32) {
                    double x = A[k * lda + j];
                    A[k * lda + j] = A[bi * lda + j];
                    A[bi * lda + j] = x;
                }
                if (lane == 0) {
                    int x = perm[k];
                    perm[k] = perm[bi];
                    perm[bi] = x;
                }
            }
            __syncwarp();
            const double piv = A[k * lda + k];
            if (piv == 0.0) {
                sing = true;
                continue;
            }
            for (int i = k + 1 + lane; i < s; i += 32) {
                double l = A[i * lda + k] / piv;
                A[i * lda + k] = l;
                if (l != 0.0)
                    for (int j = k + 1; j < s; j++)
                        A[i * lda + j] -= l * A[k * lda + j];
            }
            __syncwarp();
        }
        double est = INFINITY;
        if (!sing) {
            // Hager (1984) / Higham (1988) estimate of ||A^-1||_1
            for (int i = lane; i < s; i += 32)
                v[i] = 1.0 / s;
            __syncwarp();
            lu_solve_warp(A, lda, perm, s, v, t, lane);
            est = norm1_warp(v, s, lane);
            if (s > 1) {
                for (int i = lane; i < s; i += 32)
                    sg[i] = v[i] >= 0.0 ? 1.0 : -1.0;
                __syncwarp();
                int jold = -1;
                double est_old = est;
                for (int it = 0; it < 5; it++) {
                    for (int i = lane; i < s; i += 32)
                        v[i] = sg[i];
                    __syncwarp();
                    lu_solve_t_warp(A, lda, perm, s, v, t, lane);
                    double bv = -1.0;
                    int bj = 0;
                    for (int i = lane; i < s; i += 32)
                        if (fabs(v[i]) > bv) {
                            bv = fabs(v[i]);
                            bj = i;
                        }
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        double ob = __shfl_xor_sync(0xffffffffu, bv, o);
                        int oj = __shfl_xor_sync(0xffffffffu, bj, o);
                        if (ob > bv || (ob == bv && oj < bj)) {
                            bv = ob;
                            bj = oj;
                        }
                    }
                    if (bj == jold)
                        break;
                    for (int i = lane; i < s; i += 32)
                        v[i] = (i == bj) ? 1.0 : 0.0;
                    __syncwarp();
                    lu_solve_warp(A, lda, perm, s, v, t, lane);
                    double e = norm1_warp(v, s, lane);
                    if (e <= est_old)
                        break;
                    est = e;
                    int changed = 0;
                    for (int i = lane; i < s; i += 32) {
                        double ns = v[i] >= 0.0 ? 1.0 : -1.0;
                        changed |= (ns != sg[i]);
                        sg[i] = ns;
                    }
                    __syncwarp();
                    if (!__any_sync(0xffffffffu, changed))
                        break;
                    jold = bj;
                    est_old = est;
                }
                for (int i = lane; i < s; i += 32)
                    v[i] = ((i & 1) ? -1.0 : 1.0) * (1.0 + (double)i / (double)(s - 1));
                __syncwarp();
                lu_solve_warp(A, lda, perm, s, v, t, lane);
                double ae = 2.0 * norm1_warp(v, s, lane) / (3.0 * s);
                est = fmax(est, ae);
            }
        }
        if (lane == 0)
            J.cond[id] = sing ? INFINITY : anorm * est;
        __syncwarp();
    }
}

// ------------------------------------------------------------ host side
static int upload_exponents(int dim, int poly_deg, int *m_out) {
    int m = mp_num_poly_terms(dim, poly_deg);
    if (m <= 0 || m > MAX_M)
        return fail(MP_BAD_ARG, "poly_deg %d in %dD gives %d monomials (max %d)", poly_deg, dim, m,
                    MAX_M);
    int e[MAX_M * MAX_DIM];
    MP_TRY(mp_poly_exponents(dim, poly_deg, e));
    MP_CUDA(cudaMemcpyToSymbol(c_exps, e, sizeof(int) * m * dim));
    *m_out = m;
    return MP_OK;
}

template <int G, int W> static int launch_gj(StencilJob J, cudaStream_t s) {
    using Sh = GJShape<G, W>;
    size_t smem = (size_t)Sh::DOUBLES * Sh::GROUPS * sizeof(double);
    auto k = stencil_gj_kernel<G, W>;
    MP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, Sh::CTA, smem));
    if (per_sm < 1)
        return fail(MP_CUDA_ERROR, "stencil kernel G=%d W=%d does not fit on an SM", G, W);
    int groups_needed = (J.count + Sh::GROUPS - 1) / Sh::GROUPS;
    int grid = sm_count() * per_sm;
    if (grid > groups_needed)
        grid = groups_needed;
    if (grid < 1)
        return MP_OK;
    MP_CUDA(cudaMemsetAsync(J.queue, 0, sizeof(unsigned int), s));
    k<<<grid, Sh::CTA, smem, s>>>(J);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// Size classes: G = ceil(S/32) warps (one row per thread) and a register
// row of width W = 32G + 4 >= S + dim + 1.
static int gj_class(int S, int R) {
    for (int c = 0; c < 3; c++) {
        const int G = c + 1;
        if (S <= 32 * G && S + R <= 32 * G + 4)
            return c;
    }
    return -1;
}

static int launch_class(int cls, const StencilJob &J, cudaStream_t s) {
    switch (cls) {
    case 0: return launch_gj<1, 36>(J, s);
    case 1: return launch_gj<2, 68>(J, s);
    case 2: return launch_gj<3, 100>(J, s);
    }
    return fail(MP_BAD_ARG, "stencil size class %d", cls);
}

static int launch_cond(StencilJob J, int s_max, cudaStream_t s) {
    CondSmem L;
    L.s_max = s_max;
    L.lda = s_max | 1;
    size_t smem = (size_t)L.doubles() * sizeof(double) + sizeof(int) * s_max;
    MP_CUDA(cudaFuncSetAttribute(stencil_cond_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    int per_sm = 0;
    MP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stencil_cond_kernel, 32, smem));
    if (per_sm < 1)
        return fail(MP_CUDA_ERROR, "condition kernel does not fit (s=%d)", s_max);
    int grid = sm_count() * per_sm;
    if (grid > J.count)
        grid = J.count;
    if (grid < 1)
        return MP_OK;
    MP_CUDA(cudaMemsetAsync(J.queue, 0, sizeof(unsigned int), s));
    stencil_cond_kernel<<<grid, 32, smem, s>>>(J, L);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// Scratch for a weights call: queue counter + singular counter
struct StencilScratch {
    dbuf<unsigned int> words;
    int get(unsigned int **queue, int **singular) {
        if (!words.p)
            MP_TRY(words.alloc(8));
        *queue = words.p;
        *singular = (int *)(words.p + 4);
        return MP_OK;
    }
};

int cloud_weights_device(const double *d_xyz, int nv, int dim, const int *d_nb, int n, int phs,
                         int poly_deg, double *gx, double *gy, double *gz, double *lap,
                         double *cond, cudaStream_t s) {
    if (nv <= 0 || n <= 1 || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_stencil_weights: nv=%d n=%d dim=%d", nv, n, dim);
    if (phs != 3 && phs != 5 && phs != 7 && phs != 9 && phs != 11)  // parameters.cpp:89-93
        return fail(MP_BAD_ARG, "phs_deg should be 3, 5, 7, 9 or 11; got %d", phs);
    if (dim == 3 && !gz)
        return fail(MP_BAD_ARG, "3D weights need a grad_z output");
    int m = 0;
    MP_TRY(upload_exponents(dim, poly_deg, &m));
    const int S = n + m, R = dim + 1;
    const int cls = gj_class(S, R);
    if (cls < 0)
        return fail(MP_BAD_ARG, "stencil system %d x %d exceeds the supported %d", S, S, MAX_S);
    StencilScratch scr;
    StencilJob J{};
    MP_TRY(scr.get(&J.queue, &J.singular));
    MP_CUDA(cudaMemsetAsync(J.singular, 0, sizeof(int), s));
    J.xyz = d_xyz;
    J.nb_col = d_nb;
    J.n_fixed = n;
    J.count = nv;
    J.dim = dim;
    J.m = m;
    J.phs = phs;
    J.w0 = gx;
    J.w1 = gy;
    J.w2 = gz;
    J.w3 = lap;
    J.cond = cond;
    MP_TRY(launch_class(cls, J, s));
    if (cond)
        MP_TRY(launch_cond(J, S, s));
    int bad = 0;
    MP_CUDA(cudaMemcpyAsync(&bad, J.singular, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (bad)
        return fail(MP_SINGULAR_STENCIL, "%d stencil systems had a zero pivot (duplicate nodes?)",
                    bad);
    return MP_OK;
}

// interpolation weights of np probes from their stencils nb (np x n) of cloud xyz
int interp_weights_device(const double *d_xyz, int dim, const double *d_probe, int np,
                          const int *d_nb, int n, int phs, int poly_deg, double *w,
                          cudaStream_t s) {
    if (np <= 0 || n <= 1 || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_interp_matrix: np=%d n=%d dim=%d", np, n, dim);
    if (phs != 3 && phs != 5 && phs != 7 && phs != 9 && phs != 11)
        return fail(MP_BAD_ARG, "phs_deg should be 3, 5, 7, 9 or 11; got %d", phs);
    int m = 0;
    MP_TRY(upload_exponents(dim, poly_deg, &m));
    const int cls = gj_class(n + m, 1);
    if (cls < 0)
        return fail(MP_BAD_ARG, "interpolation system %d x %d exceeds the supported %d", n + m,
                    n + m, MAX_S);
    StencilScratch scr;
    StencilJob J{};
    MP_TRY(scr.get(&J.queue, &J.singular));
    MP_CUDA(cudaMemsetAsync(J.singular, 0, sizeof(int), s));
    J.xyz = d_xyz;
    J.nb_col = d_nb;
    J.n_fixed = n;
    J.count = np;
    J.dim = dim;
    J.m = m;
    J.phs = phs;
    J.w0 = w;
    J.probe = d_probe;
    MP_TRY(launch_class(cls, J, s));
    int bad = 0;
    MP_CUDA(cudaMemcpyAsync(&bad, J.singular, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (bad)
        return fail(MP_SINGULAR_STENCIL, "%d interpolation systems had a zero pivot", bad);
    return MP_OK;
}

int knn_probe_device(const double *d_xyz, int nv, int dim, const double *d_probe, int np, int n,
                     int *d_nb, cudaStream_t s);

}  // namespace mp

using namespace mp;

extern "C" int mp_stencil_weights(const double *xyz, int nv, int dim, const int *nb_col, int n,
                                  int phs_deg, int poly_deg, double *gx, double *gy, double *gz,
                                  double *lap, double *cond, mp_stream s) {
    cudaStream_t st = S(s);
    if (!xyz || !nb_col || !gx || !gy || !lap)
        return fail(MP_BAD_ARG, "mp_stencil_weights: null argument");
    dbuf<double> txyz;
    dbuf<int> tnb;
    const double *dxyz = nullptr;
    const int *dnb = nullptr;
    MP_TRY(stage_in(xyz, (size_t)nv * dim, txyz, &dxyz, st));
    MP_TRY(stage_in(nb_col, (size_t)nv * n, tnb, &dnb, st));
    // outputs: device pointers written in place, host pointers staged back
    double *outs[5] = {gx, gy, gz, lap, cond};
    size_t cnt[5] = {(size_t)nv * n, (size_t)nv * n, (size_t)nv * n, (size_t)nv * n, (size_t)nv};
    dbuf<double> tmp[5];
    double *dev[5];
    for (int i = 0; i < 5; i++) {
        if (!outs[i] || (i == 2 && dim == 2)) {
            dev[i] = nullptr;
            continue;
        }
        if (is_device_ptr(outs[i])) {
            dev[i] = outs[i];
        } else {
            MP_TRY(tmp[i].alloc(cnt[i]));
            dev[i] = tmp[i].p;
        }
    }
    int st_ = cloud_weights_device(dxyz, nv, dim, dnb, n, phs_deg, poly_deg, dev[0], dev[1],
                                   dev[2], dev[3], dev[4], st);
    if (st_ != MP_OK && st_ != MP_SINGULAR_STENCIL)
        return st_;
    for (int i = 0; i < 5; i++)
        if (tmp[i].p)
            MP_CUDA(cudaMemcpyAsync(outs[i], tmp[i].p, cnt[i] * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return st_;
}

extern "C" int mp_stencil_weights_batched(int nsys, const int *sizes, const int64_t *offsets,
                                          const double *pts, int dim, int phs_deg, int poly_deg,
                                          double *w, double *cond, mp_stream s) {
    cudaStream_t st = S(s);
    if (nsys <= 0)
        return MP_OK;
    if (!sizes || !offsets || !pts || !w || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_stencil_weights_batched: bad arguments");
    if (phs_deg != 3 && phs_deg != 5 && phs_deg != 7 && phs_deg != 9 && phs_deg != 11)
        return fail(MP_BAD_ARG, "phs_deg should be 3, 5, 7, 9 or 11; got %d", phs_deg);
    int m = 0;
    MP_TRY(upload_exponents(dim, poly_deg, &m));
    const int R = dim + 1;
    // size classes are chosen on the host
    std::vector<int> hs(nsys);
    std::vector<int64_t> ho(nsys);
    MP_CUDA(cudaMemcpy(hs.data(), sizes, sizeof(int) * nsys, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(ho.data(), offsets, sizeof(int64_t) * nsys, cudaMemcpyDefault));
    int64_t npts = 0;
    int s_max = 0;
    std::vector<int> lists[3];
    for (int i = 0; i < nsys; i++) {
        if (hs[i] < 2)
            return fail(MP_BAD_ARG, "system %d has %d nodes", i, hs[i]);
        int c = gj_class(hs[i] + m, R);
        if (c < 0)
            return fail(MP_BAD_ARG, "system %d: %d nodes + %d monomials exceeds %d", i, hs[i], m,
                        MAX_S);
        lists[c].push_back(i);
        if (ho[i] + hs[i] > npts)
            npts = ho[i] + hs[i];
        if (hs[i] + m > s_max)
            s_max = hs[i] + m;
    }
    dbuf<int> dsizes, dlist[3];
    dbuf<int64_t> doff;
    dbuf<double> dpts, dw, dcond;
    const int *psz = nullptr;
    const int64_t *pof = nullptr;
    const double *ppts = nullptr;
    MP_TRY(stage_in(sizes, nsys, dsizes, &psz, st));
    MP_TRY(stage_in(offsets, nsys, doff, &pof, st));
    MP_TRY(stage_in(pts, (size_t)npts * dim, dpts, &ppts, st));
    double *pw = w, *pc = cond;
    if (!is_device_ptr(w)) {
        MP_TRY(dw.alloc((size_t)npts * R));
        pw = dw.p;
    }
    if (cond && !is_device_ptr(cond)) {
        MP_TRY(dcond.alloc(nsys));
        pc = dcond.p;
    }
    // one persistent launch per size class, the classes run concurrently
    cudaEvent_t ev_fork, ev_join[3];
    cudaStream_t side[3];
    MP_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    MP_CUDA(cudaEventRecord(ev_fork, st));
    StencilScratch scr[3];
    int bad_total = 0;
    int rc = MP_OK;
    int nside = 0;
    for (int c = 0; c < 3 && rc == MP_OK; c++) {
        if (lists[c].empty())
            continue;
        MP_TRY(dlist[c].alloc(lists[c].size()));
        MP_CUDA(cudaMemcpyAsync(dlist[c].p, lists[c].data(), sizeof(int) * lists[c].size(),
                                cudaMemcpyHostToDevice, st));
    }
    MP_CUDA(cudaEventRecord(ev_fork, st));
    for (int c = 0; c < 3; c++) {
        if (lists[c].empty())
            continue;
        MP_CUDA(cudaStreamCreateWithFlags(&side[nside], cudaStreamNonBlocking));
        MP_CUDA(cudaEventCreateWithFlags(&ev_join[nside], cudaEventDisableTiming));
        cudaStream_t ss = side[nside];
        MP_CUDA(cudaStreamWaitEvent(ss, ev_fork, 0));
        StencilJob J{};
        MP_TRY(scr[c].get(&J.queue, &J.singular));
        MP_CUDA(cudaMemsetAsync(J.singular, 0, sizeof(int), ss));
        J.pts = ppts;
        J.offsets = pof;
        J.sizes = psz;
        J.list = dlist[c].p;
        J.count = (int)lists[c].size();
        J.dim = dim;
        J.m = m;
        J.phs = phs_deg;
        J.wb = pw;
        J.cond = pc;
        rc = launch_class(c, J, ss);
        if (rc == MP_OK && cond) {
            StencilJob Jc = J;
            rc = launch_cond(Jc, s_max, ss);
        }
        MP_CUDA(cudaEventRecord(ev_join[nside], ss));
        MP_CUDA(cudaStreamWaitEvent(st, ev_join[nside], 0));
        nside++;
    }
    for (int c = 0; c < 3; c++) {
        if (lists[c].empty() || !scr[c].words.p)
            continue;
        int bad = 0;
        MP_CUDA(cudaMemcpyAsync(&bad, scr[c].words.p + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        bad_total += bad;
    }
    if (dw.p)
        MP_CUDA(cudaMemcpyAsync(w, dw.p, sizeof(double) * npts * R, cudaMemcpyDeviceToHost, st));
    if (dcond.p)
        MP_CUDA(cudaMemcpyAsync(cond, dcond.p, sizeof(double) * nsys, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < nside; i++) {
        cudaStreamDestroy(side[i]);
        cudaEventDestroy(ev_join[i]);
    }
    cudaEventDestroy(ev_fork);
    if (rc != MP_OK)
        return rc;
    if (bad_total)
        return fail(MP_SINGULAR_STENCIL, "%d stencil systems had a zero pivot", bad_total);
    return MP_OK;
}

extern "C" int mp_interp_matrix(const double *xyz, int nv, int dim, const double *probe, int np,
                                int n, int phs_deg, int poly_deg, int *cols, double *w,
                                mp_stream s) {
    cudaStream_t st = S(s);
    if (!xyz || !probe || !cols || !w || nv <= 0 || np <= 0)
        return fail(MP_BAD_ARG, "mp_interp_matrix: bad arguments");
    dbuf<double> tx, tp, tw;
    dbuf<int> tc;
    const double *dx = nullptr, *dp = nullptr;
    MP_TRY(stage_in(xyz, (size_t)nv * dim, tx, &dx, st));
    MP_TRY(stage_in(probe, (size_t)np * dim, tp, &dp, st));
    int *dc = cols;
    double *dw = w;
    const bool hc = !is_device_ptr(cols), hw = !is_device_ptr(w);
    if (hc) {
        MP_TRY(tc.alloc((size_t)np * n));
        dc = tc.p;
    }
    if (hw) {
        MP_TRY(tw.alloc((size_t)np * n));
        dw = tw.p;
    }
    MP_TRY(knn_probe_device(dx, nv, dim, dp, np, n, dc, st));
    const int rc = interp_weights_device(dx, dim, dp, np, dc, n, phs_deg, poly_deg, dw, st);
    if (rc != MP_OK && rc != MP_SINGULAR_STENCIL)
        return rc;
    if (hc)
        MP_CUDA(cudaMemcpyAsync(cols, dc, sizeof(int) * np * n, cudaMemcpyDeviceToHost, st));
    if (hw)
        MP_CUDA(cudaMemcpyAsync(w, dw, sizeof(double) * np * n, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return rc;
}
