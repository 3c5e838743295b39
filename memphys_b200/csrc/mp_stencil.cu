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
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>
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

// monomial j at x; ex: the exponent table (a shared-memory copy of c_exps: lanes of a
// warp read different monomials, which constant memory would serialise)
__device__ __forceinline__ double monomial(const double *x, int j, int dim, const int *ex) {
    double t = ipow(x[0], ex[j * dim]);
    for (int d = 1; d < dim; d++)
        t *= ipow(x[d], ex[j * dim + d]);
    return t;
}

// Layout of a stencil's scale record: per-axis scales, minima, the scaled probe
// (interpolation mode) and the reciprocal scales
constexpr int SC_SCALE = 0, SC_MIN = MAX_DIM, SC_PROBE = 2 * MAX_DIM, SC_INV = 3 * MAX_DIM;
constexpr int SC_DOUBLES = 5 * MAX_DIM;  // odd multiple of MAX_DIM: keeps the GJ layout's pairs aligned

// Entry (r, j) of the augmented system [A | B] for a stencil with n nodes whose
// scaled coordinates are in sp (n x dim) and scale record in sc (divisions by the
// scales are products with their reciprocals).
__device__ double aug_entry(int r, int j, int n, int m, int dim, int phs, const double *sp,
                            const double *sc, const int *ex, const double *xp = nullptr) {
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
            return monomial(sp + r * dim, j - n, dim, ex);
        if (j < n)
            return monomial(sp + j * dim, r - n, dim, ex);
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
        return monomial(xp, r - n, dim, ex);
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
            return -phs * (sp[r * dim + c] - x0[c]) * rpow_odd(r2, phs - 2) * sc[SC_INV + c];
        if (!(fabs(r2) > 1e-14))  // :229
            return 0.0;
        double acc = 0.0, rq4 = rpow_odd(r2, phs - 4), rq2 = rpow_odd(r2, phs - 2);
        for (int d = 0; d < dim; d++) {  // :231-248
            double dk = sp[r * dim + d] - x0[d];
            double g = phs * phs * (dk * dk) * rq4;
            g = g - 2.0 * phs * (dk * dk) * rq4;
            g = g + phs * rq2;
            acc += g * (sc[SC_INV + d] * sc[SC_INV + d]);
        }
        return acc;
    }
    const int p = r - n;
    const int *e = ex + p * dim;
    if (c < dim) {  // :128-140 and siblings
        if (e[c] <= 0)
            return 0.0;
        double t = e[c] * ipow(x0[c], e[c] - 1);
        for (int d = 0; d < dim; d++)
            if (d != c)
                t *= ipow(x0[d], e[d]);
        return t * sc[SC_INV + c];
    }
    double acc = 0.0;  // :252-289
    for (int k = 0; k < dim; k++) {
        if (e[k] > 1) {
            double t = e[k] * (e[k] - 1.0) * ipow(x0[k], e[k] - 2);
            for (int d = 0; d < dim; d++)
                if (d != k)
                    t *= ipow(x0[d], e[d]);
            acc += t * (sc[SC_INV + k] * sc[SC_INV + k]);
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
                sc[SC_SCALE + d] = hi[d] - lo[d];
                sc[SC_MIN + d] = lo[d];
                sc[SC_INV + d] = 1.0 / (hi[d] - lo[d]);
            }
    }
    sync();
    for (int k = tid; k < n * dim; k += nt) {
        int d = k % dim;
        sp[k] = (sp[k] - sc[SC_MIN + d]) * sc[SC_INV + d];
    }
    sync();
}

// -------------------------------------------------------------- weights
// One thread per matrix row of a group of G warps (S <= 32 G); GROUPS groups
// per CTA work on independent systems.  Shared memory per group (each region an
// even number of doubles, so the pivot rows start on 16-byte boundaries): points,
// the scale record, the monomials of every node, the node-pair table, the pivot
// rows, the cross-warp pivot candidates, each thread's right-hand sides.
constexpr int even2(int x) { return (x + 1) / 2 * 2; }
template <int G, int W, int GROUPS> struct GJShape {
    static constexpr int NT = 32 * G;
    static constexpr int CTA = NT * GROUPS;
    static constexpr int SMAX = W - 3;               // rows of a weights system (R >= 3)
    // nodes of any system of the class: S + R <= W and S <= 32 G with R >= 1, m >= 1
    static constexpr int NMAX = (NT < W - 1 ? NT : W - 1) - 1;
    static constexpr int NP = NMAX > SMAX ? NMAX : SMAX;  // point and monomial rows
    // two pivot-row buffers (alternating steps) of W + 2 doubles each: element e of
    // the pivot row sits at [e + 1], so elements 1, 2 / 3, 4 / ... are 16-byte pairs;
    // [0] holds the reciprocal of the pivot
    static constexpr int PROW = (W + 3) / 2 * 2;
    // the pair table r_ij^phs, packed upper triangle of up to NMAX nodes
    static constexpr int TRI = NMAX * (NMAX - 1) / 2;
    static constexpr int OFF_SC = even2(NP * MAX_DIM);
    static constexpr int OFF_PM = OFF_SC + even2(SC_DOUBLES);
    static constexpr int OFF_TRI = OFF_PM + even2(NP * MAX_M);
    static constexpr int OFF_PROW = OFF_TRI + even2(TRI);
    static constexpr int OFF_AMAX = OFF_PROW + 2 * PROW;
    static constexpr int OFF_RHS = OFF_AMAX + 4 * G;
    static constexpr int DOUBLES = even2(OFF_RHS + 4 * NT);
    // CTAs per SM the register allocation must allow (one-warp systems: 16 warps per
    // SM, two-warp systems: 10; the three-warp rows need their 255 registers)
    static constexpr int WARPS_TARGET = G == 1 ? 16 : (G == 2 ? 10 : 1);
    static constexpr int MINB = (WARPS_TARGET + G * GROUPS - 1) / (G * GROUPS);
    // steps per chunk of the elimination: within a chunk the update runs over the
    // chunk's first live width, so the unrolled code stays ~W^2 / (2 CH) long
    static constexpr int CH = W <= 56 ? 4 : (W <= 84 ? 8 : 16);
    static constexpr int NCH = (W - 1 + CH - 1) / CH;  // covers every S < W
};

// Index of the pair (i, j), i < j < n, in the packed upper triangle of an n-node
// stencil: row i holds j = i + 1 .. n - 1
__device__ __forceinline__ int tri_index(int i, int j, int n) {
    return i * n - i * (i + 1) / 2 + (j - i - 1);
}

// r_ij^phs of every node pair of the stencil, once per pair (the saddle matrix's
// Phi block is symmetric): the pairs spread evenly over the group's nt threads
// (consecutive packed indices per step of the loop), so every thread takes about
// n (n - 1) / (2 nt) of the roots instead of its row's n - 1.
__device__ __forceinline__ void pair_table(double *tri, int n, int dim, int phs, const double *sp,
                                           int tid, int nt) {
    const int np = n * (n - 1) / 2;
    if (tid >= np)
        return;
    int i = 0, j = tid + 1;  // pair number tid
    while (j >= n) {
        ++i;
        j = j - n + i + 1;
    }
    for (int q = tid; q < np; q += nt) {
        double r2 = 0.0;
        for (int d = 0; d < dim; d++) {
            const double t = sp[i * dim + d] - sp[j * dim + d];
            r2 = fma(t, t, r2);
        }
        tri[q] = rpow_odd(r2, phs);
        j += nt;  // pair number q + nt
        while (j >= n && i < n) {
            ++i;
            j = j - n + i + 1;
        }
    }
}

// The right-hand sides of node row r (:108-248): the basis' gradient and Laplacian
// at the centre node 0, with one root of r^2 for all columns (phs >= 3)
__device__ __forceinline__ void node_rhs(int r, int dim, int phs, const double *sp,
                                         const double *sc, double *rhs) {
    double r2 = 0.0, dk[MAX_DIM];
    for (int d = 0; d < dim; d++) {
        dk[d] = sp[r * dim + d] - sp[d];
        r2 += dk[d] * dk[d];
    }
    const double rt = sqrt(r2);
    // r^(phs - 2) and r^(phs - 4) for odd phs >= 3 from the one root, formed as
    // rpow_odd forms them (the same products in the same order)
    double rq2 = rt, rq4 = rt;
    for (int i = 1; i < phs - 2; i += 2)
        rq2 *= r2;
    if (phs == 3)
        rq4 = 1.0 / rt;
    else
        for (int i = 1; i < phs - 4; i += 2)
            rq4 *= r2;
    for (int c = 0; c < dim; c++)  // :124-125
        rhs[c] = -phs * dk[c] * rq2 * sc[SC_INV + c];
    double acc = 0.0;
    if (fabs(r2) > 1e-14) {  // :229
        for (int d = 0; d < dim; d++) {  // :231-248
            double g = phs * phs * (dk[d] * dk[d]) * rq4;
            g = g - 2.0 * phs * (dk[d] * dk[d]) * rq4;
            g = g + phs * rq2;
            acc += g * (sc[SC_INV + d] * sc[SC_INV + d]);
        }
    }
    rhs[dim] = acc;
}

// The row of a thread: entries j < W of [A | B] for row r (coefficient_computations
// .cpp:70-106 for A, :108-292 for B, :430-454 in interpolation mode), assembled in
// registers: node-node entries from the group's pair table, polynomial entries from
// its monomial table, the right-hand sides from their formulas.
template <int W>
__device__ __forceinline__ void assemble_row(double (&a)[W], int r, int n, int m, int S, int R,
                                             int dim, int phs, const double *sp, const double *sc,
                                             const double *pm, const double *tri,
                                             const double *xp, const int *ex, double *rhs) {
    // this row's right-hand sides, through shared memory (a register copy would stay
    // live across the whole unrolled row)
    const bool node = r < n;
    if (node && !xp && phs >= 3)
        node_rhs(r, dim, phs, sp, sc, rhs);
    else
        for (int c = 0; c < R; c++)
            rhs[c] = r < S ? aug_entry(r, S + c, n, m, dim, phs, sp, sc, ex, xp) : 0.0;
    const int p = r - n;  // polynomial row index (r >= n)
    // pair (r, j) in the packed table: tri_index(r, j, n) = tr + j above the diagonal,
    // tri_index(j, r, n) = j n - (j (j + 3) / 2 + 1) + r below it
    const int tr = r * n - r * (r + 1) / 2 - r - 1;
#pragma unroll
    for (int j = 0; j < W; j++) {
        double v = 0.0;
        if (r < S) {
            if (j < n) {
                if (node) {
                    const int q = j > r ? tr + j : j * n - (j * (j + 3) / 2 + 1) + r;
                    v = j == r ? 0.0 : tri[q];
                } else {
                    v = pm[j * MAX_M + p];
                }
            } else if (j < S) {
                v = node ? pm[r * MAX_M + (j - n)] : 0.0;
            } else if (j < S + R) {
                v = rhs[j - S];
            }
        }
        a[j] = v;
    }
}

// one elimination step with the live width bounded by WC: rows drop their column
// k (a[0]) and shift left; the pivot row itself is zeroed out of the update (l = 0).
// pb holds pivot-row element e at pb[e + 1] (16-byte pairs from element 1 on) and the
// pivot's reciprocal at pb[0].
template <int W, int WC>
__device__ __forceinline__ void gj_update(double (&a)[W], const double *pb, double l) {
#pragma unroll
    for (int j = 0; j < WC - 1; j += 2) {
        const double2 q = *reinterpret_cast<const double2 *>(pb + j + 2);
        a[j] = fma(-l, q.x, a[j + 1]);
        if (j + 1 < WC - 1)
            a[j + 1] = fma(-l, q.y, a[j + 2]);
    }
    a[WC - 1] = 0.0;
}

// the pivot row's live entries into pb (element e at pb[e + 1])
template <int W, int WC>
__device__ __forceinline__ void gj_publish(const double (&a)[W], double *pb) {
    pb[1] = a[0];
#pragma unroll
    for (int e = 1; e < WC; e += 2)
        *reinterpret_cast<double2 *>(pb + e + 1) = make_double2(a[e], e + 1 < WC ? a[e + 1] : 0.0);
}

// per-thread elimination state
struct GjRow {
    bool eligible, singular;
    int my_step;
    double my_diag;
};

// chunk C of the elimination (steps C*CH .. C*CH + CH - 1): the live width of every
// row is at most WC = W - C*CH there, so the update and the pivot-row publication
// run over WC registers (a compile-time bound, registers stay statically indexed)
template <int G, int W, int GROUPS, int C, class Sync>
__device__ __forceinline__ void gj_chunks(double (&a)[W], GjRow &st, int S, int tid, int lane,
                                          int warp_in_grp, double *prow, double *amax, Sync sync) {
    using Sh = GJShape<G, W, GROUPS>;
    if constexpr (C < Sh::NCH) {
        if (C * Sh::CH >= S)
            return;
        constexpr int WC = W - C * Sh::CH;
        const int kend = min(S, (C + 1) * Sh::CH);
        for (int k = C * Sh::CH; k < kend; k++) {
            // buffers alternate between steps, so no barrier is needed between one
            // step's reads of the pivot row and the next step's publication
            double *pb = prow + (k & 1) * Sh::PROW, *am = amax + (k & 1) * 2 * G;
            // ---- pivot: largest |a[0]| among rows not yet used, lowest row on ties
            // (|a| >= 0 orders as its bit pattern: high words first, then low words)
            const unsigned long long key =
                st.eligible ? (unsigned long long)__double_as_longlong(fabs(a[0])) : 0ull;
            const unsigned khi = (unsigned)(key >> 32), klo = (unsigned)key;
            const unsigned mhi = __reduce_max_sync(0xffffffffu, khi);
            const unsigned mlo = __reduce_max_sync(0xffffffffu, khi == mhi ? klo : 0u);
            const unsigned ball =
                __ballot_sync(0xffffffffu, st.eligible && khi == mhi && klo == mlo);
            const double wmx =
                __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
            int p;
            double mx;
            if (G == 1) {
                p = __ffs(ball) - 1;
                mx = wmx;
            } else {
                if (lane == 0) {
                    am[warp_in_grp] = wmx;
                    am[G + warp_in_grp] = ball ? (double)(warp_in_grp * 32 + __ffs(ball) - 1) : -1.0;
                }
                sync();
                mx = -1.0;
                p = -1;
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const double v = am[g];
                    const int pg = (int)am[G + g];
                    if (pg >= 0 && v > mx) {
                        mx = v;
                        p = pg;
                    }
                }
            }
            if (tid == p) {
                pb[0] = 1.0 / a[0];  // the multiplier's reciprocal: one division per step
                gj_publish<W, WC>(a, pb);
                st.eligible = false;
                st.my_step = k;
                st.my_diag = a[0];
            }
            sync();
            if (!(mx > 0.0))
                st.singular = true;
            const double l = (tid == p) ? 0.0 : a[0] * pb[0];
            gj_update<W, WC>(a, pb, l);
        }
        gj_chunks<G, W, GROUPS, C + 1>(a, st, S, tid, lane, warp_in_grp, prow, amax, sync);
    }
}

template <int G, int W, int GROUPS>
__global__ void __launch_bounds__(GJShape<G, W, GROUPS>::CTA, GJShape<G, W, GROUPS>::MINB)
    stencil_gj_kernel(StencilJob J) {
    using Sh = GJShape<G, W, GROUPS>;
    extern __shared__ __align__(16) double smem_raw[];
    static_assert(Sh::OFF_PROW % 2 == 0, "pivot rows must start on a 16-byte boundary");
    const int grp = threadIdx.x / Sh::NT, tid = threadIdx.x % Sh::NT;
    const int lane = threadIdx.x & 31, warp_in_grp = tid >> 5;
    double *base = smem_raw + grp * Sh::DOUBLES;
    // sc: scales, minima, scaled probe (interpolation mode)
    double *sp = base, *sc = base + Sh::OFF_SC, *pm = base + Sh::OFF_PM;
    double *tri = base + Sh::OFF_TRI, *prow = base + Sh::OFF_PROW, *amax = base + Sh::OFF_AMAX;
    double *rhs = base + Sh::OFF_RHS + 4 * tid;
    auto sync = [&]() {
        if (G == 1)
            __syncwarp();
        else if (GROUPS == 1)
            __syncthreads();
        else
            asm volatile("bar.sync %0, %1;\n" ::"r"(1 + grp), "r"(Sh::NT) : "memory");
    };
    const int dim = J.dim, m = J.m, R = J.probe ? 1 : dim + 1;
    double *xp = J.probe ? sc + SC_PROBE : nullptr;
    __shared__ int s_item[GROUPS];
    __shared__ int s_ex[MAX_M * MAX_DIM];
    for (int q = threadIdx.x; q < MAX_M * MAX_DIM; q += blockDim.x)
        s_ex[q] = c_exps[q];
    __syncthreads();
    for (;;) {
        if (tid == 0)
            s_item[grp] = (int)atomicAdd(J.queue, 1u);
        sync();
        const int t = s_item[grp];
        sync();
        if (t >= J.count)
            break;
        const int id = sys_id(J, t);
        const int n = sys_n(J, id), S = n + m;
        load_scaled_points(J, id, n, sp, sc, tid, Sh::NT, sync);
        if (xp) {  // the probe shifted and scaled with its stencil (:23-30)
            if (tid < dim)
                xp[tid] = (J.probe[(size_t)id * dim + tid] - sc[SC_MIN + tid]) * sc[SC_INV + tid];
        }
        // monomials of every node (the P block and its transpose); consecutive lanes
        // take consecutive nodes of one monomial
        for (int q = tid; q < n * m; q += Sh::NT) {
            const int pp = q / n, i = q - pp * n;
            pm[i * MAX_M + pp] = monomial(sp + i * dim, pp, dim, s_ex);
        }
        pair_table(tri, n, dim, J.phs, sp, tid, Sh::NT);
        sync();
        double a[W];
        assemble_row<W>(a, tid, n, m, S, R, dim, J.phs, sp, sc, pm, tri, xp, s_ex, rhs);
        GjRow st{tid < S, false, -1, 1.0};
        gj_chunks<G, W, GROUPS, 0>(a, st, S, tid, lane, warp_in_grp, prow, amax, sync);
        const int my_step = st.my_step;
        const double my_diag = st.my_diag;
        const bool singular = st.singular;
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
    __host__ __device__ int doubles() const { return MAX_S * MAX_DIM + SC_DOUBLES + s_max * lda + 4 * s_max; }
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
    double *sp = sm, *sc = sp + MAX_S * MAX_DIM, *A = sc + SC_DOUBLES;
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
        // the saddle matrix (aug_entry's A block): r^phs once per node pair, written
        // to both triangles; zero diagonal; the monomials, one per lane and step of a
        // single monomial index (uniform constant-memory reads), to P and P^T; zero
        // polynomial block
        {
            const int np = n * (n - 1) / 2;
            int i = 0, j = lane + 1;
            while (j >= n && i < n) {
                ++i;
                j = j - n + i + 1;
            }
            for (int q = lane; q < np; q += 32) {
                double r2 = 0.0;
                for (int d = 0; d < dim; d++) {
                    const double tq = sp[i * dim + d] - sp[j * dim + d];
                    r2 += tq * tq;
                }
                const double v = rpow_odd(r2, J.phs);
                A[i * lda + j] = v;
                A[j * lda + i] = v;
                j += 32;
                while (j >= n && i < n) {
                    ++i;
                    j = j - n + i + 1;
                }
            }
        }
        for (int i = lane; i < n; i += 32)
            A[i * lda + i] = 0.0;
        for (int q = lane; q < n * m; q += 32) {
            const int pp = q / n, i = q - pp * n;
            const double v = monomial(sp + i * dim, pp, dim, c_exps);
            A[i * lda + n + pp] = v;
            A[(n + pp) * lda + i] = v;
        }
        for (int q = lane; q < m * m; q += 32) {
            const int a = q / m, b = q - a * m;
            A[(n + a) * lda + n + b] = 0.0;
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

template <int G, int W, int GROUPS> static int launch_gj(StencilJob J, cudaStream_t s) {
    using Sh = GJShape<G, W, GROUPS>;
    size_t smem = (size_t)Sh::DOUBLES * GROUPS * sizeof(double);
    auto k = stencil_gj_kernel<G, W, GROUPS>;
    MP_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, Sh::CTA, smem));
    if (per_sm < 1)
        return fail(MP_CUDA_ERROR, "stencil kernel G=%d W=%d x%d does not fit on an SM", G, W,
                    GROUPS);
    int groups_needed = (J.count + GROUPS - 1) / GROUPS;
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

// Size classes: a register row of width W >= S + dim + 1 (the narrowest that
// fits: the elimination's work grows with W) and G = ceil(S / 32) warps, one row per
// thread.
constexpr int GJ_CLASSES = 7;
static const int gj_width[GJ_CLASSES] = {36, 44, 56, 68, 76, 84, 100};
static const int gj_warps[GJ_CLASSES] = {1, 2, 2, 2, 3, 3, 3};

static int gj_class(int S, int R) {
    for (int c = 0; c < GJ_CLASSES; c++)
        if (S <= 32 * gj_warps[c] && S + R <= gj_width[c])
            return c;
    return -1;
}

// CTA shapes of a class: systems (groups of G warps) per CTA
constexpr int GJ_SHAPES = 4;
static const int gj_groups[GJ_CLASSES][GJ_SHAPES] = {{1, 2, 4, 8}, {1, 2, 0, 0}, {1, 2, 0, 0},
                                                     {1, 2, 0, 0}, {1, 2, 0, 0}, {1, 2, 0, 0},
                                                     {1, 2, 0, 0}};

static int launch_shape(int cls, int shape, const StencilJob &J, cudaStream_t s) {
    switch (cls * GJ_SHAPES + shape) {
    case 0: return launch_gj<1, 36, 1>(J, s);
    case 1: return launch_gj<1, 36, 2>(J, s);
    case 2: return launch_gj<1, 36, 4>(J, s);
    case 3: return launch_gj<1, 36, 8>(J, s);
    case 4: return launch_gj<2, 44, 1>(J, s);
    case 5: return launch_gj<2, 44, 2>(J, s);
    case 8: return launch_gj<2, 56, 1>(J, s);
    case 9: return launch_gj<2, 56, 2>(J, s);
    case 12: return launch_gj<2, 68, 1>(J, s);
    case 13: return launch_gj<2, 68, 2>(J, s);
    case 16: return launch_gj<3, 76, 1>(J, s);
    case 17: return launch_gj<3, 76, 2>(J, s);
    case 20: return launch_gj<3, 84, 1>(J, s);
    case 21: return launch_gj<3, 84, 2>(J, s);
    case 24: return launch_gj<3, 100, 1>(J, s);
    case 25: return launch_gj<3, 100, 2>(J, s);
    }
    return fail(MP_BAD_ARG, "stencil size class %d shape %d", cls, shape);
}

// The CTA shape of each (class, dimension), chosen by the autotuner on the first
// batched call that has enough systems of the class (-1: not tuned yet; the
// default then is 4 systems per CTA for one-warp systems, one otherwise).
static int g_gj_shape[GJ_CLASSES][2] = {{-1, -1}, {-1, -1}, {-1, -1}, {-1, -1},
                                        {-1, -1}, {-1, -1}, {-1, -1}};

static int class_shape_of(int cls, int dim) {
    const int t = g_gj_shape[cls][dim - 2];
    return t >= 0 ? t : (cls == 0 ? 2 : 0);
}

static int launch_class(int cls, const StencilJob &J, cudaStream_t s) {
    return launch_shape(cls, class_shape_of(cls, J.dim), J, s);
}

// Time every CTA shape of a class on a sample of its systems (the first
// `sample` of the class list; the sample's outputs are written, as the full run
// writes them again) with CUDA events, median of three, and keep the fastest.
static int gj_autotune(int cls, StencilJob J, int sample, cudaStream_t s) {
    if (g_gj_shape[cls][J.dim - 2] >= 0)
        return MP_OK;
    J.count = std::min(J.count, sample);
    cudaEvent_t e0, e1;
    MP_CUDA(cudaEventCreate(&e0));
    MP_CUDA(cudaEventCreate(&e1));
    int best = -1;
    float best_us = 0.f;
    for (int sh = 0; sh < GJ_SHAPES; sh++) {
        if (!gj_groups[cls][sh])
            continue;
        float t[3];
        int rc = MP_OK;
        for (int rep = 0; rep < 4 && rc == MP_OK; rep++) {
            cudaEventRecord(e0, s);
            rc = launch_shape(cls, sh, J, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0)
                t[rep - 1] = ms * 1e3f;
        }
        if (rc != MP_OK) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            return rc;
        }
        std::sort(t, t + 3);
        if (best < 0 || t[1] < best_us) {
            best = sh;
            best_us = t[1];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g_gj_shape[cls][J.dim - 2] = best;
    return MP_OK;
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

// A batch of uneven systems, classified once: the systems of each size class as a
// device list, a side stream per class forked from and joined to the caller's
// stream, the queue and singular counters.  Runs launch only.
struct mp_stencil_plan_s {
    int nsys = 0, dim = 0, m = 0, poly_deg = 0, s_max = 0;
    int64_t npts = 0;
    int count[GJ_CLASSES] = {};
    dbuf<int> list[GJ_CLASSES];
    dbuf<unsigned int> words;  // per class: queue (4 words apart), singular count
    cudaStream_t side[GJ_CLASSES] = {};
    cudaEvent_t fork = nullptr, join[GJ_CLASSES] = {};
    const int *sizes = nullptr;
    const int64_t *offsets = nullptr;
    dbuf<int> own_sizes;
    dbuf<int64_t> own_offsets;
    ~mp_stencil_plan_s() {
        for (int c = 0; c < GJ_CLASSES; c++) {
            if (side[c])
                cudaStreamDestroy(side[c]);
            if (join[c])
                cudaEventDestroy(join[c]);
        }
        if (fork)
            cudaEventDestroy(fork);
    }
};

extern "C" int mp_stencil_plan_create(int nsys, const int *sizes, const int64_t *offsets, int dim,
                                      int poly_deg, mp_stencil_plan *out) {
    if (!out || nsys <= 0 || !sizes || !offsets || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_stencil_plan_create: bad arguments");
    int m = mp_num_poly_terms(dim, poly_deg);
    if (m <= 0 || m > MAX_M)
        return fail(MP_BAD_ARG, "poly_deg %d in %dD gives %d monomials (max %d)", poly_deg, dim, m,
                    MAX_M);
    const int R = dim + 1;
    std::vector<int> hs(nsys);
    std::vector<int64_t> ho(nsys);
    MP_CUDA(cudaMemcpy(hs.data(), sizes, sizeof(int) * nsys, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(ho.data(), offsets, sizeof(int64_t) * nsys, cudaMemcpyDefault));
    std::unique_ptr<mp_stencil_plan_s> P(new mp_stencil_plan_s);
    P->nsys = nsys;
    P->dim = dim;
    P->m = m;
    P->poly_deg = poly_deg;
    std::vector<int> lists[GJ_CLASSES];
    for (int i = 0; i < nsys; i++) {
        if (hs[i] < 2)
            return fail(MP_BAD_ARG, "system %d has %d nodes", i, hs[i]);
        const int c = gj_class(hs[i] + m, R);
        if (c < 0)
            return fail(MP_BAD_ARG, "system %d: %d nodes + %d monomials exceeds %d", i, hs[i], m,
                        MAX_S);
        lists[c].push_back(i);
        P->npts = std::max<int64_t>(P->npts, ho[i] + hs[i]);
        P->s_max = std::max(P->s_max, hs[i] + m);
    }
    if (is_device_ptr(sizes) && is_device_ptr(offsets)) {
        P->sizes = sizes;
        P->offsets = offsets;
    } else {
        MP_TRY(P->own_sizes.alloc(nsys));
        MP_TRY(P->own_offsets.alloc(nsys));
        MP_CUDA(cudaMemcpy(P->own_sizes.p, hs.data(), sizeof(int) * nsys, cudaMemcpyHostToDevice));
        MP_CUDA(cudaMemcpy(P->own_offsets.p, ho.data(), sizeof(int64_t) * nsys,
                           cudaMemcpyHostToDevice));
        P->sizes = P->own_sizes.p;
        P->offsets = P->own_offsets.p;
    }
    MP_TRY(P->words.alloc(4 * GJ_CLASSES));
    MP_CUDA(cudaMemset(P->words.p, 0, sizeof(unsigned int) * 4 * GJ_CLASSES));
    MP_CUDA(cudaEventCreateWithFlags(&P->fork, cudaEventDisableTiming));
    for (int c = 0; c < GJ_CLASSES; c++) {
        P->count[c] = (int)lists[c].size();
        if (lists[c].empty())
            continue;
        MP_TRY(P->list[c].alloc(lists[c].size()));
        MP_CUDA(cudaMemcpy(P->list[c].p, lists[c].data(), sizeof(int) * lists[c].size(),
                           cudaMemcpyHostToDevice));
        MP_CUDA(cudaStreamCreateWithFlags(&P->side[c], cudaStreamNonBlocking));
        MP_CUDA(cudaEventCreateWithFlags(&P->join[c], cudaEventDisableTiming));
    }
    *out = P.release();
    return MP_OK;
}

// the jobs of the plan's classes for one run
static StencilJob plan_job(mp_stencil_plan P, int c, const double *pts, int phs, double *w,
                           double *cond) {
    StencilJob J{};
    J.queue = P->words.p + 4 * c;
    J.singular = (int *)(P->words.p + 4 * c + 1);
    J.pts = pts;
    J.offsets = P->offsets;
    J.sizes = P->sizes;
    J.list = P->list[c].p;
    J.count = P->count[c];
    J.dim = P->dim;
    J.m = P->m;
    J.phs = phs;
    J.wb = w;
    J.cond = cond;
    return J;
}

extern "C" int mp_stencil_plan_run(mp_stencil_plan P, const double *pts, int phs_deg, double *w,
                                   double *cond, mp_stream s) {
    if (!P || !pts || !w)
        return fail(MP_BAD_ARG, "mp_stencil_plan_run: null argument");
    if (phs_deg != 3 && phs_deg != 5 && phs_deg != 7 && phs_deg != 9 && phs_deg != 11)
        return fail(MP_BAD_ARG, "phs_deg should be 3, 5, 7, 9 or 11; got %d", phs_deg);
    if (!is_device_ptr(pts) || !is_device_ptr(w) || (cond && !is_device_ptr(cond)))
        return fail(MP_BAD_ARG, "mp_stencil_plan_run takes device arrays (mp_stencil_weights_"
                                "batched stages host arrays)");
    int m = 0;
    MP_TRY(upload_exponents(P->dim, P->poly_deg, &m));
    cudaStream_t st = S(s);
    // classes not tuned yet are tuned first, on a sample of their own systems
    for (int c = 0; c < GJ_CLASSES; c++)
        if (P->count[c] >= 8 * sm_count() && g_gj_shape[c][P->dim - 2] < 0)
            MP_TRY(gj_autotune(c, plan_job(P, c, pts, phs_deg, w, nullptr), 32 * sm_count(), st));
    MP_CUDA(cudaMemsetAsync(P->words.p, 0, sizeof(unsigned int) * 4 * GJ_CLASSES, st));
    MP_CUDA(cudaEventRecord(P->fork, st));
    for (int c = 0; c < GJ_CLASSES; c++) {
        if (!P->count[c])
            continue;
        cudaStream_t ss = P->side[c];
        MP_CUDA(cudaStreamWaitEvent(ss, P->fork, 0));
        const StencilJob J = plan_job(P, c, pts, phs_deg, w, cond);
        MP_TRY(launch_class(c, J, ss));
        if (cond)
            MP_TRY(launch_cond(J, P->s_max, ss));
        MP_CUDA(cudaEventRecord(P->join[c], ss));
        MP_CUDA(cudaStreamWaitEvent(st, P->join[c], 0));
    }
    return MP_OK;
}

extern "C" int mp_stencil_plan_singular(mp_stencil_plan P, int *count, mp_stream s) {
    if (!P || !count)
        return fail(MP_BAD_ARG, "mp_stencil_plan_singular: null argument");
    unsigned int words[4 * GJ_CLASSES];
    MP_CUDA(cudaMemcpyAsync(words, P->words.p, sizeof(words), cudaMemcpyDeviceToHost, S(s)));
    MP_CUDA(cudaStreamSynchronize(S(s)));
    int n = 0;
    for (int c = 0; c < GJ_CLASSES; c++)
        n += (int)words[4 * c + 1];
    *count = n;
    return MP_OK;
}

extern "C" int mp_stencil_plan_info(mp_stencil_plan P, int *class_count, int *class_shape) {
    if (!P)
        return fail(MP_BAD_ARG, "mp_stencil_plan_info: null plan");
    for (int c = 0; c < GJ_CLASSES; c++) {
        if (class_count)
            class_count[c] = P->count[c];
        if (class_shape)
            class_shape[c] = gj_groups[c][class_shape_of(c, P->dim)];
    }
    return MP_OK;
}

extern "C" int mp_stencil_plan_destroy(mp_stencil_plan P) {
    delete P;
    return MP_OK;
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
    mp_stencil_plan P = nullptr;
    MP_TRY(mp_stencil_plan_create(nsys, sizes, offsets, dim, poly_deg, &P));
    std::unique_ptr<mp_stencil_plan_s> hold(P);
    const int R = dim + 1;
    dbuf<double> dpts, dw, dcond;
    const double *ppts = nullptr;
    MP_TRY(stage_in(pts, (size_t)P->npts * dim, dpts, &ppts, st));
    double *pw = w, *pc = cond;
    if (!is_device_ptr(w)) {
        MP_TRY(dw.alloc((size_t)P->npts * R));
        pw = dw.p;
    }
    if (cond && !is_device_ptr(cond)) {
        MP_TRY(dcond.alloc(nsys));
        pc = dcond.p;
    }
    MP_TRY(mp_stencil_plan_run(P, ppts, phs_deg, pw, pc, s));
    int bad = 0;
    MP_TRY(mp_stencil_plan_singular(P, &bad, s));
    if (dw.p)
        MP_CUDA(cudaMemcpyAsync(w, dw.p, sizeof(double) * P->npts * R, cudaMemcpyDeviceToHost, st));
    if (dcond.p)
        MP_CUDA(cudaMemcpyAsync(cond, dcond.p, sizeof(double) * nsys, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (bad)
        return fail(MP_SINGULAR_STENCIL, "%d stencil systems had a zero pivot", bad);
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
