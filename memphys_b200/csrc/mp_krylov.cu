// mp_krylov.cu -- pressure-Poisson system assembly and BiCGSTAB (FP64, and
// FP32 inner iterations under FP64 iterative refinement), with the mp_ppe_*
// C ABI (SOLVER::init / SOLVER::general_solve, solver.cpp:14-79, 283-363).
#include <cstddef>
#include <cmath>
#include <vector>
#include "mp_krylov.cuh"
#include "mp_amg.cuh"
#include "mp_cloud.cuh"
#include "mp_ppe.cuh"

namespace mp {

template <class T> struct V2t;
template <> struct V2t<double> { using type = double2; };
template <> struct V2t<float> { using type = float2; };

constexpr double EPS2 = 2.220446049250313e-16 * 2.220446049250313e-16;
constexpr int KT = 256;  // threads per block in all Krylov kernels (8 slices)
// resident blocks per SM the kernels are compiled for (32 registers): the fused
// SpMV + reduction kernels wait on memory; at 48 registers and 4 blocks per SM
// they ran at 42 % warps active and 40 % of DRAM bandwidth (k_spmv_omega 62 us at
// 1M rows; 6 blocks: 50 us; 8 blocks: 46 us)
constexpr int KT_BLOCKS = 8;

__device__ __forceinline__ int gwarp() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }

// Rows r0 = 64w + 2 lane and r0 + 1 of slice w: a = (A x)_row, xs = x at the
// self column (stencil entry 0 is the row's own node).
template <class T>
__device__ __forceinline__ void ell_pair(const EllView<T> &A, int w, int lane,
                                         const T *__restrict__ x, T &a0, T &a1, T &xs0, T &xs1) {
    using V2 = typename V2t<T>::type;
    size_t base;
    int K;
    slice_span(A, w, base, K);
    base += 2 * lane;
    if constexpr (sizeof(T) == 4) {
        if (A.pk) {  // FP32 difference form as (column, value) pairs; self entry = row sum
            const int4 *P = reinterpret_cast<const int4 *>(A.pk + base);
            int4 e = __ldcs(P);
            xs0 = __ldg(x + e.x);
            xs1 = __ldg(x + e.z);
            a0 = __int_as_float(e.y) * xs0;
            a1 = __int_as_float(e.w) * xs1;
#pragma unroll 4
            for (int k = 1; k < K; k++) {
                e = __ldcs(P + (size_t)k * (SLICE / 2));
                a0 = fma(__int_as_float(e.y), __ldg(x + e.x) - xs0, a0);
                a1 = fma(__int_as_float(e.w), __ldg(x + e.z) - xs1, a1);
            }
            return;
        }
    }
    if (A.dslice && A.dslice[w]) {  // 16-bit column deltas (warp-uniform)
        const int i0 = w * SLICE + 2 * lane;
        const T *xr0 = x + i0, *xr1 = x + i0 + 1;
        short2 d = __ldcs(reinterpret_cast<const short2 *>(A.dcols + base));
        V2 v = __ldcs(reinterpret_cast<const V2 *>(A.vals + base));
        xs0 = __ldg(xr0 + d.x);
        xs1 = __ldg(xr1 + d.y);
        a0 = v.x * xs0;
        a1 = v.y * xs1;
#pragma unroll 4
        for (int k = 1; k < K; k++) {
            const size_t o = base + (size_t)k * SLICE;
            d = __ldcs(reinterpret_cast<const short2 *>(A.dcols + o));
            v = __ldcs(reinterpret_cast<const V2 *>(A.vals + o));
            a0 = fma(v.x, __ldg(xr0 + d.x), a0);
            a1 = fma(v.y, __ldg(xr1 + d.y), a1);
        }
        return;
    }
    int2 c = __ldcs(reinterpret_cast<const int2 *>(A.cols + base));
    V2 v = __ldcs(reinterpret_cast<const V2 *>(A.vals + base));
    xs0 = __ldg(x + c.x);
    xs1 = __ldg(x + c.y);
    a0 = v.x * xs0;
    a1 = v.y * xs1;
#pragma unroll 4
    for (int k = 1; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        c = __ldcs(reinterpret_cast<const int2 *>(A.cols + o));
        v = __ldcs(reinterpret_cast<const V2 *>(A.vals + o));
        a0 = fma(v.x, __ldg(x + c.x), a0);
        a1 = fma(v.y, __ldg(x + c.y), a1);
    }
}

struct RedBuf {
    double *partials;
    unsigned int *ticket;
};

// Preconditioner of a bordered system B = [A e; e^T 0] (e = ones, A e = 0: the
// all-Neumann pressure operator) under the multigrid cycle V:
//   M^-1 [r; r_n] = [V(r - a e) + c e; a],  a = w^T r / w^T e,  c = (r_n - e^T V(r - a e)) / n,
// w approximating the left null vector of A (A^T w = 0), which decides how much of r
// lies outside A's range.
// Feeding V the constant component of r (the border's column) and taking the border
// entry as it comes makes B M^-1 badly conditioned in those two directions; with them
// taken out B M^-1 is the identity up to a rank-one term for an exact V, and the
// Krylov iteration needs about what the same operator needs without the border
// (measured at 1M nodes: 26 instead of 41 sweeps for one right-hand side).  V is
// linear, so V(r - a e) = V(r) - a V(e): the cycle runs on r as before (its first
// smoothing step stays fused into the update that writes r) and the kernels after it
// apply the correction with ve = V(e), ave = A ve and sve = e^T ve, computed once.
// As A e = 0 to rounding, the c e part enters B y only through the border row, whose
// value is then r_n by construction.  The left null vector of a Laplacian with
// Neumann rows follows Green's identity, sum_i V_i (Lu)_i = sum_b S_b (du/dn)_b: a
// node's volume share on interior rows and minus its surface share on boundary rows.
// w = 1 on interior rows and beta on boundary rows, beta fitted at set-up so that
// w^T A f = 0 for f = |x|^2, did as well as the exact null vector on a 90K-node cavity
// (17 / 13 sweeps for a smooth / rough solution against 18 / 14 exact and 21 / 17 for
// the plain mean; the fractional step 14.2 against 18.3 iterations per step).
// ve == nullptr: no deflation.
template <class T> struct Defl {
    const T *ve, *ave;
    double sve;
    int nv;
    const unsigned char *bflag;  // boundary rows (weight beta)
    double beta, we;             // we = w^T e
};

#define KRYLOV_SMEM __shared__ double red_smem[32 * 4];

// ---------------------------------------------------------------- init
// r = b - A x, r0 = r, p = v = 0, scalars of Eigen's BiCGSTAB prologue.
template <class T, bool ZERO_X>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_init(EllView<T> A, int bordered, const T *x, const T *b, T *r, T *r0, T *p, T *v,
           BicgScalars *S, RedBuf R, double tol, int maxit, cudaGraphConditionalHandle h) {
    KRYLOV_SMEM
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    double acc[3] = {0, 0, 0};
    for (int w = gwarp(); w < nsl; w += nwarps) {
        T a0 = 0, a1 = 0, s0 = 0, s1 = 0;
        if (!ZERO_X)
            ell_pair(A, w, lane, x, a0, a1, s0, s1);
        const T xb = (bordered && !ZERO_X) ? x[nv] : T(0);
        const int i0 = w * SLICE + 2 * lane;
        T as[2] = {a0, a1}, ss[2] = {s0, s1};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = i0 + q;
            if (i < nv) {
                const T ri = b[i] - (as[q] + xb);
                r[i] = ri;
                r0[i] = ri;
                p[i] = 0;
                v[i] = 0;
                acc[0] += (double)ri * ri;
                acc[1] += (double)b[i] * b[i];
                acc[2] += (double)ss[q];
            }
        }
    }
    if (grid_reduce<3>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double rr = acc[0], bb = acc[1];
        if (bordered) {
            const T rn = b[nv] - (T)acc[2];
            r[nv] = rn;
            r0[nv] = rn;
            p[nv] = 0;
            v[nv] = 0;
            rr += (double)rn * rn;
            bb += (double)b[nv] * b[nv];
        }
        S->b_sq = bb;
        if (!ZERO_X)  // FP64 solves: the initial guess's residual (mixed: set by the outer residual)
            S->relres0 = bb > 0 ? sqrt(rr / bb) : 0.0;
        S->r0_sq = rr;
        S->rr = rr;
        S->rho_old = 1.0;
        S->rho = rr;
        S->alpha = 1.0;
        S->omega = 1.0;
        S->it = 0;
        S->half = 0;
        S->restarts = 0;
        S->need_restart = 0;
        S->maxit = maxit;
        // The inner solve of a refinement sweep (ZERO_X) asks for the smaller of
        // the sweep's reduction `tol` and half the reduction the outer residual
        // still needs (at most 2x per sweep): near convergence a sweep then stops
        // once the outer tolerance is in reach instead of reducing by `tol`.
        double t2 = tol * tol;
        if (ZERO_X && S->rr_true > 0.0)
            t2 = fmax(t2, fmin(0.25 * S->tol_outer2 * S->b64_sq / S->rr_true, 0.25));
        S->tol2 = ZERO_X ? t2 * bb : fmax(t2 * bb, S->abs_tol2);
        S->zero_x = (bb == 0.0);
        int done = (bb == 0.0) || !(rr > S->tol2 && maxit > 0);
        S->status = MP_OK;
        if (!isfinite(rr) || !isfinite(bb)) {
            S->status = MP_NAN_DETECTED;
            done = 1;
        }
        S->done = done;
        if (h)
            cudaGraphSetConditional(h, done ? 0u : 1u);
    }
}

// ------------------------------------------------ learned-guess weight
// With x the extrapolated guess and f a correction field: theta = <r, A f> /
// <A f, A f>, r = b - A x, over the bordered system (the border entry of f is 0,
// the border row of A f is sum f_i).  One pass over the operator for both
// products; the last block stores theta.  (Minimising the residual restricted
// to the first multigrid level instead gave more iterations at 1M nodes.)
__global__ void __launch_bounds__(KT, 4)  // two operator streams + 5 sums: 64 registers
    k_guess_mr(EllView<double> A, int bordered, const double *x, const double *b,
               const double *f, BicgScalars *S, RedBuf R) {
    __shared__ double red_smem[32 * 5];
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    double acc[5] = {0, 0, 0, 0, 0};  // <r, Af>, <Af, Af>, sum x, sum f, <r, r>
    const double xb = bordered ? x[nv] : 0.0;
    for (int w = gwarp(); w < nsl; w += nwarps) {
        size_t base;
        int K;
        slice_span(A, w, base, K);
        base += 2 * lane;
        double ax[2] = {0, 0}, af[2] = {0, 0}, sx[2] = {0, 0}, sf[2] = {0, 0};
        for (int k = 0; k < K; k++) {
            const size_t o = base + (size_t)k * SLICE;
            const int2 c = __ldcs(reinterpret_cast<const int2 *>(A.cols + o));
            const double2 v = __ldcs(reinterpret_cast<const double2 *>(A.vals + o));
            const double x0 = __ldg(x + c.x), x1 = __ldg(x + c.y);
            const double f0 = __ldg(f + c.x), f1 = __ldg(f + c.y);
            if (k == 0) {  // self column: the border row's sums
                sx[0] = x0, sx[1] = x1, sf[0] = f0, sf[1] = f1;
            }
            ax[0] = fma(v.x, x0, ax[0]);
            ax[1] = fma(v.y, x1, ax[1]);
            af[0] = fma(v.x, f0, af[0]);
            af[1] = fma(v.y, f1, af[1]);
        }
        const int i0 = w * SLICE + 2 * lane;
#pragma unroll
        for (int q = 0; q < 2; q++) {
            if (i0 + q >= nv)
                continue;
            const double r = b[i0 + q] - (ax[q] + xb);
            acc[0] += r * af[q];
            acc[1] += af[q] * af[q];
            acc[2] += sx[q];
            acc[3] += sf[q];
            acc[4] += r * r;
        }
    }
    if (grid_reduce<5>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double num = acc[0], den = acc[1], rr = acc[4];
        if (bordered) {
            const double rn = b[nv] - acc[2];
            num += rn * acc[3];
            den += acc[3] * acc[3];
            rr += rn * rn;
        }
        // ||r - th A f||^2 = rr - num^2 / den: a correction that removes under 10 % of
        // the squared residual is dropped (a small weight on a rough field helps the
        // residual norm a little and the iteration count not at all)
        double th = den > 0 ? num / den : 0.0;
        if (!(den > 0 && num * num >= 0.1 * rr * den) || !isfinite(th))
            th = 0.0;
        S->guess_theta = th;
    }
}

__global__ void k_guess_axpy(int nv, double *x, const double *f, const BicgScalars *S) {
    const double th = S->guess_theta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
        x[i] += th * f[i];
}

// Eigen's restart: r = b - A x, r0 = r, rho = r0_sq = ||r||^2 (rare path)
template <class T>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_restart(EllView<T> A, int bordered, const T *x, const T *b, T *r, T *r0, BicgScalars *S,
              RedBuf R) {
    KRYLOV_SMEM
    if (S->done || !S->need_restart)
        return;
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    double acc[2] = {0, 0};
    for (int w = gwarp(); w < nsl; w += nwarps) {
        T a0, a1, s0, s1;
        ell_pair(A, w, lane, x, a0, a1, s0, s1);
        const T xb = bordered ? x[nv] : T(0);
        const int i0 = w * SLICE + 2 * lane;
        T as[2] = {a0, a1}, ss[2] = {s0, s1};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = i0 + q;
            if (i < nv) {
                const T ri = b[i] - (as[q] + xb);
                r[i] = ri;
                r0[i] = ri;
                acc[0] += (double)ri * ri;
                acc[1] += (double)ss[q];
            }
        }
    }
    if (grid_reduce<2>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double rr = acc[0];
        if (bordered) {
            const T rn = b[nv] - (T)acc[1];
            r[nv] = rn;
            r0[nv] = rn;
            rr += (double)rn * rn;
        }
        S->r0_sq = rr;
        S->rho = rr;
        if (S->restarts++ == 0)
            S->it = 0;
        S->need_restart = 0;
    }
}

// p = r + beta (p - omega v); y = M^-1 p for the fused preconditioners; for the
// multigrid (H.d set) also the head of its cycle, H.d = H.dinv p / theta
template <class T, int PK>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_update_p(int nv, int bordered, const T *r, T *p, const T *v, T *y, const T *dinv,
               BicgScalars *S, AmgHead<T> H, RedBuf R, Defl<T> D) {
    KRYLOV_SMEM
    if (S->done)
        return;
    const double beta = (S->rho / S->rho_old) * (S->alpha / S->omega);
    const T bt = (T)beta, om = (T)S->omega;
    const int stride = gridDim.x * blockDim.x;
    double acc[1] = {0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
        const T pi = r[i] + bt * (p[i] - om * v[i]);
        p[i] = pi;
        if (PK == PK_JACOBI)
            y[i] = dinv[i] * pi;
        if (PK == PK_EXTERNAL && H.d)
            H.d[i] = H.dinv[i] * pi * H.inv_theta;
        if (D.ve)
            acc[0] += D.bflag[i] ? D.beta * pi : (double)pi;
    }
    if (bordered && blockIdx.x == 0 && threadIdx.x == 0) {
        const T pi = r[nv] + bt * (p[nv] - om * v[nv]);
        p[nv] = pi;
        if (PK != PK_NONE)
            y[nv] = pi;  // the deflated preconditioner reads p_n here (k_spmv_alpha)
    }
    if (D.ve && grid_reduce<1>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0)
        S->dfl_a[0] = acc[0] / D.we;
}

// v = B y, alpha = rho / (r0 . v).  Deflated (D.ve): y holds V(p) and p_n in its
// border entry; v = B y' for y' = [V(p) - a ve + c e; a] (see Defl), whose border
// entry replaces p_n in y for the x update
template <class T>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_spmv_alpha(EllView<T> A, int bordered, T *y, T *v, const T *r0, BicgScalars *S,
                 RedBuf R, Defl<T> D) {
    KRYLOV_SMEM
    if (S->done)
        return;
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    double acc[2] = {0, 0};
    for (int w = gwarp(); w < nsl; w += nwarps) {
        T a0, a1, s0, s1;
        ell_pair(A, w, lane, y, a0, a1, s0, s1);
        // the border column's value (read after the gathers: nothing extra stays live
        // across them)
        const T yb = D.ve ? (T)S->dfl_a[0] : (bordered ? y[nv] : T(0));
        const int i0 = w * SLICE + 2 * lane;
        T as[2] = {a0, a1}, ss[2] = {s0, s1};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = i0 + q;
            if (i < nv) {
                T vi = as[q] + yb;
                if (D.ve)
                    vi -= yb * D.ave[i];
                v[i] = vi;
                acc[0] += (double)r0[i] * vi;
                acc[1] += (double)ss[q];
            }
        }
    }
    if (grid_reduce<2>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double d = acc[0];
        if (bordered) {
            T vb = (T)acc[1];
            if (D.ve) {
                const T pn = y[nv], da = (T)S->dfl_a[0];
                S->dfl_c[0] = ((double)pn - acc[1] + (double)da * D.sve) / nv;
                vb = pn;
                y[nv] = da;
            }
            v[nv] = vb;
            d += (double)r0[nv] * vb;
        }
        S->dot_rv = d;
        S->alpha = S->rho / d;
    }
}

// s = r - alpha v; x += alpha y; z = M^-1 s for the fused preconditioners.
// ||s||^2 decides the half-step exit: when s already meets the tolerance, x is
// the solution (x + alpha y) and the iteration stops here, before the second
// preconditioner application (the later kernels of the sweep see S->done).
template <class T, int PK>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_update_s(int nv, int bordered, const T *r, const T *v, T *s, T *z, const T *dinv, T *x,
               const T *y, BicgScalars *S, RedBuf R, cudaGraphConditionalHandle h, AmgHead<T> H,
               Defl<T> D) {
    KRYLOV_SMEM
    if (S->done)
        return;
    const T al = (T)S->alpha;
    // deflated: x += alpha y' with y'_i = y_i - a ve_i + c (the border entry of y is a)
    const T da = D.ve ? (T)S->dfl_a[0] : T(0), dc = D.ve ? (T)S->dfl_c[0] : T(0);
    double acc[2] = {0, 0};
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += stride) {
        const T si = r[i] - al * v[i];
        s[i] = si;
        if (PK == PK_JACOBI)
            z[i] = dinv[i] * si;
        if (PK == PK_EXTERNAL && H.d)
            H.d[i] = H.dinv[i] * si * H.inv_theta;
        const T yi = D.ve ? y[i] - da * D.ve[i] + dc : y[i];
        x[i] = x[i] + al * yi;
        acc[0] += (double)si * si;
        if (D.ve)
            acc[1] += D.bflag[i] ? D.beta * si : (double)si;
    }
    if (grid_reduce<2>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double ss = acc[0];
        if (D.ve)
            S->dfl_a[1] = acc[1] / D.we;
        if (bordered) {
            const T si = r[nv] - al * v[nv];
            s[nv] = si;
            if (PK != PK_NONE)
                z[nv] = si;
            x[nv] = x[nv] + al * y[nv];
            ss += (double)si * si;
        }
        if (ss <= S->tol2) {  // converged at the half step (NaN compares false)
            S->rr = ss;
            S->it += 1;
            S->half = 1;
            S->done = 1;
            if (h)
                cudaGraphSetConditional(h, 0u);
        }
    }
}

// t = B z, omega = (t . s) / (t . t); deflated as k_spmv_alpha, z' = [V(s) - a ve + c e; a]
template <class T>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_spmv_omega(EllView<T> A, int bordered, T *z, T *t, const T *s, BicgScalars *S,
                 RedBuf R, Defl<T> D) {
    KRYLOV_SMEM
    if (S->done)
        return;
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    double acc[3] = {0, 0, 0};
    for (int w = gwarp(); w < nsl; w += nwarps) {
        T a0, a1, s0, s1;
        ell_pair(A, w, lane, z, a0, a1, s0, s1);
        const T zb = D.ve ? (T)S->dfl_a[1] : (bordered ? z[nv] : T(0));
        const int i0 = w * SLICE + 2 * lane;
        T as[2] = {a0, a1}, ss[2] = {s0, s1};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = i0 + q;
            if (i < nv) {
                T ti = as[q] + zb;
                if (D.ve)
                    ti -= zb * D.ave[i];
                t[i] = ti;
                acc[0] += (double)ti * ti;
                acc[1] += (double)ti * s[i];
                acc[2] += (double)ss[q];
            }
        }
    }
    if (grid_reduce<3>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double tt = acc[0], ts = acc[1];
        if (bordered) {
            T tb = (T)acc[2];
            if (D.ve) {
                const T da = (T)S->dfl_a[1];
                S->dfl_c[1] = ((double)s[nv] - acc[2] + (double)da * D.sve) / nv;
                tb = s[nv];
                z[nv] = da;
            }
            t[nv] = tb;
            tt += (double)tb * tb;
            ts += (double)tb * s[nv];
        }
        S->dot_tt = tt;
        S->dot_ts = ts;
        S->omega = tt > 0.0 ? ts / tt : 0.0;
    }
}

// x += omega z (alpha y was added with s); r = s - omega t; convergence test for
// the next sweep
template <class T>
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_update_xr(int nsys, T *x, const T *z, const T *s, const T *t, T *r, const T *r0,
                BicgScalars *S, RedBuf R, cudaGraphConditionalHandle h, Defl<T> D) {
    KRYLOV_SMEM
    if (S->done)
        return;
    const T om = (T)S->omega;
    const T da = D.ve ? (T)S->dfl_a[1] : T(0), dc = D.ve ? (T)S->dfl_c[1] : T(0);
    double acc[2] = {0, 0};
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride) {
        const T zi = (D.ve && i < D.nv) ? z[i] - da * D.ve[i] + dc : z[i];
        x[i] = x[i] + om * zi;
        const T ri = s[i] - om * t[i];
        r[i] = ri;
        acc[0] += (double)ri * ri;
        acc[1] += (double)r0[i] * ri;
    }
    if (grid_reduce<2>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        const double rr = acc[0];
        S->rr = rr;
        S->it += 1;
        S->rho_old = S->rho;
        S->rho = acc[1];
        S->need_restart = fabs(acc[1]) < EPS2 * S->r0_sq;
        int done = !(rr > S->tol2 && S->it < S->maxit);
        if (!isfinite(rr)) {
            S->status = MP_NAN_DETECTED;
            done = 1;
        }
        S->done = done;
        if (h)
            cudaGraphSetConditional(h, done ? 0u : 1u);
    }
}

// ||b - A x||^2 in FP64 (the residual solver.cpp:342-343 logs); zero x when
// ||b|| = 0 as Eigen's BiCGSTAB does.  Optionally stores r64 = b - A x.
__global__ void __launch_bounds__(KT, KT_BLOCKS)
    k_true_residual(EllView<double> A, int bordered, double *x, const double *b, double *r64,
                    BicgScalars *S, RedBuf R, int refine, cudaGraphConditionalHandle h) {
    KRYLOV_SMEM
    const int nv = A.nrows, lane = threadIdx.x & 31, nwarps = (gridDim.x * blockDim.x) >> 5;
    const int nsl = (nv + SLICE - 1) / SLICE;
    const bool zx = S->zero_x && !refine;
    double acc[3] = {0, 0, 0};
    for (int w = gwarp(); w < nsl; w += nwarps) {
        double a0 = 0, a1 = 0, s0 = 0, s1 = 0;
        if (!zx)
            ell_pair(A, w, lane, x, a0, a1, s0, s1);
        const double xb = (bordered && !zx) ? x[nv] : 0.0;
        const int i0 = w * SLICE + 2 * lane;
        double as[2] = {a0, a1}, ss[2] = {s0, s1};
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const int i = i0 + q;
            if (i < nv) {
                if (zx)
                    x[i] = 0.0;
                const double ri = b[i] - (as[q] + xb);
                if (r64)
                    r64[i] = ri;
                acc[0] += ri * ri;
                acc[1] += ss[q];
                acc[2] += b[i] * b[i];
            }
        }
    }
    if (grid_reduce<3>(acc, R.partials, R.ticket, red_smem) && threadIdx.x == 0) {
        double rr = acc[0], bb = acc[2];
        if (bordered) {
            if (zx)
                x[nv] = 0.0;
            const double rn = b[nv] - acc[1];
            if (r64)
                r64[nv] = rn;
            rr += rn * rn;
            bb += b[nv] * b[nv];
        }
        S->rr_true = rr;
        S->b64_sq = bb;
        if (refine && S->outer_it == 0)
            S->relres0 = bb > 0 ? sqrt(rr / bb) : 0.0;
        if (refine) {  // iterative-refinement loop control
            int done = !(rr > S->tol_outer2 * bb && S->outer_it < S->outer_max);
            if (bb == 0.0)
                done = 1;
            if (!isfinite(rr) || S->status == MP_NAN_DETECTED) {
                S->status = MP_NAN_DETECTED;
                done = 1;
            }
            S->outer_done = done;
            if (h)
                cudaGraphSetConditional(h, done ? 0u : 1u);
        }
    }
}

// refinement: b32 = r64 / ||r64||, e32 = 0
__global__ void k_ir_scale(int nsys, const double *r64, float *b32, float *e32, BicgScalars *S) {
    if (S->outer_done)
        return;
    const double sc = sqrt(S->rr_true);
    const double inv = sc > 0 ? 1.0 / sc : 0.0;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride) {
        b32[i] = (float)(r64[i] * inv);
        e32[i] = 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        S->scale = sc;
}

// refinement: x64 += ||r64|| * e32
__global__ void k_ir_update(int nsys, double *x, const float *e32, BicgScalars *S) {
    if (S->outer_done)
        return;
    const double sc = S->scale;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride)
        x[i] += sc * (double)e32[i];
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        S->outer_it += 1;
        S->total_inner += S->it;
        S->half_total += S->half;
    }
}

__global__ void k_jacobi_dinv(EllView<double> A, double *dinv, float *dinv32) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= A.nrows)
        return;
    double d = A.vals[ell_index(i, 0, A.K)];
    double v = (d != 0.0 && isfinite(d)) ? 1.0 / d : 1.0;
    dinv[i] = v;
    if (dinv32)
        dinv32[i] = (float)v;
}

// ------------------------------------------------------------- assembly
// solver.cpp:165-204: interior rows diff*L + conv*(Gx+Gy[+Gz]) (+ unsteady on
// the self entry); Dirichlet rows identity; Neumann rows normal . grad.
__global__ void k_assemble_ppe(int nv, int K, int dim, const int *cols, const double *gx,
                               const double *gy, const double *gz, const double *lap,
                               const uint8_t *bflag, const uint8_t *dir, const double *normal,
                               double unsteady, double conv, double diff, double *vals,
                               int *bad_self) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t total = (size_t)ell_padded_rows(nv) * K;
    if (t >= total)
        return;
    size_t slice = t / ((size_t)K * SLICE);
    int k = (int)((t / SLICE) % K);
    int row = (int)(slice * SLICE + (t % SLICE));
    if (row >= nv) {
        vals[t] = 0.0;
        return;
    }
    const int col = cols[t];
    if (k == 0 && col != row)
        atomicAdd(bad_self, 1);
    double v;
    if (bflag[row]) {
        if (dir[row]) {
            v = (k == 0) ? 1.0 : 0.0;
        } else {
            v = normal[(size_t)dim * row] * gx[t] + normal[(size_t)dim * row + 1] * gy[t];
            if (dim == 3)
                v += normal[(size_t)dim * row + 2] * gz[t];
        }
    } else {
        v = diff * lap[t];
        v += conv * gx[t];
        v += conv * gy[t];
        if (dim == 3)
            v += conv * gz[t];
        if (col == row)
            v += unsteady;
    }
    vals[t] = v;
}

// ------------------------------------------------------------ host side
static unsigned vec_blocks(int n) {
    int b = (n + KT - 1) / KT;
    int cap = sm_count() * KT_BLOCKS;
    return (unsigned)(b < cap ? (b < 1 ? 1 : b) : cap);
}
// reduction kernels walk the slices with a grid of KT_BLOCKS blocks per SM (all
// resident at once), so the last-block ticket sees a bounded number of atomics
static unsigned slice_blocks(int nv) {
    int ns = (nv + SLICE - 1) / SLICE;
    int b = (ns + 7) / 8, cap = sm_count() * KT_BLOCKS;
    return (unsigned)(b < cap ? b : cap);
}

int Krylov::alloc(int nv_, int bordered_, bool mixed, bool external_pc) {
    nv = nv_;
    bordered = bordered_;
    nsys = nv + (bordered ? 1 : 0);
    const size_t n = nsys;
    for (dbuf<double> *b : {&x, &b64, &r, &r0, &p, &v, &s, &t})
        MP_TRY(b->alloc(n));
    MP_TRY(y.alloc(n));
    MP_TRY(z.alloc(n));
    if (mixed) {
        for (dbuf<float> *q : {&e32, &b32, &r32, &r032, &p32, &v32, &s32, &t32, &y32, &z32})
            MP_TRY(q->alloc(n));
        MP_TRY(res64.alloc(n));
    }
    (void)external_pc;
    size_t maxb = slice_blocks(nv);
    if (vec_blocks(nsys) > maxb)
        maxb = vec_blocks(nsys);
    MP_TRY(partials.alloc(5 * maxb + 64));  // up to 5 sums per block (learned-guess weight)
    MP_TRY(ticket.alloc(4));
    MP_TRY(scal.alloc(1));
    MP_CUDA(cudaMemset(ticket.p, 0, 4 * sizeof(unsigned int)));
    MP_CUDA(cudaMemset(scal.p, 0, sizeof(BicgScalars)));
    return MP_OK;
}

// One BiCGSTAB sweep (everything after the prologue), issued on stream s.
template <class T>
static int issue_iteration(const PpeSystem &P, const EllView<T> &A, const T *dinv, T *x, T *b,
                           T *r, T *r0, T *p, T *v, T *s_, T *t, T *y, T *z, BicgScalars *S,
                           RedBuf R, int pk, cudaGraphConditionalHandle h, cudaStream_t st,
                           Defl<T> D) {
    const int nv = P.nv, nsys = P.nsys, bd = P.bordered;
    T *yy = pk == PK_NONE ? p : y;
    T *zz = pk == PK_NONE ? s_ : z;
    // the multigrid's first smoothing pass is fused into the updates that write its input
    const AmgHead<T> H = pk == PK_EXTERNAL ? amg_head<T>(*P.amg) : AmgHead<T>{};
    const bool head = H.d != nullptr;
    k_restart<T><<<slice_blocks(nv), KT, 0, st>>>(A, bd, x, b, r, r0, S, R);
    MP_CHECK_LAUNCH();
    if (pk == PK_JACOBI)
        k_update_p<T, PK_JACOBI><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, p, v, yy, dinv, S, H, R, D);
    else if (pk == PK_NONE)
        k_update_p<T, PK_NONE><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, p, v, yy, dinv, S, H, R, D);
    else
        k_update_p<T, PK_EXTERNAL><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, p, v, yy, dinv, S, H, R,
                                                                  D);
    MP_CHECK_LAUNCH();
    if (pk == PK_EXTERNAL)
        MP_TRY(amg_apply<T>(*P.amg, p, yy, &S->done, st, head));
    k_spmv_alpha<T><<<slice_blocks(nv), KT, 0, st>>>(A, bd, yy, v, r0, S, R, D);
    MP_CHECK_LAUNCH();
    if (pk == PK_JACOBI)
        k_update_s<T, PK_JACOBI><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, v, s_, zz, dinv, x, yy,
                                                                S, R, h, H, D);
    else if (pk == PK_NONE)
        k_update_s<T, PK_NONE><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, v, s_, zz, dinv, x, yy, S,
                                                              R, h, H, D);
    else
        k_update_s<T, PK_EXTERNAL><<<vec_blocks(nv), KT, 0, st>>>(nv, bd, r, v, s_, zz, dinv, x,
                                                                  yy, S, R, h, H, D);
    MP_CHECK_LAUNCH();
    if (pk == PK_EXTERNAL)
        MP_TRY(amg_apply<T>(*P.amg, s_, zz, &S->done, st, head));
    k_spmv_omega<T><<<slice_blocks(nv), KT, 0, st>>>(A, bd, zz, t, s_, S, R, D);
    MP_CHECK_LAUNCH();
    k_update_xr<T><<<vec_blocks(nsys), KT, 0, st>>>(nsys, x, zz, s_, t, r, r0, S, R, h, D);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int Ppe::issue_prologue64(cudaGraphConditionalHandle h, cudaStream_t st) {
    k_init<double, false><<<slice_blocks(sys.nv), KT, 0, st>>>(
        sys.A.view64(), sys.bordered, W.x.p, W.b64.p, W.r.p, W.r0.p, W.p.p, W.v.p, W.scal.p,
        RedBuf{W.partials.p, W.ticket.p}, cfg.tol, cfg.maxit, h);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int Ppe::issue_sweep64(cudaGraphConditionalHandle h, cudaStream_t st) {
    return issue_iteration<double>(sys, sys.A.view64(), sys.dinv.p, W.x.p, W.b64.p, W.r.p,
                                   W.r0.p, W.p.p, W.v.p, W.s.p, W.t.p, W.y.p, W.z.p, W.scal.p,
                                   RedBuf{W.partials.p, W.ticket.p}, pk(), h, st,
                                   Defl<double>{W.ve.p, W.ave.p, W.sve, sys.nv, W.dflag.p, W.dbeta, W.dwe});
}

int Ppe::issue_epilogue64(cudaStream_t st) {
    k_true_residual<<<slice_blocks(sys.nv), KT, 0, st>>>(sys.A.view64(), sys.bordered, W.x.p,
                                                         W.b64.p, nullptr, W.scal.p,
                                                         RedBuf{W.partials.p, W.ticket.p}, 0, 0);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// mixed precision: outer residual (sets the refinement loop condition)
int Ppe::issue_ir_residual(cudaGraphConditionalHandle h, cudaStream_t st) {
    k_true_residual<<<slice_blocks(sys.nv), KT, 0, st>>>(sys.A.view64(), sys.bordered, W.x.p,
                                                         W.b64.p, W.res64.p, W.scal.p,
                                                         RedBuf{W.partials.p, W.ticket.p}, 1, h);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int Ppe::issue_ir_inner_prologue(cudaGraphConditionalHandle h, cudaStream_t st) {
    k_ir_scale<<<vec_blocks(sys.nsys), KT, 0, st>>>(sys.nsys, W.res64.p, W.b32.p, W.e32.p,
                                                    W.scal.p);
    MP_CHECK_LAUNCH();
    // inner solve of A e = b32 from e = 0; BiCGSTAB's prologue skips the SpMV
    k_init<float, true><<<slice_blocks(sys.nv), KT, 0, st>>>(
        sys.diff32(), sys.bordered, W.e32.p, W.b32.p, W.r32.p, W.r032.p, W.p32.p, W.v32.p,
        W.scal.p, RedBuf{W.partials.p, W.ticket.p}, cfg.inner_tol, cfg.maxit, h);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int Ppe::issue_ir_sweep(cudaGraphConditionalHandle h, cudaStream_t st) {
    return issue_iteration<float>(sys, sys.diff32(), sys.dinv32.p, W.e32.p, W.b32.p, W.r32.p,
                                  W.r032.p, W.p32.p, W.v32.p, W.s32.p, W.t32.p, W.y32.p, W.z32.p,
                                  W.scal.p, RedBuf{W.partials.p, W.ticket.p}, pk(), h, st,
                                  Defl<float>{W.ve32.p, W.ave32.p, W.sve32, sys.nv, W.dflag.p, W.dbeta, W.dwe});
}

int Ppe::issue_ir_update(cudaStream_t st) {
    k_ir_update<<<vec_blocks(sys.nsys), KT, 0, st>>>(sys.nsys, W.x.p, W.e32.p, W.scal.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// Set the refinement-loop constants before a mixed solve
__global__ void k_ir_setup(BicgScalars *S, double tol, int outer_max) {
    S->tol_outer2 = tol * tol;
    S->outer_it = 0;
    S->outer_max = outer_max;
    S->total_inner = 0;
    S->half_total = 0;
    S->status = MP_OK;
}

int Ppe::issue_ir_setup(cudaStream_t st) {
    k_ir_setup<<<1, 1, 0, st>>>(W.scal.p, cfg.tol, cfg.max_refine);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int Ppe::issue_guess_min_residual(const double *f, cudaStream_t st) {
    k_guess_mr<<<slice_blocks(sys.nv), KT, 0, st>>>(sys.A.view64(), sys.bordered, W.x.p, W.b64.p,
                                                    f, W.scal.p, RedBuf{W.partials.p, W.ticket.p});
    MP_CHECK_LAUNCH();
    k_guess_axpy<<<vec_blocks(sys.nv), KT, 0, st>>>(sys.nv, W.x.p, f, W.scal.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// Build the whole solve (prologue, while loop(s), epilogue) into `gb`.
int Ppe::build_solve_graph(GraphBuilder &gb) {
    if (cfg.precision != MP_FP32) {
        cudaGraphConditionalHandle h;
        MP_TRY(gb.make_handle(&h));
        MP_TRY(gb.captured([&](cudaStream_t s) { return issue_prologue64(h, s); }));
        MP_TRY(gb.while_loop(h, [&](GraphBuilder &body) {
            return body.captured([&](cudaStream_t s) { return issue_sweep64(h, s); });
        }));
        MP_TRY(gb.captured([&](cudaStream_t s) { return issue_epilogue64(s); }));
        return MP_OK;
    }
    cudaGraphConditionalHandle ho, hi;
    MP_TRY(gb.make_handle(&ho));
    MP_TRY(gb.make_handle(&hi));
    MP_TRY(gb.captured([&](cudaStream_t s) {
        MP_TRY(issue_ir_setup(s));
        return issue_ir_residual(ho, s);
    }));
    MP_TRY(gb.while_loop(ho, [&](GraphBuilder &outer) {
        MP_TRY(outer.captured([&](cudaStream_t s) { return issue_ir_inner_prologue(hi, s); }));
        MP_TRY(outer.while_loop(hi, [&](GraphBuilder &inner) {
            return inner.captured([&](cudaStream_t s) { return issue_ir_sweep(hi, s); });
        }));
        return outer.captured([&](cudaStream_t s) {
            MP_TRY(issue_ir_update(s));
            return issue_ir_residual(ho, s);
        });
    }));
    return MP_OK;
}

// Eager (no graph) solve: host polls the device scalars every `poll` sweeps.
int Ppe::solve_eager(cudaStream_t st) {
    const int poll = 8;
    BicgScalars hs;
    auto fetch = [&]() -> int {
        MP_CUDA(cudaMemcpyAsync(&hs, W.scal.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        return MP_OK;
    };
    if (cfg.precision != MP_FP32) {
        MP_TRY(issue_prologue64(0, st));
        for (int it = 0;; it++) {
            if (it % poll == 0) {
                MP_TRY(fetch());
                if (hs.done)
                    break;
            }
            MP_TRY(issue_sweep64(0, st));
        }
        return issue_epilogue64(st);
    }
    MP_TRY(issue_ir_setup(st));
    MP_TRY(issue_ir_residual(0, st));
    for (;;) {
        MP_TRY(fetch());
        if (hs.outer_done)
            break;
        MP_TRY(issue_ir_inner_prologue(0, st));
        for (int it = 0;; it++) {
            if (it % poll == 0) {
                MP_TRY(fetch());
                if (hs.done)
                    break;
            }
            MP_TRY(issue_ir_sweep(0, st));
        }
        MP_TRY(issue_ir_update(st));
        MP_TRY(issue_ir_residual(0, st));
    }
    return MP_OK;
}

int Ppe::solve_resident(cudaStream_t st, bool use_graph) {
    if (use_graph) {
        if (!graph.e) {
            GraphBuilder gb;
            MP_TRY(gb.init_root(cap_stream()));
            int rc = build_solve_graph(gb);
            if (rc != MP_OK) {
                if (gb.g)
                    cudaGraphDestroy(gb.g);
                return rc;
            }
            MP_TRY(graph.instantiate(gb));
        }
        return graph.launch(st);
    }
    return solve_eager(st);
}

cudaStream_t Ppe::cap_stream() {
    if (!capture_stream)
        cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking);
    return capture_stream;
}

int Ppe::read_stats(cudaStream_t st, SolveStats *out) {
    BicgScalars hs;
    MP_CUDA(cudaMemcpyAsync(&hs, W.scal.p, sizeof(hs), cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    stats_of(hs, out);
    return MP_OK;
}

void Ppe::stats_of(const BicgScalars &hs, SolveStats *out) const {
    out->iters = cfg.precision != MP_FP32 ? hs.it : hs.total_inner;
    out->outer = hs.outer_it;
    out->abs_res = std::sqrt(hs.rr_true);
    out->relres = hs.b64_sq > 0 ? std::sqrt(hs.rr_true / hs.b64_sq) : 0.0;
    out->status = hs.status;
    if (hs.status == MP_OK && out->relres > cfg.tol && hs.b64_sq > 0 &&
        !(hs.rr_true <= hs.abs_tol2))
        out->status = MP_NOT_CONVERGED;
    if (hs.status == MP_OK && !std::isfinite(out->relres))
        out->status = MP_NAN_DETECTED;
}

int Ppe::set_abs_tol(double atol, cudaStream_t st) {
    const double a2 = atol * atol;
    char *field = reinterpret_cast<char *>(W.scal.p) + offsetof(BicgScalars, abs_tol2);
    MP_CUDA(cudaMemcpyAsync(field, &a2, sizeof(double), cudaMemcpyHostToDevice, st));
    MP_CUDA(cudaStreamSynchronize(st));  // a2 lives on this stack frame
    return MP_OK;
}

int Ppe::refresh_diag(cudaStream_t st) {
    if (sys.amg)
        return fail(MP_BAD_ARG, "refresh_diag: the multigrid hierarchy would be stale");
    k_jacobi_dinv<<<(sys.nv + 255) / 256, 256, 0, st>>>(sys.A.view64(), sys.dinv.p,
                                                       sys.dinv32.p ? sys.dinv32.p : nullptr);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// ------------------------------------------- deflated preconditioner set-up
__global__ void k_defl_ones(int nv, int nsys, double *e, float *e32) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsys)
        return;
    const double v = i < nv ? 1.0 : 0.0;
    if (e)
        e[i] = v;
    if (e32)
        e32[i] = (float)v;
}
__global__ void k_defl_r2(int nv, int dim, const double *xyz, double *f) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    double r2 = 0.0;
    for (int d = 0; d < dim; d++)
        r2 += xyz[(size_t)i * dim + d] * xyz[(size_t)i * dim + d];
    f[i] = r2;
}
__global__ void k_defl_f2d(int n, const float *a, double *b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        b[i] = (double)a[i];
}
__global__ void k_defl_d2f(int n, const double *a, float *b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        b[i] = (float)a[i];
}

// ve = V(e), ave = A ve and sve = e^T ve of a bordered system under a multigrid of two or
// more levels (Defl), in the precision its Krylov iteration runs: FP32 for MP_FP32's
// inner solves (the FP32 cycle; A ve formed in FP64 and rounded), FP64 otherwise.  A
// one-level hierarchy is already the bordered system's exact inverse.
static int defl_setup(Ppe &P, mp_cloud_s *c, const uint8_t *bflag,
                      const std::vector<uint8_t> &hb, cudaStream_t st) {
    PpeSystem &sys = P.sys;
    Krylov &W = P.W;
    if (P.cfg.precond != MP_PRECOND_AMG || !sys.bordered || !sys.amg || sys.amg->L.size() < 2)
        return MP_OK;
    const int nv = sys.nv, nsys = sys.nsys;
    const unsigned g = (unsigned)((nsys + 255) / 256);
    const int *zero = sys.amg->zero_flag.p;
    std::vector<double> h(nv);
    {  // the weights of the mean: beta on boundary rows from w^T A |x|^2 = 0
        const int dim = cloud_view(c).dim;
        dbuf<double> f, af;
        MP_TRY(f.alloc(nv));
        MP_TRY(af.alloc(nv));
        k_defl_r2<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(nv, dim, cloud_xyz(c), f.p);
        MP_CHECK_LAUNCH();
        MP_TRY(ell_spmv<double>(sys.A.view64(), f.p, af.p, 1.0, 0.0, st));
        MP_CUDA(cudaMemcpyAsync(h.data(), af.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        double si = 0.0, sb = 0.0;
        int nb = 0;
        for (int i = 0; i < nv; i++) {
            if (hb[i]) {
                sb += h[i];
                nb++;
            } else {
                si += h[i];
            }
        }
        double beta = (sb != 0.0 && std::isfinite(si / sb)) ? -si / sb : 1.0;
        double we = (nv - nb) + beta * nb;
        // a weight sum near zero would make the mean meaningless: the plain mean then
        if (!(std::fabs(we) > 1e-6 * ((nv - nb) + std::fabs(beta) * nb))) {
            beta = 1.0;
            we = nv;
        }
        W.dbeta = beta;
        W.dwe = we;
        MP_TRY(W.dflag.alloc(nv));
        MP_CUDA(cudaMemcpyAsync(W.dflag.p, bflag, nv, cudaMemcpyDeviceToDevice, st));
    }
    dbuf<double> ve64;
    if (P.cfg.precision == MP_FP32) {
        dbuf<float> e32;
        dbuf<double> ave64;
        MP_TRY(e32.alloc(nsys));
        MP_TRY(W.ve32.alloc(nsys));
        MP_TRY(W.ave32.alloc(nv));
        MP_TRY(ve64.alloc(nsys));
        MP_TRY(ave64.alloc(nv));
        k_defl_ones<<<g, 256, 0, st>>>(nv, nsys, nullptr, e32.p);
        MP_CHECK_LAUNCH();
        MP_CUDA(cudaMemsetAsync(W.ve32.p, 0, sizeof(float) * nsys, st));
        MP_TRY(amg_apply<float>(*sys.amg, e32.p, W.ve32.p, zero, st, false));
        k_defl_f2d<<<g, 256, 0, st>>>(nv, W.ve32.p, ve64.p);
        MP_CHECK_LAUNCH();
        MP_TRY(ell_spmv<double>(sys.A.view64(), ve64.p, ave64.p, 1.0, 0.0, st));
        k_defl_d2f<<<g, 256, 0, st>>>(nv, ave64.p, W.ave32.p);
        MP_CHECK_LAUNCH();
        MP_CUDA(cudaMemcpyAsync(h.data(), ve64.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        double sum = 0.0;
        for (double v : h)
            sum += v;
        W.sve32 = sum;
        return MP_OK;
    }
    dbuf<double> e;
    MP_TRY(e.alloc(nsys));
    MP_TRY(W.ve.alloc(nsys));
    MP_TRY(W.ave.alloc(nv));
    k_defl_ones<<<g, 256, 0, st>>>(nv, nsys, e.p, nullptr);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaMemsetAsync(W.ve.p, 0, sizeof(double) * nsys, st));
    MP_TRY(amg_apply<double>(*sys.amg, e.p, W.ve.p, zero, st, false));
    MP_TRY(ell_spmv<double>(sys.A.view64(), W.ve.p, W.ave.p, 1.0, 0.0, st));
    MP_CUDA(cudaMemcpyAsync(h.data(), W.ve.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (double v : h)
        sum += v;
    W.sve = sum;
    return MP_OK;
}

int Ppe::create(mp_cloud_s *c, const uint8_t *boundary, const uint8_t *dirichlet,
                const double *normal, double unsteady, double conv, double diff,
                const mp_solver_cfg &cfg_in, cudaStream_t st, int border_rule,
                bool stencil_order) {
    cfg = Cfg::from(cfg_in);
    if (cfg.precond == MP_PRECOND_SOR)
        border_rule = 0;  // solver.cpp:30-31: no regularisation for SOR
    CloudView cv = cloud_view(c);
    const int nv = cv.nv, K = cv.n, dim = cv.dim;
    // solver.cpp:29-38: bordered unless a boundary node is Dirichlet
    std::vector<uint8_t> hb(nv), hd(nv);
    MP_CUDA(cudaMemcpy(hb.data(), boundary, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hd.data(), dirichlet, nv, cudaMemcpyDefault));
    int bordered = border_rule;
    for (int i = 0; i < nv && bordered; i++)
        if (hb[i] && hd[i])
            bordered = 0;
    sys.nv = nv;
    sys.K = K;
    sys.bordered = bordered;
    sys.nsys = nv + bordered;
    dbuf<uint8_t> db, dd;
    dbuf<double> dn;
    dbuf<int> bad;
    MP_TRY(db.alloc(nv));
    MP_TRY(dd.alloc(nv));
    MP_TRY(dn.alloc((size_t)nv * dim));
    MP_TRY(bad.alloc(1));
    MP_CUDA(cudaMemcpyAsync(db.p, hb.data(), nv, cudaMemcpyHostToDevice, st));
    MP_CUDA(cudaMemcpyAsync(dd.p, hd.data(), nv, cudaMemcpyHostToDevice, st));
    MP_CUDA(cudaMemcpyAsync(dn.p, normal, sizeof(double) * nv * dim, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    // the system shares the cloud's stencil columns
    shared_cols = cloud_cols(c);
    sys.A.nrows = nv;
    sys.A.ncols = sys.nsys;
    sys.A.K = K;
    const size_t tot = (size_t)ell_padded_rows(nv) * K;
    MP_TRY(sys.A.cols.alloc(tot));
    MP_CUDA(cudaMemcpyAsync(sys.A.cols.p, cv.cols, sizeof(int) * tot, cudaMemcpyDeviceToDevice, st));
    MP_TRY(sys.A.v64.alloc(tot));
    k_assemble_ppe<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(
        nv, K, dim, cv.cols, cv.w[0], cv.w[1], cv.w[2], cv.w[3], db.p, dd.p, dn.p, unsteady, conv,
        diff, sys.A.v64.p, bad.p);
    MP_CHECK_LAUNCH();
    int hbad = 0;
    MP_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (hbad)
        return fail(MP_BAD_ARG, "%d stencils do not start with their own node", hbad);
    if (!stencil_order)
        MP_TRY(ell_sort_rows(sys.A, st));
    const bool mixed = cfg.precision == MP_FP32;  // FP32 Krylov + FP64 refinement
    if (mixed) {
        MP_TRY(ell_make_fp32(sys.A, st));
        MP_TRY(ell_diff32(sys.A, sys.d32, sys.dpk, st));
    }
    // 16-bit column deltas where the stencils are local (the FP64 SpMVs of the Krylov
    // iteration and of the multigrid's finest level read them)
    MP_TRY(ell_make_deltas(sys.A, st));
    MP_TRY(sys.dinv.alloc(nv));
    if (mixed)
        MP_TRY(sys.dinv32.alloc(nv));
    k_jacobi_dinv<<<(nv + 255) / 256, 256, 0, st>>>(sys.A.view64(), sys.dinv.p,
                                                   mixed ? sys.dinv32.p : nullptr);
    MP_CHECK_LAUNCH();
    if (cfg.precond == MP_PRECOND_AMG) {
        MP_TRY(amg_create(&sys.amg, sys.A, cfg,
                          mixed ? AMG_F32 : (cfg.precision == MP_MG32 ? AMG_MG32 : AMG_F64), st));
    }
    if (cfg.precond == MP_PRECOND_SOR)
        MP_TRY(sor_setup(*this, st));
    MP_TRY(W.alloc(nv, bordered, mixed, cfg.precond == MP_PRECOND_AMG));
    MP_TRY(defl_setup(*this, c, db.p, hb, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

Ppe::~Ppe() {
    graph.reset();
    if (sys.amg)
        amg_destroy(sys.amg);
    if (sor)
        sor_destroy(sor);
    if (capture_stream)
        cudaStreamDestroy(capture_stream);
}

int solver_cfg_check(const mp_solver_cfg &c) {
    if (c.tol <= 0 || c.maxit <= 0)
        return fail(MP_BAD_ARG, "solver tolerance and maxit must be positive");
    if (c.precision != MP_FP64 && c.precision != MP_FP32 && c.precision != MP_MG32)
        return fail(MP_BAD_ARG, "precision must be MP_FP64, MP_FP32 or MP_MG32");
    if (c.precond < MP_PRECOND_NONE || c.precond > MP_PRECOND_SOR)
        return fail(MP_BAD_ARG, "unknown preconditioner %d", c.precond);
    if (c.precond == MP_PRECOND_SOR && c.precision != MP_FP64)
        return fail(MP_BAD_ARG, "the sor solver type runs in FP64 only");
    if (c.precond == MP_PRECOND_SOR && !(c.sor_omega > 0.0 && c.sor_omega < 2.0))
        return fail(MP_BAD_ARG, "sor_omega must lie in (0, 2), got %g", c.sor_omega);
    if (c.guess_vectors < 0 || c.guess_vectors > 8)
        return fail(MP_BAD_ARG, "guess_vectors must be 1-8 (0 for the default 8), got %d",
                    c.guess_vectors);
    if (c.precision == MP_MG32 && c.precond != MP_PRECOND_AMG)
        return fail(MP_BAD_ARG, "MP_MG32 stores the multigrid preconditioner in FP32: it needs "
                                "MP_PRECOND_AMG");
    return MP_OK;
}

int integrator_cfg_check(const mp_solver_cfg &c) {
    MP_TRY(solver_cfg_check(c));
    if (c.precond == MP_PRECOND_SOR)
        return fail(MP_BAD_ARG, "the sor solver type is available through SOLVER (mp_ppe_*); the "
                                "time integrators need a Krylov solver type");
    return MP_OK;
}

Cfg Cfg::from(const mp_solver_cfg &c) {
    Cfg o;
    o.tol = c.tol;
    o.maxit = c.maxit;
    o.precond = c.precond;
    o.precision = c.precision;
    o.guess = c.guess;
    o.inner_tol = c.inner_tol > 0 ? c.inner_tol : 1e-3;
    o.max_refine = 12;
    o.amg_max_levels = c.amg_max_levels > 0 ? c.amg_max_levels : 12;
    o.amg_coarse_size = c.amg_coarse_size > 0 ? c.amg_coarse_size : 512;
    o.smoother_sweeps = c.smoother_sweeps > 0 ? c.smoother_sweeps : 1;
    o.cheb_lower = c.cheb_lower > 0 && c.cheb_lower < 1 ? c.cheb_lower : 1.0 / 12.0;
    o.guess_vectors = c.guess_vectors > 0 ? c.guess_vectors : 8;
    o.sor_omega = c.sor_omega > 0 && c.sor_omega < 2 ? c.sor_omega : 1.4;
    return o;
}

}  // namespace mp

using namespace mp;

extern "C" int mp_solver_cfg_default(mp_solver_cfg *c) {
    if (!c)
        return fail(MP_BAD_ARG, "null cfg");
    c->tol = 1e-8;
    c->maxit = 1000;
    c->precond = MP_PRECOND_AMG;
    c->precision = MP_FP64;
    c->guess = MP_GUESS_PREVIOUS;
    c->inner_tol = 1e-3;
    c->amg_max_levels = 12;
    c->amg_coarse_size = 512;
    c->smoother_sweeps = 1;
    c->cheb_lower = 1.0 / 12.0;
    c->guess_vectors = 8;
    c->sor_omega = 1.4;
    return MP_OK;
}

extern "C" int mp_ppe_create(mp_cloud c, const uint8_t *boundary, const uint8_t *dirichlet,
                             const double *normal, double unsteady, double conv, double diff,
                             const mp_solver_cfg *cfg, mp_ppe *out) {
    if (!c || !boundary || !dirichlet || !normal || !cfg || !out)
        return fail(MP_BAD_ARG, "mp_ppe_create: null argument");
    MP_TRY(solver_cfg_check(*cfg));
    mp_ppe p = new mp_ppe_s;
    int rc = p->P.create(c, boundary, dirichlet, normal, unsteady, conv, diff, *cfg, 0);
    if (rc != MP_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return MP_OK;
}

extern "C" int mp_ppe_system_size(mp_ppe p) { return p ? p->P.sys.nsys : -1; }

extern "C" int mp_ppe_solve(mp_ppe p, const double *rhs, double *x_inout, int *iters,
                            double *relres, double *abs_res, mp_stream s) {
    if (!p || !rhs || !x_inout)
        return fail(MP_BAD_ARG, "mp_ppe_solve: null argument");
    cudaStream_t st = S(s);
    Ppe &P = p->P;
    const size_t n = P.sys.nsys;
    MP_CUDA(cudaMemcpyAsync(P.W.b64.p, rhs, sizeof(double) * n, cudaMemcpyDefault, st));
    if (P.cfg.guess == MP_GUESS_ZERO)
        MP_CUDA(cudaMemsetAsync(P.W.x.p, 0, sizeof(double) * n, st));
    else
        MP_CUDA(cudaMemcpyAsync(P.W.x.p, x_inout, sizeof(double) * n, cudaMemcpyDefault, st));
    SolveStats ss;
    if (P.sor) {
        MP_TRY(sor_solve(P, st, &ss));
    } else {
        MP_TRY(P.solve_resident(st, p->use_graph));
    }
    MP_CUDA(cudaMemcpyAsync(x_inout, P.W.x.p, sizeof(double) * n, cudaMemcpyDefault, st));
    if (!P.sor)
        MP_TRY(P.read_stats(st, &ss));
    MP_CUDA(cudaStreamSynchronize(st));
    if (iters)
        *iters = ss.iters;
    if (relres)
        *relres = ss.relres;
    if (abs_res)
        *abs_res = ss.abs_res;
    if (ss.status == MP_NOT_CONVERGED)
        return fail(MP_NOT_CONVERGED,
                    "%s did not converge in %d %s, relative residual: %g",
                    P.sor ? "SOR" : "pressure solve", ss.iters, P.sor ? "sweeps" : "iterations",
                    ss.relres);
    if (ss.status != MP_OK)
        return fail(ss.status, "pressure solve failed (status %d), relative residual: %g",
                    ss.status, ss.relres);
    return MP_OK;
}

extern "C" int mp_ppe_destroy(mp_ppe p) {
    delete p;
    return MP_OK;
}
