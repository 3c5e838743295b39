// mp_fs1.cu -- FRACTIONAL_STEP_1 (fractional_step_1.cpp) resident on the GPU.
//
// One timestep (single_timestep_2d, :52-63):
//   calc_vel_hat  (:120-134)  src = rho(-u Gx q - v Gy q [- w Gz q]) + mu L q,
//                             q_hat = q + dt/rho (src | 1.5 src - 0.5 src_prev)
//   calc_pressure (:136-151)  b = (Gx_int u_hat + Gy_int v_hat [+ Gz w_hat]) rho/dt,
//                             boundary rows p_old (Dirichlet) or
//                             -rho ((q_old - q_hat) . n)/dt (Neumann), b[nv] = 0,
//                             then the pressure solve with p_old as initial guess
//   calc_vel_corr (:153-209)  q_new = q_hat - dt G p / rho; boundary rows without
//                             Dirichlet pressure: q_new = q_old (Dirichlet) or
//                             the normal-derivative row solved for q_new[i]
//   extras        (:211-222)  src_prev = src (Adams-Bashforth 2)
// The reference integrates 2D only; the 3D path adds the w component with the
// same steps.  Each kernel streams the stencil indices once for all the
// operators it applies.  With graphs enabled the whole step (including the
// solver's device-controlled while loop) is a single graph launch.
#include <cmath>
#include <cstring>
#include "mp_amg.cuh"
#include "mp_cloud.cuh"
#include "mp_mlp.cuh"
#include "mp_ppe.cuh"

namespace mp {

struct Fs1Const {
    double rho, mu, dt;
    int order, nv, K, bordered;
};

struct Vec3 {
    const double *q[3];
};
struct Vec3w {
    double *q[3];
};

__device__ __forceinline__ int fgwarp() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }

template <int DIM>
__global__ void __launch_bounds__(256)
    k_vel_hat(const int *__restrict__ cols, const double *__restrict__ g0,
              const double *__restrict__ g1, const double *__restrict__ g2,
              const double *__restrict__ lap, Vec3 vel, Vec3w hat, Vec3w hist, Fs1Const c,
              const int *step) {
    const int w = fgwarp(), lane = threadIdx.x & 31, K = c.K;
    if (w >= (c.nv + SLICE - 1) / SLICE)
        return;
    const size_t base = (size_t)w * K * SLICE + 2 * lane;
    // acc[op][component][row]: op 0..DIM-1 gradients, DIM Laplacian
    double acc[DIM + 1][DIM][2];
#pragma unroll
    for (int o = 0; o <= DIM; o++)
#pragma unroll
        for (int d = 0; d < DIM; d++)
            acc[o][d][0] = acc[o][d][1] = 0.0;
    const double *G[3] = {g0, g1, g2};
#pragma unroll 2
    for (int k = 0; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        const int2 cc = __ldcs(reinterpret_cast<const int2 *>(cols + o));
        double q0[DIM], q1[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            q0[d] = __ldg(vel.q[d] + cc.x);
            q1[d] = __ldg(vel.q[d] + cc.y);
        }
#pragma unroll
        for (int op = 0; op <= DIM; op++) {
            const double2 wv = __ldcs(reinterpret_cast<const double2 *>((op < DIM ? G[op] : lap) + o));
#pragma unroll
            for (int d = 0; d < DIM; d++) {
                acc[op][d][0] = fma(wv.x, q0[d], acc[op][d][0]);
                acc[op][d][1] = fma(wv.y, q1[d], acc[op][d][1]);
            }
        }
    }
    const bool euler = c.order == 1 || *step == 0;
    const double dtr = c.dt / c.rho;
    const int i0 = w * SLICE + 2 * lane;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = i0 + r;
        if (i >= c.nv)
            continue;
        double qi[DIM];
#pragma unroll
        for (int d = 0; d < DIM; d++)
            qi[d] = vel.q[d][i];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            double conv = -(qi[0] * acc[0][d][r]);
#pragma unroll
            for (int e = 1; e < DIM; e++)
                conv = conv - qi[e] * acc[e][d][r];
            const double src = c.rho * conv + c.mu * acc[DIM][d][r];
            double h;
            if (euler)
                h = qi[d] + dtr * src;
            else
                h = qi[d] + dtr * (1.5 * src - 0.5 * hist.q[d][i]);
            hat.q[d][i] = h;
            if (c.order == 2)
                hist.q[d][i] = src;
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(256)
    k_p_rhs(const int *__restrict__ cols, const double *__restrict__ g0,
            const double *__restrict__ g1, const double *__restrict__ g2, Vec3 hat, Vec3 vel,
            const uint8_t *__restrict__ bflag, const uint8_t *__restrict__ pdir,
            const double *__restrict__ normal, const double *p, double *b, Fs1Const c) {
    const int w = fgwarp(), lane = threadIdx.x & 31, K = c.K;
    if (w == 0 && lane == 0 && c.bordered)
        b[c.nv] = 0.0;
    if (w >= (c.nv + SLICE - 1) / SLICE)
        return;
    const size_t base = (size_t)w * K * SLICE + 2 * lane;
    const double *G[3] = {g0, g1, g2};
    double acc[DIM][2];
#pragma unroll
    for (int d = 0; d < DIM; d++)
        acc[d][0] = acc[d][1] = 0.0;
#pragma unroll 2
    for (int k = 0; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        const int2 cc = __ldcs(reinterpret_cast<const int2 *>(cols + o));
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const double2 wv = __ldcs(reinterpret_cast<const double2 *>(G[d] + o));
            acc[d][0] = fma(wv.x, __ldg(hat.q[d] + cc.x), acc[d][0]);
            acc[d][1] = fma(wv.y, __ldg(hat.q[d] + cc.y), acc[d][1]);
        }
    }
    const int i0 = w * SLICE + 2 * lane;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = i0 + r;
        if (i >= c.nv)
            continue;
        double v;
        if (!bflag[i]) {
            double s = acc[0][r];
#pragma unroll
            for (int d = 1; d < DIM; d++)
                s = s + acc[d][r];
            v = s * c.rho / c.dt;
        } else if (pdir[i]) {
            v = p[i];
        } else {
            double s = (vel.q[0][i] - hat.q[0][i]) * normal[(size_t)DIM * i];
#pragma unroll
            for (int d = 1; d < DIM; d++)
                s = s + (vel.q[d][i] - hat.q[d][i]) * normal[(size_t)DIM * i + d];
            v = -c.rho * s / c.dt;
        }
        b[i] = v;
    }
}

template <int DIM>
__global__ void __launch_bounds__(256)
    k_vel_corr(const int *__restrict__ cols, const double *__restrict__ g0,
               const double *__restrict__ g1, const double *__restrict__ g2, Vec3 hat, Vec3 vel_old,
               Vec3w vel_new, const double *__restrict__ p, const uint8_t *__restrict__ bflag,
               const uint8_t *__restrict__ pdir, const uint8_t *__restrict__ d0,
               const uint8_t *__restrict__ d1, const uint8_t *__restrict__ d2, Fs1Const c) {
    const int w = fgwarp(), lane = threadIdx.x & 31, K = c.K;
    if (w >= (c.nv + SLICE - 1) / SLICE)
        return;
    const size_t base = (size_t)w * K * SLICE + 2 * lane;
    const double *G[3] = {g0, g1, g2};
    const uint8_t *vd[3] = {d0, d1, d2};
    double acc[DIM][2];
#pragma unroll
    for (int d = 0; d < DIM; d++)
        acc[d][0] = acc[d][1] = 0.0;
#pragma unroll 2
    for (int k = 0; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        const int2 cc = __ldcs(reinterpret_cast<const int2 *>(cols + o));
        const double p0 = __ldg(p + cc.x), p1 = __ldg(p + cc.y);
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            const double2 wv = __ldcs(reinterpret_cast<const double2 *>(G[d] + o));
            acc[d][0] = fma(wv.x, p0, acc[d][0]);
            acc[d][1] = fma(wv.y, p1, acc[d][1]);
        }
    }
    const int i0 = w * SLICE + 2 * lane;
#pragma unroll
    for (int r = 0; r < 2; r++) {
        const int i = i0 + r;
        if (i >= c.nv)
            continue;
        const bool fix = bflag[i] && !pdir[i];
#pragma unroll
        for (int d = 0; d < DIM; d++) {
            double q = hat.q[d][i] - (c.dt * acc[d][r]) / c.rho;
            if (fix && vd[d][i])
                q = vel_old.q[d][i];
            vel_new.q[d][i] = q;
        }
    }
}

// normal-derivative velocity rows (:166-181): q[i] = -sum_{j != i} c_ij q[j] / c_ii
template <int DIM>
__global__ void k_vel_neumann(int nb, const int *__restrict__ rows, const int *__restrict__ cols,
                              const double *__restrict__ g0, const double *__restrict__ g1,
                              const double *__restrict__ g2, const double *__restrict__ normal,
                              const uint8_t *__restrict__ d0, const uint8_t *__restrict__ d1,
                              const uint8_t *__restrict__ d2, Vec3w vel_new, int K) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nb)
        return;
    const int i = rows[t];
    const double *G[3] = {g0, g1, g2};
    const uint8_t *vd[3] = {d0, d1, d2};
#pragma unroll
    for (int d = 0; d < DIM; d++) {
        if (vd[d][i])
            continue;
        double rhs = 0.0, diag = 0.0;
        for (int k = 0; k < K; k++) {
            const size_t o = ell_index(i, k, K);
            const int j = cols[o];
            double cf = G[0][o] * normal[(size_t)DIM * i];
#pragma unroll
            for (int e = 1; e < DIM; e++)
                cf = cf + G[e][o] * normal[(size_t)DIM * i + e];
            if (j == i)
                diag = cf;
            else
                rhs = rhs - cf * vel_new.q[d][j];
        }
        vel_new.q[d][i] = rhs / diag;
    }
}

__global__ void k_step_log(int *step, const BicgScalars *S, double *log, int cap, const double *x,
                           int nv, int bordered, int mixed) {
    const int s = *step;
    double *e = log + MP_LOG_FIELDS * (size_t)(s % cap);
    // iterations, a last half iteration counted as 0.5
    e[0] = mixed ? S->total_inner - 0.5 * S->half_total : S->it - 0.5 * S->half;
    e[1] = S->b64_sq > 0 ? sqrt(S->rr_true / S->b64_sq) : 0.0;
    e[2] = sqrt(S->rr_true);
    e[3] = bordered ? x[nv] : 0.0;
    e[4] = S->relres0;
    e[5] = mixed ? S->outer_it : 0;
    e[6] = S->guess_theta;
    e[7] = 0.0;
    *step = s + 1;
}

// start of the guess stage: pcur = p^n (x on entry), then the non-learned guesses
__global__ void k_guess(int nsys, int mode, double *x, double *pcur, const double *ph1,
                        const int *step) {
    const int stride = gridDim.x * blockDim.x;
    const bool have_prev = *step >= 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride) {
        const double pn = x[i];
        pcur[i] = pn;
        if (mode == MP_GUESS_ZERO)
            x[i] = 0.0;
        else if (mode == MP_GUESS_EXTRAPOLATE && have_prev)
            x[i] = 2.0 * pn - ph1[i];
    }
}

// end of a step: p^{n-2} <- p^{n-1}, p^{n-1} <- p^n
__global__ void k_hist_rotate(int nsys, const double *pcur, double *ph1, double *ph2) {
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += stride) {
        ph2[i] = ph1[i];
        ph1[i] = pcur[i];
    }
}

// ------------------------------------------------------------ projection guess
// Fischer's projection of successive right-hand sides: with D_j the last m <= 8
// pressure increments and W_j = A D_j (= b_j - b_{j-1}: each p^{j+1} solved A p = b_j to the
// tolerance), the guess p^n + sum_j c_j D_j minimises ||(b_n - b_{n-1}) - sum_j
// c_j W_j|| = ||b_n - A(p^n + sum c_j D_j)|| up to the tolerance.  The Gram matrix
// G_jl = W_j . W_l of the ring's images is kept on the device: a pushed pair adds
// its row (k_proj_push), so a step's solve forms only the m right-hand-side products
// W_j . (b_n - b_{n-1}) and its last block solves the normalised system (with a
// small ridge: successive increments are nearly parallel).
constexpr int PROJ_MAX = 8;

__global__ void __launch_bounds__(256)
    k_proj_solve(int nsys, const double *b, const double *bprev, const double *W,
                 const double *Gm, int *state, double *coef, double *partials, unsigned *ticket) {
    __shared__ double red[32 * PROJ_MAX];
    const int cnt = state[0];
    double acc[PROJ_MAX];
#pragma unroll
    for (int q = 0; q < PROJ_MAX; q++)
        acc[q] = 0.0;
    if (cnt > 0) {
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += gridDim.x * blockDim.x) {
            const double r = b[i] - bprev[i];
#pragma unroll
            for (int j = 0; j < PROJ_MAX; j++)
                if (j < cnt)
                    acc[j] = fma(W[(size_t)j * nsys + i], r, acc[j]);
        }
    }
    if (grid_reduce<PROJ_MAX>(acc, partials, ticket, red) && threadIdx.x == 0) {
        double G[PROJ_MAX][PROJ_MAX], h[PROJ_MAX], c[PROJ_MAX], sc[PROJ_MAX];
        const int m = cnt > 0 ? cnt : 0;
        for (int j = 0; j < m; j++)
            for (int l = 0; l < m; l++)
                G[j][l] = Gm[j * PROJ_MAX + l];
        bool ok = m > 0;
        for (int j = 0; j < m; j++) {
            sc[j] = G[j][j] > 0 ? 1.0 / sqrt(G[j][j]) : 0.0;
            ok = ok && G[j][j] > 0;
        }
        if (ok) {  // Cholesky of the normalised Gram matrix + 1e-12 ridge
            double L[PROJ_MAX][PROJ_MAX];
            for (int j = 0; j < m; j++) {
                h[j] = acc[j] * sc[j];
                for (int l = 0; l <= j; l++) {
                    double v = G[j][l] * sc[j] * sc[l] + (j == l ? 1e-12 : 0.0);
                    for (int k = 0; k < l; k++)
                        v -= L[j][k] * L[l][k];
                    if (j == l) {
                        if (!(v > 0)) {
                            ok = false;
                            break;
                        }
                        L[j][j] = sqrt(v);
                    } else {
                        L[j][l] = v / L[l][l];
                    }
                }
                if (!ok)
                    break;
            }
            if (ok) {
                for (int j = 0; j < m; j++) {  // L y = h
                    double v = h[j];
                    for (int k = 0; k < j; k++)
                        v -= L[j][k] * c[k];
                    c[j] = v / L[j][j];
                }
                for (int j = m - 1; j >= 0; j--) {  // L^T z = y
                    double v = c[j];
                    for (int k = j + 1; k < m; k++)
                        v -= L[k][j] * c[k];
                    c[j] = v / L[j][j];
                }
            }
        }
        for (int j = 0; j < PROJ_MAX; j++) {
            const double v = (ok && j < m) ? c[j] * sc[j] : 0.0;
            coef[j] = isfinite(v) ? v : 0.0;
        }
    }
}

// x = p^n + sum_j coef_j D_j (x holds p^n on entry)
__global__ void k_proj_apply(int nsys, double *x, const double *D, const double *coef,
                             const int *state) {
    const int cnt = state[0];
    if (cnt <= 0)
        return;
    double c[PROJ_MAX];
#pragma unroll
    for (int j = 0; j < PROJ_MAX; j++)
        c[j] = j < cnt ? coef[j] : 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += gridDim.x * blockDim.x) {
        double v = x[i];
#pragma unroll
        for (int j = 0; j < PROJ_MAX; j++)
            if (j < cnt)
                v = fma(c[j], D[(size_t)j * nsys + i], v);
        x[i] = v;
    }
}

// after the solve: the new increment and its image into the ring slot at the head,
// and that image's row of the Gram matrix against every slot holding a pair (slots
// fill from 0, so while the ring is filling they are 0..head); the first step after
// a restart only records the right-hand side
__global__ void __launch_bounds__(256)
    k_proj_push(int nsys, const double *x, const double *pcur, const double *b, double *bprev,
                double *D, double *W, const int *state, int m, double *Gm, double *partials,
                unsigned *ticket) {
    __shared__ double red[32 * PROJ_MAX];
    const int cnt = state[0], head = state[1];
    const int nval = cnt < 0 ? 0 : min(cnt + 1, m);
    double acc[PROJ_MAX];
#pragma unroll
    for (int q = 0; q < PROJ_MAX; q++)
        acc[q] = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nsys; i += gridDim.x * blockDim.x) {
        const double bi = b[i];
        if (cnt >= 0) {
            const double w = bi - bprev[i];
            D[(size_t)head * nsys + i] = x[i] - pcur[i];
            W[(size_t)head * nsys + i] = w;
#pragma unroll
            for (int j = 0; j < PROJ_MAX; j++)
                if (j < nval)
                    acc[j] = fma(w, j == head ? w : W[(size_t)j * nsys + i], acc[j]);
        }
        bprev[i] = bi;
    }
    if (cnt >= 0 && grid_reduce<PROJ_MAX>(acc, partials, ticket, red) && threadIdx.x == 0)
        for (int j = 0; j < nval; j++)
            Gm[head * PROJ_MAX + j] = Gm[j * PROJ_MAX + head] = acc[j];
}

// the ring holds m pairs
__global__ void k_proj_advance(int *state, int m) {
    if (state[0] >= 0)
        state[1] = (state[1] + 1) % m;
    state[0] = state[0] < 0 ? 0 : min(state[0] + 1, m);
}

// the projected and the learned guesses keep the increment history
static bool uses_projection(int guess) {
    return guess == MP_GUESS_PROJECT || guess == MP_GUESS_LEARNED;
}

// distance from each node to its nearest stencil member
__global__ void k_spacing(int nv, int dim, int K, const int *cols, const double *xyz, float *h) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    double best = 1e300;
    for (int k = 0; k < K; k++) {
        const int j = cols[ell_index(i, k, K)];
        if (j == i)
            continue;
        double d2 = 0;
        for (int e = 0; e < dim; e++) {
            const double t = xyz[(size_t)i * dim + e] - xyz[(size_t)j * dim + e];
            d2 += t * t;
        }
        best = fmin(best, d2);
    }
    h[i] = (float)sqrt(best);
}

}  // namespace mp

using namespace mp;

struct mp_fs1_s {
    mp_cloud c = nullptr;
    int nv = 0, K = 0, dim = 0;
    Fs1Const k{};
    dbuf<uint8_t> bflag, vdir[3], pdir;
    dbuf<double> normal;
    dbuf<int> nrows;  // boundary rows that need the Neumann velocity solve
    int n_neumann = 0;
    dbuf<double> vel[2][3], hat[3], hist[3];
    Ppe P;
    dbuf<int> step;
    dbuf<double> log;
    int log_cap = 4096;
    int guess = MP_GUESS_PREVIOUS;
    // pressure history for the extrapolated and learned guesses
    dbuf<double> pcur, ph1, ph2, norms;
    dbuf<double> corr, flt1, flt_scale;  // learned correction and its coarse-level filter
    // projection guess: the last proj_m increments D_j = p^{j+1} - p^j, their images
    // W_j = A D_j = b_j - b_{j-1}, the previous right-hand side, and on the device the
    // number of valid columns (-1: no previous right-hand side yet), the ring head and
    // the coefficients of the last guess
    dbuf<double> pD, pW, pbprev, pcoef, ppart, pG;
    int proj_m = 0;    // ring length (pairs kept)
    dbuf<int> pstate;  // [0] valid columns, [1] ring head
    dbuf<unsigned> pticket;
    // learned guess
    Mlp *mlp = nullptr;
    dbuf<float> hloc;
    dbuf<int> sidx;
    int nsample = 0, cap_steps = 0, collect = 0;
    dbuf<uint16_t> sX;
    dbuf<float> st;
    GraphExec graph[2];
    int kcounts[3] = {0, 0, 0};  // kernels per step / per sweep / per refinement sweep
    int cur = 0;
    int use_graph = 1;
};

namespace mp {

static MlpFields fs1_fields(mp_fs1_s *f) {
    const CloudView cv = cloud_view(f->c);
    MlpFields F;
    F.nv = f->nv;
    F.K = f->K;
    F.cols = cv.cols;
    F.b = f->P.W.b64.p;
    F.pcur = f->pcur.p;
    F.ph1 = f->ph1.p;
    F.ph2 = f->ph2.p;
    F.hloc = f->hloc.p;
    F.bflag = f->bflag.p;
    F.norms = f->norms.p;
    return F;
}

static int fs1_issue_pre(mp_fs1_s *f, int cur, cudaStream_t s) {
    CloudView cv = cloud_view(f->c);
    const unsigned nb = (unsigned)(((f->nv + SLICE - 1) / SLICE + 7) / 8);
    Vec3 vel{}, hatc{};
    Vec3w hat{}, hist{};
    for (int d = 0; d < f->dim; d++) {
        vel.q[d] = f->vel[cur][d].p;
        hat.q[d] = f->hat[d].p;
        hatc.q[d] = f->hat[d].p;
        hist.q[d] = f->hist[d].p;
    }
    if (f->dim == 2) {
        k_vel_hat<2><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], nullptr, cv.w[3], vel, hat, hist,
                                         f->k, f->step.p);
        MP_CHECK_LAUNCH();
        k_p_rhs<2><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], nullptr, hatc, vel, f->bflag.p,
                                       f->pdir.p, f->normal.p, f->P.W.x.p, f->P.W.b64.p, f->k);
    } else {
        k_vel_hat<3><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], cv.w[2], cv.w[3], vel, hat, hist,
                                         f->k, f->step.p);
        MP_CHECK_LAUNCH();
        k_p_rhs<3><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], cv.w[2], hatc, vel, f->bflag.p,
                                       f->pdir.p, f->normal.p, f->P.W.x.p, f->P.W.b64.p, f->k);
    }
    MP_CHECK_LAUNCH();
    if (f->guess != MP_GUESS_PREVIOUS || f->collect) {
        const int ns = f->P.sys.nsys;
        // the learned guess starts from the projection (every entry, the border too)
        const int gmode = f->guess == MP_GUESS_LEARNED ? MP_GUESS_PROJECT : f->guess;
        k_guess<<<(unsigned)std::min((ns + 255) / 256, sm_count() * 4), 256, 0, s>>>(
            ns, gmode, f->P.W.x.p, f->pcur.p, f->ph1.p, f->step.p);
        MP_CHECK_LAUNCH();
        if (uses_projection(f->guess)) {
            const unsigned g = (unsigned)std::min((ns + 255) / 256, sm_count() * 4);
            k_proj_solve<<<g, 256, 0, s>>>(ns, f->P.W.b64.p, f->pbprev.p, f->pW.p, f->pG.p,
                                           f->pstate.p, f->pcoef.p, f->ppart.p, f->pticket.p);
            MP_CHECK_LAUNCH();
            k_proj_apply<<<g, 256, 0, s>>>(ns, f->P.W.x.p, f->pD.p, f->pcoef.p, f->pstate.p);
            MP_CHECK_LAUNCH();
        }
        if (f->guess == MP_GUESS_LEARNED) {
            const MlpFields F = fs1_fields(f);
            MP_TRY(mlp_norms(F, f->norms.p, f->P.W.partials.p, f->P.W.ticket.p, s));
            // projection + the predicted second difference, low-pass filtered through
            // the first multigrid level where there is one (the pointwise noise of the
            // network would otherwise dominate the residual of the guess) and weighted
            // to minimise the guess's residual: x += theta corr, theta = 0 unless the
            // correction removes a tenth of the squared residual
            MP_TRY(mlp_predict_fields(*f->mlp, F, f->P.W.x.p, f->corr.p, f->step.p, s));
            if (f->flt_scale.p)
                MP_TRY(amg_filter(*f->P.sys.amg, f->corr.p, f->flt1.p, f->flt_scale.p,
                                  f->corr.p, s));
            MP_TRY(f->P.issue_guess_min_residual(f->corr.p, s));
        }
    }
    return MP_OK;
}

static int fs1_issue_post(mp_fs1_s *f, int cur, cudaStream_t s) {
    CloudView cv = cloud_view(f->c);
    const unsigned nb = (unsigned)(((f->nv + SLICE - 1) / SLICE + 7) / 8);
    const int nxt = 1 - cur;
    Vec3 hat{}, vo{};
    Vec3w vn{};
    for (int d = 0; d < f->dim; d++) {
        hat.q[d] = f->hat[d].p;
        vo.q[d] = f->vel[cur][d].p;
        vn.q[d] = f->vel[nxt][d].p;
    }
    const uint8_t *d2 = f->dim == 3 ? f->vdir[2].p : f->vdir[0].p;
    if (f->dim == 2)
        k_vel_corr<2><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], nullptr, hat, vo, vn, f->P.W.x.p,
                                          f->bflag.p, f->pdir.p, f->vdir[0].p, f->vdir[1].p, d2, f->k);
    else
        k_vel_corr<3><<<nb, 256, 0, s>>>(cv.cols, cv.w[0], cv.w[1], cv.w[2], hat, vo, vn, f->P.W.x.p,
                                          f->bflag.p, f->pdir.p, f->vdir[0].p, f->vdir[1].p, d2, f->k);
    MP_CHECK_LAUNCH();
    if (f->n_neumann > 0) {
        const unsigned bb = (unsigned)((f->n_neumann + 127) / 128);
        if (f->dim == 2)
            k_vel_neumann<2><<<bb, 128, 0, s>>>(f->n_neumann, f->nrows.p, cv.cols, cv.w[0], cv.w[1],
                                                 nullptr, f->normal.p, f->vdir[0].p, f->vdir[1].p,
                                                 d2, vn, f->K);
        else
            k_vel_neumann<3><<<bb, 128, 0, s>>>(f->n_neumann, f->nrows.p, cv.cols, cv.w[0], cv.w[1],
                                                 cv.w[2], f->normal.p, f->vdir[0].p, f->vdir[1].p,
                                                 d2, vn, f->K);
        MP_CHECK_LAUNCH();
    }
    if (f->collect) {  // samples for the learned guess: features of this step, solved increment
        const MlpFields F = fs1_fields(f);
        if (f->guess != MP_GUESS_LEARNED)
            MP_TRY(mlp_norms(F, f->norms.p, f->P.W.partials.p, f->P.W.ticket.p, s));
        MP_TRY(mlp_collect(F, f->sidx.p, f->nsample, f->P.W.x.p, f->sX.p, f->st.p, f->step.p,
                           f->cap_steps, s));
    }
    if (uses_projection(f->guess)) {
        const int ns = f->P.sys.nsys;
        const unsigned g = (unsigned)std::min((ns + 255) / 256, sm_count() * 4);
        k_proj_push<<<g, 256, 0, s>>>(ns, f->P.W.x.p, f->pcur.p, f->P.W.b64.p, f->pbprev.p,
                                      f->pD.p, f->pW.p, f->pstate.p, f->proj_m, f->pG.p,
                                      f->ppart.p, f->pticket.p);
        MP_CHECK_LAUNCH();
        k_proj_advance<<<1, 1, 0, s>>>(f->pstate.p, f->proj_m);
        MP_CHECK_LAUNCH();
    }
    if (f->guess != MP_GUESS_PREVIOUS || f->collect) {
        const int ns = f->P.sys.nsys;
        k_hist_rotate<<<(unsigned)std::min((ns + 255) / 256, sm_count() * 4), 256, 0, s>>>(
            ns, f->pcur.p, f->ph1.p, f->ph2.p);
        MP_CHECK_LAUNCH();
    }
    k_step_log<<<1, 1, 0, s>>>(f->step.p, f->P.W.scal.p, f->log.p, f->log_cap, f->P.W.x.p, f->nv,
                               f->P.sys.bordered, f->P.cfg.precision == MP_FP32);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

static int fs1_step_once(mp_fs1_s *f, bool graph, cudaStream_t s) {
    const int cur = f->cur;
    if (graph) {
        GraphExec &G = f->graph[cur];
        if (!G.e) {
            GraphBuilder gb;
            MP_TRY(gb.init_root(f->P.cap_stream()));
            int counts[3] = {0, 0, 0};
            gb.counts = counts;
            int rc = gb.captured([&](cudaStream_t cs) { return fs1_issue_pre(f, cur, cs); });
            if (rc == MP_OK)
                rc = f->P.build_solve_graph(gb);
            if (rc == MP_OK)
                rc = gb.captured([&](cudaStream_t cs) { return fs1_issue_post(f, cur, cs); });
            if (rc != MP_OK) {
                if (gb.g)
                    cudaGraphDestroy(gb.g);
                return rc;
            }
            MP_TRY(G.instantiate(gb));
            for (int q = 0; q < 3; q++)
                f->kcounts[q] = counts[q];
        }
        MP_TRY(G.launch(s));
    } else {
        MP_TRY(fs1_issue_pre(f, cur, s));
        MP_TRY(f->P.solve_eager(s));
        MP_TRY(fs1_issue_post(f, cur, s));
    }
    f->cur = 1 - cur;
    return MP_OK;
}

}  // namespace mp

// storage of the projection guess, its history emptied (the first step only
// records its right-hand side)
static int proj_reserve(mp_fs1 f) {
    const size_t ns = (size_t)f->P.sys.nsys;
    const int m = std::min(std::max(f->P.cfg.guess_vectors, 1), PROJ_MAX);
    if (!f->pD.p || f->proj_m != m) {
        f->proj_m = m;
        MP_TRY(f->pD.alloc(ns * m));
        MP_TRY(f->pW.alloc(ns * m));
        MP_TRY(f->pbprev.alloc(ns));
        MP_TRY(f->pcoef.alloc(PROJ_MAX));
        MP_TRY(f->ppart.alloc((size_t)PROJ_MAX * sm_count() * 4 + 64));
        MP_TRY(f->pG.alloc(PROJ_MAX * PROJ_MAX));
        MP_CUDA(cudaMemset(f->pG.p, 0, sizeof(double) * PROJ_MAX * PROJ_MAX));
        MP_TRY(f->pticket.alloc(1));
        MP_TRY(f->pstate.alloc(2));
        MP_CUDA(cudaMemset(f->pticket.p, 0, sizeof(unsigned)));
        MP_CUDA(cudaMemset(f->pcoef.p, 0, sizeof(double) * PROJ_MAX));
    }
    const int st[2] = {-1, 0};
    MP_CUDA(cudaMemcpy(f->pstate.p, st, sizeof(st), cudaMemcpyHostToDevice));
    return MP_OK;
}

extern "C" int mp_fs1_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                             const uint8_t *u_dir, const uint8_t *v_dir, const uint8_t *w_dir,
                             const uint8_t *p_dir, const mp_fs1_cfg *cfg,
                             const mp_solver_cfg *solver, mp_fs1 *out) {
    if (!c || !boundary || !normal || !u_dir || !v_dir || !p_dir || !cfg || !solver || !out)
        return fail(MP_BAD_ARG, "mp_fs1_create: null argument");
    int nv, n, dim;
    MP_TRY(mp_cloud_info(c, &nv, &n, &dim));
    if (dim == 3 && !w_dir)
        return fail(MP_BAD_ARG, "3D fractional step needs w_dirichlet");
    // fractional_step_1.cpp:78-102 (check_bc)
    std::vector<uint8_t> hu(nv), hv(nv), hw(nv, 1), hp(nv), hb(nv);
    MP_CUDA(cudaMemcpy(hu.data(), u_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hv.data(), v_dir, nv, cudaMemcpyDefault));
    if (dim == 3)
        MP_CUDA(cudaMemcpy(hw.data(), w_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hp.data(), p_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hb.data(), boundary, nv, cudaMemcpyDefault));
    long su = 0, sv = 0, sw = 0;
    for (int i = 0; i < nv; i++) {
        su += hu[i];
        sv += hv[i];
        sw += hw[i];
    }
    if (su == 0)
        return fail(MP_BAD_ARG, "Setting u_dirichlet_flag to full Neumann BC is not permitted");
    if (sv == 0)
        return fail(MP_BAD_ARG, "Setting v_dirichlet_flag to full Neumann BC is not permitted");
    if (dim == 3 && sw == 0)
        return fail(MP_BAD_ARG, "Setting w_dirichlet_flag to full Neumann BC is not permitted");
    if (cfg->rho < 0 || cfg->mu < 0)
        return fail(MP_BAD_ARG, "Some parameters are not set; rho: %g, mu: %g", cfg->rho, cfg->mu);
    if (cfg->temporal_order != 1 && cfg->temporal_order != 2)
        return fail(MP_BAD_ARG, "temporal_order should be either '1' or '2'; current value: %d",
                    cfg->temporal_order);
    if (!(cfg->dt > 0))
        return fail(MP_BAD_ARG, "dt must be positive");
    MP_TRY(integrator_cfg_check(*solver));
    mp_fs1 f = new mp_fs1_s;
    f->c = c;
    f->nv = nv;
    f->K = n;
    f->dim = dim;
    auto bail = [&](int rc) {
        delete f;
        return rc;
    };
    int rc = f->P.create(c, boundary, p_dir, normal, 0.0, 0.0, 1.0, *solver, 0);
    if (rc != MP_OK)
        return bail(rc);
    f->k.rho = cfg->rho;
    f->k.mu = cfg->mu;
    f->k.dt = cfg->dt;
    f->k.order = cfg->temporal_order;
    f->k.nv = nv;
    f->k.K = n;
    f->k.bordered = f->P.sys.bordered;
    const uint8_t *dirs[3] = {u_dir, v_dir, w_dir};
    if ((rc = f->bflag.alloc(nv)) || (rc = f->pdir.alloc(nv)) || (rc = f->normal.alloc((size_t)nv * dim)))
        return bail(rc);
    cudaMemcpy(f->bflag.p, hb.data(), nv, cudaMemcpyHostToDevice);
    cudaMemcpy(f->pdir.p, hp.data(), nv, cudaMemcpyHostToDevice);
    cudaMemcpy(f->normal.p, normal, sizeof(double) * nv * dim, cudaMemcpyDefault);
    for (int d = 0; d < dim; d++) {
        if ((rc = f->vdir[d].alloc(nv)))
            return bail(rc);
        cudaMemcpy(f->vdir[d].p, dirs[d], nv, cudaMemcpyDefault);
        for (int b = 0; b < 2; b++)
            if ((rc = f->vel[b][d].alloc(nv)))
                return bail(rc);
        if ((rc = f->hat[d].alloc(nv)) || (rc = f->hist[d].alloc(nv)))
            return bail(rc);
        cudaMemset(f->hist[d].p, 0, sizeof(double) * nv);
        cudaMemset(f->vel[0][d].p, 0, sizeof(double) * nv);
        cudaMemset(f->vel[1][d].p, 0, sizeof(double) * nv);
    }
    std::vector<int> rows;
    for (int i = 0; i < nv; i++) {
        if (!hb[i] || hp[i])
            continue;
        bool need = !hu[i] || !hv[i] || (dim == 3 && !hw[i]);
        if (need)
            rows.push_back(i);
    }
    f->n_neumann = (int)rows.size();
    if (!rows.empty()) {
        if ((rc = f->nrows.alloc(rows.size())))
            return bail(rc);
        cudaMemcpy(f->nrows.p, rows.data(), sizeof(int) * rows.size(), cudaMemcpyHostToDevice);
    }
    const int ns = f->P.sys.nsys;
    if ((rc = f->step.alloc(1)) || (rc = f->log.alloc(MP_LOG_FIELDS * (size_t)f->log_cap)) ||
        (rc = f->pcur.alloc(ns)) || (rc = f->ph1.alloc(ns)) || (rc = f->ph2.alloc(ns)) ||
        (rc = f->norms.alloc(3)))
        return bail(rc);
    for (dbuf<double> *b : {&f->pcur, &f->ph1, &f->ph2})
        cudaMemset(b->p, 0, sizeof(double) * ns);
    f->guess = solver->guess;
    if (f->guess < MP_GUESS_PREVIOUS || f->guess > MP_GUESS_PROJECT)
        return bail(fail(MP_BAD_ARG, "unknown initial-guess mode %d", f->guess));
    if (f->guess == MP_GUESS_LEARNED)
        return bail(fail(MP_BAD_ARG, "the learned guess needs a network: mp_fs1_attach_mlp, then "
                                     "mp_fs1_set_guess"));
    if (f->guess == MP_GUESS_PROJECT && (rc = proj_reserve(f)) != MP_OK)
        return bail(rc);
    cudaMemset(f->step.p, 0, sizeof(int));
    cudaMemset(f->P.W.x.p, 0, sizeof(double) * f->P.sys.nsys);
    if (cudaDeviceSynchronize() != cudaSuccess)
        return bail(fail(MP_CUDA_ERROR, "mp_fs1_create: %s", cudaGetErrorString(cudaGetLastError())));
    *out = f;
    return MP_OK;
}

extern "C" int mp_fs1_system_size(mp_fs1 f) { return f ? f->P.sys.nsys : -1; }

extern "C" int mp_fs1_set_state(mp_fs1 f, const double *const *vel, const double *p, int it,
                                mp_stream s) {
    if (!f || !vel)
        return fail(MP_BAD_ARG, "mp_fs1_set_state: null argument");
    cudaStream_t st = S(s);
    int cur_step = 0;
    MP_CUDA(cudaMemcpyAsync(&cur_step, f->step.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    for (int d = 0; d < f->dim; d++)
        MP_CUDA(cudaMemcpyAsync(f->vel[f->cur][d].p, vel[d], sizeof(double) * f->nv,
                                cudaMemcpyDefault, st));
    if (p)
        MP_CUDA(cudaMemcpyAsync(f->P.W.x.p, p, sizeof(double) * f->P.sys.nsys, cudaMemcpyDefault, st));
    MP_CUDA(cudaStreamSynchronize(st));
    // The pressure history of the extrapolated and learned guesses survives a state
    // that continues at the current step index; any other index restarts it from p.
    if (it != cur_step) {
        const size_t bytes = sizeof(double) * f->P.sys.nsys;
        for (dbuf<double> *h : {&f->pcur, &f->ph1, &f->ph2})
            MP_CUDA(cudaMemcpyAsync(h->p, f->P.W.x.p, bytes, cudaMemcpyDeviceToDevice, st));
        if (f->pstate.p) {
            const int ps[2] = {-1, 0};
            MP_CUDA(cudaMemcpyAsync(f->pstate.p, ps, sizeof(ps), cudaMemcpyHostToDevice, st));
        }
    }
    MP_CUDA(cudaMemcpyAsync(f->step.p, &it, sizeof(int), cudaMemcpyHostToDevice, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

extern "C" int mp_fs1_get_state(mp_fs1 f, double *const *vel, double *p, mp_stream s) {
    if (!f)
        return fail(MP_BAD_ARG, "null fractional-step handle");
    cudaStream_t st = S(s);
    if (vel)
        for (int d = 0; d < f->dim; d++)
            if (vel[d])
                MP_CUDA(cudaMemcpyAsync(vel[d], f->vel[f->cur][d].p, sizeof(double) * f->nv,
                                        cudaMemcpyDefault, st));
    if (p)
        MP_CUDA(cudaMemcpyAsync(p, f->P.W.x.p, sizeof(double) * f->P.sys.nsys, cudaMemcpyDefault, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

extern "C" int mp_fs1_step(mp_fs1 f, int nsteps, int use_graph, mp_stream s) {
    if (!f || nsteps < 0)
        return fail(MP_BAD_ARG, "mp_fs1_step: bad arguments");
    for (int i = 0; i < nsteps; i++)
        MP_TRY(fs1_step_once(f, use_graph != 0, S(s)));
    return MP_OK;
}

extern "C" int mp_fs1_single_timestep(mp_fs1 f, double *const *vel_new, double *p_new,
                                      const double *const *vel_old, const double *p_old, int it,
                                      mp_stream s) {
    if (!f || !vel_new || !p_new || !vel_old || !p_old)
        return fail(MP_BAD_ARG, "mp_fs1_single_timestep: null argument");
    MP_TRY(mp_fs1_set_state(f, vel_old, p_old, it, s));
    MP_TRY(fs1_step_once(f, f->use_graph != 0, S(s)));
    MP_TRY(mp_fs1_get_state(f, vel_new, p_new, s));
    int iters;
    double rr;
    MP_TRY(mp_fs1_last_stats(f, &iters, &rr, nullptr, nullptr));
    if (!(rr <= f->P.cfg.tol))
        return fail(std::isfinite(rr) ? MP_NOT_CONVERGED : MP_NAN_DETECTED,
                    "pressure solve: relative residual %g after %d iterations", rr, iters);
    return MP_OK;
}

extern "C" int mp_fs1_last_stats(mp_fs1 f, int *iters, double *relres, double *abs_res,
                                 double *alpha) {
    if (!f)
        return fail(MP_BAD_ARG, "null fractional-step handle");
    MP_CUDA(cudaDeviceSynchronize());
    int step = 0;
    MP_CUDA(cudaMemcpy(&step, f->step.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (step <= 0)
        return fail(MP_BAD_ARG, "no step has been taken");
    double e[MP_LOG_FIELDS];
    MP_CUDA(cudaMemcpy(e, f->log.p + MP_LOG_FIELDS * (size_t)((step - 1) % f->log_cap), sizeof(e),
                       cudaMemcpyDeviceToHost));
    if (iters)
        *iters = (int)e[0];
    if (relres)
        *relres = e[1];
    if (abs_res)
        *abs_res = e[2];
    if (alpha)
        *alpha = e[3];
    return MP_OK;
}

extern "C" int mp_fs1_log(mp_fs1 f, int first, int count, double *out) {
    if (!f || !out || first < 0 || count < 0 || count > f->log_cap)
        return fail(MP_BAD_ARG, "mp_fs1_log: bad arguments");
    MP_CUDA(cudaDeviceSynchronize());
    int step = 0;
    MP_CUDA(cudaMemcpy(&step, f->step.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (first + count > step || first < step - f->log_cap)
        return fail(MP_BAD_ARG, "mp_fs1_log: steps %d..%d not in the log (last step %d)", first,
                    first + count - 1, step - 1);
    for (int i = 0; i < count; i++)
        MP_CUDA(cudaMemcpy(out + MP_LOG_FIELDS * (size_t)i,
                           f->log.p + MP_LOG_FIELDS * (size_t)((first + i) % f->log_cap),
                           MP_LOG_FIELDS * sizeof(double), cudaMemcpyDeviceToHost));
    return MP_OK;
}

static void fs1_invalidate(mp_fs1 f) {
    f->graph[0].reset();
    f->graph[1].reset();
    for (int q = 0; q < 3; q++)
        f->kcounts[q] = 0;
}

extern "C" int mp_fs1_attach_mlp(mp_fs1 f, mp_mlp m, int sample_nodes, int capacity_steps,
                                 int collect) {
    if (!f || !m || sample_nodes <= 0 || capacity_steps <= 0)
        return fail(MP_BAD_ARG, "mp_fs1_attach_mlp: bad arguments");
    MP_CUDA(cudaDeviceSynchronize());
    f->mlp = mlp_of(m);
    const int nv = f->nv;
    MP_TRY(mlp_reserve_fields(*f->mlp, nv));
    // node spacing feature: distance to the nearest stencil member over its mean
    MP_TRY(f->hloc.alloc(nv));
    {
        CloudView cv = cloud_view(f->c);
        k_spacing<<<(nv + 255) / 256, 256>>>(nv, f->dim, f->K, cv.cols, cloud_xyz(f->c), f->hloc.p);
        MP_CHECK_LAUNCH();
        std::vector<float> h(nv);
        MP_CUDA(cudaMemcpy(h.data(), f->hloc.p, sizeof(float) * nv, cudaMemcpyDeviceToHost));
        double mean = 0;
        for (float v : h)
            mean += v;
        mean /= nv;
        for (float &v : h)
            v = (float)(v / mean);
        MP_CUDA(cudaMemcpy(f->hloc.p, h.data(), sizeof(float) * nv, cudaMemcpyHostToDevice));
    }
    // a fixed pseudo-random sample of nodes whose features are recorded each step
    f->nsample = std::min(sample_nodes, nv);
    std::vector<int> all(nv);
    for (int i = 0; i < nv; i++)
        all[i] = i;
    uint64_t st = 0x2545F4914F6CDD1Dull;
    for (int i = 0; i < f->nsample; i++) {  // partial Fisher-Yates
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        const int j = i + (int)(st % (uint64_t)(nv - i));
        std::swap(all[i], all[j]);
    }
    std::sort(all.begin(), all.begin() + f->nsample);
    MP_TRY(f->sidx.alloc(f->nsample));
    MP_CUDA(cudaMemcpy(f->sidx.p, all.data(), sizeof(int) * f->nsample, cudaMemcpyHostToDevice));
    f->cap_steps = capacity_steps;
    MP_TRY(f->sX.alloc((size_t)capacity_steps * f->nsample * MLP_IN));
    MP_TRY(f->st.alloc((size_t)capacity_steps * f->nsample));
    f->collect = collect ? 1 : 0;
    MP_TRY(f->corr.alloc(nv));
    if (f->P.sys.amg && amg_filter_size(*f->P.sys.amg) > 0) {
        const int n1 = amg_filter_size(*f->P.sys.amg);
        MP_TRY(f->flt1.alloc(n1));
        MP_TRY(f->flt_scale.alloc(n1));
        MP_TRY(amg_filter_setup(*f->P.sys.amg, f->flt_scale.p, 0));
    }
    fs1_invalidate(f);
    return MP_OK;
}

extern "C" int mp_fs1_set_guess(mp_fs1 f, int guess) {
    if (!f || guess < MP_GUESS_PREVIOUS || guess > MP_GUESS_PROJECT)
        return fail(MP_BAD_ARG, "mp_fs1_set_guess: unknown mode %d", guess);
    if (guess == MP_GUESS_LEARNED && !f->mlp)
        return fail(MP_BAD_ARG, "the learned guess needs mp_fs1_attach_mlp first");
    if (guess != f->guess) {
        if (uses_projection(guess))
            MP_TRY(proj_reserve(f));
        f->guess = guess;
        fs1_invalidate(f);
    }
    return MP_OK;
}

extern "C" int mp_fs1_train_mlp(mp_fs1 f, int epochs, int batch, double lr, uint64_t seed,
                                double *loss) {
    if (!f || !f->mlp)
        return fail(MP_BAD_ARG, "mp_fs1_train_mlp: no network attached");
    MP_CUDA(cudaDeviceSynchronize());
    int step = 0;
    MP_CUDA(cudaMemcpy(&step, f->step.p, sizeof(int), cudaMemcpyDeviceToHost));
    const int steps = std::min(std::max(step - 2, 0), f->cap_steps);
    const int n = steps * f->nsample;
    if (n < batch)
        return fail(MP_BAD_ARG, "only %d samples recorded (batch %d)", n, batch);
    return mlp_train(*f->mlp, f->sX.p, f->st.p, n, epochs, batch, lr, seed, loss, 0);
}

extern "C" int mp_fs1_samples(mp_fs1 f, float *X, float *t, int *nodes, int cap, int *n) {
    if (!f || !n || cap < 0)
        return fail(MP_BAD_ARG, "mp_fs1_samples: bad arguments");
    if (!f->mlp)
        return fail(MP_BAD_ARG, "mp_fs1_samples: no network attached");
    MP_CUDA(cudaDeviceSynchronize());
    int step = 0;
    MP_CUDA(cudaMemcpy(&step, f->step.p, sizeof(int), cudaMemcpyDeviceToHost));
    const int rows = std::min(std::max(step - 2, 0), f->cap_steps) * f->nsample;
    *n = rows;
    const int m = std::min(rows, cap);
    if (m == 0)
        return MP_OK;
    if (X) {
        std::vector<uint16_t> h((size_t)m * MLP_IN);
        MP_CUDA(cudaMemcpy(h.data(), f->sX.p, h.size() * 2, cudaMemcpyDeviceToHost));
        for (size_t q = 0; q < h.size(); q++) {
            const uint32_t u = (uint32_t)h[q] << 16;
            std::memcpy(X + q, &u, 4);
        }
    }
    if (t)
        MP_CUDA(cudaMemcpy(t, f->st.p, sizeof(float) * m, cudaMemcpyDefault));
    if (nodes) {
        std::vector<int> idx(f->nsample);
        MP_CUDA(cudaMemcpy(idx.data(), f->sidx.p, sizeof(int) * f->nsample,
                           cudaMemcpyDeviceToHost));
        for (int r = 0; r < m; r++)
            nodes[r] = idx[r % f->nsample];
    }
    return MP_OK;
}

extern "C" int mp_fs1_kernel_counts(mp_fs1 f, int *fixed, int *per_sweep, int *per_refine) {
    if (!f)
        return fail(MP_BAD_ARG, "null fractional-step handle");
    // FP64: fixed + iters * per_sweep; mixed: fixed + outer * per_refine + inner * per_sweep
    const bool mixed = f->P.cfg.precision == MP_FP32;
    if (fixed)
        *fixed = f->kcounts[0];
    if (per_sweep)
        *per_sweep = mixed ? f->kcounts[2] : f->kcounts[1];
    if (per_refine)
        *per_refine = mixed ? f->kcounts[1] : 0;
    return MP_OK;
}

extern "C" int mp_fs1_destroy(mp_fs1 f) {
    delete f;
    return MP_OK;
}
