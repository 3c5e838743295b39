// mp_sis.cu -- SEMI_IMPLICIT_SPLIT_SOLVER (semi_implicit_split_solver.cpp) on the GPU.
//
// One timestep (single_timestep_2d, :376-421), starting from u = u_old,
// v = v_old, p = p_old, repeated for up to n_outer_iter outer iterations:
//   modify_vel_matrix (:218-243)  interior rows of the velocity matrices
//       -mu L + rho (u_i Gx + v_i Gy) + a1 rho/dt I  (a1 = 1 at it = 0, else 1.5)
//       from the current u, v; boundary rows stay identity (Dirichlet) or n . G
//   calc_vel (:73-129)            sources (rho/dt) u_old (BDF1) or
//       2 rho/dt u_old - 0.5 rho/dt u_old_old (BDF2), minus Gx_int p; boundary rows
//       u_old (Dirichlet) or 0; u, v solved from their current values
//   calc_pressure (:131-186)      p' from the pressure-correction equation with
//       source (Gx_int u + Gy_int v) a1 rho/dt and zero initial guess; p += p';
//       non-Dirichlet boundary p from the normal momentum balance
//   calc_vel_corr (:188-204)      u -= Gx_int p' dt/(a1 rho), v likewise
//   the L1 and max changes of u, v over the iteration decide the stop (:401-418).
// The velocity matrices change every outer iteration, so their solves use
// BiCGSTAB with the Jacobi preconditioner rebuilt from the new diagonal (the
// reference keeps an ILUT factorisation for precond_freq_it steps); the
// pressure correction uses the fractional step's pressure system (multigrid).
#include <algorithm>
#include <cmath>
#include <vector>
#include "mp_cloud.cuh"
#include "mp_ppe.cuh"

namespace mp {

struct SisConst {
    int nv, K;
    double rho, mu, dt;
};

// (row, slot) of a thread over the sliced storage
__device__ __forceinline__ bool ell_slot(size_t t, int nv, int K, int &row) {
    const size_t slice = t / ((size_t)K * SLICE);
    row = (int)(slice * SLICE + (t % SLICE));
    return row < nv;
}

// interior rows of both velocity matrices (modify_vel_matrix :229-242)
__global__ void k_sis_values(SisConst c, const int *cols, const double *gx, const double *gy,
                             const double *lap, const uint8_t *bflag, const double *u,
                             const double *v, double diag, double *Au, double *Av) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)ell_padded_rows(c.nv) * c.K)
        return;
    int row;
    if (!ell_slot(t, c.nv, c.K, row) || bflag[row])
        return;
    double val = -c.mu * lap[t];
    val = val + (u[row] * c.rho * gx[t]);
    val = val + (v[row] * c.rho * gy[t]);
    if (cols[t] == row)
        val = val + diag;
    Au[t] = val;
    Av[t] = val;
}

// sum_k w[i, k] x[cols[i, k]] over the sliced storage
__device__ __forceinline__ double row_apply(const int *cols, const double *w, int i, int K,
                                            const double *x) {
    const size_t base = (size_t)(i / SLICE) * K * SLICE + (i % SLICE);
    double s = 0.0;
    for (int k = 0; k < K; k++)
        s += w[base + (size_t)k * SLICE] * x[cols[base + (size_t)k * SLICE]];
    return s;
}

// calc_vel sources (:87-128 without the body force)
__global__ void k_sis_vel_source(SisConst c, const int *cols, const double *gx, const double *gy,
                                 const uint8_t *bflag, const uint8_t *udir, const uint8_t *vdir,
                                 const double *p, const double *uo, const double *vo,
                                 const double *uoo, const double *voo, int bdf1, double *su,
                                 double *sv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.nv)
        return;
    if (bflag[i]) {
        su[i] = udir[i] ? uo[i] : 0.0;
        sv[i] = vdir[i] ? vo[i] : 0.0;
        return;
    }
    const double gxp = row_apply(cols, gx, i, c.K, p), gyp = row_apply(cols, gy, i, c.K, p);
    const double r = c.rho / c.dt;
    if (bdf1) {
        su[i] = (r * uo[i]) - gxp;
        sv[i] = (r * vo[i]) - gyp;
    } else {  // -(a2 rho/dt) u_old - (a3 rho/dt) u_old_old, a2 = -2, a3 = 0.5
        su[i] = -((-2.0 * c.rho / c.dt) * uo[i]) - ((0.5 * c.rho / c.dt) * uoo[i]) - gxp;
        sv[i] = -((-2.0 * c.rho / c.dt) * vo[i]) - ((0.5 * c.rho / c.dt) * voo[i]) - gyp;
    }
}

// pressure-correction source (:137-141); boundary rows and the border entry 0
__global__ void k_sis_p_source(SisConst c, const int *cols, const double *gx, const double *gy,
                               const uint8_t *bflag, const double *u, const double *v, double coef,
                               int nsys, double *ps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsys)
        return;
    if (i >= c.nv || bflag[i]) {
        ps[i] = 0.0;
        return;
    }
    ps[i] = (row_apply(cols, gx, i, c.K, u) + row_apply(cols, gy, i, c.K, v)) * coef;
}

__global__ void k_sis_add(int n, double *p, const double *pp) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        p[i] += pp[i];
}

// non-Dirichlet boundary pressure from the normal momentum balance (:148-185).
// Boundary stencils hold interior nodes besides their own (cloud.cpp:624-640),
// so the rows are independent; `serial` runs them one after another in index
// order for clouds where a boundary stencil holds another boundary node.
__global__ void k_sis_p_boundary(SisConst c, const int *cols, const double *gx, const double *gy,
                                 const double *lap, const uint8_t *bflag, const uint8_t *pdir,
                                 const double *normal, const double *u, const double *v,
                                 const double *uo, const double *vo, const double *uoo,
                                 const double *voo, int bdf1, int serial, double *p) {
    const int first = serial ? 0 : blockIdx.x * blockDim.x + threadIdx.x;
    const int last = serial ? c.nv : first + 1;
    if (serial && (blockIdx.x | threadIdx.x))
        return;
    for (int i = first; i < last && i < c.nv; i++) {
        if (!bflag[i] || pdir[i])
            continue;
        const double gxu = row_apply(cols, gx, i, c.K, u), gyu = row_apply(cols, gy, i, c.K, u);
        const double gxv = row_apply(cols, gx, i, c.K, v), gyv = row_apply(cols, gy, i, c.K, v);
        const double lu = row_apply(cols, lap, i, c.K, u), lv = row_apply(cols, lap, i, c.K, v);
        const double r = c.rho / c.dt;
        double mx = -c.rho * (u[i] * gxu + v[i] * gyu) + c.mu * lu;
        double my = -c.rho * (u[i] * gxv + v[i] * gyv) + c.mu * lv;
        if (bdf1) {
            mx -= r * (u[i] - uo[i]);
            my -= r * (v[i] - vo[i]);
        } else {
            mx -= r * ((1.5 * u[i]) + (-2.0 * uo[i]) + (0.5 * uoo[i]));
            my -= r * ((1.5 * v[i]) + (-2.0 * vo[i]) + (0.5 * voo[i]));
        }
        const double nx = normal[2 * (size_t)i], ny = normal[2 * (size_t)i + 1];
        double rhs = (mx * nx) + (my * ny), diag = 0.0;
        const size_t base = (size_t)(i / SLICE) * c.K * SLICE + (i % SLICE);
        for (int k = 0; k < c.K; k++) {
            const size_t e = base + (size_t)k * SLICE;
            const int j = cols[e];
            const double cf = (gx[e] * nx) + (gy[e] * ny);
            if (j == i)
                diag = cf;
            else
                rhs = rhs - (cf * p[j]);
        }
        p[i] = rhs / diag;
    }
}

// calc_vel_corr: interior rows u -= Gx p' f, v -= Gy p' f
__global__ void k_sis_vel_corr(SisConst c, const int *cols, const double *gx, const double *gy,
                               const uint8_t *bflag, const double *pp, double f, double *u,
                               double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c.nv || bflag[i])
        return;
    u[i] = u[i] - row_apply(cols, gx, i, c.K, pp) * f;
    v[i] = v[i] - row_apply(cols, gy, i, c.K, pp) * f;
}

// per-block sum |du|, sum |dv|, max |du|, max |dv|
__global__ void k_sis_err(int nv, const double *u, const double *ui, const double *v,
                          const double *vi, double *part) {
    __shared__ double s[4][256];
    double a[4] = {0, 0, 0, 0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x) {
        const double du = fabs(u[i] - ui[i]), dv = fabs(v[i] - vi[i]);
        a[0] += du;
        a[1] += dv;
        a[2] = fmax(a[2], du);
        a[3] = fmax(a[3], dv);
    }
    for (int q = 0; q < 4; q++)
        s[q][threadIdx.x] = a[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w /= 2) {
        if ((int)threadIdx.x < w) {
            s[0][threadIdx.x] += s[0][threadIdx.x + w];
            s[1][threadIdx.x] += s[1][threadIdx.x + w];
            s[2][threadIdx.x] = fmax(s[2][threadIdx.x], s[2][threadIdx.x + w]);
            s[3][threadIdx.x] = fmax(s[3][threadIdx.x], s[3][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++)
            part[4 * (size_t)blockIdx.x + q] = s[q][0];
}

// Outer-iteration state on the device: the count, the L1 and max changes of the
// last iteration, and the first failed solve (0 none, 1 u, 2 v, 3 pressure) with
// its status, iterations and relative residual.
struct SisCtl {
    int outer, status, failed, iters;
    double relres, err[2];
    double itol;  // the stopping tolerance of the L1 change, written by the host per step
};

// status of a finished solve, as Ppe::read_stats reports it
__device__ int solve_status(const BicgScalars *S, double tol, double *relres) {
    const double rr = S->b64_sq > 0 ? sqrt(S->rr_true / S->b64_sq) : 0.0;
    int st = S->status;
    if (st == MP_OK && rr > tol && S->b64_sq > 0 && !(S->rr_true <= S->abs_tol2))
        st = MP_NOT_CONVERGED;
    if (st == MP_OK && !isfinite(rr))
        st = MP_NAN_DETECTED;
    *relres = rr;
    return st;
}

__global__ void k_sis_outer_init(SisCtl *ctl, cudaGraphConditionalHandle h) {
    ctl->outer = 0;
    ctl->status = MP_OK;
    ctl->failed = 0;
    ctl->iters = 0;
    ctl->relres = 0;
    ctl->err[0] = ctl->err[1] = 0;
    if (h)
        cudaGraphSetConditional(h, 1u);
}

// End of an outer iteration: the blocks' partials to [l1 error, max error]
// (:401-404), the three solves' statuses, and whether another iteration runs
// (:405-418: the L1 change is above the tolerance, fewer than n_outer iterations
// ran, and every solve succeeded).  One block of 256 threads.
__global__ void __launch_bounds__(256)
    k_sis_outer_end(int nb, const double *part, int nv, SisCtl *ctl, const BicgScalars *Su,
                    const BicgScalars *Sv, const BicgScalars *Sp, double tol_u, double tol_v,
                    double tol_p, int n_outer, cudaGraphConditionalHandle h) {
    __shared__ double sh[4][256];
    double a[4] = {0, 0, 0, 0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        a[0] += part[4 * (size_t)b];
        a[1] += part[4 * (size_t)b + 1];
        a[2] = fmax(a[2], part[4 * (size_t)b + 2]);
        a[3] = fmax(a[3], part[4 * (size_t)b + 3]);
    }
    for (int q = 0; q < 4; q++)
        sh[q][threadIdx.x] = a[q];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w /= 2) {
        if ((int)threadIdx.x < w) {
            sh[0][threadIdx.x] += sh[0][threadIdx.x + w];
            sh[1][threadIdx.x] += sh[1][threadIdx.x + w];
            sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][threadIdx.x + w]);
            sh[3][threadIdx.x] = fmax(sh[3][threadIdx.x], sh[3][threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x)
        return;
    const double l1 = sh[0][0] / (2.0 * nv) + sh[1][0] / (2.0 * nv);
    ctl->err[0] = l1;
    ctl->err[1] = sh[2][0] / 2.0 + sh[3][0] / 2.0;
    ctl->outer += 1;
    const BicgScalars *S[3] = {Su, Sv, Sp};
    const double tol[3] = {tol_u, tol_v, tol_p};
    for (int q = 0; q < 3 && ctl->status == MP_OK; q++) {
        double rr;
        const int st = solve_status(S[q], tol[q], &rr);
        if (st != MP_OK) {
            ctl->status = st;
            ctl->failed = q + 1;
            ctl->iters = S[q]->it;
            ctl->relres = rr;
        }
    }
    if (ctl->status == MP_OK && !isfinite(l1))
        ctl->status = MP_NAN_DETECTED;
    const bool more = ctl->status == MP_OK && l1 > ctl->itol && ctl->outer < n_outer;
    if (h)
        cudaGraphSetConditional(h, more ? 1u : 0u);
}

// IMPLICIT_SCALAR_TRANSPORT_SOLVER::modify_matrix (implicit_scalar_transport_solver.cpp:87-109):
// interior rows diff L + conv (u_i Gx + v_i Gy) + unsteady_factor unsteady I
__global__ void k_ist_values(int nv, int K, const int *cols, const double *gx, const double *gy,
                             const double *lap, const uint8_t *bflag, const double *u,
                             const double *v, double diff, double conv, double diag, double *A) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)ell_padded_rows(nv) * K)
        return;
    int row;
    if (!ell_slot(t, nv, K, row) || bflag[row])
        return;
    double val = diff * lap[t];
    val = val + (u[row] * conv * gx[t]);
    val = val + (v[row] * conv * gy[t]);
    if (cols[t] == row)
        val = val + diag;
    A[t] = val;
}

// single_timestep_2d source (:153-165): unsteady phi_old (BDF1) or
// -(a2 unsteady) phi_old - (a3 unsteady) phi_old_old; boundary rows phi_old
// (Dirichlet) or 0
__global__ void k_ist_source(int nv, const uint8_t *bflag, const uint8_t *dir, const double *po,
                             const double *poo, double unsteady, int bdf1, double *src) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    if (bflag[i])
        src[i] = dir[i] ? po[i] : 0.0;
    else if (bdf1)
        src[i] = unsteady * po[i];
    else
        src[i] = -((-2.0 * unsteady) * po[i]) - ((0.5 * unsteady) * poo[i]);
}

}  // namespace mp

using namespace mp;

struct mp_sis_s {
    mp_cloud c = nullptr;
    int nv = 0, K = 0, nsys = 0, n_outer = 1, serial_pb = 0;
    double rho = 1, mu = 0, dt = 0, itol = 0;
    dbuf<uint8_t> udir, vdir, pdir;
    dbuf<double> normal;
    Ppe U, V, P;
    dbuf<double> uo, vo, uoo, voo, pn, uit, vit, part;
    dbuf<SisCtl> ctl;
    int err_blocks = 0;
    bool use_graph = true;
    GraphExec graph[2];  // the outer loop of a BDF1 and of a BDF2 step
};

extern "C" int mp_sis_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                             const uint8_t *u_dir, const uint8_t *v_dir, const uint8_t *p_dir,
                             const mp_sis_cfg *cfg, const mp_solver_cfg *vel_solver,
                             const mp_solver_cfg *p_solver, mp_sis *out) {
    if (!c || !boundary || !normal || !u_dir || !v_dir || !p_dir || !cfg || !vel_solver ||
        !p_solver || !out)
        return fail(MP_BAD_ARG, "mp_sis_create: null argument");
    int nv, n, dim;
    MP_TRY(mp_cloud_info(c, &nv, &n, &dim));
    if (dim != 2)
        return fail(MP_BAD_ARG, "the semi-implicit split solver is 2D (single_timestep_2d)");
    if (cfg->rho < 0 || cfg->mu < 0 || !(cfg->dt > 0) || cfg->n_outer_iter < 1)
        return fail(MP_BAD_ARG, "mp_sis_create: rho, mu >= 0, dt > 0 and n_outer_iter >= 1 needed");
    if (vel_solver->precond == MP_PRECOND_AMG || vel_solver->precision != MP_FP64)
        return fail(MP_BAD_ARG, "the velocity matrices change every outer iteration: their solver "
                                "takes MP_PRECOND_JACOBI or MP_PRECOND_NONE in MP_FP64");
    MP_TRY(integrator_cfg_check(*vel_solver));
    MP_TRY(integrator_cfg_check(*p_solver));
    std::vector<uint8_t> hb(nv), hu(nv), hv(nv);
    MP_CUDA(cudaMemcpy(hb.data(), boundary, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hu.data(), u_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hv.data(), v_dir, nv, cudaMemcpyDefault));
    // check_bc (:52-71): full Neumann velocity is not permitted
    int su = 0, sv = 0;
    for (int i = 0; i < nv; i++) {
        su += hu[i] != 0;
        sv += hv[i] != 0;
    }
    if (su == 0 || sv == 0)
        return fail(MP_BAD_ARG, "full Neumann BC for a velocity component is not permitted "
                                "(sum of u_dirichlet %d, v_dirichlet %d)", su, sv);
    mp_sis_s *s = new mp_sis_s;
    auto bail = [&](int rc) {
        delete s;
        return rc;
    };
    s->c = c;
    s->nv = nv;
    s->K = n;
    s->rho = cfg->rho;
    s->mu = cfg->mu;
    s->dt = cfg->dt;
    s->n_outer = cfg->n_outer_iter;
    s->itol = cfg->iterative_tolerance;
    cudaStream_t st = 0;
    int rc;
    // solver_p.init(..., 0, 0, 1, ...) (:28): the Laplacian pressure system
    if ((rc = s->P.create(c, boundary, p_dir, normal, 0.0, 0.0, 1.0, *p_solver, st)) != MP_OK ||
        (rc = s->U.create(c, boundary, u_dir, normal, 0.0, 0.0, 0.0, *vel_solver, st, 0,
                          true)) != MP_OK ||
        (rc = s->V.create(c, boundary, v_dir, normal, 0.0, 0.0, 0.0, *vel_solver, st, 0,
                          true)) != MP_OK)
        return bail(rc);
    s->nsys = s->P.sys.nsys;
    for (dbuf<uint8_t> *d : {&s->udir, &s->vdir, &s->pdir})
        if ((rc = d->alloc(nv)) != MP_OK)
            return bail(rc);
    if ((rc = s->normal.alloc((size_t)nv * 2)) != MP_OK)
        return bail(rc);
    MP_CUDA(cudaMemcpy(s->udir.p, u_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(s->vdir.p, v_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(s->pdir.p, p_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(s->normal.p, normal, sizeof(double) * nv * 2, cudaMemcpyDefault));
    for (dbuf<double> *d : {&s->uo, &s->vo, &s->uoo, &s->voo, &s->uit, &s->vit})
        if ((rc = d->alloc(nv)) != MP_OK)
            return bail(rc);
    if ((rc = s->pn.alloc(s->nsys)) != MP_OK)
        return bail(rc);
    for (dbuf<double> *d : {&s->uoo, &s->voo})
        MP_CUDA(cudaMemset(d->p, 0, sizeof(double) * nv));
    s->err_blocks = std::min((nv + 255) / 256, sm_count() * 4);
    if ((rc = s->part.alloc((size_t)4 * s->err_blocks)) != MP_OK || (rc = s->ctl.alloc(1)) != MP_OK)
        return bail(rc);
    // boundary stencils holding other boundary nodes make the boundary pressure
    // rows depend on each other: run them in index order then
    CloudView cv = cloud_view(c);
    std::vector<int> nb((size_t)nv * n);
    MP_CUDA(cudaMemcpy(nb.data(), cv.nb_rm, sizeof(int) * nb.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nv && !s->serial_pb; i++)
        if (hb[i])
            for (int k = 0; k < n; k++) {
                const int j = nb[(size_t)i * n + k];
                if (j != i && hb[j]) {
                    s->serial_pb = 1;
                    break;
                }
            }
    MP_CUDA(cudaDeviceSynchronize());
    *out = s;
    return MP_OK;
}

extern "C" int mp_sis_set_tolerance(mp_sis s, double iterative_tolerance) {
    if (!s || !(iterative_tolerance >= 0))
        return fail(MP_BAD_ARG, "mp_sis_set_tolerance: a solver and a tolerance >= 0 needed");
    s->itol = iterative_tolerance;
    return MP_OK;
}

extern "C" int mp_sis_system_size(mp_sis s, int *nsys) {
    if (!s || !nsys)
        return fail(MP_BAD_ARG, "mp_sis_system_size: null argument");
    *nsys = s->nsys;
    return MP_OK;
}

extern "C" int mp_sis_set_graph(mp_sis s, int use_graph) {
    if (!s)
        return fail(MP_BAD_ARG, "null semi-implicit solver");
    s->use_graph = use_graph != 0;
    return MP_OK;
}

// One outer iteration in three kernel sequences around the solves (each issued
// eagerly or captured): before the velocity solves, between them and the
// pressure-correction solve, and after it (ending with the stopping test).
static int sis_issue_head(mp_sis_s *s, int bdf1, cudaStream_t st) {
    const int nv = s->nv, K = s->K;
    const size_t vb = sizeof(double) * nv;
    CloudView cv = cloud_view(s->c);
    const SisConst c{nv, K, s->rho, s->mu, s->dt};
    const double a1 = bdf1 ? 1.0 : 1.5;
    double *un = s->U.W.x.p, *vn = s->V.W.x.p;
    const size_t tot = (size_t)ell_padded_rows(nv) * K;
    const unsigned eb = (unsigned)((tot + 255) / 256), rb = (unsigned)((nv + 255) / 256);
    MP_CUDA(cudaMemcpyAsync(s->uit.p, un, vb, cudaMemcpyDeviceToDevice, st));
    MP_CUDA(cudaMemcpyAsync(s->vit.p, vn, vb, cudaMemcpyDeviceToDevice, st));
    k_sis_values<<<eb, 256, 0, st>>>(c, cv.cols, cv.w[0], cv.w[1], cv.w[3], cv.bflag, un, vn,
                                     a1 * s->rho / s->dt, s->U.sys.A.v64.p, s->V.sys.A.v64.p);
    MP_CHECK_LAUNCH();
    MP_TRY(s->U.refresh_diag(st));
    MP_TRY(s->V.refresh_diag(st));
    k_sis_vel_source<<<rb, 256, 0, st>>>(c, cv.cols, cv.w[0], cv.w[1], cv.bflag, s->udir.p,
                                         s->vdir.p, s->pn.p, s->uo.p, s->vo.p, s->uoo.p, s->voo.p,
                                         bdf1, s->U.W.b64.p, s->V.W.b64.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

static int sis_issue_mid(mp_sis_s *s, int bdf1, cudaStream_t st) {
    const int ns = s->nsys;
    CloudView cv = cloud_view(s->c);
    const SisConst c{s->nv, s->K, s->rho, s->mu, s->dt};
    const double a1 = bdf1 ? 1.0 : 1.5;
    k_sis_p_source<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(
        c, cv.cols, cv.w[0], cv.w[1], cv.bflag, s->U.W.x.p, s->V.W.x.p, a1 * s->rho / s->dt, ns,
        s->P.W.b64.p);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaMemsetAsync(s->P.W.x.p, 0, sizeof(double) * ns, st));
    return MP_OK;
}

static int sis_issue_tail(mp_sis_s *s, int bdf1, cudaGraphConditionalHandle h, cudaStream_t st) {
    const int nv = s->nv, ns = s->nsys;
    CloudView cv = cloud_view(s->c);
    const SisConst c{nv, s->K, s->rho, s->mu, s->dt};
    const double a1 = bdf1 ? 1.0 : 1.5;
    double *un = s->U.W.x.p, *vn = s->V.W.x.p, *pp = s->P.W.x.p;
    const unsigned rb = (unsigned)((nv + 255) / 256);
    k_sis_add<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(ns, s->pn.p, pp);
    MP_CHECK_LAUNCH();
    k_sis_p_boundary<<<s->serial_pb ? 1 : rb, s->serial_pb ? 1 : 256, 0, st>>>(
        c, cv.cols, cv.w[0], cv.w[1], cv.w[3], cv.bflag, s->pdir.p, s->normal.p, un, vn, s->uo.p,
        s->vo.p, s->uoo.p, s->voo.p, bdf1, s->serial_pb, s->pn.p);
    MP_CHECK_LAUNCH();
    k_sis_vel_corr<<<rb, 256, 0, st>>>(c, cv.cols, cv.w[0], cv.w[1], cv.bflag, pp,
                                       s->dt / (a1 * s->rho), un, vn);
    MP_CHECK_LAUNCH();
    k_sis_err<<<s->err_blocks, 256, 0, st>>>(nv, un, s->uit.p, vn, s->vit.p, s->part.p);
    MP_CHECK_LAUNCH();
    k_sis_outer_end<<<1, 256, 0, st>>>(s->err_blocks, s->part.p, nv, s->ctl.p, s->U.W.scal.p,
                                       s->V.W.scal.p, s->P.W.scal.p, s->U.cfg.tol, s->V.cfg.tol,
                                       s->P.cfg.tol, s->n_outer, h);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// The whole outer loop as one graph: a while node whose body holds the three
// solves (each its own nested while loop) and ends with the stopping test, so a
// step makes no host round trip between its copies in and out.
static int sis_graph(mp_sis_s *s, int bdf1, GraphExec &G) {
    if (G.e)
        return MP_OK;
    GraphBuilder gb;
    MP_TRY(gb.init_root(s->P.cap_stream()));
    cudaGraphConditionalHandle h;
    int rc = gb.make_handle(&h);
    if (rc == MP_OK)
        rc = gb.captured([&](cudaStream_t cs) -> int {
            k_sis_outer_init<<<1, 1, 0, cs>>>(s->ctl.p, h);
            MP_CHECK_LAUNCH();
            return MP_OK;
        });
    if (rc == MP_OK)
        rc = gb.while_loop(h, [&](GraphBuilder &body) {
            MP_TRY(body.captured([&](cudaStream_t cs) { return sis_issue_head(s, bdf1, cs); }));
            MP_TRY(s->U.build_solve_graph(body));
            MP_TRY(s->V.build_solve_graph(body));
            MP_TRY(body.captured([&](cudaStream_t cs) { return sis_issue_mid(s, bdf1, cs); }));
            MP_TRY(s->P.build_solve_graph(body));
            return body.captured([&](cudaStream_t cs) { return sis_issue_tail(s, bdf1, h, cs); });
        });
    if (rc != MP_OK) {
        if (gb.g)
            cudaGraphDestroy(gb.g);
        return rc;
    }
    return G.instantiate(gb);
}

extern "C" int mp_sis_single_timestep(mp_sis s, const double *const *vel_old,
                                      const double *p_old, double *const *vel_new,
                                      double *p_new, int it, int *n_outer, double *l1_err,
                                      double *max_err, mp_stream stream) {
    if (!s || !vel_old || !vel_old[0] || !vel_old[1] || !p_old || !vel_new || !vel_new[0] ||
        !vel_new[1] || !p_new || it < 0)
        return fail(MP_BAD_ARG, "mp_sis_single_timestep: bad arguments");
    cudaStream_t st = S(stream);
    const int nv = s->nv, ns = s->nsys;
    const size_t vb = sizeof(double) * nv;
    const int bdf1 = it == 0;
    double *un = s->U.W.x.p, *vn = s->V.W.x.p;
    // u_new = u_old, v_new = v_old, p_new = p_old (:384)
    MP_CUDA(cudaMemcpyAsync(s->uo.p, vel_old[0], vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(s->vo.p, vel_old[1], vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(s->pn.p, p_old, sizeof(double) * ns, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(un, s->uo.p, vb, cudaMemcpyDeviceToDevice, st));
    MP_CUDA(cudaMemcpyAsync(vn, s->vo.p, vb, cudaMemcpyDeviceToDevice, st));
    SisCtl hc{};
    // the tolerance may change between steps (the reference's driver sets it from the
    // steady-state change every step); a pageable source is staged before the call returns
    MP_CUDA(cudaMemcpyAsync(&s->ctl.p->itol, &s->itol, sizeof(double), cudaMemcpyHostToDevice, st));
    if (s->use_graph) {
        GraphExec &G = s->graph[bdf1 ? 0 : 1];
        MP_TRY(sis_graph(s, bdf1, G));
        MP_TRY(G.launch(st));
        MP_CUDA(cudaMemcpyAsync(&hc, s->ctl.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
    } else {  // eager: the same sequences, the host reads the state after each iteration
        k_sis_outer_init<<<1, 1, 0, st>>>(s->ctl.p, 0);
        MP_CHECK_LAUNCH();
        for (int outer = 0; outer < s->n_outer; outer++) {
            MP_TRY(sis_issue_head(s, bdf1, st));
            MP_TRY(s->U.solve_resident(st, false));
            MP_TRY(s->V.solve_resident(st, false));
            MP_TRY(sis_issue_mid(s, bdf1, st));
            MP_TRY(s->P.solve_resident(st, false));
            MP_TRY(sis_issue_tail(s, bdf1, 0, st));
            MP_CUDA(cudaMemcpyAsync(&hc, s->ctl.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
            MP_CUDA(cudaStreamSynchronize(st));
            if (hc.status != MP_OK || !(hc.err[0] > s->itol))
                break;
        }
    }
    if (hc.status != MP_OK) {
        static const char *what[4] = {"velocity", "u", "v", "pressure-correction"};
        if (hc.failed)
            return fail(hc.status,
                        "semi-implicit step %d, outer iteration %d: %s solve status %d after %d "
                        "iterations, relres %g", it, hc.outer, what[hc.failed], hc.status,
                        hc.iters, hc.relres);
        return fail(hc.status, "semi-implicit step %d: NaN in the velocity", it);
    }
    // extras (:206-216): u_old_old = u_old
    MP_CUDA(cudaMemcpyAsync(s->uoo.p, s->uo.p, vb, cudaMemcpyDeviceToDevice, st));
    MP_CUDA(cudaMemcpyAsync(s->voo.p, s->vo.p, vb, cudaMemcpyDeviceToDevice, st));
    MP_CUDA(cudaMemcpyAsync(vel_new[0], un, vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(vel_new[1], vn, vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(p_new, s->pn.p, sizeof(double) * ns, cudaMemcpyDefault, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (n_outer)
        *n_outer = hc.outer;
    if (l1_err)
        *l1_err = hc.err[0];
    if (max_err)
        *max_err = hc.err[1];
    return MP_OK;
}

extern "C" int mp_sis_destroy(mp_sis s) {
    delete s;
    return MP_OK;
}

// ------------------------------------------- implicit scalar transport
// IMPLICIT_SCALAR_TRANSPORT_SOLVER (implicit_scalar_transport_solver.cpp, 2D): one
// implicit convection-diffusion solve per step, BDF1 at it = 0 then BDF2, the
// matrix's interior rows rebuilt from the given velocity every step (:140-151);
// BiCGSTAB with the Jacobi diagonal of that matrix, from phi_old.
struct mp_ist_s {
    mp_cloud c = nullptr;
    int nv = 0, K = 0;
    double unsteady = 0, conv = 0, diff = 0;
    dbuf<uint8_t> dir;
    dbuf<double> po, poo, u, v;
    Ppe T;
    bool use_graph = true;
};

extern "C" int mp_ist_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                             const uint8_t *dirichlet, int precond_freq_it, double unsteady_coeff,
                             double conv_coeff, double diff_coeff, const mp_solver_cfg *solver,
                             mp_ist *out) {
    if (!c || !boundary || !normal || !dirichlet || !solver || !out)
        return fail(MP_BAD_ARG, "mp_ist_create: null argument");
    (void)precond_freq_it;
    int nv, n, dim;
    MP_TRY(mp_cloud_info(c, &nv, &n, &dim));
    if (dim != 2)
        return fail(MP_BAD_ARG, "the implicit scalar transport solver is 2D (single_timestep_2d)");
    if (solver->precond == MP_PRECOND_AMG || solver->precision != MP_FP64)
        return fail(MP_BAD_ARG, "the transport matrix changes every step: its solver takes "
                                "MP_PRECOND_JACOBI or MP_PRECOND_NONE in MP_FP64");
    MP_TRY(integrator_cfg_check(*solver));
    std::vector<uint8_t> hb(nv), hd(nv);
    MP_CUDA(cudaMemcpy(hb.data(), boundary, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(hd.data(), dirichlet, nv, cudaMemcpyDefault));
    bool any_dir = false;  // :28-39: full Neumann is not permitted
    for (int i = 0; i < nv && !any_dir; i++)
        any_dir = hb[i] && hd[i];
    if (!any_dir)
        return fail(MP_BAD_ARG, "full Neumann BC is not permitted for the transported scalar");
    mp_ist_s *s = new mp_ist_s;
    auto bail = [&](int rc) {
        delete s;
        return rc;
    };
    s->c = c;
    s->nv = nv;
    s->K = n;
    s->unsteady = unsteady_coeff;
    s->conv = conv_coeff;
    s->diff = diff_coeff;
    int rc;
    if ((rc = s->T.create(c, boundary, dirichlet, normal, 0.0, 0.0, 0.0, *solver, 0, 0, true)) !=
        MP_OK)
        return bail(rc);
    if ((rc = s->dir.alloc(nv)) != MP_OK)
        return bail(rc);
    MP_CUDA(cudaMemcpy(s->dir.p, dirichlet, nv, cudaMemcpyDefault));
    for (dbuf<double> *d : {&s->po, &s->poo, &s->u, &s->v})
        if ((rc = d->alloc(nv)) != MP_OK)
            return bail(rc);
    MP_CUDA(cudaMemset(s->poo.p, 0, sizeof(double) * nv));
    MP_CUDA(cudaDeviceSynchronize());
    *out = s;
    return MP_OK;
}

extern "C" int mp_ist_set_graph(mp_ist s, int use_graph) {
    if (!s)
        return fail(MP_BAD_ARG, "null transport solver");
    s->use_graph = use_graph != 0;
    return MP_OK;
}

extern "C" int mp_ist_single_timestep(mp_ist s, const double *phi_old, const double *u_new,
                                      const double *v_new, double *phi_new, int it, int *iters,
                                      double *relres, mp_stream stream) {
    if (!s || !phi_old || !u_new || !v_new || !phi_new || it < 0)
        return fail(MP_BAD_ARG, "mp_ist_single_timestep: bad arguments");
    cudaStream_t st = S(stream);
    const int nv = s->nv, K = s->K;
    const size_t vb = sizeof(double) * nv;
    CloudView cv = cloud_view(s->c);
    MP_CUDA(cudaMemcpyAsync(s->po.p, phi_old, vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(s->u.p, u_new, vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(s->v.p, v_new, vb, cudaMemcpyDefault, st));
    const int bdf1 = it == 0;
    const size_t tot = (size_t)ell_padded_rows(nv) * K;
    k_ist_values<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(
        nv, K, cv.cols, cv.w[0], cv.w[1], cv.w[3], cv.bflag, s->u.p, s->v.p, s->diff, s->conv,
        (bdf1 ? 1.0 : 1.5) * s->unsteady, s->T.sys.A.v64.p);
    MP_CHECK_LAUNCH();
    MP_TRY(s->T.refresh_diag(st));
    k_ist_source<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(
        nv, cv.bflag, s->dir.p, s->po.p, s->poo.p, s->unsteady, bdf1, s->T.W.b64.p);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaMemcpyAsync(s->T.W.x.p, s->po.p, vb, cudaMemcpyDeviceToDevice, st));  // guess phi_old
    MP_TRY(s->T.solve_resident(st, s->use_graph));
    SolveStats ss;
    MP_TRY(s->T.read_stats(st, &ss));
    if (ss.status != MP_OK)
        return fail(ss.status, "transport solve: status %d after %d iterations, relres %g",
                    ss.status, ss.iters, ss.relres);
    MP_CUDA(cudaMemcpyAsync(phi_new, s->T.W.x.p, vb, cudaMemcpyDefault, st));
    MP_CUDA(cudaMemcpyAsync(s->poo.p, s->po.p, vb, cudaMemcpyDeviceToDevice, st));  // :172
    MP_CUDA(cudaStreamSynchronize(st));
    if (iters)
        *iters = ss.iters;
    if (relres)
        *relres = ss.relres;
    return MP_OK;
}

extern "C" int mp_ist_destroy(mp_ist s) {
    delete s;
    return MP_OK;
}
