// mp_fsf.cu -- FRACTIONAL_STEP_FOURIER (fractional_step_fourier.cpp) on the GPU.
//
// A 2D cloud extruded periodically in z: every field is nv x N (N = 2 nw + 1
// planes, column-major as Eigen's MatrixXd), and the step runs on its z-Fourier
// coefficients.  Real fields have conjugate-symmetric coefficients, so only the
// modes 0..nw are stored (real and imaginary parts, nv x (nw + 1) each); the
// reference carries all N columns and fills the upper half with conjugates
// (calc_dft, general_functions.cpp:1125-1130), which every step preserves.
// One step (single_timestep :250-266):
//   calc_vel_source (:375-398)  ft(Gx(u phi) + Gy(v phi)) + i k ft(w phi) convected,
//                               mu (L phi_ft - k^2 phi_ft) diffused, for phi = u, v, w
//   calc_vel_hat (:326-345)     Euler at it = 0 or first order, else Adams-Bashforth 2
//   calc_pressure (:400-442)    per mode the Helmholtz system L - k^2 (the first mode
//                               bordered under full-Neumann pressure, real part only),
//                               real and imaginary parts solved from the old pressure,
//                               each to tol times the largest mode's source norm
//   calc_vel_corr (:444-552)    q_ft = q_hat - G p_ft dt/rho, w: - i k p_ft dt/rho;
//                               boundary rows without Dirichlet pressure: the old
//                               value (Dirichlet) or the normal-derivative row
// The transforms use the reference's matrices (get_dft_matrix / get_idft_matrix,
// :1106-1123), whose phase carries the period as written there.
#include <algorithm>
#include <cmath>
#include <vector>
#include "mp_cloud.cuh"
#include "mp_ppe.cuh"

namespace mp {

struct FsfDims {
    int nv, K, N, M;  // nodes, stencil width, planes, stored modes (nw + 1)
};

// out (nv x M, re/im) = phys (nv x N) times the first M columns of the DFT matrix
__global__ void k_fsf_dft(FsfDims d, const double *phys, const double *twr, const double *twi,
                          double *ore, double *oim) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.M)
        return;
    const int iv = t % d.nv, iw = t / d.nv;
    double sr = 0.0, si = 0.0;
    for (int ic = 0; ic < d.N; ic++) {
        const double x = phys[(size_t)ic * d.nv + iv];
        sr += x * twr[ic * d.M + iw];
        si += x * twi[ic * d.M + iw];
    }
    ore[(size_t)iw * d.nv + iv] = sr;
    oim[(size_t)iw * d.nv + iv] = si;
}

// calc_idft (:1132-1137): phys = Re(ft_0 idft_0) + 2 sum_{iw>=1} Re(ft_iw idft_iw)
__global__ void k_fsf_idft(FsfDims d, const double *fre, const double *fim, const double *itr,
                           const double *iti, double *phys) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.N)
        return;
    const int iv = t % d.nv, ic = t / d.nv;
    double v = fre[iv] * itr[ic] - fim[iv] * iti[ic];
    double acc = 0.0;
    for (int iw = 1; iw < d.M; iw++)
        acc += fre[(size_t)iw * d.nv + iv] * itr[(size_t)iw * d.N + ic] -
               fim[(size_t)iw * d.nv + iv] * iti[(size_t)iw * d.N + ic];
    phys[(size_t)ic * d.nv + iv] = v + 2.0 * acc;
}

// node-major (nv x N, row-major: plane c of node i at i N + c) <-> plane-contiguous
// (plane c at c nv); one thread per entry, consecutive threads on consecutive nodes
// of one plane (the plane-contiguous side coalesced, the node-major side a stride
// of N doubles that L1/L2 absorb for the few planes of a Fourier step)
__global__ void k_fsf_to_planes(int nv, int N, const double *node_major, double *planes) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nv * N)
        return;
    const int i = (int)(t % nv), c = (int)(t / nv);
    planes[t] = node_major[(size_t)i * N + c];
}
__global__ void k_fsf_to_nodes(int nv, int N, const double *planes, double *node_major) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nv * N)
        return;
    const int i = (int)(t % nv), c = (int)(t / nv);
    node_major[(size_t)i * N + c] = planes[t];
}

__device__ __forceinline__ double stencil_dot(const int *cols, const double *w, int i, int K,
                                              const double *x) {
    const size_t base = (size_t)(i / SLICE) * K * SLICE + (i % SLICE);
    double s = 0.0;
    for (int k = 0; k < K; k++)
        s += w[base + (size_t)k * SLICE] * x[cols[base + (size_t)k * SLICE]];
    return s;
}

// the products u phi, v phi over all N planes (calc_vel_source :379)
__global__ void k_fsf_flux(FsfDims d, const double *u, const double *v, const double *phi,
                           double *uphi, double *vphi) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.N)
        return;
    uphi[t] = u[t] * phi[t];
    vphi[t] = v[t] * phi[t];
}

// xy := Gx(u phi) + Gy(v phi), z := w phi (:379-385)
__global__ void k_fsf_sum2(FsfDims d, const int *cols, const double *gx, const double *gy,
                           const double *uphi, const double *vphi, const double *w,
                           const double *phi, double *xy, double *z) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.N)
        return;
    const int i = t % d.nv, c = t / d.nv;
    xy[t] = stencil_dot(cols, gx, i, d.K, uphi + (size_t)c * d.nv) +
            stencil_dot(cols, gy, i, d.K, vphi + (size_t)c * d.nv);
    z[t] = w[t] * phi[t];
}

// source = -rho (xy_ft + i k z_ft) + mu (L phi_ft - k^2 phi_ft), stored modes only
__global__ void k_fsf_source(FsfDims d, const int *cols, const double *lap, const double *k,
                             double rho, double mu, const double *xyr, const double *xyi,
                             const double *zr, const double *zi, const double *pr,
                             const double *pi, double *sr, double *si) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.M)
        return;
    const int i = t % d.nv, iw = t / d.nv;
    const double kw = k[iw], k2 = kw * kw;
    const size_t o = (size_t)iw * d.nv;
    const double lr = stencil_dot(cols, lap, i, d.K, pr + o), li = stencil_dot(cols, lap, i, d.K, pi + o);
    // i k (zr + i zi) = -k zi + i k zr
    sr[t] = -rho * (xyr[t] + (-kw * zi[t])) + mu * (lr - pr[t] * k2);
    si[t] = -rho * (xyi[t] + (kw * zr[t])) + mu * (li - pi[t] * k2);
}

// calc_vel_hat: hat = old + dt/rho src (first step / order 1) or AB2
__global__ void k_fsf_hat(int n, int ab2, double c, const double *old, const double *s,
                          const double *s2, double *hat) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    hat[t] = ab2 ? old[t] + (0.5 * c) * (3.0 * s[t] - s2[t]) : old[t] + c * s[t];
}

// pressure sources of every stored mode (calc_pressure :402-415), column iw of
// (re, im); boundary rows: the old pressure (Dirichlet) or the normal momentum
__global__ void k_fsf_psrc(FsfDims d, const int *cols, const double *gx, const double *gy,
                           const double *k, const uint8_t *bflag, const uint8_t *pdir,
                           const double *normal, double rho, double dt, const double *uhr,
                           const double *uhi, const double *vhr, const double *vhi,
                           const double *whr, const double *whi, const double *uor,
                           const double *uoi, const double *vor, const double *voi,
                           const double *por, const double *poi, double *psr, double *psi) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.M)
        return;
    const int i = t % d.nv, iw = t / d.nv;
    const size_t o = (size_t)iw * d.nv;
    double r, m;
    if (bflag[i]) {
        if (pdir[i]) {
            r = por[t];
            m = poi[t];
        } else {
            const double nx = normal[2 * (size_t)i], ny = normal[2 * (size_t)i + 1];
            r = -rho * ((uor[t] - uhr[t]) * nx + (vor[t] - vhr[t]) * ny) / dt;
            m = -rho * ((uoi[t] - uhi[t]) * nx + (voi[t] - vhi[t]) * ny) / dt;
        }
    } else {
        const double kw = k[iw];
        r = (stencil_dot(cols, gx, i, d.K, uhr + o) + stencil_dot(cols, gy, i, d.K, vhr + o)) +
            (-kw * whi[t]);
        m = (stencil_dot(cols, gx, i, d.K, uhi + o) + stencil_dot(cols, gy, i, d.K, vhi + o)) +
            (kw * whr[t]);
        r = r * rho / dt;
        m = m * rho / dt;
    }
    psr[t] = r;
    psi[t] = m;
}

// velocity correction of every stored mode (:446-449)
__global__ void k_fsf_corr3(FsfDims d, const int *cols, const double *gx, const double *gy,
                            const double *k, double c, const double *pr, const double *pi,
                            const double *uhr, const double *uhi, const double *vhr,
                            const double *vhi, const double *whr, const double *whi, double *unr,
                            double *uni, double *vnr, double *vni, double *wnr, double *wni) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= d.nv * d.M)
        return;
    const int i = t % d.nv, iw = t / d.nv;
    const size_t o = (size_t)iw * d.nv;
    unr[t] = uhr[t] - stencil_dot(cols, gx, i, d.K, pr + o) * c;
    uni[t] = uhi[t] - stencil_dot(cols, gx, i, d.K, pi + o) * c;
    vnr[t] = vhr[t] - stencil_dot(cols, gy, i, d.K, pr + o) * c;
    vni[t] = vhi[t] - stencil_dot(cols, gy, i, d.K, pi + o) * c;
    // i k (pr + i pi) = -k pi + i k pr
    wnr[t] = whr[t] - (-k[iw] * pi[t]) * c;
    wni[t] = whi[t] - (k[iw] * pr[t]) * c;
}

// boundary rows without Dirichlet pressure (:460-549): Dirichlet velocity keeps the
// old coefficient, Neumann velocity solves the normal-derivative row.  Boundary
// stencils hold interior nodes besides their own, so rows are independent;
// `serial` runs them in index order otherwise.
__global__ void k_fsf_bnd(FsfDims d, const int *cols, const double *gx, const double *gy,
                          const uint8_t *bflag, const uint8_t *pdir, const uint8_t *qdir,
                          const double *normal, int serial, const double *oldr, const double *oldi,
                          double *qr, double *qi) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int first = serial ? 0 : tid, last = serial ? d.nv * d.M : tid + 1;
    if (serial && tid)
        return;
    for (int t = first; t < last && t < d.nv * d.M; t++) {
        const int i = serial ? t / d.M : t % d.nv, iw = serial ? t % d.M : t / d.nv;
        const size_t e0 = (size_t)iw * d.nv + i;
        if (!bflag[i] || pdir[i])
            continue;
        if (qdir[i]) {
            qr[e0] = oldr[e0];
            qi[e0] = oldi[e0];
            continue;
        }
        const double nx = normal[2 * (size_t)i], ny = normal[2 * (size_t)i + 1];
        const size_t base = (size_t)(i / SLICE) * d.K * SLICE + (i % SLICE);
        double rr = 0.0, ri = 0.0, diag = 0.0;
        for (int k = 0; k < d.K; k++) {
            const size_t e = base + (size_t)k * SLICE;
            const int j = cols[e];
            const double cf = (gx[e] * nx) + (gy[e] * ny);
            if (j == i) {
                diag = cf;
            } else {
                rr = rr - cf * qr[(size_t)iw * d.nv + j];
                ri = ri - cf * qi[(size_t)iw * d.nv + j];
            }
        }
        qr[e0] = rr / diag;
        qi[e0] = ri / diag;
    }
}

// sum of squares of each (column, part) of the pressure sources: out[2 iw + q]
__global__ void k_fsf_colnorm(FsfDims d, const double *re, const double *im, double *out) {
    __shared__ double red[256];
    const int col = blockIdx.x >> 1, q = blockIdx.x & 1;
    const double *x = (q ? im : re) + (size_t)col * d.nv;
    double a = 0.0;
    for (int i = threadIdx.x; i < d.nv; i += blockDim.x)
        a += x[i] * x[i];
    red[threadIdx.x] = a;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w /= 2) {
        if ((int)threadIdx.x < w)
            red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        out[blockIdx.x] = red[0];
}

}  // namespace mp

using namespace mp;

struct mp_fsf_s {
    mp_cloud c = nullptr;
    FsfDims d{};
    int order = 2, serial = 0, bordered0 = 0;
    double rho = 1, mu = 0, dt = 0;
    std::vector<Ppe *> P;
    dbuf<uint8_t> udir, vdir, wdir, pdir;
    dbuf<double> normal, k, twr, twi, itr, iti, cn;
    // spectral state (re, im; nv x M each): old fields, sources, AB2 history, hats
    dbuf<double> f[4][2], s[3][2], s2[3][2], h[3][2], ps[2];
    // scratch
    dbuf<double> phys[4], uphi, vphi, xy, z, ft[4];
    bool started = false;
    bool use_graph = true;
    // node-major fields (mp_fsf_set_layout): each passes through `stage` and a
    // device transpose on its way in and out
    bool node_major = false;
    dbuf<double> stage;
    // the modes' pressure solves are independent (each mode has its own system,
    // hierarchy and Krylov vectors): one stream per mode, joined after the solves;
    // each solve's final scalars are kept (real, imaginary) for the status check
    std::vector<cudaStream_t> ms;
    std::vector<cudaEvent_t> mev;
    cudaEvent_t fork = nullptr;
    dbuf<BicgScalars> stats;
    ~mp_fsf_s() {
        for (cudaStream_t x : ms)
            cudaStreamDestroy(x);
        for (cudaEvent_t e : mev)
            cudaEventDestroy(e);
        if (fork)
            cudaEventDestroy(fork);
    }
};

extern "C" int mp_fsf_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                             const uint8_t *u_dir, const uint8_t *v_dir, const uint8_t *w_dir,
                             const uint8_t *p_dir, double period, int nw, int temporal_order,
                             double rho, double mu, double dt, const mp_solver_cfg *solver,
                             mp_fsf *out) {
    if (!c || !boundary || !normal || !u_dir || !v_dir || !w_dir || !p_dir || !solver || !out)
        return fail(MP_BAD_ARG, "mp_fsf_create: null argument");
    int nv, n, dim;
    MP_TRY(mp_cloud_info(c, &nv, &n, &dim));
    // check_settings (:186-203)
    if (rho < 0 || mu < 0)
        return fail(MP_BAD_ARG, "rho and mu must be set (rho %g, mu %g)", rho, mu);
    if (temporal_order != 1 && temporal_order != 2)
        return fail(MP_BAD_ARG, "temporal_order should be 1 or 2; got %d", temporal_order);
    if (dim != 2)
        return fail(MP_BAD_ARG, "FRACTIONAL_STEP_FOURIER is defined for 2D clouds only");
    if (nw < 0 || !(period > 0) || !(dt > 0))
        return fail(MP_BAD_ARG, "nw >= 0, period > 0 and dt > 0 needed");
    MP_TRY(integrator_cfg_check(*solver));
    mp_fsf_s *f = new mp_fsf_s;
    auto bail = [&](int rc) {
        for (Ppe *p : f->P)
            delete p;
        delete f;
        return rc;
    };
    const int N = 2 * nw + 1, M = nw + 1;
    f->c = c;
    f->d = FsfDims{nv, n, N, M};
    f->order = temporal_order;
    f->rho = rho;
    f->mu = mu;
    f->dt = dt;
    // wave numbers (:35-41) and the transform matrices (:1106-1123)
    std::vector<double> kw(M), twr((size_t)N * M), twi((size_t)N * M), itr((size_t)M * N),
        iti((size_t)M * N);
    for (int iw = 0; iw < M; iw++)
        kw[iw] = iw * 2 * M_PI / period;
    for (int ic = 0; ic < N; ic++)
        for (int iw = 0; iw < M; iw++) {
            const double a = -2.0 * M_PI * (double)iw * (double)ic / (N * period);
            twr[(size_t)ic * M + iw] = std::cos(a);
            twi[(size_t)ic * M + iw] = std::sin(a);
            itr[(size_t)iw * N + ic] = std::cos(-a) / N;
            iti[(size_t)iw * N + ic] = std::sin(-a) / N;
        }
    int rc;
    for (auto pr : {std::make_pair(&f->k, &kw), std::make_pair(&f->twr, &twr),
                    std::make_pair(&f->twi, &twi), std::make_pair(&f->itr, &itr),
                    std::make_pair(&f->iti, &iti)}) {
        if ((rc = pr.first->alloc(pr.second->size())) != MP_OK)
            return bail(rc);
        MP_CUDA(cudaMemcpy(pr.first->p, pr.second->data(), sizeof(double) * pr.second->size(),
                           cudaMemcpyHostToDevice));
    }
    // set_p_coeff_eigen (:119-172): per stored mode the Laplacian with -k^2 on the
    // interior diagonal; only the first mode may be bordered
    for (int iw = 0; iw < M; iw++) {
        Ppe *p = new Ppe;
        f->P.push_back(p);
        if ((rc = p->create(c, boundary, p_dir, normal, -kw[iw] * kw[iw], 0.0, 1.0, *solver, 0,
                            iw == 0 ? 1 : 0)) != MP_OK)
            return bail(rc);
        MP_CUDA(cudaMemset(p->W.x.p, 0, sizeof(double) * p->sys.nsys));
    }
    f->bordered0 = f->P[0]->sys.bordered;
    f->ms.resize(M, nullptr);
    f->mev.resize(M, nullptr);
    for (int iw = 0; iw < M; iw++) {
        MP_CUDA(cudaStreamCreateWithFlags(&f->ms[iw], cudaStreamNonBlocking));
        MP_CUDA(cudaEventCreateWithFlags(&f->mev[iw], cudaEventDisableTiming));
    }
    MP_CUDA(cudaEventCreateWithFlags(&f->fork, cudaEventDisableTiming));
    if ((rc = f->stats.alloc((size_t)2 * M)) != MP_OK)
        return bail(rc);
    if ((rc = f->cn.alloc((size_t)2 * M)) != MP_OK)
        return bail(rc);
    for (dbuf<uint8_t> *b : {&f->udir, &f->vdir, &f->wdir, &f->pdir})
        if ((rc = b->alloc(nv)) != MP_OK)
            return bail(rc);
    MP_CUDA(cudaMemcpy(f->udir.p, u_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(f->vdir.p, v_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(f->wdir.p, w_dir, nv, cudaMemcpyDefault));
    MP_CUDA(cudaMemcpy(f->pdir.p, p_dir, nv, cudaMemcpyDefault));
    if ((rc = f->normal.alloc((size_t)nv * 2)) != MP_OK)
        return bail(rc);
    MP_CUDA(cudaMemcpy(f->normal.p, normal, sizeof(double) * nv * 2, cudaMemcpyDefault));
    const size_t nm = (size_t)nv * M, nn = (size_t)nv * N;
    for (int q = 0; q < 2; q++) {
        for (int a = 0; a < 4; a++)
            if ((rc = f->f[a][q].alloc(nm)) != MP_OK)
                return bail(rc);
        for (int a = 0; a < 3; a++)
            if ((rc = f->s[a][q].alloc(nm)) != MP_OK || (rc = f->s2[a][q].alloc(nm)) != MP_OK ||
                (rc = f->h[a][q].alloc(nm)) != MP_OK)
                return bail(rc);
        if ((rc = f->ps[q].alloc(nm)) != MP_OK)
            return bail(rc);
    }
    for (int a = 0; a < 4; a++)
        if ((rc = f->phys[a].alloc(nn)) != MP_OK || (rc = f->ft[a].alloc(nm)) != MP_OK)
            return bail(rc);
    for (dbuf<double> *b : {&f->uphi, &f->vphi, &f->xy, &f->z})
        if ((rc = b->alloc(nn)) != MP_OK)
            return bail(rc);
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 2; q++)
            MP_CUDA(cudaMemset(f->s2[a][q].p, 0, sizeof(double) * nm));
    // boundary stencils with other boundary nodes: boundary rows in index order
    std::vector<uint8_t> hb(nv);
    MP_CUDA(cudaMemcpy(hb.data(), boundary, nv, cudaMemcpyDefault));
    CloudView cv = cloud_view(c);
    std::vector<int> nb((size_t)nv * n);
    MP_CUDA(cudaMemcpy(nb.data(), cv.nb_rm, sizeof(int) * nb.size(), cudaMemcpyDeviceToHost));
    for (int i = 0; i < nv && !f->serial; i++)
        if (hb[i])
            for (int q = 0; q < n; q++) {
                const int j = nb[(size_t)i * n + q];
                if (j != i && hb[j]) {
                    f->serial = 1;
                    break;
                }
            }
    MP_CUDA(cudaDeviceSynchronize());
    *out = f;
    return MP_OK;
}

extern "C" int mp_fsf_set_graph(mp_fsf f, int use_graph) {
    if (!f)
        return fail(MP_BAD_ARG, "null Fourier fractional step");
    f->use_graph = use_graph != 0;
    return MP_OK;
}

extern "C" int mp_fsf_set_layout(mp_fsf f, int node_major) {
    if (!f)
        return fail(MP_BAD_ARG, "null Fourier fractional step");
    if (node_major != 0 && node_major != 1)
        return fail(MP_BAD_ARG, "mp_fsf_set_layout: node_major must be 0 or 1, not %d", node_major);
    if (node_major && !f->stage.p)
        MP_TRY(f->stage.alloc((size_t)f->d.nv * f->d.N));
    f->node_major = node_major != 0;
    return MP_OK;
}

extern "C" int mp_fsf_single_timestep(mp_fsf f, const double *const *vel_old, const double *p_old,
                                      double *const *vel_new, double *p_new, int it,
                                      mp_stream stream) {
    if (!f || !vel_old || !p_old || !vel_new || !p_new || it < 0)
        return fail(MP_BAD_ARG, "mp_fsf_single_timestep: bad arguments");
    for (int a = 0; a < 3; a++)
        if (!vel_old[a] || !vel_new[a])
            return fail(MP_BAD_ARG, "mp_fsf_single_timestep: null velocity plane");
    cudaStream_t st = S(stream);
    const FsfDims d = f->d;
    const int nv = d.nv, M = d.M;
    const size_t nn = (size_t)nv * d.N, nm = (size_t)nv * M;
    CloudView cv = cloud_view(f->c);
    const unsigned bn = (unsigned)((nn + 255) / 256), bm = (unsigned)((nm + 255) / 256);
    // physical old fields (u, v, w, p)
    const double *src_phys[4] = {vel_old[0], vel_old[1], vel_old[2], p_old};
    for (int a = 0; a < 4; a++) {
        if (f->node_major) {
            MP_CUDA(cudaMemcpyAsync(f->stage.p, src_phys[a], sizeof(double) * nn,
                                    cudaMemcpyDefault, st));
            k_fsf_to_planes<<<bn, 256, 0, st>>>(nv, d.N, f->stage.p, f->phys[a].p);
            MP_CHECK_LAUNCH();
        } else {
            MP_CUDA(cudaMemcpyAsync(f->phys[a].p, src_phys[a], sizeof(double) * nn,
                                    cudaMemcpyDefault, st));
        }
    }
    if (it == 0 || !f->started) {  // :254-258: coefficients of the old fields
        for (int a = 0; a < 4; a++) {
            k_fsf_dft<<<bm, 256, 0, st>>>(d, f->phys[a].p, f->twr.p, f->twi.p, f->f[a][0].p,
                                          f->f[a][1].p);
            MP_CHECK_LAUNCH();
        }
        f->started = true;
    }
    const double *U = f->phys[0].p, *V = f->phys[1].p, *W = f->phys[2].p;
    // calc_vel_hat: sources of u, v, w, then the hats
    for (int a = 0; a < 3; a++) {
        k_fsf_flux<<<bn, 256, 0, st>>>(d, U, V, f->phys[a].p, f->uphi.p, f->vphi.p);
        MP_CHECK_LAUNCH();
        k_fsf_sum2<<<bn, 256, 0, st>>>(d, cv.cols, cv.w[0], cv.w[1], f->uphi.p, f->vphi.p, W,
                                       f->phys[a].p, f->xy.p, f->z.p);
        MP_CHECK_LAUNCH();
        k_fsf_dft<<<bm, 256, 0, st>>>(d, f->xy.p, f->twr.p, f->twi.p, f->ft[0].p, f->ft[1].p);
        MP_CHECK_LAUNCH();
        k_fsf_dft<<<bm, 256, 0, st>>>(d, f->z.p, f->twr.p, f->twi.p, f->ft[2].p, f->ft[3].p);
        MP_CHECK_LAUNCH();
        k_fsf_source<<<bm, 256, 0, st>>>(d, cv.cols, cv.w[3], f->k.p, f->rho, f->mu, f->ft[0].p,
                                         f->ft[1].p, f->ft[2].p, f->ft[3].p, f->f[a][0].p,
                                         f->f[a][1].p, f->s[a][0].p, f->s[a][1].p);
        MP_CHECK_LAUNCH();
    }
    const int ab2 = !(f->order == 1 || it == 0);
    for (int a = 0; a < 3; a++)
        for (int q = 0; q < 2; q++) {
            k_fsf_hat<<<bm, 256, 0, st>>>((int)nm, ab2, f->dt / f->rho, f->f[a][q].p, f->s[a][q].p,
                                          f->s2[a][q].p, f->h[a][q].p);
            MP_CHECK_LAUNCH();
        }
    // calc_pressure
    k_fsf_psrc<<<bm, 256, 0, st>>>(d, cv.cols, cv.w[0], cv.w[1], f->k.p, cv.bflag, f->pdir.p,
                                   f->normal.p, f->rho, f->dt, f->h[0][0].p, f->h[0][1].p,
                                   f->h[1][0].p, f->h[1][1].p, f->h[2][0].p, f->h[2][1].p,
                                   f->f[0][0].p, f->f[0][1].p, f->f[1][0].p, f->f[1][1].p,
                                   f->f[3][0].p, f->f[3][1].p, f->ps[0].p, f->ps[1].p);
    MP_CHECK_LAUNCH();
    // every mode is solved to tol relative to the largest mode's source: a mode whose
    // source is rounding noise cannot reach tol relative to its own norm in FP64
    std::vector<double> cn(2 * M);
    k_fsf_colnorm<<<2 * M, 256, 0, st>>>(d, f->ps[0].p, f->ps[1].p, f->cn.p);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaMemcpyAsync(cn.data(), f->cn.p, sizeof(double) * 2 * M, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    double bmax = 0.0;
    for (double v : cn)
        bmax = std::max(bmax, v);
    // the modes' solves concurrently, one stream per mode (real then imaginary part of a
    // mode on its stream: they share its Krylov vectors)
    MP_CUDA(cudaEventRecord(f->fork, st));
    for (int iw = 0; iw < M; iw++) {
        Ppe &S = *f->P[iw];
        cudaStream_t ms = f->ms[iw];
        MP_CUDA(cudaStreamWaitEvent(ms, f->fork, 0));
        MP_TRY(S.set_abs_tol(S.cfg.tol * std::sqrt(bmax), ms));
        const size_t o = (size_t)iw * nv, vb = sizeof(double) * nv;
        const bool border = S.sys.nsys == nv + 1;
        for (int q = 0; q < (border ? 1 : 2); q++) {  // the bordered mode solves its real part
            MP_CUDA(cudaMemcpyAsync(S.W.b64.p, f->ps[q].p + o, vb, cudaMemcpyDeviceToDevice, ms));
            MP_CUDA(cudaMemcpyAsync(S.W.x.p, f->f[3][q].p + o, vb, cudaMemcpyDeviceToDevice, ms));
            if (border)  // the source's border entry is 0; the multiplier keeps its last value
                MP_CUDA(cudaMemsetAsync(S.W.b64.p + nv, 0, sizeof(double), ms));
            MP_TRY(S.solve_resident(ms, f->use_graph));
            MP_CUDA(cudaMemcpyAsync(f->stats.p + 2 * iw + q, S.W.scal.p, sizeof(BicgScalars),
                                    cudaMemcpyDeviceToDevice, ms));
            // the new pressure coefficients go to ft[q] (mode iw), kept apart from the old
            MP_CUDA(cudaMemcpyAsync(f->ft[q].p + o, S.W.x.p, vb, cudaMemcpyDeviceToDevice, ms));
        }
        if (border)  // the first mode's imaginary part stays 0
            MP_CUDA(cudaMemsetAsync(f->ft[1].p + o, 0, vb, ms));
        MP_CUDA(cudaEventRecord(f->mev[iw], ms));
        MP_CUDA(cudaStreamWaitEvent(st, f->mev[iw], 0));
    }
    {  // every solve's status, as Ppe::read_stats judges it
        std::vector<BicgScalars> hs((size_t)2 * M);
        MP_CUDA(cudaMemcpyAsync(hs.data(), f->stats.p, sizeof(BicgScalars) * 2 * M,
                                cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        for (int iw = 0; iw < M; iw++) {
            const Ppe &S = *f->P[iw];
            for (int q = 0; q < (S.sys.nsys == nv + 1 ? 1 : 2); q++) {
                SolveStats ss;
                S.stats_of(hs[2 * iw + q], &ss);
                if (ss.status != MP_OK)
                    return fail(ss.status,
                                "Fourier pressure solve (mode %d, %s part): status %d after %d "
                                "iterations, relres %g", iw, q ? "imaginary" : "real",
                                ss.status, ss.iters, ss.relres);
            }
        }
    }
    const double *pr = f->ft[0].p, *pi = f->ft[1].p;
    // calc_vel_corr: the new velocity coefficients go to scratch (nv x N >= nv x M)
    // until the old ones have served the boundary rows
    double *unr = f->uphi.p, *uni = f->vphi.p, *vnr = f->xy.p, *vni = f->z.p;
    double *wnr = f->ft[2].p, *wni = f->ft[3].p;
    k_fsf_corr3<<<bm, 256, 0, st>>>(d, cv.cols, cv.w[0], cv.w[1], f->k.p, f->dt / f->rho, pr, pi,
                                    f->h[0][0].p, f->h[0][1].p, f->h[1][0].p, f->h[1][1].p,
                                    f->h[2][0].p, f->h[2][1].p, unr, uni, vnr, vni, wnr, wni);
    MP_CHECK_LAUNCH();
    const unsigned bb = f->serial ? 1u : bm, tb = f->serial ? 1u : 256u;
    const uint8_t *qd[3] = {f->udir.p, f->vdir.p, f->wdir.p};
    double *qnr[3] = {unr, vnr, wnr}, *qni[3] = {uni, vni, wni};
    for (int a = 0; a < 3; a++) {
        k_fsf_bnd<<<bb, tb, 0, st>>>(d, cv.cols, cv.w[0], cv.w[1], cv.bflag, f->pdir.p, qd[a],
                                     f->normal.p, f->serial, f->f[a][0].p, f->f[a][1].p, qnr[a],
                                     qni[a]);
        MP_CHECK_LAUNCH();
    }
    // the step's end (:260-263): old <- new, source history <- this step's sources
    const size_t mb = sizeof(double) * nm;
    for (int a = 0; a < 3; a++) {
        MP_CUDA(cudaMemcpyAsync(f->f[a][0].p, qnr[a], mb, cudaMemcpyDeviceToDevice, st));
        MP_CUDA(cudaMemcpyAsync(f->f[a][1].p, qni[a], mb, cudaMemcpyDeviceToDevice, st));
        for (int q = 0; q < 2; q++)
            MP_CUDA(cudaMemcpyAsync(f->s2[a][q].p, f->s[a][q].p, mb, cudaMemcpyDeviceToDevice, st));
    }
    MP_CUDA(cudaMemcpyAsync(f->f[3][0].p, pr, mb, cudaMemcpyDeviceToDevice, st));
    MP_CUDA(cudaMemcpyAsync(f->f[3][1].p, pi, mb, cudaMemcpyDeviceToDevice, st));
    // physical new fields
    double *outs[4] = {vel_new[0], vel_new[1], vel_new[2], p_new};
    for (int a = 0; a < 4; a++) {
        k_fsf_idft<<<bn, 256, 0, st>>>(d, f->f[a][0].p, f->f[a][1].p, f->itr.p, f->iti.p,
                                       f->phys[a].p);
        MP_CHECK_LAUNCH();
        const double *res = f->phys[a].p;
        if (f->node_major) {
            // stage is free again: the inputs were transposed out of it at the start
            k_fsf_to_nodes<<<bn, 256, 0, st>>>(nv, d.N, f->phys[a].p, f->stage.p);
            MP_CHECK_LAUNCH();
            res = f->stage.p;
        }
        MP_CUDA(cudaMemcpyAsync(outs[a], res, sizeof(double) * nn, cudaMemcpyDefault, st));
    }
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

extern "C" int mp_fsf_destroy(mp_fsf f) {
    if (f) {
        for (Ppe *p : f->P)
            delete p;
        delete f;
    }
    return MP_OK;
}
