// mp_eig.cu -- largest-magnitude eigenvalue of an operator (calc_dt's eigensolve).
//
// The reference computes the time step from the eigenvalue of largest magnitude of
// grad_x, grad_y, [grad_z] and the Laplacian with Spectra's GenEigsSolver (nev = 1,
// ncv = 10, LARGEST_MAGN; general_functions.cpp:4-24, parameters.cpp:269-296).
// Here: explicitly restarted Arnoldi.  Each cycle builds an ncv-step Arnoldi
// factorisation A V = V H + h f e^T on the GPU (SpMV through the operator's ELL
// kernel, classical Gram-Schmidt applied twice, every dot product a deterministic
// two-pass reduction), the host solves the small Hessenberg eigenproblem (shifted QR
// in complex arithmetic, eigenvector by inverse iteration), and the cycle stops
// when the Ritz residual |h y_ncv| of the largest-magnitude Ritz pair falls below
// tol |lambda|.  Otherwise the next cycle starts from Re(V y) + Im(V y), which
// holds both members of a complex-conjugate pair.
#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>
#include "mp_common.cuh"
#include "mp_ell.cuh"

namespace mp {

// implemented in mp_ell.cu: the FP64 view of an operator handle
int op_view64(mp_op op, EllView<double> *view);

namespace {

constexpr int EIG_THREADS = 256;

// uniform in [0.5, 1.5) from a counter hash (splitmix64), so the start vector is
// the same on every device and run
__global__ void k_eig_start(double *v, int n, uint64_t seed) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint64_t z = seed * 0x9E3779B97F4A7C15ull + (uint64_t)i + 1;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    v[i] = 0.5 + (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// partial[k * gridDim.x + b] = sum over block b's rows of X[k][i] * w[i], k < nk
__global__ void __launch_bounds__(EIG_THREADS)
    k_eig_dots(const double *__restrict__ X, size_t ld, int nk, const double *__restrict__ w, int n,
               double *__restrict__ partial) {
    __shared__ double sm[32];
    for (int k = 0; k < nk; k++) {
        const double *x = X + (size_t)k * ld;
        double acc = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
            acc = fma(x[i], w[i], acc);
        double v[1] = {acc};
        block_sum<1>(v, sm);
        if (threadIdx.x == 0)
            partial[(size_t)k * gridDim.x + blockIdx.x] = v[0];
    }
}

// out[k] = sum of the nb partials of k, in block order (one block per k)
__global__ void k_eig_finish(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    __shared__ double sm[32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        acc += partial[(size_t)blockIdx.x * nb + b];
    double v[1] = {acc};
    block_sum<1>(v, sm);
    if (threadIdx.x == 0)
        out[blockIdx.x] = v[0];
}

// y[i] = beta * y[i] + sum_k c[k] X[k][i]
__global__ void k_eig_combine(const double *__restrict__ X, size_t ld, int nk,
                              const double *__restrict__ c, double beta, double *__restrict__ y,
                              int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double acc = beta == 0.0 ? 0.0 : beta * y[i];
    for (int k = 0; k < nk; k++)
        acc = fma(c[k], X[(size_t)k * ld + i], acc);
    y[i] = acc;
}

__global__ void k_eig_scale(const double *__restrict__ w, double s, double *__restrict__ v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] = w[i] * s;
}

using cd = std::complex<double>;

// Eigenvalues of the m x m upper Hessenberg matrix H (row-major, complex copy) by
// the shifted QR iteration: Wilkinson shift from the trailing 2 x 2 block of the
// active window, one Givens sweep for QR and its transpose for RQ, deflation when a
// subdiagonal entry falls below eps times its neighbours.
bool hessenberg_eigenvalues(int m, std::vector<cd> H, std::vector<cd> &ev) {
    const double eps = 2.220446049250313e-16;
    ev.assign(m, cd(0.0));
    auto at = [&](int i, int j) -> cd & { return H[(size_t)i * m + j]; };
    int hi = m - 1, iter = 0, total = 0;
    std::vector<cd> cs(m), sn(m);
    while (hi >= 0) {
        int lo = hi;
        while (lo > 0) {
            const double s = std::abs(at(lo - 1, lo - 1)) + std::abs(at(lo, lo));
            if (std::abs(at(lo, lo - 1)) <= eps * (s > 0 ? s : 1.0)) {
                at(lo, lo - 1) = 0.0;
                break;
            }
            lo--;
        }
        if (lo == hi) {
            ev[hi] = at(hi, hi);
            hi--;
            iter = 0;
            continue;
        }
        if (++total > 60 * m)
            return false;
        iter++;
        const cd a = at(hi - 1, hi - 1), b = at(hi - 1, hi), c = at(hi, hi - 1), d = at(hi, hi);
        const cd half_tr = 0.5 * (a + d);
        const cd disc = std::sqrt(half_tr * half_tr - (a * d - b * c));
        const cd mu1 = half_tr + disc, mu2 = half_tr - disc;
        cd mu = std::abs(mu1 - d) < std::abs(mu2 - d) ? mu1 : mu2;
        if (iter % 10 == 0)  // an exceptional shift breaks a rare cycle
            mu += cd(std::abs(c), 0.5 * std::abs(c));
        for (int k = lo; k <= hi; k++)
            at(k, k) -= mu;
        for (int k = lo; k < hi; k++) {  // H - mu I = Q R
            const cd x = at(k, k), y = at(k + 1, k);
            const double r = std::hypot(std::abs(x), std::abs(y));
            cs[k] = r > 0 ? x / r : cd(1.0);
            sn[k] = r > 0 ? y / r : cd(0.0);
            for (int j = k; j <= hi; j++) {
                const cd u = at(k, j), v = at(k + 1, j);
                at(k, j) = std::conj(cs[k]) * u + std::conj(sn[k]) * v;
                at(k + 1, j) = -sn[k] * u + cs[k] * v;
            }
        }
        for (int k = lo; k < hi; k++) {  // R Q + mu I
            const int top = std::min(k + 2, hi);
            for (int i = lo; i <= top; i++) {
                const cd u = at(i, k), v = at(i, k + 1);
                at(i, k) = u * cs[k] + v * sn[k];
                at(i, k + 1) = -u * std::conj(sn[k]) + v * std::conj(cs[k]);
            }
        }
        for (int k = lo; k <= hi; k++)
            at(k, k) += mu;
    }
    return true;
}

// Unit eigenvector of H for the eigenvalue lam: two steps of inverse iteration with
// (H - lam I) factorised once by Gaussian elimination with partial pivoting (a
// pivot that vanishes is replaced by eps |H|, the usual guard).
std::vector<cd> hessenberg_eigenvector(int m, const std::vector<cd> &H, cd lam) {
    double hn = 0.0;
    for (const cd &h : H)
        hn = std::max(hn, std::abs(h));
    const double tiny = 2.220446049250313e-16 * (hn > 0 ? hn : 1.0);
    std::vector<cd> M(H);
    for (int i = 0; i < m; i++)
        M[(size_t)i * m + i] -= lam;
    std::vector<int> piv(m);
    for (int k = 0; k < m; k++) {
        int p = k;
        for (int i = k + 1; i < m; i++)
            if (std::abs(M[(size_t)i * m + k]) > std::abs(M[(size_t)p * m + k]))
                p = i;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < m; j++)
                std::swap(M[(size_t)k * m + j], M[(size_t)p * m + j]);
        if (std::abs(M[(size_t)k * m + k]) < tiny)
            M[(size_t)k * m + k] = tiny;
        for (int i = k + 1; i < m; i++) {
            const cd f = M[(size_t)i * m + k] / M[(size_t)k * m + k];
            M[(size_t)i * m + k] = f;
            for (int j = k + 1; j < m; j++)
                M[(size_t)i * m + j] -= f * M[(size_t)k * m + j];
        }
    }
    std::vector<cd> y(m, cd(1.0));
    for (int pass = 0; pass < 2; pass++) {
        for (int k = 0; k < m; k++) {  // forward: L (unit) with the row swaps
            std::swap(y[k], y[piv[k]]);
            for (int i = k + 1; i < m; i++)
                y[i] -= M[(size_t)i * m + k] * y[k];
        }
        for (int k = m - 1; k >= 0; k--) {  // back: U
            cd s = y[k];
            for (int j = k + 1; j < m; j++)
                s -= M[(size_t)k * m + j] * y[j];
            y[k] = s / M[(size_t)k * m + k];
        }
        double nrm = 0.0;
        for (const cd &v : y)
            nrm += std::norm(v);
        nrm = std::sqrt(nrm);
        for (cd &v : y)
            v /= nrm;
    }
    return y;
}

struct Arnoldi {
    int n, m, nb;
    cudaStream_t s;
    EllView<double> A;
    dbuf<double> V, w, partial, coef;
    std::vector<double> hbuf;

    int dots(const double *X, int nk, const double *x, std::vector<double> &out) {
        k_eig_dots<<<nb, EIG_THREADS, 0, s>>>(X, (size_t)n, nk, x, n, partial.p);
        MP_CHECK_LAUNCH();
        k_eig_finish<<<nk, EIG_THREADS, 0, s>>>(partial.p, nb, coef.p);
        MP_CHECK_LAUNCH();
        out.resize(nk);
        MP_CUDA(cudaMemcpyAsync(out.data(), coef.p, sizeof(double) * nk, cudaMemcpyDeviceToHost,
                                s));
        MP_CUDA(cudaStreamSynchronize(s));
        return MP_OK;
    }
    // y = beta y + X c (c from the host)
    int combine(const double *X, int nk, const std::vector<double> &c, double beta, double *y) {
        MP_CUDA(cudaMemcpyAsync(coef.p, c.data(), sizeof(double) * nk, cudaMemcpyHostToDevice, s));
        k_eig_combine<<<(n + EIG_THREADS - 1) / EIG_THREADS, EIG_THREADS, 0, s>>>(
            X, (size_t)n, nk, coef.p, beta, y, n);
        MP_CHECK_LAUNCH();
        MP_CUDA(cudaStreamSynchronize(s));  // coef is reused by the next call
        return MP_OK;
    }
    int normalize_into(const double *x, double *v, double *nrm) {
        std::vector<double> d;
        MP_TRY(dots(x, 1, x, d));
        *nrm = std::sqrt(d[0]);
        if (!(*nrm > 0.0) || !std::isfinite(*nrm))
            return MP_OK;
        k_eig_scale<<<(n + EIG_THREADS - 1) / EIG_THREADS, EIG_THREADS, 0, s>>>(x, 1.0 / *nrm, v, n);
        MP_CHECK_LAUNCH();
        return MP_OK;
    }
    // m-step factorisation from V[0] (unit); H is (m+1) x m row-major; returns the
    // number of steps taken (fewer on breakdown, when an invariant subspace is found)
    int factorise(std::vector<double> &H, int *steps, double *scale) {
        H.assign((size_t)(m + 1) * m, 0.0);
        std::vector<double> h, h2, neg;
        for (int j = 0; j < m; j++) {
            const double *vj = V.p + (size_t)j * n;
            MP_TRY(ell_spmv<double>(A, vj, w.p, 1.0, 0.0, s));
            std::vector<double> hj(j + 1, 0.0);
            for (int pass = 0; pass < 2; pass++) {  // classical Gram-Schmidt, twice
                MP_TRY(dots(V.p, j + 1, w.p, h));
                neg.resize(j + 1);
                for (int k = 0; k <= j; k++) {
                    hj[k] += h[k];
                    neg[k] = -h[k];
                }
                MP_TRY(combine(V.p, j + 1, neg, 1.0, w.p));
            }
            double beta = 0.0;
            MP_TRY(normalize_into(w.p, V.p + (size_t)(j + 1) * n, &beta));
            for (int k = 0; k <= j; k++) {
                H[(size_t)k * m + j] = hj[k];
                *scale = std::max(*scale, std::fabs(hj[k]));
            }
            H[(size_t)(j + 1) * m + j] = beta;
            if (!(beta > 1e-13 * std::max(*scale, 1e-300))) {
                *steps = j + 1;
                return MP_OK;
            }
        }
        *steps = m;
        return MP_OK;
    }
};

}  // namespace
}  // namespace mp

using namespace mp;

extern "C" int mp_op_largest_eig(mp_op op, int ncv, double tol, int max_restarts, uint64_t seed,
                                 double *re, double *im, int *restarts, mp_stream stream) {
    if (!op || !re || !im)
        return fail(MP_BAD_ARG, "mp_op_largest_eig: null argument");
    EllView<double> A{};
    MP_TRY(op_view64(op, &A));
    if (A.nrows != A.ncols)
        return fail(MP_BAD_ARG, "mp_op_largest_eig: square operators only (%d x %d)", A.nrows,
                    A.ncols);
    if (ncv < 3 || max_restarts < 1 || !(tol > 0.0))
        return fail(MP_BAD_ARG, "mp_op_largest_eig: ncv >= 3, max_restarts >= 1, tol > 0");
    Arnoldi ar;
    ar.n = A.nrows;
    ar.m = std::min(ncv, A.nrows);
    ar.nb = std::max(1, std::min(4 * sm_count(), (ar.n + EIG_THREADS - 1) / EIG_THREADS));
    ar.s = S(stream);
    ar.A = A;
    MP_TRY(ar.V.alloc((size_t)(ar.m + 1) * ar.n));
    MP_TRY(ar.w.alloc(ar.n));
    MP_TRY(ar.partial.alloc((size_t)ar.nb * (ar.m + 1)));
    MP_TRY(ar.coef.alloc(ar.m + 1));
    k_eig_start<<<(ar.n + EIG_THREADS - 1) / EIG_THREADS, EIG_THREADS, 0, ar.s>>>(ar.w.p, ar.n,
                                                                                  seed);
    MP_CHECK_LAUNCH();
    double nrm = 0.0;
    MP_TRY(ar.normalize_into(ar.w.p, ar.V.p, &nrm));
    cd lam = 0.0;
    double res = INFINITY;
    for (int r = 0; r < max_restarts; r++) {
        std::vector<double> H;
        int k = 0;
        double scale = 0.0;
        MP_TRY(ar.factorise(H, &k, &scale));
        std::vector<cd> Hk((size_t)k * k);
        for (int i = 0; i < k; i++)
            for (int j = 0; j < k; j++)
                Hk[(size_t)i * k + j] = H[(size_t)i * ar.m + j];
        std::vector<cd> ev;
        if (!hessenberg_eigenvalues(k, Hk, ev))
            return fail(MP_NOT_CONVERGED, "mp_op_largest_eig: Hessenberg QR did not converge");
        int best = 0;
        for (int i = 1; i < k; i++) {  // largest magnitude; of a conjugate pair the + one
            const double a = std::abs(ev[i]), b = std::abs(ev[best]);
            if (a > b * (1 + 1e-12) || (a >= b * (1 - 1e-12) && ev[i].imag() > ev[best].imag()))
                best = i;
        }
        lam = ev[best];
        const std::vector<cd> y = hessenberg_eigenvector(k, Hk, lam);
        res = k < ar.m ? 0.0 : std::fabs(H[(size_t)ar.m * ar.m + (ar.m - 1)]) * std::abs(y[k - 1]);
        if (restarts)
            *restarts = r + 1;
        if (res <= tol * std::abs(lam)) {
            *re = lam.real();
            *im = lam.imag();
            return MP_OK;
        }
        // restart from Re(V y) + Im(V y), normalised
        std::vector<double> c(k);
        for (int i = 0; i < k; i++)
            c[i] = y[i].real() + y[i].imag();
        MP_TRY(ar.combine(ar.V.p, k, c, 0.0, ar.w.p));
        MP_TRY(ar.normalize_into(ar.w.p, ar.V.p, &nrm));
        if (!(nrm > 0.0))
            return fail(MP_BREAKDOWN, "mp_op_largest_eig: zero restart vector");
    }
    *re = lam.real();
    *im = lam.imag();
    return fail(MP_NOT_CONVERGED,
                "mp_op_largest_eig: Ritz residual %.3e of |lambda| %.6e after %d restarts "
                "(tol %.1e)",
                res, std::abs(lam), max_restarts, tol);
}
