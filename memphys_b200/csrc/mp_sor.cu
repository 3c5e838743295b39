// mp_sor.cu -- the reference's `sor` solver type (SOLVER::SOR, solver.cpp:243-281).
//
// The reference sweeps the rows in index order: phi = (b_i - sum_{j != i} a_ij x_j)
// / a_ii, x_i = omega phi + (1 - omega) x_i, omega = 1.4 (class.hpp:212), on the
// unbordered system (solver.cpp:30-31), n_iter sweeps.  A sweep in index order is
// sequential, so on the GPU the rows are coloured first -- greedily, in index order,
// each row taking the smallest colour that none of its stencil members and none of
// the rows whose stencils contain it already hold -- and a sweep visits the colours
// in turn, all rows of one colour in parallel (they do not read one another).  This
// is the same SOR update in another row order (multicolour SOR): it converges to
// the same solution, its iterates differ from the index-order ones.  The graph is
// that of the nonzero coefficients.  The residual is recomputed every SOR_CHECK
// sweeps; the sweeps stop once ||b - A x|| / ||b|| <= tol (the reference always
// runs n_iter sweeps) or after maxit sweeps.
#include <algorithm>
#include <cmath>
#include <vector>
#include "mp_ppe.cuh"

namespace mp {

constexpr int SOR_THREADS = 256;
constexpr int SOR_CHECK = 10;

struct Sor {
    int ncolours = 0;
    std::vector<int> start;  // rows of colour c: rows[start[c] .. start[c + 1])
    dbuf<int> rows;
    dbuf<double> partial, sums;
    int nb = 0;
};

namespace {

// one row of colour c per thread; the row's entries are K apart by SLICE in the
// sliced layout, the self entry is found by its column (solver.cpp:257-263)
__global__ void __launch_bounds__(SOR_THREADS)
    k_sor_colour(EllView<double> A, const int *__restrict__ rows, int n, const double *__restrict__ b,
                 double *__restrict__ x, double omega) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const int i = rows[t];
    const size_t base = (size_t)(i / SLICE) * A.K * SLICE + (i % SLICE);
    double s = b[i], d = 0.0;
    for (int k = 0; k < A.K; k++) {
        const int c = A.cols[base + (size_t)k * SLICE];
        const double v = A.vals[base + (size_t)k * SLICE];
        if (c == i)
            d = v;
        else
            s -= v * x[c];
    }
    x[i] = omega * (s / d) + (1.0 - omega) * x[i];
}

// partial sums of |r|, r^2, |b|, b^2 over the rows (r = b - A x), block order
__global__ void __launch_bounds__(SOR_THREADS)
    k_sor_residual(EllView<double> A, const double *__restrict__ b, const double *__restrict__ x,
                   double *__restrict__ partial) {
    __shared__ double sm[4 * 32];
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < A.nrows; i += gridDim.x * blockDim.x) {
        const size_t base = (size_t)(i / SLICE) * A.K * SLICE + (i % SLICE);
        double r = b[i];
        for (int k = 0; k < A.K; k++)
            r -= A.vals[base + (size_t)k * SLICE] * x[A.cols[base + (size_t)k * SLICE]];
        v[0] += fabs(r);
        v[1] += r * r;
        v[2] += fabs(b[i]);
        v[3] += b[i] * b[i];
    }
    block_sum<4>(v, sm);
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; q++)
            partial[(size_t)q * gridDim.x + blockIdx.x] = v[q];
}

__global__ void k_sor_finish(const double *__restrict__ partial, int nb, double *__restrict__ out) {
    __shared__ double sm[32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
        acc += partial[(size_t)blockIdx.x * nb + b];
    double v[1] = {acc};
    block_sum<1>(v, sm);
    if (threadIdx.x == 0)
        out[blockIdx.x] = v[0];
}

}  // namespace

int sor_setup(Ppe &P, cudaStream_t st) {
    const int nv = P.sys.nv, K = P.sys.K;
    const size_t tot = (size_t)ell_padded_rows(nv) * K;
    std::vector<int> cols(tot);
    std::vector<double> vals(tot);
    MP_CUDA(cudaMemcpyAsync(cols.data(), P.sys.A.cols.p, sizeof(int) * tot, cudaMemcpyDeviceToHost,
                            st));
    MP_CUDA(cudaMemcpyAsync(vals.data(), P.sys.A.v64.p, sizeof(double) * tot,
                            cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    auto at = [&](int i, int k) { return (size_t)(i / SLICE) * K * SLICE + (size_t)k * SLICE + i % SLICE; };
    // solver.cpp:264-268: a diagonal this small ends the solve in the reference
    for (int i = 0; i < nv; i++) {
        double d = 0.0;
        for (int k = 0; k < K; k++)
            if (cols[at(i, k)] == i)
                d = vals[at(i, k)];
        if (std::fabs(d) < 1e-10)
            return fail(MP_BAD_ARG, "SOLVER::SOR diag_coeff at row no.: %d is close to zero: %g", i,
                        d);
    }
    // the matrix graph is that of the nonzero coefficients (a Dirichlet row keeps its
    // stencil's columns with zero values); reverse adjacency (rows that read i), CSR
    auto link = [&](int i, int k) {
        const int j = cols[at(i, k)];
        return j != i && j >= 0 && j < nv && vals[at(i, k)] != 0.0 ? j : -1;
    };
    std::vector<int> rcount(nv + 1, 0);
    for (int i = 0; i < nv; i++)
        for (int k = 0; k < K; k++) {
            const int j = link(i, k);
            if (j >= 0)
                rcount[j + 1]++;
        }
    for (int i = 0; i < nv; i++)
        rcount[i + 1] += rcount[i];
    std::vector<int> radj(rcount[nv]), fill(rcount.begin(), rcount.end() - 1);
    for (int i = 0; i < nv; i++)
        for (int k = 0; k < K; k++) {
            const int j = link(i, k);
            if (j >= 0)
                radj[fill[j]++] = i;
        }
    // greedy colouring in index order
    std::vector<int> colour(nv, -1), mark;
    int nc = 0;
    for (int i = 0; i < nv; i++) {
        mark.assign(nc + 1, 0);
        for (int k = 0; k < K; k++) {
            const int j = link(i, k);
            if (j >= 0 && colour[j] >= 0)
                mark[colour[j]] = 1;
        }
        for (int q = rcount[i]; q < rcount[i + 1]; q++)
            if (colour[radj[q]] >= 0)
                mark[colour[radj[q]]] = 1;
        int c = 0;
        while (mark[c])
            c++;
        colour[i] = c;
        nc = std::max(nc, c + 1);
    }
    Sor *S_ = new Sor;
    P.sor = S_;
    S_->ncolours = nc;
    S_->start.assign(nc + 1, 0);
    for (int i = 0; i < nv; i++)
        S_->start[colour[i] + 1]++;
    for (int c = 0; c < nc; c++)
        S_->start[c + 1] += S_->start[c];
    std::vector<int> rows(nv), pos(S_->start.begin(), S_->start.end() - 1);
    for (int i = 0; i < nv; i++)
        rows[pos[colour[i]]++] = i;
    MP_TRY(S_->rows.alloc(nv));
    MP_CUDA(cudaMemcpyAsync(S_->rows.p, rows.data(), sizeof(int) * nv, cudaMemcpyHostToDevice, st));
    S_->nb = std::max(1, std::min(4 * sm_count(), (nv + SOR_THREADS - 1) / SOR_THREADS));
    MP_TRY(S_->partial.alloc((size_t)4 * S_->nb));
    MP_TRY(S_->sums.alloc(4));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

void sor_destroy(Sor *s) { delete s; }

// W.x holds the initial guess and receives the result; W.b64 the right-hand side
int sor_solve(Ppe &P, cudaStream_t st, SolveStats *out) {
    Sor &S_ = *P.sor;
    const EllView<double> A = P.sys.A.view64();
    const double omega = P.cfg.sor_omega;
    double sums[4] = {0, 0, 0, 0};
    auto residual = [&]() -> int {
        k_sor_residual<<<S_.nb, SOR_THREADS, 0, st>>>(A, P.W.b64.p, P.W.x.p, S_.partial.p);
        MP_CHECK_LAUNCH();
        k_sor_finish<<<4, SOR_THREADS, 0, st>>>(S_.partial.p, S_.nb, S_.sums.p);
        MP_CHECK_LAUNCH();
        MP_CUDA(cudaMemcpyAsync(sums, S_.sums.p, sizeof(sums), cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
        return MP_OK;
    };
    int sweeps = 0;
    out->status = MP_NOT_CONVERGED;
    MP_TRY(residual());
    auto relres = [&]() { return sums[3] > 0 ? std::sqrt(sums[1] / sums[3]) : std::sqrt(sums[1]); };
    if (relres() <= P.cfg.tol)
        out->status = MP_OK;
    while (out->status != MP_OK && sweeps < P.cfg.maxit) {
        const int burst = std::min(SOR_CHECK, P.cfg.maxit - sweeps);
        for (int q = 0; q < burst; q++)
            for (int c = 0; c < S_.ncolours; c++) {
                const int n = S_.start[c + 1] - S_.start[c];
                k_sor_colour<<<(n + SOR_THREADS - 1) / SOR_THREADS, SOR_THREADS, 0, st>>>(
                    A, S_.rows.p + S_.start[c], n, P.W.b64.p, P.W.x.p, omega);
                MP_CHECK_LAUNCH();
            }
        sweeps += burst;
        MP_TRY(residual());
        if (!std::isfinite(sums[1])) {
            out->status = MP_NAN_DETECTED;
            break;
        }
        if (relres() <= P.cfg.tol)
            out->status = MP_OK;
    }
    out->iters = sweeps;
    out->outer = 0;
    out->abs_res = std::sqrt(sums[1]);
    out->relres = relres();
    return MP_OK;
}

}  // namespace mp
