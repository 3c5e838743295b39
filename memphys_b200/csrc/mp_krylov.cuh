// mp_krylov.cuh -- the bordered pressure-Poisson system and its BiCGSTAB solver.
//
// System (SOLVER::calc_coeff_matrix, solver.cpp:165-214): nv stencil rows of
// width K (ELL, self column first), and when no boundary node is Dirichlet
// the regularisation border: every row i < nv gets + x[nv], and row nv is
// sum_i x_i (solver.cpp:205-213).  The border is applied inside the SpMV
// kernels: the row sum reuses the self gather of each row (stencil column 0).
//
// BiCGSTAB follows Eigen's BiCGSTAB (van der Vorst 1992, right
// preconditioned, restart when rho collapses, stop when ||r||^2 <= tol^2
// ||b||^2 or after maxit iterations; solver.cpp:154-155,339).  All scalars
// stay on the device; each kernel reads what it needs at launch and the last
// block of each reduction writes the next scalars, so an iteration is a fixed
// sequence of launches that a CUDA graph can loop over.
#pragma once
#include "mp_ell.cuh"
#include "mp_graph.cuh"

namespace mp {

struct Amg;  // aggregation multigrid preconditioner (mp_amg.cu)

struct BicgScalars {
    double rho, rho_old, alpha, omega, r0_sq, b_sq, rr, tol2;
    double dot_rv, dot_tt, dot_ts;
    double scale;       // mixed precision: norm of the FP64 residual being solved for
    double rr_true;     // ||b - A x||^2 recomputed in FP64
    int it, maxit, restarts, need_restart, done, status, zero_x;
    int half;  // 1 when the solve stopped after the first half of its last iteration
    // iterative refinement (outer) state; half_total counts the inner solves that
    // stopped after a half iteration
    int outer_it, outer_max, outer_done, total_inner, half_total;
    double tol_outer2, b64_sq;
    double relres0;     // ||b - A x0|| / ||b|| of the initial guess (first residual of a solve)
    double abs_tol2;    // absolute floor of the stopping ||r||^2 (0: the relative test alone)
    double guess_theta; // weight of the learned correction in the last initial guess
    // bordered systems under the multigrid: the mean of each preconditioner input
    // (dfl_a) and the constant that satisfies the border row (dfl_c), first and second
    // application of a sweep (see Defl in mp_krylov.cu)
    double dfl_a[2], dfl_c[2];
};

struct PpeSystem {
    int nv = 0, nsys = 0, K = 0, bordered = 0;
    Ell A;                 // stencil rows, FP64 (+FP32 copy for mixed precision)
    dbuf<double> dinv;     // Jacobi: 1 / self coefficient
    dbuf<float> dinv32;
    // FP32 Krylov: the operator in FP32 difference form, (column, value) pairs
    dbuf<float> d32;
    dbuf<int2> dpk;
    EllView<float> diff32() const {
        return EllView<float>{A.nrows, A.ncols, A.K, A.cols.p, d32.p, A.soff.p, dpk.p};
    }
    Amg *amg = nullptr;
};

// Preconditioner kinds for the fused update kernels
enum { PK_NONE = 0, PK_JACOBI = 1, PK_EXTERNAL = 2 };

struct KrylovWork;  // device vectors + scalars (mp_krylov.cu)

}  // namespace mp
