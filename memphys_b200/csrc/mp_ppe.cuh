// mp_ppe.cuh -- the pressure-solve handle (SOLVER for the pressure Poisson
// equation) used by mp_ppe_* and by the fractional-step handle.
#pragma once
#include "mp_krylov.cuh"

struct mp_cloud_s;

namespace mp {

struct Cfg {
    double tol, inner_tol, cheb_lower, sor_omega;
    int maxit, precond, precision, guess, max_refine, amg_max_levels, amg_coarse_size,
        smoother_sweeps, guess_vectors;
    static Cfg from(const mp_solver_cfg &c);
};
// MP_OK, or MP_BAD_ARG with the reason for an inconsistent solver configuration
int solver_cfg_check(const mp_solver_cfg &c);
// the same for the solvers inside a time integrator, which run as CUDA graphs:
// the SOR sweeps (MP_PRECOND_SOR, SOLVER only) are refused there
int integrator_cfg_check(const mp_solver_cfg &c);

struct SolveStats {
    int iters = 0, outer = 0, status = MP_OK;
    double relres = 0, abs_res = 0;
};

struct Sor;  // multicolour SOR sweeps (mp_sor.cu)

// Device vectors of one solve (FP64, and FP32 for mixed precision)
struct Krylov {
    int nv = 0, nsys = 0, bordered = 0;
    dbuf<double> x, b64, r, r0, p, v, s, t, y, z, res64;
    dbuf<float> e32, b32, r32, r032, p32, v32, s32, t32, y32, z32;
    dbuf<double> partials;
    dbuf<unsigned int> ticket;
    dbuf<BicgScalars> scal;
    // bordered systems under the multigrid: ve = V(1), the cycle applied to the
    // constant vector, ave = A ve and sve = sum(ve), per Krylov precision (empty when
    // the preconditioner is not deflated); the weights of the input's mean, 1 on
    // interior rows and dbeta on boundary rows (dflag), and their sum dwe
    dbuf<double> ve, ave;
    dbuf<float> ve32, ave32;
    double sve = 0.0, sve32 = 0.0;
    dbuf<unsigned char> dflag;
    double dbeta = 1.0, dwe = 0.0;
    int alloc(int nv, int bordered, bool mixed, bool external_pc);
};

struct Ppe {
    Cfg cfg{};
    PpeSystem sys;
    Krylov W;
    GraphExec graph;
    std::shared_ptr<Ell> shared_cols;
    cudaStream_t capture_stream = nullptr;
    Sor *sor = nullptr;  // MP_PRECOND_SOR: the row colouring
    ~Ppe();
    // border_rule 1: bordered unless a boundary node is Dirichlet (solver.cpp:29-38);
    // 0: never bordered (systems with a nonsingular diagonal, e.g. implicit velocity).
    // stencil_order: keep each row's entries in the cloud's stencil order (systems
    // whose values are rewritten in that order later); otherwise entries 1..K-1 are
    // sorted by column (ell_sort_rows), the same matrix with better-coalesced gathers.
    int create(mp_cloud_s *c, const uint8_t *boundary, const uint8_t *dirichlet,
               const double *normal, double unsteady, double conv, double diff,
               const mp_solver_cfg &cfg, cudaStream_t st, int border_rule = 1,
               bool stencil_order = false);
    // after the operator's values changed in place: the Jacobi diagonal again
    // (systems without a multigrid hierarchy only)
    int refresh_diag(cudaStream_t st);
    // absolute floor of the stopping residual norm, kept until changed (default 0)
    int set_abs_tol(double atol, cudaStream_t st);
    int pk() const {
        return cfg.precond == MP_PRECOND_AMG ? PK_EXTERNAL
                                             : (cfg.precond == MP_PRECOND_JACOBI ? PK_JACOBI : PK_NONE);
    }
    // kernel sequences (each can be issued eagerly or captured)
    int issue_prologue64(cudaGraphConditionalHandle h, cudaStream_t st);
    int issue_sweep64(cudaGraphConditionalHandle h, cudaStream_t st);
    int issue_epilogue64(cudaStream_t st);
    int issue_ir_setup(cudaStream_t st);
    int issue_ir_residual(cudaGraphConditionalHandle h, cudaStream_t st);
    int issue_ir_inner_prologue(cudaGraphConditionalHandle h, cudaStream_t st);
    int issue_ir_sweep(cudaGraphConditionalHandle h, cudaStream_t st);
    int issue_ir_update(cudaStream_t st);
    // initial guess x = x + theta f with theta minimising ||b - A x|| (FP64 operator,
    // border included); f has nv entries (its border entry is zero)
    int issue_guess_min_residual(const double *f, cudaStream_t st);
    int build_solve_graph(GraphBuilder &gb);
    int solve_eager(cudaStream_t st);
    // solve with W.b64 as rhs and W.x as initial guess / solution
    int solve_resident(cudaStream_t st, bool use_graph);
    int read_stats(cudaStream_t st, SolveStats *out);
    // the same judgement of a solve's final scalars already on the host
    void stats_of(const BicgScalars &hs, SolveStats *out) const;
    cudaStream_t cap_stream();
};

// MP_PRECOND_SOR (mp_sor.cu): colour the rows once; sweep with W.x as the initial
// guess and W.b64 as the right-hand side
int sor_setup(Ppe &P, cudaStream_t st);
int sor_solve(Ppe &P, cudaStream_t st, SolveStats *out);
void sor_destroy(Sor *s);

}  // namespace mp

struct mp_ppe_s {
    mp::Ppe P;
    bool use_graph = true;
};
