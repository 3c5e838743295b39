/*
 * memphys.h -- C ABI of libmemphys_cuda.so, the B200 (sm_100a) hot path of
 * the MeMPhyS meshless solver: PHS-RBF-FD stencil weights, the fixed-width
 * grad_x/grad_y/grad_z/laplacian operators applied as SpMV, and the
 * fractional-step pressure-Poisson solve.
 *
 * Conventions
 *  - Every entry point returns an int status (mp_status).  On failure a
 *    message is kept per host thread and read with mp_last_error().  The
 *    reference reports the same failures with printf + throw bad_exception()
 *    (e.g. cloud.cpp:632-636, solver.cpp:317-321); the C++ adapters in
 *    memphys_b200/host turn non-OK statuses back into that exception.
 *  - Array arguments may be host or device memory (unified addressing).
 *    Host arrays are copied in/out on the call's stream; device arrays are
 *    used in place.  Handles own their device buffers.
 *  - Handles are not re-entrant: one handle per host thread / stream.
 *  - Node ordering, stencil ordering and the CSR-aligned weight layout are
 *    those of the reference's CLOUD (cloud.cpp:251-258): stencil row i has
 *    exactly n entries, the node itself first.
 *  - Reference paths are relative to "MeMPhyS Latest Version/" of
 *    aakashvshah/MemPhys.
 */
#ifndef MEMPHYS_H_
#define MEMPHYS_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MP_OK = 0,
    MP_NOT_CONVERGED = 1,    /* solver.cpp:317-321 (HYPRE branch throws; Eigen branch only logs) */
    MP_BREAKDOWN = 2,        /* BiCGSTAB rho or omega collapsed to zero */
    MP_NAN_DETECTED = 3,     /* non-finite residual or input */
    MP_SINGULAR_STENCIL = 4, /* zero pivot in a stencil system (duplicate nodes) */
    MP_BAD_ARG = 5,          /* invalid size, flag or pointer */
    MP_CUDA_ERROR = 6,       /* a CUDA runtime call failed */
    MP_NO_DEVICE = 7,        /* no sm_100 device visible */
    MP_TIMEOUT = 8,          /* a bounded device-side wait ran out */
    MP_KNN_FAILED = 9        /* a node has fewer candidates than the stencil size */
} mp_status;

typedef void *mp_stream; /* a cudaStream_t; NULL is the legacy default stream */

/* ---------------------------------------------------------------- runtime */
int mp_last_error(char *buf, size_t len);
int mp_version(void);
int mp_device_info(int *sm_count, int *cc_major, int *cc_minor, size_t *total_mem);
int mp_set_device(int device); /* the calling host thread's current device */
int mp_malloc(void **ptr, size_t bytes);
int mp_free(void *ptr);
int mp_malloc_host(void **ptr, size_t bytes); /* pinned */
int mp_free_host(void *ptr);
int mp_memcpy(void *dst, const void *src, size_t bytes, mp_stream s); /* any direction */
int mp_memset(void *dst, int value, size_t bytes, mp_stream s);
int mp_stream_create(mp_stream *s);
int mp_stream_destroy(mp_stream s);
int mp_stream_sync(mp_stream s);
/* CUDA-event timer on a stream: mp_timer_start / mp_timer_stop -> milliseconds */
int mp_timer_start(mp_stream s, void **timer);
int mp_timer_stop(void *timer, mp_stream s, double *ms);
/* start (on != 0) / stop the profiler's capture range (cudaProfilerStart/Stop) */
int mp_profiler(int on);
/* launches of this library's kernels since the last reset (process-wide counter) */
int mp_launch_count(int64_t *count, int reset);

/* ------------------------------------------------------------- parameters */
/* parameters.cpp:122-130 (PARAMETERS::calc_cloud_num_points) */
int mp_num_poly_terms(int dim, int poly_deg);
int mp_cloud_size(int dim, int poly_deg, double cloud_size_multiplier);
/* parameters.cpp:217-267 (PARAMETERS::calc_polynomial_term_exponents); exps is m x dim */
int mp_poly_exponents(int dim, int poly_deg, int *exps);

/* ---------------------------------------------------------------- stencils */
/*
 * kNN stencils, replacing CLOUD::calc_cloud_points_fast (cloud.cpp:570-648):
 * interior node -> its n nearest nodes (itself first); boundary node ->
 * itself + its n-1 nearest interior nodes.  Ties by node index.
 * xyz: nv x dim; boundary: nv flags; nb_col: nv x n (output).
 */
int mp_knn_stencils(const double *xyz, const uint8_t *boundary, int nv, int dim, int n,
                    int *nb_col, mp_stream s);
/*
 * The same stencils without allocating device memory (no counterpart in the
 * reference, whose kNN runs on the host).  For callers that cannot allocate
 * mid-run: cudaMalloc/cudaFree synchronise the whole device (stalling solves
 * running on other streams) and fail once a run has sized its buffers to fill
 * the GPU.  Device pointers only.  Work arrays live in a fixed 4 MiB scratch
 * array per device, enough for about 140,000 nodes in 2D; larger clouds
 * return MP_BAD_ARG.  The first call on a device looks the scratch up
 * (cudaGetSymbolAddress), so make it before any stream capture.  Calls share
 * the scratch: calls that overlap in time on one device race, so order them
 * on one stream (or with events).  The scratch needs no initial contents;
 * every call clears what it counts in.
 */
int mp_knn_stencils_noalloc(const double *xyz, const uint8_t *boundary, int nv, int dim, int n,
                            int *nb_col, mp_stream s);

/*
 * calc_interp_matrix (coefficient_computations.cpp:456-518): for each of np probe
 * points its n nearest nodes of the cloud (calc_cloud_points_slow for probes,
 * :373-428: no boundary rule; here in ascending distance, ties by index) and the
 * PHS-RBF + polynomial interpolation weights (the stencil's saddle matrix with the
 * basis evaluated at the probe, :430-454, probe scaled with its stencil).
 * Row i of cols / w (np x n) is the sparse row i of the interpolation matrix.
 * n <= 64.  Host or device pointers.
 */
int mp_interp_matrix(const double *xyz, int nv, int dim, const double *probe, int np, int n,
                     int phs_deg, int poly_deg, int *cols, double *w, mp_stream s);
/* the n (1..64) nearest nodes of each probe (np x n, ascending distance, ties by
 * index): the nearest-node lookup of read_restart_tecplot_file
 * (postprocessing_functions.cpp:662-679, a nanoflann 1-NN query there) */
int mp_knn_probe(const double *xyz, int nv, int dim, const double *probe, int np, int n,
                 int *cols, mp_stream s);

/*
 * Node orderings.  order[i] = new index of node i (a permutation of 0..nv-1).
 * mp_order_rcm: CLOUD::re_order_points_reverse_cuthill_mckee (cloud.cpp:315-335)
 *   = reverse_cuthill_mckee_ordering (general_functions.cpp:806-879) on the
 *   stencil graph nb (nv x n), the order CLOUD::CLOUD applies (cloud.cpp:37);
 *   host computation (a breadth-first search), host or device pointers.
 * mp_order_morton: GPU Z-order of the points (no reference counterpart; the
 *   locality of RCM without its sequential search).
 * mp_permute_stencils: CLOUD::re_order_points (cloud.cpp:337-439) on a stencil
 *   table: nb_out row order[i] = row i with every member j replaced by order[j].
 * mp_permute_rows: out row order[i] = in row i, row_bytes bytes per row (points,
 *   normals, flags, weights).  in and out must not alias.
 */
int mp_order_rcm(const int *nb, int nv, int n, int *order);
int mp_order_morton(const double *xyz, int nv, int dim, int *order, mp_stream s);
int mp_permute_stencils(const int *nb, int nv, int n, const int *order, int *nb_out, mp_stream s);
int mp_permute_rows(const void *in, void *out, int nv, int row_bytes, const int *order,
                    mp_stream s);

/*
 * PHS-RBF-FD weights of every stencil of a cloud, replacing the loop of
 * CLOUD::calc_grad_laplace_coeffs (cloud.cpp:207-279) over
 * calc_PHS_RBF_grad_laplace_single_vert (coefficient_computations.cpp:294-328).
 * nb_col: nv x n, row i = stencil of node i with node i first.
 * gx, gy, gz (3D only, else NULL), lap: nv x n weights aligned with nb_col.
 * cond (nullable): 1/rcond of each stencil matrix as Eigen's
 *   PartialPivLU::rcond reports it (coefficient_computations.cpp:312).
 * Returns MP_SINGULAR_STENCIL if any system had a zero pivot.
 */
int mp_stencil_weights(const double *xyz, int nv, int dim, const int *nb_col, int n,
                       int phs_deg, int poly_deg, double *gx, double *gy, double *gz,
                       double *lap, double *cond, mp_stream s);

/*
 * Independent stencil systems of uneven size in one persistent launch
 * (the batched form of coefficient_computations.cpp:294-328, as the moving
 * boundary path fractional_step_fsi.cpp:239-273 re-solves subsets).
 * System i has sizes[i] nodes at pts[offsets[i] .. offsets[i]+sizes[i]) (each
 * dim coordinates, node 0 = centre); its weights go to
 * w[(dim+1)*offsets[i] ...] as (dim+1) rows of sizes[i].  cond nullable.
 * sizes[i] + m must not exceed 96.
 */
int mp_stencil_weights_batched(int nsys, const int *sizes, const int64_t *offsets,
                               const double *pts, int dim, int phs_deg, int poly_deg, double *w,
                               double *cond, mp_stream s);

/*
 * The same batch in two parts (no counterpart in the reference, which solves one
 * stencil at a time): a plan classifies the systems by size once (host work: the
 * sizes and offsets are read back), and each run launches the persistent kernels of
 * the size classes on the caller's stream, asynchronously, device arrays only.  The
 * first run of a plan whose class has at least 8 systems per SM also times the
 * class's CTA shapes on a sample of its systems and keeps the fastest (cached per
 * class and dimension in the process).  mp_stencil_plan_singular synchronises s and
 * returns the number of systems of the last run with a zero pivot;
 * mp_stencil_plan_info fills, for the 7 size classes (n + m + dim + 1 up to 36, 44,
 * 56, 68, 76, 84, 100 with n + m up to 32, 64, 64, 64, 96, 96, 96), the systems of
 * each class and the systems per CTA it runs with (arrays of 7, nullable).
 */
typedef struct mp_stencil_plan_s *mp_stencil_plan;
int mp_stencil_plan_create(int nsys, const int *sizes, const int64_t *offsets, int dim,
                           int poly_deg, mp_stencil_plan *out);
int mp_stencil_plan_run(mp_stencil_plan p, const double *pts, int phs_deg, double *w,
                        double *cond, mp_stream s);
int mp_stencil_plan_singular(mp_stencil_plan p, int *count, mp_stream s);
int mp_stencil_plan_info(mp_stencil_plan p, int *class_count, int *class_shape);
int mp_stencil_plan_destroy(mp_stencil_plan p);

/* ------------------------------------------------------------------ cloud */
typedef struct mp_cloud_s *mp_cloud;

/*
 * CLOUD::CLOUD (cloud.cpp:29-48) without the RCM reordering: GPU kNN
 * stencils + GPU weights, kept resident on the device.
 * cloud_size_multiplier as in parameters_file.csv (n = ceil(mult * m)).
 */
int mp_cloud_create(const double *xyz, const uint8_t *boundary, int nv, int dim, int phs_deg,
                    int poly_deg, double cloud_size_multiplier, int compute_cond, mp_stream s,
                    mp_cloud *out);
/* same with caller-provided stencils (nv x n) */
int mp_cloud_create_stencils(const double *xyz, const uint8_t *boundary, int nv, int dim,
                             const int *nb_col, int n, int phs_deg, int poly_deg,
                             int compute_cond, mp_stream s, mp_cloud *out);
int mp_cloud_info(mp_cloud c, int *nv, int *n, int *dim);
/* copies out CLOUD::nb_points_col / grad_*_coeff / laplacian_coeff / cond_num_RBF
 * (class.hpp:145-151); any pointer may be NULL */
int mp_cloud_get(mp_cloud c, int *nb_col, double *gx, double *gy, double *gz, double *lap,
                 double *cond, mp_stream s);
int mp_cloud_destroy(mp_cloud c);

/* -------------------------------------------------------------- operators */
typedef struct mp_op_s *mp_op;

/* operator precision; for the pressure solve (mp_solver_cfg.precision) also
 * MP_MG32: FP64 BiCGSTAB whose multigrid preconditioner stores its level
 * operators, prolongations and restrictions in FP32 (level operators in the
 * difference form (A u)_i = s_i u_i + sum_j a_ij (u_j - u_i), s_i the exact
 * row sum) and works on FP64 vectors */
enum { MP_FP64 = 0, MP_FP32 = 1, MP_MG32 = 2 };
enum { MP_GRAD_X = 0, MP_GRAD_Y = 1, MP_GRAD_Z = 2, MP_LAPLACIAN = 3 };
enum { MP_ROWS_ALL = 0, MP_ROWS_INTERNAL = 1, MP_ROWS_BOUNDARY = 2 };

/*
 * Fixed-width (ELL) operator with nrows rows of exactly `width` entries,
 * cols/vals row-major nrows x width; stored on the device in 64-row slices.
 * Replaces the Eigen::SparseMatrix<double,RowMajor> operators of POINTS
 * (class.hpp:116-124) for `matrix * vector` products.
 */
int mp_op_create_ell(int nrows, int ncols, int width, const int *cols, const double *vals,
                     int precision, mp_op *out);
/* POINTS::{grad_x,grad_y,grad_z,laplacian}_matrix_EIGEN[_internal|_boundary]
 * (cloud.cpp:89-205): rows outside the mask are zero */
int mp_op_from_cloud(mp_cloud c, int which, int rows, int precision, mp_op *out);
/* y = alpha * A x + beta * y; x, y device (or host, staged) vectors of the op's precision */
int mp_op_apply(mp_op op, const void *x, void *y, double alpha, double beta, mp_stream s);
/* y_k = A_k x for up to 4 operators sharing one column structure (one pass over the indices) */
int mp_op_apply_multi(int nops, const mp_op *ops, const void *x, void *const *ys, mp_stream s);
int mp_op_info(mp_op op, int *nrows, int *ncols, int *width, int *precision);
/*
 * calc_largest_magnitude_eigenvalue (general_functions.cpp:4-24; Spectra
 * GenEigsSolver, LARGEST_MAGN), used by PARAMETERS::calc_dt (parameters.cpp:269-296):
 * the eigenvalue of largest magnitude of a square FP64 operator, by explicitly
 * restarted Arnoldi with ncv vectors (>= 3; 30 is a good default) on the GPU.  It
 * stops once the Ritz residual is <= tol * |lambda| (MP_OK) or after max_restarts
 * cycles (MP_NOT_CONVERGED, with the last estimate written).  Of a complex-conjugate
 * pair the member with positive imaginary part is returned.  The start vector is a
 * fixed function of `seed`.  Allocates (ncv + 2) work vectors; synchronises `s`.
 */
int mp_op_largest_eig(mp_op op, int ncv, double tol, int max_restarts, uint64_t seed,
                      double *re, double *im, int *restarts, mp_stream s);
int mp_op_destroy(mp_op op);

/* --------------------------------------------------------- pressure solve */
typedef struct mp_ppe_s *mp_ppe;

/* MP_PRECOND_SOR is the reference's `sor` solver type (SOLVER::SOR, solver.cpp:243-281):
 * no Krylov method, SOR sweeps with relaxation sor_omega on the unbordered system
 * (solver.cpp:30-31), rows in multicolour order; maxit sweeps at most, stopping once
 * ||b - A x|| / ||b|| <= tol.  FP64 only; accepted by mp_ppe_* (SOLVER), not by the
 * graph-captured integrators. */
enum { MP_PRECOND_NONE = 0, MP_PRECOND_JACOBI = 1, MP_PRECOND_AMG = 2, MP_PRECOND_SOR = 3 };
/* initial guess of each fractional-step pressure solve: the previous pressure
 * (the reference's solveWithGuess(rhs, p_old)), zero, the linear extrapolation
 * 2 p^n - p^(n-1), the projection p^n + sum_j c_j (p^(j+1) - p^j) over the last
 * guess_vectors increments with c minimising the guess's residual (Fischer's projection
 * of successive right-hand sides; the increments' images are the differences of
 * successive right-hand sides, so it costs no extra matrix product), or that
 * projection plus the learned network's predicted correction, weighted to
 * minimise the residual */
enum { MP_GUESS_PREVIOUS = 0, MP_GUESS_ZERO = 1, MP_GUESS_LEARNED = 2, MP_GUESS_EXTRAPOLATE = 3,
       MP_GUESS_PROJECT = 4 };

typedef struct {
    double tol;        /* relative residual ||b - A x|| / ||b||, solver.cpp:154 */
    int maxit;         /* solver.cpp:155 */
    int precond;       /* MP_PRECOND_* */
    int precision;     /* MP_FP64; MP_FP32 = FP32 Krylov + FP64 iterative refinement; MP_MG32 */
    int guess;         /* MP_GUESS_* */
    double inner_tol;  /* mixed precision: relative reduction per refinement sweep */
    int amg_max_levels;
    int amg_coarse_size;  /* levels stop at or below this size; the coarsest is inverted densely */
    int smoother_sweeps;  /* degree-2 Chebyshev applications before and after each coarse correction */
    double cheb_lower;    /* Chebyshev interval [cheb_lower * lambda_max, 1.1 lambda_max] of D^-1 A */
    int guess_vectors;    /* MP_GUESS_PROJECT / MP_GUESS_LEARNED: pressure increments kept, 1-8 (8) */
    double sor_omega;     /* MP_PRECOND_SOR relaxation, (0, 2); 1.4 as class.hpp:212 */
} mp_solver_cfg;

/* sensible defaults for the fields above */
int mp_solver_cfg_default(mp_solver_cfg *cfg);

/*
 * SOLVER::init (solver.cpp:14-79) + calc_coeff_matrix (solver.cpp:165-214)
 * for the operator  unsteady*I + conv*(Gx+Gy[+Gz]) + diff*L  on interior rows,
 * identity on Dirichlet boundary rows and normal.grad on Neumann boundary
 * rows; bordered with the nv+1 regularisation row/column when no boundary
 * node is Dirichlet (solver.cpp:29-38, 205-213).
 */
int mp_ppe_create(mp_cloud c, const uint8_t *boundary, const uint8_t *dirichlet,
                  const double *normal, double unsteady, double conv, double diff,
                  const mp_solver_cfg *cfg, mp_ppe *out);
int mp_ppe_system_size(mp_ppe p);
/*
 * SOLVER::general_solve (solver.cpp:283-363), eigen_ilu_bicgstab branch:
 * x_inout holds the initial guess (field_old) and receives the solution.
 * iters, relres (= ||A x - b|| / ||b|| recomputed in FP64), abs_res nullable.
 * Returns MP_NOT_CONVERGED if relres > tol after maxit.
 */
int mp_ppe_solve(mp_ppe p, const double *rhs, double *x_inout, int *iters, double *relres,
                 double *abs_res, mp_stream s);
int mp_ppe_destroy(mp_ppe p);

/* ------------------------------------------------------- fractional step */
typedef struct mp_fs1_s *mp_fs1;

typedef struct {
    double rho, mu, dt;
    int temporal_order; /* 1 = Euler, 2 = Adams-Bashforth 2 (Euler on the first step) */
} mp_fs1_cfg;

/*
 * FRACTIONAL_STEP_1::FRACTIONAL_STEP_1 (fractional_step_1.cpp:22-50).
 * w_dirichlet is ignored in 2D.  Keeps u, v, [w], p resident on the device.
 */
int mp_fs1_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                  const uint8_t *u_dirichlet, const uint8_t *v_dirichlet,
                  const uint8_t *w_dirichlet, const uint8_t *p_dirichlet,
                  const mp_fs1_cfg *cfg, const mp_solver_cfg *solver, mp_fs1 *out);
int mp_fs1_system_size(mp_fs1 f);
/* resident state: vel = dim arrays of nv; p = system_size entries.  The pressure
 * history behind the extrapolated and learned guesses continues when `it` equals
 * the current step index and restarts from p otherwise. */
int mp_fs1_set_state(mp_fs1 f, const double *const *vel, const double *p, int it, mp_stream s);
int mp_fs1_get_state(mp_fs1 f, double *const *vel, double *p, mp_stream s);
/* advance the resident state nsteps timesteps (one CUDA graph launch per step
 * when use_graph); the step counter continues from set_state's `it` */
int mp_fs1_step(mp_fs1 f, int nsteps, int use_graph, mp_stream s);
/*
 * Drop-in for FRACTIONAL_STEP_1::single_timestep_2d (fractional_step_1.cpp:52-63):
 * vel_old/p_old in, vel_new/p_new out (host or device arrays; p of system_size).
 */
int mp_fs1_single_timestep(mp_fs1 f, double *const *vel_new, double *p_new,
                           const double *const *vel_old, const double *p_old, int it,
                           mp_stream s);
/* per-solve logs of the last step (class.hpp:83-84: rel_res_log, abs_res_log,
 * n_iter_actual, regul_alpha_log) */
int mp_fs1_last_stats(mp_fs1 f, int *iters, double *relres, double *abs_res, double *alpha);
/* the logs of `count` steps starting at step `first`, MP_LOG_FIELDS doubles per
 * step: iterations (mixed: inner sweeps), relative residual, absolute residual,
 * regularisation alpha, relative residual of the initial guess, refinement
 * sweeps (mixed), the weight given to the learned correction (MP_GUESS_LEARNED),
 * and one reserved field; the device keeps the last 4096 steps */
#define MP_LOG_FIELDS 8
int mp_fs1_log(mp_fs1 f, int first, int count, double *out);
/* kernels in one graph step: `fixed` once per step, `per_sweep` per BiCGSTAB
 * sweep, `per_refine` per iterative-refinement sweep (mixed precision) */
int mp_fs1_kernel_counts(mp_fs1 f, int *fixed, int *per_sweep, int *per_refine);
int mp_fs1_destroy(mp_fs1 f);

/* ------------------------------------------- semi-implicit split solver */
/*
 * SEMI_IMPLICIT_SPLIT_SOLVER (semi_implicit_split_solver.cpp, 2D): BDF2 implicit
 * velocity with outer iterations of velocity solve -> pressure correction ->
 * velocity correction until the L1 change of (u, v) is <= iterative_tolerance or
 * n_outer_iter iterations ran (single_timestep_2d :376-421).  vel_solver solves
 * the velocity matrices, which change every outer iteration (MP_PRECOND_JACOBI or
 * MP_PRECOND_NONE, MP_FP64); p_solver the pressure correction (any).
 * precond_freq_it is accepted for the reference's signature: the Jacobi
 * preconditioner is rebuilt at every outer iteration.
 */
typedef struct mp_sis_s *mp_sis;
typedef struct {
    double rho, mu, dt;
    int n_outer_iter;
    double iterative_tolerance;
    int precond_freq_it;
} mp_sis_cfg;
int mp_sis_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                  const uint8_t *u_dir, const uint8_t *v_dir, const uint8_t *p_dir,
                  const mp_sis_cfg *cfg, const mp_solver_cfg *vel_solver,
                  const mp_solver_cfg *p_solver, mp_sis *out);
/* nv + 1 when the pressure is full Neumann (bordered), else nv */
int mp_sis_system_size(mp_sis s, int *nsys);
/* solves launched as CUDA graphs (1, default) or kernel by kernel (0); with graphs
 * the whole outer loop of a step is one graph launch, its stopping test on the device */
int mp_sis_set_graph(mp_sis s, int use_graph);
/* SEMI_IMPLICIT_SPLIT_SOLVER::iterative_tolerance (class.hpp:444, a public member the
 * reference's driver resets before every step, eccentric_couette_flow_batch_ml.cpp:71-73):
 * the L1-change tolerance of the following steps */
int mp_sis_set_tolerance(mp_sis s, double iterative_tolerance);
/* single_timestep_2d (:376-421): vel_old = {u_old, v_old} (nv each), p_old
 * (system size) -> vel_new, p_new; it = timestep index (BDF1 at 0); the solver
 * keeps u_old, v_old of the call for the next BDF2 step.  Host or device
 * pointers.  Returns the outer iterations run and the last L1 / max changes. */
int mp_sis_single_timestep(mp_sis s, const double *const *vel_old, const double *p_old,
                           double *const *vel_new, double *p_new, int it, int *n_outer,
                           double *l1_err, double *max_err, mp_stream stream);
int mp_sis_destroy(mp_sis s);

/*
 * IMPLICIT_SCALAR_TRANSPORT_SOLVER (implicit_scalar_transport_solver.cpp, 2D):
 * unsteady dphi/dt + conv (u . grad) phi + diff L phi with the reference's
 * coefficient convention (interior rows diff L + conv (u_i Gx + v_i Gy) +
 * a1 unsteady I, a1 = 1 at it = 0 else 1.5), boundary rows identity
 * (Dirichlet) or n . G; one solve per step from phi_old (Jacobi or no
 * preconditioner, MP_FP64).  precond_freq_it is accepted for the signature.
 */
typedef struct mp_ist_s *mp_ist;
int mp_ist_create(mp_cloud c, const uint8_t *boundary, const double *normal,
                  const uint8_t *dirichlet, int precond_freq_it, double unsteady_coeff,
                  double conv_coeff, double diff_coeff, const mp_solver_cfg *solver, mp_ist *out);
int mp_ist_set_graph(mp_ist s, int use_graph);
/* single_timestep_2d (:136-174): phi_old, u_new, v_new (nv each) -> phi_new;
 * keeps phi_old for the next BDF2 step.  Host or device pointers. */
int mp_ist_single_timestep(mp_ist s, const double *phi_old, const double *u_new,
                           const double *v_new, double *phi_new, int it, int *iters,
                           double *relres, mp_stream stream);
int mp_ist_destroy(mp_ist s);

/* ---------------------------------------- Fourier-z fractional step */
/*
 * FRACTIONAL_STEP_FOURIER (fractional_step_fourier.cpp): a 2D cloud extruded
 * periodically in z over N = 2 nw + 1 planes of `period`; fields are nv x N,
 * column-major (plane c at offset c * nv), as the reference's Eigen::MatrixXd.
 * The pressure of each z-Fourier mode is solved by `solver` (Helmholtz
 * L - k^2 per mode; the first mode bordered under full-Neumann pressure).
 */
typedef struct mp_fsf_s *mp_fsf;
int mp_fsf_create(mp_cloud c, const uint8_t *boundary, const double *normal, const uint8_t *u_dir,
                  const uint8_t *v_dir, const uint8_t *w_dir, const uint8_t *p_dir, double period,
                  int nw, int temporal_order, double rho, double mu, double dt,
                  const mp_solver_cfg *solver, mp_fsf *out);
int mp_fsf_set_graph(mp_fsf f, int use_graph);
/* Field layout of mp_fsf_single_timestep: 0 (default) column-major nv x N, plane c at
 * offset c * nv, as the reference's Eigen::MatrixXd; 1 node-major (row-major nv x N,
 * plane c of node i at i * N + c, a C-ordered numpy (nv, N) array), transposed on the
 * device on the way in and out. */
int mp_fsf_set_layout(mp_fsf f, int node_major);
/* single_timestep (:250-266): vel_old = {u, v, w}, p_old -> vel_new, p_new (nv x N each);
 * the Fourier coefficients are taken from the old fields at it = 0 and carried by
 * the object afterwards, as the reference does.  Host or device pointers. */
int mp_fsf_single_timestep(mp_fsf f, const double *const *vel_old, const double *p_old,
                           double *const *vel_new, double *p_new, int it, mp_stream stream);
int mp_fsf_destroy(mp_fsf f);

/* ------------------------------------------------------- learned guess */
/*
 * Per-node network predicting the pressure increment of a fractional step
 * (no counterpart in the reference; its Python CNN surrogate
 * NN_functions.py:17-51 is a different model).  64 features -> 128 -> 128 ->
 * 128 (ReLU) -> 1; BF16 weights and activations, FP32 accumulation on the
 * tensor cores (tcgen05); FP32 master weights trained with Adam on the GPU.
 * Feature layout and parameter order: memphys_b200/csrc/mp_mlp.cuh.
 */
typedef struct mp_mlp_s *mp_mlp;

int mp_mlp_create(uint64_t seed, mp_mlp *out);
int mp_mlp_num_params(void);
int mp_mlp_get_params(mp_mlp m, float *theta);
int mp_mlp_set_params(mp_mlp m, const float *theta);
/* y = net(X) for n rows of 64 features (FP32 in, rounded to BF16) */
int mp_mlp_forward(mp_mlp m, const float *X, int n, float *y);
/* mean squared error over n rows and its gradient w.r.t. the parameters */
int mp_mlp_gradient(mp_mlp m, const float *X, const float *t, int n, double *loss, float *grad);
/* Adam, `epochs` passes over n rows in shuffled batches (batch a multiple of 128) */
int mp_mlp_train(mp_mlp m, const float *X, const float *t, int n, int epochs, int batch,
                 double lr, uint64_t seed, double *loss);
/* the polls of every tensor-core completion wait before the kernel gives up with
 * MP_TIMEOUT (default 4194304; 0 gives up at once, a test of that path: the
 * kernel still waits, bounded, for the MMA it already committed before it releases
 * tensor memory, and the handle stays usable) */
int mp_mlp_set_spin_limit(mp_mlp m, long long polls);
int mp_mlp_destroy(mp_mlp m);

/*
 * Attach a network to a fractional step: every step then records, for
 * `sample_nodes` fixed nodes, the features and the solved increment (up to
 * `capacity_steps` steps, oldest overwritten).  mp_fs1_train_mlp trains the
 * network on the recorded samples; mp_fs1_set_guess selects the pressure
 * solve's initial guess (MP_GUESS_*).  The solve always runs to the same
 * tolerance, so a poor prediction costs iterations, never accuracy.
 */
int mp_fs1_attach_mlp(mp_fs1 f, mp_mlp m, int sample_nodes, int capacity_steps, int collect);
int mp_fs1_train_mlp(mp_fs1 f, int epochs, int batch, double lr, uint64_t seed, double *loss);
int mp_fs1_set_guess(mp_fs1 f, int guess);
/* The recorded samples, in ring-slot order: X (n x 64 row-major features, the
 * BF16 values widened to float), t (n targets) and nodes (n sampled node
 * indices); any may be NULL.  cap is the number of rows the outputs hold; *n
 * returns the number of rows recorded (at most cap are written). */
int mp_fs1_samples(mp_fs1 f, float *X, float *t, int *nodes, int cap, int *n);

#ifdef __cplusplus
}
#endif
#endif /* MEMPHYS_H_ */
