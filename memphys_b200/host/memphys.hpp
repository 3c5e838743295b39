// memphys.hpp -- C++ host adapters over the C ABI of libmemphys_cuda.so.
//
// Class names, member names and argument order follow the reference's
// header_files/class.hpp (PARAMETERS :58-94, POINTS :96-140, CLOUD :142-169,
// SOLVER :171-217, FRACTIONAL_STEP_1 :246-270, FRACTIONAL_STEP_FOURIER :272-335,
// IMPLICIT_SCALAR_TRANSPORT_SOLVER :395-415, SEMI_IMPLICIT_SPLIT_SOLVER :417-455),
// with std::vector<double> in
// place of Eigen::VectorXd.  Every non-OK status is printed with
// mp_last_error() and turned into `throw std::bad_exception()`, the
// reference's error convention (e.g. solver.cpp:317-321).
#pragma once
#include <cmath>
#include <cstdio>
#include <exception>
#include <string>
#include <vector>

#include "../../include/memphys.h"

namespace memphys {

inline void check(int rc, const char *where) {
    if (rc != MP_OK) {
        char msg[1024];
        mp_last_error(msg, sizeof msg);
        std::printf("\n\nERROR from %s: %s (status %d)\n\n", where, msg, rc);
        throw std::bad_exception();
    }
}

struct PARAMETERS {
    int dimension = 2, poly_deg = 3, phs_deg = 3, num_poly_terms = 0, cloud_size = 0, n_iter = 1000;
    double cloud_size_multiplier = 2.0, solver_tolerance = 1e-8, dt = 0.0, rho = -10.0, mu = -10.0;
    std::string solver_type = "cuda_bicgstab_amg";
    std::vector<double> rel_res_log, abs_res_log, regul_alpha_log;
    std::vector<int> n_iter_actual;
    std::vector<int> polynomial_term_exponents;  // num_poly_terms x dimension

    PARAMETERS() { calc(); }
    void calc() {  // parameters.cpp:122-130, 217-267
        num_poly_terms = mp_num_poly_terms(dimension, poly_deg);
        cloud_size = mp_cloud_size(dimension, poly_deg, cloud_size_multiplier);
        polynomial_term_exponents.assign((size_t)num_poly_terms * dimension, 0);
        check(mp_poly_exponents(dimension, poly_deg, polynomial_term_exponents.data()),
              "PARAMETERS::calc_polynomial_term_exponents");
    }
    mp_solver_cfg solver_cfg() const {
        mp_solver_cfg c;
        mp_solver_cfg_default(&c);
        c.tol = solver_tolerance;
        c.maxit = n_iter;
        // solver_type strings as PARAMETERS::verify_parameters accepts them
        // (parameters.cpp:94-99), plus the GPU configurations by name
        if (solver_type == "cuda_bicgstab_amg_mixed")
            c.precision = MP_FP32;
        else if (solver_type == "cuda_bicgstab_amg_mg32")
            c.precision = MP_MG32;
        else if (solver_type == "cuda_bicgstab_jacobi")
            c.precond = MP_PRECOND_JACOBI;
        else if (solver_type == "cuda_bicgstab_jacobi_mixed") {
            c.precond = MP_PRECOND_JACOBI;
            c.precision = MP_FP32;
        } else if (solver_type == "cuda_bicgstab")
            c.precond = MP_PRECOND_NONE;
        else if (solver_type == "sor")
            c.precond = MP_PRECOND_SOR;
        return c;
    }
    // a time integrator's solver: the SOR sweeps run through SOLVER only, so `sor`
    // gives the integrators BiCGSTAB + multigrid to the same tolerance
    mp_solver_cfg integrator_cfg() const {
        mp_solver_cfg c = solver_cfg();
        if (c.precond == MP_PRECOND_SOR) {
            std::printf("PARAMETERS: solver_type sor -> the time integrator's pressure solve runs "
                        "BiCGSTAB + multigrid (SOR sweeps are available through SOLVER)\n");
            c.precond = MP_PRECOND_AMG;
        }
        return c;
    }
};

struct POINTS {
    int nv = 0;
    std::vector<double> xyz;              // nv x dim
    std::vector<double> normal;           // nv x dim
    std::vector<unsigned char> boundary_flag;
};

class CLOUD {
  public:
    std::vector<int> nb_points_row, nb_points_col;
    std::vector<double> grad_x_coeff, grad_y_coeff, grad_z_coeff, laplacian_coeff, cond_num_RBF;
    double cond_num_RBF_max = 0, cond_num_RBF_min = 0, cond_num_RBF_avg = 0;
    mp_cloud handle = nullptr;

    CLOUD(POINTS &points, PARAMETERS &parameters, bool compute_cond = true) {
        check(mp_cloud_create(points.xyz.data(), points.boundary_flag.data(), points.nv,
                              parameters.dimension, parameters.phs_deg, parameters.poly_deg,
                              parameters.cloud_size_multiplier, compute_cond ? 1 : 0, nullptr,
                              &handle),
              "CLOUD::CLOUD");
        int nv, n, dim;
        check(mp_cloud_info(handle, &nv, &n, &dim), "CLOUD::CLOUD");
        const size_t m = (size_t)nv * n;
        nb_points_col.resize(m);
        grad_x_coeff.resize(m);
        grad_y_coeff.resize(m);
        laplacian_coeff.resize(m);
        if (dim == 3)
            grad_z_coeff.resize(m);
        if (compute_cond)
            cond_num_RBF.resize(nv);
        check(mp_cloud_get(handle, nb_points_col.data(), grad_x_coeff.data(), grad_y_coeff.data(),
                           dim == 3 ? grad_z_coeff.data() : nullptr, laplacian_coeff.data(),
                           compute_cond ? cond_num_RBF.data() : nullptr, nullptr),
              "CLOUD::CLOUD");
        nb_points_row.resize(nv + 1);
        for (int i = 0; i <= nv; i++)
            nb_points_row[i] = i * n;
        if (compute_cond && nv > 0) {  // cloud.cpp:273-275
            cond_num_RBF_max = cond_num_RBF_min = cond_num_RBF[0];
            double s = 0;
            for (double c : cond_num_RBF) {
                cond_num_RBF_max = std::fmax(cond_num_RBF_max, c);
                cond_num_RBF_min = std::fmin(cond_num_RBF_min, c);
                s += c;
            }
            cond_num_RBF_avg = s / nv;
        }
    }
    CLOUD(const CLOUD &) = delete;
    CLOUD &operator=(const CLOUD &) = delete;
    ~CLOUD() { mp_cloud_destroy(handle); }
};

// An operator of POINTS (grad_x_matrix_EIGEN etc.), applied like `matrix * vector`
class OPERATOR {
  public:
    mp_op handle = nullptr;
    int nrows = 0;
    OPERATOR(CLOUD &cloud, int which, int rows = MP_ROWS_ALL) {
        check(mp_op_from_cloud(cloud.handle, which, rows, MP_FP64, &handle), "OPERATOR");
        check(mp_op_info(handle, &nrows, nullptr, nullptr, nullptr), "OPERATOR");
    }
    OPERATOR(const OPERATOR &) = delete;
    OPERATOR &operator=(const OPERATOR &) = delete;
    ~OPERATOR() { mp_op_destroy(handle); }
    std::vector<double> operator*(const std::vector<double> &x) const {
        std::vector<double> y(nrows);
        check(mp_op_apply(handle, x.data(), y.data(), 1.0, 0.0, nullptr), "OPERATOR::operator*");
        return y;
    }
};

class SOLVER {
  public:
    mp_ppe handle = nullptr;
    int system_size = 0;
    bool log_flag_1 = true;
    std::vector<unsigned char> dirichlet_flag_1;

    void init(POINTS &points, CLOUD &cloud, PARAMETERS &parameters,
              std::vector<bool> &dirichlet_flag, double unsteady_term_coeff,
              double conv_term_coeff, double diff_term_coeff, bool log_flag) {
        log_flag_1 = log_flag;
        dirichlet_flag_1.assign(dirichlet_flag.begin(), dirichlet_flag.end());
        mp_solver_cfg cfg = parameters.solver_cfg();
        check(mp_ppe_create(cloud.handle, points.boundary_flag.data(), dirichlet_flag_1.data(),
                            points.normal.data(), unsteady_term_coeff, conv_term_coeff,
                            diff_term_coeff, &cfg, &handle),
              "SOLVER::init");
        system_size = mp_ppe_system_size(handle);
    }
    ~SOLVER() { mp_ppe_destroy(handle); }

    // solver.cpp:283-363
    void general_solve(POINTS &points, PARAMETERS &parameters, std::vector<double> &field_new,
                       std::vector<double> &field_old, std::vector<double> &rhs) {
        field_new = field_old;
        int iters = 0;
        double rel = 0, abs_ = 0;
        int rc = mp_ppe_solve(handle, rhs.data(), field_new.data(), &iters, &rel, &abs_, nullptr);
        if (log_flag_1) {
            parameters.rel_res_log.push_back(rel);
            parameters.abs_res_log.push_back(abs_);
            parameters.n_iter_actual.push_back(iters);
            if (system_size == points.nv + 1)
                parameters.regul_alpha_log.push_back(field_new[system_size - 1]);
        }
        if (system_size == points.nv + 1)  // :361-362
            field_old[system_size - 1] = field_new[system_size - 1];
        check(rc, "SOLVER::general_solve");
    }
};

class FRACTIONAL_STEP_1 {
  public:
    mp_fs1 handle = nullptr;
    int system_size = 0;
    std::vector<unsigned char> u_d, v_d, p_d;

    FRACTIONAL_STEP_1(POINTS &points, CLOUD &cloud, PARAMETERS &parameters,
                      std::vector<bool> &u_dirichlet_flag1, std::vector<bool> &v_dirichlet_flag1,
                      std::vector<bool> &p_dirichlet_flag1, int temporal_order1) {
        u_d.assign(u_dirichlet_flag1.begin(), u_dirichlet_flag1.end());
        v_d.assign(v_dirichlet_flag1.begin(), v_dirichlet_flag1.end());
        p_d.assign(p_dirichlet_flag1.begin(), p_dirichlet_flag1.end());
        mp_fs1_cfg cfg{parameters.rho, parameters.mu, parameters.dt, temporal_order1};
        mp_solver_cfg scfg = parameters.integrator_cfg();
        check(mp_fs1_create(cloud.handle, points.boundary_flag.data(), points.normal.data(),
                            u_d.data(), v_d.data(), nullptr, p_d.data(), &cfg, &scfg, &handle),
              "FRACTIONAL_STEP_1::FRACTIONAL_STEP_1");
        system_size = mp_fs1_system_size(handle);
    }
    FRACTIONAL_STEP_1(const FRACTIONAL_STEP_1 &) = delete;
    FRACTIONAL_STEP_1 &operator=(const FRACTIONAL_STEP_1 &) = delete;
    ~FRACTIONAL_STEP_1() { mp_fs1_destroy(handle); }

    // fractional_step_1.cpp:52-63
    void single_timestep_2d(POINTS &points, CLOUD &, PARAMETERS &parameters,
                            std::vector<double> &u_new, std::vector<double> &v_new,
                            std::vector<double> &p_new, std::vector<double> &u_old,
                            std::vector<double> &v_old, std::vector<double> &p_old, int it1) {
        if ((int)p_new.size() != system_size)
            p_new.assign(system_size, 0.0);
        if ((int)p_old.size() != system_size)
            p_old.assign(system_size, 0.0);
        u_new.resize(points.nv);
        v_new.resize(points.nv);
        double *vn[2] = {u_new.data(), v_new.data()};
        const double *vo[2] = {u_old.data(), v_old.data()};
        int rc = mp_fs1_single_timestep(handle, vn, p_new.data(), vo, p_old.data(), it1, nullptr);
        int iters = 0;
        double rel = 0, abs_ = 0, alpha = 0;
        if (mp_fs1_last_stats(handle, &iters, &rel, &abs_, &alpha) == MP_OK) {
            parameters.rel_res_log.push_back(rel);
            parameters.abs_res_log.push_back(abs_);
            parameters.n_iter_actual.push_back(iters);
            if (system_size == points.nv + 1) {
                parameters.regul_alpha_log.push_back(alpha);
                p_old[system_size - 1] = p_new[system_size - 1];
            }
        }
        check(rc, "FRACTIONAL_STEP_1::single_timestep_2d");
    }
};

// implicit_scalar_transport_solver.cpp / class.hpp:395-415 (2D)
class IMPLICIT_SCALAR_TRANSPORT_SOLVER {
  public:
    mp_ist handle = nullptr;
    bool solver_log_flag = false;
    std::vector<unsigned char> d;

    IMPLICIT_SCALAR_TRANSPORT_SOLVER(POINTS &points, CLOUD &cloud, PARAMETERS &parameters,
                                     std::vector<bool> &dirichlet_flag1, int precond_freq_it1,
                                     double unsteady_coeff1, double conv_coeff1, double diff_coeff1,
                                     bool solver_log_flag1)
        : solver_log_flag(solver_log_flag1) {
        d.assign(dirichlet_flag1.begin(), dirichlet_flag1.end());
        mp_solver_cfg c = parameters.integrator_cfg();
        c.precond = MP_PRECOND_JACOBI;  // the matrix changes every step
        c.precision = MP_FP64;
        check(mp_ist_create(cloud.handle, points.boundary_flag.data(), points.normal.data(), d.data(),
                            precond_freq_it1, unsteady_coeff1, conv_coeff1, diff_coeff1, &c, &handle),
              "IMPLICIT_SCALAR_TRANSPORT_SOLVER::IMPLICIT_SCALAR_TRANSPORT_SOLVER");
    }
    IMPLICIT_SCALAR_TRANSPORT_SOLVER(const IMPLICIT_SCALAR_TRANSPORT_SOLVER &) = delete;
    IMPLICIT_SCALAR_TRANSPORT_SOLVER &operator=(const IMPLICIT_SCALAR_TRANSPORT_SOLVER &) = delete;
    ~IMPLICIT_SCALAR_TRANSPORT_SOLVER() { mp_ist_destroy(handle); }

    // :136-174; with solver_log_flag the residual and iterations are logged in parameters
    void single_timestep_2d(POINTS &points, CLOUD &, PARAMETERS &parameters,
                            std::vector<double> &phi_new, std::vector<double> &phi_old,
                            std::vector<double> &u_new, std::vector<double> &v_new, int it1) {
        phi_new.resize(points.nv);
        int iters = 0;
        double rel = 0;
        check(mp_ist_single_timestep(handle, phi_old.data(), u_new.data(), v_new.data(),
                                     phi_new.data(), it1, &iters, &rel, nullptr),
              "IMPLICIT_SCALAR_TRANSPORT_SOLVER::single_timestep_2d");
        if (solver_log_flag) {
            parameters.rel_res_log.push_back(rel);
            parameters.n_iter_actual.push_back(iters);
        }
    }
};

// semi_implicit_split_solver.cpp / class.hpp:417-455 (2D)
class SEMI_IMPLICIT_SPLIT_SOLVER {
  public:
    mp_sis handle = nullptr;
    int system_size = 0;
    // public as in the reference (class.hpp): its driver resets it before every step
    double iterative_tolerance = 0;
    std::vector<unsigned char> u_d, v_d, p_d;

    SEMI_IMPLICIT_SPLIT_SOLVER(POINTS &points, CLOUD &cloud, PARAMETERS &parameters,
                               std::vector<bool> &u_dirichlet_flag1,
                               std::vector<bool> &v_dirichlet_flag1,
                               std::vector<bool> &p_dirichlet_flag1, int n_outer_iter1,
                               double iterative_tolerance1, int precond_freq_it1) {
        u_d.assign(u_dirichlet_flag1.begin(), u_dirichlet_flag1.end());
        v_d.assign(v_dirichlet_flag1.begin(), v_dirichlet_flag1.end());
        p_d.assign(p_dirichlet_flag1.begin(), p_dirichlet_flag1.end());
        iterative_tolerance = iterative_tolerance1;
        mp_sis_cfg cfg{parameters.rho, parameters.mu, parameters.dt, n_outer_iter1,
                       iterative_tolerance1, precond_freq_it1};
        mp_solver_cfg vel = parameters.integrator_cfg(), pres = parameters.integrator_cfg();
        vel.precond = MP_PRECOND_JACOBI;  // the velocity matrices change every outer iteration
        vel.precision = MP_FP64;
        check(mp_sis_create(cloud.handle, points.boundary_flag.data(), points.normal.data(),
                            u_d.data(), v_d.data(), p_d.data(), &cfg, &vel, &pres, &handle),
              "SEMI_IMPLICIT_SPLIT_SOLVER::SEMI_IMPLICIT_SPLIT_SOLVER");
        check(mp_sis_system_size(handle, &system_size), "SEMI_IMPLICIT_SPLIT_SOLVER");
    }
    SEMI_IMPLICIT_SPLIT_SOLVER(const SEMI_IMPLICIT_SPLIT_SOLVER &) = delete;
    SEMI_IMPLICIT_SPLIT_SOLVER &operator=(const SEMI_IMPLICIT_SPLIT_SOLVER &) = delete;
    ~SEMI_IMPLICIT_SPLIT_SOLVER() { mp_sis_destroy(handle); }

    // :376-421
    void single_timestep_2d(POINTS &points, CLOUD &, PARAMETERS &, std::vector<double> &u_new,
                            std::vector<double> &v_new, std::vector<double> &p_new,
                            std::vector<double> &u_old, std::vector<double> &v_old,
                            std::vector<double> &p_old, int it1,
                            std::vector<int> &n_outer_iter_log,
                            std::vector<double> &iterative_l1_err_log,
                            std::vector<double> &iterative_max_err_log) {
        if ((int)p_new.size() != system_size)  // :380-383
            p_new.assign(system_size, 0.0);
        if ((int)p_old.size() != system_size)
            p_old.assign(system_size, 0.0);
        u_new.resize(points.nv);
        v_new.resize(points.nv);
        const double *vo[2] = {u_old.data(), v_old.data()};
        double *vn[2] = {u_new.data(), v_new.data()};
        int n = 0;
        double l1 = 0, mx = 0;
        check(mp_sis_set_tolerance(handle, iterative_tolerance),
              "SEMI_IMPLICIT_SPLIT_SOLVER::iterative_tolerance");
        check(mp_sis_single_timestep(handle, vo, p_old.data(), vn, p_new.data(), it1, &n, &l1, &mx,
                                     nullptr),
              "SEMI_IMPLICIT_SPLIT_SOLVER::single_timestep_2d");
        n_outer_iter_log.push_back(n);
        iterative_l1_err_log.push_back(l1);
        iterative_max_err_log.push_back(mx);
    }
};

// fractional_step_fourier.cpp / class.hpp:272-335 (2D cloud, Fourier in z); each
// field is nv x (2 nw + 1), column-major like the reference's Eigen::MatrixXd
class FRACTIONAL_STEP_FOURIER {
  public:
    mp_fsf handle = nullptr;
    int nv = 0, nplanes = 0;
    std::vector<unsigned char> u_d, v_d, w_d, p_d;

    FRACTIONAL_STEP_FOURIER(POINTS &points, CLOUD &cloud, PARAMETERS &parameters,
                            std::vector<bool> &u_dirichlet_flag1,
                            std::vector<bool> &v_dirichlet_flag1,
                            std::vector<bool> &w_dirichlet_flag1,
                            std::vector<bool> &p_dirichlet_flag1, double period1, int nw1,
                            int temporal_order1)
        : nv(points.nv), nplanes(2 * nw1 + 1) {
        u_d.assign(u_dirichlet_flag1.begin(), u_dirichlet_flag1.end());
        v_d.assign(v_dirichlet_flag1.begin(), v_dirichlet_flag1.end());
        w_d.assign(w_dirichlet_flag1.begin(), w_dirichlet_flag1.end());
        p_d.assign(p_dirichlet_flag1.begin(), p_dirichlet_flag1.end());
        mp_solver_cfg c = parameters.integrator_cfg();
        check(mp_fsf_create(cloud.handle, points.boundary_flag.data(), points.normal.data(),
                            u_d.data(), v_d.data(), w_d.data(), p_d.data(), period1, nw1,
                            temporal_order1, parameters.rho, parameters.mu, parameters.dt, &c,
                            &handle),
              "FRACTIONAL_STEP_FOURIER::FRACTIONAL_STEP_FOURIER");
    }
    FRACTIONAL_STEP_FOURIER(const FRACTIONAL_STEP_FOURIER &) = delete;
    FRACTIONAL_STEP_FOURIER &operator=(const FRACTIONAL_STEP_FOURIER &) = delete;
    ~FRACTIONAL_STEP_FOURIER() { mp_fsf_destroy(handle); }

    // :250-266
    void single_timestep(POINTS &, CLOUD &, PARAMETERS &, std::vector<double> &u_new,
                         std::vector<double> &v_new, std::vector<double> &w_new,
                         std::vector<double> &p_new, std::vector<double> &u_old,
                         std::vector<double> &v_old, std::vector<double> &w_old,
                         std::vector<double> &p_old, int it1) {
        const size_t m = (size_t)nv * nplanes;
        for (std::vector<double> *a : {&u_new, &v_new, &w_new, &p_new})
            a->resize(m);
        const double *vo[3] = {u_old.data(), v_old.data(), w_old.data()};
        double *vn[3] = {u_new.data(), v_new.data(), w_new.data()};
        check(mp_fsf_single_timestep(handle, vo, p_old.data(), vn, p_new.data(), it1, nullptr),
              "FRACTIONAL_STEP_FOURIER::single_timestep");
    }
};

// calc_interp_matrix (coefficient_computations.cpp:456-518): the rows of the
// interpolation matrix, row i = probe i, cloud_size entries each
struct INTERP_MATRIX {
    int rows = 0, width = 0;
    std::vector<int> cols;
    std::vector<double> vals;
};

inline INTERP_MATRIX calc_interp_matrix(std::vector<double> &xyz_probe, POINTS &points,
                                        PARAMETERS &parameters) {
    INTERP_MATRIX m;
    m.rows = (int)(xyz_probe.size() / parameters.dimension);
    m.width = parameters.cloud_size;
    m.cols.resize((size_t)m.rows * m.width);
    m.vals.resize((size_t)m.rows * m.width);
    check(mp_interp_matrix(points.xyz.data(), points.nv, parameters.dimension, xyz_probe.data(),
                           m.rows, m.width, parameters.phs_deg, parameters.poly_deg, m.cols.data(),
                           m.vals.data(), nullptr),
          "calc_interp_matrix");
    return m;
}

}  // namespace memphys
