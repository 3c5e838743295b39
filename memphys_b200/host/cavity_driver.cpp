// cavity_driver.cpp -- a C++ driver in the style of the reference's examples
// (examples/navier_stokes_2D/*.cpp): lid-driven cavity on a jittered cloud,
// stepped through the C++ adapters and the C ABI.
//   usage: cavity_driver <nx> <steps> <dt>
// Prints one line per step (iterations, relative residual) and a final
// summary line "OK max|u|=... max_relres=...".
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>
#include "memphys.hpp"

using namespace memphys;

int main(int argc, char **argv) {
    const int nx = argc > 1 ? std::atoi(argv[1]) : 64;
    const int steps = argc > 2 ? std::atoi(argv[2]) : 10;
    const double dt = argc > 3 ? std::atof(argv[3]) : 1e-4;
    const double h = 1.0 / nx;
    POINTS pts;
    std::mt19937_64 rng(20261203);
    std::uniform_real_distribution<double> jit(-0.2 * h, 0.2 * h);
    for (int j = 0; j < nx; j++)
        for (int i = 0; i < nx; i++) {
            pts.xyz.push_back((i + 0.5) * h + jit(rng));
            pts.xyz.push_back((j + 0.5) * h + jit(rng));
            pts.normal.push_back(0.0);
            pts.normal.push_back(0.0);
            pts.boundary_flag.push_back(0);
        }
    const double side[4][4] = {{0, 0, 0, -1}, {0, 1, 0, 1}, {0, 0, -1, 0}, {1, 0, 1, 0}};
    for (int s = 0; s < 4; s++)
        for (int i = 0; i < nx; i++) {
            const double t = (i + 0.5) * h;
            const bool horiz = s < 2;
            pts.xyz.push_back(horiz ? t : side[s][0]);
            pts.xyz.push_back(horiz ? side[s][1] : t);
            pts.normal.push_back(side[s][2]);
            pts.normal.push_back(side[s][3]);
            pts.boundary_flag.push_back(1);
        }
    pts.nv = (int)pts.boundary_flag.size();
    PARAMETERS prm;
    prm.rho = 1.0;
    prm.mu = 0.01;
    prm.dt = dt;
    prm.solver_tolerance = 1e-8;
    CLOUD cloud(pts, prm, false);
    std::vector<bool> udir(pts.nv), vdir(pts.nv), pdir(pts.nv, false);
    for (int i = 0; i < pts.nv; i++)
        udir[i] = vdir[i] = pts.boundary_flag[i] != 0;
    FRACTIONAL_STEP_1 fs(pts, cloud, prm, udir, vdir, pdir, 2);
    std::vector<double> u_old(pts.nv, 0.0), v_old(pts.nv, 0.0), p_old(fs.system_size, 0.0);
    for (int i = 0; i < nx; i++)
        u_old[nx * nx + nx + i] = 1.0;  // lid: the y = 1 side
    std::vector<double> u_new, v_new, p_new;
    double max_rel = 0;
    for (int it = 0; it < steps; it++) {
        fs.single_timestep_2d(pts, cloud, prm, u_new, v_new, p_new, u_old, v_old, p_old, it);
        std::printf("step %d iters %d relres %.3e\n", it, prm.n_iter_actual.back(),
                    prm.rel_res_log.back());
        max_rel = std::fmax(max_rel, prm.rel_res_log.back());
        u_old.swap(u_new);
        v_old.swap(v_new);
        p_old.swap(p_new);
    }
    double umax = 0;
    for (double u : u_old)
        umax = std::fmax(umax, std::fabs(u));
    // the divergence-free correction keeps the lid velocity as the maximum
    OPERATOR gx(cloud, MP_GRAD_X, MP_ROWS_INTERNAL);
    std::vector<double> dudx = gx * u_old;
    std::printf("OK max|u|=%.6f max_relres=%.3e grad_x_rows=%zu\n", umax, max_rel, dudx.size());
    return max_rel <= 1e-8 ? 0 : 2;
}
