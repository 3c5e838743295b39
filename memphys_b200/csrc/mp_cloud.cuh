// mp_cloud.cuh -- the resident CLOUD (stencils + operator weights) shared by
// the operator, pressure-solve and fractional-step handles.
#pragma once
#include "mp_ell.cuh"

struct mp_cloud_s;

namespace mp {

struct CloudView {
    int nv, n, dim;
    const int *cols;       // sliced stencil columns (ELL width n)
    const double *w[4];    // sliced gx, gy, gz (3D), laplacian
    const uint8_t *bflag;  // boundary flags (device)
    const int *nb_rm;      // row-major stencils nv x n (device)
};

CloudView cloud_view(mp_cloud_s *c);
const double *cloud_xyz(mp_cloud_s *c);
const Ell *cloud_operator(mp_cloud_s *c, int which);
std::shared_ptr<Ell> cloud_cols(mp_cloud_s *c);
// copy operator `which` (sliced) into dst, zeroing rows outside the mask
int cloud_masked_copy(mp_cloud_s *c, int which, int rows, double *dst, cudaStream_t s);

}  // namespace mp
