// mp_amg.cuh -- smoothed-aggregation multigrid preconditioner for the
// pressure-Poisson stencil operator.
//
// The reference has no working multigrid (multigrid.cpp builds per-level
// clouds and an SOR smoother, without transfers or a cycle), so this is a
// new design for the BiCGSTAB preconditioner:
//   setup (host, once per operator): strength of connection |a_ij| >=
//     theta * max_k |a_ik| (symmetrised), greedy aggregation, tentative
//     piecewise-constant prolongator T, smoothed P = (I - w D^-1 A) T with
//     w = 4 / (3 lambda_max(D^-1 A)), R = P^T, Galerkin A_c = R A P, until
//     the coarse size is small; the coarsest operator (singular for pure
//     Neumann problems) is bordered like solver.cpp:205-213 and inverted.
//   apply (GPU, every preconditioner call): V(1,1) cycle with degree-2
//     Chebyshev smoothing on [lambda_max / 12, lambda_max] of D^-1 A; the
//     RBF-FD Laplacian's Jacobi-scaled spectrum reaches ~2.85, where damped
//     Jacobi is unstable or weak.
// All level operators are ELL (64-row slices) padded to the level's widest row.
#pragma once
#include "mp_ell.cuh"

namespace mp {

struct Cfg;

// CSR copy of a multigrid operator for the row-group kernels (G lanes per row)
struct DCsr {
    int n = 0, m = 0;
    dbuf<int> rp, ci;
    dbuf<double> v64;
    dbuf<float> v32;
    dbuf<int2> pk;  // (column, FP32 value bits) pairs, when packed
};

// kernel schedule of one operator, chosen by the setup-time autotuner:
// 0 = sliced ELL (2 rows per lane), 1..4 = CSR with 4, 8, 16, 32 lanes per row,
// 5, 6, 7 = sliced ELL with each slice's entries split over a CTA of 8, 4, 2 warps
constexpr int OP_MODES = 8;
struct OpSched {
    int mode = 0;
    float us[OP_MODES] = {};
};

struct AmgLevel {
    int n = 0;
    Ell A;                   // level operator (level 0 borrows the PPE operator)
    bool borrowed = false;
    EllView<double> A64;
    EllView<float> A32;
    Ell P, R;                // prolongation (n x n_next), restriction (n_next x n)
    DCsr Ac, Pc, Rc;         // CSR copies (A only for levels >= 1)
    OpSched sA, sP, sR;
    dbuf<double> dinv;
    dbuf<float> dinv32;
    double lmax = 2.0;
    // work vectors (b, x, d, r) per precision
    dbuf<double> b, x, d, r;
    dbuf<float> b32, x32, d32, r32;
    // AMG_MG32: the level operator in FP32 difference form, self entry first in
    // every row holding the row sum s_i: (A u)_i = s_i u_i + sum_k a_ik (u_k - u_i).
    // Level 0 shares the PPE operator's columns and stores only values.
    Ell Ad;
    EllView<float> Ad32{};
    dbuf<int2> Adpk;         // Ad as (column, value bits) pairs
    // level 0: Ad with entries k, k + 1 of a lane's two rows side by side (values,
    // 16-bit column deltas, per-slice flags: EllView::qv/qd/qslice)
    dbuf<float4> qv;
    dbuf<short4> qd;
    dbuf<unsigned char> qslice;
    DCsr Acd;
};

// storage of the multigrid hierarchy
enum { AMG_F64 = 0, AMG_F32 = 1, AMG_MG32 = 2 };

struct Amg {
    std::vector<AmgLevel *> L;
    int nc = 0;                       // coarsest size
    dbuf<double> cinv;                // (nc+1)^2 bordered inverse, row-major
    // the coarsest operator annihilates constants and its inverse is bordered; with
    // a single level that inverse is the bordered system's own, applied in full
    dbuf<float> cinv32;
    bool coarse_bordered = false;
    double setup_seconds = 0;
    int store = AMG_F64;
    double cheb_ratio = 12.0;         // Chebyshev smoothing on [lmax / ratio, lmax]
    int sweeps = 1;                   // degree-2 Chebyshev applications per side
    dbuf<int> zero_flag;              // a device 0 used as `done` while autotuning
    ~Amg();
};

int amg_create(Amg **out, const Ell &A0, const Cfg &cfg, int store, cudaStream_t s);
// FP32 difference-form copy of a stencil operator whose rows start with their own
// node: the self slot holds the row sum, as (column, value bits) pairs in pk
int ell_diff32(const Ell &A0, dbuf<float> &v32, dbuf<int2> &pk, cudaStream_t s);
// Low-pass filter of a field through the first coarse level:
//   out = P0 diag(scale1) R0 c,   scale1 = 1 / (R0 1)   (out may alias c)
// (a locally weighted average onto the aggregates, interpolated back by the
// smoothed prolongator: smooth fields pass, node-to-node noise is averaged out).
// work1 and scale1 hold one entry per level-1 node.  No-op for a one-level hierarchy.
int amg_filter_size(const Amg &a);
int amg_filter_setup(const Amg &a, double *scale1, cudaStream_t s);
int amg_filter(const Amg &a, const double *c, double *work1, const double *scale1, double *out,
               cudaStream_t s);
void amg_destroy(Amg *a);

// out = V-cycle(in) on the first n0 entries (the border entry is handled by
// the caller); kernels return immediately while *done is set.  A one-level
// hierarchy of an operator that annihilates constants is the exact inverse of the
// bordered system: it then reads and writes entry n0 (the border) as well, since
// the inverse on the first n0 entries alone maps every vector to zero mean and the
// preconditioned system would lose its border row.  FP64 vectors use
// the FP32 difference-form operators when the hierarchy was built with AMG_MG32.
// head_ready: the caller has already written the level-0 head (see AmgHead) for
// `in`; ignored for a one-level hierarchy.
template <class T>
int amg_apply(const Amg &a, const T *in, T *out, const int *done, cudaStream_t s,
              bool head_ready = false);

// The first step of the finest level's pre-smoother from a zero guess,
// d[i] = dinv[i] * in[i] * inv_theta, which the kernel that writes the
// preconditioner's input can write alongside it (amg_apply with head_ready = true
// then skips that pass).  d == nullptr for a one-level hierarchy (the cycle is
// then a direct solve).
template <class T> struct AmgHead {
    T *d;
    const T *dinv;
    T inv_theta;
};
template <class T> AmgHead<T> amg_head(const Amg &a);

}  // namespace mp
