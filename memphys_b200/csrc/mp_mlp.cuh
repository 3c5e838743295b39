// mp_mlp.cuh -- the per-node network that predicts, from a node's stencil
// neighbourhood, how a fractional step's pressure increment departs from linear
// extrapolation (the learned initial guess).
//
//   input  64 features: for the node's first 20 stencil members, the new
//          pressure right-hand side b^{n+1} and the last two pressure
//          increments p^n - p^{n-1}, p^{n-1} - p^{n-2} (60 values, each field
//          divided by its RMS over the cloud); the node's spacing over the mean
//          spacing, its boundary flag, 1, 0
//   layers 64 -> 128 -> 128 -> 128 (ReLU) -> 1, BF16 weights and BF16
//          activations between layers, FP32 accumulation; the last hidden
//          layer stays FP32 for the output dot product
//   output the correction to the linear extrapolation,
//          (p^{n+1} - p^n) - (p^n - p^{n-1}), divided by the RMS over the cloud of
//          the last second difference (p^n - p^{n-1}) - (p^{n-1} - p^{n-2}), so
//          the network's pointwise error scales with the (small) correction,
//          not the increment; the fractional step adds the scaled prediction to
//          2 p^n - p^{n-1} after a coarse-level low-pass filter and with the
//          weight that minimises the guess's residual (mp_fs1.cu)
//
// The three hidden layers run on the 5th-generation tensor cores
// (tcgen05.mma, accumulators in tensor memory); training runs on the GPU with
// hand-written backward kernels and Adam.
#pragma once
#include "mp_common.cuh"

struct mp_mlp_s;

namespace mp {

constexpr int MLP_IN = 64, MLP_H = 128, MLP_TILE = 128, MLP_STENCIL = 20;
// flat FP32 parameter vector: W1[64][128], b1, W2[128][128], b2, W3[128][128], b3, w4[128], b4
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_IN * MLP_H;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_H * MLP_H;
constexpr int MLP_OFF_W4 = MLP_OFF_B3 + MLP_H;
constexpr int MLP_OFF_B4 = MLP_OFF_W4 + MLP_H;
constexpr int MLP_NPARAM = MLP_OFF_B4 + 1;
// packed BF16 weights (transposed, tensor-core operand layout): W1t 128x64, W2t, W3t 128x128
constexpr int MLP_PACK = MLP_H * MLP_IN + 2 * MLP_H * MLP_H;

// Feature sources when the network reads a fractional step's fields directly
struct MlpFields {
    int nv, K;               // nodes, stencil width (sliced ELL)
    const int *cols;         // sliced stencil columns
    const double *b;         // new pressure right-hand side
    const double *pcur;      // p^n
    const double *ph1;       // p^{n-1}
    const double *ph2;       // p^{n-2}
    const float *hloc;       // node spacing / mean spacing
    const uint8_t *bflag;
    const double *norms;     // [0] 1/RMS(b), [1] 1/RMS(p^n - p^{n-1}), [2] 1/RMS(second difference)
};

struct Mlp;
Mlp *mlp_of(::mp_mlp_s *h);
int mlp_create(Mlp **out, uint64_t seed);
void mlp_destroy(Mlp *m);
// The predicted correction RMS(d2p) * net(features_i) for i < nv (tensor cores),
// added to x (which holds the extrapolation 2 p^n - p^{n-1}) or, with corr set,
// written to corr.  Zero while *step < 2 (no second difference yet).
int mlp_predict_fields(Mlp &m, const MlpFields &F, double *x, double *corr, const int *step,
                       cudaStream_t s);
// buffers of the field prediction for nv nodes (allocate before any stream capture)
int mlp_reserve_fields(Mlp &m, int nv);
// row-major BF16 features of the nodes in `idx` and targets
// ((xnew - pcur) - (pcur - ph1)) / RMS(d2p), written to
// slot ((*step - 2) % cap_steps) of a sample ring; skipped while *step < 2
int mlp_collect(const MlpFields &F, const int *idx, int nidx, const double *xnew, uint16_t *X,
                float *t, const int *step, int cap_steps, cudaStream_t s);
int mlp_norms(const MlpFields &F, double *norms, double *partials, unsigned *ticket,
              cudaStream_t s);
// train on n row-major BF16 samples; returns the mean loss of the last epoch
int mlp_train(Mlp &m, const uint16_t *X, const float *t, int n, int epochs, int batch, double lr,
              uint64_t seed, double *loss, cudaStream_t s);

}  // namespace mp
