// mp_mlp.cu -- the learned pressure-increment network on sm_100a.
//
// Forward: one CTA (128 threads) owns a tile of 128 nodes.  The BF16 weights
// (transposed) and the tile's features sit in shared memory in the canonical
// K-major, non-swizzled core-matrix layout (8 rows x 16 bytes per core
// matrix; the two 8-element halves of a 16-wide K step 128 bytes apart, the
// 8-row groups K*16 bytes apart).  One elected thread issues
// tcgen05.mma.cta_group::1.kind::f16 (M = N = 128, K = 16 per instruction)
// into a 128-column FP32 accumulator in tensor memory and commits to an
// mbarrier; every thread then reads its own row back with tcgen05.ld
// (thread 32w + l owns TMEM lane 32w + l), applies bias + ReLU and writes the
// BF16 activations back to shared memory as the next layer's A operand.  The
// output layer is a per-thread dot product on the FP32 activations.
//
// Backward (training) on the tensor cores as well: the input gradients
// D_prev = (D W^T) * relu'(H_prev) per 128-row tile, and the weight gradients
// dW = A^T D as a product over the batch split into 64-row chunks across CTAs
// (each CTA accumulates its chunks in tensor memory; a second kernel sums the CTAs'
// partial products in a fixed order).  The FP32 gradients D enter the BF16 MMA as
// two parts, D = hi + lo with hi = bf16(D) and lo = bf16(D - hi) (16 significant
// bits), against operands that are exactly BF16 (the weights and activations the
// forward used), so the products carry FP32-level accuracy.  Adam updates FP32
// master weights, then the BF16 operand copies are repacked.
//
// Every mbarrier wait is bounded (the limit is a kernel argument).  A warpgroup
// whose wait runs out stops issuing MMAs and skips its epilogues, waits once more
// (bounded) for the MMA it already committed, and only then releases tensor memory;
// the host sees MP_TIMEOUT.
#include <cuda_bf16.h>
#include <algorithm>
#include <cmath>
#include <random>
#include "mp_mlp.cuh"

namespace mp {

struct Mlp {
    dbuf<float> theta, m1, m2, grad;
    dbuf<uint16_t> pack;  // W1t | W2t | W3t in core-matrix layout
    dbuf<uint16_t> packn; // W2 | W3 untransposed in core-matrix layout (backward operands)
    dbuf<float> wpart;    // weight-gradient partial products of the split batch
    long long spin = 1ll << 22;  // mbarrier wait limit (polls)
    int adam_t = 0;
    // training scratch (sized for the largest batch seen)
    int cap = 0;
    dbuf<uint16_t> h1, h2;
    dbuf<float> h3, y, d3, d2, d1, lossbuf;
    dbuf<int> idx;
    dbuf<int> err;  // device flag: an mbarrier wait ran out
    // per-node features and outputs of the field prediction (sized to the cloud)
    dbuf<uint16_t> fx;
    dbuf<float> fy;
    dbuf<float4> fq;  // per node: the three scaled fields the features gather
};

// ------------------------------------------------------------ layout helpers
__host__ __device__ __forceinline__ int cm_off(int r, int k, int K) {
    return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no swizzle: LBO = 128 B (next K half), SBO = K*16 B (next 8 rows)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, int K) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(((uint32_t)K * 16u) >> 4) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for sm_100
    return d;
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both
// K-major, N = 128 (>> 3), M = 128 (>> 4)
constexpr uint32_t MLP_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) |
                               ((128u >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db,
                                          uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
            tmem_d),
        "l"(da), "l"(db), "r"(MLP_IDESC), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void umma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
        smem_u32(mbar)));
}

// after a wait ran out: the bound of the one further wait for the MMA already committed
constexpr long long MLP_SPIN_DRAIN = 1ll << 24;

__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(mbar);
    for (long long i = 0; i < limit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(a), "r"(parity));
        if (ok)
            return true;
    }
    return false;
}

// 32 consecutive accumulator columns of this thread's row; one wait per 32
// columns keeps the tensor-memory latency off the epilogue's critical path
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++)
        v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ __forceinline__ float bf16_round(float a) {
    return __bfloat162float(__float2bfloat16_rn(a));
}

// ---------------------------------------------------------- forward kernel
enum { MLP_MODE_ROWS = 1, MLP_MODE_TRAIN = 2 };  // (template argument: k_mlp_forward<1> is the row forward)

struct MlpFwdArgs {
    int n;                   // rows
    const uint16_t *pack;    // packed BF16 weights
    const float *theta;      // biases and output weights
    // rows mode: row-major BF16 features, optional index list
    const uint16_t *X;
    const int *idx;
    float *y;                // output (rows/train)
    // train mode: stored activations
    uint16_t *h1, *h2;
    float *h3;
    int *err;
    long long spin;          // mbarrier wait limit (polls)
};

// Four warpgroups per CTA work on four tiles at once, each with its own operand
// staging buffer, mbarrier and 128 accumulator columns of tensor memory (all
// 512 columns): while some groups run their epilogues (TMEM -> registers ->
// BF16 in shared memory) the tensor core runs the others' MMAs.  The weights
// are shared.  A group's buffer holds its feature tile (K = 64) for layer 1,
// then each hidden activation (K = 128) once the MMA that read it completed.
constexpr int MLP_WG = 4;

struct MlpSmem {
    uint16_t w1[MLP_H * MLP_IN];
    uint16_t w2[MLP_H * MLP_H];
    uint16_t w3[MLP_H * MLP_H];
    uint16_t buf[MLP_WG][MLP_TILE * MLP_H];
    float bias[3][MLP_H];
    float w4[MLP_H];
    uint64_t mbar[MLP_WG];
    uint32_t tmem;
};

// barrier of one warpgroup (named barrier 1 + wg; 0 is __syncthreads)
__device__ __forceinline__ void wg_sync(int wg) {
    asm volatile("bar.sync %0, 128;\n" ::"r"(1 + wg) : "memory");
}

// the same barrier, returning whether v holds in all 128 threads of the group
__device__ __forceinline__ bool wg_all(int wg, bool v) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.b32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, 128, p;\n\t"
        "selp.b32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((int)v), "r"(1 + wg)
        : "memory");
    return r != 0;
}

template <int MODE>
__global__ void __launch_bounds__(128 * MLP_WG, 1) k_mlp_forward(MlpFwdArgs A) {
    extern __shared__ __align__(1024) unsigned char mlp_smem_raw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(mlp_smem_raw);
    const int warp = threadIdx.x >> 5, wg = threadIdx.x >> 7, tid = threadIdx.x & 127;
    // weights (already in operand layout) and vectors into shared memory
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(A.pack);
        uint4 *dst = reinterpret_cast<uint4 *>(S.w1);  // w1, w2, w3 are contiguous
        for (int i = threadIdx.x; i < MLP_PACK / 8; i += blockDim.x)
            dst[i] = src[i];
        for (int i = threadIdx.x; i < MLP_H; i += blockDim.x) {
            S.bias[0][i] = A.theta[MLP_OFF_B1 + i];
            S.bias[1][i] = A.theta[MLP_OFF_B2 + i];
            S.bias[2][i] = A.theta[MLP_OFF_B3 + i];
            S.w4[i] = A.theta[MLP_OFF_W4 + i];
        }
    }
    if (threadIdx.x == 0)
        for (int g = 0; g < MLP_WG; g++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&S.mbar[g])));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&S.tmem)),
                     "r"(MLP_H * MLP_WG));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    // this group's accumulator columns; warp w reads TMEM lanes 32 (w % 4) ..
    const uint32_t tmem = S.tmem + (uint32_t)(wg * MLP_H);
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    uint16_t *xa = S.buf[wg], *ha = S.buf[wg];
    uint64_t *mbar = &S.mbar[wg];
    const float b4 = A.theta[MLP_OFF_B4];
    uint32_t phase = 0;
    bool ok = true;
    const int ntiles = (A.n + MLP_TILE - 1) / MLP_TILE;
    // tiles interleaved over the CTAs (tile = wg * grid + cta): a batch of fewer tiles
    // than SMs gets one CTA per tile instead of sharing a few SMs' tensor cores
    const int stride = gridDim.x * MLP_WG;
    const int first = wg * gridDim.x + blockIdx.x;
    // this thread's 128-byte feature row of tile t (zeros past the end)
    auto load_row = [&](int t, uint4 (&f)[MLP_IN / 8]) {
        const int r = t * MLP_TILE + tid;
        const bool lv = t < ntiles && r < A.n;
        const int src = lv ? (A.idx ? A.idx[r] : r) : 0;
        const uint4 *xr = reinterpret_cast<const uint4 *>(A.X + (size_t)src * MLP_IN);
#pragma unroll
        for (int c = 0; c < MLP_IN / 8; c++)
            f[c] = lv ? xr[c] : make_uint4(0, 0, 0, 0);
    };
    uint4 feat[MLP_IN / 8];
    load_row(first, feat);
    for (int tile = first; tile < ntiles; tile += stride) {
        const int row = tile * MLP_TILE + tid;
        const bool live = row < A.n;
        // ---- this thread's feature row into the A operand; the next tile's row is
        // loaded while this tile's MMAs and epilogues run
#pragma unroll
        for (int c = 0; c < MLP_IN / 8; c++)
            *reinterpret_cast<uint4 *>(&xa[cm_off(tid, 8 * c, MLP_IN)]) = feat[c];
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        wg_sync(wg);
        load_row(tile + stride, feat);
        float out = b4;
        for (int layer = 0; layer < 3; layer++) {
            const int K = layer == 0 ? MLP_IN : MLP_H;
            const uint16_t *Ab = layer == 0 ? xa : ha;
            const uint16_t *Bw = layer == 0 ? S.w1 : (layer == 1 ? S.w2 : S.w3);
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t a0 = smem_u32(Ab), b0 = smem_u32(Bw);
                for (int k0 = 0; k0 < K; k0 += 16) {
                    const uint32_t koff = (uint32_t)(k0 / 8) * 128u;
                    umma_bf16(tmem, umma_desc(a0 + koff, K), umma_desc(b0 + koff, K), k0 > 0);
                }
                umma_commit(mbar);
            }
            // the group decides together: a wait that ran out anywhere stops the group
            // before any thread reads the accumulator the MMA may still be writing
            if (!wg_all(wg, mbar_wait(mbar, phase, A.spin))) {
                ok = false;
                break;
            }
            phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            // ---- epilogue: this thread's row of the accumulator
#pragma unroll 1
            for (int c0 = 0; c0 < MLP_H; c0 += 32) {
                float v[32];
                tmem_ld32(lane_addr + (uint32_t)c0, v);
#pragma unroll
                for (int i = 0; i < 32; i++)
                    v[i] = fmaxf(v[i] + S.bias[layer][c0 + i], 0.f);
                if (layer < 2) {
#pragma unroll
                    for (int h = 0; h < 32; h += 8) {
                        uint4 q;
                        q.x = pack_bf16x2(v[h], v[h + 1]);
                        q.y = pack_bf16x2(v[h + 2], v[h + 3]);
                        q.z = pack_bf16x2(v[h + 4], v[h + 5]);
                        q.w = pack_bf16x2(v[h + 6], v[h + 7]);
                        *reinterpret_cast<uint4 *>(&ha[cm_off(tid, c0 + h, MLP_H)]) = q;
                        if (MODE == MLP_MODE_TRAIN && live) {
                            uint16_t *hg = (layer == 0 ? A.h1 : A.h2) + (size_t)row * MLP_H + c0 + h;
                            *reinterpret_cast<uint4 *>(hg) = q;
                        }
                    }
                } else {
#pragma unroll
                    for (int i = 0; i < 32; i++)
                        out = fmaf(v[i], S.w4[c0 + i], out);
                    if (MODE == MLP_MODE_TRAIN && live) {
                        float4 *hg = reinterpret_cast<float4 *>(A.h3 + (size_t)row * MLP_H + c0);
#pragma unroll
                        for (int i = 0; i < 8; i++)
                            hg[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
                    }
                }
            }
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
            wg_sync(wg);
        }
        if (!ok)
            break;
        if (live)
            A.y[row] = out;
    }
    // a group that gave up waits once more, bounded, for the MMA it committed
    // (parity `phase`), so tensor memory is not released under it
    if (!ok)
        mbar_wait(mbar, phase, MLP_SPIN_DRAIN);
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(S.tmem),
                     "r"(MLP_H * MLP_WG));
    if (!ok && tid == 0 && A.err)
        atomicExch(A.err, 1);
}

// ------------------------------------------------------------ small kernels
// FP32 master weights -> BF16 operand copies: transposed (forward B operands,
// rows n) into pack; W2 and W3 as they are (rows k: the backward's B operands)
// into packn
constexpr int MLP_PACKN = 2 * MLP_H * MLP_H;
__global__ void k_mlp_pack(const float *theta, uint16_t *pack, uint16_t *packn) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PACK + MLP_PACKN)
        return;
    if (i >= MLP_PACK) {
        const int j = i - MLP_PACK;
        const int which = j / (MLP_H * MLP_H), r = j % (MLP_H * MLP_H);
        const int k = r / MLP_H, n = r % MLP_H;
        const float w = theta[(which == 0 ? MLP_OFF_W2 : MLP_OFF_W3) + k * MLP_H + n];
        __nv_bfloat16 h = __float2bfloat16_rn(w);
        packn[which * MLP_H * MLP_H + cm_off(k, n, MLP_H)] = *reinterpret_cast<uint16_t *>(&h);
        return;
    }
    int n, k, K, off;
    float w;
    if (i < MLP_H * MLP_IN) {  // W1t[n][k] = W1[k][n]
        n = i / MLP_IN;
        k = i % MLP_IN;
        K = MLP_IN;
        w = theta[MLP_OFF_W1 + k * MLP_H + n];
        off = 0;
    } else {
        const int j = i - MLP_H * MLP_IN;
        const int which = j / (MLP_H * MLP_H), r = j % (MLP_H * MLP_H);
        n = r / MLP_H;
        k = r % MLP_H;
        K = MLP_H;
        w = theta[(which == 0 ? MLP_OFF_W2 : MLP_OFF_W3) + k * MLP_H + n];
        off = MLP_H * MLP_IN + which * MLP_H * MLP_H;
    }
    __nv_bfloat16 h = __float2bfloat16_rn(w);
    pack[off + cm_off(n, k, K)] = *reinterpret_cast<uint16_t *>(&h);
}

__device__ __forceinline__ float bf(uint16_t u) {
    return __uint_as_float((uint32_t)u << 16);
}

// loss, output-layer gradients and dL/dh3 (pre-activation, masked by ReLU)
__global__ void k_mlp_out_grad(int B, const float *y, const float *t, const int *tidx,
                               const float *h3, const float *theta, float *d3, float *grad,
                               float *lossbuf) {
    const int b = blockIdx.x, c = threadIdx.x;  // blockDim = 128
    const float tb = t[tidx ? tidx[b] : b];
    const float dy = 2.f * (y[b] - tb) / (float)B;
    const float h = h3[(size_t)b * MLP_H + c];
    d3[(size_t)b * MLP_H + c] = h > 0.f ? dy * theta[MLP_OFF_W4 + c] : 0.f;
    atomicAdd(&grad[MLP_OFF_W4 + c], dy * h);
    if (c == 0) {
        atomicAdd(&grad[MLP_OFF_B4], dy);
        atomicAdd(lossbuf, (y[b] - tb) * (y[b] - tb) / (float)B);
    }
}

// FP32 values -> BF16 high part and BF16 remainder, 8 at a time (one 16-byte
// core-matrix row each)
__device__ __forceinline__ void split_bf16x8(const float (&f)[8], uint4 &hi, uint4 &lo) {
    float h[8], l[8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        h[i] = bf16_round(f[i]);
        l[i] = f[i] - h[i];
    }
    hi = make_uint4(pack_bf16x2(h[0], h[1]), pack_bf16x2(h[2], h[3]), pack_bf16x2(h[4], h[5]),
                    pack_bf16x2(h[6], h[7]));
    lo = make_uint4(pack_bf16x2(l[0], l[1]), pack_bf16x2(l[2], l[3]), pack_bf16x2(l[4], l[5]),
                    pack_bf16x2(l[6], l[7]));
}

struct MlpDgradSmem {
    uint16_t ahi[MLP_TILE * MLP_H];  // D (hi), rows b, K = n
    uint16_t alo[MLP_TILE * MLP_H];  // D (lo)
    uint16_t w[MLP_H * MLP_H];       // W, rows k, K = n
    uint64_t mbar;
    uint32_t tmem;
};

// dprev[b][k] = (sum_n d[b][n] W[k][n]) * (hprev[b][k] > 0): one 128-row tile of the
// batch per CTA, sixteen MMAs (M = N = 128, K = 16) over D's hi and lo parts
__global__ void __launch_bounds__(128, 1)
    k_mlp_dgrad_tc(int B, const float *__restrict__ d, const uint16_t *__restrict__ wn,
                   const uint16_t *__restrict__ hprev, float *__restrict__ dprev, int *err,
                   long long spin) {
    extern __shared__ __align__(1024) unsigned char mlp_bw_raw[];
    MlpDgradSmem &S = *reinterpret_cast<MlpDgradSmem *>(mlp_bw_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row = blockIdx.x * MLP_TILE + tid;
    const bool live = row < B;
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(wn);
        uint4 *dst = reinterpret_cast<uint4 *>(S.w);
        for (int i = tid; i < MLP_H * MLP_H / 8; i += 128)
            dst[i] = src[i];
    }
    const float4 *dr = reinterpret_cast<const float4 *>(d + (size_t)(live ? row : 0) * MLP_H);
#pragma unroll 4
    for (int c = 0; c < MLP_H; c += 8) {
        float f[8];
        const float4 x = live ? dr[c / 4] : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 y = live ? dr[c / 4 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        f[0] = x.x, f[1] = x.y, f[2] = x.z, f[3] = x.w, f[4] = y.x, f[5] = y.y, f[6] = y.z, f[7] = y.w;
        uint4 hi, lo;
        split_bf16x8(f, hi, lo);
        *reinterpret_cast<uint4 *>(&S.ahi[cm_off(tid, c, MLP_H)]) = hi;
        *reinterpret_cast<uint4 *>(&S.alo[cm_off(tid, c, MLP_H)]) = lo;
    }
    if (tid == 0)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&S.mbar)));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&S.tmem)),
                     "r"(MLP_H));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = S.tmem;
    if (tid == 0) {
        const uint32_t ah = smem_u32(S.ahi), al = smem_u32(S.alo), bw = smem_u32(S.w);
        for (int k0 = 0; k0 < MLP_H; k0 += 16) {
            const uint32_t koff = (uint32_t)(k0 / 8) * 128u;
            umma_bf16(tmem, umma_desc(ah + koff, MLP_H), umma_desc(bw + koff, MLP_H), k0 > 0);
        }
        for (int k0 = 0; k0 < MLP_H; k0 += 16) {
            const uint32_t koff = (uint32_t)(k0 / 8) * 128u;
            umma_bf16(tmem, umma_desc(al + koff, MLP_H), umma_desc(bw + koff, MLP_H), 1u);
        }
        umma_commit(&S.mbar);
    }
    const bool ok = __syncthreads_and(mbar_wait(&S.mbar, 0, spin)) != 0;
    if (ok) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(lane_addr + (uint32_t)c0, v);
            if (live) {
                const uint4 *hp = reinterpret_cast<const uint4 *>(hprev + (size_t)row * MLP_H + c0);
                float4 *out = reinterpret_cast<float4 *>(dprev + (size_t)row * MLP_H + c0);
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const uint4 hv = hp[q];
                    const uint32_t w4[4] = {hv.x, hv.y, hv.z, hv.w};
                    float m[8];
#pragma unroll
                    for (int t = 0; t < 4; t++) {
                        m[2 * t] = bf((uint16_t)(w4[t] & 0xFFFFu)) > 0.f ? 1.f : 0.f;
                        m[2 * t + 1] = bf((uint16_t)(w4[t] >> 16)) > 0.f ? 1.f : 0.f;
                    }
                    out[2 * q] = make_float4(v[8 * q] * m[0], v[8 * q + 1] * m[1],
                                             v[8 * q + 2] * m[2], v[8 * q + 3] * m[3]);
                    out[2 * q + 1] = make_float4(v[8 * q + 4] * m[4], v[8 * q + 5] * m[5],
                                                 v[8 * q + 6] * m[6], v[8 * q + 7] * m[7]);
                }
            }
        }
    } else {
        mbar_wait(&S.mbar, 0, MLP_SPIN_DRAIN);  // the committed MMA, before the release
        if (tid == 0)
            atomicExch(err, 1);
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(S.tmem),
                     "r"(MLP_H));
}

constexpr int MLP_WCHUNK = 64;   // batch rows per weight-gradient chunk (the MMA's K)
constexpr int MLP_WSPLIT = 16;   // most CTAs per layer (partial products)

struct MlpWgradSmem {
    uint16_t a[MLP_H * MLP_WCHUNK];    // A^T chunk: rows k (M), K = batch rows
    uint16_t bhi[MLP_H * MLP_WCHUNK];  // D^T chunk (hi): rows n (N), K = batch rows
    uint16_t blo[MLP_H * MLP_WCHUNK];
    uint64_t mbar;
    uint32_t tmem;
};

struct MlpWgradArgs {
    int B;
    const uint16_t *X, *h1, *h2;  // layer inputs (features through idx)
    const int *idx;
    const float *d1, *d2, *d3;    // layer output gradients (pre-activation)
    float *wpart, *bpart;         // [3][gridDim.x][128][128], [3][gridDim.x][128]
    int *err;
    long long spin;
};

// dW_L = A_L^T D_L over the batch: blockIdx.y = layer (0: features -> W1, 1: h1 -> W2,
// 2: h2 -> W3), blockIdx.x = one of gridDim.x CTAs that take every gridDim.x-th
// 64-row chunk; each CTA accumulates its chunks in tensor memory (M = N = 128; the
// 64 feature rows of layer 0 padded with zero rows) and writes its partial product
// and its column sums of D (the bias gradient)
__global__ void __launch_bounds__(128, 1) k_mlp_wgrad_tc(MlpWgradArgs A) {
    extern __shared__ __align__(1024) unsigned char mlp_bw_raw[];
    MlpWgradSmem &S = *reinterpret_cast<MlpWgradSmem *>(mlp_bw_raw);
    const int tid = threadIdx.x, warp = tid >> 5, L = blockIdx.y;
    const int Kin = L == 0 ? MLP_IN : MLP_H;
    const uint16_t *act = L == 0 ? A.X : (L == 1 ? A.h1 : A.h2);
    const int *aidx = L == 0 ? A.idx : nullptr;
    const float *d = L == 0 ? A.d1 : (L == 1 ? A.d2 : A.d3);
    if (tid == 0)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&S.mbar)));
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&S.tmem)),
                     "r"(MLP_H));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = S.tmem;
    const int nchunks = (A.B + MLP_WCHUNK - 1) / MLP_WCHUNK;
    float colsum = 0.f;
    uint32_t phase = 0;
    bool ok = true, any = false;
    for (int ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
        const int b0 = ch * MLP_WCHUNK;
        // thread t stages row t of A^T (activation column t) and row t of D^T
#pragma unroll 1
        for (int g = 0; g < MLP_WCHUNK; g += 8) {
            uint32_t av[4];
            float f[8];
#pragma unroll
            for (int j = 0; j < 8; j += 2) {
                const int b = b0 + g + j;
                uint32_t lo16 = 0, hi16 = 0;
                if (tid < Kin) {
                    if (b < A.B)
                        lo16 = act[(size_t)(aidx ? aidx[b] : b) * Kin + tid];
                    if (b + 1 < A.B)
                        hi16 = act[(size_t)(aidx ? aidx[b + 1] : b + 1) * Kin + tid];
                }
                av[j / 2] = lo16 | (hi16 << 16);
                f[j] = b < A.B ? d[(size_t)b * MLP_H + tid] : 0.f;
                f[j + 1] = b + 1 < A.B ? d[(size_t)(b + 1) * MLP_H + tid] : 0.f;
                colsum += f[j] + f[j + 1];
            }
            *reinterpret_cast<uint4 *>(&S.a[cm_off(tid, g, MLP_WCHUNK)]) =
                make_uint4(av[0], av[1], av[2], av[3]);
            uint4 hi, lo;
            split_bf16x8(f, hi, lo);
            *reinterpret_cast<uint4 *>(&S.bhi[cm_off(tid, g, MLP_WCHUNK)]) = hi;
            *reinterpret_cast<uint4 *>(&S.blo[cm_off(tid, g, MLP_WCHUNK)]) = lo;
        }
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (tid == 0) {
            const uint32_t aa = smem_u32(S.a), bh = smem_u32(S.bhi), bl = smem_u32(S.blo);
            for (int k0 = 0; k0 < MLP_WCHUNK; k0 += 16) {
                const uint32_t koff = (uint32_t)(k0 / 8) * 128u;
                umma_bf16(tmem, umma_desc(aa + koff, MLP_WCHUNK), umma_desc(bh + koff, MLP_WCHUNK),
                          (any || k0 > 0) ? 1u : 0u);
            }
            for (int k0 = 0; k0 < MLP_WCHUNK; k0 += 16) {
                const uint32_t koff = (uint32_t)(k0 / 8) * 128u;
                umma_bf16(tmem, umma_desc(aa + koff, MLP_WCHUNK), umma_desc(bl + koff, MLP_WCHUNK),
                          1u);
            }
            umma_commit(&S.mbar);
        }
        any = true;
        // the operands are restaged only after the MMAs that read them completed
        if (!__syncthreads_and(mbar_wait(&S.mbar, phase, A.spin))) {
            ok = false;
            break;
        }
        phase ^= 1u;
    }
    float *wp = A.wpart + ((size_t)L * gridDim.x + blockIdx.x) * MLP_H * MLP_H;
    if (ok && any) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < MLP_H; c0 += 32) {
            float v[32];
            tmem_ld32(lane_addr + (uint32_t)c0, v);
            float4 *out = reinterpret_cast<float4 *>(wp + (size_t)tid * MLP_H + c0);
#pragma unroll
            for (int q = 0; q < 8; q++)
                out[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
        }
    } else if (ok) {
        for (int c = 0; c < MLP_H; c++)
            wp[(size_t)tid * MLP_H + c] = 0.f;
    } else {
        mbar_wait(&S.mbar, phase, MLP_SPIN_DRAIN);  // the committed MMAs, before the release
        if (tid == 0)
            atomicExch(A.err, 1);
    }
    A.bpart[((size_t)L * gridDim.x + blockIdx.x) * MLP_H + tid] = colsum;
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(S.tmem),
                     "r"(MLP_H));
}

// the layers' weight and bias gradients: the partial products summed in CTA order
__global__ void k_mlp_wgrad_reduce(int G, const float *__restrict__ wpart,
                                   const float *__restrict__ bpart, float *grad) {
    const int L = blockIdx.y;
    const int Kin = L == 0 ? MLP_IN : MLP_H;
    const int offW = L == 0 ? MLP_OFF_W1 : (L == 1 ? MLP_OFF_W2 : MLP_OFF_W3);
    const int offB = L == 0 ? MLP_OFF_B1 : (L == 1 ? MLP_OFF_B2 : MLP_OFF_B3);
    const int e = blockIdx.x * blockDim.x + threadIdx.x;  // k * 128 + n, plus 128 bias rows
    if (e < Kin * MLP_H) {
        float acc = 0.f;
        for (int g = 0; g < G; g++)
            acc += wpart[((size_t)L * G + g) * MLP_H * MLP_H + e];
        grad[offW + e] += acc;
    } else if (e < Kin * MLP_H + MLP_H) {
        const int n = e - Kin * MLP_H;
        float acc = 0.f;
        for (int g = 0; g < G; g++)
            acc += bpart[((size_t)L * G + g) * MLP_H + n];
        grad[offB + n] += acc;
    }
}

__global__ void k_mlp_adam(float *theta, float *m1, float *m2, const float *g, int n, float lr,
                           float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.f - b1) * gi;
    const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    theta[i] -= lr * (a / bc1) / (sqrtf(v / bc2) + eps);
}

// spacing feature, norms, sample collection
__global__ void k_mlp_norms(MlpFields F, double *partials, unsigned *ticket, double *norms) {
    __shared__ double red[32 * 3];
    double acc[3] = {0, 0, 0};
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.nv; i += stride) {
        acc[0] += F.b[i] * F.b[i];
        const double p1 = F.ph1[i], d = F.pcur[i] - p1, d2 = d - (p1 - F.ph2[i]);
        acc[1] += d * d;
        acc[2] += d2 * d2;
    }
    if (grid_reduce<3>(acc, partials, ticket, red) && threadIdx.x == 0) {
        for (int k = 0; k < 3; k++) {
            const double r = sqrt(acc[k] / F.nv);
            norms[k] = r > 0 ? 1.0 / r : 0.0;
        }
    }
}

// the 64 features of node i (layout in mp_mlp.cuh), as BF16 into a 128-byte row
__device__ __forceinline__ void node_features(const MlpFields &F, int i, uint16_t *row) {
    const double sb = F.norms[0], sp = F.norms[1];
    float f[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; k++)
        f[k] = 0.f;
    const size_t base = (size_t)(i / 64) * F.K * 64 + (i % 64);
#pragma unroll 4
    for (int k = 0; k < MLP_STENCIL; k++) {
        const int j = F.cols[base + (size_t)k * 64];
        const double pc = F.pcur[j], p1 = F.ph1[j];
        f[3 * k] = (float)(F.b[j] * sb);
        f[3 * k + 1] = (float)((pc - p1) * sp);
        f[3 * k + 2] = (float)((p1 - F.ph2[j]) * sp);
    }
    f[60] = F.hloc[i];
    f[61] = F.bflag[i] ? 1.f : 0.f;
    f[62] = 1.f;
    uint4 *dst = reinterpret_cast<uint4 *>(row);
#pragma unroll
    for (int c = 0; c < MLP_IN; c += 8) {
        uint4 v;
        v.x = pack_bf16x2(f[c], f[c + 1]);
        v.y = pack_bf16x2(f[c + 2], f[c + 3]);
        v.z = pack_bf16x2(f[c + 4], f[c + 5]);
        v.w = pack_bf16x2(f[c + 6], f[c + 7]);
        dst[c / 8] = v;
    }
}

__global__ void k_mlp_collect(MlpFields F, const int *idx, int nidx, const double *xnew,
                              uint16_t *X, float *t, const int *step, int cap_steps) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nidx || *step < 2)
        return;
    const size_t slot = (size_t)((*step - 2) % cap_steps) * nidx;
    X += slot * MLP_IN;
    t += slot;
    const int i = idx[s];
    node_features(F, i, X + (size_t)s * MLP_IN);
    const double pc = F.pcur[i];
    t[s] = (float)(((xnew[i] - pc) - (pc - F.ph1[i])) * F.norms[2]);
}

// features of every node (skipped while *step < 2: no pressure history)
// the three gathered fields of every node, scaled and rounded to FP32 once
// (the same values node_features forms per gather), so that the feature kernel
// fetches one 16-byte record per stencil member instead of four doubles
__global__ void k_mlp_prep(MlpFields F, float4 *q, const int *step) {
    if (*step < 2)
        return;
    const double sb = F.norms[0], sp = F.norms[1];
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < F.nv; j += gridDim.x * blockDim.x) {
        const double pc = F.pcur[j], p1 = F.ph1[j];
        q[j] = make_float4((float)(F.b[j] * sb), (float)((pc - p1) * sp),
                           (float)((p1 - F.ph2[j]) * sp), 0.f);
    }
}

// features of every node from the prepared records (skipped while *step < 2: no
// pressure history)
__global__ void __launch_bounds__(256)
    k_mlp_features(MlpFields F, const float4 *__restrict__ q, uint16_t *X, const int *step) {
    if (*step < 2)
        return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.nv; i += gridDim.x * blockDim.x) {
        float f[MLP_IN];
        const size_t base = (size_t)(i / 64) * F.K * 64 + (i % 64);
#pragma unroll
        for (int k = 0; k < MLP_STENCIL; k++) {
            const float4 v = __ldg(q + F.cols[base + (size_t)k * 64]);
            f[3 * k] = v.x;
            f[3 * k + 1] = v.y;
            f[3 * k + 2] = v.z;
        }
        f[60] = F.hloc[i];
        f[61] = F.bflag[i] ? 1.f : 0.f;
        f[62] = 1.f;
        f[63] = 0.f;
        uint4 *dst = reinterpret_cast<uint4 *>(X + (size_t)i * MLP_IN);
#pragma unroll
        for (int c = 0; c < MLP_IN; c += 8) {
            uint4 v;
            v.x = pack_bf16x2(f[c], f[c + 1]);
            v.y = pack_bf16x2(f[c + 2], f[c + 3]);
            v.z = pack_bf16x2(f[c + 4], f[c + 5]);
            v.w = pack_bf16x2(f[c + 6], f[c + 7]);
            dst[c / 8] = v;
        }
    }
}

// The prediction as a pressure correction: the clamped output (8 units: the
// training targets have unit RMS) scaled back by the RMS of the second
// difference.  Written to corr when set, else added to x (which holds the
// extrapolated guess).  Zero while *step < 2 (no second difference yet).
__global__ void k_mlp_combine(MlpFields F, const float *y, double *x, double *corr,
                              const int *step) {
    const bool early = *step < 2;
    const double s2 = F.norms[2];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < F.nv; i += gridDim.x * blockDim.x) {
        const double cl = fmin(fmax((double)y[i], -8.0), 8.0);
        const double c = (early || !(s2 > 0)) ? 0.0 : cl / s2;
        if (corr)
            corr[i] = c;
        else
            x[i] += c;
    }
}

__global__ void k_f32_to_bf16(const float *a, uint16_t *b, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        __nv_bfloat16 h = __float2bfloat16_rn(a[i]);
        b[i] = *reinterpret_cast<uint16_t *>(&h);
    }
}

// --------------------------------------------------------------- host side
static int fwd_smem() { return (int)sizeof(MlpSmem) + 1024; }

template <int MODE> static int launch_forward(MlpFwdArgs &a, cudaStream_t s) {
    const int sm = fwd_smem();
    MP_CUDA(cudaFuncSetAttribute(k_mlp_forward<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    const int tiles = (a.n + MLP_TILE - 1) / MLP_TILE;
    const int grid = std::max(1, std::min(tiles, sm_count()));
    k_mlp_forward<MODE><<<grid, 128 * MLP_WG, sm, s>>>(a);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

static int repack(Mlp &m, cudaStream_t s) {
    k_mlp_pack<<<(MLP_PACK + MLP_PACKN + 255) / 256, 256, 0, s>>>(m.theta.p, m.pack.p, m.packn.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int mlp_create(Mlp **out, uint64_t seed) {
    Mlp *m = new Mlp;
    int rc;
    if ((rc = m->theta.alloc(MLP_NPARAM)) || (rc = m->m1.alloc(MLP_NPARAM)) ||
        (rc = m->m2.alloc(MLP_NPARAM)) || (rc = m->grad.alloc(MLP_NPARAM)) ||
        (rc = m->pack.alloc(MLP_PACK)) || (rc = m->packn.alloc(MLP_PACKN)) ||
        (rc = m->wpart.alloc((size_t)3 * MLP_WSPLIT * (MLP_H * MLP_H + MLP_H))) ||
        (rc = m->err.alloc(1))) {
        delete m;
        return rc;
    }
    // He-uniform initialisation from a fixed-seed generator (host)
    std::vector<float> th(MLP_NPARAM, 0.f);
    std::mt19937_64 g(seed);
    auto init = [&](int off, int fan_in, int count) {
        std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
        for (int i = 0; i < count; i++)
            th[off + i] = u(g);
    };
    init(MLP_OFF_W1, MLP_IN, MLP_IN * MLP_H);
    init(MLP_OFF_W2, MLP_H, MLP_H * MLP_H);
    init(MLP_OFF_W3, MLP_H, MLP_H * MLP_H);
    {
        std::uniform_real_distribution<float> u(-1.f / std::sqrt((float)MLP_H), 1.f / std::sqrt((float)MLP_H));
        for (int i = 0; i < MLP_H; i++)
            th[MLP_OFF_W4 + i] = 0.1f * u(g);
    }
    MP_CUDA(cudaMemcpy(m->theta.p, th.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
    MP_CUDA(cudaMemset(m->m1.p, 0, sizeof(float) * MLP_NPARAM));
    MP_CUDA(cudaMemset(m->m2.p, 0, sizeof(float) * MLP_NPARAM));
    MP_CUDA(cudaMemset(m->err.p, 0, sizeof(int)));
    MP_TRY(repack(*m, 0));
    MP_CUDA(cudaDeviceSynchronize());
    *out = m;
    return MP_OK;
}

void mlp_destroy(Mlp *m) { delete m; }

static int mlp_check_err(Mlp &m, cudaStream_t s) {
    int e = 0;
    MP_CUDA(cudaMemcpyAsync(&e, m.err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (e) {
        MP_CUDA(cudaMemsetAsync(m.err.p, 0, sizeof(int), s));
        MP_CUDA(cudaStreamSynchronize(s));
        return fail(MP_TIMEOUT, "tensor-core MLP: an mbarrier wait ran out");
    }
    return MP_OK;
}

int mlp_predict_fields(Mlp &m, const MlpFields &F, double *x, double *corr, const int *step,
                       cudaStream_t s) {
    if ((size_t)F.nv > m.fy.n)
        return fail(MP_BAD_ARG, "field prediction for %d nodes: %zu reserved", F.nv, m.fy.n);
    const unsigned g = (unsigned)std::min((F.nv + 255) / 256, sm_count() * 16);
    k_mlp_prep<<<g, 256, 0, s>>>(F, m.fq.p, step);
    MP_CHECK_LAUNCH();
    k_mlp_features<<<g, 256, 0, s>>>(F, m.fq.p, m.fx.p, step);
    MP_CHECK_LAUNCH();
    MlpFwdArgs a{};
    a.n = F.nv;
    a.pack = m.pack.p;
    a.theta = m.theta.p;
    a.X = m.fx.p;
    a.y = m.fy.p;
    a.err = m.err.p;
    a.spin = m.spin;
    MP_TRY(launch_forward<MLP_MODE_ROWS>(a, s));
    k_mlp_combine<<<g, 256, 0, s>>>(F, m.fy.p, x, corr, step);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int mlp_reserve_fields(Mlp &m, int nv) {
    if ((size_t)nv <= m.fy.n)
        return MP_OK;
    MP_TRY(m.fx.alloc((size_t)nv * MLP_IN));
    MP_TRY(m.fy.alloc(nv));
    MP_TRY(m.fq.alloc(nv));
    MP_CUDA(cudaMemset(m.fx.p, 0, m.fx.bytes()));
    return MP_OK;
}

int mlp_norms(const MlpFields &F, double *norms, double *partials, unsigned *ticket,
              cudaStream_t s) {
    const unsigned g = (unsigned)std::min((F.nv + 255) / 256, sm_count() * 4);
    k_mlp_norms<<<g, 256, 0, s>>>(F, partials, ticket, norms);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int mlp_collect(const MlpFields &F, const int *idx, int nidx, const double *xnew, uint16_t *X,
                float *t, const int *step, int cap_steps, cudaStream_t s) {
    k_mlp_collect<<<(nidx + 127) / 128, 128, 0, s>>>(F, idx, nidx, xnew, X, t, step, cap_steps);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

static int ensure_cap(Mlp &m, int B) {
    if (B <= m.cap)
        return MP_OK;
    const size_t n = (size_t)B * MLP_H;
    MP_TRY(m.h1.alloc(n));
    MP_TRY(m.h2.alloc(n));
    MP_TRY(m.h3.alloc(n));
    MP_TRY(m.d3.alloc(n));
    MP_TRY(m.d2.alloc(n));
    MP_TRY(m.d1.alloc(n));
    MP_TRY(m.y.alloc(B));
    MP_TRY(m.lossbuf.alloc(1));
    m.cap = B;
    return MP_OK;
}

static int bw_smem(size_t bytes) { return (int)bytes + 1024; }

// forward + backward of one batch: grad = dL/dtheta (accumulated from zero), loss to lossbuf
static int batch_grad(Mlp &m, const uint16_t *X, const float *t, const int *idx, int B,
                      cudaStream_t s) {
    MP_TRY(ensure_cap(m, B));
    MlpFwdArgs a{};
    a.n = B;
    a.pack = m.pack.p;
    a.theta = m.theta.p;
    a.X = X;
    a.idx = idx;
    a.y = m.y.p;
    a.h1 = m.h1.p;
    a.h2 = m.h2.p;
    a.h3 = m.h3.p;
    a.err = m.err.p;
    a.spin = m.spin;
    MP_TRY(launch_forward<MLP_MODE_TRAIN>(a, s));
    MP_CUDA(cudaMemsetAsync(m.grad.p, 0, sizeof(float) * MLP_NPARAM, s));
    MP_CUDA(cudaMemsetAsync(m.lossbuf.p, 0, sizeof(float), s));
    k_mlp_out_grad<<<B, MLP_H, 0, s>>>(B, m.y.p, t, idx, m.h3.p, m.theta.p, m.d3.p, m.grad.p,
                                      m.lossbuf.p);
    MP_CHECK_LAUNCH();
    // input gradients of layers 3 and 2 on the tensor cores
    const int ds = bw_smem(sizeof(MlpDgradSmem));
    MP_CUDA(cudaFuncSetAttribute(k_mlp_dgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, ds));
    const unsigned tiles = (unsigned)((B + MLP_TILE - 1) / MLP_TILE);
    k_mlp_dgrad_tc<<<tiles, 128, ds, s>>>(B, m.d3.p, m.packn.p + MLP_H * MLP_H, m.h2.p, m.d2.p,
                                          m.err.p, m.spin);
    MP_CHECK_LAUNCH();
    k_mlp_dgrad_tc<<<tiles, 128, ds, s>>>(B, m.d2.p, m.packn.p, m.h1.p, m.d1.p, m.err.p, m.spin);
    MP_CHECK_LAUNCH();
    // weight gradients of the three layers in one launch, the batch split across CTAs
    const int ws = bw_smem(sizeof(MlpWgradSmem));
    MP_CUDA(cudaFuncSetAttribute(k_mlp_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, ws));
    const int nch = (B + MLP_WCHUNK - 1) / MLP_WCHUNK;
    const int G = std::min(nch, MLP_WSPLIT);
    MlpWgradArgs w{};
    w.B = B;
    w.X = X;
    w.h1 = m.h1.p;
    w.h2 = m.h2.p;
    w.idx = idx;
    w.d1 = m.d1.p;
    w.d2 = m.d2.p;
    w.d3 = m.d3.p;
    w.wpart = m.wpart.p;
    w.bpart = m.wpart.p + (size_t)3 * MLP_WSPLIT * MLP_H * MLP_H;
    w.err = m.err.p;
    w.spin = m.spin;
    k_mlp_wgrad_tc<<<dim3((unsigned)G, 3), 128, ws, s>>>(w);
    MP_CHECK_LAUNCH();
    // the partial arrays are indexed with the launch's G
    k_mlp_wgrad_reduce<<<dim3((MLP_H * MLP_H + MLP_H + 255) / 256, 3), 256, 0, s>>>(
        G, w.wpart, w.bpart, m.grad.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int mlp_train(Mlp &m, const uint16_t *X, const float *t, int n, int epochs, int batch, double lr,
              uint64_t seed, double *loss, cudaStream_t s) {
    if (n < batch || batch < MLP_TILE || batch % MLP_TILE)
        return fail(MP_BAD_ARG, "mlp_train: %d samples, batch %d (multiple of %d)", n, batch,
                    MLP_TILE);
    MP_TRY(ensure_cap(m, batch));
    std::vector<int> perm(n);
    for (int i = 0; i < n; i++)
        perm[i] = i;
    std::mt19937_64 g(seed);
    MP_TRY(m.idx.alloc(n));
    const int nb = n / batch;
    double last = 0;
    for (int e = 0; e < epochs; e++) {
        std::shuffle(perm.begin(), perm.end(), g);
        MP_CUDA(cudaMemcpyAsync(m.idx.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
        double ep = 0;
        for (int bi = 0; bi < nb; bi++) {
            const int *idx = m.idx.p + (size_t)bi * batch;
            MP_TRY(batch_grad(m, X, t, idx, batch, s));
            m.adam_t++;
            const float bc1 = 1.f - std::pow(0.9f, (float)m.adam_t);
            const float bc2 = 1.f - std::pow(0.999f, (float)m.adam_t);
            k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, s>>>(m.theta.p, m.m1.p, m.m2.p, m.grad.p,
                                                                MLP_NPARAM, (float)lr, bc1, bc2);
            MP_CHECK_LAUNCH();
            MP_TRY(repack(m, s));
            if (e == epochs - 1) {
                float l = 0;
                MP_CUDA(cudaMemcpyAsync(&l, m.lossbuf.p, sizeof(float), cudaMemcpyDeviceToHost, s));
                MP_CUDA(cudaStreamSynchronize(s));
                ep += l;
            }
        }
        last = ep / nb;
    }
    MP_TRY(mlp_check_err(m, s));
    if (loss)
        *loss = last;
    return MP_OK;
}

}  // namespace mp

using namespace mp;

struct mp_mlp_s {
    Mlp *m = nullptr;
    ~mp_mlp_s() { mlp_destroy(m); }
};

// row-major FP32 (host or device) -> BF16 device rows
static int to_bf16_rows(const float *X, size_t count, dbuf<uint16_t> &out, cudaStream_t s) {
    dbuf<float> tmp;
    const float *dX;
    MP_TRY(stage_in(X, count, tmp, &dX, s));
    MP_TRY(out.alloc(count));
    k_f32_to_bf16<<<(unsigned)((count + 255) / 256), 256, 0, s>>>(dX, out.p, count);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

extern "C" int mp_mlp_num_params(void) { return MLP_NPARAM; }

extern "C" int mp_mlp_create(uint64_t seed, mp_mlp *out) {
    if (!out)
        return fail(MP_BAD_ARG, "mp_mlp_create: null out");
    mp_mlp h = new mp_mlp_s;
    int rc = mlp_create(&h->m, seed);
    if (rc != MP_OK) {
        delete h;
        return rc;
    }
    *out = h;
    return MP_OK;
}

extern "C" int mp_mlp_get_params(mp_mlp h, float *theta) {
    if (!h || !theta)
        return fail(MP_BAD_ARG, "mp_mlp_get_params: null argument");
    MP_CUDA(cudaMemcpy(theta, h->m->theta.p, sizeof(float) * MLP_NPARAM, cudaMemcpyDefault));
    return MP_OK;
}

extern "C" int mp_mlp_set_params(mp_mlp h, const float *theta) {
    if (!h || !theta)
        return fail(MP_BAD_ARG, "mp_mlp_set_params: null argument");
    MP_CUDA(cudaMemcpy(h->m->theta.p, theta, sizeof(float) * MLP_NPARAM, cudaMemcpyDefault));
    MP_TRY(repack(*h->m, 0));
    MP_CUDA(cudaDeviceSynchronize());
    return MP_OK;
}

extern "C" int mp_mlp_forward(mp_mlp h, const float *X, int n, float *y) {
    if (!h || !X || !y || n <= 0)
        return fail(MP_BAD_ARG, "mp_mlp_forward: bad arguments");
    dbuf<uint16_t> xb;
    MP_TRY(to_bf16_rows(X, (size_t)n * MLP_IN, xb, 0));
    dbuf<float> yd;
    MP_TRY(yd.alloc(n));
    MlpFwdArgs a{};
    a.n = n;
    a.pack = h->m->pack.p;
    a.theta = h->m->theta.p;
    a.X = xb.p;
    a.y = yd.p;
    a.err = h->m->err.p;
    a.spin = h->m->spin;
    MP_TRY(launch_forward<MLP_MODE_ROWS>(a, 0));
    MP_CUDA(cudaMemcpy(y, yd.p, sizeof(float) * n, cudaMemcpyDefault));
    return mlp_check_err(*h->m, 0);
}

extern "C" int mp_mlp_gradient(mp_mlp h, const float *X, const float *t, int n, double *loss,
                               float *grad) {
    if (!h || !X || !t || !grad || n <= 0)
        return fail(MP_BAD_ARG, "mp_mlp_gradient: bad arguments");
    dbuf<uint16_t> xb;
    dbuf<float> tt;
    const float *dt;
    MP_TRY(to_bf16_rows(X, (size_t)n * MLP_IN, xb, 0));
    MP_TRY(stage_in(t, (size_t)n, tt, &dt, 0));
    MP_TRY(batch_grad(*h->m, xb.p, dt, nullptr, n, 0));
    float l = 0;
    MP_CUDA(cudaMemcpy(&l, h->m->lossbuf.p, sizeof(float), cudaMemcpyDeviceToHost));
    MP_CUDA(cudaMemcpy(grad, h->m->grad.p, sizeof(float) * MLP_NPARAM, cudaMemcpyDefault));
    if (loss)
        *loss = l;
    return mlp_check_err(*h->m, 0);
}

extern "C" int mp_mlp_train(mp_mlp h, const float *X, const float *t, int n, int epochs, int batch,
                            double lr, uint64_t seed, double *loss) {
    if (!h || !X || !t)
        return fail(MP_BAD_ARG, "mp_mlp_train: null argument");
    dbuf<uint16_t> xb;
    dbuf<float> tt;
    const float *dt;
    MP_TRY(to_bf16_rows(X, (size_t)n * MLP_IN, xb, 0));
    MP_TRY(stage_in(t, (size_t)n, tt, &dt, 0));
    return mlp_train(*h->m, xb.p, dt, n, epochs, batch, lr, seed, loss, 0);
}

extern "C" int mp_mlp_set_spin_limit(mp_mlp h, long long polls) {
    if (!h || polls < 0)
        return fail(MP_BAD_ARG, "mp_mlp_set_spin_limit: a handle and a limit >= 0");
    h->m->spin = polls;
    return MP_OK;
}

extern "C" int mp_mlp_destroy(mp_mlp h) {
    delete h;
    return MP_OK;
}

namespace mp {
Mlp *mlp_of(::mp_mlp_s *h) { return h ? h->m : nullptr; }
}  // namespace mp
