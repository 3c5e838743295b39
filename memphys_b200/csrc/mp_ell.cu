// mp_ell.cu -- ELL (64-row slice) storage, packing and the plain SpMV kernel,
// plus the mp_op_* C ABI (the Eigen::SparseMatrix operators of POINTS,
// class.hpp:116-124, applied as `matrix * vector`).
#include "mp_ell.cuh"
#include "mp_cloud.cuh"

namespace mp {

template <class T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// row-major (nrows x K) -> slices; rows >= nrows get column 0 / value 0
template <class Tin, class Tout>
__global__ void ell_pack_kernel(int nrows, int nrows_pad, int K, const int *cols_rm,
                                const Tin *vals_rm, int *cols, Tout *vals) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t total = (size_t)nrows_pad * K;
    if (t >= total)
        return;
    int row = (int)(t / K), k = (int)(t % K);
    size_t o = ell_index(row, k, K);
    bool real = row < nrows;
    if (cols)
        cols[o] = real ? cols_rm[(size_t)row * K + k] : 0;
    if (vals)
        vals[o] = real ? (Tout)vals_rm[(size_t)row * K + k] : (Tout)0;
}

__global__ void f64_to_f32(const double *a, float *b, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        b[i] = (float)a[i];
}

int ell_create(Ell &E, int nrows, int ncols, int K, const int *cols, const double *vals, bool fp32,
               cudaStream_t s) {
    if (nrows <= 0 || K <= 0)
        return fail(MP_BAD_ARG, "ELL operator: nrows=%d width=%d", nrows, K);
    E.nrows = nrows;
    E.ncols = ncols;
    E.K = K;
    const int np = ell_padded_rows(nrows);
    const size_t tot = (size_t)np * K;
    dbuf<int> tc;
    dbuf<double> tv;
    const int *dc = nullptr;
    const double *dv = nullptr;
    MP_TRY(stage_in(cols, (size_t)nrows * K, tc, &dc, s));
    if (vals)
        MP_TRY(stage_in(vals, (size_t)nrows * K, tv, &dv, s));
    MP_TRY(E.cols.alloc(tot));
    const int tb = 256;
    const unsigned nb = (unsigned)((tot + tb - 1) / tb);
    if (vals) {
        MP_TRY(E.v64.alloc(tot));
        ell_pack_kernel<double, double><<<nb, tb, 0, s>>>(nrows, np, K, dc, dv, E.cols.p, E.v64.p);
        MP_CHECK_LAUNCH();
        if (fp32)
            MP_TRY(ell_make_fp32(E, s));
    } else {
        ell_pack_kernel<double, double><<<nb, tb, 0, s>>>(nrows, np, K, dc, nullptr, E.cols.p,
                                                          nullptr);
        MP_CHECK_LAUNCH();
    }
    MP_CUDA(cudaStreamSynchronize(s));  // staged inputs die at return
    return MP_OK;
}

int ell_make_fp32(Ell &E, cudaStream_t s) {
    const size_t tot = E.v64.n;
    MP_TRY(E.v32.alloc(tot));
    f64_to_f32<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(E.v64.p, E.v32.p, tot);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// one warp per slice: does every column - row of the slice fit 16 bits?  If so the
// deltas are written and the slice's flag set
__global__ void k_ell_deltas(int nrows, int K, const int *cols, short *d, unsigned char *flag,
                             unsigned *count) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nsl = (nrows + SLICE - 1) / SLICE;
    if (w >= nsl)
        return;
    const size_t base = (size_t)w * K * SLICE;
    bool fits = true;
    for (int t = lane; t < K * SLICE; t += 32) {
        const int row = w * SLICE + (t % SLICE);
        const int dl = cols[base + t] - row;
        fits = fits && dl >= -32768 && dl <= 32767;
    }
    fits = __all_sync(0xffffffffu, fits);
    if (fits)
        for (int t = lane; t < K * SLICE; t += 32)
            d[base + t] = (short)(cols[base + t] - (w * SLICE + (t % SLICE)));
    if (lane == 0) {
        flag[w] = fits ? 1 : 0;
        if (fits)
            atomicAdd(count, 1u);
    }
}

// one thread per row (padded rows included: all column 0, value 0)
constexpr int SORT_KMAX = 64;
__global__ void k_ell_sort_rows(int np, int K, int *cols, double *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np)
        return;
    const size_t base = (size_t)(i / SLICE) * K * SLICE + i % SLICE;
    int c[SORT_KMAX];
    double w[SORT_KMAX];
    for (int k = 0; k < K; k++) {
        c[k] = cols[base + (size_t)k * SLICE];
        w[k] = vals[base + (size_t)k * SLICE];
    }
    for (int k = 2; k < K; k++) {  // insertion sort of entries 1..K-1
        const int ck = c[k];
        const double wk = w[k];
        int j = k - 1;
        while (j >= 1 && c[j] > ck) {
            c[j + 1] = c[j];
            w[j + 1] = w[j];
            j--;
        }
        c[j + 1] = ck;
        w[j + 1] = wk;
    }
    for (int k = 1; k < K; k++) {
        cols[base + (size_t)k * SLICE] = c[k];
        vals[base + (size_t)k * SLICE] = w[k];
    }
}

int ell_sort_rows(Ell &E, cudaStream_t s) {
    if (E.soff.p || E.K > SORT_KMAX || !E.v64.p || E.nrows == 0)
        return MP_OK;
    const int np = ell_padded_rows(E.nrows);
    k_ell_sort_rows<<<(np + 255) / 256, 256, 0, s>>>(np, E.K, E.cols.p, E.v64.p);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int ell_make_deltas(Ell &E, cudaStream_t s, double *frac) {
    if (E.soff.p || !E.cols.p)
        return fail(MP_BAD_ARG, "ell_make_deltas: uniform-width operators only");
    const int nsl = (E.nrows + SLICE - 1) / SLICE;
    MP_TRY(E.dcols.alloc(E.cols.n));
    MP_TRY(E.dslice.alloc(nsl));
    dbuf<unsigned> cnt;
    MP_TRY(cnt.alloc(1));
    MP_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned), s));
    k_ell_deltas<<<(unsigned)((nsl + 7) / 8), 256, 0, s>>>(E.nrows, E.K, E.cols.p, E.dcols.p,
                                                           E.dslice.p, cnt.p);
    MP_CHECK_LAUNCH();
    unsigned h = 0;
    MP_CUDA(cudaMemcpyAsync(&h, cnt.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (frac)
        *frac = nsl ? (double)h / nsl : 0.0;
    return MP_OK;
}

// y = alpha*A x + beta*y, one warp per 64-row slice, two rows per lane
template <class T>
__global__ void __launch_bounds__(256)
    ell_spmv_kernel(EllView<T> A, const T *__restrict__ x, T *__restrict__ y, T alpha, T beta) {
    using V2 = typename Vec2<T>::type;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nslices = (A.nrows + SLICE - 1) / SLICE;
    if (warp >= nslices)
        return;
    size_t base;
    int K;
    slice_span(A, warp, base, K);
    base += 2 * lane;
    T a0 = 0, a1 = 0;
#pragma unroll 4
    for (int k = 0; k < K; k++) {
        const int2 c = __ldcs(reinterpret_cast<const int2 *>(A.cols + base + (size_t)k * SLICE));
        const V2 v = __ldcs(reinterpret_cast<const V2 *>(A.vals + base + (size_t)k * SLICE));
        a0 = fma(v.x, __ldg(x + c.x), a0);
        a1 = fma(v.y, __ldg(x + c.y), a1);
    }
    const int r0 = warp * SLICE + 2 * lane;
    if (r0 < A.nrows) {
        T o0 = alpha * a0;
        if (beta != T(0))
            o0 = fma(beta, y[r0], o0);
        y[r0] = o0;
    }
    if (r0 + 1 < A.nrows) {
        T o1 = alpha * a1;
        if (beta != T(0))
            o1 = fma(beta, y[r0 + 1], o1);
        y[r0 + 1] = o1;
    }
}

template <class T>
int ell_spmv(const EllView<T> &A, const T *x, T *y, double alpha, double beta, cudaStream_t s) {
    const int nslices = (A.nrows + SLICE - 1) / SLICE;
    const int blocks = (nslices + 7) / 8;
    ell_spmv_kernel<T><<<blocks, 256, 0, s>>>(A, x, y, (T)alpha, (T)beta);
    MP_CHECK_LAUNCH();
    return MP_OK;
}
template int ell_spmv<double>(const EllView<double> &, const double *, double *, double, double,
                              cudaStream_t);
template int ell_spmv<float>(const EllView<float> &, const float *, float *, double, double,
                             cudaStream_t);

// y_k = A_k x for up to 4 operators with one column structure
template <class T, int NOPS>
__global__ void __launch_bounds__(256)
    ell_spmv_multi_kernel(int nrows, int K, const int *__restrict__ cols, MultiVals<T> V,
                          const T *__restrict__ x, MultiOut<T> Y) {
    using V2 = typename Vec2<T>::type;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int nslices = (nrows + SLICE - 1) / SLICE;
    if (warp >= nslices)
        return;
    const size_t base = (size_t)warp * K * SLICE + 2 * lane;
    T a0[NOPS], a1[NOPS];
#pragma unroll
    for (int q = 0; q < NOPS; q++)
        a0[q] = a1[q] = 0;
#pragma unroll 2
    for (int k = 0; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        const int2 c = __ldcs(reinterpret_cast<const int2 *>(cols + o));
        const T x0 = __ldg(x + c.x), x1 = __ldg(x + c.y);
#pragma unroll
        for (int q = 0; q < NOPS; q++) {
            const V2 v = __ldcs(reinterpret_cast<const V2 *>(V.v[q] + o));
            a0[q] = fma(v.x, x0, a0[q]);
            a1[q] = fma(v.y, x1, a1[q]);
        }
    }
    const int r0 = warp * SLICE + 2 * lane;
#pragma unroll
    for (int q = 0; q < NOPS; q++) {
        if (r0 < nrows)
            Y.y[q][r0] = a0[q];
        if (r0 + 1 < nrows)
            Y.y[q][r0 + 1] = a1[q];
    }
}

template <class T>
int ell_spmv_multi(int nops, int nrows, int K, const int *cols, const MultiVals<T> &V, const T *x,
                   const MultiOut<T> &Y, cudaStream_t s) {
    const int blocks = ((nrows + SLICE - 1) / SLICE + 7) / 8;
    switch (nops) {
    case 1: ell_spmv_multi_kernel<T, 1><<<blocks, 256, 0, s>>>(nrows, K, cols, V, x, Y); break;
    case 2: ell_spmv_multi_kernel<T, 2><<<blocks, 256, 0, s>>>(nrows, K, cols, V, x, Y); break;
    case 3: ell_spmv_multi_kernel<T, 3><<<blocks, 256, 0, s>>>(nrows, K, cols, V, x, Y); break;
    case 4: ell_spmv_multi_kernel<T, 4><<<blocks, 256, 0, s>>>(nrows, K, cols, V, x, Y); break;
    default: return fail(MP_BAD_ARG, "mp_op_apply_multi: 1..4 operators, got %d", nops);
    }
    MP_CHECK_LAUNCH();
    return MP_OK;
}
template int ell_spmv_multi<double>(int, int, int, const int *, const MultiVals<double> &,
                                    const double *, const MultiOut<double> &, cudaStream_t);
template int ell_spmv_multi<float>(int, int, int, const int *, const MultiVals<float> &,
                                   const float *, const MultiOut<float> &, cudaStream_t);

}  // namespace mp

using namespace mp;

struct mp_op_s {
    Ell E;
    int precision = MP_FP64;
    std::shared_ptr<Ell> shared_cols;  // operators built from a cloud share its index slices
    const int *cols() const { return shared_cols ? shared_cols->cols.p : E.cols.p; }
};

namespace mp {
int op_view64(mp_op op, EllView<double> *view) {
    if (!op || op->precision != MP_FP64 || !op->E.v64.p)
        return fail(MP_BAD_ARG, "an FP64 operator is required");
    *view = EllView<double>{op->E.nrows, op->E.ncols, op->E.K, op->cols(), op->E.v64.p, nullptr};
    return MP_OK;
}
}  // namespace mp

extern "C" int mp_op_create_ell(int nrows, int ncols, int width, const int *cols,
                                const double *vals, int precision, mp_op *out) {
    if (!out || !cols || !vals)
        return fail(MP_BAD_ARG, "mp_op_create_ell: null argument");
    if (precision != MP_FP64 && precision != MP_FP32)
        return fail(MP_BAD_ARG, "precision must be MP_FP64 or MP_FP32");
    mp_op o = new mp_op_s;
    o->precision = precision;
    int st = ell_create(o->E, nrows, ncols, width, cols, vals, precision == MP_FP32, 0);
    if (st != MP_OK) {
        delete o;
        return st;
    }
    if (precision == MP_FP32)
        o->E.v64.release();
    MP_CUDA(cudaStreamSynchronize(0));
    *out = o;
    return MP_OK;
}

extern "C" int mp_op_from_cloud(mp_cloud c, int which, int rows, int precision, mp_op *out) {
    if (!c || !out)
        return fail(MP_BAD_ARG, "mp_op_from_cloud: null argument");
    if (precision != MP_FP64 && precision != MP_FP32)
        return fail(MP_BAD_ARG, "precision must be MP_FP64 or MP_FP32");
    const Ell *src = cloud_operator(c, which);
    if (!src)
        return fail(MP_BAD_ARG, "operator %d not available for this cloud", which);
    mp_op o = new mp_op_s;
    o->precision = precision;
    o->shared_cols = cloud_cols(c);
    o->E.nrows = src->nrows;
    o->E.ncols = src->ncols;
    o->E.K = src->K;
    const size_t tot = (size_t)ell_padded_rows(src->nrows) * src->K;
    int st = o->E.v64.alloc(tot);
    if (st == MP_OK)
        st = cloud_masked_copy(c, which, rows, o->E.v64.p, 0);
    if (st == MP_OK && precision == MP_FP32) {
        st = ell_make_fp32(o->E, 0);
        o->E.v64.release();
    }
    if (st == MP_OK)
        st = cudaStreamSynchronize(0) == cudaSuccess ? MP_OK : fail(MP_CUDA_ERROR, "sync failed");
    if (st != MP_OK) {
        delete o;
        return st;
    }
    *out = o;
    return MP_OK;
}

extern "C" int mp_op_info(mp_op op, int *nrows, int *ncols, int *width, int *precision) {
    if (!op)
        return fail(MP_BAD_ARG, "null operator");
    if (nrows)
        *nrows = op->E.nrows;
    if (ncols)
        *ncols = op->E.ncols;
    if (width)
        *width = op->E.K;
    if (precision)
        *precision = op->precision;
    return MP_OK;
}

template <class T>
static int op_apply_t(mp_op op, const void *x, void *y, double alpha, double beta, cudaStream_t s) {
    const T *dx = nullptr;
    dbuf<T> tx, ty;
    MP_TRY(stage_in((const T *)x, (size_t)op->E.ncols, tx, &dx, s));
    T *dy = (T *)y;
    bool host_y = !is_device_ptr(y);
    if (host_y) {
        MP_TRY(ty.alloc(op->E.nrows));
        if (beta != 0.0)
            MP_CUDA(cudaMemcpyAsync(ty.p, y, sizeof(T) * op->E.nrows, cudaMemcpyHostToDevice, s));
        dy = ty.p;
    }
    EllView<T> A{op->E.nrows, op->E.ncols, op->E.K, op->cols(),
                 std::is_same<T, double>::value ? (const T *)op->E.v64.p : (const T *)op->E.v32.p,
                 nullptr};
    MP_TRY(ell_spmv<T>(A, dx, dy, alpha, beta, s));
    if (host_y) {
        MP_CUDA(cudaMemcpyAsync(y, dy, sizeof(T) * op->E.nrows, cudaMemcpyDeviceToHost, s));
        MP_CUDA(cudaStreamSynchronize(s));
    } else if (tx.p) {
        MP_CUDA(cudaStreamSynchronize(s));
    }
    return MP_OK;
}

extern "C" int mp_op_apply(mp_op op, const void *x, void *y, double alpha, double beta,
                           mp_stream s) {
    if (!op || !x || !y)
        return fail(MP_BAD_ARG, "mp_op_apply: null argument");
    if (op->precision == MP_FP64)
        return op_apply_t<double>(op, x, y, alpha, beta, S(s));
    return op_apply_t<float>(op, x, y, alpha, beta, S(s));
}

extern "C" int mp_op_apply_multi(int nops, const mp_op *ops, const void *x, void *const *ys,
                                 mp_stream s) {
    if (nops < 1 || nops > 4 || !ops || !x || !ys)
        return fail(MP_BAD_ARG, "mp_op_apply_multi: 1..4 operators");
    const mp_op o0 = ops[0];
    for (int q = 0; q < nops; q++) {
        if (!ops[q] || ops[q]->cols() != o0->cols() || ops[q]->precision != o0->precision)
            return fail(MP_BAD_ARG, "mp_op_apply_multi: operators must share one stencil structure "
                                    "and precision (build them from the same cloud)");
        if (!is_device_ptr(ys[q]))
            return fail(MP_BAD_ARG, "mp_op_apply_multi: outputs must be device arrays");
    }
    if (!is_device_ptr(x))
        return fail(MP_BAD_ARG, "mp_op_apply_multi: x must be a device array");
    cudaStream_t st = S(s);
    if (o0->precision == MP_FP64) {
        MultiVals<double> V{};
        MultiOut<double> Y{};
        for (int q = 0; q < nops; q++) {
            V.v[q] = ops[q]->E.v64.p;
            Y.y[q] = (double *)ys[q];
        }
        return ell_spmv_multi<double>(nops, o0->E.nrows, o0->E.K, o0->cols(), V,
                                      (const double *)x, Y, st);
    }
    MultiVals<float> V{};
    MultiOut<float> Y{};
    for (int q = 0; q < nops; q++) {
        V.v[q] = ops[q]->E.v32.p;
        Y.y[q] = (float *)ys[q];
    }
    return ell_spmv_multi<float>(nops, o0->E.nrows, o0->E.K, o0->cols(), V, (const float *)x, Y,
                                 st);
}

extern "C" int mp_op_destroy(mp_op op) {
    delete op;
    return MP_OK;
}
