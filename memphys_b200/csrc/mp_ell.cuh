// mp_ell.cuh -- fixed-width sparse operators in 64-row slices.
//
// Every MeMPhyS operator row has exactly n entries (its stencil, cloud.cpp:627,644),
// so the natural layout is ELL with width K = n.  Rows are grouped in slices of
// 64; inside a slice entry k of all 64 rows is contiguous:
//     idx(row, k) = (row / 64) * K * 64 + k * 64 + (row % 64)
// One warp owns a slice and each lane two adjacent rows, so every load is a
// 16-byte (FP64 pair) or 8-byte (FP32 pair / int pair) vector and a warp reads
// 512 contiguous bytes of values and 256 of indices per stencil entry.  Padded
// rows point at column 0 with value 0.
#pragma once
#include <memory>
#include "mp_common.cuh"

namespace mp {

constexpr int SLICE = 64;

__host__ __device__ inline size_t ell_index(int row, int k, int K) {
    return (size_t)(row / SLICE) * K * SLICE + (size_t)k * SLICE + (row % SLICE);
}

__host__ __device__ inline int ell_padded_rows(int nrows) { return (nrows + SLICE - 1) / SLICE * SLICE; }

// Device ELL matrix (non-owning view).  With soff == nullptr every slice has
// width K; otherwise slice s spans entries [soff[s], soff[s+1]) of width
// soff[s+1] - soff[s] (sliced ELL with a width per 64-row slice, used for the
// multigrid operators whose row lengths vary).
template <class T> struct EllView {
    int nrows, ncols, K;
    const int *cols;
    const T *vals;
    const int *soff;
    // FP32 operators may also carry (column, value bits) pairs in the same sliced
    // order: one 16-byte load then fetches both entries of a lane's two rows
    const int2 *pk = nullptr;
    // FP64 operators may also carry 16-bit column deltas (column - row) in the same
    // sliced order, used in the slices whose flag dslice[s] is set (every delta of the
    // slice fits): 2 bytes instead of 4 per entry on the index stream
    const short *dcols = nullptr;
    const unsigned char *dslice = nullptr;
    // FP32 operators of uniform width may also carry entries k and k + 1 of a lane's
    // two rows side by side, values in one float4 (row 0 k, row 1 k, row 0 k+1,
    // row 1 k+1) and their 16-bit column deltas in one short4 of the same order, at
    // qv/qd[(slice * ceil(K/2) + k/2) * 32 + lane], used in the slices whose flag
    // qslice[s] is set: 6 instead of 8 bytes per entry, two loads per two entries
    const float4 *qv = nullptr;
    const short4 *qd = nullptr;
    const unsigned char *qslice = nullptr;
};

// start offset and width of slice w
template <class T>
__device__ __forceinline__ void slice_span(const EllView<T> &A, int w, size_t &base, int &K) {
    if (A.soff) {
        const int o0 = A.soff[w], o1 = A.soff[w + 1];
        base = (size_t)o0 * SLICE;
        K = o1 - o0;
    } else {
        base = (size_t)w * A.K * SLICE;
        K = A.K;
    }
}

// Owning ELL storage
struct Ell {
    int nrows = 0, ncols = 0, K = 0;  // K: uniform width, or the widest slice when soff is set
    dbuf<int> cols;
    dbuf<double> v64;
    dbuf<float> v32;
    dbuf<int> soff;
    dbuf<short> dcols;             // 16-bit column deltas (ell_make_deltas)
    dbuf<unsigned char> dslice;    // per slice: 1 when its deltas are used
    size_t entries() const { return v64.p ? v64.n : (v32.p ? v32.n : cols.n); }
    EllView<double> view64() const {
        return {nrows, ncols, K, cols.p, v64.p, soff.p, nullptr, dcols.p, dslice.p};
    }
    EllView<float> view32() const { return {nrows, ncols, K, cols.p, v32.p, soff.p}; }
};

// Build an Ell from row-major host or device arrays (copied).
int ell_create(Ell &E, int nrows, int ncols, int K, const int *cols, const double *vals,
               bool fp32, cudaStream_t s);
// Convert existing FP64 values to an FP32 copy on the device.
int ell_make_fp32(Ell &E, cudaStream_t s);
// 16-bit column deltas of a uniform-width operator, per slice where all of them fit
// (stencils are local in a node-ordered cloud; slices that reach far nodes, such as
// boundary nodes numbered last, keep their 32-bit columns).  Returns the fraction of
// slices that use deltas in *frac (nullable).
int ell_make_deltas(Ell &E, cudaStream_t s, double *frac = nullptr);
// Entries 1..K-1 of every row of a uniform-width FP64 operator in ascending column
// order (entry 0, a stencil's own node, stays first; widths above 64 are left as
// they are).  Consecutive rows then gather their k-th neighbours at nearly the same
// offset, and a warp's gather of entry k touches fewer cache lines.
int ell_sort_rows(Ell &E, cudaStream_t s);

// up to 4 value arrays sharing one column structure (mp_op_apply_multi)
template <class T> struct MultiVals {
    const T *v[4];
};
template <class T> struct MultiOut {
    T *y[4];
};

// y = alpha * A x + beta * y
template <class T>
int ell_spmv(const EllView<T> &A, const T *x, T *y, double alpha, double beta, cudaStream_t s);

template <class T>
int ell_spmv_multi(int nops, int nrows, int K, const int *cols, const MultiVals<T> &V, const T *x,
                   const MultiOut<T> &Y, cudaStream_t s);

}  // namespace mp
