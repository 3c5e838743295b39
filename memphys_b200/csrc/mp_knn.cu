// mp_knn.cu -- stencil selection on the GPU (replaces CLOUD::calc_cloud_points_fast,
// cloud.cpp:570-648, which queries two nanoflann KD-trees on the host).
//
// Rule (cloud.cpp:617-646): an interior node's stencil is its n nearest nodes of
// the whole cloud (itself first, at distance 0); a boundary node's stencil is the
// node itself followed by its n-1 nearest INTERIOR nodes (the reference places
// boundary nodes at infinity in the second tree, :596-601).  Neighbours are in
// ascending distance, ties broken by node index.
//
// Method: points are bucketed on a uniform grid (about two per cell) by a radix
// sort of their cell ids; each query thread scans square/cubic shells of cells
// of growing radius, keeping the best candidates in a sorted list, and stops
// once the k-th distance is within the radius already covered.  This is an
// exact search, so it selects the same stencils as the KD-tree.
#include <cub/cub.cuh>
#include <climits>
#include <cmath>
#include <mutex>
#include "mp_common.cuh"

namespace mp {

constexpr int KNN_MAX = 64;

struct Grid {
    double lo[3];
    double cell;
    int g[3];
};

__global__ void knn_cell_ids(const double *xyz, int nv, int dim, Grid G, unsigned int *cid,
                             int *idx) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    unsigned int c = 0;
    for (int d = dim - 1; d >= 0; d--) {
        int k = (int)((xyz[(size_t)i * dim + d] - G.lo[d]) / G.cell);
        k = k < 0 ? 0 : (k >= G.g[d] ? G.g[d] - 1 : k);
        c = c * G.g[d] + k;
    }
    cid[i] = c;
    idx[i] = i;
}

__global__ void knn_cell_ranges(const unsigned int *cid_sorted, int nv, int *start, int *end) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    unsigned int c = cid_sorted[i];
    if (i == 0 || cid_sorted[i - 1] != c)
        start[c] = i;
    if (i == nv - 1 || cid_sorted[i + 1] != c)
        end[c] = i + 1;
}

// Stencil queries (probe == nullptr: query q is node q, boundary rule applied) or
// probe queries (query q at probe[q], its n nearest nodes of the whole cloud, as
// calc_cloud_points_slow for probes does, coefficient_computations.cpp:373-428).
__global__ void __launch_bounds__(128)
    knn_query(const double *xyz, const uint8_t *bflag, int nv, int dim, int n, Grid G,
              const int *order, const int *start, const int *end, int *nb_col, int *failed,
              const double *probe, int nq) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (probe ? nq : nv))
        return;
    double bd[KNN_MAX];
    int bi[KNN_MAX];
    const bool isb = !probe && bflag[q] != 0;
    const int want = isb ? n - 1 : n;
    double xq[3] = {0, 0, 0};
    int qc[3] = {0, 0, 0};
    bool inside = true;  // a query outside the grid scans until the grid is covered
    for (int d = 0; d < dim; d++) {
        xq[d] = probe ? probe[(size_t)q * dim + d] : xyz[(size_t)q * dim + d];
        const double t = (xq[d] - G.lo[d]) / G.cell;
        if (!(t >= 0.0 && t <= (double)G.g[d]))
            inside = false;
        int k = (int)t;
        qc[d] = t < 0 ? 0 : (k >= G.g[d] ? G.g[d] - 1 : k);
    }
    int cnt = 0;
    for (int R = 0;; R++) {
        int zlo = dim == 3 ? qc[2] - R : 0, zhi = dim == 3 ? qc[2] + R : 0;
        for (int cz = zlo; cz <= zhi; cz++)
            for (int cy = qc[1] - R; cy <= qc[1] + R; cy++)
                for (int cx = qc[0] - R; cx <= qc[0] + R; cx++) {
                    bool shell = cx == qc[0] - R || cx == qc[0] + R || cy == qc[1] - R ||
                                 cy == qc[1] + R || (dim == 3 && (cz == zlo || cz == zhi));
                    if (!shell)
                        continue;
                    if (cx < 0 || cx >= G.g[0] || cy < 0 || cy >= G.g[1] || cz < 0 || cz >= G.g[2])
                        continue;
                    unsigned int c = ((unsigned)cz * G.g[1] + cy) * G.g[0] + cx;
                    int s0 = start[c], s1 = end[c];
                    for (int t = s0; t < s1; t++) {
                        int j = order[t];
                        if (isb && bflag[j])
                            continue;
                        double dd = 0.0;
                        for (int d = 0; d < dim; d++) {
                            double df = xyz[(size_t)j * dim + d] - xq[d];
                            dd += df * df;
                        }
                        if (cnt == want &&
                            (dd > bd[want - 1] || (dd == bd[want - 1] && j > bi[want - 1])))
                            continue;
                        int pos = cnt < want ? cnt++ : want - 1;
                        while (pos > 0 && (bd[pos - 1] > dd || (bd[pos - 1] == dd && bi[pos - 1] > j))) {
                            bd[pos] = bd[pos - 1];
                            bi[pos] = bi[pos - 1];
                            pos--;
                        }
                        bd[pos] = dd;
                        bi[pos] = j;
                    }
                }
        double reach = R * G.cell;
        bool covered = true;
        for (int d = 0; d < dim; d++)
            if (qc[d] - R > 0 || qc[d] + R < G.g[d] - 1)
                covered = false;
        if (inside && cnt == want && bd[want - 1] <= reach * reach)
            break;
        if (covered)
            break;
    }
    int *out = nb_col + (size_t)q * n;
    if (cnt < want) {
        atomicAdd(failed, 1);
        for (int k = 0; k < n; k++)
            out[k] = q;
        return;
    }
    if (isb) {
        out[0] = q;
        for (int k = 0; k < n - 1; k++)
            out[k + 1] = bi[k];
    } else {
        for (int k = 0; k < n; k++)
            out[k] = bi[k];
    }
}

// probe == nullptr: the stencils of the nodes; else the n nearest nodes of each of
// the np probes
static int knn_run(const double *d_xyz, const uint8_t *d_bflag, int nv, int dim, int n, int *d_nb,
                   const double *d_probe, int np, cudaStream_t s);

int knn_device(const double *d_xyz, const uint8_t *d_bflag, int nv, int dim, int n, int *d_nb,
               cudaStream_t s) {
    return knn_run(d_xyz, d_bflag, nv, dim, n, d_nb, nullptr, 0, s);
}

int knn_probe_device(const double *d_xyz, int nv, int dim, const double *d_probe, int np, int n,
                     int *d_nb, cudaStream_t s) {
    if (np <= 0 || n > nv)
        return fail(MP_BAD_ARG, "probe kNN: np=%d, n=%d of %d nodes", np, n, nv);
    return knn_run(d_xyz, nullptr, nv, dim, n, d_nb, d_probe, np, s);
}

static int knn_run(const double *d_xyz, const uint8_t *d_bflag, int nv, int dim, int n, int *d_nb,
                   const double *d_probe, int np, cudaStream_t s) {
    if (nv <= 0 || (dim != 2 && dim != 3) || n < (d_probe ? 1 : 2) || n > KNN_MAX)
        return fail(MP_BAD_ARG, "mp_knn_stencils: nv=%d dim=%d n=%d (n must be 2..%d)", nv, dim, n,
                    KNN_MAX);
    // bounding box on the host (one small copy; setup path)
    std::vector<double> h((size_t)nv * dim);
    MP_CUDA(cudaMemcpyAsync(h.data(), d_xyz, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    Grid G;
    double hi[3] = {0, 0, 0};
    for (int d = 0; d < 3; d++)
        G.lo[d] = 0.0, G.g[d] = 1;
    for (int d = 0; d < dim; d++)
        G.lo[d] = hi[d] = h[d];
    for (int i = 0; i < nv; i++)
        for (int d = 0; d < dim; d++) {
            double v = h[(size_t)i * dim + d];
            if (!std::isfinite(v))
                return fail(MP_BAD_ARG, "node %d has a non-finite coordinate", i);
            G.lo[d] = v < G.lo[d] ? v : G.lo[d];
            hi[d] = v > hi[d] ? v : hi[d];
        }
    double vol = 1.0;
    for (int d = 0; d < dim; d++)
        vol *= (hi[d] - G.lo[d]) > 0 ? (hi[d] - G.lo[d]) : 1.0;
    G.cell = std::pow(vol * 2.0 / nv, 1.0 / dim);
    long long ncell = 1;
    for (int d = 0; d < dim; d++) {
        G.g[d] = (int)((hi[d] - G.lo[d]) / G.cell) + 1;
        ncell *= G.g[d];
    }
    if (ncell > (1ll << 31))
        return fail(MP_BAD_ARG, "kNN grid too large (%lld cells)", ncell);
    dbuf<unsigned int> cid, cid2;
    dbuf<int> idx, idx2, st, en, failed;
    MP_TRY(cid.alloc(nv));
    MP_TRY(cid2.alloc(nv));
    MP_TRY(idx.alloc(nv));
    MP_TRY(idx2.alloc(nv));
    MP_TRY(st.alloc(ncell));
    MP_TRY(en.alloc(ncell));
    MP_TRY(failed.alloc(1));
    MP_CUDA(cudaMemsetAsync(st.p, 0, sizeof(int) * ncell, s));
    MP_CUDA(cudaMemsetAsync(en.p, 0, sizeof(int) * ncell, s));
    MP_CUDA(cudaMemsetAsync(failed.p, 0, sizeof(int), s));
    const int tb = 256, nb = (nv + tb - 1) / tb;
    knn_cell_ids<<<nb, tb, 0, s>>>(d_xyz, nv, dim, G, cid.p, idx.p);
    MP_CHECK_LAUNCH();
    size_t tmp_bytes = 0;
    int bits = 1;
    while ((1ll << bits) < ncell)
        bits++;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, cid.p, cid2.p, idx.p, idx2.p, nv, 0, bits, s);
    dbuf<char> tmp;
    MP_TRY(tmp.alloc(tmp_bytes));
    MP_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, cid.p, cid2.p, idx.p, idx2.p, nv, 0,
                                            bits, s));
    count_launch();
    knn_cell_ranges<<<nb, tb, 0, s>>>(cid2.p, nv, st.p, en.p);
    MP_CHECK_LAUNCH();
    const int nq = d_probe ? np : nv;
    knn_query<<<(nq + 127) / 128, 128, 0, s>>>(d_xyz, d_bflag, nv, dim, n, G, idx2.p, st.p, en.p,
                                                d_nb, failed.p, d_probe, np);
    MP_CHECK_LAUNCH();
    int bad = 0;
    MP_CUDA(cudaMemcpyAsync(&bad, failed.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (bad)
        return fail(MP_KNN_FAILED, "%d nodes found fewer than %d stencil candidates", bad, n);
    return MP_OK;
}

}  // namespace mp

using namespace mp;

extern "C" int mp_knn_stencils(const double *xyz, const uint8_t *boundary, int nv, int dim, int n,
                               int *nb_col, mp_stream s) {
    if (!xyz || !boundary || !nb_col)
        return fail(MP_BAD_ARG, "mp_knn_stencils: null argument");
    cudaStream_t st = S(s);
    dbuf<double> tx;
    dbuf<uint8_t> tb;
    const double *dx = nullptr;
    const uint8_t *db = nullptr;
    MP_TRY(stage_in(xyz, (size_t)nv * dim, tx, &dx, st));
    MP_TRY(stage_in(boundary, (size_t)nv, tb, &db, st));
    int *dn = nb_col;
    dbuf<int> tn;
    bool host_out = !is_device_ptr(nb_col);
    if (host_out) {
        MP_TRY(tn.alloc((size_t)nv * n));
        dn = tn.p;
    }
    MP_TRY(knn_device(dx, db, nv, dim, n, dn, st));
    if (host_out) {
        MP_CUDA(cudaMemcpyAsync(nb_col, dn, sizeof(int) * nv * n, cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
    }
    return MP_OK;
}

// ------------------------------------------------ no-allocation variant
// mp_knn_stencils_noalloc runs the same grid + radix sort + query kernels with
// every work array carved from one fixed scratch array per device, so a call
// allocates and frees no device memory.
namespace mp {

constexpr size_t KNN_SCRATCH_BYTES = (size_t)4 << 20;  // 4 MiB: ~140,000 nodes in 2D
static __device__ __align__(256) unsigned char g_knn_scratch[KNN_SCRATCH_BYTES];

constexpr int KNN_SCRATCH_DEVICES = 64;
static std::mutex g_knn_scratch_mu;
static unsigned char *g_knn_scratch_ptr[KNN_SCRATCH_DEVICES];

// device address of the current device's scratch, looked up once per device
static int knn_scratch(unsigned char **out) {
    int dev = 0;
    MP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= KNN_SCRATCH_DEVICES)
        return fail(MP_BAD_ARG, "device %d beyond the %d supported", dev, KNN_SCRATCH_DEVICES);
    std::lock_guard<std::mutex> lock(g_knn_scratch_mu);
    if (!g_knn_scratch_ptr[dev]) {
        unsigned char *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_knn_scratch);
        if (e != cudaSuccess || !p)
            return fail(MP_CUDA_ERROR, "cudaGetSymbolAddress(kNN scratch): %s",
                        cudaGetErrorString(e));
        g_knn_scratch_ptr[dev] = p;
    }
    *out = g_knn_scratch_ptr[dev];
    return MP_OK;
}

// bounding box lo[0..2], hi[0..2]; flags[0] = 0 (the query's failure count),
// flags[1] = lowest index of a node with a non-finite coordinate or INT_MAX; one block
__global__ void __launch_bounds__(256)
    knn_bbox(const double *xyz, int nv, int dim, double *box, int *flags) {
    __shared__ double slo[3][256], shi[3][256];
    __shared__ int sbad[256];
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    int first_bad = INT_MAX;
    for (int i = threadIdx.x; i < nv; i += blockDim.x)
        for (int d = 0; d < dim; d++) {
            const double v = xyz[(size_t)i * dim + d];
            if (!isfinite(v)) {
                first_bad = min(first_bad, i);
                continue;
            }
            lo[d] = fmin(lo[d], v);
            hi[d] = fmax(hi[d], v);
        }
    for (int d = 0; d < 3; d++) {
        slo[d][threadIdx.x] = lo[d];
        shi[d][threadIdx.x] = hi[d];
    }
    sbad[threadIdx.x] = first_bad;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            for (int d = 0; d < 3; d++) {
                slo[d][threadIdx.x] = fmin(slo[d][threadIdx.x], slo[d][threadIdx.x + w]);
                shi[d][threadIdx.x] = fmax(shi[d][threadIdx.x], shi[d][threadIdx.x + w]);
            }
            sbad[threadIdx.x] = min(sbad[threadIdx.x], sbad[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        for (int d = 0; d < 3; d++) {
            box[d] = slo[d][0];
            box[3 + d] = shi[d][0];
        }
        flags[0] = 0;
        flags[1] = sbad[0];
    }
}

// offsets of the work arrays inside the scratch (each 256-byte aligned)
struct KnnCarve {
    size_t off = 0;
    size_t take(size_t bytes) {
        const size_t o = off;
        off = (off + bytes + 255) / 256 * 256;
        return o;
    }
};

}  // namespace mp

extern "C" int mp_knn_stencils_noalloc(const double *xyz, const uint8_t *boundary, int nv, int dim,
                                       int n, int *nb_col, mp_stream s) {
    if (!xyz || !boundary || !nb_col)
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc: null argument");
    if (nv <= 0 || (dim != 2 && dim != 3) || n < 2 || n > KNN_MAX)
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc: nv=%d dim=%d n=%d (n must be 2..%d)", nv,
                    dim, n, KNN_MAX);
    if (!is_device_ptr(xyz) || !is_device_ptr(boundary) || !is_device_ptr(nb_col))
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc takes device pointers only (staging host "
                                "arrays would allocate); use mp_knn_stencils for host arrays");
    // the scratch and the launches belong to the current device
    if (!is_current_device_ptr(xyz) || !is_current_device_ptr(boundary) ||
        !is_current_device_ptr(nb_col))
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc: the arrays must live on the current "
                                "device (mp_set_device)");
    // the four per-node arrays alone must fit before anything runs
    if ((size_t)nv * 16 + 4096 > KNN_SCRATCH_BYTES)
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc: %d nodes exceed its %zu-byte scratch "
                                "(at most about 140000 nodes in 2D); use mp_knn_stencils", nv,
                    KNN_SCRATCH_BYTES);
    unsigned char *base = nullptr;
    MP_TRY(knn_scratch(&base));
    cudaStream_t st = S(s);
    KnnCarve cv;
    double *box = (double *)(base + cv.take(6 * sizeof(double)));
    int *flags = (int *)(base + cv.take(2 * sizeof(int)));  // [0] failed queries, [1] first non-finite
    // bounding box on the device (it also clears the flags); six numbers come back to the host
    knn_bbox<<<1, 256, 0, st>>>(xyz, nv, dim, box, flags);
    MP_CHECK_LAUNCH();
    double hb[6];
    int hf[2];
    MP_CUDA(cudaMemcpyAsync(hb, box, sizeof(hb), cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (hf[1] != INT_MAX)
        return fail(MP_BAD_ARG, "node %d has a non-finite coordinate", hf[1]);
    Grid G;
    double hi[3] = {0, 0, 0};
    for (int d = 0; d < 3; d++)
        G.lo[d] = 0.0, G.g[d] = 1;
    for (int d = 0; d < dim; d++) {
        G.lo[d] = hb[d];
        hi[d] = hb[3 + d];
    }
    double vol = 1.0;
    for (int d = 0; d < dim; d++)
        vol *= (hi[d] - G.lo[d]) > 0 ? (hi[d] - G.lo[d]) : 1.0;
    G.cell = std::pow(vol * 2.0 / nv, 1.0 / dim);
    long long ncell = 1;
    for (int d = 0; d < dim; d++) {
        G.g[d] = (int)((hi[d] - G.lo[d]) / G.cell) + 1;
        ncell *= G.g[d];
    }
    if (ncell > (1ll << 31))
        return fail(MP_BAD_ARG, "kNN grid too large (%lld cells)", ncell);
    int bits = 1;
    while ((1ll << bits) < ncell)
        bits++;
    const size_t o_cid = cv.take(sizeof(unsigned) * nv), o_cid2 = cv.take(sizeof(unsigned) * nv);
    const size_t o_idx = cv.take(sizeof(int) * nv), o_idx2 = cv.take(sizeof(int) * nv);
    const size_t o_st = cv.take(sizeof(int) * ncell), o_en = cv.take(sizeof(int) * ncell);
    unsigned *cid = (unsigned *)(base + o_cid), *cid2 = (unsigned *)(base + o_cid2);
    int *idx = (int *)(base + o_idx), *idx2 = (int *)(base + o_idx2);
    int *cst = (int *)(base + o_st), *cen = (int *)(base + o_en);
    size_t tmp_bytes = 0;  // a size query: no temporary storage is allocated
    MP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, cid, cid2, idx, idx2, nv, 0, bits,
                                            st));
    const size_t o_tmp = cv.take(tmp_bytes);
    if (cv.off > KNN_SCRATCH_BYTES)
        return fail(MP_BAD_ARG, "mp_knn_stencils_noalloc: %d nodes need %zu bytes of scratch, it "
                                "holds %zu; use mp_knn_stencils", nv, cv.off, KNN_SCRATCH_BYTES);
    MP_CUDA(cudaMemsetAsync(cst, 0, sizeof(int) * ncell, st));
    MP_CUDA(cudaMemsetAsync(cen, 0, sizeof(int) * ncell, st));
    const int tb = 256, nb = (nv + tb - 1) / tb;
    knn_cell_ids<<<nb, tb, 0, st>>>(xyz, nv, dim, G, cid, idx);
    MP_CHECK_LAUNCH();
    MP_CUDA(cub::DeviceRadixSort::SortPairs(base + o_tmp, tmp_bytes, cid, cid2, idx, idx2, nv, 0,
                                            bits, st));
    count_launch();
    knn_cell_ranges<<<nb, tb, 0, st>>>(cid2, nv, cst, cen);
    MP_CHECK_LAUNCH();
    knn_query<<<(nv + 127) / 128, 128, 0, st>>>(xyz, boundary, nv, dim, n, G, idx2, cst, cen,
                                                 nb_col, flags, nullptr, 0);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaMemcpyAsync(hf, flags, sizeof(int), cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (hf[0])
        return fail(MP_KNN_FAILED, "%d nodes found fewer than %d stencil candidates", hf[0], n);
    return MP_OK;
}

// the n nearest nodes of each probe point, ascending distance, ties by index
extern "C" int mp_knn_probe(const double *xyz, int nv, int dim, const double *probe, int np, int n,
                            int *cols, mp_stream s) {
    if (!xyz || !probe || !cols || np <= 0)
        return fail(MP_BAD_ARG, "mp_knn_probe: bad arguments");
    cudaStream_t st = S(s);
    dbuf<double> tx, tp;
    dbuf<int> tc;
    const double *dx = nullptr, *dp = nullptr;
    MP_TRY(stage_in(xyz, (size_t)nv * dim, tx, &dx, st));
    MP_TRY(stage_in(probe, (size_t)np * dim, tp, &dp, st));
    int *dc = cols;
    const bool host_out = !is_device_ptr(cols);
    if (host_out) {
        MP_TRY(tc.alloc((size_t)np * n));
        dc = tc.p;
    }
    MP_TRY(knn_probe_device(dx, nv, dim, dp, np, n, dc, st));
    if (host_out) {
        MP_CUDA(cudaMemcpyAsync(cols, dc, sizeof(int) * np * n, cudaMemcpyDeviceToHost, st));
        MP_CUDA(cudaStreamSynchronize(st));
    }
    return MP_OK;
}
