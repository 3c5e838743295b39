// mp_order.cu -- node orderings of a cloud and their application.
//
// CLOUD::CLOUD renumbers every cloud by reverse Cuthill-McKee on the stencil
// graph (cloud.cpp:37, re_order_points_reverse_cuthill_mckee :315-335,
// reverse_cuthill_mckee_ordering general_functions.cpp:806-879) and then
// permutes the points and the stencils (re_order_points, cloud.cpp:337-439).
//  * mp_order_rcm restates that ordering exactly (a breadth-first search is
//    sequential: host code).
//  * mp_order_morton is the GPU ordering: Z-order of the coordinates
//    quantised on the bounding box (16 bits per axis in 2D, 21 in 3D),
//    sorted by a radix sort, ties in index order.  It keeps stencil members
//    close in memory like RCM does, without the sequential search.
//  * mp_permute_stencils applies an ordering to a stencil table the way
//    re_order_points does: row order[i] holds row i with every member mapped.
#include <algorithm>
#include <cub/cub.cuh>
#include <vector>
#include "mp_common.cuh"

namespace mp {

// 16 / 21 bits of x spread to every 2nd / 3rd bit
__device__ __forceinline__ uint64_t spread2(uint64_t x) {
    x &= 0xFFFFull;
    x = (x | (x << 8)) & 0x00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0Full;
    x = (x | (x << 2)) & 0x33333333ull;
    x = (x | (x << 1)) & 0x55555555ull;
    return x;
}

__device__ __forceinline__ uint64_t spread3(uint64_t x) {
    x &= 0x1FFFFFull;
    x = (x | (x << 32)) & 0x1F00000000FFFFull;
    x = (x | (x << 16)) & 0x1F0000FF0000FFull;
    x = (x | (x << 8)) & 0x100F00F00F00F00Full;
    x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// per-axis minimum and maximum (one block; the cloud's bounding box)
__global__ void k_bbox(const double *xyz, int nv, int dim, double *box) {
    __shared__ double lo[3][256], hi[3][256];
    double l[3] = {1e300, 1e300, 1e300}, h[3] = {-1e300, -1e300, -1e300};
    for (int i = threadIdx.x; i < nv; i += blockDim.x)
        for (int d = 0; d < dim; d++) {
            const double v = xyz[(size_t)i * dim + d];
            l[d] = fmin(l[d], v);
            h[d] = fmax(h[d], v);
        }
    for (int d = 0; d < 3; d++) {
        lo[d][threadIdx.x] = l[d];
        hi[d][threadIdx.x] = h[d];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w /= 2) {
        if ((int)threadIdx.x < w)
            for (int d = 0; d < 3; d++) {
                lo[d][threadIdx.x] = fmin(lo[d][threadIdx.x], lo[d][threadIdx.x + w]);
                hi[d][threadIdx.x] = fmax(hi[d][threadIdx.x], hi[d][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int d = 0; d < dim; d++) {
            box[d] = lo[d][0];
            box[3 + d] = hi[d][0];
        }
}

__global__ void k_morton(const double *xyz, int nv, int dim, const double *box, uint64_t *key,
                         int *idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv)
        return;
    const int bits = dim == 3 ? 21 : 16;
    const double cells = (double)((1u << bits) - 1);
    uint64_t q[3] = {0, 0, 0};
    for (int d = 0; d < dim; d++) {
        const double ext = box[3 + d] - box[d];
        const double t = ext > 0 ? (xyz[(size_t)i * dim + d] - box[d]) / ext : 0.0;
        q[d] = (uint64_t)fmin(fmax(t * cells, 0.0), cells);
    }
    key[i] = dim == 3 ? (spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2))
                      : (spread2(q[0]) | (spread2(q[1]) << 1));
    idx[i] = i;
}

// order[sorted[r]] = r
__global__ void k_rank(const int *sorted, int nv, int *order) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < nv)
        order[sorted[r]] = r;
}

__global__ void k_permute_stencils(const int *nb, int nv, int n, const int *order, int *out,
                                   int *bad) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)nv * n)
        return;
    const int i = (int)(e / n), k = (int)(e % n);
    const int j = nb[e];
    const int oi = order[i];
    if (j < 0 || j >= nv || oi < 0 || oi >= nv) {
        atomicExch(bad, 1);
        return;
    }
    out[(size_t)oi * n + k] = order[j];
}

// out row order[i] = in row i (row_bytes bytes per row)
__global__ void k_permute_rows(const unsigned char *in, unsigned char *out, int nv, int row_bytes,
                               const int *order) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)nv * row_bytes)
        return;
    const int i = (int)(e / row_bytes), b = (int)(e % row_bytes);
    const int oi = order[i];
    if (oi >= 0 && oi < nv)
        out[(size_t)oi * row_bytes + b] = in[e];
}

}  // namespace mp

using namespace mp;

// cuthill_mckee_ordering (general_functions.cpp:806-869) + the reversal
// (:871-879): breadth-first from the first node of least degree, each node's
// unvisited neighbours appended in increasing (degree, index).  A graph that
// the search does not exhaust from that node (where the reference reads past
// its numbering) continues from the next unvisited node of least degree.
extern "C" int mp_order_rcm(const int *nb, int nv, int n, int *order) {
    if (!nb || !order || nv <= 0 || n <= 0)
        return fail(MP_BAD_ARG, "mp_order_rcm: bad arguments");
    std::vector<int> h((size_t)nv * n);
    if (is_device_ptr(nb))
        MP_CUDA(cudaMemcpy(h.data(), nb, sizeof(int) * h.size(), cudaMemcpyDeviceToHost));
    else
        std::copy(nb, nb + h.size(), h.begin());
    for (size_t e = 0; e < h.size(); e++)
        if (h[e] < 0 || h[e] >= nv)
            return fail(MP_BAD_ARG, "mp_order_rcm: stencil member %d out of range", h[e]);
    // every node's adjacency is its stencil row, so every degree is n; the
    // search keeps the general (degree, index) rule of the reference anyway
    std::vector<int> degree(nv, n), numbering;
    std::vector<char> visited(nv, 0);
    numbering.reserve(nv);
    std::vector<std::pair<int, int>> fresh;
    size_t head = 0;
    while ((int)numbering.size() < nv) {
        if (head == numbering.size()) {  // start (or restart) at the least degree
            int best = -1;
            for (int i = 0; i < nv; i++)
                if (!visited[i] && (best < 0 || degree[i] < degree[best]))
                    best = i;
            visited[best] = 1;
            numbering.push_back(best);
        }
        const int v = numbering[head++];
        fresh.clear();
        for (int k = 0; k < n; k++) {
            const int w = h[(size_t)v * n + k];
            if (!visited[w]) {
                visited[w] = 1;
                fresh.emplace_back(degree[w], w);
            }
        }
        std::sort(fresh.begin(), fresh.end());
        for (auto &f : fresh)
            numbering.push_back(f.second);
    }
    std::vector<int> ord(nv);
    for (int r = 0; r < nv; r++)
        ord[numbering[r]] = nv - r - 1;
    if (is_device_ptr(order))
        MP_CUDA(cudaMemcpy(order, ord.data(), sizeof(int) * nv, cudaMemcpyHostToDevice));
    else
        std::copy(ord.begin(), ord.end(), order);
    return MP_OK;
}

extern "C" int mp_order_morton(const double *xyz, int nv, int dim, int *order, mp_stream s) {
    if (!xyz || !order || nv <= 0 || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_order_morton: bad arguments");
    cudaStream_t st = S(s);
    dbuf<double> tx, box;
    const double *dx = nullptr;
    MP_TRY(stage_in(xyz, (size_t)nv * dim, tx, &dx, st));
    dbuf<uint64_t> key, key2;
    dbuf<int> idx, idx2, dord;
    MP_TRY(box.alloc(6));
    MP_TRY(key.alloc(nv));
    MP_TRY(key2.alloc(nv));
    MP_TRY(idx.alloc(nv));
    MP_TRY(idx2.alloc(nv));
    k_bbox<<<1, 256, 0, st>>>(dx, nv, dim, box.p);
    MP_CHECK_LAUNCH();
    const unsigned nb = (unsigned)((nv + 255) / 256);
    k_morton<<<nb, 256, 0, st>>>(dx, nv, dim, box.p, key.p, idx.p);
    MP_CHECK_LAUNCH();
    const int bits = dim == 3 ? 63 : 32;
    size_t tmp_bytes = 0;
    MP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, key.p, key2.p, idx.p, idx2.p, nv,
                                            0, bits, st));
    dbuf<unsigned char> tmp;
    MP_TRY(tmp.alloc(std::max<size_t>(tmp_bytes, 1)));
    MP_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, key.p, key2.p, idx.p, idx2.p, nv, 0,
                                            bits, st));
    int *out = order;
    const bool host_out = !is_device_ptr(order);
    if (host_out) {
        MP_TRY(dord.alloc(nv));
        out = dord.p;
    }
    k_rank<<<nb, 256, 0, st>>>(idx2.p, nv, out);
    MP_CHECK_LAUNCH();
    if (host_out)
        MP_CUDA(cudaMemcpyAsync(order, out, sizeof(int) * nv, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

extern "C" int mp_permute_stencils(const int *nb, int nv, int n, const int *order, int *nb_out,
                                   mp_stream s) {
    if (!nb || !order || !nb_out || nv <= 0 || n <= 0 || nb == nb_out)
        return fail(MP_BAD_ARG, "mp_permute_stencils: bad arguments");
    cudaStream_t st = S(s);
    dbuf<int> tn, to, tout, bad;
    const int *dn = nullptr, *dord = nullptr;
    MP_TRY(stage_in(nb, (size_t)nv * n, tn, &dn, st));
    MP_TRY(stage_in(order, (size_t)nv, to, &dord, st));
    int *dout = nb_out;
    const bool host_out = !is_device_ptr(nb_out);
    if (host_out) {
        MP_TRY(tout.alloc((size_t)nv * n));
        dout = tout.p;
    }
    MP_TRY(bad.alloc(1));
    MP_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    const size_t tot = (size_t)nv * n;
    k_permute_stencils<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(dn, nv, n, dord, dout, bad.p);
    MP_CHECK_LAUNCH();
    int hbad = 0;
    MP_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (host_out)
        MP_CUDA(cudaMemcpyAsync(nb_out, dout, sizeof(int) * tot, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    if (hbad)
        return fail(MP_BAD_ARG, "mp_permute_stencils: member or order entry out of range");
    return MP_OK;
}

extern "C" int mp_permute_rows(const void *in, void *out, int nv, int row_bytes, const int *order,
                               mp_stream s) {
    if (!in || !out || !order || nv <= 0 || row_bytes <= 0 || in == out)
        return fail(MP_BAD_ARG, "mp_permute_rows: bad arguments");
    cudaStream_t st = S(s);
    const size_t tot = (size_t)nv * row_bytes;
    dbuf<unsigned char> ti, tout;
    dbuf<int> to;
    const unsigned char *di = nullptr;
    const int *dord = nullptr;
    MP_TRY(stage_in((const unsigned char *)in, tot, ti, &di, st));
    MP_TRY(stage_in(order, (size_t)nv, to, &dord, st));
    unsigned char *dout = (unsigned char *)out;
    const bool host_out = !is_device_ptr(out);
    if (host_out) {
        MP_TRY(tout.alloc(tot));
        dout = tout.p;
    }
    k_permute_rows<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(di, dout, nv, row_bytes, dord);
    MP_CHECK_LAUNCH();
    if (host_out)
        MP_CUDA(cudaMemcpyAsync(out, dout, tot, cudaMemcpyDeviceToHost, st));
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}
