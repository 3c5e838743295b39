// mp_common.cuh -- shared helpers of libmemphys_cuda.so (sm_100a only).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "../../include/memphys.h"

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libmemphys_cuda targets sm_100a (B200) only"
#endif

namespace mp {

// ------------------------------------------------------------ error state
void set_error(const char *fmt, ...);
int fail(int status, const char *fmt, ...);
void count_launch(int n = 1);

#define MP_CUDA(call)                                                                        \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return ::mp::fail(MP_CUDA_ERROR, "%s failed: %s (%s:%d)", #call,                 \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                   \
    } while (0)

// Programmatic dependent launch (sm_90+): a kernel launched by launch_pdl may be
// scheduled while its predecessor in the stream is still draining, so its launch
// latency overlaps the predecessor's tail.  Such a kernel calls pdl_wait() before
// touching anything the predecessor wrote (it returns once that grid has
// completed and its writes are visible), and pdl_trigger() to let its own
// successor launch once all of its blocks are resident.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <class... KArgs, class... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t s,
                              Args... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
}

#define MP_CHECK_LAUNCH()                                                                    \
    do {                                                                                     \
        cudaError_t e_ = cudaGetLastError();                                                 \
        if (e_ != cudaSuccess)                                                               \
            return ::mp::fail(MP_CUDA_ERROR, "kernel launch failed: %s (%s:%d)",             \
                              cudaGetErrorString(e_), __FILE__, __LINE__);                   \
        ::mp::count_launch();                                                                \
    } while (0)

#define MP_TRY(expr)                                                                         \
    do {                                                                                     \
        int st_ = (expr);                                                                    \
        if (st_ != MP_OK)                                                                    \
            return st_;                                                                      \
    } while (0)

inline cudaStream_t S(mp_stream s) { return reinterpret_cast<cudaStream_t>(s); }

// number of SMs of the current device (cached per device)
int sm_count();

// true when p is device (or managed) memory
bool is_device_ptr(const void *p);
// true when p is memory of the current device (or managed memory)
bool is_current_device_ptr(const void *p);

// RAII device buffer (owned by handles)
template <class T> struct dbuf {
    T *p = nullptr;
    size_t n = 0;
    dbuf() = default;
    dbuf(const dbuf &) = delete;
    dbuf &operator=(const dbuf &) = delete;
    ~dbuf() { release(); }
    int alloc(size_t count) {
        release();
        if (count == 0)
            return MP_OK;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(MP_CUDA_ERROR, "cudaMalloc(%zu bytes): %s", count * sizeof(T),
                        cudaGetErrorString(e));
        }
        n = count;
        return MP_OK;
    }
    void release() {
        if (p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// Input view: device pointer used in place, host pointer staged into `tmp`.
template <class T>
int stage_in(const T *src, size_t count, dbuf<T> &tmp, const T **dev, cudaStream_t s) {
    if (count == 0 || src == nullptr) {
        *dev = src;
        return MP_OK;
    }
    if (is_device_ptr(src)) {
        *dev = src;
        return MP_OK;
    }
    MP_TRY(tmp.alloc(count));
    MP_CUDA(cudaMemcpyAsync(tmp.p, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
    *dev = tmp.p;
    return MP_OK;
}

// ------------------------------------------------------------ device side
template <class T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sum of NV values; result valid in thread 0.  smem >= 32*NV.
template <int NV, class T> __device__ __forceinline__ void block_sum(T (&v)[NV], T *smem) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; k++)
        v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; k++)
            smem[k * 32 + wid] = v[k];
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            T t = lane < nw ? smem[k * 32 + lane] : T(0);
            v[k] = warp_sum(t);
        }
    }
    __syncthreads();
}

// Deterministic grid reduction: every block writes NV partials; the last block
// to finish (atomic ticket) sums them in block order and returns true in all
// of its threads (result in out[] of thread 0).  ticket is reset for reuse.
template <int NV>
__device__ __forceinline__ bool grid_reduce(double (&v)[NV], double *partials,
                                            unsigned int *ticket, double *smem) {
    block_sum<NV>(v, smem);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++)
            partials[k * gridDim.x + blockIdx.x] = v[k];
        __threadfence();
        unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!last)
        return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; k++) {
        acc[k] = 0.0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
            acc[k] += ((volatile double *)partials)[k * gridDim.x + b];
    }
    // fixed-order combine: per-thread strided partial sums, then block sum
    block_sum<NV>(acc, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; k++)
            v[k] = acc[k];
        *ticket = 0u;
    }
    return true;
}

}  // namespace mp
