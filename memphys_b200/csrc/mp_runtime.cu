// mp_runtime.cu -- error state, memory and stream helpers of the C ABI.
#include <atomic>
#include <cstdarg>
#include <cmath>
#include <cuda_profiler_api.h>
#include "mp_common.cuh"

namespace mp {

static thread_local char g_err[1024] = {0};
static std::atomic<long long> g_launches{0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int fail(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return status;
}

void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_counter() { return g_launches.load(std::memory_order_relaxed); }

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 148;
    if (dev < 64 && cached[dev])
        return cached[dev];
    int n = 148;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (dev < 64)
        cached[dev] = n;
    return n;
}

bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

bool is_current_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (a.type == cudaMemoryTypeManaged)
        return true;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return false;
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

}  // namespace mp

using namespace mp;

extern "C" {

int mp_last_error(char *buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_err, len - 1);
        buf[len - 1] = 0;
    }
    return MP_OK;
}

int mp_version(void) { return 100; }

int mp_device_info(int *sm, int *major, int *minor, size_t *total_mem) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(MP_NO_DEVICE, "no CUDA device visible");
    }
    int dev = 0;
    MP_CUDA(cudaGetDevice(&dev));
    cudaDeviceProp p;
    MP_CUDA(cudaGetDeviceProperties(&p, dev));
    if (sm)
        *sm = p.multiProcessorCount;
    if (major)
        *major = p.major;
    if (minor)
        *minor = p.minor;
    if (total_mem)
        *total_mem = p.totalGlobalMem;
    if (p.major != 10)
        return fail(MP_NO_DEVICE, "device is sm_%d%d; the library is compiled for sm_100a (B200) only",
                    p.major, p.minor);
    return MP_OK;
}

int mp_set_device(int device) {
    MP_CUDA(cudaSetDevice(device));
    return MP_OK;
}

int mp_malloc(void **ptr, size_t bytes) {
    if (!ptr)
        return fail(MP_BAD_ARG, "mp_malloc: null out pointer");
    MP_CUDA(cudaMalloc(ptr, bytes));
    return MP_OK;
}

int mp_free(void *ptr) {
    if (ptr)
        MP_CUDA(cudaFree(ptr));
    return MP_OK;
}

int mp_malloc_host(void **ptr, size_t bytes) {
    if (!ptr)
        return fail(MP_BAD_ARG, "mp_malloc_host: null out pointer");
    MP_CUDA(cudaMallocHost(ptr, bytes));
    return MP_OK;
}

int mp_free_host(void *ptr) {
    if (ptr)
        MP_CUDA(cudaFreeHost(ptr));
    return MP_OK;
}

int mp_memcpy(void *dst, const void *src, size_t bytes, mp_stream s) {
    if (bytes == 0)
        return MP_OK;
    MP_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, S(s)));
    return MP_OK;
}

int mp_memset(void *dst, int value, size_t bytes, mp_stream s) {
    if (bytes == 0)
        return MP_OK;
    MP_CUDA(cudaMemsetAsync(dst, value, bytes, S(s)));
    return MP_OK;
}

int mp_stream_create(mp_stream *s) {
    cudaStream_t st;
    MP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    *s = (mp_stream)st;
    return MP_OK;
}

int mp_stream_destroy(mp_stream s) {
    if (s)
        MP_CUDA(cudaStreamDestroy(S(s)));
    return MP_OK;
}

int mp_stream_sync(mp_stream s) {
    MP_CUDA(cudaStreamSynchronize(S(s)));
    return MP_OK;
}

struct mp_timer_s {
    cudaEvent_t a, b;
};

int mp_timer_start(mp_stream s, void **timer) {
    mp_timer_s *t = new mp_timer_s;
    if (cudaEventCreate(&t->a) != cudaSuccess || cudaEventCreate(&t->b) != cudaSuccess) {
        delete t;
        return fail(MP_CUDA_ERROR, "cudaEventCreate failed");
    }
    MP_CUDA(cudaEventRecord(t->a, S(s)));
    *timer = t;
    return MP_OK;
}

int mp_timer_stop(void *timer, mp_stream s, double *ms) {
    mp_timer_s *t = (mp_timer_s *)timer;
    if (!t)
        return fail(MP_BAD_ARG, "null timer");
    MP_CUDA(cudaEventRecord(t->b, S(s)));
    MP_CUDA(cudaEventSynchronize(t->b));
    float f = 0.f;
    MP_CUDA(cudaEventElapsedTime(&f, t->a, t->b));
    if (ms)
        *ms = f;
    cudaEventDestroy(t->a);
    cudaEventDestroy(t->b);
    delete t;
    return MP_OK;
}

int mp_profiler(int on) {
    MP_CUDA(on ? cudaProfilerStart() : cudaProfilerStop());
    return MP_OK;
}

int mp_launch_count(int64_t *count, int reset) {
    if (count)
        *count = g_launches.load();
    if (reset)
        g_launches.store(0);
    return MP_OK;
}

// parameters.cpp:122-130
int mp_num_poly_terms(int dim, int poly_deg) {
    if (dim == 2)
        return (int)(0.5 * (poly_deg + 1) * (poly_deg + 2));
    if (dim == 3)
        return (poly_deg + 1) * (poly_deg + 2) * (poly_deg + 3) / 6;
    fail(MP_BAD_ARG, "dimension must be 2 or 3");
    return -1;
}

int mp_cloud_size(int dim, int poly_deg, double mult) {
    int m = mp_num_poly_terms(dim, poly_deg);
    if (m < 0)
        return -1;
    return (int)std::ceil(mult * m);
}

// parameters.cpp:217-267: degree blocks built from the previous block by
// multiplying with x (all terms) and y (the y/z-only tail), closed by z^deg
// (3D) or y^deg (2D).
int mp_poly_exponents(int dim, int poly_deg, int *e) {
    if ((dim != 2 && dim != 3) || poly_deg < 1 || poly_deg > 15 || !e)
        return fail(MP_BAD_ARG, "mp_poly_exponents: dim %d poly_deg %d", dim, poly_deg);
    int m = mp_num_poly_terms(dim, poly_deg);
    for (int i = 0; i < m * dim; i++)
        e[i] = 0;
    for (int d = 0; d < dim; d++)
        e[(1 + d) * dim + d] = 1;
    int prev = 1;
    for (int deg = 2; deg <= poly_deg; deg++) {
        int nprev = dim == 2 ? deg : deg * (deg + 1) / 2;
        int base = prev + nprev;
        for (int i = 0; i < nprev; i++) {
            for (int d = 0; d < dim; d++)
                e[(base + i) * dim + d] = e[(prev + i) * dim + d];
            e[(base + i) * dim] += 1;
        }
        if (dim == 2) {
            e[(base + deg) * 2] = 0;
            e[(base + deg) * 2 + 1] = deg;
        } else {
            int tail = deg * (deg - 1) / 2;  // y/z-only members of the previous block
            for (int i = tail; i < nprev; i++) {
                int r = base + i + deg;
                for (int d = 0; d < 3; d++)
                    e[r * 3 + d] = e[(prev + i) * 3 + d];
                e[r * 3 + 1] += 1;
            }
            int last = base + (deg + 1) * (deg + 2) / 2 - 1;
            e[last * 3] = 0;
            e[last * 3 + 1] = 0;
            e[last * 3 + 2] = deg;
        }
        prev = base;
    }
    return MP_OK;
}

}  // extern "C"
