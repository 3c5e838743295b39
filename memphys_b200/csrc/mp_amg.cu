// mp_amg.cu -- smoothed-aggregation multigrid: host setup, GPU V-cycle.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <type_traits>
#include <cmath>
#include <unordered_map>
#include <condition_variable>
#include "mp_amg.cuh"
#include "mp_ppe.cuh"

namespace mp {

// ------------------------------------------------------- host parallel loops
// The host setup splits its row loops into fixed chunks of rows that worker
// threads claim in any order; every chunk writes its own output range (or
// partial sum, combined in chunk order), so the hierarchy is bit-identical for
// any number of threads.  MP_HOST_THREADS overrides the thread count.
static unsigned host_threads() {
    static const unsigned n = [] {
        const char *e = getenv("MP_HOST_THREADS");
        long v = e ? strtol(e, nullptr, 10) : 0;
        if (v <= 0)
            v = (long)std::thread::hardware_concurrency();
        return (unsigned)std::max(1L, std::min(v, 64L));
    }();
    return n;
}

constexpr int HOST_CHUNK = 16384;

// fn(thread, chunk, first row, end row) for every chunk of [0, n)
template <class F> static void par_chunks(int n, F &&fn) {
    const int nch = (n + HOST_CHUNK - 1) / HOST_CHUNK;
    const unsigned nt = std::min<unsigned>(host_threads(), (unsigned)std::max(nch, 1));
    auto run = [&](unsigned t, std::atomic<int> &next) {
        for (int c; (c = next.fetch_add(1)) < nch;)
            fn(t, c, c * HOST_CHUNK, std::min(n, (c + 1) * HOST_CHUNK));
    };
    std::atomic<int> next{0};
    if (nt <= 1) {
        run(0, next);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++)
        th.emplace_back(run, t, std::ref(next));
    run(0, next);
    for (auto &x : th)
        x.join();
}

// rows produced chunk by chunk: per-chunk column/value lists and row lengths,
// then concatenated in chunk order
struct ChunkRows {
    std::vector<std::vector<int>> ci;
    std::vector<std::vector<double>> v;
    explicit ChunkRows(int n) : ci((n + HOST_CHUNK - 1) / HOST_CHUNK), v(ci.size()) {}
};

// ================================================================ host setup
struct Csr {
    int n = 0, m = 0;
    std::vector<int> rp, ci;
    std::vector<double> v;
};

// C.rp must hold the row lengths at rp[i + 1]; turns them into offsets and
// gathers the chunks' entries
static void concat_rows(Csr &C, ChunkRows &R) {
    C.rp[0] = 0;
    for (int i = 0; i < C.n; i++)
        C.rp[i + 1] += C.rp[i];
    C.ci.resize(C.rp[C.n]);
    C.v.resize(C.rp[C.n]);
    par_chunks(C.n, [&](unsigned, int c, int lo, int) {
        std::copy(R.ci[c].begin(), R.ci[c].end(), C.ci.begin() + C.rp[lo]);
        std::copy(R.v[c].begin(), R.v[c].end(), C.v.begin() + C.rp[lo]);
        std::vector<int>().swap(R.ci[c]);
        std::vector<double>().swap(R.v[c]);
    });
}

static int csr_from_ell(const Ell &E, Csr &C) {
    const int np = ell_padded_rows(E.nrows), K = E.K;
    std::vector<int> cols((size_t)np * K);
    std::vector<double> vals((size_t)np * K);
    MP_CUDA(cudaMemcpy(cols.data(), E.cols.p, sizeof(int) * cols.size(), cudaMemcpyDeviceToHost));
    MP_CUDA(cudaMemcpy(vals.data(), E.v64.p, sizeof(double) * vals.size(), cudaMemcpyDeviceToHost));
    C.n = E.nrows;
    C.m = E.nrows;
    C.rp.assign(C.n + 1, 0);
    ChunkRows R(C.n);
    std::atomic<int> bad{-1};
    par_chunks(C.n, [&](unsigned, int c, int lo, int hi) {
        std::vector<int> &ci = R.ci[c];
        std::vector<double> &v = R.v[c];
        ci.reserve((size_t)(hi - lo) * K);
        v.reserve((size_t)(hi - lo) * K);
        for (int i = lo; i < hi; i++) {
            // merge duplicate columns (setFromTriplets semantics)
            const size_t base = (size_t)(i / SLICE) * K * SLICE + (i % SLICE);
            const size_t start = ci.size();
            for (int k = 0; k < K; k++) {
                const int col = cols[base + (size_t)k * SLICE];
                const double a = vals[base + (size_t)k * SLICE];
                if (a == 0.0 && col != i)
                    continue;
                if (col < 0 || col >= C.m) {
                    bad.store(i);
                    continue;
                }
                bool merged = false;
                for (size_t t = start; t < ci.size(); t++)
                    if (ci[t] == col) {
                        v[t] += a;
                        merged = true;
                        break;
                    }
                if (!merged) {
                    ci.push_back(col);
                    v.push_back(a);
                }
            }
            C.rp[i + 1] = (int)(ci.size() - start);
        }
    });
    if (bad.load() >= 0)
        return fail(MP_BAD_ARG, "operator column out of range in row %d", bad.load());
    concat_rows(C, R);
    return MP_OK;
}

static std::vector<double> diag_of(const Csr &A) {
    std::vector<double> d(A.n, 0.0);
    for (int i = 0; i < A.n; i++)
        for (int t = A.rp[i]; t < A.rp[i + 1]; t++)
            if (A.ci[t] == i)
                d[i] += A.v[t];
    return d;
}

// difference form of a square operator: self entry first holding the row sum,
// then the off-diagonal entries, so that (A u)_i = s_i u_i + sum_j a_ij (u_j - u_i)
static Csr diff_form(const Csr &A) {
    Csr D;
    D.n = A.n;
    D.m = A.m;
    D.rp.assign(A.n + 1, 0);
    D.ci.reserve(A.ci.size() + A.n);
    D.v.reserve(A.v.size() + A.n);
    for (int i = 0; i < A.n; i++) {
        double sum = 0.0;
        for (int t = A.rp[i]; t < A.rp[i + 1]; t++)
            sum += A.v[t];
        D.ci.push_back(i);
        D.v.push_back(sum);
        for (int t = A.rp[i]; t < A.rp[i + 1]; t++)
            if (A.ci[t] != i) {
                D.ci.push_back(A.ci[t]);
                D.v.push_back(A.v[t]);
            }
        D.rp[i + 1] = (int)D.ci.size();
    }
    return D;
}

// largest |eigenvalue| of D^-1 A by power iteration (deterministic start; the
// norms are summed per row chunk, then over the chunks in order)
static double lmax_power(const Csr &A, const std::vector<double> &dinv, int iters) {
    std::vector<double> x(A.n), y(A.n);
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (int i = 0; i < A.n; i++) {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        x[i] = 0.5 + (double)(s >> 11) / 9007199254740992.0;
    }
    const int nch = (A.n + HOST_CHUNK - 1) / HOST_CHUNK;
    std::vector<double> py(nch), px(nch);
    double lam = 1.0;
    for (int it = 0; it < iters; it++) {
        par_chunks(A.n, [&](unsigned, int c, int lo, int hi) {
            double ny = 0.0, nx = 0.0;
            for (int i = lo; i < hi; i++) {
                double a = 0.0;
                for (int t = A.rp[i]; t < A.rp[i + 1]; t++)
                    a += A.v[t] * x[A.ci[t]];
                y[i] = dinv[i] * a;
                ny += y[i] * y[i];
                nx += x[i] * x[i];
            }
            py[c] = ny;
            px[c] = nx;
        });
        double ny = 0.0, nx = 0.0;
        for (int c = 0; c < nch; c++) {
            ny += py[c];
            nx += px[c];
        }
        if (ny == 0.0)
            return 1.0;
        lam = std::sqrt(ny / nx);
        const double inv = 1.0 / std::sqrt(ny);
        par_chunks(A.n, [&](unsigned, int, int lo, int hi) {
            for (int i = lo; i < hi; i++)
                x[i] = y[i] * inv;
        });
    }
    return lam;
}

static void transpose(const Csr &A, Csr &T);

// greedy aggregation on the symmetrised strong graph; isolated rows
// (Dirichlet identities) get no aggregate
static int aggregate(const Csr &A, double theta, std::vector<int> &agg) {
    const int n = A.n;
    // strong entries per row, then S = their union with the transpose (sorted,
    // duplicates removed)
    Csr G;
    G.n = G.m = n;
    G.rp.assign(n + 1, 0);
    {
        ChunkRows R(n);
        par_chunks(n, [&](unsigned, int c, int lo, int hi) {
            for (int i = lo; i < hi; i++) {
                double mx = 0.0;
                for (int t = A.rp[i]; t < A.rp[i + 1]; t++)
                    if (A.ci[t] != i)
                        mx = std::max(mx, std::fabs(A.v[t]));
                int cnt = 0;
                if (mx > 0.0)
                    for (int t = A.rp[i]; t < A.rp[i + 1]; t++) {
                        const int j = A.ci[t];
                        if (j != i && std::fabs(A.v[t]) >= theta * mx) {
                            R.ci[c].push_back(j);
                            R.v[c].push_back(0.0);
                            cnt++;
                        }
                    }
                G.rp[i + 1] = cnt;
            }
        });
        concat_rows(G, R);
    }
    Csr GT;
    transpose(G, GT);
    Csr S;
    S.n = S.m = n;
    S.rp.assign(n + 1, 0);
    {
        ChunkRows R(n);
        par_chunks(n, [&](unsigned, int c, int lo, int hi) {
            std::vector<int> row;
            for (int i = lo; i < hi; i++) {
                row.assign(G.ci.begin() + G.rp[i], G.ci.begin() + G.rp[i + 1]);
                row.insert(row.end(), GT.ci.begin() + GT.rp[i], GT.ci.begin() + GT.rp[i + 1]);
                std::sort(row.begin(), row.end());
                row.erase(std::unique(row.begin(), row.end()), row.end());
                R.ci[c].insert(R.ci[c].end(), row.begin(), row.end());
                R.v[c].resize(R.ci[c].size());
                S.rp[i + 1] = (int)row.size();
            }
        });
        concat_rows(S, R);
    }
    auto nbrs = [&](int i) {
        return std::make_pair(S.ci.begin() + S.rp[i], S.ci.begin() + S.rp[i + 1]);
    };
    agg.assign(n, -1);
    int na = 0;
    for (int i = 0; i < n; i++) {  // pass 1: roots whose neighbourhood is free
        const auto [b, e] = nbrs(i);
        if (agg[i] >= 0 || b == e)
            continue;
        bool free_ = true;
        for (auto it = b; it != e; ++it)
            if (agg[*it] >= 0) {
                free_ = false;
                break;
            }
        if (!free_)
            continue;
        agg[i] = na;
        for (auto it = b; it != e; ++it)
            agg[*it] = na;
        na++;
    }
    std::vector<int> pass1 = agg;
    for (int i = 0; i < n; i++) {  // pass 2: join a neighbouring pass-1 aggregate
        const auto [b, e] = nbrs(i);
        if (agg[i] >= 0 || b == e)
            continue;
        for (auto it = b; it != e; ++it)
            if (pass1[*it] >= 0) {
                agg[i] = pass1[*it];
                break;
            }
    }
    for (int i = 0; i < n; i++) {  // pass 3: leftovers form new aggregates
        const auto [b, e] = nbrs(i);
        if (agg[i] >= 0 || b == e)
            continue;
        agg[i] = na;
        for (auto it = b; it != e; ++it)
            if (agg[*it] < 0)
                agg[*it] = na;
        na++;
    }
    return na;
}

// C = A * B (Gustavson, rows in parallel; columns of each row sorted)
static void spgemm(const Csr &A, const Csr &B, Csr &C) {
    C.n = A.n;
    C.m = B.m;
    C.rp.assign(A.n + 1, 0);
    ChunkRows R(A.n);
    const unsigned nt = host_threads();
    std::vector<std::vector<int>> mark(nt);
    std::vector<std::vector<double>> acc(nt);
    par_chunks(A.n, [&](unsigned th, int c, int lo, int hi) {
        std::vector<int> &mk = mark[th];
        std::vector<double> &ac = acc[th];
        if (mk.empty()) {
            mk.assign(B.m, -1);
            ac.assign(B.m, 0.0);
        }
        std::vector<int> cols;
        for (int i = lo; i < hi; i++) {
            cols.clear();
            for (int t = A.rp[i]; t < A.rp[i + 1]; t++) {
                const int k = A.ci[t];
                const double a = A.v[t];
                for (int u = B.rp[k]; u < B.rp[k + 1]; u++) {
                    const int j = B.ci[u];
                    if (mk[j] != i) {
                        mk[j] = i;
                        ac[j] = 0.0;
                        cols.push_back(j);
                    }
                    ac[j] += a * B.v[u];
                }
            }
            std::sort(cols.begin(), cols.end());
            for (int j : cols) {
                R.ci[c].push_back(j);
                R.v[c].push_back(ac[j]);
            }
            C.rp[i + 1] = (int)cols.size();
        }
    });
    concat_rows(C, R);
}

static void transpose(const Csr &A, Csr &T) {
    T.n = A.m;
    T.m = A.n;
    T.rp.assign(T.n + 1, 0);
    for (int c : A.ci)
        T.rp[c + 1]++;
    for (int i = 0; i < T.n; i++)
        T.rp[i + 1] += T.rp[i];
    T.ci.resize(A.ci.size());
    T.v.resize(A.v.size());
    std::vector<int> pos(T.rp.begin(), T.rp.end() - 1);
    for (int i = 0; i < A.n; i++)
        for (int t = A.rp[i]; t < A.rp[i + 1]; t++) {
            const int p = pos[A.ci[t]]++;
            T.ci[p] = i;
            T.v[p] = A.v[t];
        }
}

// CSR -> sliced ELL on the device, each 64-row slice as wide as its longest
// row; padded entries: column `self ? row : 0`, value 0
static int upload_ell(const Csr &C, Ell &E, bool self_pad, cudaStream_t s) {
    const int ns = (C.n + SLICE - 1) / SLICE;
    std::vector<int> soff(ns + 1, 0);
    int kmax = 1;
    for (int sl = 0; sl < ns; sl++) {
        int w = 1;
        for (int i = sl * SLICE; i < std::min(C.n, (sl + 1) * SLICE); i++)
            w = std::max(w, C.rp[i + 1] - C.rp[i]);
        soff[sl + 1] = soff[sl] + w;
        kmax = std::max(kmax, w);
    }
    const size_t tot = (size_t)soff[ns] * SLICE;
    std::vector<int> cols(tot);
    std::vector<double> vals(tot, 0.0);
    par_chunks(ns * SLICE, [&](unsigned, int, int lo, int hi) {
        for (int i = lo; i < hi; i++) {
            const int sl = i / SLICE, r = i % SLICE, w = soff[sl + 1] - soff[sl];
            const int len = i < C.n ? C.rp[i + 1] - C.rp[i] : 0;
            for (int k = 0; k < w; k++) {
                const size_t o = (size_t)soff[sl] * SLICE + (size_t)k * SLICE + r;
                if (k < len) {
                    cols[o] = C.ci[C.rp[i] + k];
                    vals[o] = C.v[C.rp[i] + k];
                } else {
                    cols[o] = (self_pad && i < C.n && i < C.m) ? i : 0;
                }
            }
        }
    });
    E.nrows = C.n;
    E.ncols = C.m;
    E.K = kmax;
    MP_TRY(E.cols.alloc(cols.size()));
    MP_TRY(E.v64.alloc(vals.size()));
    MP_TRY(E.soff.alloc(soff.size()));
    MP_CUDA(cudaMemcpyAsync(E.cols.p, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(E.v64.p, vals.data(), sizeof(double) * vals.size(), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaMemcpyAsync(E.soff.p, soff.data(), sizeof(int) * soff.size(), cudaMemcpyHostToDevice, s));
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

static int upload_csr(const Csr &C, DCsr &D, cudaStream_t s) {
    D.n = C.n;
    D.m = C.m;
    MP_TRY(D.rp.alloc(C.rp.size()));
    MP_TRY(D.ci.alloc(std::max<size_t>(C.ci.size(), 1)));
    MP_TRY(D.v64.alloc(std::max<size_t>(C.v.size(), 1)));
    MP_CUDA(cudaMemcpyAsync(D.rp.p, C.rp.data(), sizeof(int) * C.rp.size(), cudaMemcpyHostToDevice, s));
    if (!C.ci.empty()) {
        MP_CUDA(cudaMemcpyAsync(D.ci.p, C.ci.data(), sizeof(int) * C.ci.size(), cudaMemcpyHostToDevice, s));
        MP_CUDA(cudaMemcpyAsync(D.v64.p, C.v.data(), sizeof(double) * C.v.size(), cudaMemcpyHostToDevice, s));
    }
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

// bordered dense inverse of the coarsest operator (LU with partial pivoting)
// An operator whose rows all sum to zero (constants in its null space, the
// all-Neumann pressure system) is bordered like solver.cpp:205-213; any other
// (Dirichlet rows, a shifted diagonal such as the Helmholtz systems of the
// Fourier modes) is inverted as [A 0; 0 1], so that the coarse correction keeps
// the constant component, which such operators do not annihilate.
static int coarse_inverse(const Csr &A, std::vector<double> &inv, bool *bordered) {
    const int n = A.n, m = n + 1;
    std::vector<double> M((size_t)m * m, 0.0);
    double max_sum = 0.0, max_abs = 0.0;
    for (int i = 0; i < n; i++) {
        double rs = 0.0, ra = 0.0;
        for (int t = A.rp[i]; t < A.rp[i + 1]; t++) {
            M[(size_t)i * m + A.ci[t]] += A.v[t];
            rs += A.v[t];
            ra += std::fabs(A.v[t]);
        }
        max_sum = std::max(max_sum, std::fabs(rs));
        max_abs = std::max(max_abs, ra);
    }
    const bool border = max_sum <= 1e-10 * max_abs;
    *bordered = border;
    for (int i = 0; i < n; i++) {
        M[(size_t)i * m + n] = border ? 1.0 : 0.0;
        M[(size_t)n * m + i] = border ? 1.0 : 0.0;
    }
    if (!border)
        M[(size_t)n * m + n] = 1.0;
    inv.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; i++)
        inv[(size_t)i * m + i] = 1.0;
    // Gauss-Jordan with partial pivoting.  Each step's pivot row is chosen and scaled
    // by thread 0, then every other row is updated by the thread that owns it (rows
    // split in fixed ranges): the rows' updates are independent, so the inverse does
    // not depend on the thread count.  Columns left of the pivot are already reduced
    // and are skipped in M.
    const unsigned nt = std::max(1u, std::min(host_threads(), (unsigned)(m / 64 + 1)));
    std::mutex mu;
    std::condition_variable cv;
    unsigned arrived = 0, gen = 0;
    auto barrier = [&]() {
        std::unique_lock<std::mutex> lk(mu);
        const unsigned g = gen;
        if (++arrived == nt) {
            arrived = 0;
            gen++;
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return gen != g; });
        }
    };
    bool singular = false;
    auto work = [&](unsigned t) {
        const int lo = (int)((long long)m * t / nt), hi = (int)((long long)m * (t + 1) / nt);
        for (int k = 0; k < m; k++) {
            if (t == 0) {
                int p = k;
                for (int i = k + 1; i < m; i++)
                    if (std::fabs(M[(size_t)i * m + k]) > std::fabs(M[(size_t)p * m + k]))
                        p = i;
                if (M[(size_t)p * m + k] == 0.0) {
                    singular = true;
                } else {
                    if (p != k)
                        for (int j = 0; j < m; j++) {
                            std::swap(M[(size_t)k * m + j], M[(size_t)p * m + j]);
                            std::swap(inv[(size_t)k * m + j], inv[(size_t)p * m + j]);
                        }
                    const double d = 1.0 / M[(size_t)k * m + k];
                    for (int j = k; j < m; j++)
                        M[(size_t)k * m + j] *= d;
                    for (int j = 0; j < m; j++)
                        inv[(size_t)k * m + j] *= d;
                }
            }
            barrier();
            if (singular)
                return;
            const double *mk = &M[(size_t)k * m], *ik = &inv[(size_t)k * m];
            for (int i = lo; i < hi; i++) {
                if (i == k)
                    continue;
                double *mi = &M[(size_t)i * m], *ii = &inv[(size_t)i * m];
                const double f = mi[k];
                if (f == 0.0)
                    continue;
                for (int j = k + 1; j < m; j++)
                    mi[j] -= f * mk[j];
                mi[k] = 0.0;
                for (int j = 0; j < m; j++)
                    ii[j] -= f * ik[j];
            }
            barrier();
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; t++)
        th.emplace_back(work, t);
    work(0);
    for (auto &x : th)
        x.join();
    if (singular)
        return fail(MP_BREAKDOWN, "multigrid coarse operator is singular");
    return MP_OK;
}

__global__ void k_to_f32(const double *a, float *b, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        b[i] = (float)a[i];
}

static int make_f32(const dbuf<double> &a, dbuf<float> &b, cudaStream_t s) {
    MP_TRY(b.alloc(a.n));
    k_to_f32<<<(unsigned)((a.n + 255) / 256), 256, 0, s>>>(a.p, b.p, a.n);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// level 0 in FP32 difference form, in the PPE operator's own sliced layout
// (its stencil rows start with the node itself); one thread per row
__global__ void k_diff_level0(EllView<double> A, float *out, int *bad) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int np = ell_padded_rows(A.nrows);
    if (i >= np)
        return;
    size_t base;
    int K;
    slice_span(A, i / SLICE, base, K);
    base += i % SLICE;
    double sum = 0.0;
    for (int k = 0; k < K; k++)
        sum += A.vals[base + (size_t)k * SLICE];
    if (i < A.nrows && K > 0 && A.cols[base] != i)
        atomicAdd(bad, 1);
    for (int k = 1; k < K; k++)
        out[base + (size_t)k * SLICE] = (float)A.vals[base + (size_t)k * SLICE];
    if (K > 0)
        out[base] = i < A.nrows ? (float)sum : 0.f;
}

__global__ void k_pack_pairs(const int *cols, const float *v, int2 *out, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = make_int2(cols[i], __float_as_int(v[i]));
}

static int pack_pairs(const int *cols, const float *v, size_t n, dbuf<int2> &out,
                      cudaStream_t s) {
    MP_TRY(out.alloc(n));
    k_pack_pairs<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(cols, v, out.p, n);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

int ell_diff32(const Ell &A0, dbuf<float> &v32, dbuf<int2> &pk, cudaStream_t s) {
    MP_TRY(v32.alloc(A0.v64.n));
    dbuf<int> bad;
    MP_TRY(bad.alloc(1));
    MP_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    const int np = ell_padded_rows(A0.nrows);
    k_diff_level0<<<(np + 255) / 256, 256, 0, s>>>(A0.view64(), v32.p, bad.p);
    MP_CHECK_LAUNCH();
    int hb = 0;
    MP_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (hb)
        return fail(MP_BAD_ARG, "FP32 difference form needs every stencil row to start with its "
                                "own node (%d rows do not)", hb);
    return pack_pairs(A0.cols.p, v32.p, A0.v64.n, pk, s);
}

// k-paired copy of a uniform-width FP32 operator (EllView::qv/qd): one warp per
// slice writes its values and deltas and sets the slice's flag when every delta
// fits 16 bits.  An odd width gets a zero entry pointing at the row itself
// (padding rows past nrows point at column 0, as everywhere in the layout).
__global__ void k_pair_deltas(int nrows, int K, const int *cols, const float *v, float *qv,
                              short *qd, unsigned char *flag) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= (nrows + SLICE - 1) / SLICE)
        return;
    const int J = (K + 1) >> 1;
    const size_t base = (size_t)w * K * SLICE;
    bool fits = true;
    for (int t = lane; t < 2 * J * SLICE; t += 32) {
        const int k = t / SLICE, r = t % SLICE, row = w * SLICE + r;
        const int col = k < K ? cols[base + (size_t)k * SLICE + r] : (row < nrows ? row : 0);
        const long long dl = (long long)col - row;
        const bool ok = dl >= -32768 && dl <= 32767;
        fits = fits && ok;
        const size_t q = (((size_t)w * J + (k >> 1)) * 32 + (r >> 1)) * 4 + (k & 1) * 2 + (r & 1);
        qv[q] = k < K ? v[base + (size_t)k * SLICE + r] : 0.f;
        qd[q] = ok ? (short)dl : (short)0;
    }
    fits = __all_sync(0xffffffffu, fits);
    if (lane == 0)
        flag[w] = fits ? 1 : 0;
}

// entries 1..K-1 of every row (the self entry stays first) in ascending column
// order, one thread per row (padded rows included): consecutive rows then meet their
// k-th neighbours at nearly the same offset, so a warp's gather of entry k touches
// few cache lines (in a 2D cavity 6.3 instead of 14.8 128-byte lines per gather,
// against the distance order of the stencil lists)
constexpr int SORT_KMAX = 64;
__global__ void k_sort_row_entries(int np, int K, const int *cols, const float *v, int *oc,
                                   float *ov) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np)
        return;
    const size_t base = (size_t)(i / SLICE) * K * SLICE + i % SLICE;
    int c[SORT_KMAX];
    float w[SORT_KMAX];
    for (int k = 0; k < K; k++) {
        c[k] = cols[base + (size_t)k * SLICE];
        w[k] = v[base + (size_t)k * SLICE];
    }
    for (int k = 2; k < K; k++) {  // insertion sort of entries 1..K-1
        const int ck = c[k];
        const float wk = w[k];
        int j = k - 1;
        while (j >= 1 && c[j] > ck) {
            c[j + 1] = c[j];
            w[j + 1] = w[j];
            j--;
        }
        c[j + 1] = ck;
        w[j + 1] = wk;
    }
    for (int k = 0; k < K; k++) {
        oc[base + (size_t)k * SLICE] = c[k];
        ov[base + (size_t)k * SLICE] = w[k];
    }
}

static int pair_deltas(const Ell &A0, const float *v32, AmgLevel &L, cudaStream_t s) {
    const int nsl = (A0.nrows + SLICE - 1) / SLICE, J = (A0.K + 1) / 2;
    const size_t nq = (size_t)nsl * J * 32;
    MP_TRY(L.qv.alloc(nq));
    MP_TRY(L.qd.alloc(nq));
    MP_TRY(L.qslice.alloc(nsl));
    const int *cols = A0.cols.p;
    const float *vals = v32;
    dbuf<int> sc;
    dbuf<float> sv;
    if (A0.K <= SORT_KMAX) {
        const int np = nsl * SLICE;
        MP_TRY(sc.alloc((size_t)np * A0.K));
        MP_TRY(sv.alloc((size_t)np * A0.K));
        k_sort_row_entries<<<(np + 255) / 256, 256, 0, s>>>(np, A0.K, A0.cols.p, v32, sc.p, sv.p);
        MP_CHECK_LAUNCH();
        cols = sc.p;
        vals = sv.p;
    }
    k_pair_deltas<<<(unsigned)(((size_t)nsl * 32 + 255) / 256), 256, 0, s>>>(
        A0.nrows, A0.K, cols, vals, reinterpret_cast<float *>(L.qv.p),
        reinterpret_cast<short *>(L.qd.p), L.qslice.p);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaStreamSynchronize(s));  // the sorted copies are freed on return
    L.Ad32.qv = L.qv.p;
    L.Ad32.qd = L.qd.p;
    L.Ad32.qslice = L.qslice.p;
    return MP_OK;
}

static int diff_level0(const Ell &A0, AmgLevel &L, cudaStream_t s) {
    const EllView<double> A = A0.view64();
    MP_TRY(L.Ad.v32.alloc(A0.v64.n));
    dbuf<int> bad;
    MP_TRY(bad.alloc(1));
    MP_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    const int np = ell_padded_rows(A0.nrows);
    k_diff_level0<<<(np + 255) / 256, 256, 0, s>>>(A, L.Ad.v32.p, bad.p);
    MP_CHECK_LAUNCH();
    int hb = 0;
    MP_CUDA(cudaMemcpyAsync(&hb, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    MP_CUDA(cudaStreamSynchronize(s));
    if (hb)
        return fail(MP_BAD_ARG, "FP32 multigrid storage needs every stencil row to start with its "
                                "own node (%d rows do not)", hb);
    MP_TRY(pack_pairs(A0.cols.p, L.Ad.v32.p, A0.v64.n, L.Adpk, s));
    L.Ad32 = EllView<float>{A0.nrows, A0.ncols, A0.K, A0.cols.p, L.Ad.v32.p, A0.soff.p, L.Adpk.p};
    if (!A0.soff.p && A0.K > 0)
        MP_TRY(pair_deltas(A0, L.Ad.v32.p, L, s));
    return MP_OK;
}

// levels >= 1: difference-form copies (sliced ELL and CSR), FP32 values
static int diff_level(const Csr &A, AmgLevel &L, cudaStream_t s) {
    const Csr D = diff_form(A);
    MP_TRY(upload_ell(D, L.Ad, true, s));
    MP_TRY(ell_make_fp32(L.Ad, s));
    MP_TRY(upload_csr(D, L.Acd, s));
    MP_TRY(make_f32(L.Acd.v64, L.Acd.v32, s));
    MP_CUDA(cudaStreamSynchronize(s));
    L.Ad.v64.release();
    L.Acd.v64.release();
    MP_TRY(pack_pairs(L.Ad.cols.p, L.Ad.v32.p, L.Ad.v32.n, L.Adpk, s));
    MP_TRY(pack_pairs(L.Acd.ci.p, L.Acd.v32.p, L.Acd.v32.n, L.Acd.pk, s));
    L.Ad32 = L.Ad.view32();
    L.Ad32.pk = L.Adpk.p;
    return MP_OK;
}

Amg::~Amg() {
    for (auto *l : L)
        delete l;
}

static int amg_autotune(Amg &a, cudaStream_t s);

int amg_create(Amg **out, const Ell &A0, const Cfg &cfg, int store, cudaStream_t s) {
    auto t0 = std::chrono::steady_clock::now();
    // Strength threshold, the Chebyshev interval [lmax / 12, 1.1 lmax] and the
    // prolongator damping 4 / (3 lmax) were chosen by sweeps on the 1M-node cavity
    // (iterations per step: ratio 6 -> 21.3, 10-15 -> 19.7-19.9, 20 -> 22.2;
    // theta 0.1 / 0.25 / 0.5 -> 29.1 / 21.3 / 30.7).
    const double theta = 0.25, lscale = 1.1;
    const int coarse_size = cfg.amg_coarse_size;
    const bool mixed = store == AMG_F32;
    Amg *a = new Amg;
    a->store = store;
    a->cheb_ratio = 1.0 / cfg.cheb_lower;
    a->sweeps = std::max(1, cfg.smoother_sweeps);
    // seconds per setup phase: operator download, aggregation, power iteration,
    // products, uploads, autotuner (printed with MP_VERBOSE)
    double ph[6] = {0, 0, 0, 0, 0, 0};
    auto tick = std::chrono::steady_clock::now();
    auto lap = [&](int q) {
        const auto now = std::chrono::steady_clock::now();
        ph[q] += std::chrono::duration<double>(now - tick).count();
        tick = now;
    };
    // with MP_VERBOSE: FNV-1a checksum of every level's operator and prolongator
    // (the host setup gives the same hierarchy for any number of threads)
    const bool verbose = getenv("MP_VERBOSE") != nullptr;
    uint64_t hsum = 0xcbf29ce484222325ull;
    auto hash_csr = [&](const Csr &C) {
        if (!verbose)
            return;
        auto mix = [&](const void *p, size_t n) {
            const unsigned char *b = (const unsigned char *)p;
            for (size_t q = 0; q < n; q++)
                hsum = (hsum ^ b[q]) * 0x100000001b3ull;
        };
        mix(C.rp.data(), sizeof(int) * C.rp.size());
        mix(C.ci.data(), sizeof(int) * C.ci.size());
        mix(C.v.data(), sizeof(double) * C.v.size());
    };
    Csr A;
    int rc = csr_from_ell(A0, A);
    lap(0);
    if (rc != MP_OK) {
        delete a;
        return rc;
    }
    auto bail = [&](int r) {
        delete a;
        return r;
    };
    for (int lev = 0;; lev++) {
        AmgLevel *L = new AmgLevel;
        a->L.push_back(L);
        L->n = A.n;
        std::vector<double> d = diag_of(A);
        std::vector<double> dinv(A.n);
        for (int i = 0; i < A.n; i++)
            dinv[i] = (d[i] != 0.0 && std::isfinite(d[i])) ? 1.0 / d[i] : 0.0;
        if (lev == 0) {
            L->borrowed = true;
            L->A64 = A0.view64();
            L->A32 = A0.view32();
            if (store != AMG_F64 && (rc = diff_level0(A0, *L, s)) != MP_OK)
                return bail(rc);
        } else {
            if ((rc = upload_ell(A, L->A, true, s)) != MP_OK || (rc = upload_csr(A, L->Ac, s)) != MP_OK)
                return bail(rc);
            L->A64 = L->A.view64();
            if (store != AMG_F64 && (rc = diff_level(A, *L, s)) != MP_OK)
                return bail(rc);
        }
        if ((rc = L->dinv.alloc(A.n)) != MP_OK)
            return bail(rc);
        MP_CUDA(cudaMemcpy(L->dinv.p, dinv.data(), sizeof(double) * A.n, cudaMemcpyHostToDevice));
        const bool coarsest = A.n <= coarse_size || lev + 1 >= cfg.amg_max_levels;
        if (!coarsest) {
            std::vector<int> agg;
            lap(4);
            const int na = aggregate(A, theta, agg);
            lap(1);
            if (na == 0 || na >= A.n) {
                // cannot coarsen further: this level becomes the coarsest
            } else {
                const double lam = lmax_power(A, dinv, 30);
                lap(2);
                L->lmax = lscale * lam;
                const double w = 4.0 / (3.0 * lam);
                // AT = A * T, then P = T - w D^-1 AT
                Csr T;
                T.n = A.n;
                T.m = na;
                T.rp.assign(A.n + 1, 0);
                for (int i = 0; i < A.n; i++) {
                    if (agg[i] >= 0) {
                        T.ci.push_back(agg[i]);
                        T.v.push_back(1.0);
                    }
                    T.rp[i + 1] = (int)T.ci.size();
                }
                Csr AT, P, R, AP, Ac;
                spgemm(A, T, AT);
                P.n = A.n;
                P.m = na;
                P.rp.assign(A.n + 1, 0);
                for (int i = 0; i < A.n; i++) {
                    const int ti = agg[i];
                    bool diag_done = false;
                    for (int t = AT.rp[i]; t < AT.rp[i + 1]; t++) {
                        double v = -w * dinv[i] * AT.v[t];
                        if (AT.ci[t] == ti) {
                            v += 1.0;
                            diag_done = true;
                        }
                        if (v != 0.0) {
                            P.ci.push_back(AT.ci[t]);
                            P.v.push_back(v);
                        }
                    }
                    if (ti >= 0 && !diag_done) {
                        P.ci.push_back(ti);
                        P.v.push_back(1.0);
                    }
                    P.rp[i + 1] = (int)P.ci.size();
                }
                transpose(P, R);
                spgemm(A, P, AP);
                spgemm(R, AP, Ac);
                lap(3);
                hash_csr(A);
                hash_csr(P);
                if ((rc = upload_ell(P, L->P, false, s)) != MP_OK ||
                    (rc = upload_ell(R, L->R, false, s)) != MP_OK ||
                    (rc = upload_csr(P, L->Pc, s)) != MP_OK || (rc = upload_csr(R, L->Rc, s)) != MP_OK)
                    return bail(rc);
                if (lev > 0) {
                    if ((rc = L->b.alloc(A.n)) != MP_OK || (rc = L->x.alloc(A.n)) != MP_OK)
                        return bail(rc);
                }
                if ((rc = L->d.alloc(A.n)) != MP_OK || (rc = L->r.alloc(A.n)) != MP_OK)
                    return bail(rc);
                A = std::move(Ac);
                continue;
            }
        }
        // coarsest level: dense inverse (bordered when singular)
        hash_csr(A);
        std::vector<double> inv;
        if ((rc = coarse_inverse(A, inv, &a->coarse_bordered)) != MP_OK)
            return bail(rc);
        a->nc = A.n;
        if ((rc = a->cinv.alloc(inv.size())) != MP_OK)
            return bail(rc);
        MP_CUDA(cudaMemcpy(a->cinv.p, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice));
        if (lev > 0) {
            if ((rc = L->b.alloc(A.n)) != MP_OK || (rc = L->x.alloc(A.n)) != MP_OK)
                return bail(rc);
        }
        break;
    }
    if (mixed) {
        for (size_t l = 0; l < a->L.size(); l++) {
            AmgLevel *L = a->L[l];
            if (!L->borrowed && L->A.v64.p) {
                if ((rc = ell_make_fp32(L->A, s)) != MP_OK)
                    return bail(rc);
                L->A32 = L->A.view32();
            }
            if (L->P.v64.p && ((rc = ell_make_fp32(L->P, s)) != MP_OK || (rc = ell_make_fp32(L->R, s)) != MP_OK))
                return bail(rc);
            for (DCsr *D : {&L->Ac, &L->Pc, &L->Rc})
                if (D->v64.p && (rc = make_f32(D->v64, D->v32, s)) != MP_OK)
                    return bail(rc);
            if ((rc = make_f32(L->dinv, L->dinv32, s)) != MP_OK)
                return bail(rc);
            for (auto pr : {std::make_pair(&L->b, &L->b32), std::make_pair(&L->x, &L->x32),
                            std::make_pair(&L->d, &L->d32), std::make_pair(&L->r, &L->r32)})
                if (pr.first->p && (rc = pr.second->alloc(pr.first->n)) != MP_OK)
                    return bail(rc);
        }
        if ((rc = make_f32(a->cinv, a->cinv32, s)) != MP_OK)
            return bail(rc);
    }
    if (store == AMG_MG32) {  // FP32 transfers; vectors, diagonal and coarse inverse stay FP64
        for (AmgLevel *L : a->L) {
            if (L->P.v64.p && ((rc = ell_make_fp32(L->P, s)) != MP_OK ||
                               (rc = ell_make_fp32(L->R, s)) != MP_OK))
                return bail(rc);
            for (DCsr *D : {&L->Pc, &L->Rc})
                if (D->v64.p && (rc = make_f32(D->v64, D->v32, s)) != MP_OK)
                    return bail(rc);
        }
    }
    lap(4);
    if ((rc = amg_autotune(*a, s)) != MP_OK)
        return bail(rc);
    MP_CUDA(cudaStreamSynchronize(s));
    lap(5);
    a->setup_seconds =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (verbose) {
        fprintf(stderr, "[memphys amg] hierarchy checksum %016llx\n", (unsigned long long)hsum);
        for (size_t l = 0; l < a->L.size(); l++) {
            const AmgLevel &L = *a->L[l];
            fprintf(stderr, "[memphys amg] level %zu n=%d A.K=%d lmax=%.3f", l, L.n, L.A64.K,
                    L.lmax);
            if (L.Ac.n)
                fprintf(stderr, " A.nnz/row=%.1f", (double)L.Ac.ci.n / L.n);
            if (L.Pc.n)
                fprintf(stderr, " P.nnz/row=%.1f R.nnz/row=%.1f", (double)L.Pc.ci.n / L.Pc.n,
                        (double)L.Rc.ci.n / L.Rc.n);
            fprintf(stderr, " sched A=%d P=%d R=%d", L.sA.mode, L.sP.mode, L.sR.mode);
            const OpSched *sc[3] = {&L.sA, &L.sP, &L.sR};
            for (int o = 0; o < 3; o++) {  // cold-L2 timings of the schedules tried
                fprintf(stderr, " (%c us:", "APR"[o]);
                for (int m = 0; m < OP_MODES; m++)
                    if (sc[o]->us[m] > 0)
                        fprintf(stderr, " %d:%.1f", m, sc[o]->us[m]);
                fprintf(stderr, ")");
            }
            fprintf(stderr, "\n");
        }
        fprintf(stderr,
                "[memphys amg] coarse n=%d setup %.2f s (download %.2f aggregate %.2f power %.2f "
                "products %.2f upload %.2f autotune %.2f; %u host threads)\n",
                a->nc, a->setup_seconds, ph[0], ph[1], ph[2], ph[3], ph[4], ph[5], host_threads());
    }
    *out = a;
    return MP_OK;
}

void amg_destroy(Amg *a) { delete a; }

// ================================================================ GPU cycle
template <class T> struct V2a;
template <> struct V2a<double> { using type = double2; };
template <> struct V2a<float> { using type = float2; };

// Operator loads.  EVF (evict first): the finest level's operators and transfers
// stream through L2 once per use (273 MB at 1M nodes, twice the L2), so their lines
// go first and leave the coarse levels resident; a coarse level's operator is read
// four times in a row inside one cycle (two smoothing steps and the residual on each
// side) and is loaded with the default policy so that its repeats hit in L2.
template <bool EVF, class P> __device__ __forceinline__ P ldop(const P *p) {
    if constexpr (EVF)
        return __ldcs(p);
    else
        return __ldg(p);
}

// Two rows of (M u): T is the vector type, V the stored value type.  With DIFF
// the first entry of each row is the self entry holding the row sum, and the
// others multiply (u_j - u_i): a = s_i u_i + sum_k a_ik (u_k - u_i).
template <class T, class V, bool DIFF, bool EVF>
__device__ __forceinline__ void spmv_pair(const EllView<V> &A, int w, int lane,
                                          const T *__restrict__ x, T &a0, T &a1) {
    using V2 = typename V2a<V>::type;
    size_t base;
    int K;
    slice_span(A, w, base, K);
    base += 2 * lane;
    a0 = 0;
    a1 = 0;
    T s0 = 0, s1 = 0;
    int k0 = 0;
    if constexpr (sizeof(V) == 4) {
        if (A.qv && A.qslice[w]) {  // entries k, k + 1 of both rows: float4 values, short4 deltas
            const int i0 = w * SLICE + 2 * lane, J = (K + 1) >> 1;
            const size_t qb = (size_t)w * J * 32 + lane;
            const float4 *QV = A.qv + qb;
            const short4 *QD = A.qd + qb;
            int j0 = 0;
            if (DIFF && K > 0) {  // the self entry (row sum) and entry 1
                s0 = i0 < A.nrows ? __ldg(x + i0) : T(0);
                s1 = i0 + 1 < A.nrows ? __ldg(x + i0 + 1) : T(0);
                const float4 v = ldop<EVF>(QV);
                const short4 c = ldop<EVF>(QD);
                const T g0 = __ldg(x + i0 + c.z), g1 = __ldg(x + i0 + 1 + c.w);
                a0 = fma((T)v.z, g0 - s0, (T)v.x * s0);
                a1 = fma((T)v.w, g1 - s1, (T)v.y * s1);
                j0 = 1;
            }
#pragma unroll 2
            for (int j = j0; j < J; j++) {
                const float4 v = ldop<EVF>(QV + (size_t)j * 32);
                const short4 c = ldop<EVF>(QD + (size_t)j * 32);
                const T g0 = __ldg(x + i0 + c.x), g1 = __ldg(x + i0 + 1 + c.y);
                const T g2 = __ldg(x + i0 + c.z), g3 = __ldg(x + i0 + 1 + c.w);
                a0 = fma((T)v.x, DIFF ? g0 - s0 : g0, a0);
                a1 = fma((T)v.y, DIFF ? g1 - s1 : g1, a1);
                a0 = fma((T)v.z, DIFF ? g2 - s0 : g2, a0);
                a1 = fma((T)v.w, DIFF ? g3 - s1 : g3, a1);
            }
            return;
        }
        if (A.pk) {  // {col, value} of both rows in one 16-byte load
            const int4 *P = reinterpret_cast<const int4 *>(A.pk + base);
            if (DIFF && K > 0) {
                const int i0 = w * SLICE + 2 * lane;
                s0 = i0 < A.nrows ? __ldg(x + i0) : T(0);
                s1 = i0 + 1 < A.nrows ? __ldg(x + i0 + 1) : T(0);
                const int4 e = ldop<EVF>(P);
                a0 = (T)__int_as_float(e.y) * s0;
                a1 = (T)__int_as_float(e.w) * s1;
                k0 = 1;
            }
#pragma unroll 4
            for (int k = k0; k < K; k++) {
                const int4 e = ldop<EVF>(P + (size_t)k * (SLICE / 2));
                const T g0 = __ldg(x + e.x), g1 = __ldg(x + e.z);
                a0 = fma((T)__int_as_float(e.y), DIFF ? g0 - s0 : g0, a0);
                a1 = fma((T)__int_as_float(e.w), DIFF ? g1 - s1 : g1, a1);
            }
            return;
        }
    }
    if (DIFF && K > 0) {
        const int i0 = w * SLICE + 2 * lane;
        s0 = i0 < A.nrows ? __ldg(x + i0) : T(0);
        s1 = i0 + 1 < A.nrows ? __ldg(x + i0 + 1) : T(0);
        const V2 v = ldop<EVF>(reinterpret_cast<const V2 *>(A.vals + base));
        a0 = (T)v.x * s0;
        a1 = (T)v.y * s1;
        k0 = 1;
    }
    if (!DIFF && A.dslice && A.dslice[w]) {  // 16-bit column deltas (warp-uniform)
        const int i0 = w * SLICE + 2 * lane;
#pragma unroll 4
        for (int k = 0; k < K; k++) {
            const size_t o = base + (size_t)k * SLICE;
            const short2 c = ldop<EVF>(reinterpret_cast<const short2 *>(A.dcols + o));
            const V2 v = ldop<EVF>(reinterpret_cast<const V2 *>(A.vals + o));
            const T x0 = __ldg(x + i0 + c.x), x1 = __ldg(x + i0 + 1 + c.y);
            a0 = fma((T)v.x, x0, a0);
            a1 = fma((T)v.y, x1, a1);
        }
        return;
    }
#pragma unroll 4
    for (int k = k0; k < K; k++) {
        const size_t o = base + (size_t)k * SLICE;
        const int2 c = ldop<EVF>(reinterpret_cast<const int2 *>(A.cols + o));
        const V2 v = ldop<EVF>(reinterpret_cast<const V2 *>(A.vals + o));
        const T x0 = __ldg(x + c.x), x1 = __ldg(x + c.y);
        a0 = fma((T)v.x, DIFF ? x0 - s0 : x0, a0);
        a1 = fma((T)v.y, DIFF ? x1 - s1 : x1, a1);
    }
}

__device__ __forceinline__ int gwarp_a() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }

// Epilogue kinds of the fused level kernels
enum { EP_CHEB_PRE = 0, EP_RESID, EP_PLAIN, EP_PROLONG, EP_CHEB_POST1, EP_CHEB_POST2, EP_RESTRICT };

struct ChebC {
    double inv_theta, theta, c1, c2, c3, c4;
};

template <class V> struct CsrView {
    int nrows;
    const int *rp, *ci;
    const V *v;
    const int2 *pk = nullptr;  // (column, FP32 value bits) pairs, when packed
};

// Row i of one fused SpMV (a = (M u)_i) followed by its epilogue:
//   EP_CHEB_PRE  : x = c1 d + c2 dinv (b - M d)            (u = d)
//   EP_RESID     : y = b - M x                              (u = x)
//   EP_PLAIN     : y = M u
//   EP_PROLONG   : x = x + M u                              (M = P, u = coarse x)
//   EP_CHEB_POST1: d = dinv (b - M x) / theta               (u = x)
//   EP_CHEB_POST2: x = x + (1 + c3) d + c4 (theta d - dinv M d)   (u = d)
//   EP_RESTRICT  : y = M u, d = dinv y / theta               (M = R; y, d, dinv and
//                  theta of the coarser level: the first step of its pre-smoother
//                  from a zero guess, written with its right-hand side)
// No kernel writes the vector it gathers.
template <class T, int EP>
__device__ __forceinline__ void level_epilogue(int i, T a, const T *b, const T *dinv, T *d, T *x,
                                               T *y, const ChebC &c) {
    if (EP == EP_CHEB_PRE) {
        x[i] = (T)c.c1 * d[i] + (T)c.c2 * dinv[i] * (b[i] - a);
    } else if (EP == EP_RESID) {
        y[i] = b[i] - a;
    } else if (EP == EP_PLAIN) {
        y[i] = a;
    } else if (EP == EP_PROLONG) {
        x[i] = x[i] + a;
    } else if (EP == EP_CHEB_POST1) {
        d[i] = dinv[i] * (b[i] - a) * (T)c.inv_theta;
    } else if (EP == EP_RESTRICT) {
        y[i] = a;
        d[i] = dinv[i] * a * (T)c.inv_theta;
    } else {
        const T di = d[i];
        x[i] = x[i] + (T)(1.0 + c.c3) * di + (T)c.c4 * ((T)c.theta * di - dinv[i] * a);
    }
}

// sliced ELL: one warp per 64-row slice, two rows per lane.  Held to 32 registers
// (8 blocks of 256 per SM): these kernels wait on memory, and occupancy is what
// keeps enough loads in flight (at 48 registers the FP32 form ran at 53 % warps
// active and 60 % of DRAM bandwidth)
template <class T, class V, bool DIFF, bool EVF, int EP>
__global__ void __launch_bounds__(256, 8)
    k_level(EllView<V> M, const T *__restrict__ u, const T *__restrict__ b,
            const T *__restrict__ dinv, T *d, T *x, T *y, ChebC c, const int *done) {
    pdl_wait();
    pdl_trigger();
    if (*done)
        return;
    const int w = gwarp_a(), lane = threadIdx.x & 31;
    if (w >= (M.nrows + SLICE - 1) / SLICE)
        return;
    T a[2];
    spmv_pair<T, V, DIFF, EVF>(M, w, lane, u, a[0], a[1]);
    const int i0 = w * SLICE + 2 * lane;
#pragma unroll
    for (int q = 0; q < 2; q++)
        if (i0 + q < M.nrows)
            level_epilogue<T, EP>(i0 + q, a[q], b, dinv, d, x, y, c);
}

// CSR: G lanes per row, partial sums combined with shuffles inside the group
// (DIFF: the row's first entry is its self entry, see spmv_pair)
template <class T, class V, int G, bool DIFF, bool EVF, int EP>
__global__ void __launch_bounds__(256)
    k_level_csr(CsrView<V> M, const T *__restrict__ u, const T *__restrict__ b,
                const T *__restrict__ dinv, T *d, T *x, T *y, ChebC c, const int *done) {
    pdl_wait();
    pdl_trigger();
    if (*done)
        return;
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const int row = gid / G, li = gid % G;
    T acc = 0;
    if (row < M.nrows) {
        const int b0 = M.rp[row], e = M.rp[row + 1];
        const T ui = DIFF ? __ldg(u + row) : T(0);
        if (M.pk) {  // (column, FP32 value) pairs: one 8-byte load per entry
#pragma unroll 4
            for (int t = b0 + li; t < e; t += G) {
                const int2 q = ldop<EVF>(M.pk + t);
                const T ut = __ldg(u + q.x);
                acc = fma((T)__int_as_float(q.y), (DIFF && t != b0) ? ut - ui : ut, acc);
            }
        } else {
#pragma unroll 4
            for (int t = b0 + li; t < e; t += G) {
                const T ut = __ldg(u + ldop<EVF>(M.ci + t));
                acc = fma((T)ldop<EVF>(M.v + t), (DIFF && t != b0) ? ut - ui : ut, acc);
            }
        }
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (row < M.nrows && li == 0)
        level_epilogue<T, EP>(row, acc, b, dinv, d, x, y, c);
}

// sliced ELL with the slice's entries split over the CTA's KS warps: one 64-row slice
// per CTA, warp q takes entries k = q, q + KS, ... of both rows of every lane, the
// partial sums meet in shared memory and warp 0 adds them in warp order and runs the
// epilogue.  For coarse levels whose slices are few and wide (level 1: 2,007 slices
// of ~35-50 entries), where one warp per slice leaves the GPU a fifth full and a
// lane's entries form a long dependent chain; KS = 8, 4, 2 trade the chain's length
// against the number of CTAs resident at once.
template <class T, class V, bool DIFF, bool EVF, int EP, int KS>
__global__ void __launch_bounds__(32 * KS)
    k_level_ks(EllView<V> M, const T *__restrict__ u, const T *__restrict__ b,
               const T *__restrict__ dinv, T *d, T *x, T *y, ChebC c, const int *done) {
    using V2 = typename V2a<V>::type;
    __shared__ T red[KS][SLICE];
    pdl_wait();
    pdl_trigger();
    if (*done)
        return;
    const int w = blockIdx.x, q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    size_t base;
    int K;
    slice_span(M, w, base, K);
    base += 2 * lane;
    const int i0 = w * SLICE + 2 * lane;
    T a0 = 0, a1 = 0, s0 = 0, s1 = 0;
    if (DIFF) {  // the self entry (k = 0) holds the row sum; the others take u_j - u_i
        s0 = i0 < M.nrows ? __ldg(u + i0) : T(0);
        s1 = i0 + 1 < M.nrows ? __ldg(u + i0 + 1) : T(0);
    }
    bool packed = false;
    if constexpr (sizeof(V) == 4) {
        if (M.qv && M.qslice[w]) {  // k-paired values and 16-bit deltas, one entry at a time
            packed = true;
            const size_t qb = (size_t)w * ((K + 1) >> 1) * 32 + lane;
            const float *QV = reinterpret_cast<const float *>(M.qv + qb);
            const short *QD = reinterpret_cast<const short *>(M.qd + qb);
#pragma unroll 2
            for (int k = q; k < K; k += KS) {
                const size_t o = (size_t)(k >> 1) * 128 + (k & 1) * 2;
                const float2 v = ldop<EVF>(reinterpret_cast<const float2 *>(QV + o));
                const short2 cd = ldop<EVF>(reinterpret_cast<const short2 *>(QD + o));
                const T g0 = __ldg(u + i0 + cd.x), g1 = __ldg(u + i0 + 1 + cd.y);
                if (DIFF && k == 0) {
                    a0 = fma((T)v.x, s0, a0);
                    a1 = fma((T)v.y, s1, a1);
                } else {
                    a0 = fma((T)v.x, DIFF ? g0 - s0 : g0, a0);
                    a1 = fma((T)v.y, DIFF ? g1 - s1 : g1, a1);
                }
            }
        } else if (M.pk) {
            packed = true;
            const int4 *P = reinterpret_cast<const int4 *>(M.pk + base);
#pragma unroll 2
            for (int k = q; k < K; k += KS) {
                const int4 e = ldop<EVF>(P + (size_t)k * (SLICE / 2));
                const T g0 = __ldg(u + e.x), g1 = __ldg(u + e.z);
                if (DIFF && k == 0) {
                    a0 = fma((T)__int_as_float(e.y), s0, a0);
                    a1 = fma((T)__int_as_float(e.w), s1, a1);
                } else {
                    a0 = fma((T)__int_as_float(e.y), DIFF ? g0 - s0 : g0, a0);
                    a1 = fma((T)__int_as_float(e.w), DIFF ? g1 - s1 : g1, a1);
                }
            }
        }
    }
    if (!packed && M.dslice && M.dslice[w]) {  // 16-bit column deltas
        packed = true;
#pragma unroll 2
        for (int k = q; k < K; k += KS) {
            const size_t o = base + (size_t)k * SLICE;
            const short2 cd = ldop<EVF>(reinterpret_cast<const short2 *>(M.dcols + o));
            const V2 v = ldop<EVF>(reinterpret_cast<const V2 *>(M.vals + o));
            const T g0 = __ldg(u + i0 + cd.x), g1 = __ldg(u + i0 + 1 + cd.y);
            if (DIFF && k == 0) {
                a0 = fma((T)v.x, s0, a0);
                a1 = fma((T)v.y, s1, a1);
            } else {
                a0 = fma((T)v.x, DIFF ? g0 - s0 : g0, a0);
                a1 = fma((T)v.y, DIFF ? g1 - s1 : g1, a1);
            }
        }
    }
    if (!packed) {
#pragma unroll 2
        for (int k = q; k < K; k += KS) {
            const size_t o = base + (size_t)k * SLICE;
            const int2 cl = ldop<EVF>(reinterpret_cast<const int2 *>(M.cols + o));
            const V2 v = ldop<EVF>(reinterpret_cast<const V2 *>(M.vals + o));
            const T g0 = __ldg(u + cl.x), g1 = __ldg(u + cl.y);
            if (DIFF && k == 0) {
                a0 = fma((T)v.x, s0, a0);
                a1 = fma((T)v.y, s1, a1);
            } else {
                a0 = fma((T)v.x, DIFF ? g0 - s0 : g0, a0);
                a1 = fma((T)v.y, DIFF ? g1 - s1 : g1, a1);
            }
        }
    }
    red[q][2 * lane] = a0;
    red[q][2 * lane + 1] = a1;
    __syncthreads();
    if (q != 0)
        return;
    T t0 = 0, t1 = 0;
#pragma unroll
    for (int r = 0; r < KS; r++) {
        t0 += red[r][2 * lane];
        t1 += red[r][2 * lane + 1];
    }
    if (i0 < M.nrows)
        level_epilogue<T, EP>(i0, t0, b, dinv, d, x, y, c);
    if (i0 + 1 < M.nrows)
        level_epilogue<T, EP>(i0 + 1, t1, b, dinv, d, x, y, c);
}

// d = dinv b / theta (start of the pre-smoother from a zero guess)
template <class T>
__global__ void k_cheb_start(int n, const T *b, const T *dinv, T *d, T inv_theta, const int *done) {
    pdl_wait();
    pdl_trigger();
    if (*done)
        return;
    const int stride = gridDim.x * blockDim.x;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        d[i] = dinv[i] * b[i] * inv_theta;
}

// coarsest level: x = first nc entries of Cinv [b; 0] (one warp per row); with
// full = 1 all nc + 1 entries of Cinv [b; b_nc] (a one-level bordered hierarchy)
template <class T>
__global__ void k_coarse(int nc, const T *__restrict__ cinv, const T *__restrict__ b, T *x,
                         const int *done, int full) {
    pdl_wait();
    pdl_trigger();
    if (*done)
        return;
    const int row = gwarp_a(), lane = threadIdx.x & 31;
    if (row >= nc + full)
        return;
    const T *ci = cinv + (size_t)row * (nc + 1);
    T acc = 0;
    for (int j = lane; j < nc + full; j += 32)
        acc = fma(ci[j], b[j], acc);
    acc = warp_sum(acc);
    if (lane == 0)
        x[row] = acc;
}

static ChebC cheb_consts(double lmax, double ratio) {
    const double lmin = lmax / ratio;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta, rho0 = 1.0 / sigma, rho1 = 1.0 / (2.0 * sigma - rho0);
    ChebC c;
    c.theta = theta;
    c.inv_theta = 1.0 / theta;
    c.c1 = 1.0 + rho1 * rho0;
    c.c2 = 2.0 * rho1 / delta;
    c.c3 = rho1 * rho0;
    c.c4 = 2.0 * rho1 / delta;
    return c;
}

// Work vectors of one vector precision
template <class T> struct LvlVec;
template <> struct LvlVec<double> {
    static const double *dinv(const AmgLevel &L) { return L.dinv.p; }
    static double *b(AmgLevel &L) { return L.b.p; }
    static double *x(AmgLevel &L) { return L.x.p; }
    static double *d(AmgLevel &L) { return L.d.p; }
    static double *r(AmgLevel &L) { return L.r.p; }
    static const double *cinv(const Amg &a) { return a.cinv.p; }
};
template <> struct LvlVec<float> {
    static const float *dinv(const AmgLevel &L) { return L.dinv32.p; }
    static float *b(AmgLevel &L) { return L.b32.p; }
    static float *x(AmgLevel &L) { return L.x32.p; }
    static float *d(AmgLevel &L) { return L.d32.p; }
    static float *r(AmgLevel &L) { return L.r32.p; }
    static const float *cinv(const Amg &a) { return a.cinv32.p; }
};

// Stored operators of one value precision (DIFF: level operators in difference form)
template <class V, bool DIFF> struct LvlOps;
template <> struct LvlOps<double, false> {
    static EllView<double> A(const AmgLevel &L) { return L.A64; }
    static CsrView<double> Ac(const AmgLevel &L) { return {L.Ac.n, L.Ac.rp.p, L.Ac.ci.p, L.Ac.v64.p}; }
    static EllView<double> P(const AmgLevel &L) { return L.P.view64(); }
    static EllView<double> R(const AmgLevel &L) { return L.R.view64(); }
    static CsrView<double> Pc(const AmgLevel &L) { return {L.Pc.n, L.Pc.rp.p, L.Pc.ci.p, L.Pc.v64.p}; }
    static CsrView<double> Rc(const AmgLevel &L) { return {L.Rc.n, L.Rc.rp.p, L.Rc.ci.p, L.Rc.v64.p}; }
};
template <> struct LvlOps<float, false> {
    static EllView<float> A(const AmgLevel &L) { return L.A32; }
    static CsrView<float> Ac(const AmgLevel &L) { return {L.Ac.n, L.Ac.rp.p, L.Ac.ci.p, L.Ac.v32.p}; }
    static EllView<float> P(const AmgLevel &L) { return L.P.view32(); }
    static EllView<float> R(const AmgLevel &L) { return L.R.view32(); }
    static CsrView<float> Pc(const AmgLevel &L) { return {L.Pc.n, L.Pc.rp.p, L.Pc.ci.p, L.Pc.v32.p}; }
    static CsrView<float> Rc(const AmgLevel &L) { return {L.Rc.n, L.Rc.rp.p, L.Rc.ci.p, L.Rc.v32.p}; }
};
template <> struct LvlOps<float, true> : LvlOps<float, false> {
    static EllView<float> A(const AmgLevel &L) { return L.Ad32; }
    static CsrView<float> Ac(const AmgLevel &L) {
        return {L.Acd.n, L.Acd.rp.p, L.Acd.ci.p, L.Acd.v32.p, L.Acd.pk.p};
    }
};

static unsigned sblocks(int n) { return (unsigned)(((n + SLICE - 1) / SLICE + 7) / 8); }

// launch one fused level operation with the operator's tuned schedule
template <class T, class V, bool DIFF, int EP, bool EVF = false>
static int level_op(int mode, const EllView<V> &E, const CsrView<V> &Cv, const T *u, const T *b,
                    const T *dinv, T *d, T *x, T *y, const ChebC &c, const int *done,
                    cudaStream_t s) {
    const int n = E.nrows;
    const dim3 blk(256);
    cudaError_t e;
    switch (mode) {
    case 0: e = launch_pdl(k_level<T, V, DIFF, EVF, EP>, dim3(sblocks(n)), blk, s, E, u, b, dinv, d, x, y, c, done); break;
    case 1: e = launch_pdl(k_level_csr<T, V, 4, DIFF, EVF, EP>, dim3((unsigned)((n * 4 + 255) / 256)), blk, s, Cv, u, b, dinv, d, x, y, c, done); break;
    case 2: e = launch_pdl(k_level_csr<T, V, 8, DIFF, EVF, EP>, dim3((unsigned)((n * 8 + 255) / 256)), blk, s, Cv, u, b, dinv, d, x, y, c, done); break;
    case 3: e = launch_pdl(k_level_csr<T, V, 16, DIFF, EVF, EP>, dim3((unsigned)((n * 16 + 255) / 256)), blk, s, Cv, u, b, dinv, d, x, y, c, done); break;
    case 4: e = launch_pdl(k_level_csr<T, V, 32, DIFF, EVF, EP>, dim3((unsigned)(((size_t)n * 32 + 255) / 256)), blk, s, Cv, u, b, dinv, d, x, y, c, done); break;
    case 5: e = launch_pdl(k_level_ks<T, V, DIFF, EVF, EP, 8>, dim3((unsigned)((n + SLICE - 1) / SLICE)), dim3(256), s, E, u, b, dinv, d, x, y, c, done); break;
    case 6: e = launch_pdl(k_level_ks<T, V, DIFF, EVF, EP, 4>, dim3((unsigned)((n + SLICE - 1) / SLICE)), dim3(128), s, E, u, b, dinv, d, x, y, c, done); break;
    default: e = launch_pdl(k_level_ks<T, V, DIFF, EVF, EP, 2>, dim3((unsigned)((n + SLICE - 1) / SLICE)), dim3(64), s, E, u, b, dinv, d, x, y, c, done); break;
    }
    if (e != cudaSuccess)
        return fail(MP_CUDA_ERROR, "multigrid launch: %s", cudaGetErrorString(e));
    MP_CHECK_LAUNCH();
    return MP_OK;
}

// level_op with the load policy of level l (evict first on the finest level)
template <class T, class V, bool DIFF, int EP>
static int level_op_at(size_t l, int mode, const EllView<V> &E, const CsrView<V> &Cv, const T *u,
                       const T *b, const T *dinv, T *d, T *x, T *y, const ChebC &c,
                       const int *done, cudaStream_t s) {
    if (l == 0)
        return level_op<T, V, DIFF, EP, true>(mode, E, Cv, u, b, dinv, d, x, y, c, done, s);
    return level_op<T, V, DIFF, EP, false>(mode, E, Cv, u, b, dinv, d, x, y, c, done, s);
}

// V(1,1) cycle from level l: T vectors, V stored values, DIFF level operators.
// head_ready: d = dinv b / theta, the first step of the pre-smoother from a zero
// guess, was written by whoever wrote b (the coarser levels' by the restriction
// epilogue; level 0's by the Krylov update that produced the preconditioner input,
// see amg_head), otherwise a kernel forms it here.
template <class T, class V, bool DIFF>
static int vcycle(const Amg &a, size_t l, const T *b, T *x, const int *done, bool head_ready,
                  cudaStream_t s) {
    using LV = LvlVec<T>;
    using LO = LvlOps<V, DIFF>;
    AmgLevel &L = *a.L[l];
    if (l + 1 == a.L.size()) {
        const int full = (l == 0 && a.coarse_bordered) ? 1 : 0;
        const cudaError_t e = launch_pdl(k_coarse<T>, dim3((unsigned)((a.nc + full + 7) / 8)),
                                         dim3(256), s, a.nc, LV::cinv(a), b, x, done, full);
        if (e != cudaSuccess)
            return fail(MP_CUDA_ERROR, "multigrid launch: %s", cudaGetErrorString(e));
        MP_CHECK_LAUNCH();
        return MP_OK;
    }
    AmgLevel &N = *a.L[l + 1];
    const ChebC c = cheb_consts(L.lmax, a.cheb_ratio);
    const EllView<V> A = LO::A(L);
    const CsrView<V> Ac = LO::Ac(L), Pc = LO::Pc(L), Rc = LO::Rc(L);
    const T *dinv = LV::dinv(L);
    T *d = LV::d(L), *r = LV::r(L);
    // the finest operator keeps one warp per slice: timed cold, the split schedules
    // come within a few percent of it and the tuner picked them at times, but inside
    // the cycle they ran slower (38-42 against 32-35 us per pass at 1M nodes)
    const int mA = l == 0 ? 0 : L.sA.mode;
    if (!head_ready) {
        const unsigned vb = (unsigned)std::min((L.n + 255) / 256, sm_count() * 8);
        const cudaError_t e = launch_pdl(k_cheb_start<T>, dim3(vb), dim3(256), s, L.n, b, dinv, d,
                                         (T)c.inv_theta, done);
        if (e != cudaSuccess)
            return fail(MP_CUDA_ERROR, "multigrid launch: %s", cudaGetErrorString(e));
        MP_CHECK_LAUNCH();
    }
    MP_TRY((level_op_at<T, V, DIFF, EP_CHEB_PRE>(l, mA, A, Ac, d, b, dinv, d, x, nullptr, c, done, s)));
    for (int k = 1; k < a.sweeps; k++) {  // further pre-smoothing from the current x
        MP_TRY((level_op_at<T, V, DIFF, EP_CHEB_POST1>(l, mA, A, Ac, x, b, dinv, d, x, nullptr, c, done, s)));
        MP_TRY((level_op_at<T, V, DIFF, EP_CHEB_POST2>(l, mA, A, Ac, d, b, dinv, d, x, nullptr, c, done, s)));
    }
    MP_TRY((level_op_at<T, V, DIFF, EP_RESID>(l, mA, A, Ac, x, b, dinv, d, x, r, c, done, s)));
    // restriction; unless the next level is the coarsest (a direct solve), it also
    // starts that level's pre-smoother
    const bool next_smooths = l + 2 < a.L.size();
    if (next_smooths) {
        const ChebC cn = cheb_consts(N.lmax, a.cheb_ratio);
        MP_TRY((level_op_at<T, V, false, EP_RESTRICT>(l, L.sR.mode, LO::R(L), Rc, r, nullptr,
                                                      LV::dinv(N), LV::d(N), nullptr, LV::b(N),
                                                      cn, done, s)));
    } else {
        MP_TRY((level_op_at<T, V, false, EP_PLAIN>(l, L.sR.mode, LO::R(L), Rc, r, nullptr, nullptr,
                                                   nullptr, nullptr, LV::b(N), c, done, s)));
    }
    MP_TRY((vcycle<T, V, DIFF>(a, l + 1, LV::b(N), LV::x(N), done, next_smooths, s)));
    MP_TRY((level_op_at<T, V, false, EP_PROLONG>(l, L.sP.mode, LO::P(L), Pc, LV::x(N), nullptr,
                                                 nullptr, nullptr, x, nullptr, c, done, s)));
    for (int k = 0; k < a.sweeps; k++) {
        MP_TRY((level_op_at<T, V, DIFF, EP_CHEB_POST1>(l, mA, A, Ac, x, b, dinv, d, x, nullptr, c, done, s)));
        MP_TRY((level_op_at<T, V, DIFF, EP_CHEB_POST2>(l, mA, A, Ac, d, b, dinv, d, x, nullptr, c, done, s)));
    }
    return MP_OK;
}

template <class T>
int amg_apply(const Amg &a, const T *in, T *out, const int *done, cudaStream_t s,
              bool head_ready) {
    if (a.L.size() < 2)
        head_ready = false;
    if constexpr (std::is_same<T, double>::value) {
        if (a.store == AMG_MG32)
            return vcycle<double, float, true>(a, 0, in, out, done, head_ready, s);
        return vcycle<double, double, false>(a, 0, in, out, done, head_ready, s);
    } else {
        return vcycle<float, float, true>(a, 0, in, out, done, head_ready, s);
    }
}
template int amg_apply<double>(const Amg &, const double *, double *, const int *, cudaStream_t,
                               bool);
template int amg_apply<float>(const Amg &, const float *, float *, const int *, cudaStream_t,
                              bool);

template <class T> AmgHead<T> amg_head(const Amg &a) {
    AmgHead<T> h{};
    if (a.L.size() < 2)
        return h;
    const AmgLevel &L = *a.L[0];
    h.d = LvlVec<T>::d(const_cast<AmgLevel &>(L));
    h.dinv = LvlVec<T>::dinv(L);
    h.inv_theta = (T)cheb_consts(L.lmax, a.cheb_ratio).inv_theta;
    return h;
}
template AmgHead<double> amg_head<double>(const Amg &);
template AmgHead<float> amg_head<float>(const Amg &);

// ------------------------------------------------------- field filter
__global__ void k_filter_scale(int n, double *s) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        s[i] = s[i] != 0.0 ? 1.0 / s[i] : 0.0;
}

__global__ void k_scale_vec(int n, const double *s, double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        v[i] *= s[i];
}

__global__ void k_fill(int n, double v, double *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        x[i] = v;
}

int amg_filter_size(const Amg &a) { return a.L.size() > 1 ? a.L[1]->n : 0; }

int amg_filter_setup(const Amg &a, double *scale1, cudaStream_t s) {
    if (a.L.size() < 2)
        return MP_OK;
    const AmgLevel &L = *a.L[0];
    dbuf<double> ones;
    MP_TRY(ones.alloc(L.n));
    k_fill<<<(L.n + 255) / 256, 256, 0, s>>>(L.n, 1.0, ones.p);
    MP_CHECK_LAUNCH();
    const ChebC c{};
    const CsrView<double> Rc{L.Rc.n, L.Rc.rp.p, L.Rc.ci.p, L.Rc.v64.p};
    MP_TRY((level_op<double, double, false, EP_PLAIN, true>(L.sR.mode, L.R.view64(), Rc, ones.p, nullptr,
                                                      nullptr, nullptr, nullptr, scale1, c,
                                                      a.zero_flag.p, s)));
    const int n1 = a.L[1]->n;
    k_filter_scale<<<(n1 + 255) / 256, 256, 0, s>>>(n1, scale1);
    MP_CHECK_LAUNCH();
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

int amg_filter(const Amg &a, const double *c, double *work1, const double *scale1, double *out,
               cudaStream_t s) {
    if (a.L.size() < 2)
        return MP_OK;
    const AmgLevel &L = *a.L[0];
    const ChebC k{};
    const CsrView<double> Rc{L.Rc.n, L.Rc.rp.p, L.Rc.ci.p, L.Rc.v64.p};
    const CsrView<double> Pc{L.Pc.n, L.Pc.rp.p, L.Pc.ci.p, L.Pc.v64.p};
    MP_TRY((level_op<double, double, false, EP_PLAIN, true>(L.sR.mode, L.R.view64(), Rc, c, nullptr,
                                                      nullptr, nullptr, nullptr, work1, k,
                                                      a.zero_flag.p, s)));
    const int n1 = a.L[1]->n;
    k_scale_vec<<<(n1 + 255) / 256, 256, 0, s>>>(n1, scale1, work1);
    MP_CHECK_LAUNCH();
    MP_TRY((level_op<double, double, false, EP_PLAIN, true>(L.sP.mode, L.P.view64(), Pc, work1, nullptr,
                                                      nullptr, nullptr, nullptr, out, k,
                                                      a.zero_flag.p, s)));
    return MP_OK;
}

// ------------------------------------------------------------- autotuner
// For each level operator and transfer, time y = M u with every schedule
// (sliced ELL with one warp or 8 / 4 / 2 warps per slice, CSR with 4/8/16/32 lanes
// per row) in the precision and form the cycle will run (FP64; FP32; FP32
// difference form for the MG32 level operators) and keep the fastest.  Each timed
// launch starts with L2 flushed (a write larger than L2), as inside the cycle,
// where the finer levels' traffic evicts a coarse operator between its uses; an
// operator timed warm from L2 ranks the schedules differently.  The mean of the
// middle five of nine launches decides.
template <class T, class V, bool DIFF>
static int tune_one(size_t l, const EllView<V> &E, const CsrView<V> &Cv, int ncols, bool allow_sell,
                    OpSched &out, const int *zero, dbuf<char> &flush, cudaStream_t s) {
    const bool csr = Cv.nrows > 0;  // level 0 has no CSR copy: sliced-ELL schedules only
    const int n = csr ? Cv.nrows : E.nrows;
    if (!n || (!csr && !allow_sell)) {
        out.mode = 0;
        return MP_OK;
    }
    dbuf<T> u, y;
    MP_TRY(u.alloc(std::max(ncols, 1)));
    MP_TRY(y.alloc(std::max(n, 1)));
    MP_CUDA(cudaMemsetAsync(u.p, 0, sizeof(T) * u.n, s));
    cudaEvent_t e0, e1;
    MP_CUDA(cudaEventCreate(&e0));
    MP_CUDA(cudaEventCreate(&e1));
    const ChebC c{};
    const bool sell = allow_sell && (E.vals || E.pk);
    // the event clock ticks in steps of about 2 us, as long as a coarse level's launch:
    // the mean of the middle of 9 cold launches resolves what one reading cannot
    constexpr int REPS = 9, TRIM = 2;
    float best = 1e30f;
    int rc = MP_OK;
    for (int mode = sell ? 0 : 1; mode < (sell ? OP_MODES : 5) && rc == MP_OK; mode++) {
        if (!csr && mode >= 1 && mode <= 4)
            continue;
        float t[REPS];
        for (int rep = 0; rep < REPS && rc == MP_OK; rep++) {
            cudaMemsetAsync(flush.p, rep & 0xff, flush.n, s);
            cudaEventRecord(e0, s);
            rc = level_op_at<T, V, DIFF, EP_PLAIN>(l, mode, E, Cv, u.p, nullptr, nullptr, nullptr,
                                                nullptr, y.p, c, zero, s);
            cudaEventRecord(e1, s);
            cudaEventSynchronize(e1);
            t[rep] = 0;
            cudaEventElapsedTime(&t[rep], e0, e1);
        }
        std::sort(t, t + REPS);
        float ms = 0.f;
        for (int r = TRIM; r < REPS - TRIM; r++)
            ms += t[r];
        ms /= (float)(REPS - 2 * TRIM);
        out.us[mode] = ms * 1e3f;
        if (ms < best) {
            best = ms;
            out.mode = mode;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

// Schedules already tuned in this process, keyed by the hierarchy's shape (device,
// store, level, rows and entries of each operator): a second solver on the same
// operator (another precision's twin, a restarted run) reuses them, so that both
// sum in the same order and reproduce each other's iteration counts.
struct TuneKey {
    int dev, store, level, n, next;
    size_t nnzA, nnzP, nnzR;
    bool operator<(const TuneKey &o) const {
        return std::tie(dev, store, level, n, next, nnzA, nnzP, nnzR) <
               std::tie(o.dev, o.store, o.level, o.n, o.next, o.nnzA, o.nnzP, o.nnzR);
    }
};
struct TuneVal {
    OpSched A, P, R;
};
static std::mutex g_tune_mu;
static std::map<TuneKey, TuneVal> g_tuned;

template <class T, class V, bool DIFF> static int tune_levels(Amg &a, cudaStream_t s) {
    using LO = LvlOps<V, DIFF>;
    using LT = LvlOps<V, false>;
    const int *z = a.zero_flag.p;
    int dev = 0;
    MP_CUDA(cudaGetDevice(&dev));
    dbuf<char> flush;  // larger than the 126 MB L2; allocated on the first miss
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (size_t l = 0; l + 1 < a.L.size(); l++) {
        AmgLevel &L = *a.L[l];
        const TuneKey key{dev,          a.store,       (int)l,        L.n,          a.L[l + 1]->n,
                          L.Ac.ci.n,    L.Pc.ci.n,     L.Rc.ci.n};
        const auto hit = g_tuned.find(key);
        if (hit != g_tuned.end()) {
            L.sA = hit->second.A;
            L.sP = hit->second.P;
            L.sR = hit->second.R;
            continue;
        }
        if (!flush.p)
            MP_TRY(flush.alloc((size_t)192 << 20));
        if (l > 0)
            MP_TRY((tune_one<T, V, DIFF>(l, LO::A(L), LO::Ac(L), L.n, true, L.sA, z, flush, s)));
        MP_TRY((tune_one<T, V, false>(l, LT::P(L), LT::Pc(L), a.L[l + 1]->n, true, L.sP, z, flush, s)));
        MP_TRY((tune_one<T, V, false>(l, LT::R(L), LT::Rc(L), L.n, true, L.sR, z, flush, s)));
        g_tuned[key] = TuneVal{L.sA, L.sP, L.sR};
    }
    return MP_OK;
}

static int amg_autotune(Amg &a, cudaStream_t s) {
    MP_TRY(a.zero_flag.alloc(1));
    MP_CUDA(cudaMemsetAsync(a.zero_flag.p, 0, sizeof(int), s));
    if (a.store == AMG_MG32)
        return tune_levels<double, float, true>(a, s);
    if (a.store == AMG_F32)
        return tune_levels<float, float, true>(a, s);
    return tune_levels<double, double, false>(a, s);
}

}  // namespace mp
