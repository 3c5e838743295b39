// mp_cloud.cu -- CLOUD (cloud.cpp:29-48) resident on the GPU: kNN stencils,
// PHS-RBF-FD weights, and the sliced operator storage built from them.
#include "mp_cloud.cuh"

namespace mp {
int knn_device(const double *d_xyz, const uint8_t *d_bflag, int nv, int dim, int n, int *d_nb,
               cudaStream_t s);
int cloud_weights_device(const double *d_xyz, int nv, int dim, const int *d_nb, int n, int phs,
                         int poly_deg, double *gx, double *gy, double *gz, double *lap,
                         double *cond, cudaStream_t s);
}  // namespace mp

using namespace mp;

struct mp_cloud_s {
    int nv = 0, n = 0, dim = 0, phs = 3, poly = 3;
    dbuf<double> xyz;
    dbuf<uint8_t> bflag;
    dbuf<int> nb_rm;
    std::shared_ptr<Ell> cols = std::make_shared<Ell>();
    Ell ops[4];  // gx, gy, gz, lap (values only; columns in `cols`)
    dbuf<double> cond;
    bool has_cond = false;
};

namespace mp {

// row-major weights -> sliced values
__global__ void pack_vals(int nrows, int nrows_pad, int K, const double *rm, double *sl) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrows_pad * K)
        return;
    int row = (int)(t / K), k = (int)(t % K);
    sl[ell_index(row, k, K)] = row < nrows ? rm[t] : 0.0;
}

__global__ void unpack_vals(int nrows, int K, const double *sl, double *rm) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nrows * K)
        return;
    int row = (int)(t / K), k = (int)(t % K);
    rm[t] = sl[ell_index(row, k, K)];
}

__global__ void masked_copy(int nrows, int K, const double *src, const uint8_t *bflag, int rows,
                            double *dst) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t total = (size_t)ell_padded_rows(nrows) * K;
    if (t >= total)
        return;
    // t indexes the sliced array directly: recover the row
    size_t slice = t / ((size_t)K * SLICE);
    int row = (int)(slice * SLICE + (t % SLICE));
    bool keep = row < nrows;
    if (keep && rows == MP_ROWS_INTERNAL)
        keep = !bflag[row];
    if (keep && rows == MP_ROWS_BOUNDARY)
        keep = bflag[row] != 0;
    dst[t] = keep ? src[t] : 0.0;
}

CloudView cloud_view(mp_cloud_s *c) {
    CloudView v;
    v.nv = c->nv;
    v.n = c->n;
    v.dim = c->dim;
    v.cols = c->cols->cols.p;
    for (int i = 0; i < 4; i++)
        v.w[i] = c->ops[i].v64.p;
    v.bflag = c->bflag.p;
    v.nb_rm = c->nb_rm.p;
    return v;
}

const double *cloud_xyz(mp_cloud_s *c) { return c->xyz.p; }

const Ell *cloud_operator(mp_cloud_s *c, int which) {
    if (which < 0 || which > 3 || !c->ops[which].v64.p)
        return nullptr;
    return &c->ops[which];
}

std::shared_ptr<Ell> cloud_cols(mp_cloud_s *c) { return c->cols; }

int cloud_masked_copy(mp_cloud_s *c, int which, int rows, double *dst, cudaStream_t s) {
    const Ell *E = cloud_operator(c, which);
    if (!E)
        return fail(MP_BAD_ARG, "operator %d not available", which);
    if (rows < MP_ROWS_ALL || rows > MP_ROWS_BOUNDARY)
        return fail(MP_BAD_ARG, "row mask %d", rows);
    size_t total = (size_t)ell_padded_rows(c->nv) * c->n;
    masked_copy<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(c->nv, c->n, E->v64.p, c->bflag.p,
                                                                rows, dst);
    MP_CHECK_LAUNCH();
    return MP_OK;
}

static int cloud_finish(mp_cloud_s *c, int compute_cond, cudaStream_t s) {
    const int nv = c->nv, n = c->n, dim = c->dim;
    const size_t rm = (size_t)nv * n;
    dbuf<double> w[4];
    for (int i = 0; i < 4; i++)
        if (i != 2 || dim == 3)
            MP_TRY(w[i].alloc(rm));
    if (compute_cond) {
        MP_TRY(c->cond.alloc(nv));
        c->has_cond = true;
    }
    int st = cloud_weights_device(c->xyz.p, nv, dim, c->nb_rm.p, n, c->phs, c->poly, w[0].p,
                                  w[1].p, w[2].p, w[3].p, compute_cond ? c->cond.p : nullptr, s);
    if (st != MP_OK)
        return st;
    // stencil columns and weights into slices
    MP_TRY(ell_create(*c->cols, nv, nv, n, c->nb_rm.p, nullptr, false, s));
    const int np = ell_padded_rows(nv);
    const size_t tot = (size_t)np * n;
    for (int i = 0; i < 4; i++) {
        if (!w[i].p)
            continue;
        Ell &E = c->ops[i];
        E.nrows = nv;
        E.ncols = nv;
        E.K = n;
        MP_TRY(E.v64.alloc(tot));
        pack_vals<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(nv, np, n, w[i].p, E.v64.p);
        MP_CHECK_LAUNCH();
    }
    MP_CUDA(cudaStreamSynchronize(s));
    return MP_OK;
}

}  // namespace mp

extern "C" int mp_cloud_create_stencils(const double *xyz, const uint8_t *boundary, int nv, int dim,
                                        const int *nb_col, int n, int phs_deg, int poly_deg,
                                        int compute_cond, mp_stream s, mp_cloud *out) {
    if (!xyz || !boundary || !nb_col || !out || nv <= 0 || n < 2 || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_cloud_create_stencils: bad arguments");
    cudaStream_t st = S(s);
    mp_cloud c = new mp_cloud_s;
    c->nv = nv;
    c->n = n;
    c->dim = dim;
    c->phs = phs_deg;
    c->poly = poly_deg;
    int rc = MP_OK;
    if ((rc = c->xyz.alloc((size_t)nv * dim)) != MP_OK || (rc = c->bflag.alloc(nv)) != MP_OK ||
        (rc = c->nb_rm.alloc((size_t)nv * n)) != MP_OK) {
        delete c;
        return rc;
    }
    cudaMemcpyAsync(c->xyz.p, xyz, sizeof(double) * nv * dim, cudaMemcpyDefault, st);
    cudaMemcpyAsync(c->bflag.p, boundary, nv, cudaMemcpyDefault, st);
    cudaMemcpyAsync(c->nb_rm.p, nb_col, sizeof(int) * nv * n, cudaMemcpyDefault, st);
    rc = cloud_finish(c, compute_cond, st);
    if (rc != MP_OK && rc != MP_SINGULAR_STENCIL) {
        delete c;
        return rc;
    }
    *out = c;
    return rc;
}

extern "C" int mp_cloud_create(const double *xyz, const uint8_t *boundary, int nv, int dim,
                               int phs_deg, int poly_deg, double mult, int compute_cond,
                               mp_stream s, mp_cloud *out) {
    if (!xyz || !boundary || !out || nv <= 0 || (dim != 2 && dim != 3))
        return fail(MP_BAD_ARG, "mp_cloud_create: bad arguments");
    if (poly_deg < 2 || poly_deg > 15)  // parameters.cpp:84-88
        return fail(MP_BAD_ARG, "poly_deg should be in range [2, 15]; current value: %d", poly_deg);
    const int n = mp_cloud_size(dim, poly_deg, mult);
    if (n < 2 || n > nv)
        return fail(MP_BAD_ARG, "cloud size %d for %d nodes", n, nv);
    cudaStream_t st = S(s);
    mp_cloud c = new mp_cloud_s;
    c->nv = nv;
    c->n = n;
    c->dim = dim;
    c->phs = phs_deg;
    c->poly = poly_deg;
    int rc = MP_OK;
    if ((rc = c->xyz.alloc((size_t)nv * dim)) != MP_OK || (rc = c->bflag.alloc(nv)) != MP_OK ||
        (rc = c->nb_rm.alloc((size_t)nv * n)) != MP_OK) {
        delete c;
        return rc;
    }
    cudaMemcpyAsync(c->xyz.p, xyz, sizeof(double) * nv * dim, cudaMemcpyDefault, st);
    cudaMemcpyAsync(c->bflag.p, boundary, nv, cudaMemcpyDefault, st);
    rc = knn_device(c->xyz.p, c->bflag.p, nv, dim, n, c->nb_rm.p, st);
    if (rc == MP_OK || rc == MP_SINGULAR_STENCIL)
        rc = cloud_finish(c, compute_cond, st);
    if (rc != MP_OK && rc != MP_SINGULAR_STENCIL) {
        delete c;
        return rc;
    }
    *out = c;
    return rc;
}

extern "C" int mp_cloud_info(mp_cloud c, int *nv, int *n, int *dim) {
    if (!c)
        return fail(MP_BAD_ARG, "null cloud");
    if (nv)
        *nv = c->nv;
    if (n)
        *n = c->n;
    if (dim)
        *dim = c->dim;
    return MP_OK;
}

extern "C" int mp_cloud_get(mp_cloud c, int *nb_col, double *gx, double *gy, double *gz,
                            double *lap, double *cond, mp_stream s) {
    if (!c)
        return fail(MP_BAD_ARG, "null cloud");
    cudaStream_t st = S(s);
    const size_t rm = (size_t)c->nv * c->n;
    if (nb_col)
        MP_CUDA(cudaMemcpyAsync(nb_col, c->nb_rm.p, sizeof(int) * rm, cudaMemcpyDefault, st));
    double *outs[4] = {gx, gy, gz, lap};
    dbuf<double> tmp;
    for (int i = 0; i < 4; i++) {
        if (!outs[i])
            continue;
        if (!c->ops[i].v64.p)
            return fail(MP_BAD_ARG, "operator %d not available (2D cloud has no grad_z)", i);
        double *dst = outs[i];
        bool host = !is_device_ptr(dst);
        if (host) {
            if (!tmp.p)
                MP_TRY(tmp.alloc(rm));
            dst = tmp.p;
        }
        unpack_vals<<<(unsigned)((rm + 255) / 256), 256, 0, st>>>(c->nv, c->n, c->ops[i].v64.p, dst);
        MP_CHECK_LAUNCH();
        if (host) {
            MP_CUDA(cudaMemcpyAsync(outs[i], tmp.p, sizeof(double) * rm, cudaMemcpyDeviceToHost, st));
            MP_CUDA(cudaStreamSynchronize(st));
        }
    }
    if (cond) {
        if (!c->has_cond)
            return fail(MP_BAD_ARG, "cloud was created without condition numbers");
        MP_CUDA(cudaMemcpyAsync(cond, c->cond.p, sizeof(double) * c->nv, cudaMemcpyDefault, st));
    }
    MP_CUDA(cudaStreamSynchronize(st));
    return MP_OK;
}

extern "C" int mp_cloud_destroy(mp_cloud c) {
    delete c;
    return MP_OK;
}
