// ref_knn.cpp -- test infrastructure: builds MeMPhyS stencils with the
// reference's own vendored nanoflann.hpp (header_files/nanoflann.hpp, v1.3.2),
// following the rule of CLOUD::calc_cloud_points_fast (cloud.cpp:570-648):
// one KD-tree over all nodes for interior queries, and one where boundary
// nodes sit at +infinity for boundary queries (self + n-1 interior nodes).
// Used only to pin the oracle's kNN; never linked into the product.
//
// usage: ref_knn <in.bin> <out.bin>
//   in:  int32 nv, int32 dim, int32 n, float64 xyz[nv*dim], uint8 bflag[nv]
//   out: int32 nb_col[nv*n]
#include <cstdio>
#include <cstdint>
#include <limits>
#include <vector>
#include "nanoflann.hpp"

struct Cloud3 {
    struct P { double x, y, z; };
    std::vector<P> pts;
    size_t kdtree_get_point_count() const { return pts.size(); }
    double kdtree_get_pt(size_t i, size_t d) const { return d == 0 ? pts[i].x : (d == 1 ? pts[i].y : pts[i].z); }
    template <class B> bool kdtree_get_bbox(B &) const { return false; }
};

typedef nanoflann::KDTreeSingleIndexAdaptor<nanoflann::L2_Simple_Adaptor<double, Cloud3>, Cloud3, 3> Tree;

int main(int argc, char **argv)
{
    if (argc != 3) return 2;
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int32_t hdr[3];
    if (std::fread(hdr, 4, 3, f) != 3) return 4;
    int nv = hdr[0], dim = hdr[1], n = hdr[2];
    std::vector<double> xyz((size_t)nv * dim);
    std::vector<uint8_t> bflag(nv);
    if (std::fread(xyz.data(), 8, xyz.size(), f) != xyz.size()) return 5;
    if (std::fread(bflag.data(), 1, nv, f) != (size_t)nv) return 6;
    std::fclose(f);
    Cloud3 all, interior;
    all.pts.resize(nv);
    interior.pts.resize(nv);
    const double inf = std::numeric_limits<double>::infinity();
    for (int i = 0; i < nv; i++) {
        Cloud3::P p{xyz[(size_t)dim * i], xyz[(size_t)dim * i + 1], dim == 3 ? xyz[(size_t)dim * i + 2] : 0.0};
        all.pts[i] = p;
        interior.pts[i] = bflag[i] ? Cloud3::P{inf, inf, inf} : p;
    }
    Tree t_all(3, all, nanoflann::KDTreeSingleIndexAdaptorParams(10));
    t_all.buildIndex();
    Tree t_int(3, interior, nanoflann::KDTreeSingleIndexAdaptorParams(10));
    t_int.buildIndex();
    std::vector<int32_t> out((size_t)nv * n);
    std::vector<size_t> idx(n);
    std::vector<double> dist(n);
    for (int i = 0; i < nv; i++) {
        double q[3] = {all.pts[i].x, all.pts[i].y, all.pts[i].z};
        int32_t *o = out.data() + (size_t)i * n;
        if (bflag[i]) {
            t_int.knnSearch(q, n, idx.data(), dist.data());
            o[0] = i;
            for (int k = 0; k < n - 1; k++) o[k + 1] = (int32_t)idx[k];
        } else {
            t_all.knnSearch(q, n, idx.data(), dist.data());
            for (int k = 0; k < n; k++) o[k] = (int32_t)idx[k];
        }
    }
    f = std::fopen(argv[2], "wb");
    if (!f) return 7;
    std::fwrite(out.data(), 4, out.size(), f);
    std::fclose(f);
    return 0;
}
