// Point and clustering helpers of the opp_* API that the apps include through their defs
// headers (apps_codegen/app_fempic_cg/fempic_defs.h includes "opp_cluster.h"; the interface is
// opp_lib/include/opp_cluster.h's).  The mesh loader reads cell centroids through
// opp::Point3D / opp::getTetraCentroid3D; the block and k-means clusterings and the triangle
// test only colour meshes for a multi-rank partition (fempic_misc_mesh_colour.h, MPI builds),
// which a one-GPU run does not do, so they are kept simple.
#ifndef OPP_CLUSTER_H
#define OPP_CLUSTER_H

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <vector>

namespace opp {

// Three coordinates, laid out as double[3] (the apps reinterpret node position arrays as it).
struct Point3D {
    double x = 0.0;
    double y = 0.0;
    double z = 0.0;
    bool operator==(const Point3D& o) const { return x == o.x && y == o.y && z == o.z; }
};

inline Point3D getTetraCentroid3D(const Point3D& a, const Point3D& b, const Point3D& c, const Point3D& d) {
    return Point3D{(a.x + b.x + c.x + d.x) / 4.0, (a.y + b.y + c.y + d.y) / 4.0, (a.z + b.z + c.z + d.z) / 4.0};
}

inline Point3D getTriangleCentroid3D(const Point3D& a, const Point3D& b, const Point3D& c) {
    return Point3D{(a.x + b.x + c.x) / 3.0, (a.y + b.y + c.y) / 3.0, (a.z + b.z + c.z) / 3.0};
}

// Whether p lies in triangle (a, b, c) projected on the x-y plane (edges included): the three
// signed areas of p with each edge share one sign.
inline bool isPointInTriangle(const Point3D& p, const Point3D& a, const Point3D& b, const Point3D& c) {
    auto side = [](const Point3D& u, const Point3D& v, const Point3D& w) {
        return (v.x - u.x) * (w.y - u.y) - (w.x - u.x) * (v.y - u.y);
    };
    const double s0 = side(a, b, p), s1 = side(b, c, p), s2 = side(c, a, p);
    const bool neg = s0 < 0 || s1 < 0 || s2 < 0, pos = s0 > 0 || s1 > 0 || s2 > 0;
    return !(neg && pos);
}

// Points split into n_clusters slabs of equal count along the axis of largest extent.
inline std::vector<int> BlockCluster(const std::vector<Point3D>& pts, int n_clusters) {
    std::vector<int> out(pts.size(), 0);
    if (pts.empty() || n_clusters <= 1) return out;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (const Point3D& p : pts) {
        const double v[3] = {p.x, p.y, p.z};
        for (int d = 0; d < 3; d++) lo[d] = std::min(lo[d], v[d]), hi[d] = std::max(hi[d], v[d]);
    }
    int axis = 0;
    for (int d = 1; d < 3; d++)
        if (hi[d] - lo[d] > hi[axis] - lo[axis]) axis = d;
    std::vector<size_t> order(pts.size());
    std::iota(order.begin(), order.end(), 0);
    auto key = [&](size_t i) { return axis == 0 ? pts[i].x : axis == 1 ? pts[i].y : pts[i].z; };
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key(a) < key(b); });
    for (size_t r = 0; r < order.size(); r++) out[order[r]] = (int)(r * (size_t)n_clusters / order.size());
    return out;
}

// Lloyd's k-means from evenly spaced seeds, at most 100 rounds.
inline std::vector<int> kMeansClustering3D(const std::vector<Point3D>& pts, int n_clusters) {
    std::vector<int> out(pts.size(), 0);
    if (pts.empty() || n_clusters <= 1) return out;
    const size_t k = std::min((size_t)n_clusters, pts.size());
    std::vector<Point3D> ctr(k);
    for (size_t c = 0; c < k; c++) ctr[c] = pts[c * pts.size() / k];
    for (int round = 0; round < 100; round++) {
        bool changed = false;
        for (size_t i = 0; i < pts.size(); i++) {
            int best = 0;
            double bd = std::numeric_limits<double>::max();
            for (size_t c = 0; c < k; c++) {
                const double dx = pts[i].x - ctr[c].x, dy = pts[i].y - ctr[c].y, dz = pts[i].z - ctr[c].z;
                const double d2 = dx * dx + dy * dy + dz * dz;
                if (d2 < bd) bd = d2, best = (int)c;
            }
            changed |= out[i] != best;
            out[i] = best;
        }
        if (!changed && round > 0) break;
        std::vector<Point3D> sum(k);
        std::vector<size_t> cnt(k, 0);
        for (size_t i = 0; i < pts.size(); i++) {
            sum[out[i]].x += pts[i].x, sum[out[i]].y += pts[i].y, sum[out[i]].z += pts[i].z;
            cnt[out[i]]++;
        }
        for (size_t c = 0; c < k; c++)
            if (cnt[c]) ctr[c] = Point3D{sum[c].x / cnt[c], sum[c].y / cnt[c], sum[c].z / cnt[c]};
    }
    return out;
}

}  // namespace opp

#endif  // OPP_CLUSTER_H
