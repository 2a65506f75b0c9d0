// Test infrastructure only: a C-ABI shim around the UNMODIFIED reference
// euclidean_cluster kernel (src/CPU/euclidean_cluster/kernel.cpp), compiled
// from its own source file where it lies in the reference tree (the path is
// passed in as REF_KERNEL by oracle/Makefile); nothing of it is copied here.
// Loaded only by tests and the golden-fixture script; the product never does.
#include <cstdint>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <vector>
#include <algorithm>

#define private public
#define protected public
#include REF_KERNEL
#undef private
#undef protected

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
void load(PointCloud &c, const float *xyz, int n) {
    c.resize(n);
    for (int i = 0; i < n; ++i) {
        c[i].x = xyz[3 * i];
        c[i].y = xyz[3 * i + 1];
        c[i].z = xyz[3 * i + 2];
    }
}
}  // namespace

// extract() (kernel.cpp:635-647): clusters of one cloud at one tolerance, in
// the reference's order; returns the cluster count (or -(needed) when `cap`
// is too small).  sizes[c] = size of cluster c, indices = concatenation.
REF_API int ref_ec_extract(const float *xyz, int n, double tol, int *sizes, int *indices, int cap) {
    PointCloud c;
    load(c, xyz, n);
    std::vector<PointIndices> clusters;
    extract(&c, clusters, tol);
    long long total = 0;
    for (auto &k : clusters) total += (long long)k.indices.size();
    if (total > cap) return -(int)total;
    int pos = 0;
    for (size_t k = 0; k < clusters.size(); ++k) {
        sizes[k] = (int)clusters[k].indices.size();
        for (int v : clusters[k].indices) indices[pos++] = v;
    }
    return (int)clusters.size();
}

// segmentByDistance (kernel.cpp:767-814) on one cloud: the colored cloud
// (x, y, z per point; the color is constant), the boxes (position xyz,
// orientation xyzw, dimensions xyz: 10 doubles each) and the centroids (xyz).
// Returns the point count; *nb / *nc = box / centroid counts.  Capacities are
// in points, boxes and centroids.
REF_API int ref_ec_segment(const float *xyz, int n, float *out_xyz, int cap_pts, double *boxes, int cap_boxes,
                           double *centroids, int cap_cent, int *nb, int *nc) {
    PointCloud c;
    load(c, xyz, n);
    euclidean_clustering k;
    PointCloudRGB out;
    BoundingboxArray bb;
    Centroid ce;
    k.segmentByDistance(&c, &out, &bb, &ce);
    if ((int)out.size() > cap_pts || (int)bb.boxes.size() > cap_boxes || (int)ce.points.size() > cap_cent) return -1;
    for (size_t i = 0; i < out.size(); ++i) {
        out_xyz[3 * i] = out[i].x;
        out_xyz[3 * i + 1] = out[i].y;
        out_xyz[3 * i + 2] = out[i].z;
    }
    for (size_t i = 0; i < bb.boxes.size(); ++i) {
        const Boundingbox &b = bb.boxes[i];
        const double v[10] = {b.position.x, b.position.y, b.position.z, b.orientation.x, b.orientation.y,
                              b.orientation.z, b.orientation.w, b.dimensions.x, b.dimensions.y, b.dimensions.z};
        std::memcpy(boxes + 10 * i, v, sizeof(v));
    }
    for (size_t i = 0; i < ce.points.size(); ++i) {
        centroids[3 * i] = ce.points[i].x;
        centroids[3 * i + 1] = ce.points[i].y;
        centroids[3 * i + 2] = ce.points[i].z;
    }
    *nb = (int)bb.boxes.size();
    *nc = (int)ce.points.size();
    return (int)out.size();
}

// The box yaw of clusterAndColor's pose estimate (kernel.cpp:720-745) for one
// cluster (xyz: its points), through the reference's own convexHull and
// rotatingCalipers, with one change: minAreaRectAngle (:479-502) hands
// rotatingCalipers the CLUSTER's point count as the hull's length and so
// reads past the end of the hull (its result then depends on heap contents);
// here the hull's own length is used, for both of its branches.  Writes the
// quaternion's z and w (x = y = 0) and returns the angle in degrees.
REF_API float ref_ec_box_yaw(const float *xyz, int n, double *qz, double *qw) {
    float min_x = std::numeric_limits<float>::max(), min_y = std::numeric_limits<float>::max();
    for (int i = 0; i < n; ++i) {
        if (xyz[3 * i] < min_x) min_x = xyz[3 * i];
        if (xyz[3 * i + 1] < min_y) min_y = xyz[3 * i + 1];
    }
    std::vector<Point2D> inner;
    for (int i = 0; i < n; ++i) {  // as :724-730
        Point2D ip;
        ip.x = (xyz[3 * i] + fabs(min_x)) * 8;
        ip.y = (xyz[3 * i + 1] + fabs(min_y)) * 8;
        inner.push_back(ip);
    }
    float angle = 0.0f;
    if (n > 0) {
        std::vector<Point2D> hull;
        convexHull(inner, hull, true, true);
        const int h = (int)hull.size();
        Point2D out[3];
        if (h > 2) {
            rotatingCalipers(hull.data(), h, (float *)out);
            angle = (float)atan2((double)out[1].y, (double)out[1].x);
        } else if (h == 2) {
            double dx = hull[1].x - hull[0].x;
            double dy = hull[1].y - hull[0].y;
            angle = (float)atan2(dy, dx);
        }
        angle = (float)(angle * 180.0 / PI);
    }
    const double rz = n > 0 ? angle * PI / 180.0 : 0.0;
    *qz = sin(rz * 0.5);
    *qw = cos(rz * 0.5);
    return angle;
}

// convexHull (kernel.cpp:376-470) of n 2-D points (clockwise, returnPoints):
// writes the hull's points to out (capacity n) and returns their count.
REF_API int ref_ec_convex_hull(const float *xy, int n, float *out) {
    std::vector<Point2D> pts(n), hull;
    for (int i = 0; i < n; ++i) pts[i] = {xy[2 * i], xy[2 * i + 1]};
    convexHull(pts, hull, true, true);
    for (size_t i = 0; i < hull.size(); ++i) {
        out[2 * i] = hull[i].x;
        out[2 * i + 1] = hull[i].y;
    }
    return (int)hull.size();
}
