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
