// Box yaw of the euclidean_cluster boxes: the pose estimate of DAPHNE's
// clusterAndColor (src/CPU/euclidean_cluster/kernel.cpp:720-745), i.e. the
// direction of the minimum-area rectangle around a cluster's points in the
// xy plane (minAreaRectAngle :479-502 over convexHull :376-470 and
// rotatingCalipers :90-289), as a quaternion about z.
//
// The reference's minAreaRectAngle hands rotatingCalipers the cluster's point
// count as the hull's length, so its calipers walk past the end of the hull
// into whatever memory follows it; its yaw is not reproducible (its shipped
// output file and a fresh run of the same binary disagree on every box).
// Here the hull's own length is used; with it, the result is the reference's
// routines' result bit for bit.
//
// The hull is Andrew's monotone chain (1979), listed clockwise (x right, y
// up) from the lowest of the leftmost points, no repeated or collinear
// vertices, with the reference's float convexity test: the vertex sequence
// the reference's Sklansky scan gives.  The rectangle is found by rotating calipers
// (Toussaint 1983: the optimal rectangle has a side on a hull edge): four
// calipers, along one base direction turned 0, 1, 2 and 3 quarter turns,
// rest on the bottom, right, top and left extreme vertices; each step turns
// all four by the smallest angle any of them has to its next hull edge and
// measures the rectangle.  The float expressions (edge vectors, inverse
// lengths, cosines, widths, heights, areas) and the tie rules (first caliper
// on equal cosines, last rectangle on equal areas) are the reference's,
// because the chosen side and the reported angle depend on their rounding.
// Compiled with -ffp-contract=off: every product and sum rounds on its own.
#include "ec_pose.h"

#include <omp.h>
#include <stdint.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace ec {
namespace {

constexpr double kPi = 3.1415926535897932384626433832795;

struct V2 {
    float x, y;
};

inline float dot(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline V2 quarter_turn(V2 a) { return {-a.y, a.x}; }  // counter-clockwise by 90 degrees
inline V2 sub(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }

// The turn a -> b -> c is clockwise (x right, y up) when this is > 0: the
// cross product of the edges b - a and c - b, negated, in float, as the
// reference's hull scan tests convexity (kernel.cpp:323-325); its rounding
// decides which nearly collinear vertices stay.
inline bool clockwise(V2 a, V2 b, V2 c) {
    const float ax = b.x - a.x, ay = b.y - a.y, bx = c.x - b.x, by = c.y - b.y;
    return ay * bx - ax * by > 0;
}

struct Work {
    std::vector<uint64_t> keys;
    std::vector<float> xs, ys, depth;  // the shifted points; per point the largest side test
    std::vector<V2> pts, hull, edge;
    std::vector<float> inv_len;
};

// The shifted points are >= +0, whose float bit patterns order as unsigned
// integers: one 64-bit key (x bits high, y bits low) sorts them by x, then y.
inline uint64_t key_of(V2 a) {
    uint32_t x, y;
    std::memcpy(&x, &a.x, 4);
    std::memcpy(&y, &a.y, 4);
    return (uint64_t)x << 32 | y;
}
inline V2 point_of(uint64_t k) {
    const uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k;
    V2 a;
    std::memcpy(&a.x, &x, 4);
    std::memcpy(&a.y, &y, 4);
    return a;
}

// Keys of the points of w.pts that can be hull vertices.  Points deep inside
// the polygon of the extreme points in eight directions (left, upper left,
// top, ..., lower left: Akl and Toussaint's 1978 quadrilateral with the
// diagonals added) are left out.  "Deep" is more than 2^-20 of the points'
// extent from each side, tested in float: the test's own rounding stays
// below half of that, and what is left (> 8 * 2^-24 of the extent) is beyond
// the relative rounding of the scan's float convexity test, so the scan's
// tests against these points are far from zero.  The polygon's vertices are
// input points whichever way the float extremes round, so it lies inside the
// hull.
void keep_outer(Work &w) {
    const float *x = w.xs.data(), *y = w.ys.data();
    const int n = (int)w.xs.size();
    w.keys.clear();
    if (n < 16) {
        for (int i = 0; i < n; ++i) w.keys.push_back(key_of({x[i], y[i]}));
        return;
    }
    // clockwise from the leftmost point: extremes of -x, y - x, y, x + y, x, x - y, -y, -x - y
    int ext[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float best[8] = {-x[0], y[0] - x[0], y[0], x[0] + y[0], x[0], x[0] - y[0], -y[0], -x[0] - y[0]};
    for (int i = 1; i < n; ++i) {
        const float u = x[i], v = y[i];
        if (-u > best[0]) best[0] = -u, ext[0] = i;
        if (v - u > best[1]) best[1] = v - u, ext[1] = i;
        if (v > best[2]) best[2] = v, ext[2] = i;
        if (u + v > best[3]) best[3] = u + v, ext[3] = i;
        if (u > best[4]) best[4] = u, ext[4] = i;
        if (u - v > best[5]) best[5] = u - v, ext[5] = i;
        if (-v > best[6]) best[6] = -v, ext[6] = i;
        if (-u - v > best[7]) best[7] = -u - v, ext[7] = i;
    }
    const double span = std::max((double)x[ext[4]] - x[ext[0]], (double)y[ext[2]] - y[ext[6]]);
    w.depth.assign(n, -std::numeric_limits<float>::infinity());
    float *depth = w.depth.data();
    int sides = 0;
    for (int d = 0; d < 8; ++d) {  // side a -> b; (p - a) . (outward normal) - bound, largest over the sides
        const int ia = ext[d], ib = ext[(d + 1) & 7];
        const float ex = x[ib] - x[ia], ey = y[ib] - y[ia];
        const double len = std::sqrt((double)ex * ex + (double)ey * ey);
        if (!(len > 0)) continue;  // coinciding extremes
        ++sides;
        const float ax = x[ia], ay = y[ia], nx = -ey, ny = ex;  // left of a -> b: outside (clockwise polygon)
        const float lim = (float)(-span * len * std::ldexp(1.0, -20));
        for (int i = 0; i < n; ++i) depth[i] = std::max(depth[i], (x[i] - ax) * nx + (y[i] - ay) * ny - lim);
    }
    const bool usable = sides >= 3 && span > 0;
    for (int i = 0; i < n; ++i)
        if (!usable || !(depth[i] < 0)) w.keys.push_back(key_of({x[i], y[i]}));
}

// Clockwise hull of the points whose keys are w.keys (reordered) into w.hull.
void hull_clockwise(Work &w) {
    std::vector<uint64_t> &k = w.keys;
    std::sort(k.begin(), k.end());
    k.erase(std::unique(k.begin(), k.end()), k.end());
    std::vector<V2> &p = w.pts, &h = w.hull;
    p.resize(k.size());
    for (size_t i = 0; i < k.size(); ++i) p[i] = point_of(k[i]);
    h.clear();
    const int n = (int)p.size();
    for (int i = 0; i < n; ++i) {  // upper chain, left to right: right turns only
        while (h.size() >= 2 && !clockwise(h[h.size() - 2], h.back(), p[i])) h.pop_back();
        h.push_back(p[i]);
    }
    const size_t upper = h.size();
    for (int i = n - 2; i >= 0; --i) {  // lower chain, right to left
        while (h.size() > upper && !clockwise(h[h.size() - 2], h.back(), p[i])) h.pop_back();
        h.push_back(p[i]);
    }
    if (h.size() > 1) h.pop_back();  // the start again
}

// Direction of the minimum-area rectangle around the clockwise hull h (> 2
// vertices), in radians, as atan2 of the rectangle's first side vector.
float rectangle_angle(Work &w) {
    const std::vector<V2> &h = w.hull;
    const int n = (int)h.size();
    w.edge.resize(n);
    w.inv_len.resize(n);
    int rest[4] = {0, 0, 0, 0};  // caliper vertices: bottom, right, top, left (first extreme in hull order)
    for (int i = 0; i < n; ++i) {
        const V2 a = h[i], b = h[i + 1 < n ? i + 1 : 0];
        const V2 d = sub(b, a);  // float differences
        w.edge[i] = d;
        w.inv_len[i] = (float)(1. / std::sqrt((double)d.x * d.x + (double)d.y * d.y));
        if (a.y < h[rest[0]].y) rest[0] = i;
        if (a.x > h[rest[1]].x) rest[1] = i;
        if (a.y > h[rest[2]].y) rest[2] = i;
        if (a.x < h[rest[3]].x) rest[3] = i;
    }
    // the hull's turning sense: the first non-zero turn between consecutive edges
    float sense = 0.f;
    for (int i = 0; i < n; ++i) {
        const V2 a = w.edge[i ? i - 1 : n - 1], b = w.edge[i];
        const double c = (double)a.x * b.y - (double)a.y * b.x;
        if (c != 0) {
            sense = c > 0 ? 1.f : -1.f;
            break;
        }
    }
    V2 base = {sense, 0.f};
    float best_area = std::numeric_limits<float>::max(), best_width = 0.f;
    V2 best_base = {0.f, 0.f};
    for (int k = 0; k < n; ++k) {
        int m_best = 0;
        float c_best = 0.f;
        V2 dir = base;
        for (int m = 0; m < 4; ++m, dir = quarter_turn(dir)) {
            const int e = rest[m];
            const float c = dot(dir, w.edge[e]) * w.inv_len[e];
            if (m == 0 || c > c_best) {
                c_best = c;
                m_best = m;
            }
        }
        const int e = rest[m_best];
        V2 lead = {w.edge[e].x * w.inv_len[e], w.edge[e].y * w.inv_len[e]};
        for (int t = 0; t < (4 - m_best) % 4; ++t) lead = quarter_turn(lead);  // back to caliper 0
        base = lead;
        rest[m_best] = rest[m_best] + 1 == n ? 0 : rest[m_best] + 1;
        const float width = dot(sub(h[rest[1]], h[rest[3]]), base);
        const float height = dot(sub(h[rest[2]], h[rest[0]]), quarter_turn(base));
        const float area = width * height;
        if (area <= best_area) {
            best_area = area;
            best_base = base;
            best_width = width;
        }
    }
    const V2 side = {best_base.x * best_width, best_base.y * best_width};
    return (float)std::atan2((double)side.y, (double)side.x);
}

}  // namespace

void box_yaw(const float *xyz, int n, float min_x, float min_y, double *qz, double *qw) {
    thread_local Work w;
    float angle = 0.f;
    if (n > 0) {
        w.xs.resize(n);
        w.ys.resize(n);
        const double ox = std::fabs((double)min_x), oy = std::fabs((double)min_y);
        for (int i = 0; i < n; ++i) {  // the reference's shifted, scaled copy of the cluster (x, y >= +0)
            w.xs[i] = (float)(((double)xyz[3 * (size_t)i] + ox) * 8);
            w.ys[i] = (float)(((double)xyz[3 * (size_t)i + 1] + oy) * 8);
        }
        keep_outer(w);
        hull_clockwise(w);
        if (w.hull.size() > 2) {
            angle = rectangle_angle(w);
        } else if (w.hull.size() == 2) {
            const V2 d = sub(w.hull[1], w.hull[0]);
            angle = (float)std::atan2((double)d.y, (double)d.x);
        }
        angle = (float)(angle * 180.0 / kPi);  // degrees, as minAreaRectAngle returns them
    }
    const double rz = angle * kPi / 180.0;
    *qz = std::sin(rz * 0.5);
    *qw = std::cos(rz * 0.5);
}

// libgomp's thread pool does not survive fork(): the first process that runs
// a parallel pass owns it, and a process forked from it after that runs its
// passes on one thread.
std::atomic<pid_t> g_pool_owner{0};

void box_yaws(const YawJob *jobs, int count) {
    // independent clusters over the host's threads (at most kYawThreads, at most the cores there are), in a
    // dynamic schedule of small chunks so that one large cluster does not hold up the others' threads
    int threads = std::max(1, std::min(kYawThreads, omp_get_num_procs()));
    if (count > 4 && threads > 1) {
        const pid_t me = getpid();
        pid_t none = 0;
        g_pool_owner.compare_exchange_strong(none, me);
        if (g_pool_owner.load() != me) threads = 1;
    }
#pragma omp parallel for schedule(dynamic, 2) num_threads(threads) if (count > 4 && threads > 1)
    for (int j = 0; j < count; ++j) box_yaw(jobs[j].xyz, jobs[j].n, jobs[j].min_x, jobs[j].min_y, jobs[j].qz, jobs[j].qw);
}

}  // namespace ec
