// Euclidean clustering on the GPU: the radius search and cluster extraction of
// DAPHNE's euclidean_cluster kernel (extractEuclideanClusters / extract,
// src/CPU/euclidean_cluster/kernel.cpp:562-647; its CUDA port builds an N x N
// boolean distance matrix, src/Cuda/euclidean_cluster/kernel.cu:506-560), and
// the host side of segmentByDistance / clusterAndColor (:652-814) around it.
//
// The reference grows each cluster breadth-first from its smallest
// unprocessed point through all points whose float squared distance
// dx*dx + dy*dy + dz*dz (each product and sum rounded) is <= r*r (float): the
// clusters are the connected components of that graph, in order of their
// smallest point index, each listed in ascending index order; those with
// [min, max] points are kept and ordered by size with std::sort over reverse
// iterators.
//
// Here: points are sorted into cells of edge r * (1 + 1e-4) (cell indices in
// FP64, so an accepted pair is never more than one cell apart on any axis;
// at most 2^28 cells per cloud) with the voxel-grid
// build's stable radix sort; one thread per point and neighbour cell tests
// that cell's points with the same float operations and joins accepted pairs
// in a lock-free union-find whose roots are always the component's smallest
// index (the larger root is linked under the smaller by atomicCAS); after a
// final compression every label is its component's smallest index.  The host
// groups the indices by label (ascending, so clusters come out in the
// reference's order), filters by size and applies the same std::sort.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "../../include/ndt_b200.h"
#include "ec_pose.h"
#include "grid_build.h"
#include "nvtx_range.h"

namespace ec {

constexpr int kThreads = 256;
constexpr int kSplit = 4;  // threads per (point, neighbour cell): dense cells are shared out
constexpr int kUnionLimit = 1 << 20;  // CAS retries of one union (never reached in practice; flags an error)

constexpr int kMaxParts = 40;  // clouds clustered in one pass (segmentByDistance: 5 rings of up to 8 clouds)

// Geometry of the clouds of one pass: part p's points are [off[p], off[p + 1])
// of the concatenation, its cells have edge cell[p] from minv[p] with dims
// dim[p], and its cell keys are base[p] + x + dx (y + dy z).
struct Parts {
    int np;
    int off[kMaxParts + 1];
    long long base[kMaxParts + 1];
    float minv[kMaxParts][3];
    float cell[kMaxParts];
    float r2[kMaxParts];
    int dim[kMaxParts][3];
};

// Cell index in FP64 (the difference of two floats is exact there), so that
// cell boundaries move by no more than ~1e-16 cells: with cells 1e-4 wider
// than the radius, points of an accepted pair are at most one cell apart.
__device__ __forceinline__ int cell_of(float v, float minv, float cell, int dim) {
    int c = (int)(((double)v - (double)minv) / (double)cell);
    return c < 0 ? 0 : (c >= dim ? dim - 1 : c);
}

// The part of point t (or of key k): the last p with first[p] <= t.
template <class T>
__device__ __forceinline__ int part_of(const T *first, int np, long long t) {
    int lo = 0, hi = np;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((long long)first[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void key_kernel(const float4 *__restrict__ pts, int n, const __grid_constant__ Parts P,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, int *__restrict__ parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int q = part_of(P.off, P.np, i);
    const float4 p = pts[i];
    const int cx = cell_of(p.x, P.minv[q][0], P.cell[q], P.dim[q][0]);
    const int cy = cell_of(p.y, P.minv[q][1], P.cell[q], P.dim[q][1]);
    const int cz = cell_of(p.z, P.minv[q][2], P.cell[q], P.dim[q][2]);
    keys[i] = (uint32_t)(P.base[q] + cx + (long long)P.dim[q][0] * (cy + (long long)P.dim[q][1] * cz));
    vals[i] = (uint32_t)i;
    parent[i] = i;
}

// cell -> first sorted position of its points (segment s), or -1
__global__ void cell_index_kernel(const int32_t *__restrict__ seg_start, const uint32_t *__restrict__ seg_key,
                                  const int *__restrict__ nseg, int *__restrict__ cell_first) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < *nseg) cell_first[seg_key[s]] = s;
}

// Union-find over parent[] with parent[v] <= v for every v (a root links
// under a smaller one only), so every chain strictly decreases and a root is
// its component's smallest index.  Reads are volatile (other threads link and
// shorten concurrently); path halving stores a valid ancestor, so any
// interleaving keeps the invariant.
__device__ __forceinline__ int find_root(int *parent, int x) {
    volatile int *p = parent;
    for (int it = 0; it < kUnionLimit; ++it) {
        const int up = p[x];
        if (up == x) return x;
        const int up2 = p[up];
        if (up2 != up) p[x] = up2;
        x = up;
    }
    return -1;
}

// kSplit threads per (point i, neighbour cell): blockIdx.y picks the cell
// offset (27 of them) and the thread's share of the cell's points (every
// kSplit-th), x walks the points in sorted order, so a warp's points share
// cells and read the same neighbours.  The thread tests the points j > i of
// its cell (cells never cross parts); i's root is found at the first accepted
// pair and kept; a pair whose roots already agree costs the reads of j's
// chain, a merge one atomicCAS (the larger root under the smaller).
__global__ void join_kernel(const float4 *__restrict__ pts, const uint32_t *__restrict__ order,
                            const uint32_t *__restrict__ keys, int n, const int32_t *__restrict__ seg_start,
                            const int *__restrict__ nseg, const int *__restrict__ cell_first,
                            const __grid_constant__ Parts P, int *__restrict__ parent, int *__restrict__ err) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int off = blockIdx.y / kSplit;  // 9 dz + 3 dy + dx, each in {0, 1, 2}
    const int part = blockIdx.y % kSplit;  // this thread's share of the cell: every kSplit-th point
    const long long key = keys[t];
    const int q = part_of(P.base, P.np, key);
    const long long local = key - P.base[q];
    const int dx0 = P.dim[q][0], dy0 = P.dim[q][1], dz0 = P.dim[q][2];
    const int x = (int)(local % dx0) + off % 3 - 1;
    const int y = (int)((local / dx0) % dy0) + (off / 3) % 3 - 1;
    const int z = (int)(local / ((long long)dx0 * dy0)) + off / 9 - 1;
    if (x < 0 || x >= dx0 || y < 0 || y >= dy0 || z < 0 || z >= dz0) return;
    const int s = cell_first[P.base[q] + x + (long long)dx0 * (y + (long long)dy0 * z)];
    if (s < 0) return;
    const int i = (int)order[t];
    const float4 p = pts[i];
    const float r2 = P.r2[q];
    const int e = s + 1 < *nseg ? seg_start[s + 1] : n;
    int ri = -2;  // not looked up yet
    for (int u = seg_start[s] + part; u < e; u += kSplit) {
        const int j = (int)order[u];
        if (j <= i) continue;
        const float4 qj = pts[j];
        const float ex = __fsub_rn(qj.x, p.x), ey = __fsub_rn(qj.y, p.y), ez = __fsub_rn(qj.z, p.z);
        const float d2 = __fadd_rn(__fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey)), __fmul_rn(ez, ez));
        if (!(d2 <= r2)) continue;
        if (ri == -2) ri = find_root(parent, i);
        int rj = find_root(parent, j);
        int it = 0;
        for (; it < kUnionLimit && ri >= 0 && rj >= 0 && ri != rj; ++it) {
            const int lo = ri < rj ? ri : rj, hi = ri < rj ? rj : ri;
            if (atomicCAS(parent + hi, hi, lo) == hi) {
                ri = lo;
                break;
            }
            ri = find_root(parent, ri);  // hi was linked meanwhile
            rj = find_root(parent, rj);
        }
        if (ri < 0 || rj < 0 || it == kUnionLimit) {
            atomicOr(err, 1);
            return;
        }
    }
}

__global__ void label_kernel(int *__restrict__ parent, int n, int *__restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int r = find_root(parent, i);
    if (r < 0) atomicOr(err, 2);
    parent[i] = r;
}

}  // namespace ec

struct ndt_ec {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    void *pts = nullptr, *scratch = nullptr, *parent = nullptr, *seg_start = nullptr, *seg_key = nullptr,
         *cell_first = nullptr, *flags = nullptr;
    size_t pts_cap = 0, scratch_cap = 0, parent_cap = 0, seg_start_cap = 0, seg_key_cap = 0, cell_cap = 0;
    float4 *h_pts = nullptr;  // pinned staging
    int *h_labels = nullptr;
    size_t h_cap = 0;
};

namespace {

constexpr long long kMaxCells = 1LL << 28;  // dense cell table (4 B per cell) of one cloud, at most

int fail(ndt_ec *h, int code, const std::string &msg) {
    if (h) h->err = msg;
    return code;
}

cudaError_t ensure(void **p, size_t *cap, size_t bytes) {
    if (*p && *cap >= bytes) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const size_t want = std::max(bytes + bytes / 2, (size_t)256);
    cudaError_t e = cudaMalloc(p, want);
    if (e == cudaSuccess) *cap = want;
    return e;
}

#define ECK(call)                                                                             \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(h, NDT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// Component labels of up to kMaxParts clouds in one pass: labels[p][i] is the
// smallest index within cloud p of point i's component (clouds never join).
int labels_of(ndt_ec *h, const std::vector<const float *> &xyz, const std::vector<int> &n,
              const std::vector<float> &tolerance, std::vector<std::vector<int>> &labels) {
    ndt::NvtxRange range("ec labels");
    const int np = (int)xyz.size();
    labels.assign(np, std::vector<int>());
    ec::Parts P;
    std::memset(&P, 0, sizeof(P));
    P.np = np;
    long long total = 0, cells = 0;
    for (int q = 0; q < np; ++q) {
        P.off[q] = (int)total;
        P.base[q] = cells;
        total += n[q];
        labels[q].assign(n[q], 0);
        float mn[3] = {0.0f, 0.0f, 0.0f}, mx[3] = {0.0f, 0.0f, 0.0f};
        for (int i = 0; i < n[q]; ++i) {
            const float *v = xyz[q] + 3 * (size_t)i;
            if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]))
                return fail(h, NDT_E_ARG, "non-finite point coordinates");
            for (int k = 0; k < 3; ++k) {
                mn[k] = i ? std::min(mn[k], v[k]) : v[k];
                mx[k] = i ? std::max(mx[k], v[k]) : v[k];
            }
        }
        P.cell[q] = tolerance[q] * 1.0001f;  // cells a little wider than the radius
        P.r2[q] = tolerance[q] * tolerance[q];
        long long G = 1;
        for (int k = 0; k < 3; ++k) {
            P.minv[q][k] = mn[k];
            const double d = std::floor(((double)mx[k] - (double)mn[k]) / (double)P.cell[q]) + 1.0;
            if (!(d >= 1.0 && d < 2147483647.0)) return fail(h, NDT_E_CAPACITY, "a cloud spans too many cells");
            P.dim[q][k] = (int)d;
            G *= P.dim[q][k];
            if (G > kMaxCells) break;
        }
        cells += n[q] ? G : 0;
        if (cells > kMaxCells) return fail(h, NDT_E_CAPACITY, "the clouds span more than 2^28 cells of the tolerance");
    }
    P.off[np] = (int)total;
    P.base[np] = cells;
    const int N = (int)total;
    if (N == 0) return NDT_OK;
    cudaStream_t st = h->stream;
    if (h->h_cap < (size_t)N) {
        if (h->h_pts) cudaFreeHost(h->h_pts);
        if (h->h_labels) cudaFreeHost(h->h_labels);
        h->h_pts = nullptr;
        h->h_labels = nullptr;
        h->h_cap = 0;
        const size_t want = (size_t)N + N / 2;
        ECK(cudaMallocHost((void **)&h->h_pts, sizeof(float4) * want));
        ECK(cudaMallocHost((void **)&h->h_labels, sizeof(int) * want));
        h->h_cap = want;
    }
    for (int q = 0; q < np; ++q)
        for (int i = 0; i < n[q]; ++i) {
            const float *v = xyz[q] + 3 * (size_t)i;
            h->h_pts[P.off[q] + i] = make_float4(v[0], v[1], v[2], 0.0f);
        }
    int bits = 1;
    while (bits < 31 && (1LL << bits) < cells) ++bits;
    ECK(ensure(&h->pts, &h->pts_cap, sizeof(float4) * (size_t)N));
    ECK(ensure(&h->scratch, &h->scratch_cap, ndt::sort_scratch_bytes(N)));
    ECK(ensure(&h->parent, &h->parent_cap, sizeof(int) * (size_t)N));
    ECK(ensure(&h->seg_start, &h->seg_start_cap, sizeof(int) * (size_t)N));
    ECK(ensure(&h->seg_key, &h->seg_key_cap, sizeof(int) * (size_t)N));
    ECK(ensure(&h->cell_first, &h->cell_cap, sizeof(int) * (size_t)cells));
    size_t fcap = 0;
    if (!h->flags) ECK(ensure(&h->flags, &fcap, 256));
    float4 *d_pts = (float4 *)h->pts;
    int *parent = (int *)h->parent, *err = (int *)h->flags;
    ECK(cudaMemcpyAsync(d_pts, h->h_pts, sizeof(float4) * (size_t)N, cudaMemcpyHostToDevice, st));
    ECK(cudaMemsetAsync(err, 0, sizeof(int), st));
    ECK(cudaMemsetAsync(h->cell_first, 0xff, sizeof(int) * (size_t)cells, st));
    ndt::SortBuffers sb = ndt::sort_buffers(h->scratch, N);
    const unsigned blocks = (unsigned)((N + ec::kThreads - 1) / ec::kThreads);
    ec::key_kernel<<<blocks, ec::kThreads, 0, st>>>(d_pts, N, P, sb.k0, sb.v0, parent);
    ndt::sort_segments(sb, N, bits, (int32_t *)h->seg_start, (uint32_t *)h->seg_key, st);
    ec::cell_index_kernel<<<blocks, ec::kThreads, 0, st>>>((const int32_t *)h->seg_start, (const uint32_t *)h->seg_key,
                                                           sb.nseg, (int *)h->cell_first);
    ec::join_kernel<<<dim3(blocks, 27 * ec::kSplit), ec::kThreads, 0, st>>>(
        d_pts, sb.v0, sb.k0, N, (const int32_t *)h->seg_start, sb.nseg, (const int *)h->cell_first, P, parent, err);
    ec::label_kernel<<<blocks, ec::kThreads, 0, st>>>(parent, N, err);
    ECK(cudaGetLastError());
    ECK(cudaMemcpyAsync(h->h_labels, parent, sizeof(int) * (size_t)N, cudaMemcpyDeviceToHost, st));
    int e = 0;
    ECK(cudaMemcpyAsync(&e, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    ECK(cudaStreamSynchronize(st));
    if (e) return fail(h, NDT_E_CUDA, "union-find retry limit reached");
    for (int q = 0; q < np; ++q)
        for (int i = 0; i < n[q]; ++i) labels[q][i] = h->h_labels[P.off[q] + i] - P.off[q];
    return NDT_OK;
}

// The reference's clusters from component labels: components in order of
// their smallest index, indices ascending, sizes in [lo, hi], then ordered by
// size with std::sort over reverse iterators (extract, kernel.cpp:635-647).
void clusters_of(const std::vector<int> &labels, int lo, int hi, std::vector<std::vector<int>> &out) {
    const int n = (int)labels.size();
    std::vector<int> size(n, 0), slot(n, -1);
    for (int i = 0; i < n; ++i) ++size[labels[i]];
    out.clear();
    for (int i = 0; i < n; ++i)
        if (labels[i] == i && size[i] >= lo && size[i] <= hi) {
            slot[i] = (int)out.size();
            out.emplace_back();
            out.back().reserve(size[i]);
        }
    for (int i = 0; i < n; ++i)
        if (slot[labels[i]] >= 0) out[slot[labels[i]]].push_back(i);
    std::sort(out.rbegin(), out.rend(),
              [](const std::vector<int> &a, const std::vector<int> &b) { return a.size() < b.size(); });
}

}  // namespace

extern "C" {

int ndt_ec_create(int device, ndt_ec **out) {
    if (!out) return NDT_E_ARG;
    *out = nullptr;
    ndt_ec *h = new ndt_ec();
    h->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete h;
        return NDT_E_CUDA;
    }
    *out = h;
    return NDT_OK;
}

void ndt_ec_destroy(ndt_ec *h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void *p : {h->pts, h->scratch, h->parent, h->seg_start, h->seg_key, h->cell_first, h->flags})
        if (p) cudaFree(p);
    if (h->h_pts) cudaFreeHost(h->h_pts);
    if (h->h_labels) cudaFreeHost(h->h_labels);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

const char *ndt_ec_last_error(const ndt_ec *h) { return h ? h->err.c_str() : "null handle"; }

int ndt_ec_labels(ndt_ec *h, const float *xyz, int n, float tolerance, int *labels) {
    if (!h || n < 0 || (n > 0 && (!xyz || !labels)) || !(tolerance > 0.0f) || !std::isfinite(tolerance))
        return fail(h, NDT_E_ARG, "bad argument");
    ECK(cudaSetDevice(h->device));
    std::vector<std::vector<int>> lab;
    if (int rc = labels_of(h, {xyz}, {n}, {tolerance}, lab)) return rc;
    if (n) std::memcpy(labels, lab[0].data(), sizeof(int) * (size_t)n);
    return NDT_OK;
}

int ndt_ec_extract(ndt_ec *h, const float *xyz, int n, float tolerance, int min_size, int max_size,
                   int *num_clusters, int *cluster_offsets, int *cluster_indices) {
    if (!h || n < 0 || (n > 0 && !xyz) || !num_clusters || !cluster_offsets || !cluster_indices ||
        !(tolerance > 0.0f) || !std::isfinite(tolerance))
        return fail(h, NDT_E_ARG, "bad argument");
    ECK(cudaSetDevice(h->device));
    std::vector<std::vector<int>> lab;
    if (int rc = labels_of(h, {xyz}, {n}, {tolerance}, lab)) return rc;
    std::vector<std::vector<int>> cl;
    clusters_of(lab[0], min_size, max_size, cl);
    int pos = 0;
    cluster_offsets[0] = 0;
    for (size_t c = 0; c < cl.size(); ++c) {
        std::memcpy(cluster_indices + pos, cl[c].data(), sizeof(int) * cl[c].size());
        pos += (int)cl[c].size();
        cluster_offsets[c + 1] = pos;
    }
    *num_clusters = (int)cl.size();
    return NDT_OK;
}

// segmentByDistance (kernel.cpp:767-814) with clusterAndColor (:652-765):
// five rings of distance from the sensor (< 15, 30, 45, 60 m, beyond) with
// tolerances 0.5, 1.1, 1.6, 2.3 and 2.6f, clusters of 20 to 100000 points.
// Clouds [c0, c1) of a packed batch in one GPU pass; outputs appended at the
// running counts np / nb.
namespace {
int segment_clouds(ndt_ec *h, const float *xyz, const int *offsets, int c0, int c1, float *out_xyz, int *out_off,
                   double *boxes, int *box_off, double *centroids, int &np, int &nb) {
    const double tol[5] = {0.5, 1.1, 1.6, 2.3, 2.6f};
    const int C = c1 - c0;
    std::vector<std::vector<float>> ring(5 * (size_t)C);
    for (int c = 0; c < C; ++c)
        for (int i = offsets[c0 + c]; i < offsets[c0 + c + 1]; ++i) {
            const float *q = xyz + 3 * (size_t)i;
            const float x = q[0], y = q[1];
            const float d = std::sqrt(x * x + y * y);
            const int r = d < 15 ? 0 : (d < 30 ? 1 : (d < 45 ? 2 : (d < 60 ? 3 : 4)));
            ring[5 * (size_t)c + r].insert(ring[5 * (size_t)c + r].end(), q, q + 3);
        }
    std::vector<const float *> parts;
    std::vector<int> sizes;
    std::vector<float> tols;
    for (int k = 0; k < 5 * C; ++k) {
        parts.push_back(ring[k].data());
        sizes.push_back((int)(ring[k].size() / 3));
        tols.push_back((float)tol[k % 5]);
    }
    std::vector<std::vector<int>> lab;
    if (int rc = labels_of(h, parts, sizes, tols, lab)) return rc;  // every ring of every cloud in one pass
    std::vector<std::vector<int>> cl;
    std::vector<ec::YawJob> yaw;
    for (int c = 0; c < C; ++c) {
        out_off[c0 + c] = np;
        box_off[c0 + c] = nb;
        for (int r = 0; r < 5; ++r) {
            const std::vector<float> &pts = ring[5 * (size_t)c + r];
            if (pts.empty()) continue;
            clusters_of(lab[5 * (size_t)c + r], 20, 100000, cl);
            for (const std::vector<int> &idx : cl) {
                double cen[3] = {0.0, 0.0, 0.0};
                float lo[3] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max(),
                               std::numeric_limits<float>::max()};
                float hi[3] = {-lo[0], -lo[1], -lo[2]};
                for (int i : idx) {
                    const float *p = &pts[3 * (size_t)i];
                    for (int k = 0; k < 3; ++k) {
                        out_xyz[3 * (size_t)np + k] = p[k];
                        cen[k] += p[k];
                        if (p[k] < lo[k]) lo[k] = p[k];
                        if (p[k] > hi[k]) hi[k] = p[k];
                    }
                    ++np;
                }
                for (int k = 0; k < 3; ++k) cen[k] /= idx.size();
                const float l = hi[0] - lo[0], w = hi[1] - lo[1], ht = hi[2] - lo[2];
                const double dim[3] = {l < 0 ? -1 * l : l, w < 0 ? -1 * w : w, ht < 0 ? -1 * ht : ht};
                if (dim[0] > 0 && dim[1] > 0 && dim[2] > 0 && dim[0] < 15 && dim[1] > 0 && dim[1] < 15 &&
                    hi[2] > -1.5 && lo[2] > -1.5 && lo[2] < 1.0) {
                    // position, orientation (x, y, z, w: z and w by the yaw pass below), dimensions
                    const double b[10] = {lo[0] + l / 2, lo[1] + w / 2, lo[2] + ht / 2, 0.0, 0.0, 0.0, 1.0,
                                          dim[0], dim[1], dim[2]};
                    std::memcpy(boxes + 10 * (size_t)nb, b, sizeof(b));
                    // the yaw only of kept boxes: the others are not output
                    yaw.push_back({out_xyz + 3 * (size_t)(np - (int)idx.size()), (int)idx.size(), lo[0], lo[1],
                                   boxes + 10 * (size_t)nb + 5, boxes + 10 * (size_t)nb + 6});
                    std::memcpy(centroids + 3 * (size_t)nb, cen, sizeof(cen));
                    ++nb;
                }
            }
        }
    }
    out_off[c1] = np;
    box_off[c1] = nb;
    {
        ndt::NvtxRange range("ec yaw");
        ec::box_yaws(yaw.data(), (int)yaw.size());
    }
    return NDT_OK;
}
}  // namespace

int ndt_ec_segment(ndt_ec *h, const float *xyz, int n, float *out_xyz, int *out_n, double *boxes, int *num_boxes,
                   double *centroids, int *num_centroids) {
    if (!h || n < 0 || (n > 0 && !xyz) || !out_xyz || !out_n || !boxes || !num_boxes || !centroids ||
        !num_centroids)
        return fail(h, NDT_E_ARG, "bad argument");
    ECK(cudaSetDevice(h->device));
    const int off[2] = {0, n};
    int oo[2], bo[2], np = 0, nb = 0;
    if (int rc = segment_clouds(h, xyz, off, 0, 1, out_xyz, oo, boxes, bo, centroids, np, nb)) return rc;
    *out_n = np;
    *num_boxes = nb;
    *num_centroids = nb;
    return NDT_OK;
}

int ndt_ec_box_yaw(const float *xyz, int n, double *qz, double *qw) {
    if (n < 0 || (n > 0 && !xyz) || !qz || !qw) return NDT_E_ARG;
    float lo[2] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < 2; ++k) {
            const float v = xyz[3 * (size_t)i + k];
            if (!std::isfinite(v)) return NDT_E_ARG;
            if (v < lo[k]) lo[k] = v;
        }
    ec::box_yaw(xyz, n, lo[0], lo[1], qz, qw);
    return NDT_OK;
}

int ndt_ec_box_yaws(int C, const float *xyz, const int *offsets, double *qz, double *qw) {
    if (C < 0 || (C > 0 && (!offsets || !qz || !qw)) || (C > 0 && offsets[0] != 0)) return NDT_E_ARG;
    if (C > 0 && offsets[C] > 0 && !xyz) return NDT_E_ARG;
    std::vector<ec::YawJob> jobs(C);
    for (int c = 0; c < C; ++c) {
        if (offsets[c + 1] < offsets[c]) return NDT_E_ARG;
        float lo[2] = {std::numeric_limits<float>::max(), std::numeric_limits<float>::max()};
        for (int i = offsets[c]; i < offsets[c + 1]; ++i)
            for (int k = 0; k < 2; ++k) {
                const float v = xyz[3 * (size_t)i + k];
                if (!std::isfinite(v)) return NDT_E_ARG;
                if (v < lo[k]) lo[k] = v;
            }
        jobs[c] = {xyz + 3 * (size_t)offsets[c], offsets[c + 1] - offsets[c], lo[0], lo[1], qz + c, qw + c};
    }
    ec::box_yaws(jobs.data(), C);
    return NDT_OK;
}

int ndt_ec_segment_batch(ndt_ec *h, int C, const float *xyz, const int *offsets, float *out_xyz, int *out_offsets,
                         double *boxes, int *box_offsets, double *centroids) {
    if (!h || C <= 0 || !offsets || !out_xyz || !out_offsets || !boxes || !box_offsets || !centroids ||
        (offsets[C] > 0 && !xyz) || offsets[0] != 0)
        return fail(h, NDT_E_ARG, "bad argument");
    for (int c = 0; c < C; ++c)
        if (offsets[c + 1] < offsets[c]) return fail(h, NDT_E_ARG, "offsets must be non-decreasing");
    ECK(cudaSetDevice(h->device));
    int np = 0, nb = 0;
    const int per_pass = ec::kMaxParts / 5;
    for (int c0 = 0; c0 < C; c0 += per_pass) {
        const int c1 = std::min(C, c0 + per_pass);
        if (int rc = segment_clouds(h, xyz, offsets, c0, c1, out_xyz, out_offsets, boxes, box_offsets, centroids,
                                    np, nb))
            return rc;
    }
    return NDT_OK;
}

}  // extern "C"
