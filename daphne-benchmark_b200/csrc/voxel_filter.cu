// Scan pre-filter: voxel-grid downsampling of a batch of raw scans on the
// device (the step that produces the align call's "filtered scan" upstream;
// it is not part of the reference kernel).
//
// Semantics (pinned by oracle/voxel_filter_ref.py):
//   * a point is kept when x, y, z are finite;
//   * its leaf is (floor(x * r), floor(y * r), floor(z * r)) with
//     r = 1 / leaf rounded to float and each product rounded to float (the
//     leaf index of the point-cloud library's voxel-grid filter, which
//     Autoware's mapping pipeline runs with a 2 m leaf before the align);
//   * every occupied leaf of a scan yields one point: the mean of its points,
//     summed in FP64 in input order and divided by their count, rounded to
//     float (x, y, z and the fourth component alike);
//   * a scan's output points are ordered by leaf, x fastest, then y, then z.
//
// Device pipeline for B scans: per scan the leaf bounding box (one block per
// scan) and its leaf-key range; an exclusive scan of the ranges gives every
// scan a disjoint key interval, so one 32-bit key per point (scan interval
// base + local leaf key) orders points by scan, then leaf; one stable radix
// sort and segmentation of all points (shared with the voxel-grid build);
// per segment the FP64 mean in input order; per-scan output counts by atomic
// increments of integers (order-independent), scanned into output offsets.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ndt_b200.h"
#include "grid_build.h"

namespace vf {

constexpr int kThreads = 256;

__device__ __forceinline__ bool finite3(float4 p) { return isfinite(p.x) && isfinite(p.y) && isfinite(p.z); }

// The product is clamped to +-2^60 before the integer conversion, so that
// any finite coordinate has a defined leaf index (a scan that far out fails
// the 2^31-leaf range check).
__device__ __forceinline__ long long leaf_of(float v, float r) {
    float q = floorf(__fmul_rn(v, r));
    q = fminf(fmaxf(q, -1.1529215e18f), 1.1529215e18f);  // 2^60
    return (long long)q;
}

struct ScanGeom {
    long long lo[3];  // leaf index minimum per axis
    long long d[3];   // leaf extent per axis
};

// Leaf bounding box and key range of scan b (one block per scan).  range[b]
// = dx * dy * dz (0 for a scan without finite points); err |= 1 when a range
// exceeds 2^31.
__global__ void scan_box_kernel(const float4 *__restrict__ pts, const int *__restrict__ offsets, float r,
                                ScanGeom *__restrict__ geom, int *__restrict__ range, int *__restrict__ err) {
    const int b = blockIdx.x;
    const int s = offsets[b], e = offsets[b + 1];
    long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
    for (int i = s + threadIdx.x; i < e; i += blockDim.x) {
        const float4 p = pts[i];
        if (!finite3(p)) continue;
        const long long q[3] = {leaf_of(p.x, r), leaf_of(p.y, r), leaf_of(p.z, r)};
        for (int k = 0; k < 3; ++k) {
            mn[k] = q[k] < mn[k] ? q[k] : mn[k];
            mx[k] = q[k] > mx[k] ? q[k] : mx[k];
        }
    }
    __shared__ long long s_mn[3][kThreads], s_mx[3][kThreads];
    for (int k = 0; k < 3; ++k) {
        s_mn[k][threadIdx.x] = mn[k];
        s_mx[k][threadIdx.x] = mx[k];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int t = 1; t < (int)blockDim.x; ++t)
        for (int k = 0; k < 3; ++k) {
            mn[k] = s_mn[k][t] < mn[k] ? s_mn[k][t] : mn[k];
            mx[k] = s_mx[k][t] > mx[k] ? s_mx[k][t] : mx[k];
        }
    ScanGeom g;
    long long span = 0;
    if (mn[0] <= mx[0]) {
        span = 1;
        for (int k = 0; k < 3; ++k) {
            g.lo[k] = mn[k];
            g.d[k] = mx[k] - mn[k] + 1;
            span = (span > (1LL << 31) / g.d[k]) ? (1LL << 32) : span * g.d[k];
        }
    } else {
        for (int k = 0; k < 3; ++k) {
            g.lo[k] = 0;
            g.d[k] = 1;
        }
    }
    if (span >= (1LL << 31)) {
        atomicOr(err, 1);
        span = 0;
    }
    geom[b] = g;
    range[b] = (int)span;
}

// key = base[scan] + local leaf key (x fastest); non-finite points get the
// key of the batch's end (sorted last, dropped); val = point index.
__global__ void key_kernel(const float4 *__restrict__ pts, const int *__restrict__ offsets, int B, float r,
                           const ScanGeom *__restrict__ geom, const int *__restrict__ base, int total_keys, int n,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, int *__restrict__ scan_of) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // scan of point i: binary search in offsets
    int lo = 0, hi = B;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (offsets[mid] <= i) lo = mid; else hi = mid;
    }
    const float4 p = pts[i];
    uint32_t k = (uint32_t)total_keys;
    if (finite3(p)) {
        const ScanGeom &g = geom[lo];
        const long long qx = leaf_of(p.x, r) - g.lo[0], qy = leaf_of(p.y, r) - g.lo[1], qz = leaf_of(p.z, r) - g.lo[2];
        k = (uint32_t)(base[lo] + (int)(qx + g.d[0] * (qy + g.d[1] * qz)));
    }
    keys[i] = k;
    vals[i] = (uint32_t)i;
    scan_of[i] = lo;
}

// One thread per segment: the FP64 mean of its points in input order (the
// stable sort keeps that order within a segment), written to out[s], and one
// count for its scan.  Segments are in key order (scan, then leaf) and the
// segment of dropped points, if any, is the last, so s is the output index.
__global__ void mean_kernel(const float4 *__restrict__ pts, const uint32_t *__restrict__ order,
                            const int32_t *__restrict__ seg_start, const uint32_t *__restrict__ seg_key,
                            const int *__restrict__ nseg, int n, uint32_t drop_key, const int *__restrict__ scan_of,
                            float4 *__restrict__ out, int *__restrict__ count) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int K = *nseg;
    if (s >= K || seg_key[s] == drop_key) return;
    const int a = seg_start[s], e = s + 1 < K ? seg_start[s + 1] : n;
    double sx = 0, sy = 0, sz = 0, sw = 0;
    for (int j = a; j < e; ++j) {
        const float4 p = pts[order[j]];
        sx += (double)p.x;
        sy += (double)p.y;
        sz += (double)p.z;
        sw += (double)p.w;
    }
    const double c = (double)(e - a);
    out[s] = make_float4((float)(sx / c), (float)(sy / c), (float)(sz / c), (float)(sw / c));
    atomicAdd(count + scan_of[order[a]], 1);
}

// Exclusive scan of n ints in place (one thread; n is the scan count + 1);
// *total = the sum, err |= 2 when it reaches 2^31 - 1.
__global__ void scan_small_kernel(int *__restrict__ data, int n, int *__restrict__ total, int *__restrict__ err) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    long long run = 0;
    for (int i = 0; i < n; ++i) {
        const long long v = data[i];
        data[i] = (int)(run < 0x7fffffffLL ? run : 0x7fffffffLL);
        run += v;
    }
    if (run >= 0x7fffffffLL) {
        if (err) atomicOr(err, 2);
        run = 0x7fffffffLL;
    }
    if (total) *total = (int)run;
}

}  // namespace vf

namespace {

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes < 256 ? 256 : bytes);
        if (e == cudaSuccess) cap = bytes < 256 ? 256 : bytes;
        return e;
    }
    ~Buf() {
        if (p) cudaFree(p);
    }
};

}  // namespace

struct ndt_filter {
    int device = 0;
    cudaStream_t stream = nullptr;
    Buf geom, range, err, keys_scratch, scan_of, seg_start, seg_key, total;
    std::string msg;
};

extern "C" {

int ndt_filter_create(int device, ndt_filter **out) {
    if (!out) return NDT_E_ARG;
    *out = nullptr;
    ndt_filter *f = new ndt_filter();
    f->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete f;
        return NDT_E_CUDA;
    }
    *out = f;
    return NDT_OK;
}

void ndt_filter_destroy(ndt_filter *f) {
    if (!f) return;
    cudaSetDevice(f->device);
    if (f->stream) {
        cudaStreamSynchronize(f->stream);
        cudaStreamDestroy(f->stream);
    }
    delete f;
}

const char *ndt_filter_last_error(const ndt_filter *f) { return f ? f->msg.c_str() : "null filter"; }

void *ndt_filter_stream(ndt_filter *f) { return f ? (void *)f->stream : nullptr; }

#define FCK(call)                                                                  \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            f->msg = std::string(#call) + ": " + cudaGetErrorString(e_);          \
            return NDT_E_CUDA;                                                     \
        }                                                                          \
    } while (0)

int ndt_voxel_filter_device(ndt_filter *f, int B, const float *d_points, const int *d_offsets, int total_points,
                            float leaf, float *d_out, int *d_out_offsets, int *out_total) {
    if (!f || B <= 0 || total_points < 0 || !d_points || !d_offsets || !d_out || !d_out_offsets || !out_total ||
        !(leaf > 0.0f) || !std::isfinite(leaf)) {
        if (f) f->msg = "bad argument";
        return NDT_E_ARG;
    }
    FCK(cudaSetDevice(f->device));
    cudaStream_t st = f->stream;
    const int n = total_points;
    const float r = 1.0f / leaf;
    FCK(f->geom.ensure(sizeof(vf::ScanGeom) * (size_t)B));
    FCK(f->range.ensure(sizeof(int) * (size_t)(B + 1)));
    FCK(f->err.ensure(sizeof(int) * 2));
    FCK(cudaMemsetAsync(f->err.p, 0, sizeof(int) * 2, st));
    int *range = (int *)f->range.p;
    int *err = (int *)f->err.p;
    vf::scan_box_kernel<<<B, vf::kThreads, 0, st>>>((const float4 *)d_points, d_offsets, r, (vf::ScanGeom *)f->geom.p,
                                                    range, err);
    FCK(cudaGetLastError());
    FCK(cudaMemsetAsync(range + B, 0, sizeof(int), st));
    vf::scan_small_kernel<<<1, 1, 0, st>>>(range, B + 1, err + 1, err);  // range -> base, total keys
    FCK(cudaGetLastError());
    int h[2] = {0, 0};
    FCK(cudaMemcpyAsync(h, err, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    if (h[0]) {
        f->msg = (h[0] & 1) ? "a scan spans 2^31 leaves or more" : "the batch spans 2^31 - 1 leaves or more";
        return NDT_E_CAPACITY;
    }
    const int total_keys = h[1];  // key total_keys marks the dropped points
    if (n == 0) {
        FCK(cudaMemsetAsync(d_out_offsets, 0, sizeof(int) * (size_t)(B + 1), st));
        FCK(cudaStreamSynchronize(st));
        *out_total = 0;
        return NDT_OK;
    }
    int bits = 1;
    while (bits < 32 && (1LL << bits) <= (long long)total_keys) ++bits;
    FCK(f->keys_scratch.ensure(ndt::sort_scratch_bytes(n)));
    FCK(f->scan_of.ensure(sizeof(int) * (size_t)n));
    FCK(f->seg_start.ensure(sizeof(int32_t) * (size_t)n));
    FCK(f->seg_key.ensure(sizeof(uint32_t) * (size_t)n));
    ndt::SortBuffers sb = ndt::sort_buffers(f->keys_scratch.p, n);
    vf::key_kernel<<<(n + vf::kThreads - 1) / vf::kThreads, vf::kThreads, 0, st>>>(
        (const float4 *)d_points, d_offsets, B, r, (const vf::ScanGeom *)f->geom.p, range, total_keys, n, sb.k0, sb.v0,
        (int *)f->scan_of.p);
    FCK(cudaGetLastError());
    ndt::sort_segments(sb, n, bits, (int32_t *)f->seg_start.p, (uint32_t *)f->seg_key.p, st);
    FCK(cudaGetLastError());
    FCK(cudaMemsetAsync(d_out_offsets, 0, sizeof(int) * (size_t)(B + 1), st));
    vf::mean_kernel<<<(n + vf::kThreads - 1) / vf::kThreads, vf::kThreads, 0, st>>>(
        (const float4 *)d_points, sb.v0, (const int32_t *)f->seg_start.p, (const uint32_t *)f->seg_key.p, sb.nseg, n,
        (uint32_t)total_keys, (const int *)f->scan_of.p, (float4 *)d_out, d_out_offsets);
    FCK(cudaGetLastError());
    FCK(f->total.ensure(sizeof(int)));
    vf::scan_small_kernel<<<1, 1, 0, st>>>(d_out_offsets, B + 1, (int *)f->total.p, nullptr);
    FCK(cudaGetLastError());
    FCK(cudaMemcpyAsync(out_total, f->total.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    return NDT_OK;
}

}  // extern "C"
