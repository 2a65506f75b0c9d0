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
// Device pipeline for B scans: the leaf bounding box of every scan (warps
// over the packed points, 64-bit atomics) and its leaf-key range; an
// exclusive scan of the ranges gives every scan a disjoint key interval, so
// one 32-bit key per point (scan interval base + local leaf key) orders
// points by scan, then leaf; one stable radix sort and segmentation of all
// points (shared with the voxel-grid build); the points gathered into key
// order; per segment the FP64 mean in input order; output offsets by lower
// bounds of the scans' key bases in the sorted segment keys.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ndt_b200.h"
#include "grid_build.h"
#include "nvtx_range.h"

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

// Scan of point (or key) i: the last b in [0, B) with first[b] <= i, for a
// non-decreasing first[] (point offsets, or key bases: with empty scans the
// search lands on the scan that owns i).
__device__ __forceinline__ int owner(const int *__restrict__ first, int B, int i) {
    int lo = 0, hi = B;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(first + mid) <= i) lo = mid; else hi = mid;
    }
    return lo;
}

constexpr int kBoxWarpPoints = 1024;  // points per warp in the box pass

// Leaf bounding boxes: box[6 b .. 6 b + 5] = min x, y, z, max x, y, z leaf
// index of scan b's finite points, by 64-bit atomics (order-independent).
// Each warp walks kBoxWarpPoints consecutive points 32 at a time and keeps a
// per-lane box while the points stay in one scan; a step that crosses a scan
// boundary flushes it and settles its points one by one.
__device__ __forceinline__ void box_flush(long long *__restrict__ box, int b, long long (&mn)[3],
                                          long long (&mx)[3]) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const long long a = __shfl_xor_sync(0xffffffffu, mn[k], o);
            const long long c = __shfl_xor_sync(0xffffffffu, mx[k], o);
            mn[k] = a < mn[k] ? a : mn[k];
            mx[k] = c > mx[k] ? c : mx[k];
        }
    if ((threadIdx.x & 31) == 0 && mn[0] <= mx[0])
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicMin(box + 6 * b + k, mn[k]);
            atomicMax(box + 6 * b + 3 + k, mx[k]);
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        mn[k] = LLONG_MAX;
        mx[k] = LLONG_MIN;
    }
}

__global__ void box_kernel(const float4 *__restrict__ pts, const int *__restrict__ offsets, int B, int n, float r,
                           long long *__restrict__ box) {
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long w0l = gw * kBoxWarpPoints;
    if (w0l >= n) return;
    const int w0 = (int)w0l, w1 = n - w0 < kBoxWarpPoints ? n : w0 + kBoxWarpPoints;
    int cur = owner(offsets, B, w0);
    int hi = __ldg(offsets + cur + 1);
    long long mn[3] = {LLONG_MAX, LLONG_MAX, LLONG_MAX}, mx[3] = {LLONG_MIN, LLONG_MIN, LLONG_MIN};
    for (int base = w0; base < w1; base += 32) {
        const int i = base + lane;
        const int last = base + 31 < w1 ? base + 31 : w1 - 1;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        bool ok = i < w1;
        if (ok) {
            p = pts[i];
            ok = finite3(p);
        }
        long long q[3] = {0, 0, 0};
        if (ok) {
            q[0] = leaf_of(p.x, r);
            q[1] = leaf_of(p.y, r);
            q[2] = leaf_of(p.z, r);
        }
        if (last < hi) {  // warp-uniform: the whole step lies in scan cur
            if (ok)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    mn[k] = q[k] < mn[k] ? q[k] : mn[k];
                    mx[k] = q[k] > mx[k] ? q[k] : mx[k];
                }
        } else {
            box_flush(box, cur, mn, mx);
            if (ok) {
                const int b = owner(offsets, B, i);
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    atomicMin(box + 6 * b + k, q[k]);
                    atomicMax(box + 6 * b + 3 + k, q[k]);
                }
            }
            if (base + 32 < w1) {
                cur = owner(offsets, B, base + 32);
                hi = __ldg(offsets + cur + 1);
            }
        }
    }
    box_flush(box, cur, mn, mx);
}

__global__ void box_init_kernel(long long *__restrict__ box, int B) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 6 * B; i += gridDim.x * blockDim.x)
        box[i] = (i % 6) < 3 ? LLONG_MAX : LLONG_MIN;
}

// One block: per scan its geometry and key range (dx * dy * dz, 0 without
// finite points), the exclusive scan of the ranges into key bases
// (base[B] = total), and the box reset for the next call.  flags[0] |= 1 when
// a scan spans 2^31 leaves or more, |= 2 when the batch spans 2^31 - 1 or
// more; flags[1] = total.
constexpr int kRangeThreads = 1024;

__global__ void __launch_bounds__(kRangeThreads) range_kernel(long long *__restrict__ box, int B,
                                                              ScanGeom *__restrict__ geom, int *__restrict__ base,
                                                              int *__restrict__ flags) {
    __shared__ long long s_sum[kRangeThreads];
    const int t = threadIdx.x;
    const int per = (B + kRangeThreads - 1) / kRangeThreads;
    const int b0 = t * per, b1 = b0 + per < B ? b0 + per : B;
    long long local = 0;
    int err = 0;
    for (int b = b0; b < b1; ++b) {
        ScanGeom g;
        long long span = 0;
        const long long *bx = box + 6 * b;
        if (bx[0] <= bx[3]) {
            span = 1;
            for (int k = 0; k < 3; ++k) {
                g.lo[k] = bx[k];
                g.d[k] = bx[3 + k] - bx[k] + 1;
                span = (span > (1LL << 31) / g.d[k]) ? (1LL << 32) : span * g.d[k];
            }
        } else {
            for (int k = 0; k < 3; ++k) {
                g.lo[k] = 0;
                g.d[k] = 1;
            }
        }
        if (span >= (1LL << 31)) {
            err |= 1;
            span = 0;
        }
        geom[b] = g;
        base[b] = (int)span;  // the range for now; the scan below makes it a base
        local += span;
        for (int k = 0; k < 6; ++k) box[6 * b + k] = k < 3 ? LLONG_MAX : LLONG_MIN;
    }
    s_sum[t] = local;
    __syncthreads();
    for (int o = 1; o < kRangeThreads; o <<= 1) {  // inclusive Hillis-Steele scan
        const long long v = t >= o ? s_sum[t - o] : 0;
        __syncthreads();
        s_sum[t] += v;
        __syncthreads();
    }
    long long run = s_sum[t] - local;
    const long long total = s_sum[kRangeThreads - 1];
    const long long cap = 0x7fffffffLL;
    for (int b = b0; b < b1; ++b) {
        const int span = base[b];
        base[b] = (int)(run < cap ? run : cap);
        run += span;
    }
    if (err) atomicOr(flags, 1);
    if (t == 0) {
        if (total >= cap) atomicOr(flags, 2);
        base[B] = (int)(total < cap ? total : cap);
        flags[1] = (int)(total < cap ? total : cap);
    }
}

// key = base[scan] + local leaf key (x fastest); non-finite points get the
// key of the batch's end (sorted last, dropped); val = point index.
__global__ void key_kernel(const float4 *__restrict__ pts, const int *__restrict__ offsets, int B, float r,
                           const ScanGeom *__restrict__ geom, const int *__restrict__ base, int total_keys, int n,
                           uint32_t *__restrict__ keys, uint32_t *__restrict__ vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pts[i];
    uint32_t k = (uint32_t)total_keys;
    if (finite3(p)) {
        const int b = owner(offsets, B, i);
        const ScanGeom &g = geom[b];
        const long long qx = leaf_of(p.x, r) - g.lo[0], qy = leaf_of(p.y, r) - g.lo[1], qz = leaf_of(p.z, r) - g.lo[2];
        k = (uint32_t)(base[b] + (int)(qx + g.d[0] * (qy + g.d[1] * qz)));
    }
    keys[i] = k;
    vals[i] = (uint32_t)i;
}

// sorted[j] = pts[order[j]]: the points in key order (one thread per point,
// so the random reads are all in flight at once; writes coalesced).
__global__ void gather_kernel(const float4 *__restrict__ pts, const uint32_t *__restrict__ order, int n,
                              float4 *__restrict__ sorted) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) sorted[j] = pts[__ldg(order + j)];
}

// One thread per segment: the FP64 mean of its points in input order (the
// stable sort keeps that order within a segment), written to out[s].
// Segments are in key order (scan, then leaf) and the segment of dropped
// points, if any, is the last, so s is the output index.
__global__ void mean_kernel(const float4 *__restrict__ sorted, const int32_t *__restrict__ seg_start,
                            const uint32_t *__restrict__ seg_key, const int *__restrict__ nseg, int n,
                            uint32_t drop_key, float4 *__restrict__ out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    const int K = *nseg;
    if (s >= K || seg_key[s] == drop_key) return;
    const int a = seg_start[s], e = s + 1 < K ? seg_start[s + 1] : n;
    double sx = 0, sy = 0, sz = 0, sw = 0;
    for (int j = a; j < e; ++j) {
        const float4 p = sorted[j];
        sx += (double)p.x;
        sy += (double)p.y;
        sz += (double)p.z;
        sw += (double)p.w;
    }
    const double c = (double)(e - a);
    out[s] = make_float4((float)(sx / c), (float)(sy / c), (float)(sz / c), (float)(sw / c));
}

// Output offsets without atomics: scan b's leaves are the segments with keys
// in [base[b], base[b + 1]), so out_off[b] = the number of segments with a
// key below base[b] (a lower bound in the sorted segment keys), b = 0 .. B
// (base[B] = the key total = the dropped points' key).
__global__ void offsets_kernel(const uint32_t *__restrict__ seg_key, const int *__restrict__ nseg,
                               const int *__restrict__ base, int B, int *__restrict__ out_off) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > B) return;
    const uint32_t k = (uint32_t)base[b];
    int lo = 0, hi = *nseg;  // first index in [lo, hi] with seg_key >= k
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (seg_key[mid] < k) lo = mid + 1; else hi = mid;
    }
    out_off[b] = lo;
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
    Buf geom, base, flags, box, sort_scratch, seg_start, seg_key, sorted;
    int box_cap = 0;
    int *h_flags = nullptr;  // pinned: error flags, key total, output total
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
    if (e == cudaSuccess) e = cudaMallocHost((void **)&f->h_flags, sizeof(int) * 4);
    if (e != cudaSuccess) {
        ndt_filter_destroy(f);
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
    if (f->h_flags) cudaFreeHost(f->h_flags);
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
    ndt::NvtxRange range("voxel filter");
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
    FCK(f->base.ensure(sizeof(int) * (size_t)(B + 1)));
    FCK(f->flags.ensure(sizeof(int) * 4));
    if (f->box_cap < B) {  // the range pass resets the boxes it read; a fresh buffer is set once
        FCK(f->box.ensure(sizeof(long long) * 6 * (size_t)B));
        vf::box_init_kernel<<<(6 * B + 255) / 256, 256, 0, st>>>((long long *)f->box.p, B);
        FCK(cudaGetLastError());
        f->box_cap = B;
    }
    long long *box = (long long *)f->box.p;
    int *base = (int *)f->base.p;
    int *flags = (int *)f->flags.p;
    FCK(cudaMemsetAsync(flags, 0, sizeof(int) * 4, st));
    if (n > 0) {
        const long long warps = ((long long)n + vf::kBoxWarpPoints - 1) / vf::kBoxWarpPoints;
        vf::box_kernel<<<(unsigned)((warps * 32 + vf::kThreads - 1) / vf::kThreads), vf::kThreads, 0, st>>>(
            (const float4 *)d_points, d_offsets, B, n, r, box);
        FCK(cudaGetLastError());
    }
    vf::range_kernel<<<1, vf::kRangeThreads, 0, st>>>(box, B, (vf::ScanGeom *)f->geom.p, base, flags);
    FCK(cudaGetLastError());
    FCK(cudaMemcpyAsync(f->h_flags, flags, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    if (f->h_flags[0]) {
        f->msg = (f->h_flags[0] & 1) ? "a scan spans 2^31 leaves or more" : "the batch spans 2^31 - 1 leaves or more";
        return NDT_E_CAPACITY;
    }
    const int total_keys = f->h_flags[1];  // key total_keys marks the dropped points
    if (n == 0) {
        FCK(cudaMemsetAsync(d_out_offsets, 0, sizeof(int) * (size_t)(B + 1), st));
        FCK(cudaStreamSynchronize(st));
        *out_total = 0;
        return NDT_OK;
    }
    int bits = 1;
    while (bits < 32 && (1LL << bits) <= (long long)total_keys) ++bits;
    FCK(f->sort_scratch.ensure(ndt::sort_scratch_bytes(n)));
    FCK(f->seg_start.ensure(sizeof(int32_t) * (size_t)n));
    FCK(f->seg_key.ensure(sizeof(uint32_t) * (size_t)n));
    FCK(f->sorted.ensure(sizeof(float4) * (size_t)n));
    ndt::SortBuffers sb = ndt::sort_buffers(f->sort_scratch.p, n);
    const unsigned pblk = (unsigned)((n + vf::kThreads - 1) / vf::kThreads);
    vf::key_kernel<<<pblk, vf::kThreads, 0, st>>>((const float4 *)d_points, d_offsets, B, r,
                                                  (const vf::ScanGeom *)f->geom.p, base, total_keys, n, sb.k0, sb.v0);
    FCK(cudaGetLastError());
    ndt::sort_segments(sb, n, bits, (int32_t *)f->seg_start.p, (uint32_t *)f->seg_key.p, st);
    FCK(cudaGetLastError());
    vf::gather_kernel<<<pblk, vf::kThreads, 0, st>>>((const float4 *)d_points, sb.v0, n, (float4 *)f->sorted.p);
    vf::mean_kernel<<<pblk, vf::kThreads, 0, st>>>((const float4 *)f->sorted.p, (const int32_t *)f->seg_start.p,
                                                   (const uint32_t *)f->seg_key.p, sb.nseg, n, (uint32_t)total_keys,
                                                   (float4 *)d_out);
    vf::offsets_kernel<<<(B + 1 + vf::kThreads - 1) / vf::kThreads, vf::kThreads, 0, st>>>(
        (const uint32_t *)f->seg_key.p, sb.nseg, base, B, d_out_offsets);
    FCK(cudaGetLastError());
    FCK(cudaMemcpyAsync(f->h_flags + 2, d_out_offsets + B, sizeof(int), cudaMemcpyDeviceToHost, st));
    FCK(cudaStreamSynchronize(st));
    *out_total = f->h_flags[2];
    return NDT_OK;
}

}  // extern "C"
