// Voxel-grid build on the device (replaces ndt_mapping::initCompute,
// src/CPU/ndt_mapping/kernel.cpp:1302-1373).
//
// Pipeline (one map):
//   bbox_partial / bbox_final   bounding box +-0.01, dims, G        (:1305-1322)
//   cell_key                    dense cell id of every map point     (:1343, :236-244)
//   radix_{upsweep,scan,down}   stable LSD sort of (cell, point index)
//   seg_{count,write}           one segment per occupied cell
//   cell_finalize_{compat,corrected}
//                               per-cell sums in point order, covariance, inverse
//
// Because the sort is stable, every cell's points are visited in the map's
// original order, so the FP64 sums of the compat finaliser are the reference's
// sequential sums bit for bit (the reference adds points in index order,
// :1341-1353).  No floating-point atomics are used anywhere.
#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

#include "grid_build.h"
#include "ndt_math.cuh"

namespace ndt {

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;                       // items per thread in the sort / segment tiles
constexpr int kSortTile = kThreads * kItems;    // 2048
constexpr int kWarps = kThreads / 32;
constexpr int kMaxDigits = 1 << 10;             // radix digits of one pass, at most
// Scratch layout: [bounding-box partials (6 x 1024 floats) + its 2 counters,
// which must stay zero between builds] [sort and segment buffers].
constexpr size_t kBboxFlagsOffset = sizeof(float) * 6 * 1024;
constexpr size_t kBboxBytes = kBboxFlagsOffset + 256;

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---------------------------------------------------------------------------
// Bounding box.  min/max are exact in any order; NaN/inf points are counted
// and make the build fail (the reference's behaviour there is undefined).
// One kernel: block partial min/max, then the last block to finish (atomic
// ticket) reduces the partials and computes the grid geometry with the
// reference's float arithmetic (kernel.cpp:1305-1322).  *flags = {ticket,
// non-finite}: zero on entry, reset to zero by the last block.
__global__ void bbox_kernel(const float4 *__restrict__ map, int m, float *__restrict__ part, int *__restrict__ flags,
                            float res, GridMeta *__restrict__ meta) {
    float mn0 = FLT_MAX, mn1 = FLT_MAX, mn2 = FLT_MAX;
    float mx0 = -FLT_MAX, mx1 = -FLT_MAX, mx2 = -FLT_MAX;
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        float4 p = map[i];
        if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) {
            bad = 1;
            continue;
        }
        mn0 = fminf(mn0, p.x); mn1 = fminf(mn1, p.y); mn2 = fminf(mn2, p.z);
        mx0 = fmaxf(mx0, p.x); mx1 = fmaxf(mx1, p.y); mx2 = fmaxf(mx2, p.z);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn0 = fminf(mn0, __shfl_xor_sync(0xffffffffu, mn0, o));
        mn1 = fminf(mn1, __shfl_xor_sync(0xffffffffu, mn1, o));
        mn2 = fminf(mn2, __shfl_xor_sync(0xffffffffu, mn2, o));
        mx0 = fmaxf(mx0, __shfl_xor_sync(0xffffffffu, mx0, o));
        mx1 = fmaxf(mx1, __shfl_xor_sync(0xffffffffu, mx1, o));
        mx2 = fmaxf(mx2, __shfl_xor_sync(0xffffffffu, mx2, o));
    }
    __shared__ float s[kWarps][6];
    __shared__ int s_last;
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s[w][0] = mn0; s[w][1] = mn1; s[w][2] = mn2;
        s[w][3] = mx0; s[w][4] = mx1; s[w][5] = mx2;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flags + 1, 1);
    if (threadIdx.x < 6) {
        float v = s[0][threadIdx.x];
        for (int k = 1; k < kWarps; ++k)
            v = threadIdx.x < 3 ? fminf(v, s[k][threadIdx.x]) : fmaxf(v, s[k][threadIdx.x]);
        part[6 * blockIdx.x + threadIdx.x] = v;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(flags, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // min/max of the block partials (exact in any order)
    const int nblk = gridDim.x;
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        for (int k = 0; k < 6; ++k) {
            const float x = __ldcg(part + 6 * b + k);
            v[k] = k < 3 ? fminf(v[k], x) : fmaxf(v[k], x);
        }
    for (int o = 16; o > 0; o >>= 1)
        for (int k = 0; k < 6; ++k) {
            float u = __shfl_xor_sync(0xffffffffu, v[k], o);
            v[k] = k < 3 ? fminf(v[k], u) : fmaxf(v[k], u);
        }
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < 6; ++k) s[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww)
        for (int k = 0; k < 6; ++k) v[k] = k < 3 ? fminf(v[k], s[ww][k]) : fmaxf(v[k], s[ww][k]);
    GridMeta g;
    g.res = res;
    g.occupied = 0;
    g.error = atomicAdd(flags + 1, 0) ? 2 : 0;
    long long G = 1;
    for (int e = 0; e < 3; ++e) {
        g.raw_min[e] = v[e];
        g.raw_max[e] = v[3 + e];
        g.minv[e] = v[e] - 0.01f;
        g.maxv[e] = v[3 + e] + 0.01f;
        float d = (g.maxv[e] - g.minv[e]) / res + 1;
        g.dim[e] = (d >= 1.0f && d < 2147483647.0f) ? (int)d : 0;
        G *= (long long)g.dim[e];
    }
    if (G <= 0 || G > 2147483647LL) {
        if (!g.error) g.error = 1;
        G = 0;
    }
    g.G = G;
    *meta = g;
    flags[0] = 0;
    flags[1] = 0;
}

// Dense cell id of each map point (linearizeCoord, kernel.cpp:236-244).
__global__ void cell_key_kernel(const float4 *__restrict__ map, int m, const GridMeta *__restrict__ meta,
                                uint32_t *__restrict__ keys, uint32_t *__restrict__ vals, int index_offset = 0) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const GridMeta g = *meta;
    if (g.error) return;
    float4 p = map[i];
    int ix = (int)((p.x - g.minv[0]) / g.res);
    int iy = (int)((p.y - g.minv[1]) / g.res);
    int iz = (int)((p.z - g.minv[2]) / g.res);
    keys[i] = (uint32_t)(ix + g.dim[0] * (iy + g.dim[1] * iz));
    vals[i] = (uint32_t)(i + index_offset);
}

// Stable merge of two key-sorted (key, value) runs, run a first on equal
// keys: element t of a lands at t + #{b keys < key}, element j of b at
// j + #{a keys <= key} (binary searches; each output position is written
// once).
__global__ void merge_kernel(const uint32_t *__restrict__ ka, const uint32_t *__restrict__ va, int na,
                             const uint32_t *__restrict__ kb, const uint32_t *__restrict__ vb, int nb,
                             uint32_t *__restrict__ ko, uint32_t *__restrict__ vo) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= na + nb) return;
    if (t < na) {
        const uint32_t key = ka[t];
        int lo = 0, hi = nb;  // first b key >= key
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(kb + mid) < key) lo = mid + 1; else hi = mid;
        }
        ko[t + lo] = key;
        vo[t + lo] = va[t];
    } else {
        const int j = t - na;
        const uint32_t key = kb[j];
        int lo = 0, hi = na;  // first a key > key
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(ka + mid) <= key) lo = mid + 1; else hi = mid;
        }
        ko[j + lo] = key;
        vo[j + lo] = vb[j];
    }
}

// ---------------------------------------------------------------------------
// Stable LSD radix sort of (key, value) pairs, `bits`-wide digit per pass.
// hist layout: digit-major, hist[d * nblk + block].
__global__ void radix_upsweep_kernel(const uint32_t *__restrict__ keys, int n, int shift, int bits,
                                     int *__restrict__ hist) {
    extern __shared__ int s_hist[];
    const int nb = 1 << bits;
    for (int d = threadIdx.x; d < nb; d += blockDim.x) s_hist[d] = 0;
    __syncthreads();
    const int base = blockIdx.x * kSortTile;
    const uint32_t mask = (uint32_t)nb - 1u;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        int i = base + k * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_hist[(keys[i] >> shift) & mask], 1);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < nb; d += blockDim.x) hist[d * gridDim.x + blockIdx.x] = s_hist[d];
}

// Exclusive scan of data[begin, end) in place by one block of 1024 threads,
// starting from `carry`; returns the running total (carry + sum) in every
// thread.  Tiles of 8192 ints are staged in shared memory with coalesced
// loads and stores; each thread scans 8 consecutive values (two 16-byte
// shared loads), the block scans the thread sums, and a carry links the tiles.
constexpr int kScanThreads = 1024, kScanItems = 8, kScanTile = kScanThreads * kScanItems;

__device__ int block_scan_range(int *__restrict__ data, int begin, int end, int carry_in) {
    constexpr int kT = kScanThreads, kI = kScanItems, kTileN = kScanTile;
    __shared__ __align__(16) int s_data[kTileN];
    __shared__ int s_warp[32];
    __shared__ int s_carry;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) s_carry = carry_in;
    for (int base = begin; base < end; base += kTileN) {
        for (int i = t; i < kTileN; i += kT) s_data[i] = base + i < end ? data[base + i] : 0;
        __syncthreads();
        const int4 a = reinterpret_cast<const int4 *>(s_data)[2 * t];
        const int4 b = reinterpret_cast<const int4 *>(s_data)[2 * t + 1];
        const int v[kI] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        int sum = 0;
#pragma unroll
        for (int k = 0; k < kI; ++k) sum += v[k];
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        if (lane == 31) s_warp[w] = incl;
        const int carry = s_carry;
        __syncthreads();
        if (w == 0) {
            const int x = s_warp[lane];
            int inc2 = x;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, inc2, o);
                if (lane >= o) inc2 += u;
            }
            s_warp[lane] = inc2 - x;
            if (lane == 31) s_carry = carry + inc2;
        }
        __syncthreads();
        int run = carry + s_warp[w] + incl - sum;
        int o[kI];
#pragma unroll
        for (int k = 0; k < kI; ++k) {
            o[k] = run;
            run += v[k];
        }
        reinterpret_cast<int4 *>(s_data)[2 * t] = make_int4(o[0], o[1], o[2], o[3]);
        reinterpret_cast<int4 *>(s_data)[2 * t + 1] = make_int4(o[4], o[5], o[6], o[7]);
        __syncthreads();
        for (int i = t; i < kTileN; i += kT)
            if (base + i < end) data[base + i] = s_data[i];
        __syncthreads();
    }
    return s_carry;
}

// Exclusive scan of n ints in place with one block; *total (optional)
// receives the sum.
__global__ void __launch_bounds__(kScanThreads) scan_single_block_kernel(int *__restrict__ data, int n,
                                                                         int *__restrict__ total) {
    const int run = block_scan_range(data, 0, n, 0);
    if (total && threadIdx.x == 0) *total = run;
}

// Multi-block form for long arrays: part[b] = sum of tile b (8192 ints) ...
__global__ void __launch_bounds__(kScanThreads) scan_tile_sum_kernel(const int *__restrict__ data, int n,
                                                                     int *__restrict__ part) {
    __shared__ int s_warp[32];
    const int base = blockIdx.x * kScanTile;
    int sum = 0;
    for (int i = threadIdx.x; i < kScanTile; i += kScanThreads)
        if (base + i < n) sum += data[base + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) s_warp[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        sum = s_warp[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (threadIdx.x == 0) part[blockIdx.x] = sum;
    }
}

// ... then, after part is scanned, tile b scans itself from carry part[b].
__global__ void __launch_bounds__(kScanThreads) scan_tile_kernel(int *__restrict__ data, int n,
                                                                 const int *__restrict__ part) {
    const int base = blockIdx.x * kScanTile;
    const int end = base + kScanTile < n ? base + kScanTile : n;
    block_scan_range(data, base, end, part[blockIdx.x]);
}

// Arrays of at most this many ints are scanned by one block (one launch);
// longer ones by tiles (three launches, part holds one int per tile).
constexpr int kSingleScanMax = 8 * kScanTile;

int scan_exclusive(int *data, int n, int *total, int *part, cudaStream_t st) {
    if (n <= kSingleScanMax) {
        scan_single_block_kernel<<<1, kScanThreads, 0, st>>>(data, n, total);
        return 1;
    }
    const int tiles = (n + kScanTile - 1) / kScanTile;
    scan_tile_sum_kernel<<<tiles, kScanThreads, 0, st>>>(data, n, part);
    scan_single_block_kernel<<<1, kScanThreads, 0, st>>>(part, tiles, total);
    scan_tile_kernel<<<tiles, kScanThreads, 0, st>>>(data, n, part);
    return 3;
}

size_t scan_part_ints(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

// Stable scatter: warp w of a block owns items [base + w*256, base + w*256 + 256)
// in 8 chunks of 32 consecutive items; ranks inside a chunk come from
// __match_any_sync peer masks, so equal digits keep their input order.
__global__ void radix_downsweep_kernel(const uint32_t *__restrict__ kin, const uint32_t *__restrict__ vin,
                                       uint32_t *__restrict__ kout, uint32_t *__restrict__ vout, int n,
                                       int shift, int bits, const int *__restrict__ hist) {
    extern __shared__ int s_cnt[];  // [kWarps][nb]
    const int nb = 1 << bits;
    const uint32_t mask = (uint32_t)nb - 1u;
    for (int d = threadIdx.x; d < kWarps * nb; d += blockDim.x) s_cnt[d] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wbase = blockIdx.x * kSortTile + w * (32 * kItems);
    int *cnt = s_cnt + w * nb;
    uint32_t key[kItems], val[kItems];
    int rank[kItems];
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        int i = wbase + k * 32 + lane;
        bool valid = i < n;
        key[k] = valid ? kin[i] : 0u;
        val[k] = valid ? vin[i] : 0u;
        uint32_t d = valid ? ((key[k] >> shift) & mask) : (uint32_t)nb;  // sentinel group
        unsigned peers = __match_any_sync(0xffffffffu, d);
        int before = valid ? cnt[d] : 0;
        __syncwarp();
        rank[k] = before + __popc(peers & lt);
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) cnt[d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps, per digit
    for (int d = threadIdx.x; d < nb; d += blockDim.x) {
        int run = 0;
        for (int ww = 0; ww < kWarps; ++ww) {
            int c = s_cnt[ww * nb + d];
            s_cnt[ww * nb + d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        int i = wbase + k * 32 + lane;
        if (i < n) {
            uint32_t d = (key[k] >> shift) & mask;
            int pos = hist[d * gridDim.x + blockIdx.x] + cnt[d] + rank[k];
            kout[pos] = key[k];
            vout[pos] = val[k];
        }
    }
}

// ---------------------------------------------------------------------------
// Segments of equal keys in the sorted order = occupied cells.
__device__ __forceinline__ bool is_head(const uint32_t *k, int i) { return i == 0 || k[i] != k[i - 1]; }

__global__ void seg_count_kernel(const uint32_t *__restrict__ keys, int n, int *__restrict__ counts) {
    int c = 0;
    const int base = blockIdx.x * kSortTile;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        int i = base + k * kThreads + threadIdx.x;
        if (i < n && is_head(keys, i)) ++c;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int s[kWarps];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < kWarps; ++k) t += s[k];
        counts[blockIdx.x] = t;
    }
}

// Writes seg_start[s] and seg_cell[s] for every segment head, s in sorted order.
__global__ void seg_write_kernel(const uint32_t *__restrict__ keys, int n, const int *__restrict__ offsets,
                                 int *__restrict__ seg_start, uint32_t *__restrict__ seg_cell) {
    __shared__ int s_warp[kWarps];
    __shared__ int s_run;
    if (threadIdx.x == 0) s_run = offsets[blockIdx.x];
    const int base = blockIdx.x * kSortTile;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int k = 0; k < kItems; ++k) {
        int i = base + k * kThreads + threadIdx.x;
        bool h = i < n && is_head(keys, i);
        unsigned b = __ballot_sync(0xffffffffu, h);
        if (lane == 0) s_warp[w] = __popc(b);
        __syncthreads();
        int before = 0, total = 0;
        for (int ww = 0; ww < kWarps; ++ww) {
            int c = s_warp[ww];
            if (ww < w) before += c;
            total += c;
        }
        int run = s_run;
        if (h) {
            int s = run + before + __popc(b & lanemask_lt());
            seg_start[s] = i;
            seg_cell[s] = keys[i];
        }
        __syncthreads();
        if (threadIdx.x == 0) s_run = run + total;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Voxel records.
__device__ bool write_records(int s, const double *mu, const double *C, GridBuffers buf) {
    bool bad = false;
    for (int k = 0; k < 9; ++k) {
        double v = C[k];
        if (!(fabs(v) <= 1e30)) bad = true;  // also catches NaN
    }
    for (int k = 0; k < 3; ++k)
        if (!isfinite(mu[k])) bad = true;
    buf.mean[s] = make_double4(mu[0], mu[1], mu[2], bad ? 1.0 : 0.0);
    const float h0 = (float)mu[0], h1 = (float)mu[1], h2 = (float)mu[2];
    float c00 = (float)C[0], c11 = (float)C[4], c22 = (float)C[8];
    float c01 = (float)((C[1] + C[3]) * 0.5), c02 = (float)((C[2] + C[6]) * 0.5), c12 = (float)((C[5] + C[7]) * 0.5);
    float4 *r = buf.vox32 + 3 * (size_t)s;  // the FP32 pair record (GridDev::vox32)
    r[0] = make_float4(h0, h1, h2, c00);
    r[1] = make_float4((float)(mu[0] - (double)h0), (float)(mu[1] - (double)h1), (float)(mu[2] - (double)h2), c01);
    r[2] = make_float4(c02, c11, c12, c22);
    for (int k = 0; k < 9; ++k) buf.icov64[9 * (size_t)s + k] = C[k];
    return bad;
}

// Reference voxel (kernel.cpp:1324-1372): sums start at mean = 0 and
// invCovariance = anti-diagonal identity; every point adds its float xyz and
// the float products x_r * x_c; then mean = sum / N and
//   S_rc = ((S_rc - 2 (sum_r mean_c)) / G + mean_r mean_c) * ((G - 1) / N)
// (G = dense cell count), inverted by adjugate (invertMatrix, :1277-1300).
__device__ void compat_cell(const float4 *__restrict__ map, const uint32_t *__restrict__ order, int lo, int hi,
                            double Gd, int s, uint32_t cell_id, GridBuffers buf) {
    double sum[3] = {0.0, 0.0, 0.0};
    double S[9] = {0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0};
    int cnt = 0;
    for (int j = lo; j < hi; ++j) {
        float4 p = map[order[j]];
        const float v[3] = {p.x, p.y, p.z};
        sum[0] += v[0];
        sum[1] += v[1];
        sum[2] += v[2];
        ++cnt;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) S[3 * r + c] += (double)(v[r] * v[c]);
    }
    double mu[3];
    for (int e = 0; e < 3; ++e) mu[e] = sum[e] / cnt;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double v = (S[3 * r + c] - 2 * (sum[r] * mu[c])) / Gd + mu[r] * mu[c];
            S[3 * r + c] = v * ((Gd - 1.0) / cnt);
        }
    // adjugate / determinant
    const double *m = S;
    double det = m[0] * (m[8] * m[4] - m[7] * m[5]) - m[3] * (m[8] * m[1] - m[7] * m[2]) +
                 m[6] * (m[5] * m[1] - m[4] * m[2]);
    double inv_det = 1.0 / det;
    double t[9];
    t[0] = m[8] * m[4] - m[7] * m[5];
    t[1] = -(m[8] * m[1] - m[7] * m[2]);
    t[2] = m[5] * m[1] - m[4] * m[2];
    t[3] = -(m[8] * m[1] - m[6] * m[5]);
    t[4] = m[8] * m[0] - m[7] * m[2];
    t[5] = -(m[5] * m[0] - m[3] * m[2]);
    t[6] = m[7] * m[3] - m[6] * m[4];
    t[7] = -(m[7] * m[0] - m[6] * m[1]);
    t[8] = m[4] * m[0] - m[3] * m[1];
    double C[9];
    for (int k = 0; k < 9; ++k) C[k] = t[k] * inv_det;
    const bool flag = write_records(s, mu, C, buf);
    buf.count[s] = cnt;
    buf.cell[s] = (int)cell_id;
    buf.index[cell_id] = s | (flag ? kSlotFlag : 0);
    buf.slot_of[cell_id] = s;
}

__global__ void cell_finalize_compat_kernel(const float4 *__restrict__ map, const uint32_t *__restrict__ order,
                                            const int *__restrict__ seg_start, const uint32_t *__restrict__ seg_cell,
                                            const int *__restrict__ nseg, int n, GridMeta *__restrict__ meta,
                                            GridBuffers buf) {
    const int K = *nseg;
    if (blockIdx.x == 0 && threadIdx.x == 0) meta->occupied = K;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= K) return;
    const int lo = seg_start[s], hi = (s + 1 < K) ? seg_start[s + 1] : n;
    compat_cell(map, order, lo, hi, (double)meta->G, s, seg_cell[s], buf);
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations (V columns =
// eigenvectors); the same algorithm as the FP64 oracle's.
__device__ void jacobi3(double A[3][3], double V[3][3], double w[3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 16; ++sweep) {
        double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double apq = A[p][q];
                if (apq == 0.0) continue;
                double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {
                    double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {
                    double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) w[i] = A[i][i];
}

// Corrected voxel: mean, centred covariance / (N - 1), usable only with at
// least min_points points, eigenvalues floored at eig_ratio * max, inverse
// as V diag(1 / w) V^T.
__device__ void corrected_cell(const float4 *__restrict__ map, const uint32_t *__restrict__ order, int lo, int hi,
                               int min_points, double eig_ratio, int s, uint32_t cell_id, GridBuffers buf) {
    const int cnt = hi - lo;
    buf.count[s] = cnt;
    buf.cell[s] = (int)cell_id;
    buf.slot_of[cell_id] = s;
    // a cell that is not usable has index -1; its records read NaN
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    const double nan3[3] = {qnan, qnan, qnan};
    const double nan9[9] = {qnan, qnan, qnan, qnan, qnan, qnan, qnan, qnan, qnan};
    if (cnt < min_points || cnt < 2) {
        write_records(s, nan3, nan9, buf);
        buf.index[cell_id] = -1;
        return;
    }
    double sum[3] = {0.0, 0.0, 0.0};
    for (int j = lo; j < hi; ++j) {
        float4 p = map[order[j]];
        sum[0] += (double)p.x;
        sum[1] += (double)p.y;
        sum[2] += (double)p.z;
    }
    double mu[3];
    for (int e = 0; e < 3; ++e) mu[e] = sum[e] / cnt;
    double m2[6] = {0, 0, 0, 0, 0, 0};
    for (int j = lo; j < hi; ++j) {
        float4 p = map[order[j]];
        double d0 = p.x - mu[0], d1 = p.y - mu[1], d2 = p.z - mu[2];
        m2[0] += d0 * d0; m2[1] += d0 * d1; m2[2] += d0 * d2;
        m2[3] += d1 * d1; m2[4] += d1 * d2; m2[5] += d2 * d2;
    }
    double A[3][3] = {{m2[0], m2[1], m2[2]}, {m2[1], m2[3], m2[4]}, {m2[2], m2[4], m2[5]}};
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q) A[r][q] /= (cnt - 1);
    double V[3][3], w[3];
    jacobi3(A, V, w);
    double wmax = fmax(w[0], fmax(w[1], w[2]));
    if (!(wmax > 0.0) || !isfinite(wmax)) {
        write_records(s, nan3, nan9, buf);
        buf.index[cell_id] = -1;
        return;
    }
    double floor_v = eig_ratio * wmax;
    double inv_w[3];
    for (int e = 0; e < 3; ++e) {
        double we = w[e] < floor_v ? floor_v : w[e];
        if (!(we > 0.0)) {
            write_records(s, nan3, nan9, buf);
            buf.index[cell_id] = -1;
            return;
        }
        inv_w[e] = 1.0 / we;
    }
    double C[9];
    for (int r = 0; r < 3; ++r)
        for (int q = 0; q < 3; ++q)
            C[3 * r + q] = V[r][0] * inv_w[0] * V[q][0] + V[r][1] * inv_w[1] * V[q][1] + V[r][2] * inv_w[2] * V[q][2];
    const bool flag = write_records(s, mu, C, buf);
    buf.index[cell_id] = s | (flag ? kSlotFlag : 0);
}

__global__ void cell_finalize_corrected_kernel(const float4 *__restrict__ map, const uint32_t *__restrict__ order,
                                               const int *__restrict__ seg_start,
                                               const uint32_t *__restrict__ seg_cell, const int *__restrict__ nseg,
                                               int n, int min_points, double eig_ratio, GridMeta *__restrict__ meta,
                                               GridBuffers buf) {
    const int K = *nseg;
    if (blockIdx.x == 0 && threadIdx.x == 0) meta->occupied = K;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= K) return;
    const int lo = seg_start[s], hi = (s + 1 < K) ? seg_start[s + 1] : n;
    corrected_cell(map, order, lo, hi, min_points, eig_ratio, s, seg_cell[s], buf);
}

// Map growth, touched cells only.  new_keys: the appended points' cell keys,
// sorted; keys / order: all points' sorted (cell, point) pairs.  Pass 1:
// fresh[j] = 1 where j is the first of its key and the cell has no slot yet;
// k_old = the slot count before the append.
__global__ void append_mark_kernel(const uint32_t *__restrict__ new_keys, int k, const int32_t *__restrict__ slot_of,
                                   const GridMeta *__restrict__ meta, int *__restrict__ fresh,
                                   int *__restrict__ k_old) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) *k_old = meta->occupied;
    if (j >= k) return;
    const uint32_t key = new_keys[j];
    const bool first = j == 0 || new_keys[j - 1] != key;
    fresh[j] = (first && slot_of[key] < 0) ? 1 : 0;
}

// Pass 2 (fresh[] exclusively scanned, *n_fresh its total): every touched
// cell, one thread per first key, is recomputed from all its points in the
// sorted order (the same arithmetic as the build, so the records equal a
// full build's); new cells take slots k_old, k_old + 1, ... in key order.
__global__ void append_cells_kernel(const float4 *__restrict__ map, const uint32_t *__restrict__ new_keys, int k,
                                    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ order, int n,
                                    const int *__restrict__ fresh, const int *__restrict__ n_fresh,
                                    const int *__restrict__ k_old, int compat, int min_points, double eig_ratio,
                                    GridMeta *__restrict__ meta, GridBuffers buf) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j == 0) meta->occupied = *k_old + *n_fresh;
    if (j >= k) return;
    const uint32_t key = new_keys[j];
    if (j > 0 && new_keys[j - 1] == key) return;
    const int old_slot = buf.slot_of[key];
    const int s = old_slot >= 0 ? old_slot : *k_old + fresh[j];
    int lo = 0, hi = n;  // first key >= key
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) < key) lo = mid + 1; else hi = mid;
    }
    const int first = lo;
    hi = n;  // first key > key
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(keys + mid) <= key) lo = mid + 1; else hi = mid;
    }
    if (compat)
        compat_cell(map, order, first, lo, (double)meta->G, s, key, buf);
    else
        corrected_cell(map, order, first, lo, min_points, eig_ratio, s, key, buf);
}

// ---------------------------------------------------------------------------
// Probe-window table (see grid_build.h).
struct WinGeom {
    int dim[3];
    int wd[3];  // dim + 2
    int W;
};

// Calls f(index entry, 9 dz + 3 dy + dx) for the usable voxels of window w in
// the reference's probe order.
template <class F>
__device__ __forceinline__ void visit_window(const int32_t *__restrict__ index, const WinGeom &g, int w, F f) {
    const int bx = w % g.wd[0] - 2;
    const int t = w / g.wd[0];
    const int by = t % g.wd[1] - 2;
    const int bz = t / g.wd[1] - 2;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz) {
        const int z = bz + dz;
        if (z < 0 || z >= g.dim[2]) continue;
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
            const int y = by + dy;
            if (y < 0 || y >= g.dim[1]) continue;
            const int row = g.dim[0] * (y + g.dim[1] * z);
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int x = bx + dx;
                if (x < 0 || x >= g.dim[0]) continue;
                const int v = __ldg(index + row + x);
                if (v >= 0) f(v, 9 * dz + 3 * dy + dx);
            }
        }
    }
}

__global__ void window_count_kernel(const int32_t *__restrict__ index, WinGeom g, int *__restrict__ ctot) {
    const int w = blockIdx.x * kThreads + threadIdx.x;
    int c = 0;
    if (w < g.W) visit_window(index, g, w, [&](int, int) { ++c; });
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int s[kWarps];
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int k = 0; k < kWarps; ++k) t += s[k];
        ctot[blockIdx.x] = t;
    }
}

// ctot holds the exclusive block offsets here.
__global__ void window_fill_kernel(const int32_t *__restrict__ index, const float4 *__restrict__ vox32, WinGeom g,
                                   const int *__restrict__ ctot, int32_t *__restrict__ off, float4 *__restrict__ ent) {
    const int w = blockIdx.x * kThreads + threadIdx.x;
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    int c = 0;
    if (w < g.W) visit_window(index, g, w, [&](int, int) { ++c; });
    int incl = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    __shared__ int s[kWarps];
    if (lane == 31) s[wp] = incl;
    __syncthreads();
    int pos = ctot[blockIdx.x] + incl - c;
    for (int k = 0; k < wp; ++k) pos += s[k];
    if (w >= g.W) return;
    off[w] = pos;
    if (w == g.W - 1) off[g.W] = pos + c;
    visit_window(index, g, w, [&](int v, int o) {
        const int slot = v & kSlotMask;
        const float4 h = __ldg(vox32 + 3 * (size_t)slot);
        const unsigned code = ((unsigned)slot << 6) | ((v & kSlotFlag) ? 32u : 0u) | (unsigned)o;
        ent[pos++] = make_float4(h.x, h.y, h.z, __uint_as_float(code));
    });
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace

// ---------------------------------------------------------------------------
size_t grid_scratch_bytes(int m) {
    return kBboxBytes + sort_scratch_bytes(m) + 4096;  // bbox partials and counters, sort buffers
}

int grid_bbox(const float4 *d_map, int m, float res, GridMeta *d_meta, void *scratch, cudaStream_t st) {
    char *p = (char *)scratch;
    float *part = (float *)p;
    int *flags = (int *)(p + kBboxFlagsOffset);  // zeroed by grid_scratch_init, left at zero
    int nblk = div_up(m, kThreads);
    if (nblk > 1024) nblk = 1024;
    bbox_kernel<<<nblk, kThreads, 0, st>>>(d_map, m, part, flags, res, d_meta);
    return (int)cudaGetLastError();
}

int grid_scratch_init(void *scratch, cudaStream_t st) {
    int *flags = (int *)((char *)scratch + kBboxFlagsOffset);
    return (int)cudaMemsetAsync(flags, 0, 2 * sizeof(int), st);
}

int64_t window_count(const GridMeta &g) {
    return (int64_t)(g.dim[0] + 2) * (int64_t)(g.dim[1] + 2) * (int64_t)(g.dim[2] + 2);
}

int grid_windows(const GridMeta &meta_host, const int32_t *index, const float4 *vox32, WindowBuffers wb,
                 cudaStream_t st, int *launches) {
    WinGeom g;
    for (int e = 0; e < 3; ++e) {
        g.dim[e] = meta_host.dim[e];
        g.wd[e] = meta_host.dim[e] + 2;
    }
    g.W = (int)window_count(meta_host);
    const int nb = div_up(g.W, kThreads);
    window_count_kernel<<<nb, kThreads, 0, st>>>(index, g, wb.ctot);
    scan_single_block_kernel<<<1, 1024, 0, st>>>(wb.ctot, nb, nullptr);
    window_fill_kernel<<<nb, kThreads, 0, st>>>(index, vox32, g, wb.ctot, wb.off, wb.ent);
    if (launches) *launches += 3;
    return (int)cudaGetLastError();
}

int radix_sort_pairs(SortBuffers &b, int n, int bits, cudaStream_t st) {
    const int nblk = div_up(n, kSortTile);
    int nl = 0;
    // digit width: passes = ceil(bits / 8), width = ceil(bits / passes).  (Wider
    // digits save a pass but make the one-block histogram scan longer than the
    // pass: 9-bit digits over 196 blocks were slower on a 400k-point map.)
    int passes = (bits + 7) / 8;
    int width = (bits + passes - 1) / passes;  // <= 8 <= log2(kMaxDigits)
    int shift = 0;
    for (int ps = 0; ps < passes; ++ps) {
        int w = width;
        if (shift + w > bits) w = bits - shift;
        size_t smem_up = sizeof(int) << w;
        size_t smem_dn = sizeof(int) * kWarps << w;
        radix_upsweep_kernel<<<nblk, kThreads, smem_up, st>>>(b.k0, n, shift, w, b.hist);
        nl += scan_exclusive(b.hist, nblk << w, nullptr, b.part, st);
        radix_downsweep_kernel<<<nblk, kThreads, smem_dn, st>>>(b.k0, b.v0, b.k1, b.v1, n, shift, w, b.hist);
        nl += 2;
        uint32_t *t = b.k0; b.k0 = b.k1; b.k1 = t;
        t = b.v0; b.v0 = b.v1; b.v1 = t;
        shift += w;
    }
    return nl;
}

int segment_sorted(const uint32_t *keys, int n, int *segc, int *nseg, int *part, int32_t *seg_start,
                   uint32_t *seg_key, cudaStream_t st) {
    const int nblk = div_up(n, kSortTile);
    seg_count_kernel<<<nblk, kThreads, 0, st>>>(keys, n, segc);
    int nl = scan_exclusive(segc, nblk, nseg, part, st);
    seg_write_kernel<<<nblk, kThreads, 0, st>>>(keys, n, segc, seg_start, seg_key);
    return nl + 2;
}

int sort_segments(SortBuffers &b, int n, int bits, int32_t *seg_start, uint32_t *seg_key, cudaStream_t st) {
    int nl = radix_sort_pairs(b, n, bits, st);
    return nl + segment_sorted(b.k0, n, b.segc, b.nseg, b.part, seg_start, seg_key, st);
}

size_t sort_scratch_bytes(int n) {
    const size_t nblk = (size_t)div_up(n, kSortTile);
    return 4 * sizeof(uint32_t) * (size_t)n + sizeof(int) * kMaxDigits * nblk + sizeof(int) * (nblk + 1) +
           sizeof(int) * scan_part_ints((size_t)kMaxDigits * nblk) + 8 * 256;
}

SortBuffers sort_buffers(void *scratch, int n) {
    const size_t nblk = (size_t)div_up(n, kSortTile);
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    SortBuffers b;
    b.k0 = (uint32_t *)take(sizeof(uint32_t) * (size_t)n);
    b.v0 = (uint32_t *)take(sizeof(uint32_t) * (size_t)n);
    b.k1 = (uint32_t *)take(sizeof(uint32_t) * (size_t)n);
    b.v1 = (uint32_t *)take(sizeof(uint32_t) * (size_t)n);
    b.hist = (int *)take(sizeof(int) * (size_t)kMaxDigits * nblk);
    b.segc = (int *)take(sizeof(int) * (nblk + 1));
    b.nseg = (int *)take(sizeof(int));
    b.part = (int *)take(sizeof(int) * scan_part_ints((size_t)kMaxDigits * nblk));
    return b;
}

// Key bits of the dense cell ids.
int key_bits(const GridMeta &meta_host) {
    int bits = 1;
    while (bits < 31 && (1LL << bits) < meta_host.G) ++bits;
    return bits;
}

// Per-voxel records from the sorted order (one launch).
int grid_finalize(const float4 *d_map, const uint32_t *order, int m, const int *nseg, GridMeta *d_meta,
                  const NdtGridOptions &opt, GridBuffers buf, cudaStream_t st) {
    // at most m segments: launch for m, kernels read the true count
    if (opt.compat) {
        cell_finalize_compat_kernel<<<div_up(m, 128), 128, 0, st>>>(d_map, order, buf.seg_start, buf.seg_cell, nseg,
                                                                    m, d_meta, buf);
    } else {
        cell_finalize_corrected_kernel<<<div_up(m, 128), 128, 0, st>>>(d_map, order, buf.seg_start, buf.seg_cell,
                                                                       nseg, m, opt.min_points, opt.eigen_ratio,
                                                                       d_meta, buf);
    }
    return 1;
}

int grid_build(const float4 *d_map, int m, const GridMeta &meta_host, GridMeta *d_meta, const NdtGridOptions &opt,
               GridBuffers buf, void *scratch, cudaStream_t st, int *launches, SortedMap *sorted) {
    SortBuffers sb = sort_buffers((char *)scratch + kBboxBytes, m);  // after the bounding-box region
    int nl = 0;

    cudaMemsetAsync(buf.index, 0xff, sizeof(int32_t) * (size_t)meta_host.G, st);
    cudaMemsetAsync(buf.slot_of, 0xff, sizeof(int32_t) * (size_t)meta_host.G, st);
    cell_key_kernel<<<div_up(m, kThreads), kThreads, 0, st>>>(d_map, m, d_meta, sb.k0, sb.v0);
    ++nl;
    nl += sort_segments(sb, m, key_bits(meta_host), buf.seg_start, buf.seg_cell, st);
    nl += grid_finalize(d_map, sb.v0, m, sb.nseg, d_meta, opt, buf, st);
    if (sorted) {
        sorted->keys = sb.k0;
        sorted->order = sb.v0;
    }
    if (launches) *launches += nl;
    return (int)cudaGetLastError();
}

size_t append_scratch_bytes(int k) {
    return sort_scratch_bytes(k) + sizeof(int) * ((size_t)k + 1) + sizeof(int) * scan_part_ints((size_t)k) + 8 * 256;
}

int grid_append(const float4 *d_map, int m_old, int k, const GridMeta &meta_host, GridMeta *d_meta,
                const NdtGridOptions &opt, GridBuffers buf, SortedMap old_sorted, uint32_t *keys_out,
                uint32_t *order_out, void *scratch, cudaStream_t st, int *launches) {
    const int n = m_old + k;
    char *p = (char *)scratch;
    auto take = [&](size_t bytes) {
        char *r = p;
        p += (bytes + 255) & ~(size_t)255;
        return (void *)r;
    };
    SortBuffers sb = sort_buffers(take(sort_scratch_bytes(k)), k);
    int *fresh = (int *)take(sizeof(int) * (size_t)k);
    int *small = (int *)take(2 * sizeof(int));  // n_fresh, k_old
    int *part = (int *)take(sizeof(int) * scan_part_ints((size_t)k));
    int nl = 0;
    // the new points' keys (point indices m_old ...), stably sorted
    cell_key_kernel<<<div_up(k, kThreads), kThreads, 0, st>>>(d_map + m_old, k, d_meta, sb.k0, sb.v0, m_old);
    ++nl;
    nl += radix_sort_pairs(sb, k, key_bits(meta_host), st);
    // merged with the map's sorted pairs: the stable sort of all n points
    merge_kernel<<<div_up(n, kThreads), kThreads, 0, st>>>(old_sorted.keys, old_sorted.order, m_old, sb.k0, sb.v0,
                                                           k, keys_out, order_out);
    // the touched cells: new slots in key order, records from all their points
    append_mark_kernel<<<div_up(k, kThreads), kThreads, 0, st>>>(sb.k0, k, buf.slot_of, d_meta, fresh, small + 1);
    nl += 2;
    nl += scan_exclusive(fresh, k, small, part, st);
    append_cells_kernel<<<div_up(k, 128), 128, 0, st>>>(d_map, sb.k0, k, keys_out, order_out, n, fresh, small, small + 1,
                                                        opt.compat, opt.min_points, opt.eigen_ratio, d_meta, buf);
    ++nl;
    if (launches) *launches += nl;
    return (int)cudaGetLastError();
}

}  // namespace ndt
