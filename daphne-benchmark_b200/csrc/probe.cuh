// Shared device code of the derivative pass: the reference's neighbour
// search (voxelRadiusSearch, src/CPU/ndt_mapping/kernel.cpp:246-286) per
// point, collecting the pair list that the pair evaluation consumes, and the
// block-reduction helpers.
//
// Every operation whose rounding decides which (point, voxel) pairs the
// reference accepts is written with explicit round-to-nearest intrinsics
// (__fadd_rn, __fsub_rn, __fmul_rn, __fdiv_rn), so this code gives the
// reference's pairs whether or not the including file is compiled with
// floating-point contraction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "derivatives.h"
#include "ndt_math.cuh"

namespace ndt {

constexpr int kAcc = 37;        // FP32 sums: score, g[6], S[21], R[9]
constexpr int kTerms = 23;      // per-point terms (see below)
constexpr int kList = 27 * 32;  // per-warp pair list: all 27 probes of all 32 lanes
constexpr unsigned kFull = 0xffffffffu;

// Per-point terms (point Jacobian columns 3-5 and point Hessian blocks), FP32.
// Index: 0 J13, 1 J23, 2 J04, 3 J14, 4 J24, 5 J05, 6 J15, 7 J25,
//        8 a1, 9 a2, 10 b1, 11 b2, 12 c1, 13 c2, 14-16 d, 17-19 e, 20-22 f.

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ double4 ldg_d4(const double4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    double2 a = __ldg(q), b = __ldg(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__device__ __forceinline__ float dot3f(float a0, float a1, float a2, const float *b) {
    return fmaf(a0, b[0], fmaf(a1, b[1], a2 * b[2]));
}

// transformPointCloud (kernel.cpp:397-400): T[r][0] x + T[r][1] y + T[r][2] z
// + T[r][3], float, left to right, every operation rounded.
__device__ __forceinline__ float transform_row(const float *T, float x, float y, float z) {
    return __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(T[0], x), __fmul_rn(T[1], y)), __fmul_rn(T[2], z)), T[3]);
}

// ---------------------------------------------------------------------------
// Probe geometry of one axis: the reference's float loop
//   for (float v = p - r; v <= p + rf; v += res)           (kernel.cpp:256-258)
// The start (float)((double)p - r) equals the float subtraction p - r: the
// double difference of two floats is exact (for |p| < 2^28 r), so both round
// the exact difference once.  The loop gives 3 coordinates for any finite |p|
// below ~1e6 m (trip count n; n = 4 only for larger or infinite
// coordinates, handled by the generic path).  For each coordinate: inside
// the bbox (kernel.cpp:261-269) and its cell index (linearizeCoord, :239-241).
struct Axis {
    float c0, c1, c2;
    int i0, i1, i2;
    unsigned in;  // bit k: coordinate k is active and inside the bbox
    int n;
};

__device__ __forceinline__ int cell_component(float v, float minv, float res, float inv_res) {
    const float d = __fsub_rn(v, minv);
    return inv_res > 0.0f ? (int)__fmul_rn(d, inv_res) : (int)__fdiv_rn(d, res);
}

__device__ __forceinline__ Axis make_axis(float p, float minv, float maxv, float res, float inv_res, float rf,
                                          bool valid) {
    Axis a;
    a.c0 = __fsub_rn(p, res);
    a.c1 = __fadd_rn(a.c0, res);
    a.c2 = __fadd_rn(a.c1, res);
    const float c3 = __fadd_rn(a.c2, res);
    const float lim = __fadd_rn(p, rf);
    // the coordinates increase, so the trip count is the number that pass
    int n = 0;
    if (valid) n = (a.c0 <= lim) + (a.c1 <= lim) + (a.c2 <= lim) + (c3 <= lim);
    a.n = n;
    unsigned in = 0;
    if (n > 0 && !(a.c0 < minv || a.c0 > maxv)) in |= 1u;
    if (n > 1 && !(a.c1 < minv || a.c1 > maxv)) in |= 2u;
    if (n > 2 && !(a.c2 < minv || a.c2 > maxv)) in |= 4u;
    a.in = in;
    a.i0 = (in & 1u) ? cell_component(a.c0, minv, res, inv_res) : 0;
    a.i1 = (in & 2u) ? cell_component(a.c1, minv, res, inv_res) : 0;
    a.i2 = (in & 4u) ? cell_component(a.c2, minv, res, inv_res) : 0;
    return a;
}

__device__ __forceinline__ int axis_i(const Axis &a, int k) { return k == 0 ? a.i0 : (k == 1 ? a.i1 : a.i2); }

// Margin of the FP32 pre-test of the radius check for a point p: the FP32
// difference hi - p and the reference's float(mean - p) (FP64 mean) differ by
// at most E = 2^-23 (|m| + |dx|) per axis, and a candidate mean lies within
// 3r of p, so |m| <= |p| + 3r; the squared distances then differ by at most
// sum_axes 2 E (|dx| + E) <= 20 r E + 3 E^2 with E = 2^-23 (|p|_1 + 14 r + 1).
__device__ __forceinline__ float radius_margin(float px, float py, float pz, float res) {
    const float E = 1.2e-7f * (fabsf(px) + fabsf(py) + fabsf(pz) + 14.0f * res + 1.0f);
    return 20.0f * res * E + 3.0f * E * E;
}

// The reference's distance test float(sqrt(dx^2 + dy^2 + dz^2)) < r,
// dx = float(mean - p) on the FP64 mean (kernel.cpp:273-278), decided as
// s <= s_max (the largest float whose correctly rounded root is below r):
// first with the FP32 mean and the margin tol, then, inside the margin,
// exactly on the FP64 mean.
__device__ __forceinline__ bool accept(const GridDev &grid, int slot, float4 hi, float px, float py, float pz,
                                       float tol) {
    const float s_max = grid.s_max;
    const float fx = hi.x - px, fy = hi.y - py, fz = hi.z - pz;
    const float sf = fmaf(fx, fx, fmaf(fy, fy, fz * fz));
    if (sf < s_max - tol) return true;
    if (sf > s_max + tol) return false;
    const double4 m = ldg_d4(grid.mean + slot);
    const float dx = (float)(m.x - (double)px);
    const float dy = (float)(m.y - (double)py);
    const float dz = (float)(m.z - (double)pz);
    const float s = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    return s <= s_max;
}

__device__ __forceinline__ unsigned pair_code(int v, int lane) {
    return ((unsigned)(v & kSlotMask) << 6) | ((v & kSlotFlag) ? 32u : 0u) | (unsigned)lane;
}

// The probe-window table (grid_build.h) holds, for a window base cell b, the
// usable voxels of cells [b, b + 2]^3 in probe order.  A lane's window is the
// one whose base is the cell of its first probe coordinate on each axis; that
// covers the reference's probe cells when each axis's in-bbox coordinates fall
// in consecutive cells inside [0, dim).  An entry is one of the reference's
// probes when its cell offset has an in-bbox coordinate on all three axes.
__device__ __forceinline__ int window_base(const Axis &a, int dim, bool &ok) {
    if (a.in == 0u) return 0;
    const int first = (a.in & 1u) ? 0 : ((a.in & 2u) ? 1 : 2);
    const int base = axis_i(a, first) - first;
#pragma unroll
    for (int k = 0; k < 3; ++k)
        if (((a.in >> k) & 1u) && (axis_i(a, k) != base + k || axis_i(a, k) >= dim)) ok = false;
    return base;
}

// Where collect_pairs puts the accepted pairs (code = slot << 6 | flag << 5 |
// lane): add() on the windows and dense paths, add_far() on the generic path.
// ListSink compacts the warp's pairs into one list (capacity 27 x 32, `n`
// entries); OwnSink keeps each lane's pairs in its own column, own[k][lane]
// for k < c (at most kOwn per lane).
struct ListSink {
    unsigned *list;
    int n;
    __device__ __forceinline__ void add(bool ok, unsigned code) {
        const unsigned bal = __ballot_sync(kFull, ok);
        if (ok) list[n + __popc(bal & lanemask_lt())] = code;
        n += __popc(bal);
    }
    __device__ __forceinline__ void add_far(bool ok, unsigned code) { add(ok, code); }
    __device__ __forceinline__ bool full() const { return n > kList - 32; }
};

struct OwnSink {
    unsigned (*own)[32];
    int c;
    __device__ __forceinline__ void add(bool ok, unsigned code) {
        if (ok) own[c++][threadIdx.x & 31] = code;
    }
    __device__ __forceinline__ void add_far(bool ok, unsigned code) { add(ok, code); }
    __device__ __forceinline__ bool full() const { return __any_sync(kFull, c >= kOwn); }
};

// The neighbour-search paths a caller compiles in (bit mask; the generic path
// is always there): kProbeWindows needs the probe-window table.
constexpr int kProbeWindows = 1;
constexpr int kProbeDenseIndex = 2;
constexpr int kProbeAll = kProbeWindows | kProbeDenseIndex;

// Collects the accepted (point, voxel) pairs of every lane's point into
// `sink`.  `resume` is 0 on the first call; it comes back -1 when the point's
// probes are done, or, on the generic path (trip counts up to 4: coordinates
// beyond ~1e6 m or inf), the probe position to continue from once the caller
// has emptied the sink.  Three paths, chosen per warp:
//   windows  the probe-window table (2 offsets + 1 record per occupied cell),
//            when the table exists and every lane's cells are consecutive;
//   dense    the 27 dense-index entries in 3 layers of 9 loads, skipping with
//            warp-uniform branches the layers and rows no lane has in bounds
//            or occupied, the distance tests of probes no lane occupies and
//            the appends of probes no lane accepted;
//   generic  one probe at a time, the reference's loop as written.
// The pairs are the reference's on every path; only their order differs.
// kPaths selects the compiled paths: without kProbeDenseIndex the warps the
// window path cannot take use the generic one; without kProbeWindows the
// table is not read.
template <class Sink, int kPaths = kProbeAll>
__device__ __forceinline__ void collect_pairs(const GridDev &grid, float px, float py, float pz, bool valid, Sink &sink,
                                              unsigned &n_probe, unsigned &n_occ, int &resume) {
    const int lane = threadIdx.x & 31;
    const GridMeta &g = grid.meta;
    const float res = g.res, inv_res = grid.inv_res, rf = grid.radius_final;
    const Axis ax = make_axis(px, g.minv[0], g.maxv[0], res, inv_res, rf, valid);
    const Axis ay = make_axis(py, g.minv[1], g.maxv[1], res, inv_res, rf, valid);
    const Axis az = make_axis(pz, g.minv[2], g.maxv[2], res, inv_res, rf, valid);
    const bool any_in = (ax.in != 0u) && (ay.in != 0u) && (az.in != 0u);
    if (!__any_sync(kFull, any_in)) {
        resume = -1;
        return;
    }
    const int mx = __reduce_max_sync(kFull, ax.n), my = __reduce_max_sync(kFull, ay.n),
              mz = __reduce_max_sync(kFull, az.n);
    const float tol = radius_margin(px, py, pz, res);
    const bool small = mx <= 3 && my <= 3 && mz <= 3;
    if ((kPaths & kProbeWindows) && small && grid.win_off) {
        bool ok = true;
        const int bx = window_base(ax, g.dim[0], ok);
        const int by = window_base(ay, g.dim[1], ok);
        const int bz = window_base(az, g.dim[2], ok);
        if (__all_sync(kFull, ok || !any_in)) {
            unsigned allowed = 0;
            int beg = 0, cnt = 0;
            if (any_in) {
#pragma unroll
                for (int dz = 0; dz < 3; ++dz)
#pragma unroll
                    for (int dy = 0; dy < 3; ++dy)
                        if ((az.in >> dz) & (ay.in >> dy) & 1u) allowed |= ax.in << (9 * dz + 3 * dy);
                const int w = (bx + 2) + grid.win_dim[0] * ((by + 2) + grid.win_dim[1] * (bz + 2));
                beg = __ldg(grid.win_off + w);
                cnt = __ldg(grid.win_off + w + 1) - beg;
                n_probe += __popc(allowed);
            }
            const int maxc = __reduce_max_sync(kFull, cnt);
            for (int j = 0; j < maxc; j += 4) {
                float4 e[4];
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    e[u] = j + u < cnt ? __ldg(grid.win_ent + beg + j + u) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const unsigned code = __float_as_uint(e[u].w);
                    const bool occ = j + u < cnt && ((allowed >> (code & 31u)) & 1u);
                    n_occ += occ;
                    const bool ok2 = occ && accept(grid, (int)(code >> 6), e[u], px, py, pz, tol);
                    sink.add(ok2, (code & ~31u) | (unsigned)lane);
                }
            }
            resume = -1;
            return;
        }
    }
    if ((kPaths & kProbeDenseIndex) && small) {
#pragma unroll 1
        for (int a = 0; a < 3; ++a) {
            const bool za = any_in && ((az.in >> a) & 1u);
            if (!__any_sync(kFull, za)) continue;
            const int zbase = g.dim[1] * axis_i(az, a);
            int v[9];
            unsigned on_mask = 0, occ = 0;
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const bool yb = za && ((ay.in >> b) & 1u);
                const int base = g.dim[0] * (axis_i(ay, b) + zbase);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const bool on = yb && ((ax.in >> c) & 1u);
                    v[3 * b + c] = on ? __ldg(grid.index + (axis_i(ax, c) + base)) : -1;
                    on_mask |= (unsigned)on << (3 * b + c);
                }
            }
#pragma unroll
            for (int k = 0; k < 9; ++k) occ |= (unsigned)(v[k] >= 0) << k;
            n_probe += __popc(on_mask);
            n_occ += __popc(occ);
            if (!__any_sync(kFull, occ != 0u)) continue;
            // one row of 3 cells at a time: means, distance tests, appends
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const unsigned row = (occ >> (3 * b)) & 7u;
                if (!__any_sync(kFull, row != 0u)) continue;
                float4 hi[3];
#pragma unroll
                for (int c = 0; c < 3; ++c)
                    if ((row >> c) & 1u) hi[c] = __ldg(grid.vox32 + 3 * (v[3 * b + c] & kSlotMask));
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (!__any_sync(kFull, (row >> c) & 1u)) continue;
                    const bool ok = ((row >> c) & 1u) && accept(grid, v[3 * b + c] & kSlotMask, hi[c], px, py, pz, tol);
                    if (__any_sync(kFull, ok)) sink.add(ok, pair_code(v[3 * b + c], lane));
                }
            }
        }
        resume = -1;
        return;
    }
    // generic: position pos = (a * my + b) * mx + c, z outer, x inner
    const int total = mz * my * mx;
    for (int pos = resume; pos < total; ++pos) {
        if (sink.full()) {
            resume = pos;
            return;
        }
        const int c = pos % mx, b = (pos / mx) % my, a = pos / (mx * my);
        float xc = ax.c0, yc = ay.c0, zc = az.c0;
        for (int k = 0; k < c; ++k) xc = __fadd_rn(xc, res);
        for (int k = 0; k < b; ++k) yc = __fadd_rn(yc, res);
        for (int k = 0; k < a; ++k) zc = __fadd_rn(zc, res);
        const bool act = a < az.n && b < ay.n && c < ax.n;
        const bool inb = act && !((xc < g.minv[0]) || (xc > g.maxv[0]) || (yc < g.minv[1]) || (yc > g.maxv[1]) ||
                                  (zc < g.minv[2]) || (zc > g.maxv[2]));
        int v = -1;
        if (inb) {
            v = __ldg(grid.index + (cell_component(xc, g.minv[0], res, inv_res) +
                                    g.dim[0] * (cell_component(yc, g.minv[1], res, inv_res) +
                                                g.dim[1] * cell_component(zc, g.minv[2], res, inv_res))));
            ++n_probe;
        }
        bool ok = false;
        if (v >= 0) {
            ++n_occ;
            ok = accept(grid, v & kSlotMask, __ldg(grid.vox32 + 3 * (v & kSlotMask)), px, py, pz, tol);
        }
        sink.add_far(ok, pair_code(v, lane));
    }
    resume = -1;
}

// ---------------------------------------------------------------------------
// Partial layout helpers.
__device__ __forceinline__ int sidx(int i, int j) {  // upper-triangle index, i <= j
    return i * 6 - (i * (i - 1)) / 2 + (j - i);
}

// Tile partial layout: [0] score, [1..6] g, [7..42] H row major, [43] pairs.
// H_ij = S_ij + kR R_ij from the FP32 sums (see derivatives_f32.cu).
__device__ __forceinline__ double h_entry(const double *tot, int i, int j, double kR, bool compat) {
    double v = tot[7 + (i <= j ? sidx(i, j) : sidx(j, i))];
    if (i >= 3 && j >= 3) {
        int a = i - 3, b = j - 3;
        double r = compat ? tot[28 + 3 * a + b] : tot[28 + 3 * (a < b ? a : b) + (a < b ? b : a)];
        v = fma(kR, r, v);  // explicit, so the result does not depend on contraction choices
    }
    return v;
}

}  // namespace ndt
