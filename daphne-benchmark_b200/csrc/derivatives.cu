// The derivative pass: score, gradient and Hessian of the NDT objective for a
// batch of alignments (computeDerivatives / computeHessian,
// src/CPU/ndt_mapping/kernel.cpp:562-705, with voxelRadiusSearch :246-286,
// computePointDerivatives :495-560 and updateDerivatives :438-493 fused in).
//
// Work decomposition: the tile list holds ceil(n_a / TILE) tiles of TILE
// consecutive points per alignment.  Block b of the persistent grid owns the
// contiguous tile range [b * per, (b + 1) * per), so the tiles of one
// alignment are met in a row; each lane keeps its FP32 sums of the current
// alignment in shared memory and the block reduces them once per alignment
// run (TwoSum-compensated across lanes and warps), writing the run's FP64
// partial to the slot of its first tile (the run's other slots get zeros).
//
// Per point (one thread):
//   1. transform by the alignment's float 3x4 (transformPointCloud :385-404,
//      same float operation order);
//   2. the reference's 27 float probe points p + {-r, 0, r}^3: coordinates by
//      the reference's float recurrence, its bounds test and cell
//      linearisation (division by r replaced by the exactly equal product
//      with 1/r when r is a power of two), one z-layer of 9 probes at a time
//      with all their loads in flight;
//   3. the reference's test float(sqrt(dx^2 + dy^2 + dz^2)) < r with
//      dx = float(mean - x) on the FP64 mean, decided without the square
//      root as s <= s_max (s_max = the largest float whose correctly rounded
//      square root is below r), first on the FP32 copy of the mean with a
//      proven error margin and, only inside that margin, exactly on the FP64
//      mean -- so the accepted (point, voxel) pairs are the reference's;
//   4. accepted pairs are compacted per warp in shared memory (ballot + popc)
//      and evaluated one per lane, so per-pair work is balanced across lanes.
// Per pair (FP32 path): x' from the (hi, lo) float split of the FP64 mean,
// q = C x', xCx, e = exp(-d2 xCx / 2), the validity test of :456, gradient
// a_i = x'^T C J_i and the Hessian split as
//   H_ij = S_ij + k R_ij,  S_ij = w (-d2 a_i a_j + J_j^T C J_i)   (i <= j)
//   compat:    R_ij = w a_i b_ij, k = -d2  (the reference's :486-488 form)
//   corrected: R_ij = w b_ij,     k = 1    (Magnusson eq. 6.13)
// with b_ij = x'^T C H_ij (nonzero for i, j >= 3 only).  Voxels flagged by the
// grid build (inverse-covariance entries non-finite or beyond 1e30) are
// evaluated in FP64 so that infinities and NaNs propagate as in the reference.
//
// The FP64 variant (precision = 1) evaluates every pair with the reference's
// literal FP64 expressions and accumulates in FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include "derivatives.h"
#include "ndt_math.cuh"

namespace ndt {

namespace {

constexpr int kAcc = 37;      // score, g[6], S[21], R[9]
constexpr int kTerms = 23;    // per-point terms (see below)
constexpr int kList = 27 * 32;  // per-warp pair list: all 27 probes of all 32 lanes
constexpr unsigned kFull = 0xffffffffu;

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

// Per-point terms (point Jacobian columns 3-5 and point Hessian blocks), FP32.
// Index: 0 J13, 1 J23, 2 J04, 3 J14, 4 J24, 5 J05, 6 J15, 7 J25,
//        8 a1, 9 a2, 10 b1, 11 b2, 12 c1, 13 c2, 14-16 d, 17-19 e, 20-22 f.

// ---------------------------------------------------------------------------
// Probe geometry of one axis: the reference's float loop
//   for (float v = p - r; v <= p + rf; v += res)           (kernel.cpp:256-258)
// gives up to 3 coordinates for any finite |p| below ~1e6 m (trip count n;
// n = 4 only for larger or infinite coordinates, handled by the generic
// path).  For each coordinate: inside the bbox (kernel.cpp:261-269) and its
// cell index (linearizeCoord, :239-241).
struct Axis {
    float c0, c1, c2;
    int i0, i1, i2;
    unsigned in;  // bit k: coordinate k is active and inside the bbox
    int n;
};

__device__ __forceinline__ int cell_component(float v, float minv, float res, float inv_res) {
    return inv_res > 0.0f ? (int)((v - minv) * inv_res) : (int)((v - minv) / res);
}

__device__ __forceinline__ Axis make_axis(float p, float minv, float maxv, float res, float inv_res, bool valid) {
    const double radius = (double)res;
    const float rf = (float)(radius + (double)0.001f);  // radiusFinal, kernel.cpp:254
    Axis a;
    a.c0 = (float)((double)p - radius);
    a.c1 = a.c0 + res;
    a.c2 = a.c1 + res;
    const float lim = p + rf;
    int n = 0;
    if (valid) {
        float v = a.c0;
        while (n < 4 && v <= lim) {
            ++n;
            v = v + res;
        }
    }
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

__device__ __forceinline__ float axis_c(const Axis &a, int k) { return k == 0 ? a.c0 : (k == 1 ? a.c1 : a.c2); }
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

// The reference's distance test for one occupied probe, decided as
// s <= s_max (see the file comment): first with the FP32 mean and the margin
// tol, then, inside the margin, exactly on the FP64 mean.
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
    const float s = dx * dx + dy * dy + dz * dz;
    return s <= s_max;
}

// Probe every lane's point in the reference's order (z outer, x inner;
// voxelRadiusSearch, kernel.cpp:256-284) and collect the accepted pairs in
// `list` (capacity 27 x 32); `consume(n)` then evaluates list[0, n) (the
// generic path calls it whenever the list could overflow).
// List code = slot << 6 | flag << 5 | lane.
template <class Consume>
__device__ __forceinline__ void probe_point(const GridDev &grid, float px, float py, float pz, bool valid,
                                            unsigned *list, unsigned &n_probe, unsigned &n_occ, Consume consume) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const GridMeta &g = grid.meta;
    const float res = g.res, inv_res = grid.inv_res;
    const Axis ax = make_axis(px, g.minv[0], g.maxv[0], res, inv_res, valid);
    const Axis ay = make_axis(py, g.minv[1], g.maxv[1], res, inv_res, valid);
    const Axis az = make_axis(pz, g.minv[2], g.maxv[2], res, inv_res, valid);
    const int mx = __reduce_max_sync(kFull, ax.n), my = __reduce_max_sync(kFull, ay.n),
              mz = __reduce_max_sync(kFull, az.n);
    const float tol = radius_margin(px, py, pz, res);
    int n = 0;
    if (mx <= 3 && my <= 3 && mz <= 3) {
        // no lane has an in-bounds probe: nothing to do
        if (!__any_sync(kFull, (ax.in != 0u) && (ay.in != 0u) && (az.in != 0u))) return;
#pragma unroll 1
        for (int a = 0; a < mz; ++a) {
            const bool za = (az.in >> a) & 1u;
            if (!__any_sync(kFull, za && ax.in != 0u && ay.in != 0u)) continue;
            const int zbase = g.dim[1] * axis_i(az, a);
            int slot[9];
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const bool yb = za && ((ay.in >> b) & 1u);
                const int base = g.dim[0] * (axis_i(ay, b) + zbase);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const bool on = yb && ((ax.in >> c) & 1u);
                    slot[3 * b + c] = on ? __ldg(grid.index + (axis_i(ax, c) + base)) : -2;
                }
            }
            float4 hi[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                n_probe += slot[k] != -2;
                if (slot[k] >= 0) hi[k] = __ldg(grid.mean_hi + (slot[k] & kSlotMask));
            }
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int v = slot[k];
                bool acc = false;
                if (v >= 0) {
                    ++n_occ;
                    acc = accept(grid, v & kSlotMask, hi[k], px, py, pz, tol);
                }
                const unsigned b = __ballot_sync(kFull, acc);
                if (acc) list[n + __popc(b & lt)] = ((unsigned)(v & kSlotMask) << 6) | ((v & kSlotFlag) ? 32u : 0u) | lane;
                n += __popc(b);
            }
        }
        __syncwarp();
        consume(n);
        __syncwarp();
        return;
    }
    // generic path: trip counts up to 4 (coordinates beyond ~1e6 m or inf)
    float zc = (float)((double)pz - (double)res);
    for (int a = 0; a < mz; ++a, zc = zc + res) {
        float yc = (float)((double)py - (double)res);
        for (int b = 0; b < my; ++b, yc = yc + res) {
            float xc = (float)((double)px - (double)res);
            for (int c = 0; c < mx; ++c, xc = xc + res) {
                const bool act = a < az.n && b < ay.n && c < ax.n;
                const bool inb = act && !((xc < g.minv[0]) || (xc > g.maxv[0]) || (yc < g.minv[1]) ||
                                          (yc > g.maxv[1]) || (zc < g.minv[2]) || (zc > g.maxv[2]));
                int v = -1;
                if (inb) {
                    v = __ldg(grid.index + (cell_component(xc, g.minv[0], res, inv_res) +
                                            g.dim[0] * (cell_component(yc, g.minv[1], res, inv_res) +
                                                        g.dim[1] * cell_component(zc, g.minv[2], res, inv_res))));
                    ++n_probe;
                }
                bool acc = false;
                if (v >= 0) {
                    ++n_occ;
                    acc = accept(grid, v & kSlotMask, __ldg(grid.mean_hi + (v & kSlotMask)), px, py, pz, tol);
                }
                if (n > kList - 32) {
                    __syncwarp();
                    consume(n);
                    __syncwarp();
                    n = 0;
                }
                const unsigned bb = __ballot_sync(kFull, acc);
                if (acc) list[n + __popc(bb & lt)] = ((unsigned)(v & kSlotMask) << 6) | ((v & kSlotFlag) ? 32u : 0u) | lane;
                n += __popc(bb);
            }
        }
    }
    __syncwarp();
    consume(n);
    __syncwarp();
}

// ---------------------------------------------------------------------------
// FP32 pair evaluation.
struct AccF {
    float v[kAcc];
};

__device__ __forceinline__ int sidx(int i, int j) {  // upper-triangle index, i <= j
    return i * 6 - (i * (i - 1)) / 2 + (j - i);
}

__device__ __forceinline__ void pair_fp32(AccF &A, const float (*terms)[32], int owner, float p0, float p1, float p2,
                                          float4 ca, float4 cb, float d1, float d2, bool hess, bool compat) {
    const float c00 = ca.x, c01 = ca.y, c02 = ca.z, c11 = ca.w, c12 = cb.x, c22 = cb.y;
    const float q0 = fmaf(c00, p0, fmaf(c01, p1, c02 * p2));
    const float q1 = fmaf(c01, p0, fmaf(c11, p1, c12 * p2));
    const float q2 = fmaf(c02, p0, fmaf(c12, p1, c22 * p2));
    const float xCx = fmaf(p0, q0, fmaf(p1, q1, p2 * q2));
    const float e = expf(-d2 * xCx * 0.5f);
    const float e2 = d2 * e;
    if (!(e2 <= 1.0f && e2 >= 0.0f)) return;  // kernel.cpp:456 (also rejects NaN)
    const float w = d1 * e2;
    A.v[0] += -d1 * e;
    // M_i = C J_i for i = 3, 4, 5
    const float J13 = terms[0][owner], J23 = terms[1][owner], J04 = terms[2][owner], J14 = terms[3][owner];
    const float J24 = terms[4][owner], J05 = terms[5][owner], J15 = terms[6][owner], J25 = terms[7][owner];
    const float M30 = fmaf(c01, J13, c02 * J23), M31 = fmaf(c11, J13, c12 * J23), M32 = fmaf(c12, J13, c22 * J23);
    const float M40 = fmaf(c00, J04, fmaf(c01, J14, c02 * J24));
    const float M41 = fmaf(c01, J04, fmaf(c11, J14, c12 * J24));
    const float M42 = fmaf(c02, J04, fmaf(c12, J14, c22 * J24));
    const float M50 = fmaf(c00, J05, fmaf(c01, J15, c02 * J25));
    const float M51 = fmaf(c01, J05, fmaf(c11, J15, c12 * J25));
    const float M52 = fmaf(c02, J05, fmaf(c12, J15, c22 * J25));
    float a[6];
    a[0] = q0;
    a[1] = q1;
    a[2] = q2;
    a[3] = fmaf(p0, M30, fmaf(p1, M31, p2 * M32));
    a[4] = fmaf(p0, M40, fmaf(p1, M41, p2 * M42));
    a[5] = fmaf(p0, M50, fmaf(p1, M51, p2 * M52));
    float u[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        u[i] = w * a[i];
        A.v[1 + i] += u[i];
    }
    if (!hess) return;
    // column vectors M_i (i < 3: columns of C)
    const float M[6][3] = {{c00, c01, c02}, {c01, c11, c12}, {c02, c12, c22},
                           {M30, M31, M32}, {M40, M41, M42}, {M50, M51, M52}};
    // J_j . M_i
    auto jm = [&](int j, int i) -> float {
        switch (j) {
            case 0: return M[i][0];
            case 1: return M[i][1];
            case 2: return M[i][2];
            case 3: return fmaf(J13, M[i][1], J23 * M[i][2]);
            case 4: return fmaf(J04, M[i][0], fmaf(J14, M[i][1], J24 * M[i][2]));
            default: return fmaf(J05, M[i][0], fmaf(J15, M[i][1], J25 * M[i][2]));
        }
    };
    const float nd2 = -d2;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float ui = nd2 * u[i];
#pragma unroll
        for (int j = i; j < 6; ++j) A.v[7 + sidx(i, j)] += fmaf(ui, a[j], w * jm(j, i));
    }
    // b_ij = q . H_ij, i, j in 3..5
#define T_(k) terms[k][owner]
    const float b33 = fmaf(q1, T_(8), q2 * T_(9));
    const float b34 = fmaf(q1, T_(10), q2 * T_(11));
    const float b35 = fmaf(q1, T_(12), q2 * T_(13));
    const float b44 = fmaf(q0, T_(14), fmaf(q1, T_(15), q2 * T_(16)));
    const float b45 = fmaf(q0, T_(17), fmaf(q1, T_(18), q2 * T_(19)));
    const float b55 = fmaf(q0, T_(20), fmaf(q1, T_(21), q2 * T_(22)));
#undef T_
    const float B[3][3] = {{b33, b34, b35}, {b34, b44, b45}, {b35, b45, b55}};
    if (compat) {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) A.v[28 + 3 * i + j] += u[3 + i] * B[i][j];
    } else {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = i; j < 3; ++j) A.v[28 + 3 * i + j] += w * B[i][j];
    }
}

// Flagged voxel in the FP32 kernel: the same decomposition in FP64 with the
// full (unsymmetrised) inverse covariance of the reference.  Contributions go
// to the alignment's FP64 side buffer (exc[44], same layout as a tile
// partial) with atomics; they are 0, inf or NaN in practice (a flagged
// covariance puts xCx far from 0), so their order does not matter.
__device__ void pair_fp64_flagged(double *exc, const float *t, float p0f, float p1f, float p2f, const double *C,
                                  double d1, double d2, bool hess, bool compat) {
    const double p[3] = {p0f, p1f, p2f};
    double xCx = C[0] * p[0] * p[0] + C[4] * p[1] * p[1] + C[8] * p[2] * p[2] + (C[1] + C[3]) * p[0] * p[1] +
                 (C[2] + C[6]) * p[0] * p[2] + (C[5] + C[7]) * p[1] * p[2];
    double e = exp(-d2 * (xCx) / 2);
    double sc = -d1 * e;
    e = d2 * e;
    if (e > 1 || e < 0 || e != e) return;
    double w = e * d1;
    double J[3][6] = {{1, 0, 0, 0, t[2], t[5]}, {0, 1, 0, t[0], t[3], t[6]}, {0, 0, 1, t[1], t[4], t[7]}};
    double Mv[6][3], a[6];
    for (int i = 0; i < 6; ++i) {
        for (int r = 0; r < 3; ++r) Mv[i][r] = C[3 * r] * J[0][i] + C[3 * r + 1] * J[1][i] + C[3 * r + 2] * J[2][i];
        a[i] = p[0] * Mv[i][0] + p[1] * Mv[i][1] + p[2] * Mv[i][2];
    }
    auto add = [&](int k, double v) {
        if (v != 0.0) atomicAdd(exc + k, v);
    };
    add(0, sc);
    for (int i = 0; i < 6; ++i) add(1 + i, w * a[i]);
    if (!hess) return;
    // q' = C^T x' (b_ij = x'^T C H_ij)
    double qt[3];
    for (int c = 0; c < 3; ++c) qt[c] = C[c] * p[0] + C[3 + c] * p[1] + C[6 + c] * p[2];
    const double hb[3][3][3] = {
        {{0, t[8], t[9]}, {0, t[10], t[11]}, {0, t[12], t[13]}},
        {{0, t[10], t[11]}, {t[14], t[15], t[16]}, {t[17], t[18], t[19]}},
        {{0, t[12], t[13]}, {t[17], t[18], t[19]}, {t[20], t[21], t[22]}}};
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) {
            double jm = J[0][j] * Mv[i][0] + J[1][j] * Mv[i][1] + J[2][j] * Mv[i][2];
            double h = w * (-d2 * a[i] * a[j] + jm);
            if (i >= 3 && j >= 3) {
                const double *hv = hb[i - 3][j - 3];
                double b = qt[0] * hv[0] + qt[1] * hv[1] + qt[2] * hv[2];
                h += compat ? -d2 * w * a[i] * b : w * b;
            }
            add(7 + 6 * i + j, h);
        }
}

__device__ __forceinline__ void warp_two_sum_reduce(float &s, float &e) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        float so = __shfl_xor_sync(kFull, s, o);
        float eo = __shfl_xor_sync(kFull, e, o);
        float t, err;
        two_sum(s, so, t, err);
        s = t;
        e = __fadd_rn(__fadd_rn(e, eo), err);
    }
}

// Tile partial layout: [0] score, [1..6] g, [7..42] H row major, [43] pairs.
__device__ __forceinline__ double h_entry(const double *tot, int i, int j, double kR, bool compat) {
    double v = tot[7 + (i <= j ? sidx(i, j) : sidx(j, i))];
    if (i >= 3 && j >= 3) {
        int a = i - 3, b = j - 3;
        double r = compat ? tot[28 + 3 * a + b] : tot[28 + 3 * (a < b ? a : b) + (a < b ? b : a)];
        v += kR * r;
    }
    return v;
}

// Pairs with a flagged voxel queued by the FP32 pass: (alignment, point,
// slot).  The point is transformed and its per-point terms recomputed exactly
// as the FP32 pass does, then the pair is evaluated in FP64.
__global__ void flagged_kernel(EvalArgs args) {
    const unsigned n = *args.flag_n;
    const unsigned m = n < args.flag_cap ? n : args.flag_cap;
    for (unsigned q = blockIdx.x * blockDim.x + threadIdx.x; q < m; q += gridDim.x * blockDim.x) {
        const int4 e = args.flag_q[q];
        const AlignState &st = args.states[e.x];
        const int mode = st.eval_mode;
        const bool hess = mode != kEvalGradient;
        const float4 x = args.points[e.y];
        float px, py, pz;
        if (args.trans) {
            const float4 y = args.trans[e.y];
            px = y.x; py = y.y; pz = y.z;
        } else {
            const float *T = st.T;
            px = T[0] * x.x + T[1] * x.y + T[2] * x.z + T[3];
            py = T[4] * x.x + T[5] * x.y + T[6] * x.z + T[7];
            pz = T[8] * x.x + T[9] * x.y + T[10] * x.z + T[11];
        }
        float t[kTerms];
        for (int k = 0; k < 8; ++k) t[k] = dot3f(x.x, x.y, x.z, st.angf + 3 * k);
        for (int k = 0; k < 15; ++k) t[8 + k] = dot3f(x.x, x.y, x.z, st.angf + 24 + 3 * k);
        const float4 hi = args.grid.mean_hi[e.z];
        const float4 lo = args.grid.mean_lo[e.z];
        pair_fp64_flagged(args.exc + (size_t)e.x * kPartial, t, (px - hi.x) - lo.x, (py - hi.y) - lo.y,
                          (pz - hi.z) - lo.z, args.grid.icov64 + 9 * (size_t)e.z, args.d1, args.d2, hess,
                          args.compat != 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && n > args.flag_cap) atomicOr(args.flag_overflow, 1);
}

// Dynamic shared memory of the FP32 kernel (W warps).
template <int W>
struct F32Smem {
    float acc[kAcc][W * 32];      // per-lane sums of the current alignment run
    float terms[W][kTerms][32];   // per-point terms of each warp's 32 points
    float xt[W][3][32];           // transformed points
    unsigned list[W][kList];      // accepted pairs of the current tile
    float2 red[W][kAcc];
};

// Block-wide reduction of the per-lane sums of one alignment run (TwoSum
// compensated across lanes and warps), written as the FP64 partial of the
// run's first tile; resets the sums.
template <int W>
__device__ void reduce_run(F32Smem<W> &sm, double *s_tot, const unsigned (*s_cnt)[3], double *out, double kR,
                           bool compat) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
#pragma unroll 1
    for (int k = 0; k < kAcc; ++k) {
        float s = sm.acc[k][threadIdx.x], e = 0.0f;
        sm.acc[k][threadIdx.x] = 0.0f;
        warp_two_sum_reduce(s, e);
        if (lane == 0) sm.red[warp][k] = make_float2(s, e);
    }
    __syncthreads();
    if (threadIdx.x < kAcc) {
        float s = sm.red[0][threadIdx.x].x, e = sm.red[0][threadIdx.x].y;
        for (int w = 1; w < W; ++w) {
            float t, err;
            two_sum(s, sm.red[w][threadIdx.x].x, t, err);
            s = t;
            e = __fadd_rn(__fadd_rn(e, sm.red[w][threadIdx.x].y), err);
        }
        s_tot[threadIdx.x] = (double)s + (double)e;
    }
    __syncthreads();
    if (threadIdx.x < kPartial) {
        const int k = threadIdx.x;
        double v;
        if (k < 7) {
            v = s_tot[k];
        } else if (k < 43) {
            v = h_entry(s_tot, (k - 7) / 6, (k - 7) % 6, kR, compat);
        } else {
            unsigned np = 0;
            for (int w = 0; w < W; ++w) np += s_cnt[w][2];
            v = (double)np;
        }
        out[k] = v;
    }
}

template <int TILE, int MINB>
__global__ void __launch_bounds__(TILE, MINB) derivative_f32_kernel(EvalArgs args) {
    constexpr int kW = TILE / 32;
    __shared__ float s_T[12];
    __shared__ float s_ang[kAngle];
    __shared__ int s_mode;
    __shared__ double s_tot[kAcc];
    __shared__ unsigned s_cnt[kW][3];
    extern __shared__ __align__(16) unsigned char s_dyn[];
    F32Smem<kW> &sm = *reinterpret_cast<F32Smem<kW> *>(s_dyn);

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool compat = args.compat != 0;
    const float d1f = (float)args.d1, d2f = (float)args.d2;
    const double kR = compat ? -args.d2 : 1.0;
    const GridDev &grid = args.grid;
    float (*terms)[32] = sm.terms[warp];
    float (*xts)[32] = sm.xt[warp];
    unsigned *list = sm.list[warp];
    float *acc = &sm.acc[0][threadIdx.x];

    const int nt = *args.num_tiles;
    const int per = (nt + gridDim.x - 1) / gridDim.x;
    const int t_begin = blockIdx.x * per;
    const int t_end = min(nt, t_begin + per);
    for (int k = 0; k < kAcc; ++k) acc[k * TILE] = 0.0f;
    if (lane == 0) s_cnt[warp][0] = s_cnt[warp][1] = s_cnt[warp][2] = 0;
    unsigned long long blk_probe = 0, blk_occ = 0, blk_pair = 0, blk_pts = 0, blk_tiles = 0;
    int cur = -1, run_first = -1, mode = kEvalNone;
    double *exc = nullptr;

    for (int ti = t_begin; ti < t_end; ++ti) {
        const Tile tile = args.tiles[ti];
        if (tile.align != cur) {
            if (cur >= 0 && mode != kEvalNone) {
                reduce_run<kW>(sm, s_tot, s_cnt, args.partials + (size_t)run_first * kPartial, kR, compat);
                __syncthreads();
                if (lane == 0) s_cnt[warp][0] = s_cnt[warp][1] = s_cnt[warp][2] = 0;
            }
            __syncthreads();
            const AlignState *st = args.states + tile.align;
            if (threadIdx.x == 0) s_mode = st->eval_mode;
            if (threadIdx.x < 12) s_T[threadIdx.x] = st->T[threadIdx.x];
            if (threadIdx.x < kAngle) s_ang[threadIdx.x] = st->angf[threadIdx.x];
            __syncthreads();
            cur = tile.align;
            run_first = ti;
            mode = s_mode;
            exc = args.exc + (size_t)tile.align * kPartial;
        } else if (mode != kEvalNone && threadIdx.x < kPartial) {
            args.partials[(size_t)ti * kPartial + threadIdx.x] = 0.0;
        }
        if (mode == kEvalNone) continue;
        const bool hess = mode != kEvalGradient;

        const int i = tile.start + threadIdx.x;
        const bool valid = i < tile.end;
        const float4 x = valid ? args.points[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        // transformPointCloud (kernel.cpp:397-400), float, left to right
        float px, py, pz;
        if (args.trans) {
            const float4 y = valid ? args.trans[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            px = y.x; py = y.y; pz = y.z;
        } else {
            px = s_T[0] * x.x + s_T[1] * x.y + s_T[2] * x.z + s_T[3];
            py = s_T[4] * x.x + s_T[5] * x.y + s_T[6] * x.z + s_T[7];
            pz = s_T[8] * x.x + s_T[9] * x.y + s_T[10] * x.z + s_T[11];
        }
        __syncwarp();
        xts[0][lane] = px;
        xts[1][lane] = py;
        xts[2][lane] = pz;
        unsigned n_probe = 0, n_occ = 0, n_pair = 0;
        bool have_terms = false;
        // evaluate list[0, n): one entry per lane per round
        auto consume = [&](int n) {
            if (n == 0) return;
            if (!have_terms) {
                // per-point terms of the ORIGINAL point (computePointDerivatives),
                // computed once a warp has pairs to evaluate
                const float *ja = s_ang;
#pragma unroll
                for (int k = 0; k < 8; ++k) terms[k][lane] = dot3f(x.x, x.y, x.z, ja + 3 * k);
                const float *h = s_ang + 24;
#pragma unroll
                for (int k = 0; k < 15; ++k) terms[8 + k][lane] = dot3f(x.x, x.y, x.z, h + 3 * k);
                have_terms = true;
                __syncwarp();
            }
            AccF A;
#pragma unroll
            for (int k = 0; k < kAcc; ++k) A.v[k] = 0.0f;
            for (int base = 0; base < n; base += 32) {
                const int k = base + lane;
                if (k >= n) break;
                const unsigned code = list[k];
                const int owner = code & 31;
                const int slot = (int)(code >> 6);
                const float4 hi = __ldg(grid.mean_hi + slot);
                const float4 lo = __ldg(grid.mean_lo + slot);
                // x' = x_trans - mean (kernel.cpp:692-694) from the (hi, lo) split
                const float p0 = (xts[0][owner] - hi.x) - lo.x;
                const float p1 = (xts[1][owner] - hi.y) - lo.y;
                const float p2 = (xts[2][owner] - hi.z) - lo.z;
                ++n_pair;
                if (code & 32) {
                    // FP64 side path, evaluated by flagged_kernel after this pass
                    const unsigned q = atomicAdd(args.flag_n, 1u);
                    if (q < args.flag_cap)
                        args.flag_q[q] = make_int4(tile.align, tile.start + warp * 32 + owner, slot, 0);
                } else {
                    const float4 ca = __ldg(grid.icov32 + 2 * slot);
                    const float4 cb = __ldg(grid.icov32 + 2 * slot + 1);
                    pair_fp32(A, terms, owner, p0, p1, p2, ca, cb, d1f, d2f, hess, compat);
                }
            }
#pragma unroll
            for (int k = 0; k < kAcc; ++k) acc[k * TILE] += A.v[k];
        };
        __syncwarp();
        probe_point(grid, px, py, pz, valid, list, n_probe, n_occ, consume);
        // per-warp work counters (pairs feed the partial's count)
        for (int o = 16; o > 0; o >>= 1) {
            n_probe += __shfl_xor_sync(kFull, n_probe, o);
            n_occ += __shfl_xor_sync(kFull, n_occ, o);
            n_pair += __shfl_xor_sync(kFull, n_pair, o);
        }
        if (lane == 0) s_cnt[warp][2] += n_pair;
        blk_probe += n_probe;
        blk_occ += n_occ;
        blk_pair += n_pair;
        blk_pts += (unsigned long long)(tile.end - tile.start);
        blk_tiles += 1;
    }
    if (cur >= 0 && mode != kEvalNone)
        reduce_run<kW>(sm, s_tot, s_cnt, args.partials + (size_t)run_first * kPartial, kR, compat);
    if (args.counters && lane == 0 && blk_tiles) {
        if (warp == 0) {
            atomicAdd(&args.counters->points, blk_pts);
            atomicAdd(&args.counters->tiles, blk_tiles);
        }
        atomicAdd(&args.counters->probes, blk_probe);
        atomicAdd(&args.counters->occupied_probes, blk_occ);
        atomicAdd(&args.counters->pairs, blk_pair);
    }
}

// ---------------------------------------------------------------------------
// FP64 variant: the reference's updateDerivatives / updateHessian expressions
// literally (compat) or the Magnusson eq. 6.13 Hessian (corrected), in FP64.
struct AccD {
    double v[43];  // score, g[6], H[36]
};

__device__ void pair_fp64(AccD &A, const double *x, const double *ang, const double *xt, const double *C, double d1,
                          double d2, bool hess, bool compat) {
    // point derivatives (computePointDerivatives, kernel.cpp:495-560)
    auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    double J[3][6] = {{1, 0, 0, 0, 0, 0}, {0, 1, 0, 0, 0, 0}, {0, 0, 1, 0, 0, 0}};
    J[1][3] = dot(x, ang + 0);
    J[2][3] = dot(x, ang + 3);
    J[0][4] = dot(x, ang + 6);
    J[1][4] = dot(x, ang + 9);
    J[2][4] = dot(x, ang + 12);
    J[0][5] = dot(x, ang + 15);
    J[1][5] = dot(x, ang + 18);
    J[2][5] = dot(x, ang + 21);
    const double *h = ang + 24;
    double blk[6][3];  // a b c d e f
    blk[0][0] = 0; blk[0][1] = dot(x, h + 0); blk[0][2] = dot(x, h + 3);
    blk[1][0] = 0; blk[1][1] = dot(x, h + 6); blk[1][2] = dot(x, h + 9);
    blk[2][0] = 0; blk[2][1] = dot(x, h + 12); blk[2][2] = dot(x, h + 15);
    blk[3][0] = dot(x, h + 18); blk[3][1] = dot(x, h + 21); blk[3][2] = dot(x, h + 24);
    blk[4][0] = dot(x, h + 27); blk[4][1] = dot(x, h + 30); blk[4][2] = dot(x, h + 33);
    blk[5][0] = dot(x, h + 36); blk[5][1] = dot(x, h + 39); blk[5][2] = dot(x, h + 42);
    const int bmap[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
    // updateDerivatives (kernel.cpp:438-493)
    double xCx = C[0] * xt[0] * xt[0] + C[4] * xt[1] * xt[1] + C[8] * xt[2] * xt[2] +
                 (C[1] + C[3]) * xt[0] * xt[1] + (C[2] + C[6]) * xt[0] * xt[2] + (C[5] + C[7]) * xt[1] * xt[2];
    double e = exp(-d2 * (xCx) / 2);
    double score_inc = -d1 * e;
    e = d2 * e;
    if (e > 1 || e < 0 || e != e) return;
    e *= d1;
    double cov[3];
    for (int i = 0; i < 6; ++i) {
        for (int r = 0; r < 3; ++r) {
            cov[r] = 0;
            for (int c = 0; c < 3; ++c) cov[r] += C[3 * r + c] * J[c][i];
        }
        A.v[1 + i] += dot(xt, cov) * e;
        if (!hess) continue;
        for (int j = 0; j < 6; ++j) {
            double col[3] = {J[0][j], J[1][j], J[2][j]};
            double hb[3] = {0, 0, 0};
            if (i >= 3 && j >= 3) {
                const double *bb = blk[bmap[i - 3][j - 3]];
                hb[0] = bb[0]; hb[1] = bb[1]; hb[2] = bb[2];
            }
            if (compat) {
                double colh[3] = {col[0] + hb[0], col[1] + hb[1], col[2] + hb[2]};
                double mp[3];
                for (int r = 0; r < 3; ++r) {
                    mp[r] = 0;
                    for (int c = 0; c < 3; ++c) mp[r] += C[3 * r + c] * colh[c];
                }
                A.v[7 + 6 * i + j] += e * (-d2 * dot(xt, cov) * dot(xt, mp) + dot(col, cov));
            } else {
                double cj[3], ch[3];
                for (int r = 0; r < 3; ++r) {
                    cj[r] = C[3 * r] * col[0] + C[3 * r + 1] * col[1] + C[3 * r + 2] * col[2];
                    ch[r] = C[3 * r] * hb[0] + C[3 * r + 1] * hb[1] + C[3 * r + 2] * hb[2];
                }
                A.v[7 + 6 * i + j] += e * (-d2 * dot(xt, cov) * dot(xt, cj) + dot(xt, ch) + dot(col, cov));
            }
        }
    }
    A.v[0] += score_inc;
}

constexpr int kTile64 = 256;

__global__ void __launch_bounds__(kTile64, 1) derivative_f64_kernel(EvalArgs args) {
    constexpr int kW = kTile64 / 32;
    __shared__ float s_T[12];
    __shared__ double s_ang[kAngle];
    __shared__ int s_mode;
    __shared__ float s_pts[kW][6][32];  // original xyz, transformed xyz
    __shared__ unsigned s_list[kW][kList];
    __shared__ double s_red[kW][43];
    __shared__ unsigned s_cnt[kW][3];

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool compat = args.compat != 0;
    const GridDev &grid = args.grid;
    unsigned *list = s_list[warp];
    float (*pts)[32] = s_pts[warp];

    for (int ti = blockIdx.x, nt = *args.num_tiles; ti < nt; ti += gridDim.x) {
        const Tile tile = args.tiles[ti];
        const AlignState *st = args.states + tile.align;
        __syncthreads();
        if (threadIdx.x == 0) s_mode = st->eval_mode;
        if (threadIdx.x < 12) s_T[threadIdx.x] = st->T[threadIdx.x];
        if (threadIdx.x < kAngle) s_ang[threadIdx.x] = st->angd[threadIdx.x];
        __syncthreads();
        const int mode = s_mode;
        if (mode == kEvalNone) continue;
        const bool hess = mode != kEvalGradient;
        const int i = tile.start + threadIdx.x;
        const bool valid = i < tile.end;
        const float4 x = valid ? args.points[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        float px, py, pz;
        if (args.trans) {
            const float4 y = valid ? args.trans[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            px = y.x; py = y.y; pz = y.z;
        } else {
            px = s_T[0] * x.x + s_T[1] * x.y + s_T[2] * x.z + s_T[3];
            py = s_T[4] * x.x + s_T[5] * x.y + s_T[6] * x.z + s_T[7];
            pz = s_T[8] * x.x + s_T[9] * x.y + s_T[10] * x.z + s_T[11];
        }
        __syncwarp();
        pts[0][lane] = x.x; pts[1][lane] = x.y; pts[2][lane] = x.z;
        pts[3][lane] = px; pts[4][lane] = py; pts[5][lane] = pz;
        AccD A;
        for (int k = 0; k < 43; ++k) A.v[k] = 0.0;
        unsigned n_probe = 0, n_occ = 0, n_pair = 0;
        auto consume = [&](int n) {
            for (int base = 0; base < n; base += 32) {
                const int kk = base + lane;
                if (kk >= n) break;
                const unsigned code = list[kk];
                const int owner = code & 31;
                const int slot = (int)(code >> 6);
                const double4 m = ldg_d4(grid.mean + slot);
                const double xo[3] = {pts[0][owner], pts[1][owner], pts[2][owner]};
                const double xt[3] = {(double)pts[3][owner] - m.x, (double)pts[4][owner] - m.y,
                                      (double)pts[5][owner] - m.z};
                pair_fp64(A, xo, s_ang, xt, grid.icov64 + 9 * (size_t)slot, args.d1, args.d2, hess, compat);
                ++n_pair;
            }
        };
        __syncwarp();
        probe_point(grid, px, py, pz, valid, list, n_probe, n_occ, consume);
        for (int k = 0; k < 43; ++k) {
            double v = A.v[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
            if (lane == 0) s_red[warp][k] = v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            n_probe += __shfl_xor_sync(kFull, n_probe, o);
            n_occ += __shfl_xor_sync(kFull, n_occ, o);
            n_pair += __shfl_xor_sync(kFull, n_pair, o);
        }
        if (lane == 0) {
            s_cnt[warp][0] = n_probe;
            s_cnt[warp][1] = n_occ;
            s_cnt[warp][2] = n_pair;
        }
        __syncthreads();
        double *out = args.partials + (size_t)tile.slot * kPartial;
        if (threadIdx.x < kPartial) {
            const int k = threadIdx.x;
            double v = 0.0;
            if (k < 43) {
                for (int w = 0; w < kW; ++w) v += s_red[w][k];
            } else {
                unsigned np = 0;
                for (int w = 0; w < kW; ++w) np += s_cnt[w][2];
                v = (double)np;
            }
            out[k] = v;
        }
        if (threadIdx.x == 0 && args.counters) {
            unsigned long long a0 = 0, a1 = 0, a2 = 0;
            for (int w = 0; w < kW; ++w) {
                a0 += s_cnt[w][0];
                a1 += s_cnt[w][1];
                a2 += s_cnt[w][2];
            }
            atomicAdd(&args.counters->probes, a0);
            atomicAdd(&args.counters->occupied_probes, a1);
            atomicAdd(&args.counters->pairs, a2);
            atomicAdd(&args.counters->points, (unsigned long long)(tile.end - tile.start));
            atomicAdd(&args.counters->tiles, 1ull);
        }
    }
}

template <int TILE, int MINB>
cudaError_t prepare_one() {
    return cudaFuncSetAttribute(derivative_f32_kernel<TILE, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(F32Smem<TILE / 32>));
}

template <int TILE, int MINB>
void launch_one(const EvalArgs &args, int blocks, cudaStream_t st) {
    derivative_f32_kernel<TILE, MINB><<<blocks, TILE, sizeof(F32Smem<TILE / 32>), st>>>(args);
}

}  // namespace

const DerivVariant kDerivVariants[kNumDerivVariants] = {
    {256, 2}, {256, 1}, {128, 4}, {128, 3}, {256, 3},
};

int prepare_derivatives() {
    cudaError_t e = cudaSuccess, r;
    if ((r = prepare_one<256, 2>()) != cudaSuccess) e = r;
    if ((r = prepare_one<256, 1>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 4>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 3>()) != cudaSuccess) e = r;
    if ((r = prepare_one<256, 3>()) != cudaSuccess) e = r;
    return (int)e;
}

int launch_derivatives(const EvalArgs &args, int precision, int variant, int sms, cudaStream_t st) {
    if (args.max_tiles <= 0) return 0;
    if (precision == 1) {
        if (args.tile_size != kTile64) return (int)cudaErrorInvalidValue;
        int blocks = sms < args.max_tiles ? sms : args.max_tiles;
        derivative_f64_kernel<<<blocks, kTile64, 0, st>>>(args);
        return (int)cudaGetLastError();
    }
    if (variant < 0 || variant >= kNumDerivVariants) variant = 0;
    const DerivVariant v = kDerivVariants[variant];
    if (args.tile_size != v.tile) return (int)cudaErrorInvalidValue;
    long long want = (long long)sms * v.min_blocks;
    int blocks = (int)(want < args.max_tiles ? want : args.max_tiles);
    cudaMemsetAsync(args.flag_n, 0, sizeof(unsigned), st);
    switch (variant) {
        case 0: launch_one<256, 2>(args, blocks, st); break;
        case 1: launch_one<256, 1>(args, blocks, st); break;
        case 2: launch_one<128, 4>(args, blocks, st); break;
        case 3: launch_one<128, 3>(args, blocks, st); break;
        default: launch_one<256, 3>(args, blocks, st); break;
    }
    flagged_kernel<<<sms, 128, 0, st>>>(args);
    return (int)cudaGetLastError();
}

}  // namespace ndt
