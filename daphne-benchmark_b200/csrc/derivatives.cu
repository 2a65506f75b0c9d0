// The derivative pass: score, gradient and Hessian of the NDT objective for a
// batch of alignments (computeDerivatives / computeHessian,
// src/CPU/ndt_mapping/kernel.cpp:562-705, with voxelRadiusSearch :246-286,
// computePointDerivatives :495-560 and updateDerivatives :438-493 fused in).
//
// One block (256 threads) handles one tile of up to 256 consecutive points of
// ONE alignment; blocks loop over the tile list (persistent grid), skipping
// tiles whose alignment has nothing to evaluate this round.
//
// Per point (one thread):
//   1. transform by the alignment's float 3x4 (transformPointCloud :385-404,
//      same float operation order);
//   2. the reference's 27 float probe points p + {-r, 0, r}^3 with its bounds
//      test, cell linearisation and the `dist < r` test on the FP64 voxel mean,
//      all with the reference's float/double roundings, so the set and order
//      of accepted (point, voxel) pairs equals the reference's;
//   3. accepted pairs are appended to a per-warp ring in shared memory
//      (ballot + popc); whenever 32 are queued the warp evaluates them one per
//      lane, so the per-pair work stays load-balanced across lanes whatever
//      the neighbour counts are.
// Per pair (FP32 path): q = C x', xCx, e = exp(-d2 xCx / 2), the validity test
// of :456, gradient a_i = x'^T C J_i and the Hessian split as
//   H_ij = S_ij + k R_ij,  S_ij = w (-d2 a_i a_j + J_j^T C J_i)   (i <= j)
//   compat:    R_ij = w a_i b_ij, k = -d2  (the reference's :486-488 form)
//   corrected: R_ij = w b_ij,     k = 1    (Magnusson eq. 6.13)
// with b_ij = x'^T C H_ij (nonzero for i, j >= 3 only).  37 FP32 lane sums are
// reduced with error-free TwoSum across the warp and the block; the tile
// partial is written as FP64 (hi + lo).  Voxels flagged by the grid build
// (inverse-covariance entries non-finite or beyond 1e30) are evaluated in
// FP64 so that infinities and NaNs propagate as in the reference.
//
// The FP64 variant (precision = 1) evaluates every pair with the reference's
// literal FP64 expressions and accumulates in FP64.
#include <cuda_runtime.h>
#include <stdint.h>

#include "derivatives.h"
#include "ndt_math.cuh"

namespace ndt {

namespace {

constexpr int kWarpsE = kTile / 32;
constexpr int kAcc = 37;    // score, g[6], S[21], R[9]
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
constexpr int kTerms = 23;

// The reference's probe walk for one transformed point: trip counts of the
// three float loops (z outer, x inner), capped at 4 (the reference's loops run
// 3 times for finite coordinates below ~1e6 m; the cap only stops the endless
// loop it enters for infinite coordinates).
struct ProbeStart {
    float x0, y0, z0;
    int nx, ny, nz;
};

__device__ __forceinline__ int trips(float start, float limit, float res) {
    int n = 0;
    float v = start;
    while (n < 4 && v <= limit) {
        ++n;
        v = v + res;
    }
    return n;
}

__device__ __forceinline__ ProbeStart probe_start(float px, float py, float pz, float res, bool valid) {
    const double radius = (double)res;
    const float rf = (float)(radius + (double)0.001f);  // radiusFinal, kernel.cpp:254
    ProbeStart s;
    s.x0 = (float)((double)px - radius);
    s.y0 = (float)((double)py - radius);
    s.z0 = (float)((double)pz - radius);
    s.nx = valid ? trips(s.x0, px + rf, res) : 0;
    s.ny = valid ? trips(s.y0, py + rf, res) : 0;
    s.nz = valid ? trips(s.z0, pz + rf, res) : 0;
    return s;
}

constexpr int kList = 27 * 32;  // per-warp pair list: all 27 probes of all 32 lanes

// Append the accepted (point, voxel) pairs of one probe step of the warp to
// the list (code = slot << 6 | flag << 5 | lane), in lane order.
__device__ __forceinline__ void list_append(unsigned *list, int &n, bool acc, unsigned code, unsigned lt) {
    const unsigned b = __ballot_sync(kFull, acc);
    if (acc) list[n + __popc(b & lt)] = code;
    n += __popc(b);
}

// Probe the reference's 27 cells around every lane's point (z outer, x
// inner; voxelRadiusSearch, kernel.cpp:246-286) and collect the accepted
// pairs in `list`.  Fast path (trip counts <= 3, i.e. every finite coordinate
// below ~1e6 m): the 27 index loads, then the voxel-mean loads of one
// z-layer at a time, are all in flight together, and the list (27 x 32
// entries) cannot overflow.  Generic path (up to 4 x 4 x 4 probes): one probe
// at a time, calling flush(n) whenever the list could overflow.
template <class Flush>
__device__ __forceinline__ int probe_list(const GridDev &grid, float px, float py, float pz, bool valid,
                                          unsigned *list, unsigned &n_probe, unsigned &n_occ, Flush flush) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const GridMeta &g = grid.meta;
    const float res = g.res;
    const double radius = (double)res;
    const ProbeStart ps = probe_start(px, py, pz, res, valid);
    const int mz = __reduce_max_sync(kFull, ps.nz);
    const int my = __reduce_max_sync(kFull, ps.ny);
    const int mx = __reduce_max_sync(kFull, ps.nx);
    int n = 0;
    if (mz <= 3 && my <= 3 && mx <= 3) {
        float zc[3], yc[3], xc[3];
        zc[0] = ps.z0; zc[1] = zc[0] + res; zc[2] = zc[1] + res;
        yc[0] = ps.y0; yc[1] = yc[0] + res; yc[2] = yc[1] + res;
        xc[0] = ps.x0; xc[1] = xc[0] + res; xc[2] = xc[1] + res;
        int v[27];
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float z = zc[a], y = yc[b], x = xc[c];
                    const bool act = a < ps.nz && b < ps.ny && c < ps.nx;
                    const bool inb = act && !((x < g.minv[0]) || (x > g.maxv[0]) || (y < g.minv[1]) ||
                                              (y > g.maxv[1]) || (z < g.minv[2]) || (z > g.maxv[2]));
                    int slot = -1;
                    if (inb) {
                        const int ix = (int)((x - g.minv[0]) / res);
                        const int iy = (int)((y - g.minv[1]) / res);
                        const int iz = (int)((z - g.minv[2]) / res);
                        slot = __ldg(grid.index + (ix + g.dim[0] * (iy + g.dim[1] * iz)));
                        ++n_probe;
                    }
                    v[9 * a + 3 * b + c] = slot;
                }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            float4 mf[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int slot = v[9 * a + k];
                if (slot >= 0) mf[k] = __ldg(grid.mean32 + (slot & kSlotMask));
            }
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                const int slot = v[9 * a + k];
                bool acc = false;
                if (slot >= 0) {
                    ++n_occ;
                    // FP32-mean distance; it differs from the reference's
                    // (FP64 mean, float differences) by less than tol, so
                    // only distances within tol of r need the exact test
                    const float fx = mf[k].x - px, fy = mf[k].y - py, fz = mf[k].z - pz;
                    const float fd = sqrtf(fx * fx + fy * fy + fz * fz);
                    const float tol = 1e-6f + 2.384185791e-7f * (fabsf(mf[k].x) + fabsf(mf[k].y) + fabsf(mf[k].z));
                    if (fd < res - tol) {
                        acc = true;
                    } else if (fd <= res + tol) {
                        const double4 m = ldg_d4(grid.mean + (slot & kSlotMask));
                        const float dx = (float)(m.x - (double)px);
                        const float dy = (float)(m.y - (double)py);
                        const float dz = (float)(m.z - (double)pz);
                        const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
                        acc = (double)dist < radius;
                    }
                }
                const unsigned code = ((unsigned)(slot & kSlotMask) << 6) | ((slot & kSlotFlag) ? 32u : 0u) | lane;
                list_append(list, n, acc, code, lt);
            }
        }
        return n;
    }
    // generic path
    float zc = ps.z0;
    for (int az = 0; az < mz; ++az, zc = zc + res) {
        float yc = ps.y0;
        for (int ay = 0; ay < my; ++ay, yc = yc + res) {
            float xc = ps.x0;
            for (int ax = 0; ax < mx; ++ax, xc = xc + res) {
                const bool act = az < ps.nz && ay < ps.ny && ax < ps.nx;
                const bool inb = act && !((xc < g.minv[0]) || (xc > g.maxv[0]) || (yc < g.minv[1]) ||
                                          (yc > g.maxv[1]) || (zc < g.minv[2]) || (zc > g.maxv[2]));
                int slot = -1;
                if (inb) {
                    const int ix = (int)((xc - g.minv[0]) / res);
                    const int iy = (int)((yc - g.minv[1]) / res);
                    const int iz = (int)((zc - g.minv[2]) / res);
                    slot = __ldg(grid.index + (ix + g.dim[0] * (iy + g.dim[1] * iz)));
                    ++n_probe;
                }
                bool acc = false;
                if (slot >= 0) {
                    ++n_occ;
                    const double4 m = ldg_d4(grid.mean + (slot & kSlotMask));
                    const float dx = (float)(m.x - (double)px);
                    const float dy = (float)(m.y - (double)py);
                    const float dz = (float)(m.z - (double)pz);
                    const float dist = sqrtf(dx * dx + dy * dy + dz * dz);
                    acc = (double)dist < radius;
                }
                if (n > kList - 32) {
                    __syncwarp();
                    flush(n);
                    __syncwarp();
                    n = 0;
                }
                const unsigned code = ((unsigned)(slot & kSlotMask) << 6) | ((slot & kSlotFlag) ? 32u : 0u) | lane;
                list_append(list, n, acc, code, lt);
            }
        }
    }
    return n;
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
__device__ __noinline__ void pair_fp64_flagged(double *exc, const float (*terms)[32], int owner, float p0f, float p1f,
                                               float p2f, const double *C, double d1, double d2, bool hess,
                                               bool compat) {
    float t[kTerms];
    for (int k = 0; k < kTerms; ++k) t[k] = terms[k][owner];
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

// Dynamic shared memory of the FP32 kernel (W warps).
template <int W>
struct F32Smem {
    float acc[kAcc][W * 32];  // per-lane sums of the current alignment run
    float terms[W][kTerms][32];
    float xt[W][3][32];
    unsigned list[W][kList];
    float2 red[W][kAcc];
};

// Generic-path overflow (coordinates beyond ~1e6 m only): evaluate the queued
// pairs through the FP64 side path, whose sums land in exc with atomics.
__device__ __noinline__ void flush_fp64(const unsigned *list, int n, const float (*terms)[32], const float (*xts)[32],
                                        const GridDev &grid, double *exc, double d1, double d2, bool hess,
                                        bool compat) {
    const int lane = threadIdx.x & 31;
    for (int k = lane; k < n; k += 32) {
        const unsigned code = list[k];
        const int owner = code & 31;
        const int slot = (int)(code >> 6);
        const double4 m = ldg_d4(grid.mean + slot);
        pair_fp64_flagged(exc, terms, owner, (float)((double)xts[0][owner] - m.x), (float)((double)xts[1][owner] - m.y),
                          (float)((double)xts[2][owner] - m.z), grid.icov64 + 9 * (size_t)slot, d1, d2, hess, compat);
    }
}

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

// FP32 derivative pass.  Block b owns the contiguous tile range
// [b * per, (b + 1) * per) of the tile list (tiles of one alignment are
// consecutive), keeps per-lane sums in shared memory across the tiles of one
// alignment and reduces once per alignment run; the run's partial goes to the
// slot of its first tile, the other slots of the run get zeros.
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

    const int nt = *args.num_tiles;
    const int per = (nt + gridDim.x - 1) / gridDim.x;
    const int t_begin = blockIdx.x * per;
    const int t_end = min(nt, t_begin + per);
    for (int k = 0; k < kAcc; ++k) sm.acc[k][threadIdx.x] = 0.0f;
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
        // per-point terms of the ORIGINAL point (computePointDerivatives)
        {
            const float *ja = s_ang;
#pragma unroll
            for (int k = 0; k < 8; ++k) terms[k][lane] = dot3f(x.x, x.y, x.z, ja + 3 * k);
            const float *h = s_ang + 24;
#pragma unroll
            for (int k = 0; k < 15; ++k) terms[8 + k][lane] = dot3f(x.x, x.y, x.z, h + 3 * k);
        }
        unsigned n_probe = 0, n_occ = 0, n_pair = 0;
        auto flush = [&](int n) {
            flush_fp64(list, n, terms, xts, grid, exc, args.d1, args.d2, hess, compat);
            n_pair += (lane < n) ? (unsigned)((n - lane + 31) / 32) : 0u;
        };
        __syncwarp();
        const int n = probe_list(grid, px, py, pz, valid, list, n_probe, n_occ, flush);
        __syncwarp();
        AccF A;
#pragma unroll
        for (int k = 0; k < kAcc; ++k) A.v[k] = 0.0f;
        // evaluate list[0, n): one entry per lane per round
        for (int base = 0; base < n; base += 32) {
            const int k = base + lane;
            if (k >= n) break;
            const unsigned code = list[k];
            const int owner = code & 31;
            const int slot = (int)(code >> 6);
            const double2 *q = reinterpret_cast<const double2 *>(grid.mean + slot);
            const double2 m01 = __ldg(q);
            const double m2 = __ldg(reinterpret_cast<const double *>(q + 1));
            // x' = x_trans - mean (kernel.cpp:692-694), rounded to float
            const float p0 = (float)((double)xts[0][owner] - m01.x);
            const float p1 = (float)((double)xts[1][owner] - m01.y);
            const float p2 = (float)((double)xts[2][owner] - m2);
            ++n_pair;
            if (code & 32) {
                pair_fp64_flagged(exc, terms, owner, p0, p1, p2, grid.icov64 + 9 * (size_t)slot, args.d1, args.d2,
                                  hess, compat);
            } else {
                const float4 ca = __ldg(grid.icov32 + 2 * slot);
                const float4 cb = __ldg(grid.icov32 + 2 * slot + 1);
                pair_fp32(A, terms, owner, p0, p1, p2, ca, cb, d1f, d2f, hess, compat);
            }
        }
#pragma unroll
        for (int k = 0; k < kAcc; ++k) sm.acc[k][threadIdx.x] += A.v[k];
        // per-warp work counters of the run (pairs feed the partial's count)
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
        // every warp holds the warp-summed counts; warp 0 reports per-block totals of probes and pairs
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

__global__ void __launch_bounds__(kTile, 1) derivative_f64_kernel(EvalArgs args) {
    __shared__ float s_T[12];
    __shared__ double s_ang[kAngle];
    __shared__ int s_mode;
    __shared__ float s_pts[kWarpsE][6][32];  // original xyz, transformed xyz
    __shared__ unsigned s_list[kWarpsE][kList];
    __shared__ double s_red[kWarpsE][43];
    __shared__ unsigned s_cnt[kWarpsE][3];

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
        pts[0][lane] = x.x; pts[1][lane] = x.y; pts[2][lane] = x.z;
        pts[3][lane] = px; pts[4][lane] = py; pts[5][lane] = pz;
        AccD A;
        for (int k = 0; k < 43; ++k) A.v[k] = 0.0;
        unsigned n_probe = 0, n_occ = 0, n_pair = 0;
        auto process = [&](int n) {
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
        const int n = probe_list(grid, px, py, pz, valid, list, n_probe, n_occ, process);
        __syncwarp();
        process(n);
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
                for (int w = 0; w < kWarpsE; ++w) v += s_red[w][k];
            } else {
                unsigned np = 0;
                for (int w = 0; w < kWarpsE; ++w) np += s_cnt[w][2];
                v = (double)np;
            }
            out[k] = v;
        }
        if (threadIdx.x == 0 && args.counters) {
            unsigned long long a0 = 0, a1 = 0, a2 = 0;
            for (int w = 0; w < kWarpsE; ++w) {
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

}  // namespace

namespace {
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
    {256, 2}, {256, 1}, {128, 4}, {128, 3}, {128, 2},
};

int prepare_derivatives() {
    cudaError_t e = cudaSuccess;
    cudaError_t r;
    if ((r = prepare_one<256, 2>()) != cudaSuccess) e = r;
    if ((r = prepare_one<256, 1>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 4>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 3>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 2>()) != cudaSuccess) e = r;
    return (int)e;
}

int launch_derivatives(const EvalArgs &args, int precision, int variant, int sms, cudaStream_t st) {
    if (args.max_tiles <= 0) return 0;
    if (precision == 1) {
        if (args.tile_size != kTile) return (int)cudaErrorInvalidValue;
        int blocks = sms < args.max_tiles ? sms : args.max_tiles;
        derivative_f64_kernel<<<blocks, kTile, 0, st>>>(args);
        return (int)cudaGetLastError();
    }
    if (variant < 0 || variant >= kNumDerivVariants) variant = 0;
    const DerivVariant v = kDerivVariants[variant];
    if (args.tile_size != v.tile) return (int)cudaErrorInvalidValue;
    long long want = (long long)sms * v.min_blocks;
    int blocks = (int)(want < args.max_tiles ? want : args.max_tiles);
    switch (variant) {
        case 0: launch_one<256, 2>(args, blocks, st); break;
        case 1: launch_one<256, 1>(args, blocks, st); break;
        case 2: launch_one<128, 4>(args, blocks, st); break;
        case 3: launch_one<128, 3>(args, blocks, st); break;
        default: launch_one<128, 2>(args, blocks, st); break;
    }
    return (int)cudaGetLastError();
}

}  // namespace ndt
