// The FP32 derivative pass: score, gradient and Hessian of the NDT
// objective for a batch of alignments (computeDerivatives / computeHessian,
// src/CPU/ndt_mapping/kernel.cpp:562-705, with voxelRadiusSearch :246-286,
// computePointDerivatives :495-560 and updateDerivatives :438-493 fused in).
//
// Work decomposition: the tile list holds ceil(n_a / TILE) tiles of TILE
// consecutive points per alignment, handed out to the persistent blocks in
// chunks of consecutive tiles.  Each lane keeps its FP32 sums of the current
// alignment in shared memory and the block reduces them once per alignment
// run, adding the FP32 lane sums in FP64 in a fixed order (across lanes, then
// warps), writing the run's FP64 partial to the slot of its first tile (the
// run's other slots get zeros).
//
// Per point (one thread): the float transform and the reference's neighbour
// search of probe.cuh (exact: the accepted pairs are the reference's), each
// lane's pairs in its own column of shared memory.  Then, per warp:
//   dense  (more than 32 pairs in the warp): each lane sums its own pairs
//          into 16 FP32 point sums and contracts them with its point's
//          Jacobian and Hessian terms once (factored form below);
//   sparse: the pairs are appended to a per-warp ring and evaluated 32 at a
//          time, one pair per lane, each contracted on its own; the ring is
//          emptied at the end of the alignment run.
// Both kinds go through one evaluation loop (eval_steps), so the pair sums
// and the contraction appear once in the kernel; compat and corrected mode,
// and maps with and without a probe-window table, are separate
// instantiations.  The kernel's instruction footprint is what this buys:
// each instantiation carries only the code it runs.
// Voxels flagged by the grid build (inverse-covariance entries non-finite or
// beyond 1e30) are queued and evaluated in FP64 by flagged_kernel, so that
// infinities and NaNs propagate as in the reference.
//
// This file is compiled with floating-point contraction (the pair arithmetic
// is FP32 with FMA); the exact parts live in probe.cuh with explicit
// rounding intrinsics.
#include <cuda_runtime.h>
#include <stdint.h>

#include "derivatives.h"
#include "ndt_math.cuh"
#include "probe.cuh"

namespace ndt {

namespace {

// ---------------------------------------------------------------------------
// FP32 pair evaluation, factored through the point.
//
// For a point x with Jacobian J (3 x 6; columns e0, e1, e2, J_3, J_4, J_5) and
// point-Hessian vectors h_ij (i, j >= 3), the pairs (x, voxel v) contribute,
// with x' = x_trans - mean_v, C = C_v, q = C x', e = exp(-d2 x'^T q / 2),
// w = d1 d2 e (kept when 0 <= d2 e <= 1, kernel.cpp:456) and a_i = q . J_i:
//   score   sum -d1 e
//   g_i     sum w a_i                              = J_i . U
//   S_ij    sum w (-d2 a_i a_j + J_j^T C J_i)      = J_i^T (W - d2 Q) J_j
//   R_ij    compat:    sum w a_i (q . h_ij)        = J_i^T Q h_ij
//           corrected: sum w (q . h_ij)            = U . h_ij
// with the point's sums U = sum w q, Q = sum w q q^T, W = sum w C.  A pair
// therefore costs 16 FMA-type sums (PairSums) and a point one contraction
// with its J and h (contract_add), however many pairs it has.  H = S + k R,
// k = -d2 (compat, the reference's :486-488 form) or 1 (corrected, Magnusson
// eq. 6.13), is assembled from the block totals.
struct PairSums {
    float s, u0, u1, u2;
    float q00, q01, q02, q11, q12, q22;
    float w00, w01, w02, w11, w12, w22;
};

__device__ __forceinline__ void zero(PairSums &F) {
    F.s = F.u0 = F.u1 = F.u2 = 0.0f;
    F.q00 = F.q01 = F.q02 = F.q11 = F.q12 = F.q22 = 0.0f;
    F.w00 = F.w01 = F.w02 = F.w11 = F.w12 = F.w22 = 0.0f;
}

__device__ __forceinline__ void pair_sums(PairSums &F, float p0, float p1, float p2, float c00, float c01, float c02,
                                          float c11, float c12, float c22, float d1, float d2, bool hess) {
    const float q0 = fmaf(c00, p0, fmaf(c01, p1, c02 * p2));
    const float q1 = fmaf(c01, p0, fmaf(c11, p1, c12 * p2));
    const float q2 = fmaf(c02, p0, fmaf(c12, p1, c22 * p2));
    const float xCx = fmaf(p0, q0, fmaf(p1, q1, p2 * q2));
    const float e = expf(-d2 * xCx * 0.5f);
    const float e2 = d2 * e;
    if (!(e2 <= 1.0f && e2 >= 0.0f)) return;  // kernel.cpp:456 (also rejects NaN)
    const float w = d1 * e2;
    F.s = fmaf(-d1, e, F.s);
    // every multiply-add is written as fmaf or as separately rounded
    // operations, so the FP32 results do not depend on the compiler's
    // contraction choices (which can change with the surrounding code)
    const float wq0 = __fmul_rn(w, q0), wq1 = __fmul_rn(w, q1), wq2 = __fmul_rn(w, q2);
    F.u0 = fmaf(w, q0, F.u0);
    F.u1 = fmaf(w, q1, F.u1);
    F.u2 = fmaf(w, q2, F.u2);
    if (!hess) return;
    F.q00 = fmaf(wq0, q0, F.q00);
    F.q01 = fmaf(wq0, q1, F.q01);
    F.q02 = fmaf(wq0, q2, F.q02);
    F.q11 = fmaf(wq1, q1, F.q11);
    F.q12 = fmaf(wq1, q2, F.q12);
    F.q22 = fmaf(wq2, q2, F.q22);
    F.w00 = fmaf(w, c00, F.w00);
    F.w01 = fmaf(w, c01, F.w01);
    F.w02 = fmaf(w, c02, F.w02);
    F.w11 = fmaf(w, c11, F.w11);
    F.w12 = fmaf(w, c12, F.w12);
    F.w22 = fmaf(w, c22, F.w22);
}

// Symmetric 3 x 3 (m00 m01 m02 m11 m12 m22) times v.
__device__ __forceinline__ void sym_mul(float m00, float m01, float m02, float m11, float m12, float m22, float v0,
                                        float v1, float v2, float &r0, float &r1, float &r2) {
    r0 = fmaf(m00, v0, fmaf(m01, v1, m02 * v2));
    r1 = fmaf(m01, v0, fmaf(m11, v1, m12 * v2));
    r2 = fmaf(m02, v0, fmaf(m12, v1, m22 * v2));
}

// Adds a point's contribution (its PairSums F contracted with its J and h) to
// the lane's accumulators acc[k * stride]: [0] score, [1..6] g, [7..27] S
// (upper triangle), [28..36] R (compat: 3 x 3; corrected: upper triangle).
// ang = the alignment's FP32 angle terms (j_ang a..h, h_ang a2..f3, 3 each).
__device__ __forceinline__ void contract_add(const PairSums &F, float x0, float x1, float x2, const float *ang,
                                             float *acc, int stride, float d2, bool hess, bool compat) {
    // J_3 = (0, J13, J23), J_4 = (J04, J14, J24), J_5 = (J05, J15, J25)
    // (computePointDerivatives, kernel.cpp:512-521)
    const float J13 = dot3f(x0, x1, x2, ang + 0), J23 = dot3f(x0, x1, x2, ang + 3);
    const float J04 = dot3f(x0, x1, x2, ang + 6), J14 = dot3f(x0, x1, x2, ang + 9);
    const float J24 = dot3f(x0, x1, x2, ang + 12), J05 = dot3f(x0, x1, x2, ang + 15);
    const float J15 = dot3f(x0, x1, x2, ang + 18), J25 = dot3f(x0, x1, x2, ang + 21);
    acc[0] += F.s;
    acc[1 * stride] += F.u0;
    acc[2 * stride] += F.u1;
    acc[3 * stride] += F.u2;
    acc[4 * stride] += fmaf(J13, F.u1, J23 * F.u2);
    acc[5 * stride] += fmaf(J04, F.u0, fmaf(J14, F.u1, J24 * F.u2));
    acc[6 * stride] += fmaf(J05, F.u0, fmaf(J15, F.u1, J25 * F.u2));
    if (!hess) return;
    // P = W - d2 Q
    const float nd2 = -d2;
    const float P00 = fmaf(nd2, F.q00, F.w00), P01 = fmaf(nd2, F.q01, F.w01), P02 = fmaf(nd2, F.q02, F.w02);
    const float P11 = fmaf(nd2, F.q11, F.w11), P12 = fmaf(nd2, F.q12, F.w12), P22 = fmaf(nd2, F.q22, F.w22);
    float a0, a1, a2, b0, b1, b2, c0, c1, c2;  // P J_3, P J_4, P J_5
    sym_mul(P00, P01, P02, P11, P12, P22, 0.0f, J13, J23, a0, a1, a2);
    sym_mul(P00, P01, P02, P11, P12, P22, J04, J14, J24, b0, b1, b2);
    sym_mul(P00, P01, P02, P11, P12, P22, J05, J15, J25, c0, c1, c2);
    float *S = acc + 7 * stride;  // sidx order: (0,0..5), (1,1..5), (2,2..5), (3,3..5), (4,4..5), (5,5)
    S[0 * stride] += P00;
    S[1 * stride] += P01;
    S[2 * stride] += P02;
    S[3 * stride] += a0;
    S[4 * stride] += b0;
    S[5 * stride] += c0;
    S[6 * stride] += P11;
    S[7 * stride] += P12;
    S[8 * stride] += a1;
    S[9 * stride] += b1;
    S[10 * stride] += c1;
    S[11 * stride] += P22;
    S[12 * stride] += a2;
    S[13 * stride] += b2;
    S[14 * stride] += c2;
    S[15 * stride] += fmaf(J13, a1, J23 * a2);
    S[16 * stride] += fmaf(J13, b1, J23 * b2);
    S[17 * stride] += fmaf(J13, c1, J23 * c2);
    S[18 * stride] += fmaf(J04, b0, fmaf(J14, b1, J24 * b2));
    S[19 * stride] += fmaf(J04, c0, fmaf(J14, c1, J24 * c2));
    S[20 * stride] += fmaf(J05, c0, fmaf(J15, c1, J25 * c2));
    // point-Hessian vectors (computePointDerivatives, kernel.cpp:523-558):
    // h33 = (0, a2, a3), h34 = (0, b2, b3), h35 = (0, c2, c3), h44 = d,
    // h45 = e, h55 = f
    const float *h = ang + 24;
    const float h33y = dot3f(x0, x1, x2, h + 0), h33z = dot3f(x0, x1, x2, h + 3);
    const float h34y = dot3f(x0, x1, x2, h + 6), h34z = dot3f(x0, x1, x2, h + 9);
    const float h35y = dot3f(x0, x1, x2, h + 12), h35z = dot3f(x0, x1, x2, h + 15);
    const float h44x = dot3f(x0, x1, x2, h + 18), h44y = dot3f(x0, x1, x2, h + 21), h44z = dot3f(x0, x1, x2, h + 24);
    const float h45x = dot3f(x0, x1, x2, h + 27), h45y = dot3f(x0, x1, x2, h + 30), h45z = dot3f(x0, x1, x2, h + 33);
    const float h55x = dot3f(x0, x1, x2, h + 36), h55y = dot3f(x0, x1, x2, h + 39), h55z = dot3f(x0, x1, x2, h + 42);
    float *R = acc + 28 * stride;
    if (compat) {
        // R[a][b] = J_{3+a} . (Q h_{3+a,3+b})
        float t0, t1, t2;
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, 0.0f, h33y, h33z, t0, t1, t2);
        R[0] += fmaf(J13, t1, J23 * t2);
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, 0.0f, h34y, h34z, t0, t1, t2);
        R[1 * stride] += fmaf(J13, t1, J23 * t2);
        R[3 * stride] += fmaf(J04, t0, fmaf(J14, t1, J24 * t2));
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, 0.0f, h35y, h35z, t0, t1, t2);
        R[2 * stride] += fmaf(J13, t1, J23 * t2);
        R[6 * stride] += fmaf(J05, t0, fmaf(J15, t1, J25 * t2));
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, h44x, h44y, h44z, t0, t1, t2);
        R[4 * stride] += fmaf(J04, t0, fmaf(J14, t1, J24 * t2));
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, h45x, h45y, h45z, t0, t1, t2);
        R[5 * stride] += fmaf(J04, t0, fmaf(J14, t1, J24 * t2));
        R[7 * stride] += fmaf(J05, t0, fmaf(J15, t1, J25 * t2));
        sym_mul(F.q00, F.q01, F.q02, F.q11, F.q12, F.q22, h55x, h55y, h55z, t0, t1, t2);
        R[8 * stride] += fmaf(J05, t0, fmaf(J15, t1, J25 * t2));
    } else {
        // R[a][b] = U . h_{3+a,3+b}, a <= b
        R[0] += fmaf(F.u1, h33y, F.u2 * h33z);
        R[1 * stride] += fmaf(F.u1, h34y, F.u2 * h34z);
        R[2 * stride] += fmaf(F.u1, h35y, F.u2 * h35z);
        R[4 * stride] += fmaf(F.u0, h44x, fmaf(F.u1, h44y, F.u2 * h44z));
        R[5 * stride] += fmaf(F.u0, h45x, fmaf(F.u1, h45y, F.u2 * h45z));
        R[8 * stride] += fmaf(F.u0, h55x, fmaf(F.u1, h55y, F.u2 * h55z));
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

// Pairs with a flagged voxel queued by the FP32 pass: (alignment, point,
// slot).  The point is transformed and its per-point terms recomputed exactly
// as the FP32 pass does, then the pair is evaluated in FP64.
__global__ void flagged_kernel(const __grid_constant__ EvalArgs args) {
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
            px = transform_row(st.T, x.x, x.y, x.z);
            py = transform_row(st.T + 4, x.x, x.y, x.z);
            pz = transform_row(st.T + 8, x.x, x.y, x.z);
        }
        float t[kTerms];
        for (int k = 0; k < 8; ++k) t[k] = dot3f(x.x, x.y, x.z, st.angf + 3 * k);
        for (int k = 0; k < 15; ++k) t[8 + k] = dot3f(x.x, x.y, x.z, st.angf + 24 + 3 * k);
        const float4 hi = args.grid.vox32[3 * (size_t)e.z];
        const float4 lo = args.grid.vox32[3 * (size_t)e.z + 1];
        pair_fp64_flagged(args.exc + (size_t)e.x * kPartial, t, __fsub_rn(__fsub_rn(px, hi.x), lo.x),
                          __fsub_rn(__fsub_rn(py, hi.y), lo.y), __fsub_rn(__fsub_rn(pz, hi.z), lo.z),
                          args.grid.icov64 + 9 * (size_t)e.z, args.d1, args.d2, hess, args.compat != 0);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && n > args.flag_cap) atomicOr(args.flag_overflow, 1);
}

// Dynamic shared memory of the FP32 kernel (W warps).
// A warp with more pairs than kDenseThreshold in one collect call evaluates
// them per point; fewer go to its ring of deferred pairs.  The ring holds
// fewer than 32 pairs between calls and receives at most kDenseThreshold, so
// kDefer >= 31 + kDenseThreshold; 64 keeps the 128-thread block at 35.7 KB of
// shared memory, so that 6 blocks fit on an SM.
constexpr int kDefer = 64;            // per-warp ring of deferred pairs (power of two)
constexpr int kDenseThreshold = 32;
static_assert(kDefer >= 31 + kDenseThreshold, "the deferred ring must hold a collect call's pairs");

template <int W>
struct F32Smem {
    float acc[kAcc][W * 32];         // per-lane sums of the current alignment run
    unsigned own[W][kOwn][32];       // each lane's accepted pairs of the current tile
    uint2 defer[W][kDefer];          // deferred pairs: (slot << 6 | flag << 5, point index)
};

// Block-wide reduction of the per-lane FP32 sums of one chunk into the
// chunk's FP64 partial; resets the sums.  Warp w reduces the values w,
// w + W, ...: each lane adds W of the block's lane sums in FP64 (conflict-free
// rows of shared memory), then the warp adds its 32 lane sums with a fixed
// shuffle tree, also in FP64 (B200 issues FP64 adds at half the FP32 rate, and
// the sums of FP32 values stay exact or nearly so).  Fixed order, so the
// result does not depend on timing.  A chunk in which no warp found a pair
// writes its zeros directly.
template <int W>
__device__ void reduce_run(F32Smem<W> &sm, double *s_tot, const unsigned *s_pairs, double *out, double kR,
                           bool compat) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    unsigned np = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) np += s_pairs[w];
    if (np == 0) {  // block-uniform
        if (threadIdx.x < kPartial) out[threadIdx.x] = 0.0;
        return;
    }
    // (not unrolled: the unrolled loop adds ~11 KB of code to a kernel whose hot
    // loop is already larger than the instruction cache)
#pragma unroll 1
    for (int k = warp; k < kAcc; k += W) {
        double sum = 0.0;
#pragma unroll
        for (int r = 0; r < W; ++r) {
            const float v = sm.acc[k][32 * r + lane];
            sm.acc[k][32 * r + lane] = 0.0f;
            sum += (double)v;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(kFull, sum, o);
        if (lane == 0) s_tot[k] = sum;
    }
    __syncthreads();
    if (threadIdx.x < kPartial) {
        const int k = threadIdx.x;
        double v;
        if (k < 7)
            v = s_tot[k];
        else if (k < 43)
            v = h_entry(s_tot, (k - 7) / 6, (k - 7) % 6, kR, compat);
        else
            v = (double)np;
        out[k] = v;
    }
}

// Per-warp context of the pair evaluation.
struct WarpPairs {
    const EvalArgs *args;
    const GridDev *grid;
    const float *T;      // the alignment's transform (shared memory)
    const float *ang;    // its FP32 angle terms (shared memory)
    float *acc;          // this lane's accumulators, stride = block size
    int stride;
    int align;
    float d1, d2;
    bool hess;
};

// Queues a pair with a flagged voxel for flagged_kernel (FP64).
__device__ __forceinline__ void queue_flagged(const EvalArgs &args, int align, int point, int slot) {
    const unsigned q = atomicAdd(args.flag_n, 1u);
    if (q < args.flag_cap) args.flag_q[q] = make_int4(align, point, slot, 0);
}

// x' = x_trans - mean (kernel.cpp:692-694) from the (hi, lo) float split of
// the FP64 mean, and the pair's sums.
__device__ __forceinline__ void add_pair(const WarpPairs &P, PairSums &F, int slot, float px, float py, float pz) {
    const GridDev &g = *P.grid;
    const float4 *r = g.vox32 + 3 * slot;  // one 48-byte record
    const float4 hi = __ldg(r), lo = __ldg(r + 1), cc = __ldg(r + 2);
    const float p0 = __fsub_rn(__fsub_rn(px, hi.x), lo.x);
    const float p1 = __fsub_rn(__fsub_rn(py, hi.y), lo.y);
    const float p2 = __fsub_rn(__fsub_rn(pz, hi.z), lo.z);
    pair_sums(F, p0, p1, p2, hi.w, lo.w, cc.x, cc.y, cc.z, cc.w, P.d1, P.d2, P.hess);
}

// The evaluation steps after one collect call of a warp: first the dense
// step (dense: each lane sums its own pairs own[0..c) and contracts them once
// with its point), then full rounds of 32 deferred pairs from the warp's ring
// (one pair per lane: the lane reloads the pair's point, transforms it again
// with the same float operations and contracts the single pair), and, when
// `flush` is set (the chunk's last collect call), the ring's remainder.  Both
// kinds share this one loop, so the pair sums and the contraction are inlined
// once in the kernel (a smaller instruction footprint).  Pairs with a flagged
// voxel are queued for flagged_kernel instead.
template <bool COMPAT>
__device__ __forceinline__ void eval_steps(const WarpPairs &P, const unsigned (*own)[32], const uint2 *ring,
                                           unsigned &head, unsigned tail, bool dense, bool flush, int c, int i,
                                           float4 x, float px, float py, float pz) {
    const int lane = threadIdx.x & 31;
    for (;;) {
        int cnt = 0, pi = i;
        float4 xe = x;
        float ex = px, ey = py, ez = pz;
        bool from_ring = false;
        unsigned rcode = 0;
        if (dense) {
            dense = false;
            cnt = c;
        } else {
            const unsigned avail = tail - head;
            if (avail == 0u || (avail < 32u && !flush)) break;
            const int take = avail < 32u ? (int)avail : 32;
            __syncwarp();
            from_ring = true;
            if (lane < take) {
                const uint2 d = ring[(head + lane) & (kDefer - 1)];
                rcode = d.x;
                pi = (int)d.y;
                cnt = 1;
                xe = __ldg(P.args->points + pi);
                if (P.args->trans) {
                    const float4 y = __ldg(P.args->trans + pi);
                    ex = y.x; ey = y.y; ez = y.z;
                } else {
                    ex = transform_row(P.T, xe.x, xe.y, xe.z);
                    ey = transform_row(P.T + 4, xe.x, xe.y, xe.z);
                    ez = transform_row(P.T + 8, xe.x, xe.y, xe.z);
                }
            }
            head += (unsigned)take;
        }
        PairSums F;
        zero(F);
        const int maxc = __reduce_max_sync(kFull, cnt);
        for (int k = 0; k < maxc; ++k) {
            if (k < cnt) {
                const unsigned code = from_ring ? rcode : own[k][lane];
                const int slot = (int)(code >> 6);
                if (code & 32u)
                    queue_flagged(*P.args, P.align, pi, slot);
                else
                    add_pair(P, F, slot, ex, ey, ez);
            }
        }
        if (cnt > 0 && !(from_ring && (rcode & 32u)))
            contract_add(F, xe.x, xe.y, xe.z, P.ang, P.acc, P.stride, P.d2, P.hess, COMPAT);
    }
}

// The chunks of the alignments that ask for an evaluation, in a list the FP32
// pass hands out (warp-aggregated appends; the order of the list does not
// change any result, since each chunk writes its own partial slot).
__global__ void active_chunks_kernel(const __grid_constant__ EvalArgs args) {
    const int nc = *args.num_chunks;
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x; base < nc; base += gridDim.x * blockDim.x) {
        const int c = base + threadIdx.x;
        const bool act = c < nc && args.states[args.chunks[c].align].eval_mode != kEvalNone;
        const unsigned bal = __ballot_sync(0xffffffffu, act);
        int at = 0;
        if (lane == 0 && bal) at = atomicAdd(args.num_active, __popc(bal));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (act) args.active_chunks[at + __popc(bal & ((1u << lane) - 1u))] = c;
    }
}

// COMPAT: the reference's Hessian form and pose build (else corrected); WIN: the
// map has a probe-window table (the neighbour search compiles only the paths it
// can take, a smaller instruction footprint).
template <int TILE, int MINB, bool COMPAT, bool WIN>
__global__ void __launch_bounds__(TILE, MINB) derivative_f32_kernel(const __grid_constant__ EvalArgs args) {
    constexpr int kW = TILE / 32;
    static_assert(TILE >= kPartial, "the partial is written by one thread per entry");
    __shared__ float s_T[12];
    __shared__ float s_ang[kAngle];
    __shared__ int s_mode;
    __shared__ double s_tot[kAcc];
    __shared__ unsigned s_pairs[kW];  // pairs each warp found in the current chunk
    __shared__ int s_chunk[2];
    // per-warp work counters (points, tiles, probes, occupied probes, pairs), kept
    // only when the caller asked for counters (in shared memory: no registers)
    __shared__ unsigned long long s_work[kW][5];
    extern __shared__ __align__(16) unsigned char s_dyn[];
    F32Smem<kW> &sm = *reinterpret_cast<F32Smem<kW> *>(s_dyn);

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr bool compat = COMPAT;
    const GridDev &grid = args.grid;
    unsigned (*own)[32] = sm.own[warp];
    uint2 *ring = sm.defer[warp];

    WarpPairs P;
    P.args = &args;
    P.grid = &grid;
    P.T = s_T;
    P.ang = s_ang;
    P.acc = &sm.acc[0][threadIdx.x];
    P.stride = TILE;
    P.d1 = (float)args.d1;
    P.d2 = (float)args.d2;

    const int nc = args.num_active ? *args.num_active : *args.num_chunks;
    for (int k = 0; k < kAcc; ++k) P.acc[k * TILE] = 0.0f;
    if (lane == 0) s_pairs[warp] = 0;
    if (lane == 0)
        for (int q = 0; q < 5; ++q) s_work[warp][q] = 0;
    unsigned head = 0, tail = 0;  // deferred ring of this warp (warp-uniform)
    int parity = 0;

    // Chunks are handed out dynamically (one atomic per chunk), so blocks
    // finish together however uneven the alignments are.  A chunk's partial
    // sums depend only on its own tiles, so results do not depend on which
    // block takes which chunk.  (No block takes more than nc chunks; the
    // bound only guards against a corrupted counter.)
    for (int it = 0; it <= nc; ++it) {
        if (threadIdx.x == 0) {
            const int k = atomicAdd(args.work_counter, 1);
            s_chunk[parity] = k < nc ? (args.active_chunks ? args.active_chunks[k] : k) : -1;
        }
        __syncthreads();
        const int chunk = s_chunk[parity];
        parity ^= 1;
        if (chunk < 0) break;
        const Chunk ck = args.chunks[chunk];
        const AlignState *st = args.states + ck.align;
        if (threadIdx.x == 0) s_mode = st->eval_mode;
        if (threadIdx.x < 12) s_T[threadIdx.x] = st->T[threadIdx.x];
        for (int k = threadIdx.x; k < kAngle; k += TILE) s_ang[k] = st->angf[k];
        __syncthreads();
        const int mode = s_mode;
        if (mode == kEvalNone) continue;  // s_mode is rewritten only after the next chunk's barrier
        P.align = ck.align;
        P.hess = mode != kEvalGradient;
        for (int ti = ck.first; ti < ck.end; ++ti) {
            const Tile tile = args.tiles[ti];
            const int i = tile.start + threadIdx.x;
            const bool valid = i < tile.end;
            const float4 x = valid ? args.points[i] : make_float4(0.f, 0.f, 0.f, 0.f);
            // transformPointCloud (kernel.cpp:397-400), float, left to right
            float px, py, pz;
            if (args.trans) {
                const float4 y = valid ? args.trans[i] : make_float4(0.f, 0.f, 0.f, 0.f);
                px = y.x; py = y.y; pz = y.z;
            } else {
                px = transform_row(s_T, x.x, x.y, x.z);
                py = transform_row(s_T + 4, x.x, x.y, x.z);
                pz = transform_row(s_T + 8, x.x, x.y, x.z);
            }
            unsigned n_probe = 0, n_occ = 0, n_pair = 0;
            int resume = 0;
            do {
                __syncwarp();
                OwnSink sink{own, 0};
                collect_pairs<OwnSink, WIN ? kProbeWindows : kProbeDenseIndex>(grid, px, py, pz, valid, sink, n_probe,
                                                                               n_occ, resume);
                __syncwarp();
                const int c = sink.c;
                n_pair += c;
                const int n = __reduce_add_sync(kFull, c);
                // dense (more than kDenseThreshold pairs in the warp): per point;
                // sparse: into the ring, evaluated in rounds of 32
                const bool dense = n > kDenseThreshold;
                if (!dense && n > 0) {
                    int pre = c;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int v = __shfl_up_sync(kFull, pre, o);
                        if (lane >= o) pre += v;
                    }
                    pre -= c;
                    for (int k = 0; k < c; ++k)
                        ring[(tail + pre + k) & (kDefer - 1)] = make_uint2(own[k][lane] & ~31u, (unsigned)i);
                    tail += n;
                }
                // the chunk's last collect call also empties the ring
                const bool flush = resume < 0 && ti + 1 == ck.end;
                eval_steps<COMPAT>(P, own, ring, head, tail, dense, flush, c, i, x, px, py, pz);
            } while (resume >= 0);
            // per-warp work counters: the pairs feed the partial's count; the
            // others only when the caller asked for counters
            n_pair = __reduce_add_sync(kFull, n_pair);
            if (lane == 0) s_pairs[warp] += n_pair;
            if (args.counters) {
                const unsigned probes = __reduce_add_sync(kFull, n_probe);
                const unsigned occupied = __reduce_add_sync(kFull, n_occ);
                if (lane == 0) {
                    s_work[warp][0] += (unsigned)(tile.end - tile.start);
                    s_work[warp][1] += 1;
                    s_work[warp][2] += probes;
                    s_work[warp][3] += occupied;
                    s_work[warp][4] += n_pair;
                }
            }
        }
        // end of the chunk (the last collect call emptied the ring): the block's sums
        head = tail = 0;
        reduce_run<kW>(sm, s_tot, s_pairs, args.partials + (size_t)ck.slot * kPartial, compat ? -args.d2 : 1.0, compat);
        __syncthreads();
        if (lane == 0) s_pairs[warp] = 0;
    }
    if (args.counters && lane == 0 && s_work[warp][1]) {
        if (warp == 0) {  // every warp of the block saw the same tiles
            atomicAdd(&args.counters->points, s_work[warp][0]);
            atomicAdd(&args.counters->tiles, s_work[warp][1]);
        }
        atomicAdd(&args.counters->probes, s_work[warp][2]);
        atomicAdd(&args.counters->occupied_probes, s_work[warp][3]);
        atomicAdd(&args.counters->pairs, s_work[warp][4]);
    }
}

template <int TILE, int MINB>
cudaError_t prepare_one() {
    const int bytes = (int)sizeof(F32Smem<TILE / 32>);
    const void *k[4] = {(const void *)derivative_f32_kernel<TILE, MINB, true, true>,
                        (const void *)derivative_f32_kernel<TILE, MINB, true, false>,
                        (const void *)derivative_f32_kernel<TILE, MINB, false, true>,
                        (const void *)derivative_f32_kernel<TILE, MINB, false, false>};
    cudaError_t e = cudaSuccess;
    for (const void *f : k) {
        const cudaError_t r = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (r != cudaSuccess) e = r;
    }
    return e;
}

template <int TILE, int MINB>
void launch_one(const EvalArgs &args, int blocks, cudaStream_t st) {
    const size_t smem = sizeof(F32Smem<TILE / 32>);
    const bool win = args.grid.win_off != nullptr;
    if (args.compat) {
        if (win)
            derivative_f32_kernel<TILE, MINB, true, true><<<blocks, TILE, smem, st>>>(args);
        else
            derivative_f32_kernel<TILE, MINB, true, false><<<blocks, TILE, smem, st>>>(args);
    } else {
        if (win)
            derivative_f32_kernel<TILE, MINB, false, true><<<blocks, TILE, smem, st>>>(args);
        else
            derivative_f32_kernel<TILE, MINB, false, false><<<blocks, TILE, smem, st>>>(args);
    }
}

}  // namespace

const DerivVariant kDerivVariants[kNumDerivVariants] = {
    {256, 2}, {256, 1}, {128, 4}, {128, 3}, {256, 3}, {128, 5}, {128, 6},
};

int prepare_derivatives() {
    cudaError_t e = cudaSuccess, r;
    if ((r = prepare_one<256, 2>()) != cudaSuccess) e = r;
    if ((r = prepare_one<256, 1>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 4>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 3>()) != cudaSuccess) e = r;
    if ((r = prepare_one<256, 3>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 5>()) != cudaSuccess) e = r;
    if ((r = prepare_one<128, 6>()) != cudaSuccess) e = r;
    return (int)e;
}

int launch_derivatives(const EvalArgs &args, int precision, int variant, int sms, cudaStream_t st) {
    if (args.max_tiles <= 0) return 0;
    if (precision == 1) return launch_derivatives_f64(args, sms, st);
    if (variant < 0 || variant >= kNumDerivVariants) variant = 0;
    const DerivVariant v = kDerivVariants[variant];
    if (args.tile_size != v.tile) return (int)cudaErrorInvalidValue;
    long long want = (long long)sms * v.min_blocks;
    int blocks = (int)(want < args.max_tiles ? want : args.max_tiles);
    cudaMemsetAsync(args.flag_n, 0, sizeof(unsigned), st);
    cudaMemsetAsync(args.work_counter, 0, sizeof(int), st);
    if (args.active_chunks) {
        cudaMemsetAsync(args.num_active, 0, sizeof(int), st);
        active_chunks_kernel<<<sms * 4, 256, 0, st>>>(args);
    }
    switch (variant) {
        case 0: launch_one<256, 2>(args, blocks, st); break;
        case 1: launch_one<256, 1>(args, blocks, st); break;
        case 2: launch_one<128, 4>(args, blocks, st); break;
        case 3: launch_one<128, 3>(args, blocks, st); break;
        case 5: launch_one<128, 5>(args, blocks, st); break;
        case 6: launch_one<128, 6>(args, blocks, st); break;
        default: launch_one<256, 3>(args, blocks, st); break;
    }
    flagged_kernel<<<sms, 128, 0, st>>>(args);
    return (int)cudaGetLastError();
}

}  // namespace ndt
