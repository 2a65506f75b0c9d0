// The FP32 derivative pass: score, gradient and Hessian of the NDT
// objective for a batch of alignments (computeDerivatives / computeHessian,
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
// Per point (one thread): the float transform and the reference's neighbour
// search of probe.cuh (exact: the accepted pairs are the reference's); the
// accepted pairs are compacted per warp in shared memory and evaluated one per
// lane, so the per-pair work is balanced across lanes.
// Per pair: x' from the (hi, lo) float split of the FP64 mean, q = C x', xCx,
// e = exp(-d2 xCx / 2), the validity test of :456, gradient a_i = x'^T C J_i
// and the Hessian split as
//   H_ij = S_ij + k R_ij,  S_ij = w (-d2 a_i a_j + J_j^T C J_i)   (i <= j)
//   compat:    R_ij = w a_i b_ij, k = -d2  (the reference's :486-488 form)
//   corrected: R_ij = w b_ij,     k = 1    (Magnusson eq. 6.13)
// with b_ij = x'^T C H_ij (nonzero for i, j >= 3 only).  Voxels flagged by the
// grid build (inverse-covariance entries non-finite or beyond 1e30) are queued
// and evaluated in FP64 by flagged_kernel, so that infinities and NaNs
// propagate as in the reference.
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
            px = transform_row(st.T, x.x, x.y, x.z);
            py = transform_row(st.T + 4, x.x, x.y, x.z);
            pz = transform_row(st.T + 8, x.x, x.y, x.z);
        }
        float t[kTerms];
        for (int k = 0; k < 8; ++k) t[k] = dot3f(x.x, x.y, x.z, st.angf + 3 * k);
        for (int k = 0; k < 15; ++k) t[8 + k] = dot3f(x.x, x.y, x.z, st.angf + 24 + 3 * k);
        const float4 hi = args.grid.mean_hi[e.z];
        const float4 lo = args.grid.mean_lo[e.z];
        pair_fp64_flagged(args.exc + (size_t)e.x * kPartial, t, __fsub_rn(__fsub_rn(px, hi.x), lo.x),
                          __fsub_rn(__fsub_rn(py, hi.y), lo.y), __fsub_rn(__fsub_rn(pz, hi.z), lo.z),
                          args.grid.icov64 + 9 * (size_t)e.z, args.d1, args.d2, hess, args.compat != 0);
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
};

// Block-wide reduction of the per-lane sums of one alignment run, written as
// the FP64 partial of the run's first tile; resets the sums.  Warp w reduces
// the values w, w + W, ...: each lane sums W of the block's lane sums
// (conflict-free rows of shared memory) with TwoSum compensation, then the
// warp combines its 32 (sum, error) pairs with shuffles.  Fixed order, so the
// result does not depend on timing.
template <int W>
__device__ void reduce_run(F32Smem<W> &sm, double *s_tot, const unsigned (*s_cnt)[3], double *out, double kR,
                           bool compat) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    for (int k = warp; k < kAcc; k += W) {
        float s = 0.0f, e = 0.0f;
#pragma unroll
        for (int r = 0; r < W; ++r) {
            const float v = sm.acc[k][32 * r + lane];
            sm.acc[k][32 * r + lane] = 0.0f;
            float t, err;
            two_sum(s, v, t, err);
            s = t;
            e = __fadd_rn(e, err);
        }
        warp_two_sum_reduce(s, e);
        if (lane == 0) s_tot[k] = (double)s + (double)e;
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
    const int K = args.chunk_tiles;
    for (int k = 0; k < kAcc; ++k) acc[k * TILE] = 0.0f;
    if (lane == 0) s_cnt[warp][0] = s_cnt[warp][1] = s_cnt[warp][2] = 0;
    unsigned long long blk_probe = 0, blk_occ = 0, blk_pair = 0, blk_pts = 0, blk_tiles = 0;
    int cur = -1, run_first = -1, mode = kEvalNone;
    double *exc = nullptr;
    __shared__ int s_chunk[2];
    int parity = 0;

    // Chunks of K consecutive tiles are handed out dynamically (one atomic per
    // chunk), so blocks finish together however uneven the alignments are.  A
    // chunk's partial sums depend only on its tiles, so results do not depend
    // on which block takes which chunk.
    for (;;) {
        if (threadIdx.x == 0) s_chunk[parity] = atomicAdd(args.work_counter, 1);
        __syncthreads();
        const int chunk = s_chunk[parity];
        parity ^= 1;
        const int t_begin = chunk * K;
        if (t_begin >= nt) break;
        const int t_end = min(nt, t_begin + K);
    for (int ti = t_begin; ti < t_end; ++ti) {
        const Tile tile = args.tiles[ti];
        if (tile.align != cur || ti == t_begin) {
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
            px = transform_row(s_T, x.x, x.y, x.z);
            py = transform_row(s_T + 4, x.x, x.y, x.z);
            pz = transform_row(s_T + 8, x.x, x.y, x.z);
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
                const float p0 = __fsub_rn(__fsub_rn(xts[0][owner], hi.x), lo.x);
                const float p1 = __fsub_rn(__fsub_rn(xts[1][owner], hi.y), lo.y);
                const float p2 = __fsub_rn(__fsub_rn(xts[2][owner], hi.z), lo.z);
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
        // the run of this chunk ends with the chunk
        if (cur >= 0 && mode != kEvalNone) {
            reduce_run<kW>(sm, s_tot, s_cnt, args.partials + (size_t)run_first * kPartial, kR, compat);
            __syncthreads();
            if (lane == 0) s_cnt[warp][0] = s_cnt[warp][1] = s_cnt[warp][2] = 0;
        }
        cur = -1;
    }
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
    if (precision == 1) return launch_derivatives_f64(args, sms, st);
    if (variant < 0 || variant >= kNumDerivVariants) variant = 0;
    const DerivVariant v = kDerivVariants[variant];
    if (args.tile_size != v.tile) return (int)cudaErrorInvalidValue;
    long long want = (long long)sms * v.min_blocks;
    int blocks = (int)(want < args.max_tiles ? want : args.max_tiles);
    cudaMemsetAsync(args.flag_n, 0, sizeof(unsigned), st);
    cudaMemsetAsync(args.work_counter, 0, sizeof(int), st);
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
