// The FP64 derivative pass (precision = 1): every (point, voxel) pair is
// evaluated with the reference's literal FP64 expressions (updateDerivatives /
// updateHessian, src/CPU/ndt_mapping/kernel.cpp:438-493, 604-649, compat) or the
// Magnusson eq. 6.13 Hessian (corrected), and accumulated in FP64.  The
// neighbour search is the exact one of probe.cuh.  Compiled without
// floating-point contraction, like the reference's x86-64 code.
#include <cuda_runtime.h>
#include <stdint.h>

#include "derivatives.h"
#include "ndt_math.cuh"
#include "probe.cuh"

namespace ndt {

namespace {

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

__global__ void __launch_bounds__(kTile64, 1) derivative_f64_kernel(const __grid_constant__ EvalArgs args) {
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
            px = transform_row(s_T, x.x, x.y, x.z);
            py = transform_row(s_T + 4, x.x, x.y, x.z);
            pz = transform_row(s_T + 8, x.x, x.y, x.z);
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
        int resume = 0;
        do {
            __syncwarp();
            ListSink sink{list, 0};
            collect_pairs(grid, px, py, pz, valid, sink, n_probe, n_occ, resume);
            __syncwarp();
            consume(sink.n);
        } while (resume >= 0);
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

}  // namespace

int launch_derivatives_f64(const EvalArgs &args, int sms, cudaStream_t st) {
    if (args.tile_size != kTile64) return (int)cudaErrorInvalidValue;
    int blocks = sms < args.max_tiles ? sms : args.max_tiles;
    derivative_f64_kernel<<<blocks, kTile64, 0, st>>>(args);
    return (int)cudaGetLastError();
}

}  // namespace ndt
