// Learned initial pose: a point-feature network (PointNet-style) that reads a
// scan transformed by its guess and proposes a pose correction, which the
// plain NDT then refines.  Forward and backward kernels of our own:
//
//   per point  u (3)  -> h1 = ReLU(W1 u + b1)        (64,  FP32, CUDA cores)
//              h1     -> z2 = W2 bf16(h1) + b2       (128, BF16 x BF16 -> FP32 on
//                                                     the tensor cores: tcgen05.mma,
//                                                     accumulator in TMEM)
//              h2 = ReLU(z2); g = max over points (with the argmax point)
//   per scan   g (128) -> h3 = ReLU(W3 g + b3) (64) -> y = W4 h3 + b4 (6)
//              (head_tc_kernel: 128 scans per CTA, both products on the
//              tensor cores)
//
// The network input u is the scan point transformed by the guess into the map
// frame, centred and scaled by the map's extent (u = (T_guess x - c) / s).
// y is the pose correction in units of `delta_scale` (see ndt_b200.h).
//
// Backward: every product of the head's backward is a GEMM over the batch and
// runs on the tensor cores in head_tc_kernel (dH3 = dY W4, dG = dH3 W3 and the
// weight gradients dH3^T G, dY^T H3 summed over each 128-scan tile).  The
// max-pool routes the gradient of channel c of scan b to one point (its
// argmax), so the shared layers' gradient touches at most 128 points per scan
// with a different point per channel: a gather, not a GEMM, computed on CUDA
// cores per scan (shared_bwd_kernel) with the same BF16 operands the forward
// used (h1 and W2 rounded to BF16).  Gradients are summed over the batch in a
// fixed order (deterministic) and applied with Adam to FP32 master weights; W2
// is then re-packed to BF16.
//
// Tensor-core tile of the shared layer (one CTA of 128 threads per scan, 128
// sampled points per tile): A = W2 [128 outputs x 64] and B = bf16(h1) [128
// points x 64], both K-major in shared memory in the interleaved (no-swizzle)
// core-matrix layout: element (r, k) at (r / 8) * 1024 + (k / 8) * 128 +
// (r % 8) * 16 + (k % 8) * 2 bytes, so a descriptor's leading byte offset
// (next 8 K-elements) is 128 B and its stride byte offset (next 8 rows) is
// 1024 B (K * 16 B in general, opk()).  Four MMAs of K = 16 (start addresses
// 256 B apart) give D = A B^T (channels x points), 128 x 128
// FP32 in 128 TMEM columns; thread c reads its channel's row (TMEM lane c)
// back with tcgen05.ld and keeps the running maximum over the points.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ndt_b200.h"
#include "mlp_internal.h"
#include "umma_desc.h"

namespace pn {

constexpr int kH1 = 64, kH2 = 128, kH3 = 64, kOut = 6;
// FP32 weight blob layout
constexpr int oW1 = 0, oB1 = oW1 + kH1 * 3, oW2 = oB1 + kH1, oB2 = oW2 + kH2 * kH1, oW3 = oB2 + kH2,
              oB3 = oW3 + kH3 * kH2, oW4 = oB3 + kH3, oB4 = oW4 + kOut * kH3, kNumW = oB4 + kOut;
constexpr int kTileRows = 128;                  // points per tensor-core tile (MMA M)
constexpr int kOperandBytes = kTileRows * kH1 * 2;  // 16 KB per BF16 operand
constexpr uint32_t kTmemCols = 128;             // FP32 accumulator columns (MMA N)

// Byte offset of element (r, k) in an interleaved K-major operand (64 K).
__host__ __device__ __forceinline__ uint32_t op_offset(int r, int k) {
    return (uint32_t)((r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long pack_max(float v, int idx) {
    // v >= 0 (after ReLU): its bits order like the value; ties keep the smaller index
    return ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)(0xffffffffu - (unsigned)idx);
}

// Map-frame feature of point i of the scan: u = (T x - c) * inv_s.
__device__ __forceinline__ void point_feature(const float *T, float4 x, const Norm &nm, float u[3]) {
    const float px = T[0] * x.x + T[1] * x.y + T[2] * x.z + T[3];
    const float py = T[4] * x.x + T[5] * x.y + T[6] * x.z + T[7];
    const float pz = T[8] * x.x + T[9] * x.y + T[10] * x.z + T[11];
    u[0] = (px - nm.cx) * nm.inv_s;
    u[1] = (py - nm.cy) * nm.inv_s;
    u[2] = (pz - nm.cz) * nm.inv_s;
}

// Index of the j-th of P sampled points of an n-point scan (evenly strided).
__device__ __forceinline__ int sample_index(int j, int P, int n) { return (int)(((long long)j * n) / P); }

// ---------------------------------------------------------------------------
// W2 (FP32 [128][64]) -> BF16 interleaved operand.
__global__ void pack_w2_kernel(const float *__restrict__ w, uint8_t *__restrict__ w2op) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= kH2 * kH1) return;
    const int r = t / kH1, k = t % kH1;
    *reinterpret_cast<__nv_bfloat16 *>(w2op + op_offset(r, k)) = __float2bfloat16_rn(w[oW2 + t]);
}

// ---------------------------------------------------------------------------
// Shared layers + max-pool, one CTA per scan.  gmax[b][c] = packed (max
// value, ~argmax sample index); err is set when an mbarrier wait gives up.
struct PointArgs {
    const float4 *points;
    const int *offsets;
    const float *guesses;      // B x 16
    const float *w;            // FP32 weights
    const uint8_t *w2op;       // BF16 W2 operand (16 KB)
    unsigned long long *gmax;  // B x 128
    int *err;
    Norm nm;
    int B;
    int scans;                 // candidate b reads scan b % scans (several starts of one scan)
    int max_points;
    unsigned wait_limit;       // polls of the MMA barrier before the wait gives up
};

__global__ void __launch_bounds__(128, 1) point_kernel(const __grid_constant__ PointArgs a) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sA = smem;                                  // 16 KB
    uint8_t *sB = smem + kOperandBytes;                  // 16 KB
    float *sW1 = reinterpret_cast<float *>(smem + 2 * kOperandBytes);  // 192 + 64 (b1) + 128 (b2)
    float *sB1 = sW1 + kH1 * 3;
    float *sB2 = sB1 + kH1;
    uint64_t *sBar = reinterpret_cast<uint64_t *>(sB2 + kH2);  // 8-byte aligned (offset 32768 + 1536)
    uint32_t *sTmem = reinterpret_cast<uint32_t *>(sBar + 1);
    __shared__ float sT[12];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int b = blockIdx.x;
    if (b >= a.B) return;  // (grid = B: never taken)
    const int sb = b % a.scans;
    const int start = a.offsets[sb], n = a.offsets[sb + 1] - start;
    const int P = n < a.max_points ? n : a.max_points;

    // operands and small weights into shared memory
    for (int i = tid; i < kOperandBytes / 16; i += 128)
        reinterpret_cast<uint4 *>(sB)[i] = reinterpret_cast<const uint4 *>(a.w2op)[i];
    for (int i = tid; i < kH1 * 3; i += 128) sW1[i] = a.w[oW1 + i];
    for (int i = tid; i < kH1; i += 128) sB1[i] = a.w[oB1 + i];
    for (int i = tid; i < kH2; i += 128) sB2[i] = a.w[oB2 + i];
    if (tid < 12) sT[tid] = a.guesses[16 * (size_t)b + tid];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(sBar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {  // TMEM: 128 columns for the 128 x 128 FP32 accumulator
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(sTmem)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *sTmem;

    // D = W2 h1^T: 128 channels (TMEM lanes; thread 32 warp + lane owns
    // channel c) x 128 points of the tile (columns).  The max-pool is then a
    // per-thread reduction over its own row; bias and ReLU are monotonic, so
    // they apply once to the final maximum.
    const uint32_t idesc = umma::instr_desc_bf16_f32(kH2, kTileRows);
    const int c = tid;
    float best = -INFINITY;
    int best_j = 0;
    uint32_t phase = 0;
    const int tiles = (P + kTileRows - 1) / kTileRows;
    for (int t = 0; t < tiles; ++t) {
        // layer 1 for this thread's point (sample j = t * 128 + tid), row tid of the h1 operand
        const int j = t * kTileRows + tid;
        const bool valid = j < P;
        float u[3] = {0.f, 0.f, 0.f};
        if (valid) {
            const float4 x = a.points[start + sample_index(j, P, n)];
            point_feature(sT, x, a.nm, u);
        }
#pragma unroll
        for (int kc = 0; kc < kH1 / 8; ++kc) {
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const int k = kc * 8 + e;
                float v = fmaf(sW1[3 * k], u[0], fmaf(sW1[3 * k + 1], u[1], fmaf(sW1[3 * k + 2], u[2], sB1[k])));
                v = valid ? fmaxf(v, 0.0f) : 0.0f;
                h[e] = __float2bfloat16_rn(v);
            }
            *reinterpret_cast<uint4 *>(sA + op_offset(tid, kc * 8)) = *reinterpret_cast<const uint4 *>(h);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (tid == 0) {
#pragma unroll
            for (int kk = 0; kk < kH1 / 16; ++kk) {
                // A = W2 (channels x K), B = h1 (points x K), both K-major
                const uint64_t da = umma::smem_desc_kmajor_interleaved(smem_u32(sB) + kk * 256, 128, 1024);
                const uint64_t db = umma::smem_desc_kmajor_interleaved(smem_u32(sA) + kk * 256, 128, 1024);
                const uint32_t accumulate = kk > 0 ? 1u : 0u;
                const uint32_t no_mask = 0;  // disable-output-lane mask: all lanes written
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(no_mask), "r"(no_mask), "r"(no_mask),
                    "r"(no_mask));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(sBar))
                         : "memory");
        }
        // wait for the MMAs (bounded).  A wait that gives up sets the error
        // flag; the MMAs it gave up on may still be running, so the thread
        // then waits for them with the full limit before the block leaves
        // the tile loop and releases its TMEM.
        bool gave_up = false;
        {
            uint32_t done = 0;
            unsigned it = 0;
            while (!done) {
                if (it++ >= a.wait_limit) {
                    gave_up = true;
                    break;
                }
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.b32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_u32(sBar)), "r"(phase)
                    : "memory");
            }
            if (gave_up) {
                atomicExch(a.err, 1);
                for (unsigned k = 0; k < kWaitLimit && !done; ++k)
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.b32 %0, 1, 0, p;\n\t}\n"
                        : "=r"(done)
                        : "r"(smem_u32(sBar)), "r"(phase)
                        : "memory");
            }
            phase ^= 1u;
        }
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (__syncthreads_or(gave_up)) break;  // the same decision in every thread of the block
        // this channel's 128 values: columns 32 q .. 32 q + 31 = points t * 128 + column
        const int nvalid = min(kTileRows, P - t * kTileRows);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t r[32];
            const uint32_t addr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(32 * q);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
            for (int e = 0; e < 32; ++e) {
                const int col = 32 * q + e;
                const float z = __uint_as_float(r[e]);
                if (col < nvalid && z > best) {  // strict: the smallest index among equal maxima
                    best = z;
                    best_j = t * kTileRows + col;
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // all TMEM reads and operand reads done before the next tile's writes and MMAs
    }
    {
        // g_c = ReLU(max_p z + b2_c); a zero maximum routes no gradient: report sample 0
        float g = P > 0 ? fmaxf(best + sB2[c], 0.0f) : 0.0f;
        const int j = g > 0.0f ? best_j : 0;
        a.gmax[(size_t)b * kH2 + c] = P > 0 ? pack_max(g, j) : 0ull;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// ---------------------------------------------------------------------------
// Head on the tensor cores, 128 scans per CTA (row r of every operand =
// scan r of the tile; invalid rows are zero and contribute nothing):
//   D1 = G  W3^T            G = the max-pooled features (128 x 128), W3 (64 x 128)
//   H3 = ReLU(D1 + b3);     D2 = H3 W4^T (N padded to 16);  Y = D2 + b4
// and, when training (dY = d loss_b / dY = 2 (Y - T) / 6 per scan):
//   D3 = dY W4 -> dH3 = D3 [H3 > 0]                      (K = 16, 6 used)
//   D4 = dH3 W3 -> dG = D4 [G > 0]                        (to the shared layers)
//   D5 = dH3^T G  = this tile's sum over scans of dW3     (M padded to 128)
//   D6 = dY^T H3  = this tile's sum over scans of dW4     (M padded to 128)
// BF16 operands, FP32 accumulators in TMEM (512 columns: D1 0, D2 64, D3 128,
// D4 192, D5 320, D6 448), one elected thread issues the MMAs.  Bias
// gradients are summed over the tile's rows in a fixed order.
constexpr int kOutPad = 16;
constexpr int kHeadPart = kNumW;  // per-CTA partial: the head's weights and biases at their blob offsets

// Byte offset of element (r, k) in a K-major interleaved operand with K columns.
__host__ __device__ __forceinline__ uint32_t opk(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct HeadTcArgs {
    const float *w;
    const unsigned long long *gmax;  // B x 128 (value bits << 32 | ~argmax)
    const float *target;             // B x 6 or null (inference)
    float *y;                        // B x 6 out (may be null)
    float *dg;                       // B x 128 out (training)
    float *loss_scan;                // B out (training)
    float *head_part;                // gridDim.x x kHeadPart out (training)
    int *err;
    int B;
    unsigned wait_limit;
};

// Shared memory of head_tc_kernel (bytes).
constexpr uint32_t hG = 0, hGt = hG + 32768, hW3 = hGt + 32768, hW3t = hW3 + 16384, hH3 = hW3t + 16384,
                   hH3t = hH3 + 16384, hW4 = hH3t + 16384, hW4t = hW4 + 2048, hDY = hW4t + 2048, hDYt = hDY + 4096,
                   hDH3 = hDYt + 32768, hDH3t = hDH3 + 16384, hBar = hDH3t + 32768, hTmem = hBar + 8,
                   kHeadSmem = hTmem + 8;

__device__ __forceinline__ void st_bf16(uint8_t *base, uint32_t off, float v) {
    *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint32_t a_smem, uint32_t b_smem, int K_a, int K_b,
                                         int ksteps, uint32_t idesc, bool accumulate_first) {
    for (int kk = 0; kk < ksteps; ++kk) {
        const uint64_t da = umma::smem_desc_kmajor_interleaved(a_smem + kk * 256, 128, (uint32_t)K_a * 16);
        const uint64_t db = umma::smem_desc_kmajor_interleaved(b_smem + kk * 256, 128, (uint32_t)K_b * 16);
        const uint32_t acc = (kk > 0 || accumulate_first) ? 1u : 0u;
        const uint32_t no_mask = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(no_mask), "r"(no_mask), "r"(no_mask), "r"(no_mask));
    }
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Bounded wait on the MMA barrier (see point_kernel); returns true when any
// thread of the block gave up (the same in every thread).
__device__ bool mma_wait(uint32_t bar, uint32_t &phase, unsigned limit, int *err) {
    bool gave_up = false;
    uint32_t done = 0;
    unsigned it = 0;
    while (!done) {
        if (it++ >= limit) {
            gave_up = true;
            break;
        }
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(phase)
            : "memory");
    }
    if (gave_up) {
        atomicExch(err, 1);
        for (unsigned k = 0; k < kWaitLimit && !done; ++k)
            asm volatile(
                "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(bar), "r"(phase)
                : "memory");
    }
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    return __syncthreads_or(gave_up);
}

// n columns (a multiple of 32) of this thread's TMEM lane, from column c0.
template <int N>
__device__ __forceinline__ void tmem_row(uint32_t tmem, int warp, int c0, float *out) {
#pragma unroll
    for (int q = 0; q < N / 32; ++q) {
        uint32_t r[32];
        const uint32_t addr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(c0 + 32 * q);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
            "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
              "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
              "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 32; ++e) out[32 * q + e] = __uint_as_float(r[e]);
    }
}

__global__ void __launch_bounds__(128, 1) head_tc_kernel(const __grid_constant__ HeadTcArgs a) {
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const int b = blockIdx.x * 128 + tid;
    const bool valid = b < a.B;
    const bool train = a.target != nullptr;
    const float *w = a.w;
    const uint32_t s0 = smem_u32(sm), bar = s0 + hBar;

    // operands: zero the padded ones, then fill
    if (train) {
        for (uint32_t i = tid; i < (32768u + 32768u) / 16; i += 128) {  // dY^T and dH3^T (rows beyond 6 / 64)
            const uint32_t o = (i < 2048u) ? hDYt + 16 * i : hDH3t + 16 * (i - 2048u);
            *reinterpret_cast<uint4 *>(sm + o) = make_uint4(0, 0, 0, 0);
        }
    }
    for (int i = tid; i < kH3 * kH2; i += 128) {  // W3 (64 x 128) and its transpose
        const int j = i / kH2, c = i % kH2;
        const float v = w[oW3 + i];
        st_bf16(sm, hW3 + opk(j, c, kH2), v);
        st_bf16(sm, hW3t + opk(c, j, kH3), v);
    }
    for (int i = tid; i < kOutPad * kH3; i += 128) {  // W4 (6 x 64) padded to 16 rows, and its transpose
        const int o = i / kH3, j = i % kH3;
        const float v = o < kOut ? w[oW4 + o * kH3 + j] : 0.0f;
        st_bf16(sm, hW4 + opk(o, j, kH3), v);
        st_bf16(sm, hW4t + opk(j, o, kOutPad), v);
    }
    float g[kH2];
    {
        const unsigned long long *gm = a.gmax + (size_t)(valid ? b : 0) * kH2;
#pragma unroll 4
        for (int c = 0; c < kH2; ++c) {
            g[c] = valid ? __uint_as_float((unsigned)(gm[c] >> 32)) : 0.0f;
            st_bf16(sm, hG + opk(tid, c, kH2), g[c]);
            st_bf16(sm, hGt + opk(c, tid, 128), g[c]);
        }
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(s0 + hTmem), "r"(512));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *reinterpret_cast<const uint32_t *>(sm + hTmem);
    uint32_t phase = 0;
    bool failed = false;

    // D1 = G W3^T (N = 64, K = 128)
    if (tid == 0) {
        mma_bf16(tmem + 0, s0 + hG, s0 + hW3, kH2, kH2, kH2 / 16, umma::instr_desc_bf16_f32(128, kH3), false);
        mma_commit(bar);
    }
    failed = mma_wait(bar, phase, a.wait_limit, a.err);
    float h3[kH3];
    if (!failed) {
        tmem_row<kH3>(tmem, warp, 0, h3);
#pragma unroll
        for (int j = 0; j < kH3; ++j) {
            h3[j] = valid ? fmaxf(h3[j] + w[oB3 + j], 0.0f) : 0.0f;
            st_bf16(sm, hH3 + opk(tid, j, kH3), h3[j]);
            st_bf16(sm, hH3t + opk(j, tid, 128), h3[j]);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // D2 = H3 W4^T (N = 16, K = 64)
    if (!failed) {
        if (tid == 0) {
            mma_bf16(tmem + 64, s0 + hH3, s0 + hW4, kH3, kH3, kH3 / 16, umma::instr_desc_bf16_f32(128, kOutPad),
                     false);
            mma_commit(bar);
        }
        failed = mma_wait(bar, phase, a.wait_limit, a.err);
    }
    float dy[kOut];
    if (!failed) {
        float d2[32];
        tmem_row<32>(tmem, warp, 64, d2);  // columns 64..95: D2 (16) and unused columns
        float l = 0.0f;
#pragma unroll
        for (int o = 0; o < kOut; ++o) {
            const float yo = d2[o] + w[oB4 + o];
            if (valid && a.y) a.y[(size_t)b * kOut + o] = yo;
            dy[o] = 0.0f;
            if (train && valid) {
                const float d = yo - a.target[(size_t)b * kOut + o];
                l += d * d;
                dy[o] = d * (2.0f / kOut);
            }
        }
        if (train && valid) a.loss_scan[b] = l / kOut;
    }
    if (!train || failed) {
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
        return;
    }
#pragma unroll
    for (int o = 0; o < kOutPad; ++o) st_bf16(sm, hDY + opk(tid, o, kOutPad), o < kOut ? dy[o] : 0.0f);
#pragma unroll
    for (int o = 0; o < kOut; ++o) st_bf16(sm, hDYt + opk(o, tid, 128), dy[o]);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // D3 = dY W4 (N = 64, K = 16)
    if (tid == 0) {
        mma_bf16(tmem + 128, s0 + hDY, s0 + hW4t, kOutPad, kOutPad, 1, umma::instr_desc_bf16_f32(128, kH3), false);
        mma_commit(bar);
    }
    failed = mma_wait(bar, phase, a.wait_limit, a.err);
    float dh3[kH3];
    if (!failed) {
        tmem_row<kH3>(tmem, warp, 128, dh3);
#pragma unroll
        for (int j = 0; j < kH3; ++j) {
            dh3[j] = h3[j] > 0.0f ? dh3[j] : 0.0f;
            st_bf16(sm, hDH3 + opk(tid, j, kH3), dh3[j]);
            st_bf16(sm, hDH3t + opk(j, tid, 128), dh3[j]);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // D4 = dH3 W3 (N = 128, K = 64); D5 = dH3^T G (N = 128, K = 128 scans); D6 = dY^T H3 (N = 64, K = 128)
    if (!failed) {
        if (tid == 0) {
            mma_bf16(tmem + 192, s0 + hDH3, s0 + hW3t, kH3, kH3, kH3 / 16, umma::instr_desc_bf16_f32(128, kH2), false);
            mma_bf16(tmem + 320, s0 + hDH3t, s0 + hGt, 128, 128, 8, umma::instr_desc_bf16_f32(128, kH2), false);
            mma_bf16(tmem + 448, s0 + hDYt, s0 + hH3t, 128, 128, 8, umma::instr_desc_bf16_f32(128, kH3), false);
            mma_commit(bar);
        }
        failed = mma_wait(bar, phase, a.wait_limit, a.err);
    }
    if (!failed) {
        float d4[kH2];
        tmem_row<kH2>(tmem, warp, 192, d4);
        if (valid)
            for (int c = 0; c < kH2; ++c) a.dg[(size_t)b * kH2 + c] = g[c] > 0.0f ? d4[c] : 0.0f;
        float *part = a.head_part + (size_t)blockIdx.x * kHeadPart;
        if (warp < 2) {  // rows 0..63 of D5: dW3
            float r[kH2];
            tmem_row<kH2>(tmem, warp, 320, r);
            for (int c = 0; c < kH2; ++c) part[oW3 + tid * kH2 + c] = r[c];
        }
        if (warp == 0) {  // rows 0..5 of D6: dW4
            float r[kH3];
            tmem_row<kH3>(tmem, warp, 448, r);
            if (tid < kOut)
                for (int j = 0; j < kH3; ++j) part[oW4 + tid * kH3 + j] = r[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
    if (failed) return;
    // bias gradients: column sums over the tile's rows in row order (the G operand's space is free now)
    float *red = reinterpret_cast<float *>(sm + hG);  // 128 rows x (64 + 6) floats
#pragma unroll
    for (int j = 0; j < kH3; ++j) red[tid * (kH3 + kOut) + j] = dh3[j];
#pragma unroll
    for (int o = 0; o < kOut; ++o) red[tid * (kH3 + kOut) + kH3 + o] = dy[o];
    __syncthreads();
    if (tid < kH3 + kOut) {
        float sacc = 0.0f;
        for (int r = 0; r < 128; ++r) sacc += red[r * (kH3 + kOut) + tid];
        float *part = a.head_part + (size_t)blockIdx.x * kHeadPart;
        part[tid < kH3 ? oB3 + tid : oB4 + (tid - kH3)] = sacc;
    }
}

// The shared layers' gradient of one scan (one CTA of 128 threads): the
// max-pool routes channel c's gradient dg[c] to one point (its argmax), so
// this is a gather over at most 128 points, with the BF16 operands of the
// forward (h1 and W2 rounded to BF16):
//   dW2[c][k] = dg[c] bf16(h1[p_c][k]),  db2[c] = dg[c],
//   dz1[c][k] = dg[c] bf16(W2[c][k]) [z1[p_c][k] > 0],  dW1[k] = sum_c dz1[c][k] u[p_c],  db1[k] = sum_c dz1[c][k].
struct SharedBwdArgs {
    const float4 *points;
    const int *offsets;
    const float *guesses;
    const float *w;
    const unsigned long long *gmax;
    const float *dg;     // B x 128
    float *grad_scan;    // B x kNumW (the shared layers' entries)
    Norm nm;
    int B;
    int max_points;
};

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

__global__ void __launch_bounds__(128) shared_bwd_kernel(const __grid_constant__ SharedBwdArgs a) {
    __shared__ float dgs[kH2];
    __shared__ int arg[kH2];
    __shared__ float sT[12];
    const int tid = threadIdx.x, b = blockIdx.x;
    if (b >= a.B) return;
    const float *w = a.w;
    {
        const unsigned long long m = a.gmax[(size_t)b * kH2 + tid];
        arg[tid] = (int)(0xffffffffu - (unsigned)(m & 0xffffffffu));
        dgs[tid] = a.dg[(size_t)b * kH2 + tid];
    }
    if (tid < 12) sT[tid] = a.guesses[16 * (size_t)b + tid];
    __syncthreads();
    float *G = a.grad_scan + (size_t)b * kNumW;
    const int start = a.offsets[b], n = a.offsets[b + 1] - start;
    const int P = n < a.max_points ? n : a.max_points;
    {
        const int c = tid;
        const float d = dgs[c];
        float u[3] = {0.f, 0.f, 0.f};
        if (d != 0.0f && P > 0) point_feature(sT, a.points[start + sample_index(arg[c], P, n)], a.nm, u);
        for (int k = 0; k < kH1; ++k) {
            const float v = fmaf(w[oW1 + 3 * k], u[0], fmaf(w[oW1 + 3 * k + 1], u[1], fmaf(w[oW1 + 3 * k + 2], u[2],
                                                                                            w[oB1 + k])));
            G[oW2 + c * kH1 + k] = d * bf16r(fmaxf(v, 0.0f));
        }
        G[oB2 + c] = d;
    }
    if (tid < kH1) {
        const int k = tid;
        float gw0 = 0.f, gw1 = 0.f, gw2 = 0.f, gb = 0.f;
        for (int c = 0; c < kH2; ++c) {
            const float d = dgs[c];
            if (d == 0.0f) continue;
            float u[3];
            point_feature(sT, a.points[start + sample_index(arg[c], P, n)], a.nm, u);
            const float z = fmaf(w[oW1 + 3 * k], u[0], fmaf(w[oW1 + 3 * k + 1], u[1], fmaf(w[oW1 + 3 * k + 2], u[2],
                                                                                            w[oB1 + k])));
            if (!(z > 0.0f)) continue;
            const float dz = bf16r(w[oW2 + c * kH1 + k]) * d;
            gw0 = fmaf(dz, u[0], gw0);
            gw1 = fmaf(dz, u[1], gw1);
            gw2 = fmaf(dz, u[2], gw2);
            gb += dz;
        }
        G[oW1 + 3 * k] = gw0;
        G[oW1 + 3 * k + 1] = gw1;
        G[oW1 + 3 * k + 2] = gw2;
        G[oB1 + k] = gb;
    }
}

// Batch gradient (mean over the scans: the shared layers' per-scan gradients
// in scan order, the head's per-tile sums in tile order) and loss; optionally
// an Adam step on the FP32 weights.
struct AdamArgs {
    float *w, *m, *v;
    const float *grad_scan;  // B x kNumW: the shared layers' entries (W1, b1, W2, b2)
    const float *head_part;  // parts x kNumW: the head's entries (W3, b3, W4, b4), summed over 128 scans each
    int parts;
    const float *loss_scan;
    float *grad;   // kNumW out (batch gradient)
    float *loss;   // 1 out
    int B;
    float lr, beta1, beta2, eps, bc1, bc2;  // bc = 1 - beta^t
    int update;
};

__global__ void reduce_adam_kernel(const __grid_constant__ AdamArgs a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        float l = 0.f;
        for (int b = 0; b < a.B; ++b) l += a.loss_scan[b];
        *a.loss = l / a.B;
    }
    if (i >= kNumW) return;
    float s = 0.f;
    if (i < oW3)
        for (int b = 0; b < a.B; ++b) s += a.grad_scan[(size_t)b * kNumW + i];
    else
        for (int t = 0; t < a.parts; ++t) s += a.head_part[(size_t)t * kNumW + i];
    const float gi = s / a.B;
    a.grad[i] = gi;
    if (!a.update) return;
    const float m = a.beta1 * a.m[i] + (1.0f - a.beta1) * gi;
    const float v = a.beta2 * a.v[i] + (1.0f - a.beta2) * gi * gi;
    a.m[i] = m;
    a.v[i] = v;
    a.w[i] -= a.lr * (m / a.bc1) / (sqrtf(v / a.bc2) + a.eps);
}

// proposal = T(pose(guess) + y * dscale)
__global__ void apply_kernel(const float *__restrict__ guesses, const float *__restrict__ y, Norm nm, int B,
                             float *__restrict__ out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double p[6];
    pose_of(guesses + 16 * (size_t)b, p);
    for (int i = 0; i < 6; ++i) p[i] += (double)y[6 * (size_t)b + i] * (double)nm.dscale[i];
    matrix_of(p, out + 16 * (size_t)b);
}

// The NDT's judgement: start from the proposal where its score is at least
// the raw guess's, from the guess otherwise.
__global__ void judge_kernel(const float *__restrict__ prop, const float *__restrict__ guess,
                             const double *__restrict__ s_prop, const double *__restrict__ s_guess, int B,
                             float *__restrict__ start, int *__restrict__ used) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const bool u = s_prop[b] >= s_guess[b];
    for (int k = 0; k < 16; ++k) start[16 * (size_t)b + k] = u ? prop[16 * (size_t)b + k] : guess[16 * (size_t)b + k];
    if (used) used[b] = u ? 1 : 0;
}

}  // namespace pn

// ---------------------------------------------------------------------------
// C ABI (struct ndt_mlp: mlp_internal.h)

namespace {

int mlp_fail(ndt_mlp *c, cudaError_t e, const char *what) {
    if (c) c->msg = std::string(what) + ": " + cudaGetErrorString(e);
    return NDT_E_CUDA;
}

#define MCK(call)                                               \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return mlp_fail(c, e_, #call);   \
    } while (0)

constexpr size_t kPointSmem = 2 * pn::kOperandBytes + (pn::kH1 * 3 + pn::kH1 + pn::kH2) * 4 + 64;
// keep at most 4 CTAs per SM, so that 4 x 128 TMEM columns fit
constexpr size_t kPointSmemAlloc = kPointSmem < 48 * 1024 ? 48 * 1024 : kPointSmem;

int ensure_batch(ndt_mlp *c, int B) {
    if ((size_t)B <= c->cap_b) return NDT_OK;
    cudaFree(c->gmax);
    cudaFree(c->grad_scan);
    cudaFree(c->loss_scan);
    cudaFree(c->dg);
    cudaFree(c->head_part);
    c->gmax = nullptr;
    c->grad_scan = c->loss_scan = c->dg = c->head_part = nullptr;
    c->cap_b = 0;
    MCK(cudaMalloc(&c->gmax, sizeof(unsigned long long) * pn::kH2 * (size_t)B));
    MCK(cudaMalloc(&c->grad_scan, sizeof(float) * pn::kNumW * (size_t)B));
    MCK(cudaMalloc(&c->loss_scan, sizeof(float) * (size_t)B));
    MCK(cudaMalloc(&c->dg, sizeof(float) * pn::kH2 * (size_t)B));
    MCK(cudaMalloc(&c->head_part, sizeof(float) * pn::kHeadPart * (size_t)((B + 127) / 128)));
    c->cap_b = (size_t)B;
    return NDT_OK;
}

// The head on the tensor cores over B candidates (inference: target null).
int run_head(ndt_mlp *c, int B, const float *d_target6, float *d_y6) {
    pn::HeadTcArgs h;
    std::memset(&h, 0, sizeof(h));
    h.w = c->w;
    h.gmax = c->gmax;
    h.target = d_target6;
    h.y = d_y6;
    h.dg = c->dg;
    h.loss_scan = c->loss_scan;
    h.head_part = c->head_part;
    h.err = c->err;
    h.B = B;
    h.wait_limit = c->wait_limit;
    pn::head_tc_kernel<<<(B + 127) / 128, 128, pn::kHeadSmem, c->stream>>>(h);
    MCK(cudaGetLastError());
    return NDT_OK;
}

int run_forward(ndt_mlp *c, int B, const float *d_points, const int *d_offsets, const float *d_guesses,
                int max_points, int scans) {
    if (int rc = ensure_batch(c, B)) return rc;
    pn::PointArgs a;
    a.points = reinterpret_cast<const float4 *>(d_points);
    a.offsets = d_offsets;
    a.guesses = d_guesses;
    a.w = c->w;
    a.w2op = c->w2op;
    a.gmax = c->gmax;
    a.err = c->err;
    a.wait_limit = c->wait_limit;
    a.nm = c->nm;
    a.B = B;
    a.scans = scans;
    a.max_points = max_points;
    pn::point_kernel<<<B, 128, kPointSmemAlloc, c->stream>>>(a);
    MCK(cudaGetLastError());
    return NDT_OK;
}

}  // namespace

extern "C" {

int ndt_mlp_num_weights(void) { return pn::kNumW; }

int ndt_mlp_create(int device, ndt_mlp **out) {
    if (!out) return NDT_E_ARG;
    *out = nullptr;
    ndt_mlp *c = new ndt_mlp();
    c->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    c->stream = c->own_stream;
    if (e == cudaSuccess) e = cudaMalloc(&c->w, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess) e = cudaMalloc(&c->m, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess) e = cudaMalloc(&c->v, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess) e = cudaMalloc(&c->grad, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess) e = cudaMalloc(&c->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->w2op, pn::kOperandBytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(c->m, 0, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess) e = cudaMemset(c->v, 0, sizeof(float) * pn::kNumW);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pn::point_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPointSmemAlloc);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(pn::head_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pn::kHeadSmem);
    if (e != cudaSuccess) {
        ndt_mlp_destroy(c);
        return NDT_E_CUDA;
    }
    for (int i = 0; i < 6; ++i) c->nm.dscale[i] = 1.0f;
    c->nm.inv_s = 1.0f;
    *out = c;
    return NDT_OK;
}

void ndt_mlp_destroy(ndt_mlp *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *bufs[] = {c->w, c->m, c->v, c->grad, c->loss, c->w2op, c->err, c->gmax, c->grad_scan, c->loss_scan,
                    c->dg, c->head_part};
    for (void *p : bufs)
        if (p) cudaFree(p);
    learned_buffers_free(c->lb);
    for (cudaEvent_t e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

const char *ndt_mlp_last_error(const ndt_mlp *c) { return c ? c->msg.c_str() : "null network"; }

int ndt_mlp_set_input_frame(ndt_mlp *c, const float center3[3], float scale, const float delta_scale6[6]) {
    if (!c || !center3 || !delta_scale6 || !(scale > 0.0f)) return NDT_E_ARG;
    c->nm.cx = center3[0];
    c->nm.cy = center3[1];
    c->nm.cz = center3[2];
    c->nm.inv_s = 1.0f / scale;
    for (int i = 0; i < 6; ++i) c->nm.dscale[i] = delta_scale6[i];
    return NDT_OK;
}

int ndt_mlp_set_weights(ndt_mlp *c, const float *w, int n) {
    if (!c || !w || n != pn::kNumW) return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    MCK(cudaMemcpyAsync(c->w, w, sizeof(float) * pn::kNumW, cudaMemcpyHostToDevice, c->stream));
    MCK(cudaMemsetAsync(c->m, 0, sizeof(float) * pn::kNumW, c->stream));
    MCK(cudaMemsetAsync(c->v, 0, sizeof(float) * pn::kNumW, c->stream));
    pn::pack_w2_kernel<<<(pn::kH2 * pn::kH1 + 255) / 256, 256, 0, c->stream>>>(c->w, c->w2op);
    MCK(cudaGetLastError());
    MCK(cudaStreamSynchronize(c->stream));
    c->step = 0;
    return NDT_OK;
}

int ndt_mlp_get_weights(ndt_mlp *c, float *w, int n) {
    if (!c || !w || n != pn::kNumW) return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    MCK(cudaMemcpyAsync(w, c->w, sizeof(float) * pn::kNumW, cudaMemcpyDeviceToHost, c->stream));
    MCK(cudaStreamSynchronize(c->stream));
    return NDT_OK;
}

int ndt_mlp_forward_device(ndt_mlp *c, int B, const float *d_points, const int *d_offsets, const float *d_guesses,
                           int max_points, float *d_y6) {
    if (!c || B <= 0 || !d_points || !d_offsets || !d_guesses || !d_y6 || max_points <= 0) return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    return mlp_forward(c, B, B, d_points, d_offsets, d_guesses, max_points, d_y6);
}

}  // extern "C"

int mlp_forward(ndt_mlp *c, int B, int scans, const float *d_points, const int *d_offsets, const float *d_guesses,
                int max_points, float *d_y6) {
    if (int rc = run_forward(c, B, d_points, d_offsets, d_guesses, max_points, scans)) return rc;
    return run_head(c, B, nullptr, d_y6);
}

int mlp_propose(ndt_mlp *c, int B, int scans, const float *d_points, const int *d_offsets, const float *d_guesses,
                int max_points, int passes, float *d_y6, float *d_prop16) {
    const float *g = d_guesses;
    for (int k = 0; k < passes; ++k) {
        if (int rc = mlp_forward(c, B, scans, d_points, d_offsets, g, max_points, d_y6)) return rc;
        pn::apply_kernel<<<(B + 127) / 128, 128, 0, c->stream>>>(g, d_y6, c->nm, B, d_prop16);
        MCK(cudaGetLastError());
        g = d_prop16;  // the next pass reads the previous proposal (in place: each thread reads its own row first)
    }
    return NDT_OK;
}

extern "C" {

int ndt_mlp_train_step_device(ndt_mlp *c, int B, const float *d_points, const int *d_offsets, const float *d_guesses,
                              const float *d_target6, int max_points, float lr, int update, float *h_loss,
                              float *h_grad) {
    if (!c || B <= 0 || !d_points || !d_offsets || !d_guesses || !d_target6 || max_points <= 0) return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    if (int rc = run_forward(c, B, d_points, d_offsets, d_guesses, max_points, B)) return rc;
    if (int rc = run_head(c, B, d_target6, nullptr)) return rc;
    pn::SharedBwdArgs sb;
    sb.points = reinterpret_cast<const float4 *>(d_points);
    sb.offsets = d_offsets;
    sb.guesses = d_guesses;
    sb.w = c->w;
    sb.gmax = c->gmax;
    sb.dg = c->dg;
    sb.grad_scan = c->grad_scan;
    sb.nm = c->nm;
    sb.B = B;
    sb.max_points = max_points;
    pn::shared_bwd_kernel<<<B, 128, 0, c->stream>>>(sb);
    MCK(cudaGetLastError());
    if (update) ++c->step;
    pn::AdamArgs a;
    a.w = c->w;
    a.m = c->m;
    a.v = c->v;
    a.grad_scan = c->grad_scan;
    a.head_part = c->head_part;
    a.parts = (B + 127) / 128;
    a.loss_scan = c->loss_scan;
    a.grad = c->grad;
    a.loss = c->loss;
    a.B = B;
    a.lr = lr;
    a.beta1 = 0.9f;
    a.beta2 = 0.999f;
    a.eps = 1e-8f;
    a.bc1 = 1.0f - std::pow(0.9f, (float)(c->step > 0 ? c->step : 1));
    a.bc2 = 1.0f - std::pow(0.999f, (float)(c->step > 0 ? c->step : 1));
    a.update = update;
    pn::reduce_adam_kernel<<<(pn::kNumW + 255) / 256, 256, 0, c->stream>>>(a);
    MCK(cudaGetLastError());
    if (update) {
        pn::pack_w2_kernel<<<(pn::kH2 * pn::kH1 + 255) / 256, 256, 0, c->stream>>>(c->w, c->w2op);
        MCK(cudaGetLastError());
    }
    if (h_loss) MCK(cudaMemcpyAsync(h_loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    if (h_grad) MCK(cudaMemcpyAsync(h_grad, c->grad, sizeof(float) * pn::kNumW, cudaMemcpyDeviceToHost, c->stream));
    if (h_loss || h_grad) MCK(cudaStreamSynchronize(c->stream));
    return NDT_OK;
}

int ndt_mlp_maxpool_device(ndt_mlp *c, unsigned long long *d_out, int B) {
    if (!c || !d_out || B <= 0 || (size_t)B > c->cap_b) return NDT_E_ARG;
    MCK(cudaMemcpyAsync(d_out, c->gmax, sizeof(unsigned long long) * pn::kH2 * (size_t)B,
                        cudaMemcpyDeviceToDevice, c->stream));
    return NDT_OK;
}

int ndt_mlp_synchronize(ndt_mlp *c, int *tc_error) {
    if (!c) return NDT_E_ARG;
    MCK(cudaStreamSynchronize(c->stream));
    int e = 0;
    MCK(cudaMemcpy(&e, c->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) MCK(cudaMemset(c->err, 0, sizeof(int)));  // reported once: the flag covers the calls since the last one
    if (tc_error) *tc_error = e;
    return NDT_OK;
}

int ndt_mlp_set_wait_limit(ndt_mlp *c, int polls) {
    if (!c) return NDT_E_ARG;
    c->wait_limit = polls < 0 ? pn::kWaitLimit : (unsigned)polls;
    return NDT_OK;
}

void *ndt_mlp_stream(ndt_mlp *c) { return c ? (void *)c->stream : nullptr; }

int ndt_mlp_set_stream(ndt_mlp *c, void *stream) {
    if (!c) return NDT_E_ARG;
    MCK(cudaStreamSynchronize(c->stream));
    c->stream = stream ? (cudaStream_t)stream : c->own_stream;
    return NDT_OK;
}

int ndt_mlp_propose_device(ndt_mlp *c, int B, const float *d_points, const int *d_offsets, const float *d_guesses,
                           int max_points, int passes, float *d_y6, float *d_prop16) {
    if (!c || B <= 0 || !d_points || !d_offsets || !d_guesses || !d_y6 || !d_prop16 || max_points <= 0 || passes < 1)
        return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    return mlp_propose(c, B, B, d_points, d_offsets, d_guesses, max_points, passes, d_y6, d_prop16);
}

int ndt_mlp_judge_device(ndt_mlp *c, int B, const float *d_prop16, const float *d_guesses, const double *d_score_prop,
                         const double *d_score_guess, float *d_start16, int *d_used) {
    if (!c || B <= 0 || !d_prop16 || !d_guesses || !d_score_prop || !d_score_guess || !d_start16) return NDT_E_ARG;
    MCK(cudaSetDevice(c->device));
    pn::judge_kernel<<<(B + 127) / 128, 128, 0, c->stream>>>(d_prop16, d_guesses, d_score_prop, d_score_guess, B,
                                                             d_start16, d_used);
    MCK(cudaGetLastError());
    return NDT_OK;
}

}  // extern "C"
