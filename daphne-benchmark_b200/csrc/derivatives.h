// Derivative pass launcher (see derivatives.cu).
#pragma once
#include <cuda_runtime.h>

#include "ndt_types.h"

namespace ndt {

struct EvalArgs {  // (GridDev is in ndt_types.h)
    GridDev grid;
    const float4 *points;  // all scans, concatenated (original coordinates)
    const float4 *trans;   // optional: already transformed points (then T is not applied)
    const Tile *tiles;
    const int *num_tiles;  // device: number of tiles
    const Chunk *chunks;   // chunks of tiles (FP32 pass; the FP64 pass uses chunks of 1 tile)
    const int *num_chunks; // device: number of chunks
    int max_tiles;         // host-side upper bound (grid sizing)
    int tile_size;         // points per tile (must equal the kernel variant's block size)
    AlignState *states;
    double *partials;      // [chunk][kPartial]
    double *exc;           // [alignment][kPartial] FP64 side sums of flagged voxels (FP32 path)
    double d1, d2;         // Gauss constants (kernel.cpp:1181-1185)
    int compat;
    Counters *counters;    // may be null
    int4 *flag_q;          // FP32 path: queue of pairs with flagged voxels (align, point, slot, -)
    unsigned *flag_n;      // queue length (reset by launch_derivatives)
    unsigned flag_cap;     // queue capacity
    int *flag_overflow;    // set when the queue overflowed
    int *work_counter;     // FP32 pass: next chunk (reset by launch_derivatives)
    // FP32 pass, optional: the pass first compacts the chunks whose alignment
    // asks for an evaluation into active_chunks (capacity: the chunk count)
    // and hands out only those (batches whose alignments finish at different
    // rounds); null: every chunk is handed out and inactive ones skipped.
    int *active_chunks = nullptr;
    int *num_active = nullptr;
};

constexpr int kOwn = 27;        // accepted pairs of one point per collect call, at most (3 x 3 x 3 probes)
constexpr int kChunkBig = 8;    // tiles per large chunk of the FP32 pass by default (the FP64 pass: 1)
constexpr int kMaxChunkTiles = 64;
// the chunk sizes the autotuner times (8 suits batches of many large scans,
// c5: 21k chunks per pass; 4 the smaller c3 / c4 batches, where the end of
// the pass is a larger share)
constexpr int kChunkChoices[] = {4, 6, 8};
constexpr int kChunkSmall = 4;  // tiles per small chunk of the FP32 pass, at most the large size (the FP64 pass: 1)

// Per-device set-up (dynamic shared memory opt-in); call with the device current.
int prepare_derivatives();

// FP32 derivative-pass launch shapes the autotuner chooses from:
// (points per tile = threads per block, resident blocks per SM).
struct DerivVariant {
    int tile;
    int min_blocks;
};
constexpr int kNumDerivVariants = 7;
// The shape a new context starts with: 128 threads x 6 blocks per SM (80
// registers, 35.7 KB of shared memory per block), the fastest on B200 for the
// corrected-mode workloads (c5: 2M-point map at 0.5 m); on c2 compat 128 x 5
// is within 1 %.
constexpr int kDefaultDerivVariant = 6;
extern const DerivVariant kDerivVariants[kNumDerivVariants];

// precision 0 = FP32 pair arithmetic (launch shape `variant`), 1 = FP64
// (256-point tiles).  The persistent grid is sms x resident blocks; blocks
// loop over the tiles.
int launch_derivatives(const EvalArgs &args, int precision, int variant, int sms, cudaStream_t st);
// The FP64 pass alone (256-point tiles).
int launch_derivatives_f64(const EvalArgs &args, int sms, cudaStream_t st);
// Kernel launches per launch_derivatives call (FP32: pass + flagged pairs; FP64: pass).
constexpr int kDerivLaunchesFP32 = 2;

}  // namespace ndt
