// Derivative pass launcher (see derivatives.cu).
#pragma once
#include <cuda_runtime.h>

#include "ndt_types.h"

namespace ndt {

struct EvalArgs {
    GridDev grid;
    const float4 *points;  // all scans, concatenated (original coordinates)
    const float4 *trans;   // optional: already transformed points (then T is not applied)
    const Tile *tiles;
    const int *num_tiles;  // device: number of tiles
    int max_tiles;         // host-side upper bound (grid sizing)
    AlignState *states;
    double *partials;      // [tile slot][kPartial]
    double *exc;           // [alignment][kPartial] FP64 side sums of flagged voxels (FP32 path)
    double d1, d2;         // Gauss constants (kernel.cpp:1181-1185)
    int compat;
    Counters *counters;    // may be null
};

// precision 0 = FP32 pair arithmetic, 1 = FP64.  grid_blocks caps the
// persistent grid (blocks loop over tiles).
int launch_derivatives(const EvalArgs &args, int precision, int grid_blocks, cudaStream_t st);

}  // namespace ndt
