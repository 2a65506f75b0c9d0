// Device voxel-grid build (see grid_build.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ndt_types.h"

namespace ndt {

// Output buffers of one grid (capacities: index G, per-voxel arrays m).
struct GridBuffers {
    int32_t *index;      // G dense cell -> voxel slot (-1 = no usable voxel)
    double4 *mean;       // slot -> mean xyz, w = 1 if the FP32 pair path must not be used
    float4 *mean_hi;     // slot -> float(mean) xyz
    float4 *mean_lo;     // slot -> float(mean - float(mean)) xyz
    float4 *icov32;      // slot -> 2 float4 (symmetrised FP32 inverse covariance)
    double *icov64;      // slot -> 9 doubles
    int32_t *count;      // slot -> points in the cell
    int32_t *cell;       // slot -> dense cell id
    int32_t *seg_start;  // slot -> first position in the sorted order
    uint32_t *seg_cell;  // slot -> dense cell id (sort output)
};

struct NdtGridOptions {
    int compat;
    int min_points;
    double eigen_ratio;
};

size_t grid_scratch_bytes(int m);

// Phase 1: bounding box and dims into *d_meta (the caller reads it back to
// size the dense index table).
int grid_bbox(const float4 *d_map, int m, float res, GridMeta *d_meta, void *scratch, cudaStream_t st);

// Phase 2: keys, stable sort, segments, per-voxel records.
int grid_build(const float4 *d_map, int m, const GridMeta &meta_host, GridMeta *d_meta, const NdtGridOptions &opt,
               GridBuffers buf, void *scratch, cudaStream_t st, int *launches);

}  // namespace ndt
