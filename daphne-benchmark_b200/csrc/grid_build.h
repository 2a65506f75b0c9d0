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

// Probe-window table.  The FP32 derivative pass probes, for a point p, the
// cells [b, b + 2] on each axis, b = cell(p - res) (the reference's 3 x 3 x 3
// probe loop, kernel.cpp:256-260, whenever its three coordinates fall in
// consecutive cells).  Window w of base cell b, each component in
// [-2, dim - 1], lists the usable voxels of those 27 cells in the reference's
// probe order (z outer, x inner) as float4 {float(mean) xyz, code}, code =
// slot << 6 | flag << 5 | 9 dz + 3 dy + dx, so a point reads 2 offsets and one
// record per occupied cell instead of 27 dense-index entries.
struct WindowBuffers {
    int32_t *off;   // W + 1 entry offsets
    float4 *ent;    // entries (capacity 27 * min(m, G))
    int32_t *ctot;  // per-block totals (ceil(W / 256) + 1)
};

int64_t window_count(const GridMeta &g);  // W = (dim_x + 2)(dim_y + 2)(dim_z + 2)

// Builds the table from the finished dense index (after grid_build).
int grid_windows(const GridMeta &meta_host, const int32_t *index, const float4 *mean_hi, WindowBuffers wb,
                 cudaStream_t st, int *launches);

// Stable LSD radix sort of n (key, value) pairs on the low `bits` key bits,
// then the segments of equal keys: seg_start[s] = first sorted position of
// segment s, seg_key[s] = its key, *b.nseg = segment count (device).  After
// the call b.k0 / b.v0 hold the sorted keys and values.  Returns the number of
// kernel launches.
struct SortBuffers {
    uint32_t *k0, *v0, *k1, *v1;
    int *hist, *segc, *nseg, *part;
};
size_t sort_scratch_bytes(int n);
SortBuffers sort_buffers(void *scratch, int n);
int sort_segments(SortBuffers &b, int n, int bits, int32_t *seg_start, uint32_t *seg_key, cudaStream_t st);

size_t grid_scratch_bytes(int m);
// Zeroes the scratch's bounding-box counters (once, after the scratch is allocated).
int grid_scratch_init(void *scratch, cudaStream_t st);

// Phase 1: bounding box and dims into *d_meta (the caller reads it back to
// size the dense index table).
int grid_bbox(const float4 *d_map, int m, float res, GridMeta *d_meta, void *scratch, cudaStream_t st);

// Phase 2: keys, stable sort, segments, per-voxel records.
int grid_build(const float4 *d_map, int m, const GridMeta &meta_host, GridMeta *d_meta, const NdtGridOptions &opt,
               GridBuffers buf, void *scratch, cudaStream_t st, int *launches);

}  // namespace ndt
