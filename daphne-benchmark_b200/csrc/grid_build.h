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
    float4 *vox32;       // slot -> 3 float4, the FP32 pair record (GridDev::vox32)
    double *icov64;      // slot -> 9 doubles
    int32_t *count;      // slot -> points in the cell
    int32_t *cell;       // slot -> dense cell id
    int32_t *seg_start;  // slot -> first position in the sorted order
    uint32_t *seg_cell;  // slot -> dense cell id (sort output)
    int32_t *slot_of;    // G dense cell -> its slot, usable or not (-1 = no points)
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
int grid_windows(const GridMeta &meta_host, const int32_t *index, const float4 *vox32, WindowBuffers wb,
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
// The two halves: the radix passes alone (b.k0 / b.v0 sorted afterwards), and
// the segments of sorted keys (segc: ceil(n / 2048) + 1 ints, part: the
// multi-block scan's tile sums).
int radix_sort_pairs(SortBuffers &b, int n, int bits, cudaStream_t st);
int segment_sorted(const uint32_t *keys, int n, int *segc, int *nseg, int *part, int32_t *seg_start,
                   uint32_t *seg_key, cudaStream_t st);

// The map's points sorted by dense cell (key) and, within a cell, by point
// index: what the last build or append left, the input of the next append.
struct SortedMap {
    const uint32_t *keys;
    const uint32_t *order;
};

size_t grid_scratch_bytes(int m);
// Zeroes the scratch's bounding-box counters (once, after the scratch is allocated).
int grid_scratch_init(void *scratch, cudaStream_t st);

// Phase 1: bounding box and dims into *d_meta (the caller reads it back to
// size the dense index table).
int grid_bbox(const float4 *d_map, int m, float res, GridMeta *d_meta, void *scratch, cudaStream_t st);

// Phase 2: keys, stable sort, segments, per-voxel records.  *sorted (optional)
// receives the sorted (cell, point) pairs, which stay valid in the scratch
// until the next build.
int grid_build(const float4 *d_map, int m, const GridMeta &meta_host, GridMeta *d_meta, const NdtGridOptions &opt,
               GridBuffers buf, void *scratch, cudaStream_t st, int *launches, SortedMap *sorted = nullptr);

// Incremental map growth: the map's points [0, m_old) were built into the
// grid (same meta: the appended points lie inside the old points' bounding
// box) and sorted as old_sorted; points [m_old, m_old + k) of d_map are new.
// Their keys are sorted and merged with old_sorted (old first on equal keys:
// exactly the stable sort of all m_old + k points) into keys_out / order_out
// (capacity m_old + k).  Only the cells the new points fall in are recomputed,
// each from all its points in that order with the build's arithmetic, so the
// records equal a full build's bit for bit; cells new to the grid take the
// next slots (slot numbers may differ from a full build's; the records per
// cell do not).  The record arrays must hold m_old + k slots with the old
// slots kept.  Scratch: append_scratch_bytes(k).
size_t append_scratch_bytes(int k);
int grid_append(const float4 *d_map, int m_old, int k, const GridMeta &meta_host, GridMeta *d_meta,
                const NdtGridOptions &opt, GridBuffers buf, SortedMap old_sorted, uint32_t *keys_out,
                uint32_t *order_out, void *scratch, cudaStream_t st, int *launches);

}  // namespace ndt
