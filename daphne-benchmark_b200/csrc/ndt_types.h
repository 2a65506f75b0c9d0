// Types shared by the host engine and the device kernels.
#pragma once
#include <stdint.h>

namespace ndt {

constexpr int kTile = 256;      // scan points per derivative-pass tile (= threads per block)
constexpr int kPartial = 44;    // per-tile partial: score, g[6], H[36], pair count
constexpr int kAngle = 69;      // angle terms: j_ang a..h (8 x 3) + h_ang a2..f3 (15 x 3)

// Dense index entries: voxel slot in the low bits, kSlotFlag set when the
// voxel's inverse covariance must be evaluated in FP64 (non-finite entries or
// entries beyond 1e30); -1 = no usable voxel.
constexpr int32_t kSlotFlag = 1 << 30;
constexpr int32_t kSlotMask = kSlotFlag - 1;

// What the derivative pass must compute for one alignment this round.
enum EvalMode : int32_t {
    kEvalNone = 0,
    kEvalFull = 1,      // score, gradient, Hessian (computeDerivatives(..., true))
    kEvalGradient = 2,  // score, gradient; Hessian reset to 0 (computeDerivatives(..., false))
    kEvalHessian = 3,   // Hessian only (computeHessian)
};

// Phases of the per-alignment registration state machine (one Newton
// iteration = solve + More-Thuente step length + pose update).
enum Phase : int32_t {
    kPhaseInitEval = 0,  // waiting for the first evaluation at the guess
    kPhaseMTFirst = 1,   // waiting for the first line-search evaluation
    kPhaseMTIter = 2,    // waiting for a later line-search evaluation
    kPhaseMTHess = 3,    // waiting for the closing Hessian pass
    kPhaseDone = 4,
};

// Grid geometry (dense addressing as the reference's initCompute).
struct GridMeta {
    float minv[3];
    float maxv[3];
    float raw_min[3];  // min / max of the map points themselves (minv = raw_min - 0.01f, maxv = raw_max + 0.01f)
    float raw_max[3];
    int32_t dim[3];
    float res;
    int64_t G;         // dense cell count
    int32_t occupied;  // cells with >= 1 point (compat) / usable cells (corrected)
    int32_t error;     // nonzero: G does not fit 32-bit indices
};

// Device pointers of a built grid.
struct GridDev {
    GridMeta meta;
    const int32_t *index;    // G: dense cell -> voxel slot | kSlotFlag, -1 = none
    const double4 *mean;     // K: mean xyz (FP64), w = 1 when the FP32 path must not be used
    // 3K: a voxel's FP32 pair record, one 48-byte gather: {float(mean) xyz, c00},
    // {float(mean - float(mean)) xyz, c01}, {c02 c11 c12 c22} (the symmetrised
    // inverse covariance); x' = (x - hi) - lo, and hi is the probe's first,
    // conservative distance test
    const float4 *vox32;
    float s_max;             // largest float s with sqrtf(s) < res (the radius test without sqrt)
    float inv_res;           // 1 / res when res is a power of two (exact), else 0 (divide)
    float radius_final;      // (float)(res + 0.001f): the probe loop bound of kernel.cpp:254
    const double *icov64;    // 9K: inverse covariance as the reference stores it (row major)
    // probe-window table (grid_build.h), nullptr when not built
    const int32_t *win_off;  // W + 1
    const float4 *win_ent;   // {float(mean) xyz, slot << 6 | flag << 5 | cell offset}
    int32_t win_dim[2];      // dim_x + 2, dim_y + 2
};

// Per-alignment state (FP64 control, float transform), one per alignment.
struct __align__(16) AlignState {
    // evaluation request read by the derivative pass
    float T[16];             // final_transformation_ used for the current evaluation
    float angf[kAngle];      // angle terms (FP32 copy)
    int32_t eval_mode;
    int32_t phase;
    double angd[kAngle];     // angle terms (FP64)
    // Newton / More-Thuente state (kernel.cpp:1015-1272 variables)
    double p[6];             // current pose vector
    double x_t[6];           // trial pose
    double dir[6];           // step direction (delta_p)
    double g[6];
    double H[36];
    double score;
    double phi_0, d_phi_0, a_l, f_l, g_l, a_u, f_u, g_u, a_t, phi_t, d_phi_t, psi_t, d_psi_t;
    double step_max, step_min;
    int32_t nr_iterations;
    int32_t step_iterations;
    int32_t open_interval;
    int32_t interval_converged;
    int32_t converged;
    int32_t evals;
    int32_t status;
    int32_t n;               // scan points
};

// Work counters (device, 64-bit).
struct Counters {
    unsigned long long evaluations;
    unsigned long long points;
    unsigned long long probes;
    unsigned long long occupied_probes;
    unsigned long long pairs;
    unsigned long long tiles;
    unsigned long long rounds;  // lockstep rounds (derivative pass + step) of the batch
};

struct Tile {
    int32_t align;
    int32_t start;   // first point (global index into the concatenated scans)
    int32_t end;     // one past the last point
    int32_t slot;    // index of this tile in the tile list
};

// Consecutive tiles of one alignment: the unit of work the derivative pass
// hands out, with one partial-sum slot (partials[slot]; an alignment's slots
// are contiguous, chunk_begin[b] .. chunk_begin[b + 1]).  An alignment's
// tiles are cut, from its first tile, into large chunks and then a few small
// ones (the last tiles); the list holds every large chunk of the batch before
// any small one, so the blocks finish together.  Chunk boundaries depend only
// on the alignment's own point count, so its sums are the same in any batch.
struct Chunk {
    int32_t align;
    int32_t first;   // first tile
    int32_t end;     // one past the last tile
    int32_t slot;    // partial-sum slot
};

// Tile and chunk lists of a batch (device).
struct TileLists {
    int *tile_begin;   // B + 1: first tile of each alignment
    Tile *tiles;
    int *num_tiles;
    int *chunk_begin;  // B + 1: first partial slot of each alignment
    Chunk *chunks;     // large chunks, then small chunks
    int *num_chunks;
    int *big_begin;    // B + 1: scratch (large chunks before each alignment)
    int *small_begin;  // B + 1: scratch (small chunks before each alignment)
    int *num_big;      // total large chunks
};

}  // namespace ndt
