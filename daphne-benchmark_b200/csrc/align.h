// Per-alignment control kernels (see align.cu).
#pragma once
#include <cuda_runtime.h>

#include "ndt_types.h"

namespace ndt {

constexpr int NDT_ST_WATCHDOG_DEV = 1;
constexpr int NDT_ST_OVERFLOW_DEV = 2;

struct StepParams {
    int compat;
    int max_iterations;
    double eps;        // transformation_epsilon: |step| < eps stop test
    double step_max;   // step_size
    double step_min;   // eps / 2
    int watchdog_evals;
};

// Tiles of `tile` points and chunks (large: kb tiles, small: ks tiles) for
// the alignments of a batch (d_offsets: B + 1 point offsets; tile and chunk
// capacity: total / tile + B + 1).
int launch_tiles(const int *d_offsets, int B, int tile, int kb, int ks, const TileLists &L, cudaStream_t st);
int launch_init(AlignState *d_states, const float *d_guesses, const int *d_offsets, int B, const StepParams &P,
                double *d_exc, cudaStream_t st);
int launch_step(AlignState *d_states, const double *d_partials, const int *d_chunk_begin, double *d_exc, int B,
                const StepParams &P, int *d_active, Counters *d_counters, cudaStream_t st);
int launch_prepare_eval(AlignState *d_state, const double *d_p6, int n, double *d_exc, int compat, cudaStream_t st);
int launch_score(const double *d_partials, const int *d_chunk_begin, const double *d_exc, int B, double *d_score,
                 cudaStream_t st);
int launch_finalize(const AlignState *d_states, int B, float *d_out, int *d_conv, double *d_fit, int *d_status,
                    const int *d_overflow, cudaStream_t st);

}  // namespace ndt
