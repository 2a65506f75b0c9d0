// Per-alignment control on the device: set-up from the guess, the Newton /
// More-Thuente state machine between derivative passes, and the result write.
//
// The reference runs, per alignment (computeTransformation,
// src/CPU/ndt_mapping/kernel.cpp:1175-1272, computeStepLengthMT :1015-1144):
//   eval(guess) ; repeat { solve ; step length (1 + <= 10 line-search evals +
//   optional Hessian pass) ; pose update ; convergence test }.
// Here every alignment of a batch is a small state machine in AlignState; a
// round is one derivative pass over all tiles of the alignments that asked for
// an evaluation, then one step_kernel call in which each such alignment
// consumes its result and advances until it needs the next evaluation (or is
// done).  All control arithmetic is FP64 with the reference's operation order.
#include <cuda_runtime.h>
#include <stdint.h>

#include "align.h"
#include "ndt_math.cuh"

namespace ndt {

namespace {

constexpr double kMu = 1.e-4;     // sufficient decrease (kernel.cpp:1042)
constexpr double kNu = 0.9;       // curvature condition (kernel.cpp:1044)
constexpr int kMaxStepIterations = 10;  // kernel.cpp:1039

__device__ void set_angles(AlignState &s, const double *pose, bool compat) {
    double a[kAngle];
    angle_terms(pose, a, compat);
    for (int k = 0; k < kAngle; ++k) {
        s.angd[k] = a[k];
        s.angf[k] = (float)a[k];
    }
}

__device__ void set_pose(AlignState &s, const StepParams &P) {
    if (P.compat)
        build_tm_compat(s.T, s.x_t);
    else
        build_tm_corrected(s.T, s.x_t);
    set_angles(s, s.x_t, P.compat);
}

__device__ __forceinline__ double dot6(const double *a, const double *b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2] + a[3] * b[3] + a[4] * b[4] + a[5] * b[5];
}

// Request an evaluation, unless the watchdog budget is spent.
__device__ bool request(AlignState &s, const StepParams &P, int mode, int phase) {
    if (s.evals >= P.watchdog_evals) {
        s.status = NDT_ST_WATCHDOG_DEV;
        s.converged = 0;
        s.phase = kPhaseDone;
        s.eval_mode = kEvalNone;
        return false;
    }
    s.eval_mode = mode;
    s.phase = phase;
    return true;
}

// Start of a Newton iteration (kernel.cpp:1214-1245) and of the step-length
// search up to its first evaluation (:1019-1066).  Returns true when an
// evaluation was requested; false when the step ended without one (then the
// caller continues with newton_end) or the alignment finished (phase Done).
__device__ bool newton_start(AlignState &s, const StepParams &P) {
    double A[6][6], b[6], dp[6];
    for (int i = 0; i < 6; ++i) {
        b[i] = -s.g[i];
        for (int j = 0; j < 6; ++j) A[i][j] = s.H[6 * i + j];
    }
    solve6(dp, A, b);
    double norm = sqrt(dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2] + dp[3] * dp[3] + dp[4] * dp[4] + dp[5] * dp[5]);
    if (P.compat) norm = 1;  // kernel.cpp:1231
    if (norm == 0 || norm != norm) {
        s.converged = norm == norm;
        s.phase = kPhaseDone;
        s.eval_mode = kEvalNone;
        return false;
    }
    for (int i = 0; i < 6; ++i) s.dir[i] = dp[i] / norm;
    // computeStepLengthMT(p, dir, step_init = norm, step_max, step_min)
    s.phi_0 = -s.score;
    s.d_phi_0 = -(dot6(s.g, s.dir));
    if (s.d_phi_0 >= 0) {
        if (s.d_phi_0 == 0) {
            s.a_t = 0;  // not a descent direction: step 0, no evaluation
            return false;
        }
        s.d_phi_0 *= -1;
        for (int i = 0; i < 6; ++i) s.dir[i] *= -1;
    }
    s.step_iterations = 0;
    s.a_l = 0;
    s.a_u = 0;
    s.f_l = psi_mt(s.a_l, s.phi_0, s.phi_0, s.d_phi_0, kMu);
    s.g_l = dpsi_mt(s.d_phi_0, s.d_phi_0, kMu);
    s.f_u = psi_mt(s.a_u, s.phi_0, s.phi_0, s.d_phi_0, kMu);
    s.g_u = dpsi_mt(s.d_phi_0, s.d_phi_0, kMu);
    // the reference tests "> 0" (kernel.cpp:1053), which skips the search
    // whenever step_max > step_min; the corrected NDT tests "< 0"
    s.interval_converged = P.compat ? (s.step_max - s.step_min) > 0 : (s.step_max - s.step_min) < 0;
    s.open_interval = 1;
    double a_t = norm;
    a_t = std_min(a_t, s.step_max);
    a_t = std_max(a_t, s.step_min);
    s.a_t = a_t;
    for (int i = 0; i < 6; ++i) s.x_t[i] = s.p[i] + s.dir[i] * a_t;
    set_pose(s, P);
    return request(s, P, kEvalFull, kPhaseMTFirst);
}

// Pose update and convergence test after a step (kernel.cpp:1246-1266).
// Returns true when the alignment is done.
__device__ bool newton_end(AlignState &s, const StepParams &P) {
    double dp[6];
    for (int i = 0; i < 6; ++i) dp[i] = s.dir[i] * s.a_t;
    for (int i = 0; i < 6; ++i) s.p[i] = s.p[i] + dp[i];
    if (s.nr_iterations > P.max_iterations || (s.nr_iterations && (fabs(s.a_t) < P.eps))) s.converged = 1;
    s.nr_iterations++;
    if (s.converged) {
        s.phase = kPhaseDone;
        s.eval_mode = kEvalNone;
        return true;
    }
    return false;
}

// Loop test of the line search (kernel.cpp:1076) and its next trial point
// (:1078-1099).  Returns true when an evaluation was requested.
__device__ bool mt_continue(AlignState &s, const StepParams &P) {
    if (!s.interval_converged && s.step_iterations < kMaxStepIterations &&
        !(s.psi_t <= 0 && s.d_phi_t <= -kNu * s.d_phi_0)) {
        double a_t;
        if (s.open_interval)
            a_t = trial_value(s.a_l, s.f_l, s.g_l, s.a_u, s.f_u, s.g_u, s.a_t, s.psi_t, s.d_psi_t);
        else
            a_t = trial_value(s.a_l, s.f_l, s.g_l, s.a_u, s.f_u, s.g_u, s.a_t, s.phi_t, s.d_phi_t);
        a_t = std_min(a_t, s.step_max);
        a_t = std_max(a_t, s.step_min);
        s.a_t = a_t;
        for (int i = 0; i < 6; ++i) s.x_t[i] = s.p[i] + s.dir[i] * a_t;
        set_pose(s, P);
        return request(s, P, kEvalGradient, kPhaseMTIter);
    }
    if (s.step_iterations) return request(s, P, kEvalHessian, kPhaseMTHess);  // computeHessian (:1141-1142)
    return false;
}

// Consume the evaluation result held in s.score/g/H and advance until the
// next evaluation is requested or the alignment is done.
__device__ void advance(AlignState &s, const StepParams &P) {
    int phase = s.phase;
    if (phase == kPhaseMTFirst || phase == kPhaseMTIter) {
        s.phi_t = -s.score;
        s.d_phi_t = -(dot6(s.g, s.dir));
        s.psi_t = psi_mt(s.a_t, s.phi_t, s.phi_0, s.d_phi_0, kMu);
        s.d_psi_t = dpsi_mt(s.d_phi_t, s.d_phi_0, kMu);
        if (phase == kPhaseMTIter) {
            if (s.open_interval && (s.psi_t <= 0 && s.d_psi_t >= 0)) {
                s.open_interval = 0;
                s.f_l = s.f_l + s.phi_0 - kMu * s.d_phi_0 * s.a_l;
                s.g_l = s.g_l + kMu * s.d_phi_0;
                s.f_u = s.f_u + s.phi_0 - kMu * s.d_phi_0 * s.a_u;
                s.g_u = s.g_u + kMu * s.d_phi_0;
            }
            bool ic;
            if (s.open_interval)
                ic = update_interval(s.a_l, s.f_l, s.g_l, s.a_u, s.f_u, s.g_u, s.a_t, s.psi_t, s.d_psi_t);
            else
                ic = update_interval(s.a_l, s.f_l, s.g_l, s.a_u, s.f_u, s.g_u, s.a_t, s.phi_t, s.d_phi_t);
            s.interval_converged = ic;
            s.step_iterations++;
        }
        if (mt_continue(s, P)) return;
        if (s.phase == kPhaseDone) return;
        if (newton_end(s, P)) return;
    } else if (phase == kPhaseMTHess) {
        if (newton_end(s, P)) return;
    } else if (phase != kPhaseInitEval) {
        return;
    }
    // bounded: each pass either requests an evaluation, finishes, or
    // completes a Newton iteration without one (d_phi_0 == 0)
    for (int guard = 0; guard < 1024; ++guard) {
        if (newton_start(s, P)) return;
        if (s.phase == kPhaseDone) return;
        if (newton_end(s, P)) return;
    }
    s.status = NDT_ST_WATCHDOG_DEV;
    s.converged = 0;
    s.phase = kPhaseDone;
    s.eval_mode = kEvalNone;
}

// One warp per alignment; lane 0 works on a shared-memory copy of the
// alignment's state (the state machine is serial FP64 code that touches
// hundreds of fields), and the warp moves the state between global and
// shared memory in 16-byte pieces.
constexpr int kStateWarps = 4;
constexpr int kStateVecs = (int)(sizeof(AlignState) / sizeof(uint4));
static_assert(sizeof(AlignState) % sizeof(uint4) == 0, "AlignState is copied in 16-byte pieces");

__device__ __forceinline__ void copy_state(AlignState *dst, const AlignState *src, int lane) {
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    for (int i = lane; i < kStateVecs; i += 32) d[i] = s[i];
}

__global__ void init_kernel(AlignState *__restrict__ states, const float *__restrict__ guesses,
                            const int *__restrict__ offsets, int B, StepParams P, double *__restrict__ exc) {
    __shared__ AlignState s_st[kStateWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.x * kStateWarps + warp;
    if (b >= B) return;
    for (int k = lane; k < kPartial; k += 32) exc[(size_t)b * kPartial + k] = 0.0;
    AlignState &s = s_st[warp];
    if (lane == 0) {
        for (int k = 0; k < 16; ++k) s.T[k] = guesses[16 * (size_t)b + k];
        pose_vector(P.compat != 0, s.T, s.p);
        if (!P.compat) build_tm_corrected(s.T, s.p);
        for (int i = 0; i < 6; ++i) {
            s.x_t[i] = s.p[i];
            s.dir[i] = 0.0;
            s.g[i] = 0.0;
        }
        for (int k = 0; k < 36; ++k) s.H[k] = 0.0;
        s.score = 0.0;
        s.phi_0 = s.d_phi_0 = s.a_l = s.f_l = s.g_l = s.a_u = s.f_u = s.g_u = s.a_t = 0.0;
        s.phi_t = s.d_phi_t = s.psi_t = s.d_psi_t = 0.0;
        s.step_max = P.step_max;
        s.step_min = P.step_min;
        s.nr_iterations = 0;
        s.step_iterations = 0;
        s.open_interval = 1;
        s.interval_converged = 0;
        s.converged = 0;
        s.evals = 0;
        s.status = 0;
        s.n = offsets[b + 1] - offsets[b];
        set_angles(s, s.p, P.compat);
        s.eval_mode = kEvalFull;
        s.phase = kPhaseInitEval;
    }
    __syncwarp();
    copy_state(states + b, &s, lane);
}

// FP64 sum of the alignment's chunk partials in chunk order (deterministic;
// each lane sums the values k = lane, lane + 32 with its loads issued 8 at a
// time), then lane 0 advances the state machine.
__global__ void step_kernel(AlignState *__restrict__ states, const double *__restrict__ partials,
                            const int *__restrict__ chunk_begin, double *__restrict__ exc, int B, StepParams P,
                            int *__restrict__ active, Counters *__restrict__ counters) {
    __shared__ double s_v[kStateWarps][kPartial];
    __shared__ AlignState s_st[kStateWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&counters->rounds, 1ull);
    const int b = blockIdx.x * kStateWarps + warp;
    if (b >= B) return;
    AlignState *st = states + b;
    const int mode = st->eval_mode;
    if (mode == kEvalNone) return;
    const int c0 = chunk_begin[b], c1 = chunk_begin[b + 1];
    for (int k = lane; k < kPartial; k += 32) {
        double v = 0.0;
        int c = c0;
        for (; c + 8 <= c1; c += 8) {
            double t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) t[u] = partials[(size_t)(c + u) * kPartial + k];
#pragma unroll
            for (int u = 0; u < 8; ++u) v += t[u];
        }
        for (; c < c1; ++c) v += partials[(size_t)c * kPartial + k];
        double *e = exc + (size_t)b * kPartial + k;
        v += *e;
        *e = 0.0;
        s_v[warp][k] = v;
    }
    AlignState &s = s_st[warp];
    copy_state(&s, st, lane);
    __syncwarp();
    if (lane == 0) {
        const double *v = s_v[warp];
        if (mode == kEvalFull || mode == kEvalGradient) {
            s.score = v[0];
            for (int i = 0; i < 6; ++i) s.g[i] = v[1 + i];
        }
        if (mode == kEvalFull || mode == kEvalHessian) {
            for (int k = 0; k < 36; ++k) s.H[k] = v[7 + k];
        } else {
            for (int k = 0; k < 36; ++k) s.H[k] = 0.0;  // computeDerivatives zeroes it (kernel.cpp:667)
        }
        s.evals++;
        s.eval_mode = kEvalNone;
        advance(s, P);
        if (s.eval_mode != kEvalNone) atomicAdd(active, 1);
        if (counters) atomicAdd(&counters->evaluations, 1ull);
    }
    __syncwarp();
    copy_state(st, &s, lane);
}

__global__ void finalize_kernel(const AlignState *__restrict__ states, int B, float *__restrict__ out,
                                int *__restrict__ conv, double *__restrict__ fit, int *__restrict__ status,
                                const int *__restrict__ overflow) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const AlignState &s = states[b];
    for (int k = 0; k < 16; ++k) out[16 * (size_t)b + k] = s.T[k];
    conv[b] = s.converged;
    fit[b] = s.n > 0 ? s.score / (double)s.n : 0.0;
    int st = s.status;
    if (s.phase != kPhaseDone && st == 0) st = NDT_ST_WATCHDOG_DEV;
    if (overflow && *overflow) st |= NDT_ST_OVERFLOW_DEV;
    if (status) status[b] = st;
}

// Chunk plan of an alignment with t tiles: large chunks of kb tiles over the
// first tiles, leaving at least 4 small chunks' worth (4 ks tiles, or all of
// them when t is smaller) for small chunks of ks tiles.
__device__ __forceinline__ void chunk_plan(int t, int kb, int ks, int &nb, int &ns) {
    const int keep = min(t, 4 * ks);
    nb = (t - keep) / kb;
    const int rest = t - nb * kb;
    ns = (rest + ks - 1) / ks;
}

// Tile list: ceil(n_b / tile) tiles per alignment, in alignment order; the
// large and small chunk counts per alignment.
__global__ void tile_count_kernel(const int *__restrict__ offsets, int B, int tile, int kb, int ks, TileLists L) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b > B) return;
    if (b == B) {
        L.tile_begin[B] = 0;
        L.big_begin[B] = 0;
        L.small_begin[B] = 0;
        return;
    }
    const int n = offsets[b + 1] - offsets[b];
    const int t = n > 0 ? (n + tile - 1) / tile : 0;
    int nb, ns;
    chunk_plan(t, kb, ks, nb, ns);
    L.tile_begin[b] = t;
    L.big_begin[b] = nb;
    L.small_begin[b] = ns;
}

// Exclusive scans in place of three arrays of n ints, one block of 1024
// threads per array (block k scans arrays[k], total to *totals[k]).
struct ScanArgs {
    int *data[3];
    int *total[3];
};

__global__ void scan3_kernel(ScanArgs a, int n) {
    __shared__ int s_warp[32];
    int *data = a.data[blockIdx.x];
    int *total = a.total[blockIdx.x];
    const int t = threadIdx.x, nt = blockDim.x;
    const int chunk = (n + nt - 1) / nt;
    const int lo = min(n, t * chunk), hi = min(n, lo + chunk);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += data[i];
    int lane = t & 31, w = t >> 5;
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        int v = (lane < (nt >> 5)) ? s_warp[lane] : 0;
        int inc2 = v;
        for (int o = 1; o < 32; o <<= 1) {
            int u = __shfl_up_sync(0xffffffffu, inc2, o);
            if (lane >= o) inc2 += u;
        }
        s_warp[lane] = inc2 - v;
    }
    __syncthreads();
    int run = s_warp[w] + incl - sum;
    for (int i = lo; i < hi; ++i) {
        int v = data[i];
        data[i] = run;
        run += v;
    }
    if (total && t == nt - 1) *total = run;
}

// One warp per alignment writes its tiles, its chunks (large ones at the
// front of the list, small ones after every large one) and its slot range.
__global__ void tile_fill_kernel(const int *__restrict__ offsets, int B, int tile, int kb, int ks, TileLists L) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= B) return;
    const int lo = offsets[warp], hi = offsets[warp + 1];
    const int t0 = L.tile_begin[warp], t1 = L.tile_begin[warp + 1];
    for (int t = t0 + lane; t < t1; t += 32) {
        Tile x;
        x.align = warp;
        x.start = lo + (t - t0) * tile;
        x.end = min(hi, x.start + tile);
        x.slot = t;
        L.tiles[t] = x;
    }
    const int b0 = L.big_begin[warp], nb = L.big_begin[warp + 1] - b0;
    const int s0 = L.small_begin[warp], ns = L.small_begin[warp + 1] - s0;
    const int slot0 = b0 + s0;
    const int total_big = *L.num_big;
    if (lane == 0) {
        L.chunk_begin[warp] = slot0;
        if (warp == B - 1) L.chunk_begin[B] = *L.num_chunks = slot0 + nb + ns;
    }
    for (int j = lane; j < nb + ns; j += 32) {
        Chunk x;
        x.align = warp;
        int pos;
        if (j < nb) {
            x.first = t0 + j * kb;
            x.end = x.first + kb;
            pos = b0 + j;
        } else {
            x.first = t0 + nb * kb + (j - nb) * ks;
            x.end = min(t1, x.first + ks);
            pos = total_big + s0 + (j - nb);
        }
        x.slot = slot0 + j;
        L.chunks[pos] = x;
    }
}

// One evaluation request at pose p (test hook: the caller supplies the
// transformed points, so T is the identity).
__global__ void prepare_eval_kernel(AlignState *__restrict__ s, const double *__restrict__ p6, int n,
                                    double *__restrict__ exc, int compat) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int k = 0; k < 16; ++k) s->T[k] = (k % 5 == 0) ? 1.0f : 0.0f;
    for (int i = 0; i < 6; ++i) s->x_t[i] = s->p[i] = p6[i];
    double a[kAngle];
    angle_terms(p6, a, compat != 0);
    for (int k = 0; k < kAngle; ++k) {
        s->angd[k] = a[k];
        s->angf[k] = (float)a[k];
    }
    s->n = n;
    s->eval_mode = kEvalFull;
    s->phase = kPhaseInitEval;
    for (int k = 0; k < kPartial; ++k) exc[k] = 0.0;
}

}  // namespace

int launch_prepare_eval(AlignState *d_state, const double *d_p6, int n, double *d_exc, int compat, cudaStream_t st) {
    prepare_eval_kernel<<<1, 32, 0, st>>>(d_state, d_p6, n, d_exc, compat);
    return (int)cudaGetLastError();
}

int launch_tiles(const int *d_offsets, int B, int tile, int kb, int ks, const TileLists &L, cudaStream_t st) {
    tile_count_kernel<<<(B + 1 + 255) / 256, 256, 0, st>>>(d_offsets, B, tile, kb, ks, L);
    ScanArgs a;
    a.data[0] = L.tile_begin;
    a.total[0] = L.num_tiles;
    a.data[1] = L.big_begin;
    a.total[1] = L.num_big;
    a.data[2] = L.small_begin;
    a.total[2] = nullptr;
    scan3_kernel<<<3, 1024, 0, st>>>(a, B + 1);
    tile_fill_kernel<<<(B * 32 + 255) / 256, 256, 0, st>>>(d_offsets, B, tile, kb, ks, L);
    return (int)cudaGetLastError();
}

int launch_init(AlignState *d_states, const float *d_guesses, const int *d_offsets, int B, const StepParams &P,
                double *d_exc, cudaStream_t st) {
    init_kernel<<<(B + kStateWarps - 1) / kStateWarps, 32 * kStateWarps, 0, st>>>(d_states, d_guesses, d_offsets, B,
                                                                                  P, d_exc);
    return (int)cudaGetLastError();
}

int launch_step(AlignState *d_states, const double *d_partials, const int *d_chunk_begin, double *d_exc, int B,
                const StepParams &P, int *d_active, Counters *d_counters, cudaStream_t st) {
    step_kernel<<<(B + kStateWarps - 1) / kStateWarps, 32 * kStateWarps, 0, st>>>(d_states, d_partials, d_chunk_begin,
                                                                                  d_exc, B, P, d_active, d_counters);
    return (int)cudaGetLastError();
}

// score[b] = the alignment's NDT score (sum over its chunk partials in chunk
// order, plus its FP64 side sum) after one derivative pass.
__global__ void score_kernel(const double *__restrict__ partials, const int *__restrict__ chunk_begin,
                             const double *__restrict__ exc, int B, double *__restrict__ score) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    double v = 0.0;
    for (int c = chunk_begin[b]; c < chunk_begin[b + 1]; ++c) v += partials[(size_t)c * kPartial];
    score[b] = v + exc[(size_t)b * kPartial];
}

int launch_score(const double *d_partials, const int *d_chunk_begin, const double *d_exc, int B, double *d_score,
                 cudaStream_t st) {
    score_kernel<<<(B + 127) / 128, 128, 0, st>>>(d_partials, d_chunk_begin, d_exc, B, d_score);
    return (int)cudaGetLastError();
}

int launch_finalize(const AlignState *d_states, int B, float *d_out, int *d_conv, double *d_fit, int *d_status,
                    const int *d_overflow, cudaStream_t st) {
    finalize_kernel<<<(B + 127) / 128, 128, 0, st>>>(d_states, B, d_out, d_conv, d_fit, d_status, d_overflow);
    return (int)cudaGetLastError();
}

}  // namespace ndt
