// Learned-init batched NDT: the network proposes, the NDT judges and refines
// (ndt_align_batch_learned_device; no counterpart in the reference, whose
// align call starts the NDT at the caller's guess: partial_points_callback,
// src/CPU/ndt_mapping/kernel.cpp:1405-1414).
//
// For B scans with guesses, against contexts `levels[0 .. L)` that hold the
// same map at coarse-to-fine resolutions:
//   1. starts: every guess is moved by a fixed pattern of K offsets (a
//      grid_xy x grid_xy grid of translations in the guess's heading frame
//      times grid_yaw yaw offsets; K = 1 is the guess alone);
//   2. proposals: the network runs `passes` times from each of the K x B
//      starts (each pass reads the previous proposal); the K starts of a
//      scan share its points (candidate c reads scan c % B);
//   3. the judge: the NDT score of every proposal and of the raw guess, on an
//      evenly strided subsample of each scan, with the map of
//      levels[judge_level], in one score pass over (K + 1) x B candidates;
//      each scan starts from its best-scoring candidate -- the raw guess
//      whenever no proposal scores higher (the fallback);
//   4. refinement: the plain NDT from that start through every level in
//      order, each level starting at the previous level's result; the last
//      level's result is the output.
// Each step is enqueued on the stream of the object that does it (the
// network's stream, then the contexts' streams), ordered by events; nothing
// waits on the host.  Buffers are kept by the network object and only grow.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/ndt_b200.h"
#include "ctx_view.h"
#include "mlp_internal.h"

namespace {

struct Buf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(256, bytes + bytes / 4);
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    template <class T>
    T *as() const {
        return reinterpret_cast<T *>(p);
    }
};

}  // namespace

struct LearnedBuffers {
    Buf h_points, h_offsets, h_guesses, h_out, h_conv, h_fit, h_status, h_choice;  // device copies of host batches
    Buf starts, y, cand, scores, start, choice_tmp;
    Buf judge_count, judge_prefix, judge_dec, rep, rep_off;
    Buf lvl_count[NDT_LEARNED_MAX_LEVELS], lvl_prefix[NDT_LEARNED_MAX_LEVELS], lvl_dec[NDT_LEARNED_MAX_LEVELS];
    Buf out[NDT_LEARNED_MAX_LEVELS], conv[NDT_LEARNED_MAX_LEVELS], fit[NDT_LEARNED_MAX_LEVELS],
        status[NDT_LEARNED_MAX_LEVELS];
};

void learned_buffers_free(LearnedBuffers *lb) {
    if (!lb) return;
    Buf *all[] = {&lb->h_points, &lb->h_offsets, &lb->h_guesses, &lb->h_out, &lb->h_conv, &lb->h_fit,
                  &lb->h_status, &lb->h_choice, &lb->starts, &lb->y, &lb->cand, &lb->scores, &lb->start, &lb->choice_tmp, &lb->judge_count,
                  &lb->judge_prefix, &lb->judge_dec, &lb->rep, &lb->rep_off};
    for (Buf *b : all)
        if (b->p) cudaFree(b->p);
    for (int l = 0; l < NDT_LEARNED_MAX_LEVELS; ++l) {
        Buf *per[] = {&lb->lvl_count[l], &lb->lvl_prefix[l], &lb->lvl_dec[l], &lb->out[l], &lb->conv[l],
                      &lb->fit[l], &lb->status[l]};
        for (Buf *b : per)
            if (b->p) cudaFree(b->p);
    }
    delete lb;
}

namespace {

// counts[b] = min(n_b, cap), n_b = the scan's point count (cap <= 0: n_b).
__global__ void sub_count_kernel(const int *__restrict__ offsets, int B, int cap, int *__restrict__ counts) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const int n = offsets[b + 1] - offsets[b];
    counts[b] = (cap > 0 && n > cap) ? cap : n;
}

// prefix[0..B] = exclusive prefix sums of counts (one block of 1024 threads;
// each thread sums a contiguous run, the block scans the run totals).
__global__ void prefix_kernel(const int *__restrict__ counts, int B, int *__restrict__ prefix) {
    __shared__ int s_warp[32];
    const int t = threadIdx.x, nt = blockDim.x, lane = t & 31, w = t >> 5;
    const int chunk = (B + nt - 1) / nt;
    const int lo = min(B, t * chunk), hi = min(B, lo + chunk);
    int sum = 0;
    for (int i = lo; i < hi; ++i) sum += counts[i];
    int incl = sum;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int v = lane < (nt >> 5) ? s_warp[lane] : 0;
        int inc2 = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, inc2, o);
            if (lane >= o) inc2 += u;
        }
        s_warp[lane] = inc2 - v;
    }
    __syncthreads();
    int run = s_warp[w] + incl - sum;
    for (int i = lo; i < hi; ++i) {
        prefix[i] = run;
        run += counts[i];
    }
    if (t == nt - 1) prefix[B] = run;
}

// The evenly strided subsample of every scan (one block per scan): point j of
// m_b = prefix[b + 1] - prefix[b] is point (j * n_b) / m_b of the scan.
__global__ void subsample_kernel(const float4 *__restrict__ pts, const int *__restrict__ offsets,
                                 const int *__restrict__ prefix, float4 *__restrict__ out) {
    const int b = blockIdx.x;
    const int s = offsets[b], n = offsets[b + 1] - s;
    const int o = prefix[b], m = prefix[b + 1] - o;
    for (int j = threadIdx.x; j < m; j += blockDim.x) out[o + j] = pts[s + (int)(((long long)j * n) / m)];
}

// Candidate c of C = (K + 1) B reads scan c % B: its subsample copied to its
// own range of `rep` (the score pass takes one point range per candidate).
__global__ void replicate_kernel(const float4 *__restrict__ sub, const int *__restrict__ prefix, int B, int C,
                                 float4 *__restrict__ rep, int *__restrict__ rep_off) {
    const int c = blockIdx.x;
    const int b = c % B, k = c / B;
    const int S = prefix[B];
    const int src = prefix[b], m = prefix[b + 1] - src;
    const long long dst = (long long)k * S + src;
    if (threadIdx.x == 0) {
        rep_off[c] = (int)dst;
        if (c == C - 1) rep_off[C] = (int)((long long)(k + 1) * S);
    }
    for (int j = threadIdx.x; j < m; j += blockDim.x) rep[dst + j] = sub[src + j];
}

// Start k of scan b (candidate k B + b): the guess moved by the k-th offset
// of the pattern, translations in the guess's heading frame.
__global__ void start_kernel(const float *__restrict__ guesses, int B, int gxy, int gyaw, float step_xy,
                             float step_yaw, float *__restrict__ starts) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    const int K = gxy * gxy * gyaw;
    if (c >= K * B) return;
    const int b = c % B, k = c / B;
    const int iyaw = k % gyaw, ixy = k / gyaw;
    const int ix = ixy % gxy, iy = ixy / gxy;
    const double dx = (ix - 0.5 * (gxy - 1)) * (double)step_xy;
    const double dy = (iy - 0.5 * (gxy - 1)) * (double)step_xy;
    const double dyaw = (iyaw - 0.5 * (gyaw - 1)) * (double)step_yaw;
    double p[6];
    pn::pose_of(guesses + 16 * (size_t)b, p);
    double s, co;
    sincos(p[5], &s, &co);
    p[0] += co * dx - s * dy;
    p[1] += s * dx + co * dy;
    p[5] += dyaw;
    pn::matrix_of(p, starts + 16 * (size_t)c);
}

// The judge: scan b starts from its best-scoring candidate (ties: the lower
// index; NaN scores never win); candidate K, the raw guess, when no proposal
// scores higher.
__global__ void select_kernel(const float *__restrict__ cand, const double *__restrict__ scores, int B, int K,
                              float *__restrict__ start, int *__restrict__ choice) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    int best = K;
    double bs = scores[(size_t)K * B + b];
    for (int k = 0; k < K; ++k) {
        const double v = scores[(size_t)k * B + b];
        if (v > bs || (bs != bs && v == v)) {
            bs = v;
            best = k;
        }
    }
    const float *src = cand + 16 * ((size_t)best * B + b);
    for (int i = 0; i < 16; ++i) start[16 * (size_t)b + i] = src[i];
    if (choice) choice[b] = best;
}

// status[b] = OR of the levels' statuses.
struct StatusList {
    const int *s[NDT_LEARNED_MAX_LEVELS];
    int n;
};

__global__ void status_or_kernel(StatusList L, int B, int *__restrict__ out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    int v = 0;
    for (int l = 0; l < L.n; ++l) v |= L.s[l][b];
    out[b] = v;
}

int fail(ndt_mlp *c, int code, const char *msg) {
    c->msg = msg;
    return code;
}

int cuda_fail(ndt_mlp *c, cudaError_t e, const char *what) {
    c->msg = std::string(what) + ": " + cudaGetErrorString(e);
    return NDT_E_CUDA;
}

#define LCK(call)                                             \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
    } while (0)

// Subsample (cap points per scan, evenly strided) of the B scans into `dec`
// with prefix offsets `prefix`; returns the host-side upper bound of its
// point count in *bound.
int subsample(ndt_mlp *c, cudaStream_t st, const float *d_points, const int *d_offsets, int B, int cap,
              Buf &count, Buf &prefix, Buf &dec, long long total, long long *bound) {
    const long long ub = cap > 0 ? std::min<long long>(total, (long long)cap * B) : total;
    LCK(count.ensure(sizeof(int) * (size_t)B));
    LCK(prefix.ensure(sizeof(int) * (size_t)(B + 1)));
    LCK(dec.ensure(sizeof(float4) * (size_t)std::max<long long>(1, ub)));
    sub_count_kernel<<<(B + 255) / 256, 256, 0, st>>>(d_offsets, B, cap, count.as<int>());
    prefix_kernel<<<1, 1024, 0, st>>>(count.as<int>(), B, prefix.as<int>());
    subsample_kernel<<<B, 256, 0, st>>>(reinterpret_cast<const float4 *>(d_points), d_offsets, prefix.as<int>(),
                                        dec.as<float4>());
    LCK(cudaGetLastError());
    *bound = ub;
    return NDT_OK;
}

}  // namespace

extern "C" {

void ndt_learned_params_default(ndt_learned_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->max_points = 1024;
    p->passes = 2;
    p->grid_xy = 3;
    p->grid_yaw = 3;
    p->step_xy = 2.5f;
    p->step_yaw_deg = 10.0f;
    p->judge_level = 0;
    p->judge_points = 2048;
}

int ndt_align_batch_learned_device(ndt_mlp *c, ndt_ctx *const *levels, int n_levels, const ndt_learned_params *lp,
                                   int B, const float *d_points, const int *d_offsets, int total_points,
                                   const float *d_guesses, float *d_out, int *d_conv, double *d_fit, int *d_status,
                                   int *d_choice, float *d_start16) {
    if (!c) return NDT_E_ARG;
    if (!levels || n_levels < 1 || n_levels > NDT_LEARNED_MAX_LEVELS || !lp || B <= 0 || total_points < 0 ||
        !d_points || !d_offsets || !d_guesses || !d_out || !d_conv || !d_fit)
        return fail(c, NDT_E_ARG, "ndt_align_batch_learned_device: bad argument");
    if (lp->max_points <= 0 || lp->passes < 0 || lp->grid_xy < 1 || lp->grid_yaw < 1 || lp->judge_level < 0 ||
        lp->judge_level >= n_levels || lp->judge_points < 0)
        return fail(c, NDT_E_ARG, "ndt_align_batch_learned_device: bad learned parameters");
    const int K = lp->grid_xy * lp->grid_xy * lp->grid_yaw;
    const long long C = (long long)(K + 1) * B;
    if (C > (1LL << 30)) return fail(c, NDT_E_CAPACITY, "ndt_align_batch_learned_device: too many candidates");
    cudaStream_t s_lvl[NDT_LEARNED_MAX_LEVELS];
    for (int l = 0; l < n_levels; ++l) {
        ndt::CtxEvalView v;
        if (!levels[l] || ndt::ctx_eval_view(levels[l], &v) != 0)
            return fail(c, NDT_E_ARG, "ndt_align_batch_learned_device: null level context");
        if (!v.have_map) return fail(c, NDT_E_NOMAP, "ndt_align_batch_learned_device: a level has no map");
        if (v.device != c->device)
            return fail(c, NDT_E_ARG, "ndt_align_batch_learned_device: contexts and network on different devices");
        s_lvl[l] = v.stream;
    }
    LCK(cudaSetDevice(c->device));
    for (int i = 0; i < kMlpEvents; ++i)
        if (!c->ev[i]) LCK(cudaEventCreateWithFlags(&c->ev[i], cudaEventDisableTiming));
    if (!c->lb) c->lb = new LearnedBuffers();
    LearnedBuffers &lb = *c->lb;
    const cudaStream_t s_net = c->stream;

    // the previous call's work on the levels' streams reads buffers this call rewrites
    for (int l = 0; l < n_levels; ++l) {
        LCK(cudaEventRecord(c->ev[1 + l], s_lvl[l]));
        LCK(cudaStreamWaitEvent(s_net, c->ev[1 + l], 0));
    }

    // 1-2. starts and the network's proposals (candidates 0 .. K B), then the raw guesses (K B .. (K + 1) B)
    LCK(lb.starts.ensure(sizeof(float) * 16 * (size_t)K * B));
    LCK(lb.y.ensure(sizeof(float) * 6 * (size_t)K * B));
    LCK(lb.cand.ensure(sizeof(float) * 16 * (size_t)C));
    float *cand = lb.cand.as<float>();
    start_kernel<<<(int)((K * (long long)B + 127) / 128), 128, 0, s_net>>>(
        d_guesses, B, lp->grid_xy, lp->grid_yaw, lp->step_xy, (float)(lp->step_yaw_deg * (3.14159265358979323846 / 180.0)),
        lb.starts.as<float>());
    LCK(cudaGetLastError());
    if (lp->passes > 0) {
        if (int rc = mlp_propose(c, K * B, B, d_points, d_offsets, lb.starts.as<float>(), lp->max_points, lp->passes,
                                 lb.y.as<float>(), cand))
            return rc;
    } else {
        LCK(cudaMemcpyAsync(cand, lb.starts.p, sizeof(float) * 16 * (size_t)K * B, cudaMemcpyDeviceToDevice, s_net));
    }
    LCK(cudaMemcpyAsync(cand + 16 * (size_t)K * B, d_guesses, sizeof(float) * 16 * (size_t)B,
                        cudaMemcpyDeviceToDevice, s_net));

    // 3. the judge's subsample, one copy per candidate
    long long judge_bound = 0;
    if (int rc = subsample(c, s_net, d_points, d_offsets, B, lp->judge_points, lb.judge_count, lb.judge_prefix,
                           lb.judge_dec, total_points, &judge_bound))
        return rc;
    const long long rep_bound = judge_bound * (K + 1);
    if (rep_bound >= (1LL << 31)) return fail(c, NDT_E_CAPACITY, "ndt_align_batch_learned_device: judge subsample "
                                                                 "too large (lower judge_points)");
    LCK(lb.rep.ensure(sizeof(float4) * (size_t)std::max<long long>(1, rep_bound)));
    LCK(lb.rep_off.ensure(sizeof(int) * (size_t)(C + 1)));
    replicate_kernel<<<(int)C, 256, 0, s_net>>>(lb.judge_dec.as<float4>(), lb.judge_prefix.as<int>(), B, (int)C,
                                                lb.rep.as<float4>(), lb.rep_off.as<int>());
    LCK(cudaGetLastError());
    // subsamples of the refinement levels that read fewer points
    const float *lvl_pts[NDT_LEARNED_MAX_LEVELS];
    const int *lvl_off[NDT_LEARNED_MAX_LEVELS];
    int lvl_total[NDT_LEARNED_MAX_LEVELS];
    for (int l = 0; l < n_levels; ++l) {
        const int cap = lp->level_points[l];
        if (cap <= 0) {
            lvl_pts[l] = d_points;
            lvl_off[l] = d_offsets;
            lvl_total[l] = total_points;
            continue;
        }
        long long bound = 0;
        if (int rc = subsample(c, s_net, d_points, d_offsets, B, cap, lb.lvl_count[l], lb.lvl_prefix[l],
                               lb.lvl_dec[l], total_points, &bound))
            return rc;
        lvl_pts[l] = lb.lvl_dec[l].as<float>();
        lvl_off[l] = lb.lvl_prefix[l].as<int>();
        lvl_total[l] = (int)bound;
    }
    LCK(cudaEventRecord(c->ev[0], s_net));

    // 3. scores of all candidates at the judge level, then the choice
    const int J = lp->judge_level;
    LCK(cudaStreamWaitEvent(s_lvl[J], c->ev[0], 0));
    LCK(lb.scores.ensure(sizeof(double) * (size_t)C));
    LCK(lb.start.ensure(sizeof(float) * 16 * (size_t)B));
    if (int rc = ndt_score_batch_device(levels[J], (int)C, lb.rep.as<float>(), lb.rep_off.as<int>(), (int)rep_bound,
                                        cand, lb.scores.as<double>())) {
        c->msg = std::string("judge: ") + ndt_last_error(levels[J]);
        return rc;
    }
    select_kernel<<<(B + 127) / 128, 128, 0, s_lvl[J]>>>(cand, lb.scores.as<double>(), B, K, lb.start.as<float>(),
                                                         d_choice);
    LCK(cudaGetLastError());
    if (d_start16)
        LCK(cudaMemcpyAsync(d_start16, lb.start.p, sizeof(float) * 16 * (size_t)B, cudaMemcpyDeviceToDevice,
                            s_lvl[J]));
    // a stream's wait takes the event's latest record at the time of the
    // wait, so one event carries the order from each step to the next
    const cudaEvent_t prev = c->ev[kMlpEvents - 1];
    LCK(cudaEventRecord(prev, s_lvl[J]));

    // 4. refinement through the levels
    StatusList sl;
    sl.n = n_levels;
    const float *cur = lb.start.as<float>();
    for (int l = 0; l < n_levels; ++l) {
        const bool last = l == n_levels - 1;
        LCK(lb.status[l].ensure(sizeof(int) * (size_t)B));
        if (!last) {
            LCK(lb.out[l].ensure(sizeof(float) * 16 * (size_t)B));
            LCK(lb.conv[l].ensure(sizeof(int) * (size_t)B));
            LCK(lb.fit[l].ensure(sizeof(double) * (size_t)B));
        }
        float *o = last ? d_out : lb.out[l].as<float>();
        int *cv = last ? d_conv : lb.conv[l].as<int>();
        double *ft = last ? d_fit : lb.fit[l].as<double>();
        LCK(cudaStreamWaitEvent(s_lvl[l], prev, 0));
        if (int rc = ndt_align_batch_device(levels[l], B, lvl_pts[l], lvl_off[l], lvl_total[l], cur, o, cv, ft,
                                            lb.status[l].as<int>())) {
            c->msg = std::string("refinement: ") + ndt_last_error(levels[l]);
            return rc;
        }
        sl.s[l] = lb.status[l].as<int>();
        cur = o;
        if (!last) LCK(cudaEventRecord(prev, s_lvl[l]));
    }
    if (d_status) {
        status_or_kernel<<<(B + 127) / 128, 128, 0, s_lvl[n_levels - 1]>>>(sl, B, d_status);
        LCK(cudaGetLastError());
    }
    return NDT_OK;
}

int ndt_align_batch_learned(ndt_mlp *c, ndt_ctx *const *levels, int n_levels, const ndt_learned_params *lp, int B,
                            const float *points, const int *offsets, const float *guesses, float *out, int *conv,
                            double *fit, int *status, int *choice, float *start16) {
    if (!c) return NDT_E_ARG;
    if (!levels || n_levels < 1 || n_levels > NDT_LEARNED_MAX_LEVELS || B <= 0 || !points || !offsets || !guesses ||
        !out || !conv || !fit)
        return fail(c, NDT_E_ARG, "ndt_align_batch_learned: bad argument");
    if (offsets[0] != 0) return fail(c, NDT_E_ARG, "ndt_align_batch_learned: offsets[0] must be 0");
    for (int b = 0; b < B; ++b)
        if (offsets[b + 1] < offsets[b]) return fail(c, NDT_E_ARG, "ndt_align_batch_learned: decreasing offsets");
    const int total = offsets[B];
    ndt::CtxEvalView v;
    if (!levels[n_levels - 1] || ndt::ctx_eval_view(levels[n_levels - 1], &v) != 0)
        return fail(c, NDT_E_ARG, "ndt_align_batch_learned: null level context");
    const cudaStream_t s_last = v.stream;
    LCK(cudaSetDevice(c->device));
    if (!c->lb) c->lb = new LearnedBuffers();
    LearnedBuffers &lb = *c->lb;
    // the previous call's read-back must be done before its buffers are refilled
    LCK(cudaStreamSynchronize(s_last));
    LCK(lb.h_points.ensure(sizeof(float4) * (size_t)std::max(1, total)));
    LCK(lb.h_offsets.ensure(sizeof(int) * (size_t)(B + 1)));
    LCK(lb.h_guesses.ensure(sizeof(float) * 16 * (size_t)B));
    LCK(lb.h_out.ensure(sizeof(float) * 16 * (size_t)B));
    LCK(lb.h_conv.ensure(sizeof(int) * (size_t)B));
    LCK(lb.h_fit.ensure(sizeof(double) * (size_t)B));
    LCK(lb.h_status.ensure(sizeof(int) * (size_t)B));
    LCK(lb.h_choice.ensure(sizeof(int) * (size_t)B));
    const cudaStream_t s_net = c->stream;
    LCK(cudaMemcpyAsync(lb.h_points.p, points, sizeof(float4) * (size_t)total, cudaMemcpyHostToDevice, s_net));
    LCK(cudaMemcpyAsync(lb.h_offsets.p, offsets, sizeof(int) * (size_t)(B + 1), cudaMemcpyHostToDevice, s_net));
    LCK(cudaMemcpyAsync(lb.h_guesses.p, guesses, sizeof(float) * 16 * (size_t)B, cudaMemcpyHostToDevice, s_net));
    if (int rc = ndt_align_batch_learned_device(c, levels, n_levels, lp, B, lb.h_points.as<float>(),
                                                lb.h_offsets.as<int>(), total, lb.h_guesses.as<float>(),
                                                lb.h_out.as<float>(), lb.h_conv.as<int>(), lb.h_fit.as<double>(),
                                                lb.h_status.as<int>(), lb.h_choice.as<int>(), nullptr))
        return rc;
    LCK(cudaMemcpyAsync(out, lb.h_out.p, sizeof(float) * 16 * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    LCK(cudaMemcpyAsync(conv, lb.h_conv.p, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    LCK(cudaMemcpyAsync(fit, lb.h_fit.p, sizeof(double) * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    if (status)
        LCK(cudaMemcpyAsync(status, lb.h_status.p, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    if (choice)
        LCK(cudaMemcpyAsync(choice, lb.h_choice.p, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    if (start16)
        LCK(cudaMemcpyAsync(start16, lb.start.p, sizeof(float) * 16 * (size_t)B, cudaMemcpyDeviceToHost, s_last));
    LCK(cudaStreamSynchronize(s_last));
    return NDT_OK;
}

}  // extern "C"
