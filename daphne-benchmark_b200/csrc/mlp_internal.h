// Internals shared by the point-feature network (posenet.cu) and the
// learned-init alignment pipeline (learned_pipeline.cu): the network object
// behind the C ABI's ndt_mlp handle, its input frame, and the FP64 pose
// helpers of the corrected parametrisation T = Trans Rx Ry Rz.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/ndt_b200.h"

namespace pn {

constexpr unsigned kWaitLimit = 1u << 26;  // bounded mbarrier wait (error flag when exceeded)

struct Norm {
    float cx, cy, cz, inv_s;  // input centring and scale
    float dscale[6];          // pose-correction units
};

// Pose vector (x, y, z, roll, pitch, yaw) of T = Trans Rx Ry Rz and back, FP64.
__device__ __forceinline__ void pose_of(const float *T, double p[6]) {
    p[0] = T[3];
    p[1] = T[7];
    p[2] = T[11];
    p[3] = atan2(-(double)T[6], (double)T[10]);
    p[4] = asin(fmin(1.0, fmax(-1.0, (double)T[2])));
    p[5] = atan2(-(double)T[1], (double)T[0]);
}

__device__ __forceinline__ void matrix_of(const double p[6], float *T) {
    double sa, ca, sb, cb, sc, cc;
    sincos(p[3], &sa, &ca);
    sincos(p[4], &sb, &cb);
    sincos(p[5], &sc, &cc);
    T[0] = (float)(cb * cc);
    T[1] = (float)(-cb * sc);
    T[2] = (float)sb;
    T[3] = (float)p[0];
    T[4] = (float)(ca * sc + sa * sb * cc);
    T[5] = (float)(ca * cc - sa * sb * sc);
    T[6] = (float)(-sa * cb);
    T[7] = (float)p[1];
    T[8] = (float)(sa * sc - ca * sb * cc);
    T[9] = (float)(sa * cc + ca * sb * sc);
    T[10] = (float)(ca * cb);
    T[11] = (float)p[2];
    T[12] = T[13] = T[14] = 0.0f;
    T[15] = 1.0f;
}

}  // namespace pn

struct LearnedBuffers;  // device buffers of the learned-init pipeline (learned_pipeline.cu)
void learned_buffers_free(LearnedBuffers *lb);

constexpr int kMlpEvents = NDT_LEARNED_MAX_LEVELS + 2;  // events that order the pipeline's streams

struct ndt_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;  // created with the network; `stream` may be a caller's
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    uint8_t *w2op = nullptr;
    int *err = nullptr;
    unsigned long long *gmax = nullptr;
    float *grad_scan = nullptr, *loss_scan = nullptr;
    float *dg = nullptr;         // B x 128: the head's gradient at the max-pooled features
    float *head_part = nullptr;  // per 128-scan tile: the head's weight and bias gradient sums
    size_t cap_b = 0;
    int step = 0;
    pn::Norm nm{};
    unsigned wait_limit = pn::kWaitLimit;
    LearnedBuffers *lb = nullptr;
    cudaEvent_t ev[kMlpEvents] = {};
    std::string msg;
};

// The network on B candidates (pose guesses) whose scans are shared: candidate
// b reads scan b % scans of (d_points, d_offsets).  mlp_forward writes y (B x
// 6); mlp_propose runs `passes` forward passes, each applied to the previous
// proposal, and writes the last proposals (B x 16) and y.  Work goes to the
// network's stream.
int mlp_forward(ndt_mlp *c, int B, int scans, const float *d_points, const int *d_offsets, const float *d_guesses,
                int max_points, float *d_y6);
int mlp_propose(ndt_mlp *c, int B, int scans, const float *d_points, const int *d_offsets, const float *d_guesses,
                int max_points, int passes, float *d_y6, float *d_prop16);
