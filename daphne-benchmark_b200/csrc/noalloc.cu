// ndt_derivatives_noalloc: one derivative evaluation (score, gradient,
// Hessian of one scan against the context's voxel grid) that allocates no
// memory at call time.
//
// Who needs it: callers that must not allocate device memory while they
// run -- a real-time control loop with a fixed memory budget (cudaMalloc can
// block, synchronise the device and take unbounded time), or code that runs
// while another component owns the device's memory and has handed out all of
// it.  They set up a context and its map beforehand, then call this as often
// as they like.
//
// Its scratch memory (tile and chunk lists, one alignment state, per-chunk
// partial sums, the FP64 side queue, counters) is the file-scope array
// ndt_noalloc_scratch below, sized for at most kNoAllocMaxPoints scan points.
// Every GPU that loads this library holds that array (at most 256 KB) until
// the process exits.  Host code cannot take the array's address directly (in
// host code the symbol is a host-side stand-in); the first call on each
// device, with that device current, looks the device address up with
// cudaGetSymbolAddress and caches it -- make that first call before any
// stream capture.
//
// Every call shares the one array and keeps the previous call's contents:
// each call clears what must start at zero before it runs, and two calls whose
// work overlaps on the GPU (different streams, or contexts on different host
// threads using the same device) race on it.  Calls on one context's stream
// are ordered and do not overlap.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "../../include/ndt_b200.h"
#include "align.h"
#include "ctx_view.h"
#include "derivatives.h"
#include "ndt_math.cuh"

namespace ndt {
namespace {

constexpr int kNoAllocMaxPoints = 65536;
constexpr int kNoAllocMaxTiles = kNoAllocMaxPoints / 128 + 2;  // smallest tile: 128 points
constexpr unsigned kNoAllocFlagCap = 2048;

// Layout of the scratch array.
struct NoAllocScratch {
    AlignState state;
    Counters counters;
    int offsets[2];
    int tile_begin[2];
    int num_tiles;
    int chunk_begin[2];
    int num_chunks;
    int big_begin[2];
    int small_begin[2];
    int num_big;
    unsigned flag_n;
    int flag_overflow;
    int work_counter;
    double exc[kPartial];
    Tile tiles[kNoAllocMaxTiles];
    Chunk chunks[kNoAllocMaxTiles];
    int4 flag_q[kNoAllocFlagCap];
    double partials[kNoAllocMaxTiles * kPartial];
};

constexpr size_t kNoAllocScratchBytes = (sizeof(NoAllocScratch) + 255) & ~(size_t)255;
static_assert(kNoAllocScratchBytes <= 256 * 1024, "the static scratch is documented as at most 256 KB");

static __device__ __align__(256) unsigned char ndt_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices];  // device address of ndt_noalloc_scratch, per device

// Clears the zero-initialised parts and sets the one evaluation request:
// transformed points given by the caller (T unused), angle terms of p.
struct Pose6 {
    double p[6];
};

__global__ void noalloc_setup_kernel(NoAllocScratch *s, Pose6 pose, int n, int compat) {
    const int t = threadIdx.x;
    if (t < kPartial) s->exc[t] = 0.0;
    if (t == 0) {
        s->counters.evaluations = s->counters.points = s->counters.probes = 0;
        s->counters.occupied_probes = s->counters.pairs = s->counters.tiles = s->counters.rounds = 0;
        s->offsets[0] = 0;
        s->offsets[1] = n;
        s->flag_n = 0;
        s->flag_overflow = 0;
        AlignState &st = s->state;
        for (int k = 0; k < 16; ++k) st.T[k] = (k % 5 == 0) ? 1.0f : 0.0f;
        for (int i = 0; i < 6; ++i) st.x_t[i] = st.p[i] = pose.p[i];
        double a[kAngle];
        angle_terms(pose.p, a, compat != 0);
        for (int k = 0; k < kAngle; ++k) {
            st.angd[k] = a[k];
            st.angf[k] = (float)a[k];
        }
        st.n = n;
        st.eval_mode = kEvalFull;
        st.phase = kPhaseInitEval;
    }
}

// out[k] = sum over chunks (in chunk order) + side sums; out[43] = pairs, or -1
// when the FP64 side queue overflowed.
__global__ void noalloc_reduce_kernel(const NoAllocScratch *s, double *out) {
    const int k = threadIdx.x;
    if (k >= kPartial) return;
    double v = 0.0;
    for (int t = 0; t < s->num_chunks; ++t) v += s->partials[(size_t)t * kPartial + k];
    v += s->exc[k];
    if (k == kPartial - 1 && (s->flag_overflow || s->flag_n > kNoAllocFlagCap)) v = -1.0;
    out[k] = v;
}

// Makes `device` current for its lifetime and puts the caller's current
// device back when it ends, so that the call leaves the calling thread's
// device selection as it found it.
class DeviceGuard {
public:
    explicit DeviceGuard(int device) {
        if (cudaGetDevice(&prev_) != cudaSuccess) prev_ = -1;
        err_ = (prev_ == device) ? cudaSuccess : cudaSetDevice(device);
    }
    ~DeviceGuard() {
        if (prev_ >= 0 && err_ == cudaSuccess) cudaSetDevice(prev_);
    }
    cudaError_t error() const { return err_; }

private:
    int prev_ = -1;
    cudaError_t err_ = cudaSuccess;
};

}  // namespace
}  // namespace ndt

using namespace ndt;

extern "C" int ndt_derivatives_noalloc(ndt_ctx *ctx, const float *d_scan, const float *d_trans, int n,
                                       const double p6[6], double *d_out) {
    CtxEvalView v;
    if (!ctx || !d_scan || !d_trans || !p6 || !d_out || n <= 0) {
        ctx_set_error(ctx, "ndt_derivatives_noalloc: null pointer or empty scan");
        return NDT_E_ARG;
    }
    ctx_eval_view(ctx, &v);
    if (!v.have_map) {
        ctx_set_error(ctx, "ndt_derivatives_noalloc: no map set");
        return NDT_E_NOMAP;
    }
    if (n > kNoAllocMaxPoints) {
        ctx_set_error(ctx, "ndt_derivatives_noalloc: more than 65536 scan points (the static scratch limit)");
        return NDT_E_CAPACITY;
    }
    // The kernels read the scans as float4 and write d_out as doubles: a
    // misaligned pointer would fault on the device, so it is refused here.
    if ((reinterpret_cast<uintptr_t>(d_scan) | reinterpret_cast<uintptr_t>(d_trans)) & 15u ||
        reinterpret_cast<uintptr_t>(d_out) & 7u) {
        ctx_set_error(ctx, "ndt_derivatives_noalloc: d_scan and d_trans must be 16-byte aligned, d_out 8-byte aligned");
        return NDT_E_ARG;
    }
    if (v.device < 0 || v.device >= kMaxDevices) {
        ctx_set_error(ctx, "ndt_derivatives_noalloc: device ordinal out of range");
        return NDT_E_ARG;
    }
    DeviceGuard guard(v.device);
    cudaError_t e = guard.error();
    if (e != cudaSuccess) {
        ctx_set_error(ctx, cudaGetErrorString(e));
        return NDT_E_CUDA;
    }
    void *addr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_scratch_addr[v.device]) {
            e = cudaGetSymbolAddress(&g_scratch_addr[v.device], ndt_noalloc_scratch);
            if (e != cudaSuccess) {
                g_scratch_addr[v.device] = nullptr;
                ctx_set_error(ctx, cudaGetErrorString(e));
                return NDT_E_CUDA;
            }
        }
        addr = g_scratch_addr[v.device];
    }
    NoAllocScratch *s = reinterpret_cast<NoAllocScratch *>(addr);
    const cudaStream_t st = v.stream;
    const int tile = v.precision == 1 ? kTile : kDerivVariants[v.variant].tile;
    Pose6 pose;
    for (int i = 0; i < 6; ++i) pose.p[i] = p6[i];
    noalloc_setup_kernel<<<1, 64, 0, st>>>(s, pose, n, v.compat);
    TileLists L;
    L.tile_begin = s->tile_begin;
    L.tiles = s->tiles;
    L.num_tiles = &s->num_tiles;
    L.chunk_begin = s->chunk_begin;
    L.chunks = s->chunks;
    L.num_chunks = &s->num_chunks;
    L.big_begin = s->big_begin;
    L.small_begin = s->small_begin;
    L.num_big = &s->num_big;
    const bool f64 = v.precision == 1;
    int rc = launch_tiles(s->offsets, 1, tile, f64 ? 1 : kChunkBig, f64 ? 1 : kChunkSmall, L, st);
    if (rc) {
        ctx_set_error(ctx, cudaGetErrorString((cudaError_t)rc));
        return NDT_E_CUDA;
    }
    EvalArgs ea;
    ea.grid = v.grid;
    ea.points = reinterpret_cast<const float4 *>(d_scan);
    ea.trans = reinterpret_cast<const float4 *>(d_trans);
    ea.tiles = s->tiles;
    ea.num_tiles = &s->num_tiles;
    ea.chunks = s->chunks;
    ea.num_chunks = &s->num_chunks;
    ea.max_tiles = n / tile + 2;
    ea.tile_size = tile;
    ea.states = &s->state;
    ea.partials = s->partials;
    ea.exc = s->exc;
    ea.d1 = v.d1;
    ea.d2 = v.d2;
    ea.compat = v.compat;
    ea.counters = &s->counters;
    ea.flag_q = s->flag_q;
    ea.flag_n = &s->flag_n;
    ea.flag_cap = kNoAllocFlagCap;
    ea.flag_overflow = &s->flag_overflow;
    ea.work_counter = &s->work_counter;
    rc = launch_derivatives(ea, v.precision, v.variant, v.sms, st);
    if (rc) {
        ctx_set_error(ctx, cudaGetErrorString((cudaError_t)rc));
        return NDT_E_CUDA;
    }
    noalloc_reduce_kernel<<<1, 64, 0, st>>>(s, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        ctx_set_error(ctx, cudaGetErrorString(e));
        return NDT_E_CUDA;
    }
    return NDT_OK;
}
