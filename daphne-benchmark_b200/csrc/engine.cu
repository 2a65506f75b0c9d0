// C ABI of the library (include/ndt_b200.h): context, device memory, the
// per-batch launch sequence and the host-buffer entry points.
//
// Device memory is owned by the context and grows on demand (never shrinks),
// so steady-state calls allocate nothing.  All work of a context is ordered on
// its own non-blocking stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ndt_b200.h"
#include "align.h"
#include "ctx_view.h"
#include "nvtx_range.h"
#include "derivatives.h"
#include "grid_build.h"
#include "ndt_types.h"

using namespace ndt;

namespace {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
    // Contents are not kept.  A buffer that has to grow takes half as much
    // again, so that a slowly growing size (a map grown scan by scan)
    // reallocates only now and then.
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        const bool regrow = p != nullptr;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes < 256 ? 256 : bytes;
        if (regrow) want += want / 2;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    // Grows to at least `bytes` keeping the first `keep` bytes (copied on
    // stream st, which is synchronised before the old buffer is freed).
    cudaError_t grow_keep(size_t bytes, size_t keep, cudaStream_t st) {
        if (bytes <= cap && p) return cudaSuccess;
        void *fresh = nullptr;
        const size_t want = bytes + bytes / 2;
        cudaError_t e = cudaMalloc(&fresh, want);
        if (e != cudaSuccess) return e;
        if (p && keep) {
            e = cudaMemcpyAsync(fresh, p, keep < cap ? keep : cap, cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                cudaFree(fresh);
                return e;
            }
        }
        if (p) cudaFree(p);
        p = fresh;
        cap = want;
        return cudaSuccess;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T *as() const {
        return (T *)p;
    }
};

struct HostBuf {
    void *p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        size_t want = bytes < 256 ? 256 : bytes;
        cudaError_t e = cudaMallocHost(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T>
    T *as() const {
        return (T *)p;
    }
};

// Everything one batch enqueues (pointers, sizes, parameters): the key of its
// cached CUDA graph, compared byte for byte (zero-filled before use).
struct RunPlan {
    EvalArgs ea;
    TileLists L;
    StepParams P;
    const int *d_offsets;
    const float *d_guesses;
    float *d_out;
    int *d_conv;
    double *d_fit;
    int *d_status;
    int *active;
    int *round_no;
    unsigned long long *dev_launches;
    int B, tile, kb, ks, max_rounds, precision, variant, sms, fixed;
};

struct BatchGraph {
    RunPlan key;
    cudaGraphExec_t exec;
    unsigned long long last_use;
};

}  // namespace

struct ndt_ctx {
    ndt_params prm{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;  // host-to-device copies of host-buffer batches
    cudaStream_t aux_stream = nullptr;   // capture of the round body of batch graphs
    bool use_graphs = true;              // device batches as CUDA graphs (when profiling is off)
    std::vector<BatchGraph> graphs;      // cached batch graphs, least recently used evicted
    unsigned long long graph_clock = 0;
    std::vector<cudaEvent_t> copy_ev;    // one per copied alignment group
    int num_sms = 148;
    std::string err;
    double d1 = 0, d2 = 0;
    // grid
    DevBuf map, index, slot_of, mean, vox32, icov64, count, cell, seg_start, seg_cell, scratch, meta;
    DevBuf win_off, win_ent, win_ctot;
    GridMeta meta_host{};
    bool have_map = false;
    bool have_windows = false;
    int map_points = 0;
    // map growth (ndt_map_append): the current map's points on the device
    // (the context's own buffer `map`, or the caller's for ndt_set_map_device),
    // its cell-sorted pairs (in the build scratch, or in sorted_keys / _order
    // [sorted_in]) and the append's own scratch
    const float4 *map_src = nullptr;
    ndt::SortedMap sorted{nullptr, nullptr};
    int sorted_in = -1;  // -1: in `scratch`, else the index of the buffer pair
    DevBuf sorted_keys[2], sorted_order[2], append_scratch, meta_tmp;
    // the grid build after its bounding box, as a cached CUDA graph (the same
    // map pointer, size, bounding box and buffers launch it again)
    struct GridGraphKey {
        const float4 *map;
        int m;
        GridMeta meta;
        ndt::NdtGridOptions opt;
        ndt::GridBuffers buf;
        void *scratch;
        int windows;
        ndt::WindowBuffers wb;
    } grid_key;
    cudaGraphExec_t grid_exec = nullptr;
    int grid_nl = 0;
    ndt::SortedMap grid_sorted{nullptr, nullptr};
    // batch
    DevBuf chunks, chunk_begin, num_chunks, big_begin, small_begin, num_big, round_no, dev_launches;
    DevBuf points, offsets, guesses, states, tiles, tile_begin, num_tiles, partials, exc, out_T, out_conv, out_fit,
        out_status, active, counters, p6, trans, flag_q, flag_n, flag_overflow, work_counter, active_chunks, num_active;
    HostBuf h_offsets, h_active, h_counters, h_out;
    ndt_counters last{};
    long long launches = 0;
    int variant = kDefaultDerivVariant;  // FP32 derivative-pass launch shape (kDerivVariants)
    int chunk_tiles = kChunkBig;         // FP32 derivative pass: tiles per large chunk
    unsigned flag_cap = 1u << 20;  // FP64 side-queue capacity in pairs per derivative pass
    float s_max = 1.0f;    // radius test threshold (see radius_threshold)
    float inv_res = 0.0f;  // 1 / res when res is a power of two
    // profiling: event pairs around derivative launches and the grid build
    bool profiling = false;
    std::vector<cudaEvent_t> ev;
    int ev_used = 0;
    cudaEvent_t grid_ev[2] = {nullptr, nullptr};
    bool grid_timed = false;
};

namespace {

int fail(ndt_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(ndt_ctx *c, cudaError_t e, const char *what) {
    return fail(c, NDT_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                             \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
    } while (0)

// Gauss fitting constants, with the reference's host arithmetic
// (computeTransformation, kernel.cpp:1181-1185).
void gauss_constants(const ndt_params &p, double &d1, double &d2) {
    double outlier = p.outlier_ratio;
    float res = p.resolution;
    double c1 = 10 * (1 - outlier);
    double c2 = outlier / std::pow((double)res, 3.0);
    double d3 = -std::log(c2);
    d1 = -std::log(c1 + c2) - d3;
    d2 = -2 * std::log((-std::log(c1 * std::exp(-0.5) + c2) - d3) / d1);
}

// The reference accepts a voxel when float(sqrt(s)) < r (s = dx^2 + dy^2 +
// dz^2 in float, kernel.cpp:276-278).  The correctly rounded float square root
// is monotonic, so that is s <= s_max for the largest float s_max whose root
// rounds below r.
float radius_threshold(float r) {
    float s = r * r;
    while (std::sqrt(s) >= r) s = std::nextafter(s, 0.0f);
    while (std::sqrt(std::nextafter(s, INFINITY)) < r) s = std::nextafter(s, INFINITY);
    return s;
}

// 1 / r when r is a power of two (then (v - min) / r == (v - min) * (1 / r)
// exactly), otherwise 0 (the kernels divide).
float exact_reciprocal(float r) {
    int e;
    float m = std::frexp(r, &e);
    return m == 0.5f ? 1.0f / r : 0.0f;
}

StepParams step_params(const ndt_params &p) {
    StepParams s;
    s.compat = p.compat;
    s.max_iterations = p.max_iterations;
    s.eps = p.transformation_epsilon;
    s.step_max = p.step_size;
    s.step_min = p.transformation_epsilon / 2;
    s.watchdog_evals = p.watchdog_evals > 0 ? p.watchdog_evals : 1024;
    return s;
}

GridBuffers grid_buffers(ndt_ctx *c) {
    GridBuffers b;
    b.index = c->index.as<int32_t>();
    b.mean = c->mean.as<double4>();
    b.vox32 = c->vox32.as<float4>();
    b.icov64 = c->icov64.as<double>();
    b.count = c->count.as<int32_t>();
    b.cell = c->cell.as<int32_t>();
    b.seg_start = c->seg_start.as<int32_t>();
    b.seg_cell = c->seg_cell.as<uint32_t>();
    b.slot_of = c->slot_of.as<int32_t>();
    return b;
}

GridDev grid_dev(ndt_ctx *c) {
    GridDev g;
    g.meta = c->meta_host;
    g.index = c->index.as<int32_t>();
    g.mean = c->mean.as<double4>();
    g.vox32 = c->vox32.as<float4>();
    g.s_max = c->s_max;
    g.inv_res = c->inv_res;
    g.radius_final = (float)((double)c->prm.resolution + (double)0.001f);
    g.icov64 = c->icov64.as<double>();
    g.win_off = c->have_windows ? c->win_off.as<int32_t>() : nullptr;
    g.win_ent = c->have_windows ? c->win_ent.as<float4>() : nullptr;
    g.win_dim[0] = c->meta_host.dim[0] + 2;
    g.win_dim[1] = c->meta_host.dim[1] + 2;
    return g;
}

cudaEvent_t next_event(ndt_ctx *c) {
    if (c->ev_used >= (int)c->ev.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        c->ev.push_back(e);
    }
    return c->ev[c->ev_used++];
}

int set_device(ndt_ctx *c) {
    CK(cudaSetDevice(c->device));
    return NDT_OK;
}

constexpr long long kMaxWindows = 1LL << 28;        // probe windows (4 B offset each)
constexpr long long kMaxWindowEntries = 1LL << 28;  // window entries (16 B each)

// Grid build from a device-resident map (any device pointer valid on the
// context's stream for the duration of the call).
// Probe-window table of the finished dense index: W + 1 offsets and at most
// 27 entries per usable voxel (skipped when it would not fit, or with
// dense_probe set).  prepare_windows sizes the buffers (false: no table);
// enqueue_windows launches the build.
int prepare_windows(ndt_ctx *c, int m, bool &use, WindowBuffers &wb) {
    const size_t G = (size_t)c->meta_host.G;
    const long long W = (long long)window_count(c->meta_host);
    const long long ent_cap = 27LL * (long long)std::min<size_t>((size_t)m, G);
    use = !c->prm.dense_probe && W < kMaxWindows && ent_cap < kMaxWindowEntries;
    std::memset(&wb, 0, sizeof(wb));
    if (!use) return NDT_OK;
    CK(c->win_off.ensure(sizeof(int32_t) * (size_t)(W + 1)));
    CK(c->win_ent.ensure(sizeof(float4) * (size_t)ent_cap));
    CK(c->win_ctot.ensure(sizeof(int32_t) * (size_t)(W / 256 + 2)));
    wb.off = c->win_off.as<int32_t>();
    wb.ent = c->win_ent.as<float4>();
    wb.ctot = c->win_ctot.as<int32_t>();
    return NDT_OK;
}

int enqueue_windows(ndt_ctx *c, const WindowBuffers &wb, int *nl) {
    int rc = grid_windows(c->meta_host, c->index.as<int32_t>(), c->vox32.as<float4>(), wb, c->stream, nl);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_windows");
    return NDT_OK;
}

int build_windows(ndt_ctx *c, int m) {
    bool use = false;
    WindowBuffers wb;
    c->have_windows = false;
    if (int rc = prepare_windows(c, m, use, wb)) return rc;
    if (!use) return NDT_OK;
    int nl = 0;
    if (int rc = enqueue_windows(c, wb, &nl)) return rc;
    c->launches += nl;
    c->have_windows = true;
    return NDT_OK;
}

// Per-voxel record buffers for m slots, keeping the first `keep` slots.
int grow_records(ndt_ctx *c, int m, int keep) {
    cudaStream_t st = c->stream;
    const size_t n = (size_t)m, k = (size_t)keep;
    CK(c->mean.grow_keep(sizeof(double4) * n, sizeof(double4) * k, st));
    CK(c->vox32.grow_keep(3 * sizeof(float4) * n, 3 * sizeof(float4) * k, st));
    CK(c->icov64.grow_keep(9 * sizeof(double) * n, 9 * sizeof(double) * k, st));
    CK(c->count.grow_keep(sizeof(int32_t) * n, sizeof(int32_t) * k, st));
    CK(c->cell.grow_keep(sizeof(int32_t) * n, sizeof(int32_t) * k, st));
    return NDT_OK;
}

// Per-voxel record buffers for a map of m points.
int ensure_records(ndt_ctx *c, int m) {
    CK(c->mean.ensure(sizeof(double4) * (size_t)m));
    CK(c->vox32.ensure(3 * sizeof(float4) * (size_t)m));
    CK(c->icov64.ensure(9 * sizeof(double) * (size_t)m));
    CK(c->count.ensure(sizeof(int32_t) * (size_t)m));
    CK(c->cell.ensure(sizeof(int32_t) * (size_t)m));
    CK(c->seg_start.ensure(sizeof(int32_t) * (size_t)m));
    CK(c->seg_cell.ensure(sizeof(uint32_t) * (size_t)m));
    return NDT_OK;
}

int build_grid(ndt_ctx *c, const float4 *d_map, int m) {
    NvtxRange range("grid build");
    if (m <= 0) return fail(c, NDT_E_ARG, "map must have at least one point");
    // voxel slots travel in 26 bits of a packed pair code (slot << 6 | flag << 5 | lane)
    if (m >= (1 << 25)) return fail(c, NDT_E_CAPACITY, "map larger than 2^25 points");
    c->have_map = false;
    c->have_windows = false;
    c->grid_timed = false;
    if (c->profiling) {
        if (!c->grid_ev[0]) CK(cudaEventCreate(&c->grid_ev[0]));
        if (!c->grid_ev[1]) CK(cudaEventCreate(&c->grid_ev[1]));
        CK(cudaEventRecord(c->grid_ev[0], c->stream));
    }
    {
        void *old = c->scratch.p;
        CK(c->scratch.ensure(ndt::grid_scratch_bytes(m)));
        if (c->scratch.p != old) CK((cudaError_t)grid_scratch_init(c->scratch.p, c->stream));
    }
    CK(c->meta.ensure(sizeof(GridMeta)));
    int rc = grid_bbox(d_map, m, c->prm.resolution, c->meta.as<GridMeta>(), c->scratch.p, c->stream);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_bbox");
    c->launches += 1;
    CK(cudaMemcpyAsync(&c->meta_host, c->meta.p, sizeof(GridMeta), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (c->meta_host.error == 2) return fail(c, NDT_E_ARG, "map has non-finite coordinates");
    if (c->meta_host.error) return fail(c, NDT_E_GRID, "voxel grid does not fit 32-bit cell indices");
    const size_t G = (size_t)c->meta_host.G;
    CK(c->index.ensure(sizeof(int32_t) * G));
    CK(c->slot_of.ensure(sizeof(int32_t) * G));
    if (int rc0 = ensure_records(c, m)) return rc0;
    NdtGridOptions opt;
    opt.compat = c->prm.compat;
    opt.min_points = c->prm.min_points_per_voxel;
    opt.eigen_ratio = c->prm.eigen_ratio;
    bool windows = false;
    WindowBuffers wb;
    if (int rc0 = prepare_windows(c, m, windows, wb)) return rc0;
    // the rest of the build (keys, sort, segments, records, windows): replayed
    // from the cached graph when nothing it depends on has changed
    ndt_ctx::GridGraphKey key;
    std::memset(&key, 0, sizeof(key));
    key.map = d_map;
    key.m = m;
    {  // field by field: the struct's padding bytes are not part of the key
        const GridMeta &g = c->meta_host;
        for (int e = 0; e < 3; ++e) {
            key.meta.minv[e] = g.minv[e];
            key.meta.maxv[e] = g.maxv[e];
            key.meta.raw_min[e] = g.raw_min[e];
            key.meta.raw_max[e] = g.raw_max[e];
            key.meta.dim[e] = g.dim[e];
        }
        key.meta.res = g.res;
        key.meta.G = g.G;
        key.meta.occupied = g.occupied;
        key.meta.error = g.error;
    }
    key.opt = opt;
    key.buf = grid_buffers(c);
    key.scratch = c->scratch.p;
    key.windows = windows ? 1 : 0;
    key.wb = wb;
    cudaStream_t st = c->stream;
    if (!(c->use_graphs && c->grid_exec && std::memcmp(&key, &c->grid_key, sizeof(key)) == 0)) {
        if (c->grid_exec) cudaGraphExecDestroy(c->grid_exec);
        c->grid_exec = nullptr;
        int nl = 0;
        ndt::SortedMap sorted{nullptr, nullptr};
        if (c->use_graphs) CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        rc = grid_build(d_map, m, c->meta_host, c->meta.as<GridMeta>(), opt, key.buf, c->scratch.p, st, &nl, &sorted);
        int rc2 = rc ? 0 : (windows ? enqueue_windows(c, wb, &nl) : 0);
        if (c->use_graphs) {
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(st, &g);
            if (rc || rc2 || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_build");
                if (rc2) return rc2;
                return cuda_fail(c, e, "grid build capture");
            }
            e = cudaGraphInstantiate(&c->grid_exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                c->grid_exec = nullptr;
                return cuda_fail(c, e, "cudaGraphInstantiate (grid build)");
            }
            c->grid_key = key;
        } else {
            if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_build");
            if (rc2) return rc2;
        }
        c->grid_nl = nl;
        c->grid_sorted = sorted;
    }
    if (c->grid_exec) CK(cudaGraphLaunch(c->grid_exec, st));
    c->launches += c->grid_nl;
    c->sorted = c->grid_sorted;
    c->sorted_in = -1;
    c->have_windows = windows;
    if (c->profiling) {
        CK(cudaEventRecord(c->grid_ev[1], c->stream));
        c->grid_timed = true;
    }
    c->map_src = d_map;
    c->have_map = true;
    c->map_points = m;
    return NDT_OK;
}

constexpr unsigned kFlagCap = 1u << 20;     // default side-queue capacity (pairs per derivative pass)
constexpr unsigned kFlagCapMax = 1u << 24;  // largest capacity ndt_set_side_queue_capacity accepts

int prepare_flag_queue(ndt_ctx *c, EvalArgs &ea) {
    CK(c->flag_q.ensure(sizeof(int4) * c->flag_cap));
    CK(c->flag_n.ensure(sizeof(unsigned)));
    CK(c->flag_overflow.ensure(sizeof(int)));
    ea.flag_q = c->flag_q.as<int4>();
    ea.flag_n = c->flag_n.as<unsigned>();
    ea.flag_cap = c->flag_cap;
    ea.flag_overflow = c->flag_overflow.as<int>();
    CK(c->work_counter.ensure(sizeof(int)));
    ea.work_counter = c->work_counter.as<int>();
    return NDT_OK;
}

// Tile and chunk lists for B alignments (capacity max_tiles each); the FP32
// pass takes chunks of kChunkBig and kChunkSmall tiles, the FP64 pass chunks
// of one tile.
int prepare_lists(ndt_ctx *c, int B, int max_tiles, TileLists &L) {
    CK(c->tile_begin.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->tiles.ensure(sizeof(Tile) * (size_t)max_tiles));
    CK(c->num_tiles.ensure(sizeof(int)));
    CK(c->chunk_begin.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->chunks.ensure(sizeof(Chunk) * (size_t)max_tiles));
    CK(c->num_chunks.ensure(sizeof(int)));
    L.tile_begin = c->tile_begin.as<int>();
    L.tiles = c->tiles.as<Tile>();
    L.num_tiles = c->num_tiles.as<int>();
    L.chunk_begin = c->chunk_begin.as<int>();
    L.chunks = c->chunks.as<Chunk>();
    L.num_chunks = c->num_chunks.as<int>();
    CK(c->big_begin.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->small_begin.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->num_big.ensure(sizeof(int)));
    L.big_begin = c->big_begin.as<int>();
    L.small_begin = c->small_begin.as<int>();
    L.num_big = c->num_big.as<int>();
    return NDT_OK;
}

int chunk_big(const ndt_ctx *c) { return c->prm.precision == 1 ? 1 : c->chunk_tiles; }
int chunk_small(const ndt_ctx *c) { return c->prm.precision == 1 ? 1 : std::min(kChunkSmall, c->chunk_tiles); }

// Device-side batch: everything already on the device.
// Round-loop condition of a batch graph: another round while an alignment
// asked for an evaluation and the round budget (the evaluation watchdog) is
// not spent, so the loop always ends.
__global__ void round_cond_kernel(cudaGraphConditionalHandle h, const int *active, int *round_no, int max_rounds,
                                  unsigned long long *launches, int per_round) {
    const int r = ++*round_no;
    *launches += (unsigned long long)per_round;
    cudaGraphSetConditional(h, (*active > 0 && r < max_rounds) ? 1u : 0u);
}

int enqueue_prologue(ndt_ctx *c, const RunPlan &R, cudaStream_t st) {
    CK(cudaMemsetAsync(R.ea.flag_overflow, 0, sizeof(int), st));
    CK(cudaMemsetAsync(R.round_no, 0, sizeof(int), st));
    int rc = launch_tiles(R.d_offsets, R.B, R.tile, R.kb, R.ks, R.L, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_tiles");
    rc = launch_init(R.ea.states, R.d_guesses, R.d_offsets, R.B, R.P, R.ea.exc, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_init");
    return NDT_OK;
}

// One round: the derivative pass, then the step kernel (which counts in
// *active the alignments that ask for another evaluation).
int enqueue_round(ndt_ctx *c, const RunPlan &R, cudaStream_t st, bool profile) {
    cudaEvent_t e0 = profile ? next_event(c) : nullptr;
    if (e0) CK(cudaEventRecord(e0, st));
    int rc = launch_derivatives(R.ea, R.precision, R.variant, R.sms, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_derivatives");
    cudaEvent_t e1 = profile ? next_event(c) : nullptr;
    if (e1) CK(cudaEventRecord(e1, st));
    CK(cudaMemsetAsync(R.active, 0, sizeof(int), st));
    rc = launch_step(R.ea.states, R.ea.partials, R.L.chunk_begin, R.ea.exc, R.B, R.P, R.active, R.ea.counters, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_step");
    return NDT_OK;
}

int enqueue_epilogue(ndt_ctx *c, const RunPlan &R, cudaStream_t st) {
    int rc = launch_finalize(R.ea.states, R.B, R.d_out, R.d_conv, R.d_fit, R.d_status, R.ea.flag_overflow, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_finalize");
    return NDT_OK;
}

// Kernel launches of one round (derivative pass + step kernel).
int round_launches(const RunPlan &R) {
    return 1 + (R.precision == 1 ? 1 : kDerivLaunchesFP32 + (R.ea.active_chunks ? 1 : 0));
}

// The batch as one CUDA graph: prologue, a conditional WHILE node whose body
// is one round plus round_cond_kernel, epilogue.  Built by stream capture
// (the round body on the auxiliary stream, into the WHILE node's body graph).
int build_batch_graph(ndt_ctx *c, const RunPlan &R, cudaGraphExec_t *out) {
    cudaGraph_t g = nullptr;
    CK(cudaGraphCreate(&g, 0));
    cudaStream_t st = c->stream;
    auto abort_capture = [&](int code) {
        cudaGraph_t tmp = nullptr;
        cudaStreamEndCapture(st, &tmp);
        cudaGraphDestroy(g);
        return code;
    };
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(c, e, "cudaGraphConditionalHandleCreate");
    }
    e = cudaStreamBeginCaptureToGraph(st, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(c, e, "cudaStreamBeginCaptureToGraph");
    }
    if (int rc = enqueue_prologue(c, R, st)) return abort_capture(rc);
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    e = cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd);
    if (e != cudaSuccess) return abort_capture(cuda_fail(c, e, "cudaStreamGetCaptureInfo"));
    // (cudaGraphNodeParams has no default constructor: zeroed raw storage)
    alignas(cudaGraphNodeParams) unsigned char np_raw[sizeof(cudaGraphNodeParams)];
    std::memset(np_raw, 0, sizeof(np_raw));
    cudaGraphNodeParams &np = *reinterpret_cast<cudaGraphNodeParams *>(np_raw);
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, cg, deps, nd, &np);
    if (e != cudaSuccess) return abort_capture(cuda_fail(c, e, "cudaGraphAddNode (while)"));
    e = cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies);
    if (e != cudaSuccess) return abort_capture(cuda_fail(c, e, "cudaStreamUpdateCaptureDependencies"));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(c->aux_stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return abort_capture(cuda_fail(c, e, "cudaStreamBeginCaptureToGraph (body)"));
    int rc = enqueue_round(c, R, c->aux_stream, false);
    if (!rc) {
        round_cond_kernel<<<1, 1, 0, c->aux_stream>>>(h, R.active, R.round_no, R.max_rounds, R.dev_launches,
                                                       round_launches(R) + 1);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_fail(c, e, "round_cond_kernel");
    }
    cudaGraph_t body_out = nullptr;
    e = cudaStreamEndCapture(c->aux_stream, &body_out);
    if (rc) return abort_capture(rc);
    if (e != cudaSuccess) return abort_capture(cuda_fail(c, e, "cudaStreamEndCapture (body)"));
    if (int rc2 = enqueue_epilogue(c, R, st)) return abort_capture(rc2);
    cudaGraph_t g_out = nullptr;
    e = cudaStreamEndCapture(st, &g_out);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(c, e, "cudaStreamEndCapture");
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
    return NDT_OK;
}

constexpr size_t kMaxGraphs = 8;  // cached batch graphs per context

int get_batch_graph(ndt_ctx *c, const RunPlan &R, cudaGraphExec_t *out) {
    ++c->graph_clock;
    for (BatchGraph &b : c->graphs) {
        if (std::memcmp(&b.key, &R, sizeof(RunPlan)) == 0) {
            b.last_use = c->graph_clock;
            *out = b.exec;
            return NDT_OK;
        }
    }
    cudaGraphExec_t exec = nullptr;
    if (int rc = build_batch_graph(c, R, &exec)) return rc;
    if (c->graphs.size() >= kMaxGraphs) {
        size_t lru = 0;
        for (size_t i = 1; i < c->graphs.size(); ++i)
            if (c->graphs[i].last_use < c->graphs[lru].last_use) lru = i;
        cudaGraphExecDestroy(c->graphs[lru].exec);
        c->graphs.erase(c->graphs.begin() + (long)lru);
    }
    BatchGraph b;
    std::memcpy(&b.key, &R, sizeof(RunPlan));
    b.exec = exec;
    b.last_use = c->graph_clock;
    c->graphs.push_back(b);
    *out = exec;
    return NDT_OK;
}

// first = false continues the counters and profiling events of the previous
// call (alignment groups of one host batch).
int run_batch(ndt_ctx *c, int B, const float4 *d_points, const int *d_offsets, int total, const float *d_guesses,
              float *d_out, int *d_conv, double *d_fit, int *d_status, bool first = true) {
    NvtxRange range("rounds");
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    if (B <= 0 || total < 0) return fail(c, NDT_E_ARG, "empty batch");
    const int tile = c->prm.precision == 1 ? kTile : kDerivVariants[c->variant].tile;
    const int max_tiles = total / tile + B + 1;
    CK(c->states.ensure(sizeof(AlignState) * (size_t)B));
    RunPlan R;
    std::memset(&R, 0, sizeof(R));
    if (int rc0 = prepare_lists(c, B, max_tiles, R.L)) return rc0;
    CK(c->partials.ensure(sizeof(double) * kPartial * (size_t)max_tiles));
    CK(c->exc.ensure(sizeof(double) * kPartial * (size_t)B));
    CK(c->active.ensure(sizeof(int)));
    CK(c->counters.ensure(sizeof(Counters)));
    CK(c->h_active.ensure(sizeof(int)));
    CK(c->round_no.ensure(sizeof(int)));
    cudaStream_t st = c->stream;
    if (first) {
        CK(cudaMemsetAsync(c->counters.p, 0, sizeof(Counters), st));
        c->ev_used = 0;
    }
    R.P = step_params(c->prm);
    EvalArgs &ea = R.ea;
    ea.grid = grid_dev(c);
    ea.points = d_points;
    ea.trans = nullptr;
    ea.tiles = c->tiles.as<Tile>();
    ea.num_tiles = c->num_tiles.as<int>();
    ea.chunks = R.L.chunks;
    ea.num_chunks = R.L.num_chunks;
    ea.max_tiles = max_tiles;
    ea.tile_size = tile;
    ea.states = c->states.as<AlignState>();
    ea.partials = c->partials.as<double>();
    ea.exc = c->exc.as<double>();
    ea.d1 = c->d1;
    ea.d2 = c->d2;
    ea.compat = c->prm.compat;
    ea.counters = c->counters.as<Counters>();
    if (int rc2 = prepare_flag_queue(c, ea)) return rc2;
    R.d_offsets = d_offsets;
    R.d_guesses = d_guesses;
    R.d_out = d_out;
    R.d_conv = d_conv;
    R.d_fit = d_fit;
    R.d_status = d_status;
    R.active = c->active.as<int>();
    R.round_no = c->round_no.as<int>();
    R.dev_launches = c->dev_launches.as<unsigned long long>();
    R.B = B;
    R.tile = tile;
    R.kb = chunk_big(c);
    R.ks = chunk_small(c);
    R.precision = c->prm.precision;
    R.variant = c->variant;
    R.sms = c->num_sms;
    // With the reference's line-search test (compat, step_max > step_min)
    // every Newton iteration takes at most one evaluation, so the round count
    // is fixed.
    R.fixed = R.P.compat && (R.P.step_max - R.P.step_min) > 0;
    R.max_rounds = R.fixed ? R.P.max_iterations + 3 : R.P.watchdog_evals + 1;
    if (!R.fixed && R.precision == 0) {
        // alignments finish at different rounds: each FP32 pass hands out only the chunks of active ones
        CK(c->active_chunks.ensure(sizeof(int) * (size_t)max_tiles));
        CK(c->num_active.ensure(sizeof(int)));
        ea.active_chunks = c->active_chunks.as<int>();
        ea.num_active = c->num_active.as<int>();
    }

    if (c->use_graphs && !c->profiling) {
        // one graph launch: the rounds run on the device until no alignment
        // asks for an evaluation, with no host synchronisation
        cudaGraphExec_t exec = nullptr;
        if (int rc = get_batch_graph(c, R, &exec)) return rc;
        CK(cudaGraphLaunch(exec, st));
        c->launches += 5;  // tiles (3), init, finalize; the rounds count themselves on the device
        return NDT_OK;
    }
    long long nl = 0;
    if (int rc = enqueue_prologue(c, R, st)) return rc;
    nl += 4;
    const int poll_every = 4;
    for (int r = 0; r < R.max_rounds; ++r) {
        if (int rc = enqueue_round(c, R, st, c->profiling)) return rc;
        nl += round_launches(R);
        if (!R.fixed && (r + 1) % poll_every == 0) {
            CK(cudaMemcpyAsync(c->h_active.p, c->active.p, sizeof(int), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (*c->h_active.as<int>() == 0) break;
        }
    }
    if (int rc = enqueue_epilogue(c, R, st)) return rc;
    nl += 1;
    c->launches += nl;
    return NDT_OK;
}

int read_counters(ndt_ctx *c) {
    CK(c->h_counters.ensure(sizeof(Counters)));
    CK(cudaMemcpyAsync(c->h_counters.p, c->counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    const Counters *k = c->h_counters.as<Counters>();
    c->last.rounds = (int64_t)k->rounds;
    unsigned long long dl = 0;
    if (c->dev_launches.p) CK(cudaMemcpy(&dl, c->dev_launches.p, sizeof(dl), cudaMemcpyDeviceToHost));
    c->last.launches = c->launches + (long long)dl;
    c->last.points = (int64_t)k->points;
    c->last.probes = (int64_t)k->probes;
    c->last.occupied_probes = (int64_t)k->occupied_probes;
    c->last.pairs = (int64_t)k->pairs;
    c->last.tiles = (int64_t)k->tiles;
    c->last.evaluations = (int64_t)k->evaluations;
    double ms = 0.0;
    int n = 0;
    for (int i = 0; i + 1 < c->ev_used; i += 2) {
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, c->ev[i], c->ev[i + 1]));
        ms += t;
        ++n;
    }
    c->last.deriv_ms = ms;
    c->last.deriv_launches = n;
    c->last.grid_ms = 0.0;
    if (c->grid_timed) {
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, c->grid_ev[0], c->grid_ev[1]));
        c->last.grid_ms = t;
    }
    return NDT_OK;
}

// Number of alignment groups of a host-buffer batch: each group's points are
// copied on the copy stream while the compute stream runs the previous
// group's rounds (and, for the first group, the grid build of a map set just
// before).  By size: about 2^20 points per group, at most 4 groups (each
// group repeats the per-round fixed costs, so small groups do not pay).
int copy_group_count(const ndt_ctx *c, int B, long long total) {
    int g = c->prm.copy_groups > 0 ? c->prm.copy_groups : (int)std::min<long long>(4, total >> 20);
    if (g < 1) g = 1;
    if (g > B) g = B;
    return g;
}

// Host batch: offsets (off[0] = 0) and guesses are host arrays; copy(b0, b1,
// stream) enqueues the host-to-device copy of the points of alignments
// [b0, b1) into c->points at off[b0].  Alignments are split into groups of
// about equal point counts; group k's rounds wait only for group k's copy.
// A host batch in copy groups: every group's points are copied on the copy
// stream (all copies enqueued first, one event each), then each group's
// rounds run on the compute stream once its event has fired, so the copies
// of later groups overlap the rounds of earlier ones.  `before_copies` and
// `before_runs` (optional) run before the copies are enqueued and before the
// first group's rounds: the map of ndt_align_batch_packed_with_map is
// uploaded in the first and built in the second, so its grid build overlaps
// the scans' copies.
template <class CopyFn, class PreFn, class MidFn>
int staged_batch(ndt_ctx *c, int B, const int *off, const float *guesses, float *out, int *conv, double *fit,
                 int *status, CopyFn copy, PreFn before_copies, MidFn before_runs) {
    const long long total = off[B];
    cudaStream_t st = c->stream, cs = c->copy_stream;
    CK(c->points.ensure(sizeof(float4) * (size_t)(total > 0 ? total : 1)));
    CK(c->offsets.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->guesses.ensure(sizeof(float) * 16 * (size_t)B));
    CK(c->out_T.ensure(sizeof(float) * 16 * (size_t)B));
    CK(c->out_conv.ensure(sizeof(int) * (size_t)B));
    CK(c->out_fit.ensure(sizeof(double) * (size_t)B));
    CK(c->out_status.ensure(sizeof(int) * (size_t)B));
    const int G = copy_group_count(c, B, total);
    while ((int)c->copy_ev.size() < G) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->copy_ev.push_back(e);
    }
    // group k ends at the first alignment whose start reaches (k + 1) / G of the points
    std::vector<int> bound(G + 1, 0);
    bound[G] = B;
    for (int k = 0; k + 1 < G; ++k) {
        const long long target = total * (k + 1) / G;
        int b1 = bound[k] + 1;
        while (b1 < B - (G - 1 - k) && off[b1] < target) ++b1;
        bound[k + 1] = b1;
    }
    NvtxRange range("host batch");
    if (int rc = before_copies()) return rc;
    CK(cudaMemcpyAsync(c->offsets.p, off, sizeof(int) * (size_t)(B + 1), cudaMemcpyHostToDevice, cs));
    CK(cudaMemcpyAsync(c->guesses.p, guesses, sizeof(float) * 16 * (size_t)B, cudaMemcpyHostToDevice, cs));
    for (int k = 0; k < G; ++k) {
        if (int rc = copy(bound[k], bound[k + 1], cs)) return rc;
        CK(cudaEventRecord(c->copy_ev[k], cs));
    }
    if (int rc = before_runs()) {
        cudaStreamSynchronize(cs);
        return rc;
    }
    if (!c->have_map) {
        cudaStreamSynchronize(cs);
        return fail(c, NDT_E_NOMAP, "no map set");
    }
    for (int k = 0; k < G; ++k) {
        const int b0 = bound[k], b1 = bound[k + 1];
        CK(cudaStreamWaitEvent(st, c->copy_ev[k], 0));
        int rc = run_batch(c, b1 - b0, c->points.as<float4>(), c->offsets.as<int>() + b0, off[b1] - off[b0],
                           c->guesses.as<float>() + 16 * (size_t)b0, c->out_T.as<float>() + 16 * (size_t)b0,
                           c->out_conv.as<int>() + b0, c->out_fit.as<double>() + b0, c->out_status.as<int>() + b0,
                           k == 0);
        if (rc) {
            cudaStreamSynchronize(cs);
            return rc;
        }
    }
    CK(cudaMemcpyAsync(out, c->out_T.p, sizeof(float) * 16 * (size_t)B, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(conv, c->out_conv.p, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(fit, c->out_fit.p, sizeof(double) * (size_t)B, cudaMemcpyDeviceToHost, st));
    if (status) CK(cudaMemcpyAsync(status, c->out_status.p, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return NDT_OK;
}

int no_hook() { return NDT_OK; }

// Host batch of separate scan buffers.
int host_batch(ndt_ctx *c, int B, const float *const *scans, const int *ns, const float *guesses, float *out,
               int *conv, double *fit, int *status) {
    if (B <= 0 || !scans || !ns || !guesses || !out || !conv || !fit) return fail(c, NDT_E_ARG, "null argument");
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    CK(c->h_offsets.ensure(sizeof(int) * (size_t)(B + 1)));
    int *off = c->h_offsets.as<int>();
    long long total = 0;
    off[0] = 0;
    for (int b = 0; b < B; ++b) {
        if (ns[b] < 0 || (ns[b] > 0 && !scans[b])) return fail(c, NDT_E_ARG, "bad scan");
        total += ns[b];
        if (total > (1LL << 31) - 1) return fail(c, NDT_E_CAPACITY, "batch larger than 2^31 points");
        off[b + 1] = (int)total;
    }
    return staged_batch(c, B, off, guesses, out, conv, fit, status, [&](int b0, int b1, cudaStream_t cs) -> int {
        for (int b = b0; b < b1; ++b)
            if (ns[b] > 0)
                CK(cudaMemcpyAsync(c->points.as<float4>() + off[b], scans[b], sizeof(float4) * (size_t)ns[b],
                                   cudaMemcpyHostToDevice, cs));
        return NDT_OK;
    }, no_hook, no_hook);
}

// Host batch from one packed host buffer; with map != nullptr the batch's map
// comes along (uploaded first, built while the scans are copied).
int packed_batch(ndt_ctx *c, int B, const float *points, const int *offsets, const float *guesses, float *out,
                 int *conv, double *fit, int *status, const float *map = nullptr, int m = 0) {
    if (B <= 0 || !points || !offsets || !guesses || !out || !conv || !fit) return fail(c, NDT_E_ARG, "null argument");
    if (!map && !c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    if (map && m <= 0) return fail(c, NDT_E_ARG, "empty map");
    if (offsets[0] != 0) return fail(c, NDT_E_ARG, "offsets[0] must be 0");
    for (int b = 0; b < B; ++b)
        if (offsets[b + 1] < offsets[b]) return fail(c, NDT_E_ARG, "offsets must be non-decreasing");
    auto upload_map = [&]() -> int {
        if (!map) return NDT_OK;
        c->have_map = false;
        CK(c->map.ensure(sizeof(float4) * (size_t)m));
        CK(cudaMemcpyAsync(c->map.p, map, sizeof(float4) * (size_t)m, cudaMemcpyHostToDevice, c->stream));
        return NDT_OK;
    };
    auto build_map = [&]() -> int { return map ? build_grid(c, c->map.as<float4>(), m) : NDT_OK; };
    return staged_batch(c, B, offsets, guesses, out, conv, fit, status, [&](int b0, int b1, cudaStream_t cs) -> int {
        const long long n = (long long)offsets[b1] - offsets[b0];
        if (n > 0)
            CK(cudaMemcpyAsync(c->points.as<float4>() + offsets[b0], points + 4 * (size_t)offsets[b0],
                               sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, cs));
        return NDT_OK;
    }, upload_map, build_map);
}

}  // namespace

namespace ndt {

int ctx_eval_view(ndt_ctx *c, CtxEvalView *v) {
    if (!c || !v) return NDT_E_ARG;
    v->grid = grid_dev(c);
    v->d1 = c->d1;
    v->d2 = c->d2;
    v->compat = c->prm.compat;
    v->precision = c->prm.precision;
    v->variant = c->variant;
    v->sms = c->num_sms;
    v->device = c->device;
    v->stream = c->stream;
    v->have_map = c->have_map;
    return NDT_OK;
}

void ctx_set_error(ndt_ctx *c, const char *msg) {
    if (c) c->err = msg;
}

}  // namespace ndt

extern "C" {

void ndt_params_reference(ndt_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->resolution = 1.0f;
    p->outlier_ratio = 0.55;
    p->step_size = 0.1;
    p->transformation_epsilon = 0.1;
    p->max_iterations = 0;
    p->compat = 1;
    p->min_points_per_voxel = 0;
    p->precision = 0;
    p->eigen_ratio = 0.0;
    p->watchdog_evals = 0;
}

void ndt_params_corrected(ndt_params *p) {
    if (!p) return;
    ndt_params_reference(p);
    p->transformation_epsilon = 0.01;
    p->max_iterations = 30;
    p->compat = 0;
    p->min_points_per_voxel = 6;
    p->eigen_ratio = 0.01;
}

int ndt_create(const ndt_params *params, int device, ndt_ctx **out) {
    if (!out) return NDT_E_ARG;
    *out = nullptr;
    if (!params) return NDT_E_ARG;
    if (!(params->resolution > 0.0f) || !std::isfinite(params->resolution)) return NDT_E_ARG;
    if (params->precision != 0 && params->precision != 1) return NDT_E_ARG;
    if (params->outlier_ratio <= 0.0 || params->outlier_ratio >= 1.0) return NDT_E_ARG;
    ndt_ctx *c = new ndt_ctx();
    c->prm = *params;
    c->device = device;
    gauss_constants(c->prm, c->d1, c->d2);
    c->s_max = radius_threshold(c->prm.resolution);
    c->inv_res = exact_reciprocal(c->prm.resolution);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = c->dev_launches.ensure(sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(c->dev_launches.p, 0, sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = (cudaError_t)prepare_derivatives();
    if (e != cudaSuccess) {
        delete c;
        return NDT_E_CUDA;
    }
    *out = c;
    return NDT_OK;
}

void ndt_destroy(ndt_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    DevBuf *bufs[] = {&c->win_off, &c->win_ent, &c->win_ctot, &c->map, &c->index, &c->mean, &c->vox32,
                      &c->icov64, &c->count, &c->cell, &c->seg_start, &c->seg_cell,
                      &c->scratch, &c->meta, &c->points, &c->offsets, &c->guesses, &c->states,
                      &c->tiles, &c->tile_begin, &c->num_tiles, &c->chunks, &c->chunk_begin, &c->num_chunks,
                      &c->big_begin, &c->small_begin, &c->num_big, &c->round_no, &c->dev_launches,
                      &c->partials, &c->exc, &c->out_T, &c->out_conv,
                      &c->out_fit, &c->out_status, &c->active, &c->counters, &c->p6, &c->trans,
                      &c->flag_q, &c->flag_n, &c->flag_overflow, &c->work_counter, &c->active_chunks,
                      &c->num_active};
    for (DevBuf *b : bufs) b->release();
    HostBuf *hb[] = {&c->h_offsets, &c->h_active, &c->h_counters, &c->h_out};
    for (HostBuf *b : hb) b->release();
    for (cudaEvent_t e : c->ev) cudaEventDestroy(e);
    for (cudaEvent_t e : c->copy_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : c->grid_ev)
        if (e) cudaEventDestroy(e);
    for (BatchGraph &b : c->graphs) cudaGraphExecDestroy(b.exec);
    if (c->grid_exec) cudaGraphExecDestroy(c->grid_exec);
    c->graphs.clear();
    if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *ndt_last_error(const ndt_ctx *c) { return c ? c->err.c_str() : "null context"; }

void *ndt_stream(ndt_ctx *c) { return c ? (void *)c->stream : nullptr; }

int ndt_synchronize(ndt_ctx *c) {
    if (!c) return NDT_E_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return NDT_OK;
}

int ndt_set_map(ndt_ctx *c, const float *map, int m) {
    if (!c || !map || m <= 0) return fail(c, NDT_E_ARG, "null map or empty map");
    if (int rc = set_device(c)) return rc;
    CK(c->map.ensure(sizeof(float4) * (size_t)m));
    CK(cudaMemcpyAsync(c->map.p, map, sizeof(float4) * (size_t)m, cudaMemcpyHostToDevice, c->stream));
    return build_grid(c, c->map.as<float4>(), m);
}

int ndt_set_map_device(ndt_ctx *c, const float *d_map, int m) {
    if (!c || !d_map || m <= 0) return fail(c, NDT_E_ARG, "null map or empty map");
    if (int rc = set_device(c)) return rc;
    return build_grid(c, (const float4 *)d_map, m);
}

// Appends k points (host or device) to the current map and brings the grid up
// to date: incrementally (merge of the new points' sorted cells into the
// map's, then the voxel records) when they lie inside the old points'
// bounding box, else by a full build of the grown map.  Either way the grid
// equals ndt_set_map of the whole grown map.
int map_append(ndt_ctx *c, const float *pts, int k, bool host) {
    NvtxRange range("map append");
    if (!c) return NDT_E_ARG;
    if (k < 0 || (k > 0 && !pts)) return fail(c, NDT_E_ARG, "null points or negative count");
    if (int rc = set_device(c)) return rc;
    if (!c->have_map || !c->map_src) return fail(c, NDT_E_NOMAP, "no map set");
    if (k == 0) return NDT_OK;
    const int m = c->map_points;
    const long long nl_total = (long long)m + k;
    if (nl_total >= (1LL << 25)) return fail(c, NDT_E_CAPACITY, "map larger than 2^25 points");
    const int n = (int)nl_total;
    cudaStream_t st = c->stream;
    // 1. the grown map in the context's own buffer (grown by half again when full)
    const size_t need = sizeof(float4) * (size_t)n;
    if (c->map_src != c->map.as<float4>() || c->map.cap < need) {
        void *fresh = nullptr;
        const size_t want = std::max(need + need / 2, (size_t)4096);
        CK(cudaMalloc(&fresh, want));
        cudaError_t e = cudaMemcpyAsync(fresh, c->map_src, sizeof(float4) * (size_t)m, cudaMemcpyDeviceToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            cudaFree(fresh);
            return cuda_fail(c, e, "copy of the map");
        }
        c->map.release();
        c->map.p = fresh;
        c->map.cap = want;
        c->map_src = c->map.as<float4>();
    }
    float4 *map = c->map.as<float4>();
    CK(cudaMemcpyAsync(map + m, pts, sizeof(float4) * (size_t)k,
                       host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
    // 2. the new points' bounding box against the old points'
    CK(c->meta_tmp.ensure(sizeof(GridMeta)));
    int rc = grid_bbox(map + m, k, c->prm.resolution, c->meta_tmp.as<GridMeta>(), c->scratch.p, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_bbox");
    c->launches += 1;
    GridMeta nm;
    CK(cudaMemcpyAsync(&nm, c->meta_tmp.p, sizeof(GridMeta), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (nm.error == 2) return fail(c, NDT_E_ARG, "appended points have non-finite coordinates");
    bool inside = true;
    for (int e = 0; e < 3; ++e)
        if (!(nm.raw_min[e] >= c->meta_host.raw_min[e] && nm.raw_max[e] <= c->meta_host.raw_max[e])) inside = false;
    if (!inside) return build_grid(c, map, n);
    // 3. incremental: merge, the touched cells' records, windows
    c->have_map = false;
    c->grid_timed = false;
    if (c->profiling) {
        if (!c->grid_ev[0]) CK(cudaEventCreate(&c->grid_ev[0]));
        if (!c->grid_ev[1]) CK(cudaEventCreate(&c->grid_ev[1]));
        CK(cudaEventRecord(c->grid_ev[0], st));
    }
    if (int rc0 = grow_records(c, n, m)) return rc0;
    const int out = c->sorted_in == 0 ? 1 : 0;
    CK(c->sorted_keys[out].ensure(sizeof(uint32_t) * (size_t)n));
    CK(c->sorted_order[out].ensure(sizeof(uint32_t) * (size_t)n));
    CK(c->append_scratch.ensure(ndt::append_scratch_bytes(k)));
    NdtGridOptions opt;
    opt.compat = c->prm.compat;
    opt.min_points = c->prm.min_points_per_voxel;
    opt.eigen_ratio = c->prm.eigen_ratio;
    int nl = 0;
    rc = grid_append(map, m, k, c->meta_host, c->meta.as<GridMeta>(), opt, grid_buffers(c), c->sorted,
                     c->sorted_keys[out].as<uint32_t>(), c->sorted_order[out].as<uint32_t>(), c->append_scratch.p, st,
                     &nl);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "grid_append");
    c->launches += nl;
    c->sorted.keys = c->sorted_keys[out].as<uint32_t>();
    c->sorted.order = c->sorted_order[out].as<uint32_t>();
    c->sorted_in = out;
    if (int rc2 = build_windows(c, n)) return rc2;
    if (c->profiling) {
        CK(cudaEventRecord(c->grid_ev[1], st));
        c->grid_timed = true;
    }
    c->have_map = true;
    c->map_points = n;
    return NDT_OK;
}

int ndt_map_append(ndt_ctx *c, const float *points, int k) { return map_append(c, points, k, true); }

int ndt_map_append_device(ndt_ctx *c, const float *d_points, int k) { return map_append(c, d_points, k, false); }

int ndt_align(ndt_ctx *c, const float *scan, int n, const float guess16[16], float out16[16], int *converged,
              double *fitness) {
    if (!c || !guess16 || !out16 || !converged || !fitness || n < 0 || (n > 0 && !scan))
        return fail(c, NDT_E_ARG, "null argument");
    if (int rc = set_device(c)) return rc;
    const float *scans[1] = {scan};
    int ns[1] = {n};
    int status = 0;
    if (int rc = host_batch(c, 1, scans, ns, guess16, out16, converged, fitness, &status)) return rc;
    if (status & NDT_ST_WATCHDOG) return fail(c, NDT_E_WATCHDOG, "the evaluation watchdog stopped the alignment");
    if (status & NDT_ST_OVERFLOW) return fail(c, NDT_E_CAPACITY, "the FP64 side queue overflowed");
    return NDT_OK;
}

int ndt_align_with_map(ndt_ctx *c, const float *scan, int n, const float guess16[16], const float *map, int m,
                       float out16[16], int *converged, double *fitness) {
    if (int rc = ndt_set_map(c, map, m)) return rc;
    return ndt_align(c, scan, n, guess16, out16, converged, fitness);
}

int ndt_align_batch(ndt_ctx *c, int B, const float *const *scans, const int *ns, const float *guesses, float *out,
                    int *converged, double *fitness, int *status) {
    if (!c) return NDT_E_ARG;
    if (int rc = set_device(c)) return rc;
    return host_batch(c, B, scans, ns, guesses, out, converged, fitness, status);
}

int ndt_align_batch_packed(ndt_ctx *c, int B, const float *points, const int *offsets, const float *guesses,
                           float *out, int *converged, double *fitness, int *status) {
    if (!c) return NDT_E_ARG;
    if (int rc = set_device(c)) return rc;
    return packed_batch(c, B, points, offsets, guesses, out, converged, fitness, status);
}

int ndt_align_batch_packed_with_map(ndt_ctx *c, const float *map, int m, int B, const float *points,
                                    const int *offsets, const float *guesses, float *out, int *converged,
                                    double *fitness, int *status) {
    if (!c || !map) return fail(c, NDT_E_ARG, "null argument");
    if (int rc = set_device(c)) return rc;
    return packed_batch(c, B, points, offsets, guesses, out, converged, fitness, status, map, m);
}

int ndt_score_batch_device(ndt_ctx *c, int B, const float *d_points, const int *d_offsets, int total_points,
                           const float *d_poses, double *d_score) {
    if (!c || !d_points || !d_offsets || !d_poses || !d_score) return fail(c, NDT_E_ARG, "null argument");
    if (int rc = set_device(c)) return rc;
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    if (B <= 0 || total_points < 0) return fail(c, NDT_E_ARG, "empty batch");
    const int tile = c->prm.precision == 1 ? kTile : kDerivVariants[c->variant].tile;
    const int max_tiles = total_points / tile + B + 1;
    CK(c->states.ensure(sizeof(AlignState) * (size_t)B));
    RunPlan R;
    std::memset(&R, 0, sizeof(R));
    if (int rc0 = prepare_lists(c, B, max_tiles, R.L)) return rc0;
    CK(c->partials.ensure(sizeof(double) * kPartial * (size_t)max_tiles));
    CK(c->exc.ensure(sizeof(double) * kPartial * (size_t)B));
    CK(c->counters.ensure(sizeof(Counters)));
    CK(c->round_no.ensure(sizeof(int)));
    cudaStream_t st = c->stream;
    CK(cudaMemsetAsync(c->counters.p, 0, sizeof(Counters), st));
    c->ev_used = 0;
    R.P = step_params(c->prm);
    EvalArgs &ea = R.ea;
    ea.grid = grid_dev(c);
    ea.points = (const float4 *)d_points;
    ea.trans = nullptr;
    ea.tiles = c->tiles.as<Tile>();
    ea.num_tiles = c->num_tiles.as<int>();
    ea.chunks = R.L.chunks;
    ea.num_chunks = R.L.num_chunks;
    ea.max_tiles = max_tiles;
    ea.tile_size = tile;
    ea.states = c->states.as<AlignState>();
    ea.partials = c->partials.as<double>();
    ea.exc = c->exc.as<double>();
    ea.d1 = c->d1;
    ea.d2 = c->d2;
    ea.compat = c->prm.compat;
    ea.counters = c->counters.as<Counters>();
    if (int rc2 = prepare_flag_queue(c, ea)) return rc2;
    R.d_offsets = d_offsets;
    R.d_guesses = d_poses;
    R.round_no = c->round_no.as<int>();
    R.B = B;
    R.tile = tile;
    R.kb = chunk_big(c);
    R.ks = chunk_small(c);
    R.precision = c->prm.precision;
    R.variant = c->variant;
    R.sms = c->num_sms;
    if (int rc = enqueue_prologue(c, R, st)) return rc;
    int rc = launch_derivatives(R.ea, R.precision, R.variant, R.sms, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_derivatives");
    rc = launch_score(R.ea.partials, R.L.chunk_begin, R.ea.exc, B, d_score, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_score");
    c->launches += 4 + (R.precision == 1 ? 1 : kDerivLaunchesFP32) + 1;
    return NDT_OK;
}

int ndt_set_batch_graphs(ndt_ctx *c, int on) {
    if (!c) return NDT_E_ARG;
    c->use_graphs = on != 0;
    return NDT_OK;
}

int ndt_set_profiling(ndt_ctx *c, int on) {
    if (!c) return NDT_E_ARG;
    c->profiling = on != 0;
    return NDT_OK;
}

int ndt_align_batch_device(ndt_ctx *c, int B, const float *d_points, const int *d_offsets, int total_points,
                           const float *d_guesses, float *d_out, int *d_conv, double *d_fit, int *d_status) {
    if (!c || !d_points || !d_offsets || !d_guesses || !d_out || !d_conv || !d_fit)
        return fail(c, NDT_E_ARG, "null argument");
    if (int rc = set_device(c)) return rc;
    return run_batch(c, B, (const float4 *)d_points, d_offsets, total_points, d_guesses, d_out, d_conv, d_fit,
                     d_status);
}

int ndt_kernel_variants(void) { return kNumDerivVariants; }

int ndt_set_side_queue_capacity(ndt_ctx *c, int pairs) {
    if (!c || pairs < 0 || (unsigned)pairs > kFlagCapMax) return fail(c, NDT_E_ARG, "bad side-queue capacity");
    c->flag_cap = pairs == 0 ? kFlagCap : (unsigned)pairs;
    return NDT_OK;
}

int ndt_get_kernel_variant(ndt_ctx *c) { return c ? c->variant : NDT_E_ARG; }

// Times a device batch with every launch shape of the FP32 derivative pass
// (one untimed warm call each, then `repeats` calls timed with CUDA events on
// the context stream; the minimum counts) and selects the fastest; then, with
// that shape, every chunk size of kChunkChoices, and selects the fastest.
// Results go to the context's own output buffers.
int ndt_autotune_batch_device(ndt_ctx *c, int B, const float *d_points, const int *d_offsets, int total_points,
                              const float *d_guesses, int repeats, int *best, float *ms_per_variant) {
    if (!c || !d_points || !d_offsets || !d_guesses || B <= 0 || repeats < 1)
        return fail(c, NDT_E_ARG, "ndt_autotune_batch_device: bad argument");
    if (int rc = set_device(c)) return rc;
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    if (c->prm.precision == 1) {  // one launch shape only
        if (best) *best = c->variant;
        return NDT_OK;
    }
    CK(c->out_T.ensure(sizeof(float) * 16 * (size_t)B));
    CK(c->out_conv.ensure(sizeof(int) * (size_t)B));
    CK(c->out_fit.ensure(sizeof(double) * (size_t)B));
    CK(c->out_status.ensure(sizeof(int) * (size_t)B));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    cudaError_t ee = cudaEventCreate(&e1);
    if (ee != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(c, ee, "cudaEventCreate");
    }
    // the fastest of `repeats` timed calls of the current configuration, after one warm call
    auto time_config = [&](float &best_ms) -> int {
        best_ms = -1.0f;
        for (int r = 0; r <= repeats; ++r) {
            if (r > 0 && (ee = cudaEventRecord(e0, c->stream)) != cudaSuccess) return cuda_fail(c, ee, "cudaEventRecord");
            if (int rc = run_batch(c, B, (const float4 *)d_points, d_offsets, total_points, d_guesses,
                                   c->out_T.as<float>(), c->out_conv.as<int>(), c->out_fit.as<double>(),
                                   c->out_status.as<int>()))
                return rc;
            if (r == 0) continue;
            float ms = 0.0f;
            if ((ee = cudaEventRecord(e1, c->stream)) != cudaSuccess || (ee = cudaEventSynchronize(e1)) != cudaSuccess ||
                (ee = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess)
                return cuda_fail(c, ee, "autotune timing");
            if (best_ms < 0.0f || ms < best_ms) best_ms = ms;
        }
        return NDT_OK;
    };
    const int keep = c->variant, keep_chunk = c->chunk_tiles;
    int winner = keep, rc = NDT_OK;
    float winner_ms = 0.0f;
    for (int v = 0; v < kNumDerivVariants && rc == NDT_OK; ++v) {
        c->variant = v;
        float ms = 0.0f;
        if ((rc = time_config(ms)) != NDT_OK) break;
        if (ms_per_variant) ms_per_variant[v] = ms;
        if (v == 0 || ms < winner_ms) {
            winner = v;
            winner_ms = ms;
        }
    }
    int chunk = keep_chunk;
    if (rc == NDT_OK) {
        c->variant = winner;
        for (int k : kChunkChoices) {
            if (k == keep_chunk) continue;  // timed above with the winning shape
            c->chunk_tiles = k;
            float ms = 0.0f;
            if ((rc = time_config(ms)) != NDT_OK) break;
            if (ms < winner_ms) {
                chunk = k;
                winner_ms = ms;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->variant = rc ? keep : winner;
    c->chunk_tiles = rc ? keep_chunk : chunk;
    if (rc) return rc;
    if (best) *best = winner;
    return NDT_OK;
}

// The same from host buffers (packed scans as ndt_align_batch_packed takes
// them): the batch is uploaded once, then tuned on the device.
int ndt_autotune_batch(ndt_ctx *c, int B, const float *points, const int *offsets, const float *guesses,
                       int repeats, int *best, float *ms_per_variant) {
    if (!c || !points || !offsets || !guesses || B <= 0) return fail(c, NDT_E_ARG, "ndt_autotune_batch: bad argument");
    if (int rc = set_device(c)) return rc;
    const long long total = offsets[B];
    if (total < 0 || offsets[0] != 0) return fail(c, NDT_E_ARG, "ndt_autotune_batch: bad offsets");
    CK(c->points.ensure(sizeof(float4) * (size_t)std::max<long long>(1, total)));
    CK(c->offsets.ensure(sizeof(int) * (size_t)(B + 1)));
    CK(c->guesses.ensure(sizeof(float) * 16 * (size_t)B));
    CK(cudaMemcpyAsync(c->points.p, points, sizeof(float4) * (size_t)total, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->offsets.p, offsets, sizeof(int) * (size_t)(B + 1), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->guesses.p, guesses, sizeof(float) * 16 * (size_t)B, cudaMemcpyHostToDevice, c->stream));
    return ndt_autotune_batch_device(c, B, c->points.as<float>(), c->offsets.as<int>(), (int)total,
                                     c->guesses.as<float>(), repeats, best, ms_per_variant);
}

int ndt_set_kernel_variant(ndt_ctx *c, int variant) {
    if (!c || variant < 0 || variant >= kNumDerivVariants) return fail(c, NDT_E_ARG, "bad kernel variant");
    c->variant = variant;
    return NDT_OK;
}

int ndt_set_chunk_tiles(ndt_ctx *c, int tiles) {
    if (!c || tiles < 1 || tiles > kMaxChunkTiles) return fail(c, NDT_E_ARG, "chunk tiles out of range");
    c->chunk_tiles = tiles;
    return NDT_OK;
}

int ndt_get_chunk_tiles(ndt_ctx *c) { return c ? c->chunk_tiles : NDT_E_ARG; }

int ndt_kernel_variant_shape(int variant, int *tile, int *blocks_per_sm) {
    if (variant < 0 || variant >= kNumDerivVariants || !tile || !blocks_per_sm) return NDT_E_ARG;
    *tile = kDerivVariants[variant].tile;
    *blocks_per_sm = kDerivVariants[variant].min_blocks;
    return NDT_OK;
}

int ndt_get_counters(ndt_ctx *c, ndt_counters *out) {
    if (!c || !out) return NDT_E_ARG;
    if (!c->counters.p) {
        std::memset(out, 0, sizeof(*out));
        return NDT_OK;
    }
    if (int rc = read_counters(c)) return rc;
    *out = c->last;
    return NDT_OK;
}

int ndt_grid_info(ndt_ctx *c, float *bbox6, int *dims3, int *occupied) {
    if (!c) return NDT_E_ARG;
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    CK(cudaMemcpyAsync(&c->meta_host, c->meta.p, sizeof(GridMeta), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int e = 0; e < 3; ++e) {
        if (bbox6) {
            bbox6[e] = c->meta_host.minv[e];
            bbox6[3 + e] = c->meta_host.maxv[e];
        }
        if (dims3) dims3[e] = c->meta_host.dim[e];
    }
    if (occupied) *occupied = c->meta_host.occupied;
    return NDT_OK;
}

int ndt_grid_cells(ndt_ctx *c, int cap, int *cell_index, int *count, double *mean3, double *icov9) {
    int K = 0;
    if (int rc = ndt_grid_info(c, nullptr, nullptr, &K)) return rc;
    if (cap < K) return fail(c, NDT_E_CAPACITY, "cell arrays too small");
    std::vector<double4> mean(K);
    cudaStream_t st = c->stream;
    if (K) {
        if (cell_index) CK(cudaMemcpyAsync(cell_index, c->cell.p, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost, st));
        if (count) CK(cudaMemcpyAsync(count, c->count.p, sizeof(int) * (size_t)K, cudaMemcpyDeviceToHost, st));
        if (mean3) CK(cudaMemcpyAsync(mean.data(), c->mean.p, sizeof(double4) * (size_t)K, cudaMemcpyDeviceToHost, st));
        if (icov9)
            CK(cudaMemcpyAsync(icov9, c->icov64.p, sizeof(double) * 9 * (size_t)K, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    if (mean3)
        for (int k = 0; k < K; ++k) {
            mean3[3 * k] = mean[k].x;
            mean3[3 * k + 1] = mean[k].y;
            mean3[3 * k + 2] = mean[k].z;
        }
    return K;
}

int ndt_window_info(ndt_ctx *c, long long *windows, long long *entries) {
    if (!c) return NDT_E_ARG;
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    long long W = 0, E = 0;
    if (c->have_windows) {
        W = (long long)window_count(c->meta_host);
        int32_t e = 0;
        CK(cudaMemcpyAsync(&e, c->win_off.as<int32_t>() + W, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        E = e;
    }
    if (windows) *windows = W;
    if (entries) *entries = E;
    return NDT_OK;
}

int ndt_derivatives(ndt_ctx *c, const float *scan, const float *trans, int n, const double p6[6], double *score,
                    double g6[6], double H36[36]) {
    if (!c || !scan || !trans || n <= 0 || !p6 || !score || !g6 || !H36) return fail(c, NDT_E_ARG, "null argument");
    if (!c->have_map) return fail(c, NDT_E_NOMAP, "no map set");
    if (int rc = set_device(c)) return rc;
    cudaStream_t st = c->stream;
    const int tile = c->prm.precision == 1 ? kTile : kDerivVariants[c->variant].tile;
    const int max_tiles = n / tile + 2;
    CK(c->points.ensure(sizeof(float4) * (size_t)n));
    CK(c->trans.ensure(sizeof(float4) * (size_t)n));
    CK(c->offsets.ensure(sizeof(int) * 2));
    CK(c->states.ensure(sizeof(AlignState)));
    TileLists L;
    if (int rc0 = prepare_lists(c, 1, max_tiles, L)) return rc0;
    CK(c->partials.ensure(sizeof(double) * kPartial * (size_t)max_tiles));
    CK(c->exc.ensure(sizeof(double) * kPartial));
    CK(c->p6.ensure(sizeof(double) * 6));
    CK(c->counters.ensure(sizeof(Counters)));
    CK(c->h_offsets.ensure(sizeof(int) * 2));
    int *off = c->h_offsets.as<int>();
    off[0] = 0;
    off[1] = n;
    CK(cudaMemcpyAsync(c->points.p, scan, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->trans.p, trans, sizeof(float4) * (size_t)n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->offsets.p, off, sizeof(int) * 2, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->p6.p, p6, sizeof(double) * 6, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(c->counters.p, 0, sizeof(Counters), st));
    int rc = launch_tiles(c->offsets.as<int>(), 1, tile, chunk_big(c), chunk_small(c), L, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_tiles");
    rc = launch_prepare_eval(c->states.as<AlignState>(), c->p6.as<double>(), n, c->exc.as<double>(), c->prm.compat,
                             st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_prepare_eval");
    EvalArgs ea;
    ea.grid = grid_dev(c);
    ea.points = c->points.as<float4>();
    ea.trans = c->trans.as<float4>();
    ea.tiles = c->tiles.as<Tile>();
    ea.num_tiles = c->num_tiles.as<int>();
    ea.chunks = L.chunks;
    ea.num_chunks = L.num_chunks;
    ea.max_tiles = max_tiles;
    ea.tile_size = tile;
    ea.states = c->states.as<AlignState>();
    ea.partials = c->partials.as<double>();
    ea.exc = c->exc.as<double>();
    ea.d1 = c->d1;
    ea.d2 = c->d2;
    ea.compat = c->prm.compat;
    ea.counters = c->counters.as<Counters>();
    if (int rc2 = prepare_flag_queue(c, ea)) return rc2;
    rc = launch_derivatives(ea, c->prm.precision, c->variant, c->num_sms, st);
    if (rc) return cuda_fail(c, (cudaError_t)rc, "launch_derivatives");
    int nt = 0;
    std::vector<double> part((size_t)max_tiles * kPartial), exc(kPartial);
    CK(cudaMemcpyAsync(&nt, c->num_chunks.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpyAsync(part.data(), c->partials.p, sizeof(double) * kPartial * (size_t)nt, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(exc.data(), c->exc.p, sizeof(double) * kPartial, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double v[kPartial] = {0};
    for (int t = 0; t < nt; ++t)
        for (int k = 0; k < kPartial; ++k) v[k] += part[(size_t)t * kPartial + k];
    for (int k = 0; k < kPartial; ++k) v[k] += exc[k];
    *score = v[0];
    for (int i = 0; i < 6; ++i) g6[i] = v[1 + i];
    for (int k = 0; k < 36; ++k) H36[k] = v[7 + k];
    return read_counters(c);
}

}  // extern "C"
