// The ndt_mapping input file on the fast path: the file is memory-mapped and
// indexed once (no per-value reads), its pages are registered with the CUDA
// driver so that scans and maps go to the device by asynchronous DMA straight
// from the mapping, and a run of test cases is aligned in chunks whose
// uploads (on a copy stream, double-buffered) overlap the previous chunk's
// alignments.  The reference reads the same format one value at a time
// (parseInitGuess / parseFilteredScan, src/CPU/ndt_mapping/kernel.cpp:143-173,
// read_next_testcases :192-229).
//
// Format (little-endian, packed): int32 T; T times: float32[16] guess (row
// major), int32 N + N x float32[4] scan, int32 M + M x float32[4] map.
//
// Map reuse: at open the maps are compared with their predecessors (threads
// over the test cases): a map byte-identical to the previous case's reuses
// the grid; a map that is the previous map followed by more points grows it
// (ndt_map_append); any other map is built anew.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <stdint.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ndt_b200.h"
#include "ctx_view.h"
#include "nvtx_range.h"

struct ndt_dat {
    int fd = -1;
    const unsigned char *base = nullptr;
    size_t size = 0;
    int device = -1;          // device the mapping is registered on (-1: not registered)
    bool registered = false;
    int T = 0;
    std::vector<const float *> guess, scan, map;
    std::vector<int> n, m;
    std::vector<uint8_t> rel;  // NDT_DAT_MAP_*: relation of case i's map to case i - 1's
    std::string err;
    // runner buffers (on `device`)
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr}, used[2] = {nullptr, nullptr};
    float *d_pts[2] = {nullptr, nullptr};
    size_t pts_cap[2] = {0, 0};
    int *d_off[2] = {nullptr, nullptr};
    float *d_guess[2] = {nullptr, nullptr};
    int chunk_cap = 0;
    int *h_off = nullptr;    // pinned: 2 x (chunk_cap + 1)
    float *h_guess = nullptr;  // pinned: 2 x chunk_cap x 16
    float *d_out = nullptr;
    int *d_conv = nullptr, *d_status = nullptr;
    double *d_fit = nullptr;
    int out_cap = 0;
};

namespace {

constexpr int kChunk = 512;  // test cases per alignment batch of the runner

int fail(ndt_dat *d, int code, const std::string &msg) {
    if (d) d->err = msg;
    return code;
}

// Compares ranges of two maps in parallel (the maps are megabytes).
bool equal_bytes(const void *a, const void *b, size_t bytes) {
    if (a == b) return true;
    const size_t kPiece = 1 << 20;
    if (bytes <= 4 * kPiece) return std::memcmp(a, b, bytes) == 0;
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    std::atomic<bool> same{true};
    std::atomic<size_t> next{0};
    auto work = [&]() {
        for (;;) {
            const size_t off = next.fetch_add(kPiece);
            if (off >= bytes || !same.load()) return;
            const size_t len = std::min(kPiece, bytes - off);
            if (std::memcmp((const char *)a + off, (const char *)b + off, len) != 0) same = false;
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < hw; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    return same.load();
}

int ensure_dev(ndt_dat *d, void **p, size_t *cap, size_t bytes) {
    if (*cap >= bytes && *p) return NDT_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    const size_t want = std::max(bytes + bytes / 2, (size_t)4096);
    cudaError_t e = cudaMalloc(p, want);
    if (e != cudaSuccess) return fail(d, NDT_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    *cap = want;
    return NDT_OK;
}

void release_runner(ndt_dat *d) {
    if (d->device < 0) return;
    cudaSetDevice(d->device);
    if (d->copy) cudaStreamSynchronize(d->copy);
    for (int b = 0; b < 2; ++b) {
        if (d->copied[b]) cudaEventDestroy(d->copied[b]);
        if (d->used[b]) cudaEventDestroy(d->used[b]);
        if (d->d_pts[b]) cudaFree(d->d_pts[b]);
        if (d->d_off[b]) cudaFree(d->d_off[b]);
        if (d->d_guess[b]) cudaFree(d->d_guess[b]);
    }
    if (d->h_off) cudaFreeHost(d->h_off);
    if (d->h_guess) cudaFreeHost(d->h_guess);
    if (d->d_out) cudaFree(d->d_out);
    if (d->d_conv) cudaFree(d->d_conv);
    if (d->d_status) cudaFree(d->d_status);
    if (d->d_fit) cudaFree(d->d_fit);
    if (d->copy) cudaStreamDestroy(d->copy);
    if (d->registered) cudaHostUnregister((void *)d->base);
    d->registered = false;
    d->device = -1;
}

// Per-device set-up of the runner: the copy stream, events, pinned staging of
// offsets and guesses, and the registration of the mapping (if the driver
// refuses it, uploads read the mapping as pageable memory).
int prepare_runner(ndt_dat *d, int device) {
    if (d->device == device) return NDT_OK;
    release_runner(d);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->copy, cudaStreamNonBlocking);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaEventCreateWithFlags(&d->copied[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&d->used[b], cudaEventDisableTiming);
    }
    d->chunk_cap = kChunk;
    if (e == cudaSuccess) e = cudaMallocHost((void **)&d->h_off, sizeof(int) * 2 * (kChunk + 1));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&d->h_guess, sizeof(float) * 2 * kChunk * 16);
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMalloc((void **)&d->d_off[b], sizeof(int) * (kChunk + 1));
        if (e == cudaSuccess) e = cudaMalloc((void **)&d->d_guess[b], sizeof(float) * kChunk * 16);
    }
    d->device = device;
    if (e != cudaSuccess) {
        std::string msg = std::string("runner set-up: ") + cudaGetErrorString(e);
        release_runner(d);
        return fail(d, NDT_E_CUDA, msg);
    }
    if (d->size > 0) {
        e = cudaHostRegister((void *)d->base, d->size, cudaHostRegisterReadOnly);
        d->registered = e == cudaSuccess;
        if (e != cudaSuccess) cudaGetLastError();  // clear: pageable uploads still work
    }
    return NDT_OK;
}

}  // namespace

extern "C" {

int ndt_dat_open(const char *path, ndt_dat **out) {
    if (!out) return NDT_E_ARG;
    ndt_dat *d = new ndt_dat();
    *out = d;
    if (!path) return fail(d, NDT_E_ARG, "null path");
    d->fd = open(path, O_RDONLY);
    if (d->fd < 0) return fail(d, NDT_E_ARG, std::string("Error opening the testcase file: ") + std::strerror(errno));
    struct stat sb;
    if (fstat(d->fd, &sb) != 0) return fail(d, NDT_E_ARG, std::string("fstat: ") + std::strerror(errno));
    d->size = (size_t)sb.st_size;
    if (d->size < 4) return fail(d, NDT_E_ARG, "Error reading number of test cases");
    void *p = mmap(nullptr, d->size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, d->fd, 0);
    if (p == MAP_FAILED) return fail(d, NDT_E_ARG, std::string("mmap: ") + std::strerror(errno));
    d->base = (const unsigned char *)p;
    int32_t T;
    std::memcpy(&T, d->base, 4);
    if (T < 0) return fail(d, NDT_E_ARG, "negative test case count");
    size_t off = 4;
    auto need = [&](size_t bytes) { return off + bytes <= d->size; };
    for (int i = 0; i < T; ++i) {
        if (!need(64)) return fail(d, NDT_E_ARG, "file ends inside test case " + std::to_string(i) + " (guess)");
        d->guess.push_back((const float *)(d->base + off));
        off += 64;
        for (int k = 0; k < 2; ++k) {
            int32_t cnt;
            if (!need(4)) return fail(d, NDT_E_ARG, "file ends inside test case " + std::to_string(i) + " (count)");
            std::memcpy(&cnt, d->base + off, 4);
            off += 4;
            if (cnt < 0) return fail(d, NDT_E_ARG, "negative point count in test case " + std::to_string(i));
            if (!need(16 * (size_t)cnt))
                return fail(d, NDT_E_ARG, "file ends inside test case " + std::to_string(i) + " (points)");
            (k == 0 ? d->scan : d->map).push_back((const float *)(d->base + off));
            (k == 0 ? d->n : d->m).push_back(cnt);
            off += 16 * (size_t)cnt;
        }
    }
    d->T = T;
    // map relations, compared in parallel over the test cases
    d->rel.assign(T, NDT_DAT_MAP_NEW);
    std::atomic<int> next{1};
    auto work = [&]() {
        for (int i = next.fetch_add(1); i < T; i = next.fetch_add(1)) {
            const size_t a = 16 * (size_t)d->m[i - 1], b = 16 * (size_t)d->m[i];
            if (d->m[i] > 0 && d->m[i - 1] > 0 && a <= b && std::memcmp(d->map[i], d->map[i - 1], 16) == 0 &&
                equal_bytes(d->map[i], d->map[i - 1], a))
                d->rel[i] = a == b ? NDT_DAT_MAP_SAME : NDT_DAT_MAP_GROWN;
        }
    };
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < hw; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    d->err.clear();
    return NDT_OK;
}

void ndt_dat_close(ndt_dat *d) {
    if (!d) return;
    release_runner(d);
    if (d->base) munmap((void *)d->base, d->size);
    if (d->fd >= 0) close(d->fd);
    delete d;
}

const char *ndt_dat_last_error(const ndt_dat *d) { return d ? d->err.c_str() : "null handle"; }

int ndt_dat_count(const ndt_dat *d) { return d ? d->T : 0; }

int ndt_dat_case(const ndt_dat *d, int i, const float **guess16, const float **scan, int *n, const float **map,
                 int *m) {
    if (!d || i < 0 || i >= d->T) return NDT_E_ARG;
    if (guess16) *guess16 = d->guess[i];
    if (scan) *scan = d->scan[i];
    if (n) *n = d->n[i];
    if (map) *map = d->map[i];
    if (m) *m = d->m[i];
    return NDT_OK;
}

int ndt_dat_map_relation(const ndt_dat *d, int i) {
    if (!d || i < 0 || i >= d->T) return NDT_E_ARG;
    return d->rel[i];
}

int ndt_dat_align(ndt_ctx *ctx, ndt_dat *d, int first, int count, float *out16, int *converged, double *fitness,
                  int *status) {
    ndt::NvtxRange range("dat align");
    if (!ctx || !d || first < 0 || count < 0 || (long long)first + count > d->T ||
        (count > 0 && (!out16 || !converged || !fitness)))
        return d ? fail(d, NDT_E_ARG, "bad argument") : NDT_E_ARG;
    if (count == 0) return NDT_OK;
    ndt::CtxEvalView v;
    if (ndt::ctx_eval_view(ctx, &v) != 0) return fail(d, NDT_E_ARG, "bad context");
    if (int rc = prepare_runner(d, v.device)) return rc;
    cudaStream_t st = v.stream, cp = d->copy;
#define DCK(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(d, NDT_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
    if (d->out_cap < count) {
        if (d->d_out) cudaFree(d->d_out);
        if (d->d_conv) cudaFree(d->d_conv);
        if (d->d_status) cudaFree(d->d_status);
        if (d->d_fit) cudaFree(d->d_fit);
        d->d_out = nullptr;
        d->d_conv = d->d_status = nullptr;
        d->d_fit = nullptr;
        d->out_cap = 0;
        DCK(cudaMalloc((void **)&d->d_out, sizeof(float) * 16 * (size_t)count));
        DCK(cudaMalloc((void **)&d->d_conv, sizeof(int) * (size_t)count));
        DCK(cudaMalloc((void **)&d->d_status, sizeof(int) * (size_t)count));
        DCK(cudaMalloc((void **)&d->d_fit, sizeof(double) * (size_t)count));
        d->out_cap = count;
    }
    // chunks: runs of test cases that share a map, at most kChunk each
    int chunk_no = 0;
    const float *cur_map = nullptr;  // the map the context holds (a pointer into the mapping)
    int cur_m = 0;
    for (int i = first; i < first + count;) {
        // the map of case i
        const bool same = cur_map && (d->map[i] == cur_map ||
                                      (i > first && d->rel[i] == NDT_DAT_MAP_SAME && d->map[i - 1] == cur_map));
        if (!same) {
            int rc;
            if (cur_map && i > first && d->rel[i] == NDT_DAT_MAP_GROWN && d->map[i - 1] == cur_map)
                rc = ndt_map_append(ctx, d->map[i] + 4 * (size_t)cur_m, d->m[i] - cur_m);
            else
                rc = ndt_set_map(ctx, d->map[i], d->m[i]);
            if (rc != NDT_OK) return fail(d, rc, std::string("map of test case ") + std::to_string(i) + ": " +
                                                      ndt_last_error(ctx));
            cur_map = d->map[i];
            cur_m = d->m[i];
        }
        int j = i + 1;
        while (j < first + count && j - i < kChunk && d->rel[j] == NDT_DAT_MAP_SAME) ++j;
        const int B = j - i, buf = chunk_no & 1;
        // the buffer's previous chunk must have finished aligning before it is overwritten
        DCK(cudaStreamWaitEvent(cp, d->used[buf], 0));
        int *ho = d->h_off + buf * (kChunk + 1);
        float *hg = d->h_guess + (size_t)buf * kChunk * 16;
        // pinned staging is reused only after the copy that read it has run
        DCK(cudaEventSynchronize(d->copied[buf]));
        ho[0] = 0;
        for (int b = 0; b < B; ++b) {
            ho[b + 1] = ho[b] + d->n[i + b];
            std::memcpy(hg + 16 * b, d->guess[i + b], 64);
        }
        const int total = ho[B];
        if (int rc = ensure_dev(d, (void **)&d->d_pts[buf], &d->pts_cap[buf], 16 * (size_t)std::max(total, 1)))
            return rc;
        for (int b = 0; b < B; ++b)
            if (d->n[i + b] > 0)
                DCK(cudaMemcpyAsync(d->d_pts[buf] + 4 * (size_t)ho[b], d->scan[i + b], 16 * (size_t)d->n[i + b],
                                    cudaMemcpyHostToDevice, cp));
        DCK(cudaMemcpyAsync(d->d_off[buf], ho, sizeof(int) * (B + 1), cudaMemcpyHostToDevice, cp));
        DCK(cudaMemcpyAsync(d->d_guess[buf], hg, sizeof(float) * 16 * B, cudaMemcpyHostToDevice, cp));
        DCK(cudaEventRecord(d->copied[buf], cp));
        DCK(cudaStreamWaitEvent(st, d->copied[buf], 0));
        const int r = i - first;
        int rc = ndt_align_batch_device(ctx, B, d->d_pts[buf], d->d_off[buf], total, d->d_guess[buf],
                                        d->d_out + 16 * (size_t)r, d->d_conv + r, d->d_fit + r, d->d_status + r);
        if (rc != NDT_OK) return fail(d, rc, std::string("alignments: ") + ndt_last_error(ctx));
        DCK(cudaEventRecord(d->used[buf], st));
        ++chunk_no;
        i = j;
    }
    DCK(cudaMemcpyAsync(out16, d->d_out, sizeof(float) * 16 * (size_t)count, cudaMemcpyDeviceToHost, st));
    DCK(cudaMemcpyAsync(converged, d->d_conv, sizeof(int) * (size_t)count, cudaMemcpyDeviceToHost, st));
    DCK(cudaMemcpyAsync(fitness, d->d_fit, sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost, st));
    if (status) DCK(cudaMemcpyAsync(status, d->d_status, sizeof(int) * (size_t)count, cudaMemcpyDeviceToHost, st));
    DCK(cudaStreamSynchronize(st));
#undef DCK
    return NDT_OK;
}

}  // extern "C"
