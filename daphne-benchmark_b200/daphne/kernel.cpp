// DAPHNE ndt_mapping front end on the B200 library: the benchmark kernel the
// reference harness runs (src/CPU/ndt_mapping/kernel.cpp:22-137, 192-229,
// 345-377, 1416-1506), with the per-test-case align call replaced by batched
// GPU alignments through the C ABI of include/ndt_b200.h.
//
// Behaviour kept from the reference: the data file formats and default paths
// (../../../data/ndt_input.dat, ../../../data/ndt_output.dat), the -p block
// size, timer pauses around reading and checking, the acceptance rule of
// check_next_outputs (including its running max_delta) and the exit(-3) on
// I/O errors.  Different: run() hands a whole block of test cases to the GPU
// at once; test cases whose maps are byte-identical share one voxel-grid
// build (the maps are compared while reading, with the timer paused).
//
// The derivative pass's launch shape is autotuned on the first batch (timer
// paused; NDT_AUTOTUNE=0 keeps the library's default shape).
//
// Environment: NDT_INPUT / NDT_OUTPUT override the data paths,
// NDT_DATAGEN_OUT writes every result in the output-file format (the
// reference's datagen variant), NDT_PRECISION=1 selects FP64 pair arithmetic,
// NDT_DEVICE the CUDA device.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/ndt_b200.h"
#include "benchmark.h"

namespace {

constexpr double kMaxTranslationEps = 0.001;  // kernel.cpp:18
constexpr double kMaxEps = 2;                 // kernel.cpp:20

struct Testcase {
    float guess[16];
    std::vector<float> scan;  // n x 4
    std::vector<float> map;   // m x 4
    uint64_t map_hash = 0;
};

struct Result {
    float T[16];
    double fitness;
    int converged;
};

uint64_t fnv1a(const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    uint64_t h = 1469598103934665603ull;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}

const char *env_or(const char *name, const char *dflt) {
    const char *v = std::getenv(name);
    return (v && *v) ? v : dflt;
}

}  // namespace

class ndt_mapping : public kernel {
public:
    ~ndt_mapping() {
        if (ctx_) ndt_destroy(ctx_);
    }
    void init() override;
    void run(int p = 1) override;
    bool check_output() override;

protected:
    int read_next_testcases(int count) override;
    void check_next_outputs(int count);
    void align_block(int count);

private:
    std::ifstream input_file_, output_file_;
    std::ofstream datagen_;
    int read_testcases_ = 0;
    std::vector<Testcase> cases_;
    std::vector<Result> results_;
    bool error_so_far_ = false;
    double max_delta_ = 0.0;
    ndt_ctx *ctx_ = nullptr;
    bool tuned_ = false;
};

void ndt_mapping::init() {
    std::cout << "init\n";
    input_file_.exceptions(std::ifstream::failbit | std::ifstream::badbit);
    output_file_.exceptions(std::ifstream::failbit | std::ifstream::badbit);
    try {
        input_file_.open(env_or("NDT_INPUT", "../../../data/ndt_input.dat"), std::ios::binary);
    } catch (std::ifstream::failure &) {
        std::cerr << "Error opening the testcase file" << std::endl;
        std::exit(-3);
    }
    try {
        output_file_.open(env_or("NDT_OUTPUT", "../../../data/ndt_output.dat"), std::ios::binary);
    } catch (std::ifstream::failure &) {
        std::cerr << "Error opening the results file" << std::endl;
        std::exit(-3);
    }
    if (const char *dg = std::getenv("NDT_DATAGEN_OUT")) datagen_.open(dg, std::ios::binary);
    try {
        int32_t n = 0;
        input_file_.read((char *)&n, sizeof(int32_t));
        testcases = (uint32_t)n;
    } catch (std::ios_base::failure &) {
        std::cerr << "Error reading number of test cases" << std::endl;
        std::exit(-3);
    }
    ndt_params prm;
    ndt_params_reference(&prm);
    prm.precision = std::atoi(env_or("NDT_PRECISION", "0")) == 1 ? 1 : 0;
    int rc = ndt_create(&prm, std::atoi(env_or("NDT_DEVICE", "0")), &ctx_);
    if (rc != NDT_OK) {
        std::cerr << "ndt_create failed (" << rc << "): no usable CUDA device" << std::endl;
        std::exit(-3);
    }
    error_so_far_ = false;
    max_delta_ = 0.0;
    std::cout << "done\n" << std::endl;
}

// parseInitGuess / parseFilteredScan (kernel.cpp:143-173): float[16] guess,
// int32 N + N x float[4] scan, int32 M + M x float[4] map.
int ndt_mapping::read_next_testcases(int count) {
    cases_.clear();
    cases_.resize(count);
    int i = 0;
    for (; i < count && read_testcases_ < (int)testcases; ++i, ++read_testcases_) {
        Testcase &t = cases_[i];
        try {
            input_file_.read((char *)t.guess, sizeof(float) * 16);
            for (std::vector<float> *cloud : {&t.scan, &t.map}) {
                int32_t n = 0;
                input_file_.read((char *)&n, sizeof(int32_t));
                if (n < 0) throw std::ios_base::failure("negative point count");
                cloud->resize(4 * (size_t)n);
                if (n) input_file_.read((char *)cloud->data(), sizeof(float) * 4 * (size_t)n);
            }
        } catch (std::ios_base::failure &e) {
            std::cerr << e.what() << std::endl;
            std::exit(-3);
        }
        t.map_hash = fnv1a(t.map.data(), sizeof(float) * t.map.size());
    }
    cases_.resize(i);
    return i;
}

// One GPU batch per distinct map of the block.
void ndt_mapping::align_block(int count) {
    results_.assign(count, Result{});
    std::vector<char> done(count, 0);
    for (int i = 0; i < count; ++i) {
        if (done[i]) continue;
        const Testcase &lead = cases_[i];
        std::vector<int> members;
        for (int j = i; j < count; ++j) {
            const Testcase &t = cases_[j];
            if (!done[j] && t.map_hash == lead.map_hash && t.map.size() == lead.map.size() &&
                std::memcmp(t.map.data(), lead.map.data(), sizeof(float) * t.map.size()) == 0) {
                members.push_back(j);
                done[j] = 1;
            }
        }
        int rc = ndt_set_map(ctx_, lead.map.data(), (int)(lead.map.size() / 4));
        if (rc != NDT_OK) {
            std::cerr << "ndt_set_map failed: " << ndt_last_error(ctx_) << std::endl;
            std::exit(-3);
        }
        const int B = (int)members.size();
        std::vector<const float *> scans(B);
        std::vector<int> ns(B), conv(B), status(B);
        std::vector<float> guesses(16 * (size_t)B), out(16 * (size_t)B);
        std::vector<double> fit(B);
        for (int b = 0; b < B; ++b) {
            const Testcase &t = cases_[members[b]];
            scans[b] = t.scan.data();
            ns[b] = (int)(t.scan.size() / 4);
            std::memcpy(&guesses[16 * (size_t)b], t.guess, sizeof(float) * 16);
        }
        if (!tuned_) {
            // the launch shape of the derivative pass, tuned once on the first batch (timer paused: set-up)
            tuned_ = true;
            if (std::strcmp(env_or("NDT_AUTOTUNE", "1"), "0") != 0) {
                std::vector<int> offs(B + 1, 0);
                for (int b = 0; b < B; ++b) offs[b + 1] = offs[b] + ns[b];
                std::vector<float> packed(4 * (size_t)offs[B]);
                for (int b = 0; b < B; ++b)
                    std::memcpy(&packed[4 * (size_t)offs[b]], scans[b], sizeof(float) * 4 * (size_t)ns[b]);
                if (pause_func) pause_func();
                int best = 0;
                rc = ndt_autotune_batch(ctx_, B, packed.data(), offs.data(), guesses.data(), 1, &best, nullptr);
                if (unpause_func) unpause_func();
                if (rc != NDT_OK) {
                    std::cerr << "ndt_autotune_batch failed: " << ndt_last_error(ctx_) << std::endl;
                    std::exit(-3);
                }
            }
        }
        rc = ndt_align_batch(ctx_, B, scans.data(), ns.data(), guesses.data(), out.data(), conv.data(), fit.data(),
                             status.data());
        if (rc != NDT_OK) {
            std::cerr << "ndt_align_batch failed: " << ndt_last_error(ctx_) << std::endl;
            std::exit(-3);
        }
        for (int b = 0; b < B; ++b) {
            Result &r = results_[members[b]];
            std::memcpy(r.T, &out[16 * (size_t)b], sizeof(float) * 16);
            r.fitness = fit[b];
            r.converged = conv[b];
        }
    }
}

// ndt_mapping::run (kernel.cpp:1416-1434).
void ndt_mapping::run(int p) {
    pause_func();
    while (read_testcases_ < (int)testcases) {
        int count = read_next_testcases(p);
        unpause_func();
        align_block(count);
        pause_func();
        check_next_outputs(count);
    }
}

// check_next_outputs (kernel.cpp:1436-1496): converged equal, NaN pattern
// equal, translation column within 0.001 and the transformed test point within
// 2; a threshold is tested only when a new maximum delta is set, as there.
void ndt_mapping::check_next_outputs(int count) {
    for (int i = 0; i < count; ++i) {
        float ref[16];
        double ref_fit = 0;
        bool ref_conv = false;
        try {
            output_file_.read((char *)ref, sizeof(float) * 16);
            output_file_.read((char *)&ref_fit, sizeof(double));
            output_file_.read((char *)&ref_conv, sizeof(bool));
        } catch (std::ios_base::failure &e) {
            std::cerr << e.what() << std::endl;
            std::exit(-3);
        }
        const Result &r = results_[i];
        if (datagen_.is_open()) {
            bool c = r.converged != 0;
            datagen_.write((const char *)r.T, sizeof(float) * 16);
            datagen_.write((const char *)&r.fitness, sizeof(double));
            datagen_.write((const char *)&c, sizeof(bool));
        }
        if ((r.converged != 0) != ref_conv) error_so_far_ = true;
        for (int h = 0; h < 4; ++h) {
            for (int w = 0; w < 4; ++w)
                if (std::isnan(r.T[4 * h + w]) != std::isnan(ref[4 * h + w])) error_so_far_ = true;
            float delta = std::fabs(r.T[4 * h + 3] - ref[4 * h + 3]);
            if (delta > max_delta_) {
                max_delta_ = delta;
                if (delta > kMaxTranslationEps) error_so_far_ = true;
            }
        }
        const float origin[4] = {0.724f, 0.447f, 0.525f, 1.0f};
        float res_pt[4] = {0, 0, 0, 0}, ref_pt[4] = {0, 0, 0, 0};
        for (int h = 0; h < 4; ++h)
            for (int w = 0; w < 4; ++w) {
                res_pt[h] += r.T[4 * h + w] * origin[w];
                ref_pt[h] += ref[4 * h + w] * origin[w];
            }
        for (int w = 0; w < 4; ++w) {
            float delta = std::fabs(res_pt[w] - ref_pt[w]);
            if (delta > max_delta_) {
                max_delta_ = delta;
                if (delta > kMaxEps) error_so_far_ = true;
            }
        }
    }
}

bool ndt_mapping::check_output() {
    std::cout << "checking output \n";
    input_file_.close();
    output_file_.close();
    if (datagen_.is_open()) datagen_.close();
    std::cout << "max delta: " << max_delta_ << "\n";
    return !error_so_far_;
}

static ndt_mapping the_kernel;
kernel &myKernel = the_kernel;
