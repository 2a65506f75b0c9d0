// DAPHNE euclidean_cluster front end on the B200 library: the benchmark kernel
// the reference harness runs (src/CPU/euclidean_cluster/kernel.cpp:906-1127),
// with segmentByDistance replaced by batched GPU clustering through the C ABI
// of include/ndt_b200.h (ndt_ec_segment_batch: a block of clouds per call).
//
// Kept from the reference: the data formats and default paths
// (../../../data/ec_input.dat, ../../../data/ec_output.dat), the -p block
// size, timer pauses around reading and checking, the acceptance rule of
// check_next_outputs (both sides sorted, equal sizes, max |difference| of
// points, box position / dimensions / orientation x and y, centroids,
// <= 0.001) and exit(-3) on I/O errors.  The library computes the box yaw
// (orientation z, w) too; the rule does not compare it.
//
// Environment: EC_INPUT / EC_OUTPUT override the data paths, EC_DEVICE the
// CUDA device.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "../../include/ndt_b200.h"
#include "../daphne/benchmark.h"

namespace {

constexpr double kMaxEps = 0.001;  // kernel.cpp:22

struct PointRGB {
    float x, y, z;
    uint8_t r, g, b;
};
struct Box {  // the output file's fields
    double px, py, ox, oy, oz, ow, dx, dy;
};

const char *env_or(const char *name, const char *dflt) {
    const char *v = std::getenv(name);
    return (v && *v) ? v : dflt;
}

bool less_point(const PointRGB &a, const PointRGB &b) {
    if (a.x != b.x) return a.x < b.x;
    if (a.y != b.y) return a.y < b.y;
    return a.z < b.z;
}
bool less_box(const Box &a, const Box &b) {
    if (a.px != b.px) return a.px < b.px;
    if (a.py != b.py) return a.py < b.py;
    if (a.dx != b.dx) return a.dx < b.dx;
    return a.dy < b.dy;
}
bool less_centroid(const double *a, const double *b) {
    if (a[0] != b[0]) return a[0] < b[0];
    if (a[1] != b[1]) return a[1] < b[1];
    return a[2] < b[2];
}

template <class T>
void read_exact(std::ifstream &f, T *p, size_t n, const char *what) {
    f.read((char *)p, sizeof(T) * n);
    if (!f) {
        std::cerr << what << std::endl;
        std::exit(-3);
    }
}

}  // namespace

class euclidean_clustering : public kernel {
public:
    ~euclidean_clustering() {
        if (ec_) ndt_ec_destroy(ec_);
    }
    void init() override;
    void run(int p = 1) override;
    bool check_output() override;

protected:
    int read_next_testcases(int count) override;
    void check_next_outputs(int count);

private:
    std::ifstream input_file_, output_file_;
    int read_testcases_ = 0;
    std::vector<float> xyz_;  // the block's clouds, packed
    std::vector<int> off_;
    std::vector<float> out_xyz_;
    std::vector<int> out_off_, box_off_;
    std::vector<double> boxes_, centroids_;
    bool error_so_far_ = false;
    double max_delta_ = 0.0;
    ndt_ec *ec_ = nullptr;
};

void euclidean_clustering::init() {
    std::cout << "init\n";
    input_file_.open(env_or("EC_INPUT", "../../../data/ec_input.dat"), std::ios::binary);
    if (!input_file_) {
        std::cerr << "Error opening the input data file" << std::endl;
        std::exit(-3);
    }
    output_file_.open(env_or("EC_OUTPUT", "../../../data/ec_output.dat"), std::ios::binary);
    if (!output_file_) {
        std::cerr << "Error opening the output data file" << std::endl;
        std::exit(-3);
    }
    int32_t n = 0;
    read_exact(input_file_, &n, 1, "Error reading the number of testcases");
    testcases = (uint32_t)n;
    if (ndt_ec_create(std::atoi(env_or("EC_DEVICE", "0")), &ec_) != NDT_OK) {
        std::cerr << "ndt_ec_create failed: no usable CUDA device" << std::endl;
        std::exit(-3);
    }
    error_so_far_ = false;
    max_delta_ = 0.0;
    std::cout << "done\n" << std::endl;
}

// parsePointCloud (kernel.cpp:816-835): int32 n + n x float32[3].
int euclidean_clustering::read_next_testcases(int count) {
    xyz_.clear();
    off_.assign(1, 0);
    int i = 0;
    for (; i < count && read_testcases_ < (int)testcases; ++i, ++read_testcases_) {
        int32_t n = 0;
        read_exact(input_file_, &n, 1, "Error reading point cloud");
        if (n < 0) {
            std::cerr << "Error reading point cloud" << std::endl;
            std::exit(-3);
        }
        const size_t at = xyz_.size();
        xyz_.resize(at + 3 * (size_t)n);
        if (n) read_exact(input_file_, xyz_.data() + at, 3 * (size_t)n, "Error reading point cloud");
        off_.push_back(off_.back() + n);
    }
    return i;
}

// euclidean_clustering::run (kernel.cpp:971-993), one GPU call per block.
void euclidean_clustering::run(int p) {
    pause_func();
    while (read_testcases_ < (int)testcases) {
        const int count = read_next_testcases(p);
        unpause_func();
        const size_t n = (size_t)off_.back();
        out_xyz_.resize(3 * std::max<size_t>(n, 1));
        boxes_.resize(10 * std::max<size_t>(n, 1));
        centroids_.resize(3 * std::max<size_t>(n, 1));
        out_off_.assign(count + 1, 0);
        box_off_.assign(count + 1, 0);
        const int rc = ndt_ec_segment_batch(ec_, count, xyz_.data(), off_.data(), out_xyz_.data(), out_off_.data(),
                                            boxes_.data(), box_off_.data(), centroids_.data());
        if (rc != NDT_OK) {
            std::cerr << "ndt_ec_segment_batch failed: " << ndt_ec_last_error(ec_) << std::endl;
            std::exit(-3);
        }
        pause_func();
        check_next_outputs(count);
    }
}

// check_next_outputs (kernel.cpp:1034-1093).
void euclidean_clustering::check_next_outputs(int count) {
    for (int c = 0; c < count; ++c) {
        int32_t n = 0;
        read_exact(output_file_, &n, 1, "Error reading reference cloud");
        std::vector<PointRGB> ref(n > 0 ? n : 0);
        for (PointRGB &q : ref) {
            read_exact(output_file_, &q.x, 3, "Error reading reference cloud");
            read_exact(output_file_, &q.r, 3, "Error reading reference cloud");
        }
        int32_t nb = 0;
        read_exact(output_file_, &nb, 1, "Error reading reference bounding boxes");
        std::vector<Box> rb(nb > 0 ? nb : 0);
        for (Box &b : rb) read_exact(output_file_, &b.px, 8, "Error reading reference bounding boxes");
        int32_t nc = 0;
        read_exact(output_file_, &nc, 1, "Error reading reference centroids");
        std::vector<double> rc(3 * (size_t)(nc > 0 ? nc : 0));
        if (nc > 0) read_exact(output_file_, rc.data(), rc.size(), "Error reading reference centroids");
        // ours
        std::vector<PointRGB> pts;
        for (int i = out_off_[c]; i < out_off_[c + 1]; ++i)
            pts.push_back({out_xyz_[3 * (size_t)i], out_xyz_[3 * (size_t)i + 1], out_xyz_[3 * (size_t)i + 2], 10, 20,
                           30});
        std::vector<Box> bx;
        std::vector<double> ce;
        for (int i = box_off_[c]; i < box_off_[c + 1]; ++i) {
            const double *b = &boxes_[10 * (size_t)i];
            bx.push_back({b[0], b[1], b[3], b[4], b[5], b[6], b[7], b[8]});
            ce.insert(ce.end(), &centroids_[3 * (size_t)i], &centroids_[3 * (size_t)i] + 3);
        }
        std::sort(ref.begin(), ref.end(), less_point);
        std::sort(pts.begin(), pts.end(), less_point);
        std::sort(rb.begin(), rb.end(), less_box);
        std::sort(bx.begin(), bx.end(), less_box);
        std::vector<const double *> rcp, cep;
        for (size_t i = 0; i < rc.size(); i += 3) rcp.push_back(&rc[i]);
        for (size_t i = 0; i < ce.size(); i += 3) cep.push_back(&ce[i]);
        std::sort(rcp.begin(), rcp.end(), less_centroid);
        std::sort(cep.begin(), cep.end(), less_centroid);
        if (ref.size() != pts.size() || rb.size() != bx.size() || rcp.size() != cep.size()) {
            error_so_far_ = true;
            continue;
        }
        for (size_t j = 0; j < ref.size(); ++j) {
            max_delta_ = std::fmax(std::fabs(pts[j].x - ref[j].x), max_delta_);
            max_delta_ = std::fmax(std::fabs(pts[j].y - ref[j].y), max_delta_);
            max_delta_ = std::fmax(std::fabs(pts[j].z - ref[j].z), max_delta_);
        }
        for (size_t j = 0; j < rb.size(); ++j) {
            max_delta_ = std::fmax(std::fabs(bx[j].px - rb[j].px), max_delta_);
            max_delta_ = std::fmax(std::fabs(bx[j].py - rb[j].py), max_delta_);
            max_delta_ = std::fmax(std::fabs(bx[j].dx - rb[j].dx), max_delta_);
            max_delta_ = std::fmax(std::fabs(bx[j].dy - rb[j].dy), max_delta_);
            max_delta_ = std::fmax(std::fabs(bx[j].ox - rb[j].ox), max_delta_);
            max_delta_ = std::fmax(std::fabs(bx[j].oy - rb[j].oy), max_delta_);
        }
        for (size_t j = 0; j < rcp.size(); ++j)
            for (int k = 0; k < 3; ++k) max_delta_ = std::fmax(std::fabs(cep[j][k] - rcp[j][k]), max_delta_);
    }
}

bool euclidean_clustering::check_output() {
    std::cout << "checking output \n";
    input_file_.close();
    output_file_.close();
    std::cout << "max delta: " << max_delta_ << "\n";
    return !(max_delta_ > kMaxEps || error_so_far_);
}

static euclidean_clustering the_kernel;
kernel &myKernel = the_kernel;
