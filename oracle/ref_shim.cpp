// Test infrastructure only: a C-ABI shim around the UNMODIFIED reference
// ndt_mapping kernel, compiled from its own source file where it lies in the
// reference tree (the path is passed in as REF_KERNEL by oracle/Makefile).
// Nothing of the reference is copied here; the file is #included at build time.
//
// Only tests, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
// arm load the resulting library (oracle/_ref/libref_ndt_*.so).  The product
// path never does.
//
// The reference keeps the members we need to reach (partial_points_callback,
// initCompute, computeDerivatives, ...) private, so access specifiers are
// widened for the reference translation unit only.  Standard headers are
// included first so the redefinition never reaches them.
#include <cstdint>
#include <cmath>
#include <cstring>
#include <chrono>
#include <fstream>
#include <iostream>
#include <limits>
#include <thread>
#include <vector>
#include <algorithm>
#include <atomic>

#define private public
#define protected public
#include REF_KERNEL
#undef private
#undef protected

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {

void load_cloud(PointCloud &c, const float *xyzi, int n) {
    c.resize(n);
    if (n) std::memcpy(c.data(), xyzi, sizeof(float) * 4 * (size_t)n);
}

void load_matrix(Matrix4f &m, const float *m16) {
    std::memcpy(&m.data[0][0], m16, sizeof(float) * 16);
}

// One reference object per host thread: the reference object is not
// re-entrant, but independent objects are (all state lives in members).
ndt_mapping &thread_instance() {
    static thread_local ndt_mapping inst;
    return inst;
}

int align_one(ndt_mapping &k, const float *scan, int n, const float *guess16,
              const float *map, int m, float *out16, int *converged) {
    if (n <= 0 || m <= 0) return -1;
    PointCloud s, t;
    load_cloud(s, scan, n);
    load_cloud(t, map, m);
    Matrix4f g;
    load_matrix(g, guess16);
    CallbackResult r = k.partial_points_callback(s, g, t);
    std::memcpy(out16, &r.final_transformation.data[0][0], sizeof(float) * 16);
    *converged = r.converged ? 1 : 0;
    return 0;
}

}  // namespace

// partial_points_callback (kernel.cpp:1405) on this thread's reference object.
REF_API int ref_align(const float *scan, int n, const float *guess16,
                      const float *map, int m, float *out16, int *converged) {
    return align_one(thread_instance(), scan, n, guess16, map, m, out16, converged);
}

// Independent alignments on `nthreads` host threads, one reference object per
// thread.  scans/maps are arrays of pointers; outs is B x 16 floats.
REF_API int ref_align_batch(int B, const float *const *scans, const int *ns,
                            const float *guesses, const float *const *maps,
                            const int *ms, float *outs, int *convs, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    std::atomic<int> next(0), err(0);
    auto worker = [&]() {
        ndt_mapping *k = new ndt_mapping();
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= B) break;
            if (align_one(*k, scans[i], ns[i], guesses + 16 * (size_t)i, maps[i], ms[i],
                          outs + 16 * (size_t)i, convs + i))
                err = -1;
        }
        delete k;
    };
    std::vector<std::thread> th;
    for (int t = 1; t < nthreads; ++t) th.emplace_back(worker);
    worker();
    for (auto &x : th) x.join();
    return err.load();
}

// initCompute (kernel.cpp:1302): dense grid of the map.  Writes bbox
// (min xyz, max xyz), dims, and for every cell: mean[3], invCov[9], count
// (13 doubles per cell) when cells != NULL and cap >= G.  Returns G.
REF_API long long ref_grid(const float *map, int m, float *bbox6, int *dims3,
                           double *cells, long long cap) {
    ndt_mapping &k = thread_instance();
    PointCloud t;
    load_cloud(t, map, m);
    k.target_ = &t;
    k.initCompute();
    for (int i = 0; i < 3; ++i) {
        bbox6[i] = k.minVoxel.data[i];
        bbox6[3 + i] = k.maxVoxel.data[i];
        dims3[i] = k.voxelDimension[i];
    }
    long long G = (long long)k.target_cells_.size();
    if (cells && cap >= G) {
        for (long long c = 0; c < G; ++c) {
            const Voxel &v = k.target_cells_[c];
            double *o = cells + 13 * c;
            for (int i = 0; i < 3; ++i) o[i] = v.mean[i];
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) o[3 + 3 * r + q] = v.invCovariance.data[r][q];
            o[12] = (double)v.numberPoints;
        }
    }
    k.target_ = nullptr;
    return G;
}

// computeDerivatives (kernel.cpp:651) for a given map, original scan, already
// transformed scan and pose vector p.  gauss_d1/d2 are inputs (the reference
// computes them in computeTransformation, kernel.cpp:1181-1185).
REF_API double ref_derivatives(const float *map, int m, const float *scan, const float *trans,
                               int n, const double *p6, double d1, double d2, int hessian,
                               double *g6, double *H36) {
    ndt_mapping &k = thread_instance();
    PointCloud t, s, tr;
    load_cloud(t, map, m);
    load_cloud(s, scan, n);
    load_cloud(tr, trans, n);
    k.target_ = &t;
    k.input_ = &s;
    k.initCompute();
    k.gauss_d1_ = d1;
    k.gauss_d2_ = d2;
    std::memset(k.point_gradient_.data, 0, sizeof(k.point_gradient_.data));
    k.point_gradient_.data[0][0] = 1.0;
    k.point_gradient_.data[1][1] = 1.0;
    k.point_gradient_.data[2][2] = 1.0;
    std::memset(k.point_hessian_.data, 0, sizeof(k.point_hessian_.data));
    Vec6 p, g;
    Mat66 H;
    for (int i = 0; i < 6; ++i) p[i] = p6[i];
    double score = k.computeDerivatives(g, H, tr, p, hessian != 0);
    for (int i = 0; i < 6; ++i) g6[i] = g[i];
    if (hessian)
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j) H36[6 * i + j] = H.data[i][j];
    k.target_ = nullptr;
    k.input_ = nullptr;
    return score;
}

// computeAngleDerivatives (kernel.cpp:707-825) at pose p6: out69 = j_ang a..h,
// then h_ang a2 a3 b2 b3 c2 c3 d1 d2 d3 e1 e2 e3 f1 f2 f3 (3 each).
REF_API void ref_angle_terms(const double *p6, double *out69) {
    ndt_mapping &k = thread_instance();
    Vec6 p;
    for (int i = 0; i < 6; ++i) p[i] = p6[i];
    k.computeAngleDerivatives(p, true);
    const double *terms[23] = {k.j_ang_a_, k.j_ang_b_, k.j_ang_c_, k.j_ang_d_, k.j_ang_e_, k.j_ang_f_,
                               k.j_ang_g_, k.j_ang_h_, k.h_ang_a2_, k.h_ang_a3_, k.h_ang_b2_, k.h_ang_b3_,
                               k.h_ang_c2_, k.h_ang_c3_, k.h_ang_d1_, k.h_ang_d2_, k.h_ang_d3_, k.h_ang_e1_,
                               k.h_ang_e2_, k.h_ang_e3_, k.h_ang_f1_, k.h_ang_f2_, k.h_ang_f3_};
    for (int t = 0; t < 23; ++t)
        for (int c = 0; c < 3; ++c) out69[3 * t + c] = terms[t][c];
}

// One pair through the reference's own routines: computeAngleDerivatives(p)
// (kernel.cpp:707), computePointDerivatives(x) (:495) and updateDerivatives
// (:438) with the scan point x, its offset from the cell mean xt and the
// cell's inverse covariance C (row major).  g6 / H36 are accumulated in
// place; returns the score increment (0 when the pair is rejected).
REF_API double ref_update_pair(const double *p6, const double *x3, const double *xt3, const double *C9, double d1,
                               double d2, int hessian, double *g6, double *H36) {
    ndt_mapping &k = thread_instance();
    k.gauss_d1_ = d1;
    k.gauss_d2_ = d2;
    std::memset(k.point_gradient_.data, 0, sizeof(k.point_gradient_.data));
    k.point_gradient_.data[0][0] = 1.0;
    k.point_gradient_.data[1][1] = 1.0;
    k.point_gradient_.data[2][2] = 1.0;
    std::memset(k.point_hessian_.data, 0, sizeof(k.point_hessian_.data));
    Vec6 p, g;
    Vec3 x, xt;
    Mat33 C;
    Mat66 H;
    for (int i = 0; i < 6; ++i) p[i] = p6[i], g[i] = g6[i];
    for (int i = 0; i < 3; ++i) x[i] = x3[i], xt[i] = xt3[i];
    for (int i = 0; i < 9; ++i) C.data[i / 3][i % 3] = C9[i];
    for (int i = 0; i < 36; ++i) H.data[i / 6][i % 6] = H36[i];
    k.computeAngleDerivatives(p, hessian != 0);
    k.computePointDerivatives(x, hessian != 0);
    const double inc = k.updateDerivatives(g, H, xt, C, hessian != 0);
    for (int i = 0; i < 6; ++i) g6[i] = g[i];
    for (int i = 0; i < 36; ++i) H36[i] = H.data[i / 6][i % 6];
    return inc;
}

// voxelRadiusSearch (kernel.cpp:246) on the grid of `map`: number of
// neighbour voxels of point xyz; their means go to means3 (up to cap).
REF_API int ref_radius_search(const float *map, int m, const float *pt4, double *means3, int cap) {
    ndt_mapping &k = thread_instance();
    PointCloud t;
    load_cloud(t, map, m);
    k.target_ = &t;
    k.initCompute();
    PointXYZI p;
    std::memcpy(p.data, pt4, sizeof(float) * 4);
    std::vector<Voxel> nb;
    std::vector<float> dist;
    int r = k.voxelRadiusSearch(k.target_cells_, p, k.resolution_, nb, dist);
    for (int i = 0; i < r && i < cap; ++i)
        for (int c = 0; c < 3; ++c) means3[3 * i + c] = nb[i].mean[c];
    k.target_ = nullptr;
    return r;
}

// buildTransformationMatrix (kernel.cpp:949): writes into m16 in place
// (cells the reference does not touch keep their input values).
REF_API void ref_build_tm(const double *p6, float *m16) {
    ndt_mapping &k = thread_instance();
    Matrix4f m;
    load_matrix(m, m16);
    Vec6 p;
    for (int i = 0; i < 6; ++i) p[i] = p6[i];
    k.buildTransformationMatrix(m, p);
    std::memcpy(m16, &m.data[0][0], sizeof(float) * 16);
}

// eulerAngles (kernel.cpp:1146).
REF_API void ref_euler(const float *m16, double *out3) {
    ndt_mapping &k = thread_instance();
    Matrix4f m;
    load_matrix(m, m16);
    Vec3 r;
    k.eulerAngles(m, r);
    for (int i = 0; i < 3; ++i) out3[i] = r[i];
}

// solve (kernel.cpp:293).
REF_API void ref_solve(const double *A36, const double *b6, double *x6) {
    Mat66 A;
    Vec6 b, x;
    for (int i = 0; i < 6; ++i) {
        b[i] = b6[i];
        for (int j = 0; j < 6; ++j) A.data[i][j] = A36[6 * i + j];
    }
    solve(x, A, b);
    for (int i = 0; i < 6; ++i) x6[i] = x[i];
}

// invertMatrix (kernel.cpp:1277), in place on a row-major 3x3.
REF_API void ref_invert(double *m9) {
    Mat33 m;
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m.data[r][c] = m9[3 * r + c];
    invertMatrix(m);
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) m9[3 * r + c] = m.data[r][c];
}

// transformPointCloud (kernel.cpp:385).
REF_API void ref_transform(const float *in, int n, const float *m16, float *out) {
    PointCloud a, b;
    load_cloud(a, in, n);
    Matrix4f m;
    load_matrix(m, m16);
    transformPointCloud(a, b, m);
    for (int i = 0; i < n; ++i) std::memcpy(out + 4 * (size_t)i, b[i].data, sizeof(float) * 4);
}

// trialValueSelectionMT (kernel.cpp:867).
REF_API double ref_trial_value(double a_l, double f_l, double g_l, double a_u, double f_u,
                               double g_u, double a_t, double f_t, double g_t) {
    return thread_instance().trialValueSelectionMT(a_l, f_l, g_l, a_u, f_u, g_u, a_t, f_t, g_t);
}

// updateIntervalMT (kernel.cpp:827); io6 = {a_l, f_l, g_l, a_u, f_u, g_u} in/out.
REF_API int ref_update_interval(double *io6, double a_t, double f_t, double g_t) {
    return thread_instance().updateIntervalMT(io6[0], io6[1], io6[2], io6[3], io6[4], io6[5],
                                              a_t, f_t, g_t)
               ? 1
               : 0;
}
