// Host-side check of the exact parts of daphne-benchmark_b200/csrc/probe.cuh
// (compiled with g++ as host code and run by tests/test_probe_host.py; no GPU):
//  * make_axis: the probe coordinates, trip count, in-box flags and cells of
//    one axis, against the reference's float probe loop (voxelRadiusSearch,
//    src/CPU/ndt_mapping/kernel.cpp:246-286, as oracle/ndt_oracle.cpp restates
//    it: x = p - r; x <= p + r_final; x += r, each skipped outside the box);
//  * accept: the radius test with its FP32 pre-test margin, against the
//    reference's float(sqrt(dx^2 + dy^2 + dz^2)) < r with dx = float(mean - p),
//    on pairs placed within a few ulps of the radius, at coordinates up to 1e5 m;
//  * window_base: when it accepts a lane, the window's cells are the probe cells.
// Prints the number of disagreements per part; exit status 1 if any.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <random>

// host versions of the device intrinsics (round to nearest, no contraction: -ffp-contract=off)
inline float __fadd_rn(float a, float b) { return a + b; }
inline float __fsub_rn(float a, float b) { return a - b; }
inline float __fmul_rn(float a, float b) { return a * b; }
inline float __fdiv_rn(float a, float b) { return a / b; }
template <class T>
inline T __ldg(const T *p) { return *p; }
// warp intrinsics: declared for the warp-cooperative parts of the header, which this check does not call
unsigned __ballot_sync(unsigned, int);
int __any_sync(unsigned, int);
int __all_sync(unsigned, int);
unsigned __reduce_max_sync(unsigned, unsigned);
int __popc(unsigned);
unsigned __float_as_uint(float);
extern uint3 threadIdx;

#include "probe.cuh"

namespace {

// the reference's float probe loop for one axis: coordinates, and for each whether it is inside [lo, hi]
int reference_axis(float p, float lo, float hi, float res, float rf, float *c, bool *in) {
    int n = 0;
    for (float x = p - res; x <= p + rf && n < 4; x += res, ++n) {
        c[n] = x;
        in[n] = !(x < lo || x > hi);
    }
    return n;
}

// largest float s whose correctly rounded square root is below r
float threshold(float r) {
    float s = r * r;
    while (std::sqrt(s) >= r) s = std::nextafter(s, 0.0f);
    while (std::sqrt(std::nextafter(s, INFINITY)) < r) s = std::nextafter(s, INFINITY);
    return s;
}

bool reference_accept(const double *m, float px, float py, float pz, float r) {
    const float dx = (float)(m[0] - px), dy = (float)(m[1] - py), dz = (float)(m[2] - pz);
    const float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
    return (double)dist < (double)r;
}

}  // namespace

int main() {
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const float resolutions[] = {1.0f, 0.5f, 2.0f, 0.3f};
    long bad_axis = 0, bad_accept = 0, bad_window = 0, axes = 0, pairs = 0, near = 0;
    for (float res : resolutions) {
        int e2;
        const float inv = std::frexp(res, &e2) == 0.5f ? 1.0f / res : 0.0f;  // power of two: exact reciprocal
        const float rf = (float)((double)res + (double)0.001f);
        // axis checks: a box [lo, hi] and points spread over it and beyond, many right at its edges and
        // on cell boundaries
        for (int t = 0; t < 200000; ++t) {
            const float lo = (float)(U(rng) * 2000.0 - 1000.0);
            const int dim = 1 + (int)(U(rng) * 200);
            const float hi = lo + (float)dim * res - 0.02f;
            float p;
            const int kind = t % 4;
            if (kind == 0) p = (float)(lo + (hi - lo) * (U(rng) * 1.4 - 0.2));
            else if (kind == 1) p = std::nextafter(lo + res * (float)(int)(U(rng) * dim), U(rng) < 0.5 ? -INFINITY : INFINITY);
            else if (kind == 2) p = (U(rng) < 0.5 ? lo : hi) + (float)((U(rng) - 0.5) * 2.5 * res);
            else p = lo + res * (float)(int)(U(rng) * dim) + (float)((U(rng) - 0.5) * 1e-4);
            float c[4];
            bool in[4];
            const int n = reference_axis(p, lo, hi, res, rf, c, in);
            const ndt::Axis a = ndt::make_axis(p, lo, hi, res, inv, rf, true);
            bool ok = a.n == n;
            const float ac[3] = {a.c0, a.c1, a.c2};
            for (int k = 0; k < 3 && ok; ++k) {
                const bool rin = k < n && in[k];
                ok = ((a.in >> k) & 1u) == (unsigned)rin;
                if (ok && rin) ok = ac[k] == c[k] && ndt::axis_i(a, k) == (int)((c[k] - lo) / res);
            }
            bad_axis += !ok;
            ++axes;
            // window decision: accepted only when the in-box cells are consecutive from the base and inside dim
            bool wok = true;
            const int base = ndt::window_base(a, dim, wok);
            if (wok)
                for (int k = 0; k < 3; ++k)
                    if (k < n && in[k] && (int)((c[k] - lo) / res) != base + k) ++bad_window;
        }
        // radius test on pairs near the sphere of radius res
        ndt::GridDev g = {};
        g.s_max = threshold(res);
        double4 mean[1];
        g.mean = mean;
        for (int t = 0; t < 1000000; ++t) {
            const double scale = t % 3 == 0 ? 1e5 : (t % 3 == 1 ? 1e3 : 50.0);
            const float px = (float)((U(rng) - 0.5) * 2 * scale), py = (float)((U(rng) - 0.5) * 2 * scale),
                        pz = (float)((U(rng) - 0.5) * 20);
            double ux = U(rng) - 0.5, uy = U(rng) - 0.5, uz = U(rng) - 0.5;
            const double un = std::sqrt(ux * ux + uy * uy + uz * uz);
            const double d = (double)res * (1.0 + (U(rng) - 0.5) * 4e-6 * (t % 7 == 0 ? 100.0 : 1.0));
            const double m[3] = {px + d * ux / un, py + d * uy / un, pz + d * uz / un};
            mean[0] = make_double4(m[0], m[1], m[2], 0.0);
            const float4 hi = make_float4((float)m[0], (float)m[1], (float)m[2], 0.0f);
            const float tol = ndt::radius_margin(px, py, pz, res);
            const bool ours = ndt::accept(g, 0, hi, px, py, pz, tol);
            const bool ref = reference_accept(m, px, py, pz, res);
            bad_accept += ours != ref;
            ++pairs;
            near += ref != reference_accept(m, px, py, pz, std::nextafter(res, 0.0f));
        }
    }
    std::printf("axes %ld bad %ld; window disagreements %ld; pairs %ld (%ld within one ulp of the radius) bad %ld\n",
                axes, bad_axis, bad_window, pairs, near, bad_accept);
    return (bad_axis || bad_accept || bad_window) ? 1 : 0;
}
