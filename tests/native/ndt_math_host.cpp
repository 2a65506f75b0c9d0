// Host build of daphne-benchmark_b200/csrc/ndt_math.cuh (the device-side
// angle terms, pose build, pose vector, 6x6 solve and More-Thuente helpers) behind a C ABI,
// for tests/test_ndt_math_host.py to compare with the reference's own routines
// (oracle/_ref) on many random inputs.  Compiled with g++ -ffp-contract=off,
// like the library's --fmad=false build: every product and sum rounds on its
// own; cos / sin / atan2 / sqrt are the host's, as in the reference's build.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "ndt_math.cuh"

#define API extern "C" __attribute__((visibility("default")))

API void ndtm_angle_terms(const double *p6, int compat, double *out69) { ndt::angle_terms(p6, out69, compat != 0); }

API void ndtm_build_tm_compat(const double *t6, float *m16) { ndt::build_tm_compat(m16, t6); }

API void ndtm_build_tm_corrected(const double *p6, float *m16) { ndt::build_tm_corrected(m16, p6); }

API void ndtm_pose_vector(int compat, const float *m16, double *p6) { ndt::pose_vector(compat != 0, m16, p6); }

API void ndtm_solve6(const double *A36, const double *b6, double *x6) {
    double A[6][6], b[6];
    std::memcpy(A, A36, sizeof(A));
    std::memcpy(b, b6, sizeof(b));
    ndt::solve6(x6, A, b);
}

API double ndtm_trial_value(double a_l, double f_l, double g_l, double a_u, double f_u, double g_u, double a_t,
                            double f_t, double g_t) {
    return ndt::trial_value(a_l, f_l, g_l, a_u, f_u, g_u, a_t, f_t, g_t);
}

API int ndtm_update_interval(double *io6, double a_t, double f_t, double g_t) {
    return ndt::update_interval(io6[0], io6[1], io6[2], io6[3], io6[4], io6[5], a_t, f_t, g_t) ? 1 : 0;
}
