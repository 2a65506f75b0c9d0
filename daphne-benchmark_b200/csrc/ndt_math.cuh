// Device-side NDT math: pose build, pose vector, angle derivatives, 6x6
// solve and More-Thuente helpers.
//
// The library is compiled with --fmad=false, so every expression here rounds
// each product and sum on its own, as the reference's x86-64 SSE2 code does
// (src/CPU/ndt_mapping/kernel.cpp); the operation order of each expression is
// the reference's where the corrected mode does not change the formula.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "ndt_types.h"

namespace ndt {

// std::min / std::max semantics (NaN in the first argument propagates), as the
// reference's line search uses them (kernel.cpp:932-934, 1055-1056).
__device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }

// Angle derivative terms, eq. 6.19 / 6.21 (computeAngleDerivatives,
// kernel.cpp:707-825).  out[0..23] = j_ang a..h (3 each), out[24..68] =
// h_ang a2 a3 b2 b3 c2 c3 d1 d2 d3 e1 e2 e3 f1 f2 f3 (3 each).  One term
// differs by mode: the second derivative of the rotated x component in pitch,
// d^2/db^2 (cy cz, -cy sz, sy) = (-cy cz, cy sz, -sy), has +sy in the
// reference's h_ang_d1 (kernel.cpp:795-797); compat keeps it, the corrected
// mode uses -sy.
__device__ inline void angle_terms(const double *p, double *o, bool compat) {
    double cx, cy, cz, sx, sy, sz;
    if (fabs(p[3]) < 10e-5) { cx = 1.0; sx = 0.0; } else { cx = cos(p[3]); sx = sin(p[3]); }
    if (fabs(p[4]) < 10e-5) { cy = 1.0; sy = 0.0; } else { cy = cos(p[4]); sy = sin(p[4]); }
    if (fabs(p[5]) < 10e-5) { cz = 1.0; sz = 0.0; } else { cz = cos(p[5]); sz = sin(p[5]); }
    // j_ang a .. h
    o[0] = (-sx * sz + cx * sy * cz);  o[1] = (-sx * cz - cx * sy * sz);  o[2] = (-cx * cy);
    o[3] = (cx * sz + sx * sy * cz);   o[4] = (cx * cz - sx * sy * sz);   o[5] = (-sx * cy);
    o[6] = (-sy * cz);                 o[7] = sy * sz;                    o[8] = cy;
    o[9] = sx * cy * cz;               o[10] = (-sx * cy * sz);           o[11] = sx * sy;
    o[12] = (-cx * cy * cz);           o[13] = cx * cy * sz;              o[14] = (-cx * sy);
    o[15] = (-cy * sz);                o[16] = (-cy * cz);                o[17] = 0;
    o[18] = (cx * cz - sx * sy * sz);  o[19] = (-cx * sz - sx * sy * cz); o[20] = 0;
    o[21] = (sx * cz + cx * sy * sz);  o[22] = (cx * sy * cz - sx * sz);  o[23] = 0;
    // h_ang a2 a3 b2 b3 c2 c3 d1 d2 d3 e1 e2 e3 f1 f2 f3
    double *h = o + 24;
    h[0] = (-cx * sz - sx * sy * cz);  h[1] = (-cx * cz + sx * sy * sz);  h[2] = sx * cy;
    h[3] = (-sx * sz + cx * sy * cz);  h[4] = (-cx * sy * sz - sx * cz);  h[5] = (-cx * cy);
    h[6] = (cx * cy * cz);             h[7] = (-cx * cy * sz);            h[8] = (cx * sy);
    h[9] = (sx * cy * cz);             h[10] = (-sx * cy * sz);           h[11] = (sx * sy);
    h[12] = (-sx * cz - cx * sy * sz); h[13] = (sx * sz - cx * sy * cz);  h[14] = 0;
    h[15] = (cx * cz - sx * sy * sz);  h[16] = (-sx * sy * cz - cx * sz); h[17] = 0;
    h[18] = (-cy * cz);                h[19] = (cy * sz);                 h[20] = compat ? sy : -sy;
    h[21] = (-sx * sy * cz);           h[22] = (sx * sy * sz);            h[23] = (sx * cy);
    h[24] = (cx * sy * cz);            h[25] = (-cx * sy * sz);           h[26] = (-cx * cy);
    h[27] = (sy * sz);                 h[28] = (sy * cz);                 h[29] = 0;
    h[30] = (-sx * cy * sz);           h[31] = (-sx * cy * cz);           h[32] = 0;
    h[33] = (cx * cy * sz);            h[34] = (cx * cy * cz);            h[35] = 0;
    h[36] = (-cy * cz);                h[37] = (cy * sz);                 h[38] = 0;
    h[39] = (-cx * sz - sx * sy * cz); h[40] = (-cx * cz + sx * sy * sz); h[41] = 0;
    h[42] = (-sx * sz + cx * sy * cz); h[43] = (-cx * sy * sz - sx * cz); h[44] = 0;
}

// Reference pose build (buildTransformationMatrix, kernel.cpp:949-1013):
// float quaternion products with permuted components; writes the rotation
// block and row 3 only, the translation column keeps its value.
__device__ inline void build_tm_compat(float *M, const double *t) {
    const float q_ha = 0.5f * t[3];
    const float q_w = cos((double)q_ha);
    const float q_x = sin((double)q_ha);
    const float q_y = 0.0f, q_z = 0.0f;
    const float q_ha2 = 0.5f * t[4];
    const float q_w2 = cos((double)q_ha2);
    const float q_x2 = 0.0f;
    const float q_y2 = sin((double)q_ha2);
    const float q_z2 = 0.0f;
    const float q_ha3 = 0.5f * t[5];
    const float q_w3 = cos((double)q_ha3);
    const float q_x3 = 0.0f, q_y3 = 0.0f;
    const float q_z3 = sin((double)q_ha3);
    const float r_x = q_w * q_w2 - q_x * q_x2 - q_y * q_y2 - q_z * q_z2;
    const float r_y = q_w * q_x2 + q_x * q_w2 + q_y * q_z2 - q_z * q_y2;
    const float r_z = q_w * q_y2 + q_y * q_w2 + q_z * q_x2 - q_x * q_z2;
    const float r_w = q_w * q_z2 + q_z * q_w2 + q_x * q_y2 - q_y * q_x2;
    const float r2_x = r_w * q_w3 - r_x * q_x3 - r_y * q_y3 - r_z * q_z3;
    const float r2_y = r_w * q_x3 + r_x * q_w3 + r_y * q_z3 - r_z * q_y3;
    const float r2_z = r_w * q_y3 + r_y * q_w3 + r_z * q_x3 - r_x * q_z3;
    const float r2_w = r_w * q_z3 + r_z * q_w3 + r_x * q_y3 - r_y * q_x3;
    const float tx = 2.0f * r2_x, ty = 2.0f * r2_y, tz = 2.0f * r2_z;
    const float twx = tx * r2_w, twy = ty * r2_w, twz = tz * r2_w;
    const float txx = tx * r2_x, txy = ty * r2_x, txz = tz * r2_x;
    const float tyy = ty * r2_y, tyz = tz * r2_y, tzz = tz * r2_z;
    M[12] = 0.0f; M[13] = 0.0f; M[14] = 0.0f; M[15] = 1.0f;
    M[0] = 1.0f - (tyy + tzz);
    M[1] = txy - twz;
    M[2] = txz + twy;
    M[4] = txy + twz;
    M[5] = 1.0f - (txx + tzz);
    M[6] = tyz - twx;
    M[8] = txz - twy;
    M[9] = tyz + twx;
    M[10] = 1.0f - (txx + tyy);
}

// Rotation R = Rx(a) Ry(b) Rz(c) (the parametrisation eq. 6.19 / 6.21
// differentiate), row major.
__device__ inline void rot_xyz(const double *p, double *R) {
    double ca = cos(p[3]), sa = sin(p[3]);
    double cb = cos(p[4]), sb = sin(p[4]);
    double cc = cos(p[5]), sc = sin(p[5]);
    R[0] = cb * cc;                R[1] = -cb * sc;               R[2] = sb;
    R[3] = ca * sc + sa * sb * cc; R[4] = ca * cc - sa * sb * sc; R[5] = -sa * cb;
    R[6] = sa * sc - ca * sb * cc; R[7] = sa * cc + ca * sb * sc; R[8] = ca * cb;
}

// Corrected pose build: T = Trans(p0..2) * Rx * Ry * Rz, FP64 then rounded.
__device__ inline void build_tm_corrected(float *M, const double *p) {
    double R[9];
    rot_xyz(p, R);
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) M[4 * r + c] = (float)R[3 * r + c];
        M[4 * r + 3] = (float)p[r];
    }
    M[12] = 0.0f; M[13] = 0.0f; M[14] = 0.0f; M[15] = 1.0f;
}

// Pose vector of a 4x4: translation column + angles.  compat: the reference's
// negated Euler extraction (eulerAngles, kernel.cpp:1146-1173); corrected:
// the exact inverse of rot_xyz.
__device__ inline void pose_vector(bool compat, const float *M, double *p) {
    p[0] = M[3];
    p[1] = M[7];
    p[2] = M[11];
    if (compat) {
        const double kPi = 3.1415926535897932384626433832795;
        double r0 = atan2((double)M[6], (double)M[10]), r1;
        double n1 = M[0], n2 = M[1];
        double c2 = sqrt(n1 * n1 + n2 * n2);
        if (r0 > 0.0) {
            r0 -= kPi;
            r1 = atan2((double)-M[2], -c2);
        } else {
            r1 = atan2((double)-M[2], c2);
        }
        double s1 = sin(r0), c1 = cos(r0);
        double r2 = atan2(s1 * M[8] - c1 * M[4], c1 * M[5] - s1 * M[9]);
        p[3] = -r0;
        p[4] = -r1;
        p[5] = -r2;
    } else {
        double r12 = M[6], r22 = M[10], r02 = M[2], r00 = M[0], r01 = M[1];
        p[3] = atan2(-r12, r22);
        p[4] = atan2(r02, sqrt(r00 * r00 + r01 * r01));
        p[5] = atan2(-r01, r00);
    }
}

// 6x6 Gaussian elimination with partial pivoting; a zero pivot column is
// replaced by 0.001 (solve, kernel.cpp:293-343).  A and b are clobbered.
__device__ inline void solve6(double *x, double (*A)[6], double *b) {
    for (int j = 0; j < 6; ++j) {
        double mx = fabs(A[j][j]);
        int mi = j;
        for (int i = j + 1; i < 6; ++i)
            if (fabs(A[i][j]) > mx) {
                mi = i;
                mx = fabs(A[i][j]);
            }
        if (mi != j)
            for (int i = 0; i < 6; ++i) {
                double t = A[mi][i];
                A[mi][i] = A[j][i];
                A[j][i] = t;
            }
        if (mx == 0.0) A[j][j] = 0.001;
        for (int i = j + 1; i < 6; ++i) {
            double piv = A[i][j] / A[j][j];
            for (int k = 0; k < 6; ++k) A[i][k] = A[i][k] - piv * A[j][k];
            b[i] = b[i] - piv * b[j];
        }
    }
    x[5] = b[5] / A[5][5];
    for (int i = 4; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1; j < 6; ++j) sum = sum + A[i][j] * x[j];
        x[i] = (b[i] - sum) / A[i][i];
    }
}

// More-Thuente auxiliary functions and interval updates
// (kernel.cpp:425-436, 827-946; More & Thuente 1994, Sun & Yuan 2006).
__device__ __forceinline__ double psi_mt(double a, double f_a, double f_0, double g_0, double mu) {
    return (f_a - f_0 - mu * g_0 * a);
}
__device__ __forceinline__ double dpsi_mt(double g_a, double g_0, double mu) { return (g_a - mu * g_0); }

__device__ inline bool update_interval(double &a_l, double &f_l, double &g_l, double &a_u, double &f_u,
                                       double &g_u, double a_t, double f_t, double g_t) {
    if (f_t > f_l) {
        a_u = a_t; f_u = f_t; g_u = g_t;
        return false;
    } else if (g_t * (a_l - a_t) > 0) {
        a_l = a_t; f_l = f_t; g_l = g_t;
        return false;
    } else if (g_t * (a_l - a_t) < 0) {
        a_u = a_l; f_u = f_l; g_u = g_l;
        a_l = a_t; f_l = f_t; g_l = g_t;
        return false;
    }
    return true;
}

__device__ inline double trial_value(double a_l, double f_l, double g_l, double a_u, double f_u, double g_u,
                                     double a_t, double f_t, double g_t) {
    if (f_t > f_l) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_q = a_l - 0.5 * (a_l - a_t) * g_l / (g_l - (f_l - f_t) / (a_l - a_t));
        if (fabs(a_c - a_l) < fabs(a_q - a_l)) return a_c;
        return 0.5 * (a_q + a_c);
    } else if (g_t * g_l < 0) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_s = a_l - (a_l - a_t) / (g_l - g_t) * g_l;
        if (fabs(a_c - a_t) >= fabs(a_s - a_t)) return a_c;
        return a_s;
    } else if (fabs(g_t) <= fabs(g_l)) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_s = a_l - (a_l - a_t) / (g_l - g_t) * g_l;
        double a_t_next = (fabs(a_c - a_t) < fabs(a_s - a_t)) ? a_c : a_s;
        if (a_t > a_l) return std_min(a_t + 0.66 * (a_u - a_t), a_t_next);
        return std_max(a_t + 0.66 * (a_u - a_t), a_t_next);
    }
    double z = 3 * (f_t - f_u) / (a_t - a_u) - g_t - g_u;
    double w = sqrt(z * z - g_t * g_u);
    return (a_u + (a_t - a_u) * (w - g_u - z) / (g_t - g_u + 2 * w));
}

}  // namespace ndt
