// CPU oracle for the NDT align path -- TEST INFRASTRUCTURE ONLY (see ndt_oracle.h).
//
// Mode R (compat = 1) restates src/CPU/ndt_mapping/kernel.cpp function by
// function; each routine cites the lines it follows.  Floating-point
// expressions keep the reference's operation order and types (float where the
// reference computes in float, double where it computes in double), and the
// library is compiled with -ffp-contract=off, so results agree bit for bit
// with the compiled reference on x86-64.
//
// Mode F (compat = 0) is the corrected NDT in FP64 (see ndt_b200.h).
#include "ndt_oracle.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr double kPi = 3.1415926535897932384626433832795;  // datatypes.h:73

// ---------------------------------------------------------------------------
// Voxel grid.  Mode R keeps every dense cell (kernel.cpp:1324-1338); Mode F
// keeps the same dense addressing but marks cells below min_points invalid.
struct Grid {
    float res = 1.0f;
    float minv[3] = {0, 0, 0}, maxv[3] = {0, 0, 0};
    int dim[3] = {0, 0, 0};
    long long G = 0;
    std::vector<double> mean;   // 3 per cell
    std::vector<double> icov;   // 9 per cell, row major
    std::vector<int> count;     // per cell
    std::vector<unsigned char> valid;  // Mode F: usable cell
};

// linearizeAddr / linearizeCoord (kernel.cpp:231-244): float subtraction and
// division, truncation to int, int linearisation.
inline int cell_of(const Grid &g, float x, float y, float z) {
    int ix = (int)((x - g.minv[0]) / g.res);
    int iy = (int)((y - g.minv[1]) / g.res);
    int iz = (int)((z - g.minv[2]) / g.res);
    return ix + g.dim[0] * (iy + g.dim[1] * iz);
}

// Bounding box and dims (kernel.cpp:1305-1322).
bool grid_bbox(Grid &g, const float *map, int m, float res) {
    g.res = res;
    for (int e = 0; e < 3; ++e) g.minv[e] = g.maxv[e] = map[e];
    for (int i = 1; i < m; ++i)
        for (int e = 0; e < 3; ++e) {
            float v = map[4 * (size_t)i + e];
            if (v > g.maxv[e]) g.maxv[e] = v;
            if (v < g.minv[e]) g.minv[e] = v;
        }
    for (int e = 0; e < 3; ++e) {
        g.minv[e] -= 0.01f;
        g.maxv[e] += 0.01f;
        g.dim[e] = (int)((g.maxv[e] - g.minv[e]) / res + 1);
    }
    long long G = (long long)g.dim[0] * g.dim[1] * g.dim[2];
    if (G <= 0 || G > INT_MAX) return false;
    g.G = G;
    return true;
}

// invertMatrix (kernel.cpp:1277-1300): adjugate over the determinant.
void invert3(double *m) {
    double det = m[0] * (m[8] * m[4] - m[7] * m[5]) - m[3] * (m[8] * m[1] - m[7] * m[2]) +
                 m[6] * (m[5] * m[1] - m[4] * m[2]);
    double inv_det = 1.0 / det;
    double t[9];
    t[0] = m[8] * m[4] - m[7] * m[5];
    t[1] = -(m[8] * m[1] - m[7] * m[2]);
    t[2] = m[5] * m[1] - m[4] * m[2];
    t[3] = -(m[8] * m[1] - m[6] * m[5]);
    t[4] = m[8] * m[0] - m[7] * m[2];
    t[5] = -(m[5] * m[0] - m[3] * m[2]);
    t[6] = m[7] * m[3] - m[6] * m[4];
    t[7] = -(m[7] * m[0] - m[6] * m[1]);
    t[8] = m[4] * m[0] - m[3] * m[1];
    for (int i = 0; i < 9; ++i) m[i] = t[i] * inv_det;
}

// Mode R grid (kernel.cpp:1324-1372): single-pass sums into cells whose
// inverse-covariance slot starts as the anti-diagonal identity, then the
// covariance scaled by the dense cell count G, then the adjugate inverse.
bool build_grid_r(Grid &g, const float *map, int m, float res) {
    if (!grid_bbox(g, map, m, res)) return false;
    const long long G = g.G;
    g.mean.assign(3 * G, 0.0);
    g.icov.assign(9 * G, 0.0);
    g.count.assign(G, 0);
    for (long long c = 0; c < G; ++c) {
        g.icov[9 * c + 6] = 1.0;  // [2][0]
        g.icov[9 * c + 4] = 1.0;  // [1][1]
        g.icov[9 * c + 2] = 1.0;  // [0][2]
    }
    for (int i = 0; i < m; ++i) {
        const float *p = map + 4 * (size_t)i;
        int c = cell_of(g, p[0], p[1], p[2]);
        double *mu = &g.mean[3 * (size_t)c];
        mu[0] += p[0];
        mu[1] += p[1];
        mu[2] += p[2];
        g.count[c]++;
        double *S = &g.icov[9 * (size_t)c];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) S[3 * r + q] += p[r] * p[q];  // float product
    }
    const double Gd = (double)(size_t)G;
    for (long long c = 0; c < G; ++c) {
        double *mu = &g.mean[3 * c];
        double *S = &g.icov[9 * c];
        double ps[3] = {mu[0], mu[1], mu[2]};
        int n = g.count[c];
        mu[0] /= n;
        mu[1] /= n;
        mu[2] /= n;
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
                S[3 * r + q] = (S[3 * r + q] - 2 * (ps[r] * mu[q])) / Gd + mu[r] * mu[q];
                S[3 * r + q] *= (Gd - 1.0) / n;
            }
        invert3(S);
    }
    return true;
}

// Symmetric 3x3 eigen-decomposition by cyclic Jacobi rotations.  A is
// overwritten; V receives eigenvectors as columns; w the eigenvalues.
void jacobi3(double A[3][3], double V[3][3], double w[3]) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 16; ++sweep) {
        double off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        double diag = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (off <= 1e-30 * diag || off == 0.0) break;
        for (int p = 0; p < 2; ++p)
            for (int q = p + 1; q < 3; ++q) {
                double apq = A[p][q];
                if (apq == 0.0) continue;
                double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 3; ++k) {  // A <- A J (columns p, q)
                    double akp = A[k][p], akq = A[k][q];
                    A[k][p] = c * akp - s * akq;
                    A[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < 3; ++k) {  // A <- J^T A (rows p, q)
                    double apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c * apk - s * aqk;
                    A[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < 3; ++k) {
                    double vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c * vkp - s * vkq;
                    V[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < 3; ++i) w[i] = A[i][i];
}

// Mode F grid: per-voxel mean, centred covariance / (N-1), cells with fewer
// than min_points points unusable, eigenvalues floored at eigen_ratio * max.
bool build_grid_f(Grid &g, const float *map, int m, float res, int min_points, double eig_ratio) {
    if (!grid_bbox(g, map, m, res)) return false;
    const long long G = g.G;
    g.mean.assign(3 * G, 0.0);
    g.icov.assign(9 * G, 0.0);
    g.count.assign(G, 0);
    g.valid.assign(G, 0);
    std::vector<int> cell(m);
    const double nan = std::nan("");
    for (int i = 0; i < m; ++i) {
        const float *p = map + 4 * (size_t)i;
        int c = cell_of(g, p[0], p[1], p[2]);
        cell[i] = c;
        g.count[c]++;
        for (int e = 0; e < 3; ++e) g.mean[3 * (size_t)c + e] += (double)p[e];
    }
    for (long long c = 0; c < G; ++c)
        if (g.count[c] > 0)
            for (int e = 0; e < 3; ++e) g.mean[3 * c + e] /= g.count[c];
    std::vector<double> M2(6 * G, 0.0);  // xx xy xz yy yz zz
    for (int i = 0; i < m; ++i) {
        const float *p = map + 4 * (size_t)i;
        int c = cell[i];
        double d0 = p[0] - g.mean[3 * (size_t)c], d1 = p[1] - g.mean[3 * (size_t)c + 1],
               d2 = p[2] - g.mean[3 * (size_t)c + 2];
        double *s = &M2[6 * (size_t)c];
        s[0] += d0 * d0; s[1] += d0 * d1; s[2] += d0 * d2;
        s[3] += d1 * d1; s[4] += d1 * d2; s[5] += d2 * d2;
    }
    for (long long c = 0; c < G; ++c) {
        int n = g.count[c];
        if (n < min_points || n < 2) continue;
        const double *s = &M2[6 * c];
        double A[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) A[r][q] /= (n - 1);
        double V[3][3], w[3];
        jacobi3(A, V, w);
        double wmax = std::max(w[0], std::max(w[1], w[2]));
        if (!(wmax > 0.0) || !std::isfinite(wmax)) continue;
        double floor_v = eig_ratio * wmax;
        double inv_w[3];
        bool ok = true;
        for (int e = 0; e < 3; ++e) {
            double we = w[e] < floor_v ? floor_v : w[e];
            if (!(we > 0.0)) ok = false;
            inv_w[e] = 1.0 / we;
        }
        if (!ok) continue;
        double *C = &g.icov[9 * c];
        for (int e = 0; e < 9; ++e) C[e] = 0.0;
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q)
                C[3 * r + q] = V[r][0] * inv_w[0] * V[q][0] + V[r][1] * inv_w[1] * V[q][1] +
                               V[r][2] * inv_w[2] * V[q][2];
        g.valid[c] = 1;
    }
    // unusable cells: NaN mean, so the radius test never accepts them
    for (long long c = 0; c < G; ++c)
        if (!g.valid[c])
            for (int e = 0; e < 3; ++e) g.mean[3 * c + e] = nan;
    return true;
}

// ---------------------------------------------------------------------------
// Neighbour search.
// Mode R: voxelRadiusSearch (kernel.cpp:246-286) -- 27 float probe points
// p + {-r, 0, r}^3 (z outer, x inner), each skipped outside the bbox, mapped
// to its cell, kept when the float distance to the cell mean is < r.
int radius_search_r(const Grid &g, const float *pt, double radius, int *out) {
    int k = 0;
    float radius_final = radius + 0.001f;
    const float res = g.res;
    // Each float loop runs 3 times for any finite coordinate below ~1e6 m;
    // the cap of 4 only stops the endless loop the reference enters for
    // infinite or huge coordinates (where z + res == z).
    int iz = 0;
    for (float z = pt[2] - radius; z <= pt[2] + radius_final && iz < 4; z += res, ++iz) {
        int iy = 0;
        for (float y = pt[1] - radius; y <= pt[1] + radius_final && iy < 4; y += res, ++iy) {
            int ix = 0;
            for (float x = pt[0] - radius; x <= pt[0] + radius_final && ix < 4; x += res, ++ix) {
                if ((x < g.minv[0]) || (x > g.maxv[0]) || (y < g.minv[1]) || (y > g.maxv[1]) ||
                    (z < g.minv[2]) || (z > g.maxv[2]))
                    continue;
                int idx = cell_of(g, x, y, z);
                const double *c = &g.mean[3 * (size_t)idx];
                float dx = c[0] - pt[0];
                float dy = c[1] - pt[1];
                float dz = c[2] - pt[2];
                float dist = std::sqrt(dx * dx + dy * dy + dz * dz);
                if (dist < radius) out[k++] = idx;
            }
        }
    }
    return k;
}

// ---------------------------------------------------------------------------
// Angle derivatives, eq. 6.19 / 6.21 (kernel.cpp:707-825).  jang[8][3] =
// j_ang a..h, hang[15][3] = h_ang a2 a3 b2 b3 c2 c3 d1 d2 d3 e1 e2 e3 f1 f2 f3.
struct AngleTerms {
    double j[8][3];
    double h[15][3];
};

void angle_terms(const double *p, AngleTerms &A, bool compat) {
    double cx, cy, cz, sx, sy, sz;
    if (std::fabs(p[3]) < 10e-5) { cx = 1.0; sx = 0.0; } else { cx = std::cos(p[3]); sx = std::sin(p[3]); }
    if (std::fabs(p[4]) < 10e-5) { cy = 1.0; sy = 0.0; } else { cy = std::cos(p[4]); sy = std::sin(p[4]); }
    if (std::fabs(p[5]) < 10e-5) { cz = 1.0; sz = 0.0; } else { cz = std::cos(p[5]); sz = std::sin(p[5]); }
    double(*j)[3] = A.j;
    j[0][0] = (-sx * sz + cx * sy * cz); j[0][1] = (-sx * cz - cx * sy * sz); j[0][2] = (-cx * cy);
    j[1][0] = (cx * sz + sx * sy * cz);  j[1][1] = (cx * cz - sx * sy * sz);  j[1][2] = (-sx * cy);
    j[2][0] = (-sy * cz);                j[2][1] = sy * sz;                   j[2][2] = cy;
    j[3][0] = sx * cy * cz;              j[3][1] = (-sx * cy * sz);           j[3][2] = sx * sy;
    j[4][0] = (-cx * cy * cz);           j[4][1] = cx * cy * sz;              j[4][2] = (-cx * sy);
    j[5][0] = (-cy * sz);                j[5][1] = (-cy * cz);                j[5][2] = 0;
    j[6][0] = (cx * cz - sx * sy * sz);  j[6][1] = (-cx * sz - sx * sy * cz); j[6][2] = 0;
    j[7][0] = (sx * cz + cx * sy * sz);  j[7][1] = (cx * sy * cz - sx * sz);  j[7][2] = 0;
    double(*h)[3] = A.h;
    h[0][0] = (-cx * sz - sx * sy * cz);  h[0][1] = (-cx * cz + sx * sy * sz);  h[0][2] = sx * cy;      // a2
    h[1][0] = (-sx * sz + cx * sy * cz);  h[1][1] = (-cx * sy * sz - sx * cz);  h[1][2] = (-cx * cy);   // a3
    h[2][0] = (cx * cy * cz);             h[2][1] = (-cx * cy * sz);            h[2][2] = (cx * sy);    // b2
    h[3][0] = (sx * cy * cz);             h[3][1] = (-sx * cy * sz);            h[3][2] = (sx * sy);    // b3
    h[4][0] = (-sx * cz - cx * sy * sz);  h[4][1] = (sx * sz - cx * sy * cz);   h[4][2] = 0;            // c2
    h[5][0] = (cx * cz - sx * sy * sz);   h[5][1] = (-sx * sy * cz - cx * sz);  h[5][2] = 0;            // c3
    // d1: d^2/db^2 of the rotated x component is (-cy cz, cy sz, -sy); the
    // reference has +sy (kernel.cpp:795-797), kept in compat mode only
    h[6][0] = (-cy * cz);                 h[6][1] = (cy * sz);                  h[6][2] = compat ? sy : -sy;
    h[7][0] = (-sx * sy * cz);            h[7][1] = (sx * sy * sz);             h[7][2] = (sx * cy);    // d2
    h[8][0] = (cx * sy * cz);             h[8][1] = (-cx * sy * sz);            h[8][2] = (-cx * cy);   // d3
    h[9][0] = (sy * sz);                  h[9][1] = (sy * cz);                  h[9][2] = 0;            // e1
    h[10][0] = (-sx * cy * sz);           h[10][1] = (-sx * cy * cz);           h[10][2] = 0;           // e2
    h[11][0] = (cx * cy * sz);            h[11][1] = (cx * cy * cz);            h[11][2] = 0;           // e3
    h[12][0] = (-cy * cz);                h[12][1] = (cy * sz);                 h[12][2] = 0;           // f1
    h[13][0] = (-cx * sz - sx * sy * cz); h[13][1] = (-cx * cz + sx * sy * sz); h[13][2] = 0;           // f2
    h[14][0] = (-sx * sz + cx * sy * cz); h[14][1] = (-cx * sy * sz - sx * cz); h[14][2] = 0;           // f3
}

inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Point Jacobian (3x6) and point Hessian (18x6), eq. 6.18 / 6.20
// (computePointDerivatives, kernel.cpp:495-560); J columns 0-2 are the
// identity (kernel.cpp:1191-1194), all other unset entries are zero.
struct PointTerms {
    double J[3][6];
    double H[18][6];
};

void point_terms(const AngleTerms &A, const double *x, PointTerms &P) {
    std::memset(&P, 0, sizeof(P));
    P.J[0][0] = 1.0; P.J[1][1] = 1.0; P.J[2][2] = 1.0;
    P.J[1][3] = dot3(x, A.j[0]); P.J[2][3] = dot3(x, A.j[1]);
    P.J[0][4] = dot3(x, A.j[2]); P.J[1][4] = dot3(x, A.j[3]); P.J[2][4] = dot3(x, A.j[4]);
    P.J[0][5] = dot3(x, A.j[5]); P.J[1][5] = dot3(x, A.j[6]); P.J[2][5] = dot3(x, A.j[7]);
    double a[3], b[3], c[3], d[3], e[3], f[3];
    a[0] = 0; a[1] = dot3(x, A.h[0]); a[2] = dot3(x, A.h[1]);
    b[0] = 0; b[1] = dot3(x, A.h[2]); b[2] = dot3(x, A.h[3]);
    c[0] = 0; c[1] = dot3(x, A.h[4]); c[2] = dot3(x, A.h[5]);
    d[0] = dot3(x, A.h[6]); d[1] = dot3(x, A.h[7]); d[2] = dot3(x, A.h[8]);
    e[0] = dot3(x, A.h[9]); e[1] = dot3(x, A.h[10]); e[2] = dot3(x, A.h[11]);
    f[0] = dot3(x, A.h[12]); f[1] = dot3(x, A.h[13]); f[2] = dot3(x, A.h[14]);
    const double *blk[3][3] = {{a, b, c}, {b, d, e}, {c, e, f}};
    for (int bi = 0; bi < 3; ++bi)
        for (int bj = 0; bj < 3; ++bj)
            for (int r = 0; r < 3; ++r) P.H[3 * (3 + bi) + r][3 + bj] = blk[bi][bj][r];
}

struct Gauss {
    double d1, d2;
};

// updateDerivatives (kernel.cpp:438-493) when compat, otherwise the
// Magnusson eq. 6.12 / 6.13 Hessian.  Returns the score increment (0 when
// the reference's validity test rejects the pair).
double update_pair(const Gauss &G, const PointTerms &P, const double *xt, const double *C,
                   bool hess, bool compat, double *g6, double *H36) {
    double xCx = C[0] * xt[0] * xt[0] + C[4] * xt[1] * xt[1] + C[8] * xt[2] * xt[2] +
                 (C[1] + C[3]) * xt[0] * xt[1] + (C[2] + C[6]) * xt[0] * xt[2] +
                 (C[5] + C[7]) * xt[1] * xt[2];
    double e = std::exp(-G.d2 * (xCx) / 2);
    double score_inc = -G.d1 * e;
    e = G.d2 * e;
    if (e > 1 || e < 0 || e != e) return 0;
    e *= G.d1;
    double cov_dxd_pi[3];
    for (int i = 0; i < 6; ++i) {
        for (int r = 0; r < 3; ++r) {
            cov_dxd_pi[r] = 0;
            for (int q = 0; q < 3; ++q) cov_dxd_pi[r] += C[3 * r + q] * P.J[q][i];
        }
        g6[i] += dot3(xt, cov_dxd_pi) * e;
        if (!hess) continue;
        for (int j = 0; j < 6; ++j) {
            double col[3] = {P.J[0][j], P.J[1][j], P.J[2][j]};
            if (compat) {
                double colh[3] = {col[0] + P.H[3 * i][j], col[1] + P.H[3 * i + 1][j],
                                  col[2] + P.H[3 * i + 2][j]};
                double mp[3];
                for (int r = 0; r < 3; ++r) {
                    mp[r] = 0;
                    for (int q = 0; q < 3; ++q) mp[r] += C[3 * r + q] * colh[q];
                }
                H36[6 * i + j] += e * (-G.d2 * dot3(xt, cov_dxd_pi) * dot3(xt, mp) + dot3(col, cov_dxd_pi));
            } else {
                double hb[3] = {P.H[3 * i][j], P.H[3 * i + 1][j], P.H[3 * i + 2][j]};
                double cj[3], ch[3];
                for (int r = 0; r < 3; ++r) {
                    cj[r] = C[3 * r] * col[0] + C[3 * r + 1] * col[1] + C[3 * r + 2] * col[2];
                    ch[r] = C[3 * r] * hb[0] + C[3 * r + 1] * hb[1] + C[3 * r + 2] * hb[2];
                }
                H36[6 * i + j] += e * (-G.d2 * dot3(xt, cov_dxd_pi) * dot3(xt, cj) + dot3(xt, ch) +
                                       dot3(col, cov_dxd_pi));
            }
        }
    }
    return score_inc;
}

// ---------------------------------------------------------------------------
// Pose build and pose vector.
// Mode R: buildTransformationMatrix (kernel.cpp:949-1013): float quaternion
// products with permuted components; only the rotation block and row 3 are
// written (the translation column keeps its previous value).
void build_tm_r(float *M, const double *t) {
    const float q_ha = 0.5f * t[3];
    const float q_w = std::cos((double)q_ha);  // double cos of the float, as the reference
    const float q_x = std::sin((double)q_ha);
    const float q_y = 0.0, q_z = 0.0;
    const float q_ha2 = 0.5f * t[4];
    const float q_w2 = std::cos((double)q_ha2);
    const float q_x2 = 0.0;
    const float q_y2 = std::sin((double)q_ha2);
    const float q_z2 = 0.0;
    const float q_ha3 = 0.5f * t[5];
    const float q_w3 = std::cos((double)q_ha3);
    const float q_x3 = 0.0, q_y3 = 0.0;
    const float q_z3 = std::sin((double)q_ha3);
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

// Mode F: T = Trans(p0..2) * Rx(p3) * Ry(p4) * Rz(p5), FP64 then rounded.
void build_tm_f(float *M, const double *p) {
    double ca = std::cos(p[3]), sa = std::sin(p[3]);
    double cb = std::cos(p[4]), sb = std::sin(p[4]);
    double cc = std::cos(p[5]), sc = std::sin(p[5]);
    double R[9] = {cb * cc, -cb * sc, sb,
                   ca * sc + sa * sb * cc, ca * cc - sa * sb * sc, -sa * cb,
                   sa * sc - ca * sb * cc, sa * cc + ca * sb * sc, ca * cb};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) M[4 * r + c] = (float)R[3 * r + c];
        M[4 * r + 3] = (float)p[r];
    }
    M[12] = 0.0f; M[13] = 0.0f; M[14] = 0.0f; M[15] = 1.0f;
}

// Mode R: eulerAngles (kernel.cpp:1146-1173), negated.
void euler_r(const float *M, double *out) {
    double res[3];
    res[0] = std::atan2((double)M[4 * 1 + 2], (double)M[4 * 2 + 2]);
    double n1 = M[0];
    double n2 = M[1];
    double c2 = std::sqrt(n1 * n1 + n2 * n2);
    if (res[0] > 0.0) {
        res[0] -= kPi;
        res[1] = std::atan2((double)-M[2], -c2);
    } else {
        res[1] = std::atan2((double)-M[2], c2);
    }
    double s1 = std::sin(res[0]);
    double c1 = std::cos(res[0]);
    res[2] = std::atan2(s1 * M[4 * 2 + 0] - c1 * M[4 * 1 + 0], c1 * M[4 * 1 + 1] - s1 * M[4 * 2 + 1]);
    out[0] = -res[0];
    out[1] = -res[1];
    out[2] = -res[2];
}

// Pose vector of a transform: translation column + angles.
void pose_vector(bool compat, const float *M, double *p) {
    p[0] = M[3];
    p[1] = M[7];
    p[2] = M[11];
    if (compat) {
        euler_r(M, p + 3);
    } else {
        double r12 = M[6], r22 = M[10], r02 = M[2], r00 = M[0], r01 = M[1];
        p[3] = std::atan2(-r12, r22);
        p[4] = std::atan2(r02, std::sqrt(r00 * r00 + r01 * r01));
        p[5] = std::atan2(-r01, r00);
    }
}

// solve (kernel.cpp:293-343): Gaussian elimination with partial pivoting;
// a zero pivot column is replaced by 0.001 (MAX_TRANSLATION_EPS).
void solve6(double *x, double A[6][6], double *b) {
    for (int j = 0; j < 6; ++j) {
        double mx = std::fabs(A[j][j]);
        int mi = j;
        for (int i = j + 1; i < 6; ++i)
            if (std::fabs(A[i][j]) > mx) {
                mi = i;
                mx = std::fabs(A[i][j]);
            }
        if (mi != j)
            for (int i = 0; i < 6; ++i) std::swap(A[mi][i], A[j][i]);
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

// transformPointCloud (kernel.cpp:385-404), float arithmetic.
void transform_cloud(const float *in, int n, const float *M, float *out) {
    for (int i = 0; i < n; ++i) {
        const float *p = in + 4 * (size_t)i;
        float *o = out + 4 * (size_t)i;
        for (int r = 0; r < 3; ++r)
            o[r] = M[4 * r] * p[0] + M[4 * r + 1] * p[1] + M[4 * r + 2] * p[2] + M[4 * r + 3];
        o[3] = 0.0f;
    }
}

// More-Thuente helpers (kernel.cpp:425-436, 827-946).
inline double psi_mt(double a, double f_a, double f_0, double g_0, double mu) { return (f_a - f_0 - mu * g_0 * a); }
inline double dpsi_mt(double g_a, double g_0, double mu) { return (g_a - mu * g_0); }

bool update_interval(double &a_l, double &f_l, double &g_l, double &a_u, double &f_u, double &g_u,
                     double a_t, double f_t, double g_t) {
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

double trial_value(double a_l, double f_l, double g_l, double a_u, double f_u, double g_u,
                   double a_t, double f_t, double g_t) {
    if (f_t > f_l) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = std::sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_q = a_l - 0.5 * (a_l - a_t) * g_l / (g_l - (f_l - f_t) / (a_l - a_t));
        if (std::fabs(a_c - a_l) < std::fabs(a_q - a_l)) return a_c;
        return 0.5 * (a_q + a_c);
    } else if (g_t * g_l < 0) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = std::sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_s = a_l - (a_l - a_t) / (g_l - g_t) * g_l;
        if (std::fabs(a_c - a_t) >= std::fabs(a_s - a_t)) return a_c;
        return a_s;
    } else if (std::fabs(g_t) <= std::fabs(g_l)) {
        double z = 3 * (f_t - f_l) / (a_t - a_l) - g_t - g_l;
        double w = std::sqrt(z * z - g_t * g_l);
        double a_c = a_l + (a_t - a_l) * (w - g_l - z) / (g_t - g_l + 2 * w);
        double a_s = a_l - (a_l - a_t) / (g_l - g_t) * g_l;
        double a_t_next = (std::fabs(a_c - a_t) < std::fabs(a_s - a_t)) ? a_c : a_s;
        if (a_t > a_l) return std::min(a_t + 0.66 * (a_u - a_t), a_t_next);
        return std::max(a_t + 0.66 * (a_u - a_t), a_t_next);
    }
    double z = 3 * (f_t - f_u) / (a_t - a_u) - g_t - g_u;
    double w = std::sqrt(z * z - g_t * g_u);
    return (a_u + (a_t - a_u) * (w - g_u - z) / (g_t - g_u + 2 * w));
}

// ---------------------------------------------------------------------------
// One registration (ndt_align + computeTransformation, kernel.cpp:1175-1272,
// 1375-1392) on a prebuilt grid.
struct Aligner {
    const ndt_params &prm;
    const Grid &grid;
    bool compat;
    Gauss gs;
    const float *scan = nullptr;
    int n = 0;
    std::vector<float> trans_f;   // float transformed cloud
    float final_T[16];
    int evals = 0;
    long long pairs = 0;
    long long *eval_pairs = nullptr;  // optional per-evaluation pair counts
    int eval_pairs_cap = 0;

    Aligner(const ndt_params &p, const Grid &g, Gauss gauss)
        : prm(p), grid(g), compat(p.compat != 0), gs(gauss) {}

    // transformPointCloud (kernel.cpp:385-404): float matrix, float arithmetic,
    // in both modes (the corrected mode builds the float matrix from the FP64
    // pose vector).
    void apply(const float *M) {
        trans_f.resize(4 * (size_t)n);
        transform_cloud(scan, n, M, trans_f.data());
    }

    // computeDerivatives (kernel.cpp:651-705) / computeHessian (:562-602).
    double derivatives(double *g6, double *H36, const double *p, bool hess, bool hessian_only) {
        const long long pairs_before = pairs;
        struct Log {
            Aligner *a;
            long long before;
            ~Log() {
                if (a->eval_pairs && a->evals - 1 < a->eval_pairs_cap) a->eval_pairs[a->evals - 1] = a->pairs - before;
            }
        } log_guard{this, pairs_before};
        ++evals;
        if (!hessian_only) std::memset(g6, 0, sizeof(double) * 6);
        std::memset(H36, 0, sizeof(double) * 36);
        double dummy_g[6];
        double *gg = hessian_only ? dummy_g : g6;
        AngleTerms A;
        angle_terms(p, A, prm.compat != 0);
        double score = 0.0;
        int nb[64];
        PointTerms P;
        for (int idx = 0; idx < n; ++idx) {
            // the reference's neighbour search in both modes; the corrected
            // grid marks cells below min_points unusable (radius_search_r
            // skips them through their NaN means)
            const float *tp = &trans_f[4 * (size_t)idx];
            const int k = radius_search_r(grid, tp, grid.res, nb);
            const double xt0[3] = {tp[0], tp[1], tp[2]};
            if (!k) continue;
            const float *sp = scan + 4 * (size_t)idx;
            double x[3] = {sp[0], sp[1], sp[2]};
            point_terms(A, x, P);
            for (int q = 0; q < k; ++q) {
                int c = nb[q];
                const double *mu = &grid.mean[3 * (size_t)c];
                double xt[3] = {xt0[0] - mu[0], xt0[1] - mu[1], xt0[2] - mu[2]};
                ++pairs;
                double inc = update_pair(gs, P, xt, &grid.icov[9 * (size_t)c], hess, compat, gg, H36);
                score += inc;
            }
        }
        return score;
    }

    void set_pose(const double *x_t) {
        if (compat)
            build_tm_r(final_T, x_t);
        else
            build_tm_f(final_T, x_t);
        apply(final_T);
    }

    // computeStepLengthMT (kernel.cpp:1015-1144).
    double step_length(const double *x, double *dir, double step_init, double step_max, double step_min,
                       double &score, double *g6, double *H36) {
        const double mu = 1.e-4, nu = 0.9;
        double phi_0 = -score;
        double d_phi_0 = -(g6[0] * dir[0] + g6[1] * dir[1] + g6[2] * dir[2] + g6[3] * dir[3] + g6[4] * dir[4] + g6[5] * dir[5]);
        double x_t[6] = {0, 0, 0, 0, 0, 0};
        if (d_phi_0 >= 0) {
            if (d_phi_0 == 0) return 0;
            d_phi_0 *= -1;
            for (int i = 0; i < 6; ++i) dir[i] *= -1;
        }
        const int max_step_iterations = 10;
        int step_iterations = 0;
        double a_l = 0, a_u = 0;
        double f_l = psi_mt(a_l, phi_0, phi_0, d_phi_0, mu);
        double g_l = dpsi_mt(d_phi_0, d_phi_0, mu);
        double f_u = psi_mt(a_u, phi_0, phi_0, d_phi_0, mu);
        double g_u = dpsi_mt(d_phi_0, d_phi_0, mu);
        // The reference tests "> 0" here (kernel.cpp:1053), which skips the
        // search whenever step_max > step_min; the corrected NDT tests "< 0".
        bool interval_converged = compat ? (step_max - step_min) > 0 : (step_max - step_min) < 0;
        bool open_interval = true;
        double a_t = step_init;
        a_t = std::min(a_t, step_max);
        a_t = std::max(a_t, step_min);
        for (int i = 0; i < 6; ++i) x_t[i] = x[i] + dir[i] * a_t;
        set_pose(x_t);
        score = derivatives(g6, H36, x_t, true, false);
        double phi_t = -score;
        double d_phi_t = -(g6[0] * dir[0] + g6[1] * dir[1] + g6[2] * dir[2] + g6[3] * dir[3] + g6[4] * dir[4] + g6[5] * dir[5]);
        double psi_t = psi_mt(a_t, phi_t, phi_0, d_phi_0, mu);
        double d_psi_t = dpsi_mt(d_phi_t, d_phi_0, mu);
        while (!interval_converged && step_iterations < max_step_iterations &&
               !(psi_t <= 0 && d_phi_t <= -nu * d_phi_0)) {
            if (open_interval)
                a_t = trial_value(a_l, f_l, g_l, a_u, f_u, g_u, a_t, psi_t, d_psi_t);
            else
                a_t = trial_value(a_l, f_l, g_l, a_u, f_u, g_u, a_t, phi_t, d_phi_t);
            a_t = std::min(a_t, step_max);
            a_t = std::max(a_t, step_min);
            for (int i = 0; i < 6; ++i) x_t[i] = x[i] + dir[i] * a_t;
            set_pose(x_t);
            score = derivatives(g6, H36, x_t, false, false);
            phi_t = -score;
            d_phi_t = -(g6[0] * dir[0] + g6[1] * dir[1] + g6[2] * dir[2] + g6[3] * dir[3] + g6[4] * dir[4] + g6[5] * dir[5]);
            psi_t = psi_mt(a_t, phi_t, phi_0, d_phi_0, mu);
            d_psi_t = dpsi_mt(d_phi_t, d_phi_0, mu);
            if (open_interval && (psi_t <= 0 && d_psi_t >= 0)) {
                open_interval = false;
                f_l = f_l + phi_0 - mu * d_phi_0 * a_l;
                g_l = g_l + mu * d_phi_0;
                f_u = f_u + phi_0 - mu * d_phi_0 * a_u;
                g_u = g_u + mu * d_phi_0;
            }
            if (open_interval)
                interval_converged = update_interval(a_l, f_l, g_l, a_u, f_u, g_u, a_t, psi_t, d_psi_t);
            else
                interval_converged = update_interval(a_l, f_l, g_l, a_u, f_u, g_u, a_t, phi_t, d_phi_t);
            step_iterations++;
        }
        if (step_iterations) derivatives(g6, H36, x_t, true, true);
        return a_t;
    }

    // computeTransformation (kernel.cpp:1175-1272).
    void run(const float *scan_in, int npts, const float *guess, float *out, int *converged, double *fitness) {
        scan = scan_in;
        n = npts;
        std::memcpy(final_T, guess, sizeof(float) * 16);
        double p[6], dp[6], g6[6], H36[36];
        pose_vector(compat, final_T, p);
        if (!compat) build_tm_f(final_T, p);
        apply(final_T);
        double score = derivatives(g6, H36, p, true, false);
        bool conv = false;
        int nr_iterations = 0;
        const double eps = prm.transformation_epsilon;
        while (!conv) {
            double A[6][6], neg_g[6];
            for (int i = 0; i < 6; ++i) {
                neg_g[i] = -g6[i];
                for (int j = 0; j < 6; ++j) A[i][j] = H36[6 * i + j];
            }
            solve6(dp, A, neg_g);
            double dp_norm = std::sqrt(dp[0] * dp[0] + dp[1] * dp[1] + dp[2] * dp[2] + dp[3] * dp[3] +
                                       dp[4] * dp[4] + dp[5] * dp[5]);
            if (compat) dp_norm = 1;  // kernel.cpp:1231
            if (dp_norm == 0 || dp_norm != dp_norm) {
                conv = dp_norm == dp_norm;
                break;
            }
            for (int i = 0; i < 6; ++i) dp[i] /= dp_norm;
            dp_norm = step_length(p, dp, dp_norm, prm.step_size, eps / 2, score, g6, H36);
            for (int i = 0; i < 6; ++i) dp[i] *= dp_norm;
            for (int i = 0; i < 6; ++i) p[i] = p[i] + dp[i];
            if (nr_iterations > prm.max_iterations || (nr_iterations && (std::fabs(dp_norm) < eps))) conv = true;
            nr_iterations++;
        }
        std::memcpy(out, final_T, sizeof(float) * 16);
        *converged = conv ? 1 : 0;
        *fitness = score / (double)n;
    }
};

void gauss_consts(const ndt_params &prm, Gauss &g) {
    // kernel.cpp:1181-1185
    double outlier = prm.outlier_ratio;
    float res = prm.resolution;
    double c1 = 10 * (1 - outlier);
    double c2 = outlier / std::pow(res, 3);
    double d3 = -std::log(c2);
    g.d1 = -std::log(c1 + c2) - d3;
    g.d2 = -2 * std::log((-std::log(c1 * std::exp(-0.5) + c2) - d3) / g.d1);
}

bool build_grid(const ndt_params &prm, Grid &g, const float *map, int m) {
    if (m <= 0) return false;
    if (prm.compat) return build_grid_r(g, map, m, prm.resolution);
    return build_grid_f(g, map, m, prm.resolution, prm.min_points_per_voxel, prm.eigen_ratio);
}

}  // namespace

#define ORACLE_API extern "C" __attribute__((visibility("default")))

ORACLE_API void oracle_gauss(const ndt_params *prm, double *d1, double *d2) {
    Gauss g;
    gauss_consts(*prm, g);
    *d1 = g.d1;
    *d2 = g.d2;
}

ORACLE_API int oracle_align(const ndt_params *prm, const float *scan, int n, const float *guess16,
                            const float *map, int m, float *out16, int *converged, double *fitness,
                            int *evals) {
    if (!prm || !scan || !guess16 || !map || n <= 0 || m <= 0) return NDT_E_ARG;
    Grid g;
    if (!build_grid(*prm, g, map, m)) return NDT_E_GRID;
    Gauss gs;
    gauss_consts(*prm, gs);
    Aligner a(*prm, g, gs);
    a.run(scan, n, guess16, out16, converged, fitness);
    if (evals) *evals = a.evals;
    return NDT_OK;
}

// Per-evaluation (point, voxel) pair counts of one alignment (diagnostics).
ORACLE_API int oracle_align_trace(const ndt_params *prm, const float *scan, int n, const float *guess16,
                                  const float *map, int m, long long *pairs, int cap) {
    Grid g;
    if (!build_grid(*prm, g, map, m)) return NDT_E_GRID;
    Gauss gs;
    gauss_consts(*prm, gs);
    Aligner a(*prm, g, gs);
    a.eval_pairs = pairs;
    a.eval_pairs_cap = cap;
    float out[16];
    int conv;
    double fit;
    a.run(scan, n, guess16, out, &conv, &fit);
    return a.evals;
}

ORACLE_API int oracle_align_batch(const ndt_params *prm, int B, const float *const *scans,
                                  const int *ns, const float *guesses, const float *map, int m,
                                  float *out16, int *converged, double *fitness, int *evals,
                                  int nthreads) {
    if (!prm || B < 0 || !map || m <= 0) return NDT_E_ARG;
    Grid g;
    if (!build_grid(*prm, g, map, m)) return NDT_E_GRID;
    Gauss gs;
    gauss_consts(*prm, gs);
    int err = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int b = 0; b < B; ++b) {
        if (ns[b] <= 0) {
            err = NDT_E_ARG;
            continue;
        }
        Aligner a(*prm, g, gs);
        a.run(scans[b], ns[b], guesses + 16 * (size_t)b, out16 + 16 * (size_t)b, converged + b, fitness + b);
        if (evals) evals[b] = a.evals;
    }
    return err;
}

ORACLE_API long long oracle_grid(const ndt_params *prm, const float *map, int m, float *bbox6,
                                 int *dims3, double *cells, long long cap) {
    Grid g;
    if (!build_grid(*prm, g, map, m)) return NDT_E_GRID;
    for (int e = 0; e < 3; ++e) {
        bbox6[e] = g.minv[e];
        bbox6[3 + e] = g.maxv[e];
        dims3[e] = g.dim[e];
    }
    if (cells && cap >= g.G)
        for (long long c = 0; c < g.G; ++c) {
            double *o = cells + 13 * c;
            for (int e = 0; e < 3; ++e) o[e] = g.mean[3 * c + e];
            for (int e = 0; e < 9; ++e) o[3 + e] = g.icov[9 * c + e];
            o[12] = (!prm->compat && !g.valid[c]) ? -(double)g.count[c] : (double)g.count[c];
        }
    return g.G;
}

// One pair: angle terms of p, point terms of x, then update_pair with the
// offset xt from the cell mean and the inverse covariance C (row major);
// g6 / H36 accumulate in place; returns the score increment.
ORACLE_API double oracle_update_pair(const ndt_params *prm, const double *p6, const double *x3, const double *xt3,
                                     const double *C9, int hessian, double *g6, double *H36) {
    Gauss gs;
    gauss_consts(*prm, gs);
    AngleTerms A;
    angle_terms(p6, A, prm->compat != 0);
    PointTerms P;
    point_terms(A, x3, P);
    return update_pair(gs, P, xt3, C9, hessian != 0, prm->compat != 0, g6, H36);
}

// voxelRadiusSearch (kernel.cpp:246-286) of Mode R on the grid of `map`:
// number of neighbour cells of point pt4 (their means to means3, up to cap).
ORACLE_API int oracle_radius_search(const ndt_params *prm, const float *map, int m, const float *pt4,
                                    double *means3, int cap) {
    Grid g;
    if (!prm->compat || !build_grid(*prm, g, map, m)) return NDT_E_GRID;
    int idx[64];
    const int k = radius_search_r(g, pt4, g.res, idx);
    for (int i = 0; i < k && i < cap; ++i)
        for (int e = 0; e < 3; ++e) means3[3 * i + e] = g.mean[3 * (size_t)idx[i] + e];
    return k;
}

ORACLE_API double oracle_derivatives(const ndt_params *prm, const float *map, int m,
                                     const float *scan, const float *trans, int n, const double *p6,
                                     int hessian, double *g6, double *H36, long long *pairs) {
    Grid g;
    if (!build_grid(*prm, g, map, m)) return NAN;
    Gauss gs;
    gauss_consts(*prm, gs);
    Aligner a(*prm, g, gs);
    a.scan = scan;
    a.n = n;
    a.trans_f.assign(trans, trans + 4 * (size_t)n);
    double Hd[36];
    double s = a.derivatives(g6, H36 ? H36 : Hd, p6, hessian != 0, false);
    if (pairs) *pairs = a.pairs;
    return s;
}

ORACLE_API void oracle_build_tm(int compat, const double *p6, float *m16) {
    if (compat) build_tm_r(m16, p6);
    else build_tm_f(m16, p6);
}

ORACLE_API void oracle_pose_vector(int compat, const float *m16, double *p6) { pose_vector(compat != 0, m16, p6); }

ORACLE_API void oracle_solve(const double *A36, const double *b6, double *x6) {
    double A[6][6], b[6];
    for (int i = 0; i < 6; ++i) {
        b[i] = b6[i];
        for (int j = 0; j < 6; ++j) A[i][j] = A36[6 * i + j];
    }
    solve6(x6, A, b);
}

ORACLE_API void oracle_invert(double *m9) { invert3(m9); }

ORACLE_API void oracle_transform(const float *in, int n, const float *m16, float *out) {
    transform_cloud(in, n, m16, out);
}

ORACLE_API double oracle_trial_value(double a_l, double f_l, double g_l, double a_u, double f_u,
                                     double g_u, double a_t, double f_t, double g_t) {
    return trial_value(a_l, f_l, g_l, a_u, f_u, g_u, a_t, f_t, g_t);
}

ORACLE_API int oracle_update_interval(double *io6, double a_t, double f_t, double g_t) {
    return update_interval(io6[0], io6[1], io6[2], io6[3], io6[4], io6[5], a_t, f_t, g_t) ? 1 : 0;
}
