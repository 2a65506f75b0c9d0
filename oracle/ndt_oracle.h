/*
 * CPU oracle for the NDT align path -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg may
 * load this library, and only as the checker (or the timed CPU port): the
 * product path (daphne-benchmark_b200/) never links or calls it.
 *
 * Two modes behind one parameter block (ndt_params from include/ndt_b200.h):
 *  - compat = 1 (Mode R): an FP64 restatement of the reference kernel
 *    src/CPU/ndt_mapping/kernel.cpp, with the same floating-point operation
 *    order, so that it agrees bit for bit with the compiled reference
 *    (pinned by tests/test_oracle_pin.py against oracle/_ref and the golden
 *    fixtures in tests/golden/).
 *  - compat = 0 (Mode F): the corrected NDT in FP64 -- the accuracy oracle for
 *    the GPU's corrected mode.
 */
#ifndef NDT_ORACLE_H
#define NDT_ORACLE_H
#include "../include/ndt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Gauss fitting constants d1, d2 (kernel.cpp:1181-1185). */
void oracle_gauss(const ndt_params *prm, double *d1, double *d2);

/* Full alignment.  evals (may be NULL) receives the derivative evaluations. */
int oracle_align(const ndt_params *prm, const float *scan, int n, const float *guess16,
                 const float *map, int m, float *out16, int *converged, double *fitness,
                 int *evals);

/* B alignments against ONE shared map (grid built once), nthreads host threads. */
int oracle_align_batch(const ndt_params *prm, int B, const float *const *scans, const int *ns,
                       const float *guesses, const float *map, int m, float *out16,
                       int *converged, double *fitness, int *evals, int nthreads);

/* Grid: bbox6, dims3, and per cell 13 doubles (mean3, icov9, count). Returns G. */
long long oracle_grid(const ndt_params *prm, const float *map, int m, float *bbox6, int *dims3,
                      double *cells, long long cap);

/* One derivative evaluation of `trans` (already transformed scan). */
double oracle_derivatives(const ndt_params *prm, const float *map, int m, const float *scan,
                          const float *trans, int n, const double *p6, int hessian, double *g6,
                          double *H36, long long *pairs);

/* Pose helpers. */
void oracle_build_tm(int compat, const double *p6, float *m16);
void oracle_pose_vector(int compat, const float *m16, double *p6);
void oracle_solve(const double *A36, const double *b6, double *x6);
void oracle_invert(double *m9);
void oracle_transform(const float *in, int n, const float *m16, float *out);
double oracle_trial_value(double a_l, double f_l, double g_l, double a_u, double f_u, double g_u,
                          double a_t, double f_t, double g_t);
int oracle_update_interval(double *io6, double a_t, double f_t, double g_t);

#ifdef __cplusplus
}
#endif
#endif
