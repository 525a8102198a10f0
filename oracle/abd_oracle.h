/*
 * abd_oracle.h — CPU oracle for the ABD Newton step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C FP64 restatement of the
 * reference's ABD path (Luke-Skycrawler/colb: abd.py, contact.py,
 * barrier.py, ortho.py, abd_simple.py, gauss_newton.py).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may call it, as a
 * checker or a timed CPU baseline; the product (colb_b200) never does.
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors,
 * and three of its functions live in the empty ipctk_wp submodule, so the
 * restatement follows the published formulas it names (IPC squared
 * distances, Ericson's segment closest point, additive CCD).  Its
 * derivatives are pinned by finite differences and its pair set by a
 * float32 numpy restatement of the same predicate (tests/golden).
 */
#ifndef ABD_ORACLE_H
#define ABD_ORACLE_H
#include "../include/abd_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- primitive math (exported for known-answer / FD tests) ---------- */
void oracle_barrier(int kind, double x, double xhat, double out3[3]);
void oracle_ortho(const double q9[9], double k, double* e, double g9[9], double H81[81]);
/* Ericson closest points between segments, in float (contact.py:166) */
void oracle_seg_seg_f32(const float p1[3], const float q1[3], const float p2[3],
                        const float q2[3], float eps, float out_std[3]);
void oracle_seg_seg_f64(const double p1[3], const double q1[3], const double p2[3],
                        const double q2[3], double eps, double out_std[3]);
/* squared distances with gradient and Hessian */
void oracle_d2_pp(const double x6[6], double* f, double g6[6], double H36[36]);
void oracle_d2_pe(const double x9[9], double* f, double g9[9], double H81[81]);
void oracle_d2_ee_line(const double x12[12], double* f, double g12[12], double H144[144]);
void oracle_d2_pt_plane(const double x12[12], double* f, double g12[12], double H144[144]);
/* point-triangle region: 0..2 vertex t0..t2, 3 edge t0t1, 4 edge t1t2, 5 edge t2t0, 6 face */
int oracle_pt_region(const double p[3], const double a[3], const double b[3], const double c[3]);
double oracle_pt_dist2(const double p[3], const double a[3], const double b[3], const double c[3]);
void oracle_psd_project(int n, double* H);
/* additive CCD along linear displacement; kind 0 EE (x12, p12), 1 PT.
 * returns 1 on hit with *toi, 0 otherwise */
int oracle_accd(int kind, const double x12[12], const double p12[12], double s,
                double tmax, double* toi);

/* ---- whole-scene oracle -------------------------------------------- */
typedef struct OracleWorld OracleWorld;

OracleWorld* oracle_create(const AbdParams* params, const AbdSceneDesc* scenes, int n_scenes);
void oracle_destroy(OracleWorld* w);
int oracle_set_state(OracleWorld* w, const double* st);
int oracle_get_state(OracleWorld* w, double* st);
int oracle_get_vertices(OracleWorld* w, double* x);
/* sorted candidate list like abd_get_pairs */
int oracle_get_pairs(OracleWorld* w, int32_t* out4, int32_t* kinds, int cap, int* n);
int oracle_energy(OracleWorld* w, double* e_per_scene);
int oracle_assemble(OracleWorld* w, double* grad, double* hess_dense);
int oracle_solve(OracleWorld* w, double* du, int* iters);
int oracle_step(OracleWorld* w, int n_steps, AbdStepStats* stats);
int oracle_get_profile(OracleWorld* w, int scene, double* res, double* alpha, int* iters_per_step,
                       int cap, int* n);
int oracle_set_warm_start(OracleWorld* w, const float* dq12, int nb);
int oracle_count_intersections(OracleWorld* w, int* count);
void oracle_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
