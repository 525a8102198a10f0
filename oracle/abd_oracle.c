/*
 * abd_oracle.c — FP64 CPU oracle of the ABD Newton step with barrier contact.
 *
 * TEST INFRASTRUCTURE ONLY (see abd_oracle.h).  It restates, loop by loop,
 * what the reference computes:
 *   state / transform ......... abd_simple.py:26-49, quat_util.py:40-47, BDF1.py:11-14
 *   inertia + orthogonality ... abd.py:53-64, :77-85, :108-166; ortho.py:9-41
 *   barrier ................... barrier.py:6-65
 *   candidate pairs ........... contact.py:25-32, :133-169 (float32 predicate)
 *   contact grad/Hessian ...... abd.py:168-571 (EE / PE / PP classification)
 *   linear solve .............. abd.py:631-658 (here: block-Jacobi BiCGSTAB / PCG)
 *   line search ............... gauss_newton.py:98-115, abd.py:725-746, :768-785
 *   Newton loop, forward ...... abd.py:574-581, :674-702
 * plus the components the reference does not have (point-triangle and
 * half-space contacts, additive CCD, batched scenes), restated from the
 * published methods named at each function.
 *
 * Build: gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off (oracle/Makefile).
 * -ffp-contract=off keeps every float32 operation of the segment predicate
 * individually rounded, which is how the CUDA kernels evaluate it.
 */
#include "abd_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* small vector helpers                                                 */
/* ------------------------------------------------------------------ */
static inline double dot3(const double* a, const double* b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
static inline void sub3(const double* a, const double* b, double* o) { o[0]=a[0]-b[0]; o[1]=a[1]-b[1]; o[2]=a[2]-b[2]; }
static inline void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1]*b[2] - a[2]*b[1]; o[1] = a[2]*b[0] - a[0]*b[2]; o[2] = a[0]*b[1] - a[1]*b[0];
}
/* [a]x such that [a]x b = a x b, row-major 3x3 */
static inline void skew3(const double* a, double* S) {
    S[0]=0;     S[1]=-a[2]; S[2]=a[1];
    S[3]=a[2];  S[4]=0;     S[5]=-a[0];
    S[6]=-a[1]; S[7]=a[0];  S[8]=0;
}
static inline void matmul3(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
        double s = 0; for (int k = 0; k < 3; k++) s += A[3*i+k]*B[3*k+j]; C[3*i+j] = s;
    }
}
static inline double clampd(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------ */
/* barrier.py:6-65 — all three barriers in x = d^2, zero for x >= xh   */
/* ------------------------------------------------------------------ */
void oracle_barrier(int kind, double x, double xh, double out[3]) {
    out[0] = out[1] = out[2] = 0.0;
    if (!(x < xh)) return;
    double t = x - xh;
    if (kind == ABD_BARRIER_CUBIC) {            /* barrier.py:47-65 */
        out[0] = -t * t * t;
        out[1] = -3.0 * t * t;
        out[2] = -6.0 * t;
    } else if (kind == ABD_BARRIER_QUADRATIC) { /* barrier.py:23-44 */
        out[0] = t * t;
        out[1] = 2.0 * t;
        out[2] = 2.0;
    } else {                                    /* barrier.py:6-21, normalised by xh^2 */
        double l = log(x / xh);
        out[0] = -t * t * l / (xh * xh);
        out[1] = (xh - x) * (2.0 * l + t / x) / (xh * xh);
        out[2] = -(2.0 * l + t / x + t * (2.0 / x + xh / (x * x))) / (xh * xh);
    }
}

/* ------------------------------------------------------------------ */
/* ortho.py:9-41 — E = k sum_ij (a_i.a_j - delta_ij)^2 over rows a_i     */
/* ------------------------------------------------------------------ */
void oracle_ortho(const double q[9], double k, double* e, double g[9], double H[81]) {
    const double* a[3] = {q, q + 3, q + 6};
    if (e) {
        double s = 0;
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
            double t = dot3(a[i], a[j]) - (i == j ? 1.0 : 0.0);
            s += t * t;
        }
        *e = s * k;
    }
    if (g) {
        for (int i = 0; i < 3; i++) {
            double gi[3] = {-a[i][0], -a[i][1], -a[i][2]};
            for (int j = 0; j < 3; j++) {
                double d = dot3(a[i], a[j]);
                for (int c = 0; c < 3; c++) gi[c] += d * a[j][c];
            }
            for (int c = 0; c < 3; c++) g[3*i+c] = gi[c] * 4.0 * k;
        }
    }
    if (H) {
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
            double B[9];
            if (i == j) {
                double d = dot3(a[i], a[i]) - 1.0;
                for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) {
                    double s = 0;
                    for (int m = 0; m < 3; m++) s += a[m][r] * a[m][c];
                    s += a[i][r] * a[i][c] + (r == c ? d : 0.0);
                    B[3*r+c] = s;
                }
            } else {
                double d = dot3(a[j], a[i]);
                for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++)
                    B[3*r+c] = a[j][r] * a[i][c] + (r == c ? d : 0.0);
            }
            for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++)
                H[(3*i+r)*9 + 3*j+c] = B[3*r+c] * 4.0 * k;
        }
    }
}

/* ------------------------------------------------------------------ */
/* Closest points between two segments: Ericson, Real-Time Collision    */
/* Detection (2005) §5.1.9, in float32 as contact.py:166 / abd.py:190   */
/* call it.  Returns (s, t, |c1-c2|).  Every operation is one IEEE      */
/* rounding (no contraction), dot = (x*x + y*y) + z*z.                   */
/* ------------------------------------------------------------------ */
static inline float dotf(const float* a, const float* b) { return (a[0]*b[0] + a[1]*b[1]) + a[2]*b[2]; }
void oracle_seg_seg_f32(const float p1[3], const float q1[3], const float p2[3], const float q2[3],
                        float eps, float out[3]) {
    float d1[3], d2[3], r[3];
    for (int k = 0; k < 3; k++) { d1[k] = q1[k] - p1[k]; d2[k] = q2[k] - p2[k]; r[k] = p1[k] - p2[k]; }
    float a = dotf(d1, d1), e = dotf(d2, d2), f = dotf(d2, r);
    float s, t;
    if (a <= eps && e <= eps) { s = 0.f; t = 0.f; }
    else if (a <= eps) { s = 0.f; t = clampf(f / e, 0.f, 1.f); }
    else {
        float c = dotf(d1, r);
        if (e <= eps) { t = 0.f; s = clampf(-c / a, 0.f, 1.f); }
        else {
            float b = dotf(d1, d2);
            float denom = a * e - b * b;
            s = (denom != 0.f) ? clampf((b * f - c * e) / denom, 0.f, 1.f) : 0.f;
            t = (b * s + f) / e;
            if (t < 0.f) { t = 0.f; s = clampf(-c / a, 0.f, 1.f); }
            else if (t > 1.f) { t = 1.f; s = clampf((b - c) / a, 0.f, 1.f); }
        }
    }
    float dv[3];
    for (int k = 0; k < 3; k++) dv[k] = (p1[k] + d1[k] * s) - (p2[k] + d2[k] * t);
    out[0] = s; out[1] = t; out[2] = sqrtf(dotf(dv, dv));
}
void oracle_seg_seg_f64(const double p1[3], const double q1[3], const double p2[3], const double q2[3],
                        double eps, double out[3]) {
    double d1[3], d2[3], r[3];
    for (int k = 0; k < 3; k++) { d1[k] = q1[k] - p1[k]; d2[k] = q2[k] - p2[k]; r[k] = p1[k] - p2[k]; }
    double a = dot3(d1, d1), e = dot3(d2, d2), f = dot3(d2, r);
    double s, t;
    if (a <= eps && e <= eps) { s = 0; t = 0; }
    else if (a <= eps) { s = 0; t = clampd(f / e, 0, 1); }
    else {
        double c = dot3(d1, r);
        if (e <= eps) { t = 0; s = clampd(-c / a, 0, 1); }
        else {
            double b = dot3(d1, d2);
            double denom = a * e - b * b;
            s = (denom != 0.0) ? clampd((b * f - c * e) / denom, 0, 1) : 0.0;
            t = (b * s + f) / e;
            if (t < 0) { t = 0; s = clampd(-c / a, 0, 1); }
            else if (t > 1) { t = 1; s = clampd((b - c) / a, 0, 1); }
        }
    }
    double dv[3];
    for (int k = 0; k < 3; k++) dv[k] = (p1[k] + d1[k] * s) - (p2[k] + d2[k] * t);
    out[0] = s; out[1] = t; out[2] = sqrt(dot3(dv, dv));
}

/* ------------------------------------------------------------------ */
/* Squared distances (IPC, Li et al. 2020, §4 / supplement): value,    */
/* gradient and Hessian w.r.t. the stencil points.  A stencil function  */
/* is written in a few auxiliary vectors y = L x; the map L has entries */
/* in {-1,0,1} per (point, aux) and is applied at the end.              */
/* ------------------------------------------------------------------ */
static void map_aux(int np, int na, const int C[4][3], const double* gy, const double* Hy,
                    double* gx, double* Hx) {
    /* gy: 3*na, Hy: (3na)^2 row-major; gx: 3*np, Hx: (3np)^2 */
    int ny = 3 * na, nx = 3 * np;
    for (int i = 0; i < np; i++) for (int k = 0; k < 3; k++) {
        double s = 0;
        for (int a = 0; a < na; a++) s += C[i][a] * gy[3*a+k];
        gx[3*i+k] = s;
    }
    for (int i = 0; i < np; i++) for (int j = 0; j < np; j++)
        for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) {
            double s = 0;
            for (int a = 0; a < na; a++) if (C[i][a])
                for (int b = 0; b < na; b++) if (C[j][b])
                    s += C[i][a] * C[j][b] * Hy[(3*a+r)*ny + 3*b+c];
            Hx[(3*i+r)*nx + 3*j+c] = s;
        }
}

/* point-point: f = |x0 - x1|^2 */
void oracle_d2_pp(const double x[6], double* f, double g[6], double H[36]) {
    double d[3]; sub3(x, x + 3, d);
    *f = dot3(d, d);
    for (int k = 0; k < 3; k++) { g[k] = 2*d[k]; g[3+k] = -2*d[k]; }
    memset(H, 0, 36*sizeof(double));
    for (int k = 0; k < 3; k++) {
        H[k*6+k] = 2; H[(3+k)*6+3+k] = 2; H[k*6+3+k] = -2; H[(3+k)*6+k] = -2;
    }
}

/* point-line: stencil (p, e0, e1); w = p - e0, e = e1 - e0,
 * f = w.w - (w.e)^2/(e.e) = |w x e|^2/|e|^2 */
void oracle_d2_pe(const double x[9], double* f, double g[9], double H[81]) {
    double w[3], e[3]; sub3(x, x + 3, w); sub3(x + 6, x + 3, e);
    double c = dot3(w, e), s = dot3(e, e);
    *f = dot3(w, w) - c * c / s;
    double gy[6], Hy[36];
    for (int k = 0; k < 3; k++) {
        gy[k] = 2*w[k] - 2*c/s*e[k];
        gy[3+k] = -2*c/s*w[k] + 2*c*c/(s*s)*e[k];
    }
    for (int r = 0; r < 3; r++) for (int q = 0; q < 3; q++) {
        double I = (r == q) ? 1.0 : 0.0;
        Hy[r*6+q] = 2*I - 2/s*e[r]*e[q];                                          /* ww */
        double we = -2/s*e[r]*w[q] - 2*c/s*I + 4*c/(s*s)*e[r]*e[q];               /* d(g_w)_r/de_q */
        Hy[r*6+3+q] = we;
        Hy[(3+q)*6+r] = we;
        Hy[(3+r)*6+3+q] = -2/s*w[r]*w[q] + 4*c/(s*s)*(w[r]*e[q] + e[r]*w[q])
                          - 8*c*c/(s*s*s)*e[r]*e[q] + 2*c*c/(s*s)*I;               /* ee */
    }
    static const int C[4][3] = {{1, 0, 0}, {-1, -1, 0}, {0, 1, 0}, {0, 0, 0}};
    map_aux(3, 2, C, gy, Hy, g, H);
}

/* f = (w.n)^2/(n.n), n = u x v, derivatives w.r.t. y = (w, u, v) */
static void d2_wn(const double* w, const double* u, const double* v, double* f, double gy[9], double Hy[81]) {
    double n[3]; cross3(u, v, n);
    double a = dot3(w, n), b = dot3(n, n);
    *f = a * a / b;
    double ga[9], gb[9];
    double vw[3], wu[3], vn[3], nu[3];
    cross3(v, w, vw); cross3(w, u, wu); cross3(v, n, vn); cross3(n, u, nu);
    for (int k = 0; k < 3; k++) {
        ga[k] = n[k]; ga[3+k] = vw[k]; ga[6+k] = wu[k];
        gb[k] = 0;    gb[3+k] = 2*vn[k]; gb[6+k] = 2*nu[k];
    }
    double Ha[81], Hb[81];
    memset(Ha, 0, sizeof Ha); memset(Hb, 0, sizeof Hb);
    double Su[9], Sv[9], Sw[9], Sn[9];
    skew3(u, Su); skew3(v, Sv); skew3(w, Sw); skew3(n, Sn);
    /* Ha: [w][u] = -[v]x, [w][v] = [u]x, [u][v] = -[w]x, and transposes */
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) {
        Ha[(0+r)*9 + 3+c] = -Sv[3*r+c]; Ha[(3+c)*9 + 0+r] = -Sv[3*r+c];
        Ha[(0+r)*9 + 6+c] =  Su[3*r+c]; Ha[(6+c)*9 + 0+r] =  Su[3*r+c];
        Ha[(3+r)*9 + 6+c] = -Sw[3*r+c]; Ha[(6+c)*9 + 3+r] = -Sw[3*r+c];
    }
    /* Hb = 2 Jn^T Jn + 2 sum_k n_k d2 n_k, Jn = [-[v]x, [u]x] */
    double SvT_Sv[9], Sv_Su[9], Su_Sv[9], SuT_Su[9], SvT[9], SuT[9];
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) { SvT[3*r+c] = Sv[3*c+r]; SuT[3*r+c] = Su[3*c+r]; }
    matmul3(SvT, Sv, SvT_Sv); matmul3(Sv, Su, Sv_Su); matmul3(Su, Sv, Su_Sv); matmul3(SuT, Su, SuT_Su);
    for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) {
        Hb[(3+r)*9 + 3+c] = 2*SvT_Sv[3*r+c];
        Hb[(3+r)*9 + 6+c] = 2*Sv_Su[3*r+c] - 2*Sn[3*r+c];
        Hb[(6+r)*9 + 3+c] = 2*Su_Sv[3*r+c] + 2*Sn[3*r+c];
        Hb[(6+r)*9 + 6+c] = 2*SuT_Su[3*r+c];
    }
    for (int i = 0; i < 9; i++) gy[i] = 2*a/b*ga[i] - a*a/(b*b)*gb[i];
    for (int i = 0; i < 9; i++) for (int j = 0; j < 9; j++)
        Hy[i*9+j] = 2/b*ga[i]*ga[j] + 2*a/b*Ha[i*9+j]
                  - 2*a/(b*b)*(ga[i]*gb[j] + gb[i]*ga[j])
                  + 2*a*a/(b*b*b)*gb[i]*gb[j] - a*a/(b*b)*Hb[i*9+j];
}

/* line-line: stencil (ea0, ea1, eb0, eb1); w = ea0-eb0, u = ea1-ea0, v = eb1-eb0 */
void oracle_d2_ee_line(const double x[12], double* f, double g[12], double H[144]) {
    double w[3], u[3], v[3], gy[9], Hy[81];
    sub3(x, x + 6, w); sub3(x + 3, x, u); sub3(x + 9, x + 6, v);
    d2_wn(w, u, v, f, gy, Hy);
    static const int C[4][3] = {{1, -1, 0}, {0, 1, 0}, {-1, 0, -1}, {0, 0, 1}};
    map_aux(4, 3, C, gy, Hy, g, H);
}
/* point-plane: stencil (p, t0, t1, t2); w = p-t0, u = t1-t0, v = t2-t0 */
void oracle_d2_pt_plane(const double x[12], double* f, double g[12], double H[144]) {
    double w[3], u[3], v[3], gy[9], Hy[81];
    sub3(x, x + 3, w); sub3(x + 6, x + 3, u); sub3(x + 9, x + 3, v);
    d2_wn(w, u, v, f, gy, Hy);
    static const int C[4][3] = {{1, 0, 0}, {-1, -1, -1}, {0, 1, 0}, {0, 0, 1}};
    map_aux(4, 3, C, gy, Hy, g, H);
}

/* Closest-point region of p on triangle abc: Ericson §5.1.5. */
int oracle_pt_region(const double p[3], const double a[3], const double b[3], const double c[3]) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
    sub3(b, a, ab); sub3(c, a, ac); sub3(p, a, ap);
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) return 0;
    sub3(p, b, bp);
    double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3 >= 0 && d4 <= d3) return 1;
    double vc = d1*d4 - d3*d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return 3;
    sub3(p, c, cp);
    double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) return 2;
    double vb = d5*d2 - d1*d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return 5;
    double va = d3*d6 - d5*d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) return 4;
    return 6;
}
double oracle_pt_dist2(const double p[3], const double a[3], const double b[3], const double c[3]) {
    int r = oracle_pt_region(p, a, b, c);
    const double* T[3] = {a, b, c};
    double f, g[12], H[144], x[12];
    if (r <= 2) { double d[3]; sub3(p, T[r], d); return dot3(d, d); }
    if (r <= 5) {
        int i0 = r - 3, i1 = (r - 3 + 1) % 3;
        memcpy(x, p, 24); memcpy(x + 3, T[i0], 24); memcpy(x + 6, T[i1], 24);
        oracle_d2_pe(x, &f, g, H); return f;
    }
    memcpy(x, p, 24); memcpy(x + 3, a, 24); memcpy(x + 6, b, 24); memcpy(x + 9, c, 24);
    oracle_d2_pt_plane(x, &f, g, H); return f;
}

/* ------------------------------------------------------------------ */
/* Symmetric eigen-decomposition by cyclic Jacobi rotations and the PSD  */
/* projection V max(L,0) V^T (used where the reference calls            */
/* x_to_grad_psd_hess_ee, abd.py:247).  A matrix whose Cholesky         */
/* factorization succeeds is returned unchanged.  The entry a rotation  */
/* annihilates is set to zero rather than left at rounding level, so   */
/* the sweeps end once the off-diagonal mass has decayed.                */
/* ------------------------------------------------------------------ */
/* Cholesky without storing the factor: 1 when every pivot is positive, in
 * which case the matrix is its own PSD projection. */
static int is_pd(int n, const double* H) {
    double L[144];
    memcpy(L, H, (size_t)n * n * sizeof(double));
    for (int k = 0; k < n; k++) {
        double d = L[k*n+k];
        if (!(d > 0)) return 0;
        d = sqrt(d);
        for (int i = k + 1; i < n; i++) L[i*n+k] /= d;
        for (int i = k + 1; i < n; i++)
            for (int j = k + 1; j <= i; j++) L[i*n+j] -= L[i*n+k] * L[j*n+k];
    }
    return 1;
}

void oracle_psd_project(int n, double* H) {
    double A[144], V[144];
    if (is_pd(n, H)) return;
    memcpy(A, H, (size_t)n * n * sizeof(double));
    for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) V[i*n+j] = (i == j);
    double fro = 0; for (int i = 0; i < n*n; i++) fro += A[i]*A[i];
    if (fro == 0) return;
    /* a rotation is skipped when |a_pq| is at rounding level against its
     * diagonal pair (1e-15 of their geometric mean) or against the whole
     * matrix (1e-14 of its Frobenius norm, above the fill rotations leave);
     * the sweeps stop when none was applied (scale-invariant) */
    for (int sweep = 0; sweep < 50; sweep++) {
        int rotated = 0;
        for (int p = 0; p < n; p++) for (int q = p + 1; q < n; q++) {
            double apq = A[p*n+q];
            if (fabs(apq) <= fmax(1e-15 * sqrt(fabs(A[p*n+p] * A[q*n+q])), 1e-14 * sqrt(fro))) continue;
            rotated = 1;
            double theta = (A[q*n+q] - A[p*n+p]) / (2 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta*theta + 1));
            double c = 1 / sqrt(t*t + 1), s = t * c;
            for (int k = 0; k < n; k++) {          /* A <- A R */
                double akp = A[k*n+p], akq = A[k*n+q];
                A[k*n+p] = c*akp - s*akq; A[k*n+q] = s*akp + c*akq;
            }
            for (int k = 0; k < n; k++) {          /* A <- R^T A */
                double apk = A[p*n+k], aqk = A[q*n+k];
                A[p*n+k] = c*apk - s*aqk; A[q*n+k] = s*apk + c*aqk;
            }
            for (int k = 0; k < n; k++) {
                double vkp = V[k*n+p], vkq = V[k*n+q];
                V[k*n+p] = c*vkp - s*vkq; V[k*n+q] = s*vkp + c*vkq;
            }
            A[p*n+q] = A[q*n+p] = 0.0;      /* the rotation annihilates it */
        }
        if (!rotated) break;
    }
    for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) {
        double s = 0;
        for (int k = 0; k < n; k++) { double l = A[k*n+k]; if (l > 0) s += V[i*n+k]*l*V[j*n+k]; }
        H[i*n+j] = s;
    }
}

/* ------------------------------------------------------------------ */
/* Additive CCD (Li, Kaufman, Jiang 2021, "Codimensional Incremental    */
/* Potential Contact", Alg. 1) with thickness 0: advance along the      */
/* relative linear motion by steps bounded by the current distance      */
/* over the relative speed bound, stopping once the distance falls      */
/* below s times its start value.                                        */
/* ------------------------------------------------------------------ */
static double prim_dist2(int kind, const double* x) {
    if (kind == 0) { double o[3]; oracle_seg_seg_f64(x, x+3, x+6, x+9, 0.0, o); return o[2]*o[2]; }
    return oracle_pt_dist2(x, x+3, x+6, x+9);
}
#define ACCD_MAX_ITERS 100000
static int g_ccd_cap_hit = 0;
int oracle_accd(int kind, const double x0[12], const double p0[12], double s, double tmax, double* toi) {
    double x[12], p[12], pm[3] = {0, 0, 0};
    memcpy(x, x0, sizeof x); memcpy(p, p0, sizeof p);
    for (int i = 0; i < 4; i++) for (int k = 0; k < 3; k++) pm[k] += p[3*i+k] * 0.25;
    for (int i = 0; i < 4; i++) for (int k = 0; k < 3; k++) p[3*i+k] -= pm[k];
    double n[4]; for (int i = 0; i < 4; i++) n[i] = sqrt(dot3(p + 3*i, p + 3*i));
    double lp = (kind == 0) ? fmax(n[0], n[1]) + fmax(n[2], n[3])
                            : n[0] + fmax(n[1], fmax(n[2], n[3]));
    if (lp == 0) return 0;
    double d2 = prim_dist2(kind, x), d = sqrt(d2);
    if (d == 0.0) { *toi = 0.0; return 1; }
    double g = s * d;                /* (d^2 - xi^2)/(d + xi) with xi = 0 */
    double t = 0, tl = (1 - s) * d / lp;
    for (int it = 0; it < ACCD_MAX_ITERS; it++) {
        for (int i = 0; i < 12; i++) x[i] += tl * p[i];
        d2 = prim_dist2(kind, x); d = sqrt(d2);
        if (t > 0 && d < g) { *toi = t; return 1; }
        t += tl;
        if (t > tmax) return 0;
        tl = 0.9 * d / lp;
    }
    g_ccd_cap_hit = 1;
    *toi = t; return 1;
}

/* ------------------------------------------------------------------ */
/* scene storage                                                        */
/* ------------------------------------------------------------------ */
#define ST_NOW 0
#define ST_NXT 24
#define ST_C 0
#define ST_Q 3
#define ST_V 12
#define ST_QD 15

typedef struct { int kind, a, b; } Cand;

typedef struct {
    int nb, nv, ne, nt, np;
    double *xbar, *mass, *J, *st, *planes, *x;
    int *vbody, *edges, *tris;
    Cand* cand; int nc, ccap;
    double *ws; int has_ws;
    double *prof_res, *prof_alpha; int *prof_iters; int prof_n, prof_steps, prof_cap;
    double *box_cache;
} OScene;

struct OracleWorld { AbdParams P; int ns; OScene* s; };

static int g_threads = 1;
void oracle_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

static void* xalloc(size_t n) { void* p = calloc(1, n ? n : 1); return p; }

OracleWorld* oracle_create(const AbdParams* P, const AbdSceneDesc* d, int ns) {
    OracleWorld* w = (OracleWorld*)xalloc(sizeof *w);
    w->P = *P; w->ns = ns;
    w->s = (OScene*)xalloc(sizeof(OScene) * ns);
    for (int i = 0; i < ns; i++) {
        OScene* S = &w->s[i]; const AbdSceneDesc* D = &d[i];
        S->nb = D->n_bodies; S->nv = D->n_verts; S->ne = D->n_edges; S->nt = D->n_tris; S->np = D->n_planes;
        S->xbar = xalloc(sizeof(double) * 3 * S->nv); memcpy(S->xbar, D->xbar, sizeof(double) * 3 * S->nv);
        S->vbody = xalloc(sizeof(int) * S->nv); memcpy(S->vbody, D->vert_body, sizeof(int) * S->nv);
        S->edges = xalloc(sizeof(int) * 2 * S->ne); if (S->ne) memcpy(S->edges, D->edges, sizeof(int) * 2 * S->ne);
        S->tris = xalloc(sizeof(int) * 3 * S->nt); if (S->nt) memcpy(S->tris, D->tris, sizeof(int) * 3 * S->nt);
        S->mass = xalloc(sizeof(double) * S->nb); memcpy(S->mass, D->mass, sizeof(double) * S->nb);
        S->J = xalloc(sizeof(double) * S->nb); memcpy(S->J, D->inertia_J, sizeof(double) * S->nb);
        S->st = xalloc(sizeof(double) * 48 * S->nb); memcpy(S->st, D->state, sizeof(double) * 48 * S->nb);
        S->planes = xalloc(sizeof(double) * 4 * S->np); if (S->np) memcpy(S->planes, D->planes, sizeof(double) * 4 * S->np);
        S->x = xalloc(sizeof(double) * 3 * S->nv);
        S->ccap = 1024; S->cand = xalloc(sizeof(Cand) * S->ccap);
        S->ws = xalloc(sizeof(double) * 12 * S->nb);
    }
    return w;
}
void oracle_destroy(OracleWorld* w) {
    if (!w) return;
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        free(S->xbar); free(S->vbody); free(S->edges); free(S->tris); free(S->mass); free(S->J);
        free(S->st); free(S->planes); free(S->x); free(S->cand); free(S->ws);
        free(S->prof_res); free(S->prof_alpha); free(S->prof_iters);
    }
    free(w->s); free(w);
}
int oracle_set_state(OracleWorld* w, const double* st) {
    for (int i = 0; i < w->ns; i++) { memcpy(w->s[i].st, st, sizeof(double) * 48 * w->s[i].nb); st += 48 * w->s[i].nb; }
    return 0;
}
int oracle_get_state(OracleWorld* w, double* st) {
    for (int i = 0; i < w->ns; i++) { memcpy(st, w->s[i].st, sizeof(double) * 48 * w->s[i].nb); st += 48 * w->s[i].nb; }
    return 0;
}

/* x = q^T xbar + c of the nxt state (abd_simple.py:26-35), evaluated as
 * c_k + q0k xb0 + q1k xb1 + q2k xb2 with fused multiply-adds. */
static void transform(const OScene* S, const double* st, double* x) {
    for (int v = 0; v < S->nv; v++) {
        const double* s = st + 48 * S->vbody[v] + ST_NXT;
        const double* xb = S->xbar + 3 * v;
        for (int k = 0; k < 3; k++) {
            double t = s[ST_C + k];
            t = fma(s[ST_Q + 0 + k], xb[0], t);
            t = fma(s[ST_Q + 3 + k], xb[1], t);
            t = fma(s[ST_Q + 6 + k], xb[2], t);
            x[3*v + k] = t;
        }
    }
}
int oracle_get_vertices(OracleWorld* w, double* x) {
    for (int i = 0; i < w->ns; i++) { transform(&w->s[i], w->s[i].st, x); x += 3 * w->s[i].nv; }
    return 0;
}

static inline int dynamic(const OScene* S, int b) { return S->mass[b] > 0.0; }

/* ------------------------------------------------------------------ */
/* Broad phase: sort-and-sweep on x over padded boxes.                  */
/* ------------------------------------------------------------------ */
typedef struct { double lo[3], hi[3]; int id, set; } Box;
static int box_cmp(const void* a, const void* b) {
    double x = ((const Box*)a)->lo[0], y = ((const Box*)b)->lo[0];
    if (x < y) return -1; if (x > y) return 1;
    int i = ((const Box*)a)->set * 0x40000000 + ((const Box*)a)->id;
    int j = ((const Box*)b)->set * 0x40000000 + ((const Box*)b)->id;
    return (i > j) - (i < j);
}
static int cand_cmp(const void* a, const void* b) {
    const Cand* x = (const Cand*)a; const Cand* y = (const Cand*)b;
    if (x->kind != y->kind) return x->kind - y->kind;
    if (x->a != y->a) return (x->a > y->a) - (x->a < y->a);
    return (x->b > y->b) - (x->b < y->b);
}
typedef struct { Cand* v; int n, cap; } CandVec;
static void cv_push(CandVec* c, int kind, int a, int b) {
    if (c->n == c->cap) { c->cap = c->cap ? 2 * c->cap : 256; c->v = realloc(c->v, sizeof(Cand) * c->cap); }
    c->v[c->n].kind = kind; c->v[c->n].a = a; c->v[c->n].b = b; c->n++;
}

/* pairs of boxes (set 0 with set 0 when two_sets == 0, else set 0 with set 1) */
typedef void (*pair_fn)(void* ctx, CandVec* out, int ida, int idb);
static void sweep(Box* bx, int n, int two_sets, pair_fn fn, void* ctx, CandVec* out) {
    qsort(bx, n, sizeof(Box), box_cmp);
    int nt = g_threads;
    CandVec* loc = (CandVec*)xalloc(sizeof(CandVec) * nt);
    #pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        for (int j = i + 1; j < n && bx[j].lo[0] <= bx[i].hi[0]; j++) {
            if (bx[j].lo[1] > bx[i].hi[1] || bx[j].hi[1] < bx[i].lo[1]) continue;
            if (bx[j].lo[2] > bx[i].hi[2] || bx[j].hi[2] < bx[i].lo[2]) continue;
            if (!two_sets) {
                int a = bx[i].id, b = bx[j].id;
                if (a > b) { int t = a; a = b; b = t; }
                fn(ctx, &loc[tid], a, b);
            } else if (bx[i].set != bx[j].set) {
                if (bx[i].set == 0) fn(ctx, &loc[tid], bx[i].id, bx[j].id);
                else fn(ctx, &loc[tid], bx[j].id, bx[i].id);
            }
        }
    }
    for (int t = 0; t < nt; t++) { for (int k = 0; k < loc[t].n; k++) cv_push(out, loc[t].v[k].kind, loc[t].v[k].a, loc[t].v[k].b); free(loc[t].v); }
    free(loc);
}

typedef struct { const OracleWorld* w; const OScene* S; const double* x; double filt; } DetCtx;

/* EE candidate predicate (contact.py:158-168): i<j, no shared vertex,
 * distance < filter; float32 closest points when ee_f32. */
static int ee_dist(const AbdParams* P, const OScene* S, const double* x, int i, int j, double out[3]) {
    const int* ea = S->edges + 2*i; const int* eb = S->edges + 2*j;
    if (P->ee_f32) {
        float p1[3], q1[3], p2[3], q2[3], o[3];
        for (int k = 0; k < 3; k++) {
            p1[k] = (float)x[3*ea[0]+k]; q1[k] = (float)x[3*ea[1]+k];
            p2[k] = (float)x[3*eb[0]+k]; q2[k] = (float)x[3*eb[1]+k];
        }
        oracle_seg_seg_f32(p1, q1, p2, q2, 1e-6f, o);
        out[0] = o[0]; out[1] = o[1]; out[2] = o[2];
        return 1;
    }
    oracle_seg_seg_f64(x + 3*ea[0], x + 3*ea[1], x + 3*eb[0], x + 3*eb[1], 1e-12, out);
    return 0;
}
static int ee_filter_pass(const AbdParams* P, const double* o, double filt) {
    if (P->ee_f32) return (float)o[2] < (float)filt;
    return o[2] < filt;
}
static void ee_cb(void* c, CandVec* out, int i, int j) {
    DetCtx* d = (DetCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* ea = S->edges + 2*i; const int* eb = S->edges + 2*j;
    if (ea[0] == eb[0] || ea[0] == eb[1] || ea[1] == eb[0] || ea[1] == eb[1]) return;
    if (!P->self_contact && S->vbody[ea[0]] == S->vbody[eb[0]]) return;
    double o[3]; ee_dist(P, S, d->x, i, j, o);
    if (ee_filter_pass(P, o, d->filt)) cv_push(out, ABD_CONTACT_EE, i, j);
}
static void pt_cb(void* c, CandVec* out, int p, int t) {
    DetCtx* d = (DetCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* tr = S->tris + 3*t;
    if (p == tr[0] || p == tr[1] || p == tr[2]) return;
    if (!P->self_contact && S->vbody[p] == S->vbody[tr[0]]) return;
    double f = oracle_pt_dist2(d->x + 3*p, d->x + 3*tr[0], d->x + 3*tr[1], d->x + 3*tr[2]);
    if (f < d->filt * d->filt) cv_push(out, ABD_CONTACT_PT, p, t);
}

/* Candidate list at positions x with distance filter filt, sorted. */
static void detect(const OracleWorld* w, OScene* S, const double* x, double filt) {
    const AbdParams* P = &w->P;
    CandVec out = {0};
    DetCtx ctx = {w, S, x, filt};
    double pad = 0.5 * filt * (1.0 + 1e-6) + 1e-7;
    if (P->contact_ee && S->ne > 1) {
        Box* bx = (Box*)xalloc(sizeof(Box) * S->ne);
        for (int e = 0; e < S->ne; e++) {
            const double* a = x + 3*S->edges[2*e]; const double* b = x + 3*S->edges[2*e+1];
            for (int k = 0; k < 3; k++) {
                double lo = fmin(a[k], b[k]), hi = fmax(a[k], b[k]);
                if (P->ee_f32) { lo = fmin((double)(float)a[k], (double)(float)b[k]); hi = fmax((double)(float)a[k], (double)(float)b[k]); }
                bx[e].lo[k] = lo - pad; bx[e].hi[k] = hi + pad;
            }
            bx[e].id = e; bx[e].set = 0;
        }
        sweep(bx, S->ne, 0, ee_cb, &ctx, &out);
        free(bx);
    }
    if (P->contact_pt && S->nt > 0) {
        Box* bx = (Box*)xalloc(sizeof(Box) * (S->nv + S->nt));
        for (int v = 0; v < S->nv; v++) {
            for (int k = 0; k < 3; k++) { bx[v].lo[k] = x[3*v+k] - pad; bx[v].hi[k] = x[3*v+k] + pad; }
            bx[v].id = v; bx[v].set = 0;
        }
        for (int t = 0; t < S->nt; t++) {
            Box* B = &bx[S->nv + t];
            for (int k = 0; k < 3; k++) {
                double a = x[3*S->tris[3*t]+k], b = x[3*S->tris[3*t+1]+k], c = x[3*S->tris[3*t+2]+k];
                B->lo[k] = fmin(a, fmin(b, c)) - pad; B->hi[k] = fmax(a, fmax(b, c)) + pad;
            }
            B->id = t; B->set = 1;
        }
        sweep(bx, S->nv + S->nt, 1, pt_cb, &ctx, &out);
        free(bx);
    }
    for (int pl = 0; pl < S->np; pl++) {
        const double* n = S->planes + 4*pl;
        for (int v = 0; v < S->nv; v++) {
            double d = dot3(n, x + 3*v) - n[3];
            if (d < filt) cv_push(&out, ABD_CONTACT_PG, v, pl);
        }
    }
    qsort(out.v, out.n, sizeof(Cand), cand_cmp);
    if (out.n > S->ccap) { S->ccap = out.n; S->cand = realloc(S->cand, sizeof(Cand) * S->ccap); }
    if (out.n) memcpy(S->cand, out.v, sizeof(Cand) * out.n);
    S->nc = out.n;
    free(out.v);
}

int oracle_get_pairs(OracleWorld* w, int32_t* out4, int32_t* kinds, int cap, int* n) {
    int tot = 0;
    int voff = 0, eoff = 0, toff = 0, poff = 0;
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        transform(S, S->st, S->x);
        detect(w, S, S->x, w->P.cand_dist);
        for (int c = 0; c < S->nc && tot < cap; c++, tot++) {
            const Cand* C = &S->cand[c];
            int32_t* o = out4 + 4*tot;
            if (C->kind == ABD_CONTACT_EE) {
                o[0] = S->edges[2*C->a] + voff; o[1] = S->edges[2*C->a+1] + voff;
                o[2] = S->edges[2*C->b] + voff; o[3] = S->edges[2*C->b+1] + voff;
            } else if (C->kind == ABD_CONTACT_PT) {
                o[0] = C->a + voff; o[1] = S->tris[3*C->b] + voff; o[2] = S->tris[3*C->b+1] + voff; o[3] = S->tris[3*C->b+2] + voff;
            } else { o[0] = C->a + voff; o[1] = C->b + poff; o[2] = -1; o[3] = -1; }
            if (kinds) kinds[tot] = C->kind;
        }
        voff += S->nv; eoff += S->ne; toff += S->nt; poff += S->np;
    }
    *n = tot;
    return 0;
}

/* ------------------------------------------------------------------ */
/* One contact: stencil, barrier argument, gradient and Hessian on the  */
/* stencil points (abd.py:198-571 for EE/PE/PP).                        */
/* ------------------------------------------------------------------ */
typedef struct { int n; int v[4]; double e, noise; double g[12]; double H[144]; int active; int type; } CEval;

#define T_PP 0
#define T_PE 1
#define T_EE 2
#define T_PT 3
#define T_PG 4

static void eval_contact(const OracleWorld* w, const OScene* S, const double* x, const Cand* C,
                         int deriv, CEval* out) {
    const AbdParams* P = &w->P;
    double xh = P->dhat * P->dhat;
    double sc = P->kappa * P->dt * P->dt;
    out->active = 0; out->e = 0; out->noise = 0; out->n = 0;
    double xb = 0;  /* barrier argument */
    double f = 0, g[12], H[144], pts[12];
    int type = -1;
    if (C->kind == ABD_CONTACT_EE) {
        int i0 = S->edges[2*C->a], i1 = S->edges[2*C->a+1], i2 = S->edges[2*C->b], i3 = S->edges[2*C->b+1];
        double o[3]; int f32 = ee_dist(P, S, x, C->a, C->b, o);
        double d = o[2];
        if (!(d < P->dhat)) return;
        int a0 = o[0] == 0.0, a1 = o[0] == 1.0, b0 = o[1] == 0.0, b1 = o[1] == 1.0;
        if ((a0 || a1) && (b0 || b1)) {                       /* abd.py:352-361 */
            type = T_PP; out->n = 2;
            out->v[0] = a0 ? i0 : i1; out->v[1] = b0 ? i2 : i3;
        } else if (a0 || a1 || b0 || b1) {                    /* abd.py:457-464 */
            type = T_PE; out->n = 3;
            if (a0) { out->v[0] = i0; out->v[1] = i2; out->v[2] = i3; }
            else if (a1) { out->v[0] = i1; out->v[1] = i2; out->v[2] = i3; }
            else if (b0) { out->v[0] = i2; out->v[1] = i0; out->v[2] = i1; }
            else { out->v[0] = i3; out->v[1] = i0; out->v[2] = i1; }
        } else {
            type = T_EE; out->n = 4;
            out->v[0] = i0; out->v[1] = i1; out->v[2] = i2; out->v[3] = i3;
        }
        for (int k = 0; k < out->n; k++) memcpy(pts + 3*k, x + 3*out->v[k], 24);
        if (type == T_PP) oracle_d2_pp(pts, &f, g, H);
        else if (type == T_PE) oracle_d2_pe(pts, &f, g, H);
        else oracle_d2_ee_line(pts, &f, g, H);
        xb = f32 ? d * d : f;
    } else if (C->kind == ABD_CONTACT_PT) {
        const int* tr = S->tris + 3*C->b;
        int p = C->a;
        int r = oracle_pt_region(x + 3*p, x + 3*tr[0], x + 3*tr[1], x + 3*tr[2]);
        out->v[0] = p;
        if (r <= 2) { type = T_PP; out->n = 2; out->v[1] = tr[r]; }
        else if (r <= 5) { type = T_PE; out->n = 3; out->v[1] = tr[r-3]; out->v[2] = tr[(r-3+1)%3]; }
        else { type = T_PT; out->n = 4; out->v[1] = tr[0]; out->v[2] = tr[1]; out->v[3] = tr[2]; }
        for (int k = 0; k < out->n; k++) memcpy(pts + 3*k, x + 3*out->v[k], 24);
        if (type == T_PP) oracle_d2_pp(pts, &f, g, H);
        else if (type == T_PE) oracle_d2_pe(pts, &f, g, H);
        else oracle_d2_pt_plane(pts, &f, g, H);
        if (!(f < xh)) return;
        xb = f;
    } else {
        const double* n = S->planes + 4*C->b;
        int p = C->a;
        double d = dot3(n, x + 3*p) - n[3];
        if (!(d < P->dhat)) return;
        type = T_PG; out->n = 1; out->v[0] = p;
        f = d * d;
        for (int k = 0; k < 3; k++) g[k] = 2 * d * n[k];
        for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++) H[r*3+c] = 2 * n[r] * n[c];
        xb = f;
    }
    double B[3]; oracle_barrier(P->barrier, xb, xh, B);
    out->active = 1; out->type = type;
    out->e = B[0] * sc;
    {
        /* scale of the FP64 evaluation error: the term, plus the barrier
         * slope times the error of x from positions rounded at magnitude L
         * (FP32 distances carry 2^29 times the FP64 rounding) */
        double L = 0;
        for (int k = 0; k < out->n; k++) for (int c = 0; c < 3; c++) L = fmax(L, fabs(x[3*out->v[k] + c]));
        double mult = 1.0;
        if (C->kind == ABD_CONTACT_EE && P->ee_f32) mult = 536870912.0;
        if (C->kind == ABD_CONTACT_PG) L = fmax(L, fabs(S->planes[4*C->b + 3]));
        out->noise = sc * (fabs(B[0]) + fabs(B[1]) * 8.0 * sqrt(fabs(xb)) * L * mult) * DBL_EPSILON;
    }
    if (!deriv) return;
    int m = 3 * out->n;
    if (P->hess_mode == ABD_HESS_REFERENCE) {
        if (type == T_EE) oracle_psd_project(12, H);             /* abd.py:247 */
        for (int i = 0; i < m; i++) for (int j = 0; j < m; j++) {
            double h = (type == T_PP) ? 0.0 : B[1] * H[i*m+j];    /* abd.py:381-382 */
            out->H[i*m+j] = (h + B[2] * g[i] * g[j]) * sc;
        }
    } else {
        for (int i = 0; i < m; i++) for (int j = 0; j < m; j++)
            out->H[i*m+j] = B[1] * H[i*m+j] + B[2] * g[i] * g[j];
        oracle_psd_project(m, out->H);
        for (int i = 0; i < m*m; i++) out->H[i] *= sc;
    }
    for (int i = 0; i < m; i++) out->g[i] = g[i] * B[1] * sc;
}

/* ------------------------------------------------------------------ */
/* Energy (abd.py:53-75, :725-735)                                       */
/* ------------------------------------------------------------------ */
/* scale of the FP64 evaluation error of the orthogonality energy:
 * k sum_ij (t_ij^2 + 4 |t_ij| |a_i| |a_j|), t_ij = a_i.a_j - delta_ij */
static double ortho_noise(const double q[9], double k) {
    double na[3], e = 0;
    for (int i = 0; i < 3; i++) na[i] = sqrt(dot3(q + 3*i, q + 3*i));
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) {
        double t = dot3(q + 3*i, q + 3*j) - (i == j);
        e += t * t + 4.0 * fabs(t) * na[i] * na[j];
    }
    return e * k;
}
/* inertia + orthogonality energy of one body; *noise (may be NULL) gets the
 * scale of its FP64 evaluation error */
static double body_energy(const OracleWorld* w, const OScene* S, const double* st, int b, double* noise) {
    const AbdParams* P = &w->P; double dt = P->dt;
    const double* s = st + 48*b;
    const double* now = s + ST_NOW; const double* nx = s + ST_NXT;
    double eo; oracle_ortho(nx + ST_Q, P->k_ortho, &eo, NULL, NULL);
    double dq0[3], n1 = 0, s0 = 0, s1 = 0;
    for (int k = 0; k < 3; k++) {
        double ct = now[ST_C+k] + dt * now[ST_V+k] + dt * dt * P->gravity[k];
        dq0[k] = nx[ST_C+k] - ct;
        s0 += fabs(dq0[k]) * (fabs(nx[ST_C+k]) + fabs(ct));
    }
    for (int r = 0; r < 9; r++) {
        double qt = now[ST_Q+r] + dt * now[ST_QD+r];
        double d = nx[ST_Q+r] - qt; n1 += d * d;
        s1 += fabs(d) * (fabs(nx[ST_Q+r]) + fabs(qt));
    }
    double nm = dot3(dq0, dq0) * S->mass[b] + n1 * S->J[b];
    double e = eo * dt * dt + 0.5 * nm;
    if (noise) *noise = (e + s0 * fabs(S->mass[b]) + s1 * fabs(S->J[b]) + dt * dt * ortho_noise(nx + ST_Q, P->k_ortho)) * DBL_EPSILON;
    return e;
}
/* total energy of a scene; *noise (may be NULL) gets the scale of its FP64
 * evaluation error (sum over terms) */
static double scene_energy(const OracleWorld* w, OScene* S, const double* st, double* noise) {
    double e = 0, en = 0;
    for (int b = 0; b < S->nb; b++) { double nb_; e += body_energy(w, S, st, b, &nb_); en += nb_; }
    transform(S, st, S->x);
    detect(w, S, S->x, w->P.cand_dist);   /* abd.py:732: re-detect with the candidate filter */
    double* ec = (double*)xalloc(sizeof(double) * 2 * (S->nc + 1));
    #pragma omp parallel for num_threads(g_threads) schedule(dynamic, 64)
    for (int c = 0; c < S->nc; c++) { CEval ce; eval_contact(w, S, S->x, &S->cand[c], 0, &ce); ec[2*c] = ce.e; ec[2*c+1] = ce.noise; }
    for (int c = 0; c < S->nc; c++) { e += ec[2*c]; en += ec[2*c+1]; }
    free(ec);
    if (noise) *noise = en;
    return e;
}
int oracle_energy(OracleWorld* w, double* e) {
    for (int i = 0; i < w->ns; i++) e[i] = scene_energy(w, &w->s[i], w->s[i].st, NULL);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Block-sparse matrix of 12x12 body blocks                             */
/* ------------------------------------------------------------------ */
typedef struct { int r, c; double v[144]; } Blk;
typedef struct { int nb; int* rowptr; int* col; double* val; int nnzb; } BSR;
static int blk_cmp(const void* a, const void* b) {
    const Blk* x = (const Blk*)a; const Blk* y = (const Blk*)b;
    if (x->r != y->r) return x->r - y->r; return x->c - y->c;
}
static void bsr_free(BSR* A) { free(A->rowptr); free(A->col); free(A->val); memset(A, 0, sizeof *A); }
static void bsr_from_blocks(int nb, Blk* bl, int n, BSR* A) {
    qsort(bl, n, sizeof(Blk), blk_cmp);
    int m = 0;
    for (int i = 0; i < n; i++) {
        if (m > 0 && bl[m-1].r == bl[i].r && bl[m-1].c == bl[i].c) { for (int k = 0; k < 144; k++) bl[m-1].v[k] += bl[i].v[k]; }
        else { if (m != i) bl[m] = bl[i]; m++; }
    }
    A->nb = nb; A->nnzb = m;
    A->rowptr = (int*)xalloc(sizeof(int) * (nb + 1));
    A->col = (int*)xalloc(sizeof(int) * (m + 1));
    A->val = (double*)xalloc(sizeof(double) * 144 * (m + 1));
    for (int i = 0; i < m; i++) { A->rowptr[bl[i].r + 1]++; A->col[i] = bl[i].c; memcpy(A->val + 144*i, bl[i].v, sizeof(double) * 144); }
    for (int r = 0; r < nb; r++) A->rowptr[r+1] += A->rowptr[r];
}
static void bsr_mv(const BSR* A, const double* x, double* y) {
    #pragma omp parallel for num_threads(g_threads)
    for (int r = 0; r < A->nb; r++) {
        double acc[12] = {0};
        for (int k = A->rowptr[r]; k < A->rowptr[r+1]; k++) {
            const double* V = A->val + 144*k; const double* xc = x + 12*A->col[k];
            for (int i = 0; i < 12; i++) { double s = 0; for (int j = 0; j < 12; j++) s += V[12*i+j] * xc[j]; acc[i] += s; }
        }
        memcpy(y + 12*r, acc, sizeof acc);
    }
}

/* gradient + Hessian of one scene at its nxt state, with the candidate
 * list of that state (abd.py:681-688) */
typedef struct { double* g; BSR A; int n_active; } Assembly;

static void add_block(Blk** bl, int* n, int* cap, int r, int c, const double* v) {
    if (*n == *cap) { *cap = *cap ? 2 * *cap : 1024; *bl = realloc(*bl, sizeof(Blk) * *cap); }
    (*bl)[*n].r = r; (*bl)[*n].c = c; memcpy((*bl)[*n].v, v, sizeof(double) * 144); (*n)++;
}

static void assemble_scene(const OracleWorld* w, OScene* S, Assembly* out) {
    const AbdParams* P = &w->P; double dt = P->dt;
    int nb = S->nb;
    out->g = (double*)xalloc(sizeof(double) * 12 * nb);
    Blk* bl = NULL; int nbl = 0, cap = 0;
    transform(S, S->st, S->x);
    detect(w, S, S->x, P->cand_dist);
    /* abd.py:108-149 inertia + orthogonality */
    for (int b = 0; b < nb; b++) {
        double blk[144] = {0};
        double* g = out->g + 12*b;
        if (dynamic(S, b)) {
            const double* now = S->st + 48*b + ST_NOW; const double* nx = S->st + 48*b + ST_NXT;
            double go[9], Ho[81];
            oracle_ortho(nx + ST_Q, P->k_ortho, NULL, go, Ho);
            for (int k = 0; k < 3; k++) {
                double ct = now[ST_C+k] + dt * now[ST_V+k] + dt * dt * P->gravity[k];
                g[k] = (nx[ST_C+k] - ct) * S->mass[b];
            }
            for (int r = 0; r < 9; r++) {
                double qt = now[ST_Q+r] + dt * now[ST_QD+r];
                g[3+r] = dt * dt * go[r] + (nx[ST_Q+r] - qt) * S->J[b];
            }
            for (int i = 0; i < 81; i++) Ho[i] *= dt * dt;
            if (P->hess_mode == ABD_HESS_PROJECTED) oracle_psd_project(9, Ho);
            for (int k = 0; k < 3; k++) blk[k*12+k] = S->mass[b];
            for (int i = 0; i < 9; i++) for (int j = 0; j < 9; j++)
                blk[(3+i)*12 + 3+j] = Ho[i*9+j] + (i == j ? S->J[b] : 0.0);
        } else {
            for (int k = 0; k < 12; k++) blk[k*12+k] = P->pinned_diag;
        }
        add_block(&bl, &nbl, &cap, b, b, blk);
    }
    /* abd.py:198-571 contacts */
    CEval* ce = (CEval*)xalloc(sizeof(CEval) * (S->nc + 1));
    #pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
    for (int c = 0; c < S->nc; c++) eval_contact(w, S, S->x, &S->cand[c], 1, &ce[c]);
    int nact = 0;
    for (int c = 0; c < S->nc; c++) {
        CEval* E = &ce[c];
        if (!E->active) continue;
        nact++;
        int m = 3 * E->n;
        for (int i = 0; i < E->n; i++) {
            int v = E->v[i], b = S->vbody[v];
            if (!dynamic(S, b)) continue;
            const double* xb = S->xbar + 3*v;
            double Jv[4] = {1, xb[0], xb[1], xb[2]};
            for (int al = 0; al < 4; al++) for (int k = 0; k < 3; k++) out->g[12*b + 3*al + k] += Jv[al] * E->g[3*i+k];
        }
        for (int i = 0; i < E->n; i++) for (int j = 0; j < E->n; j++) {
            int vi = E->v[i], vj = E->v[j], bi = S->vbody[vi], bj = S->vbody[vj];
            if (!dynamic(S, bi) || !dynamic(S, bj)) continue;
            const double* xi = S->xbar + 3*vi; const double* xj = S->xbar + 3*vj;
            double Ji[4] = {1, xi[0], xi[1], xi[2]}, Jj[4] = {1, xj[0], xj[1], xj[2]};
            double blk[144];
            for (int al = 0; al < 4; al++) for (int be = 0; be < 4; be++)
                for (int r = 0; r < 3; r++) for (int cc = 0; cc < 3; cc++)
                    blk[(3*al+r)*12 + 3*be+cc] = Ji[al] * Jj[be] * E->H[(3*i+r)*m + 3*j+cc];
            add_block(&bl, &nbl, &cap, bi, bj, blk);
        }
    }
    free(ce);
    out->n_active = nact;
    bsr_from_blocks(nb, bl, nbl, &out->A);
    free(bl);
}

int oracle_assemble(OracleWorld* w, double* grad, double* hess) {
    int off = 0, tot = 0;
    for (int i = 0; i < w->ns; i++) tot += w->s[i].nb;
    if (hess) memset(hess, 0, sizeof(double) * 144 * (size_t)tot * tot);
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        Assembly as; assemble_scene(w, S, &as);
        memcpy(grad + 12*off, as.g, sizeof(double) * 12 * S->nb);
        if (hess) {
            int n = 12 * tot;
            for (int r = 0; r < S->nb; r++) for (int k = as.A.rowptr[r]; k < as.A.rowptr[r+1]; k++) {
                int c = as.A.col[k];
                for (int a = 0; a < 12; a++) for (int b = 0; b < 12; b++)
                    hess[(size_t)(12*(off+r)+a)*n + 12*(off+c)+b] = as.A.val[144*k + 12*a + b];
            }
        }
        free(as.g); bsr_free(&as.A);
        off += S->nb;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Block-Jacobi preconditioned Krylov solvers (abd.py:631-636)          */
/* ------------------------------------------------------------------ */
static int inv12(const double* A, double* Ai) {
    double M[12][24];
    for (int i = 0; i < 12; i++) for (int j = 0; j < 24; j++) M[i][j] = j < 12 ? A[12*i+j] : (j - 12 == i);
    for (int c = 0; c < 12; c++) {
        int p = c; for (int r = c + 1; r < 12; r++) if (fabs(M[r][c]) > fabs(M[p][c])) p = r;
        if (M[p][c] == 0.0) return -1;
        if (p != c) for (int j = 0; j < 24; j++) { double t = M[p][j]; M[p][j] = M[c][j]; M[c][j] = t; }
        double iv = 1.0 / M[c][c];
        for (int j = 0; j < 24; j++) M[c][j] *= iv;
        for (int r = 0; r < 12; r++) if (r != c) {
            double f = M[r][c]; if (f == 0.0) continue;
            for (int j = 0; j < 24; j++) M[r][j] -= f * M[c][j];
        }
    }
    for (int i = 0; i < 12; i++) for (int j = 0; j < 12; j++) Ai[12*i+j] = M[i][12+j];
    return 0;
}
static void precond(int nb, const double* Dinv, const double* x, double* y) {
    for (int b = 0; b < nb; b++) for (int i = 0; i < 12; i++) {
        double s = 0; for (int j = 0; j < 12; j++) s += Dinv[144*b + 12*i + j] * x[12*b + j]; y[12*b + i] = s;
    }
}
static double vdot(int n, const double* a, const double* b) { double s = 0; for (int i = 0; i < n; i++) s += a[i]*b[i]; return s; }

static int krylov(const AbdParams* P, const BSR* A, const double* b, double* x, int* iters) {
    int nb = A->nb, n = 12 * nb;
    if (nb <= 0) { *iters = 0; return 0; }
    double* Dinv = (double*)xalloc(sizeof(double) * 144 * nb);
    for (int r = 0; r < nb; r++) {
        const double* D = NULL;
        for (int k = A->rowptr[r]; k < A->rowptr[r+1]; k++) if (A->col[k] == r) D = A->val + 144*k;
        if (!D || inv12(D, Dinv + 144*r)) { memset(Dinv + 144*r, 0, sizeof(double)*144); for (int i = 0; i < 12; i++) Dinv[144*r + 13*i] = 1.0; }
    }
    double *r = xalloc(8*n), *p = xalloc(8*n), *v = xalloc(8*n), *y = xalloc(8*n), *s = xalloc(8*n), *z = xalloc(8*n), *t = xalloc(8*n), *rh = xalloc(8*n);
    memset(x, 0, 8*(size_t)n);
    memcpy(r, b, 8*(size_t)n);
    double bn = sqrt(vdot(n, b, b)), tol = P->lin_tol * bn;
    int it = 0, status = 0;
    if (bn == 0) { *iters = 0; goto done; }
    if (P->linear_solver == ABD_SOLVER_PCG) {
        precond(nb, Dinv, r, z); memcpy(p, z, 8*n);
        double rz = vdot(n, r, z);
        for (it = 0; it < P->lin_max_iter; it++) {
            bsr_mv(A, p, v);
            double pAp = vdot(n, p, v);
            if (!(pAp > 0)) { status = 1; break; }
            double al = rz / pAp;
            for (int i = 0; i < n; i++) { x[i] += al * p[i]; r[i] -= al * v[i]; }
            if (sqrt(vdot(n, r, r)) <= tol) { it++; break; }
            precond(nb, Dinv, r, z);
            double rz2 = vdot(n, r, z), be = rz2 / rz; rz = rz2;
            for (int i = 0; i < n; i++) p[i] = z[i] + be * p[i];
        }
    } else {
        memcpy(rh, r, 8*n);
        double rho = 1, al = 1, om = 1;
        for (it = 0; it < P->lin_max_iter; it++) {
            double rho2 = vdot(n, rh, r);
            if (rho2 == 0) { status = 1; break; }
            double be = (rho2 / rho) * (al / om); rho = rho2;
            for (int i = 0; i < n; i++) p[i] = r[i] + be * (p[i] - om * v[i]);
            precond(nb, Dinv, p, y);
            bsr_mv(A, y, v);
            double rv = vdot(n, rh, v);
            if (rv == 0) { status = 1; break; }
            al = rho / rv;
            for (int i = 0; i < n; i++) { x[i] += al * y[i]; s[i] = r[i] - al * v[i]; }
            if (sqrt(vdot(n, s, s)) <= tol) { memcpy(r, s, 8*n); it++; break; }
            precond(nb, Dinv, s, z);
            bsr_mv(A, z, t);
            double tt = vdot(n, t, t);
            if (tt == 0) { status = 1; break; }
            om = vdot(n, t, s) / tt;
            for (int i = 0; i < n; i++) { x[i] += om * z[i]; r[i] = s[i] - om * t[i]; }
            if (sqrt(vdot(n, r, r)) <= tol) { it++; break; }
            if (om == 0) { status = 1; break; }
        }
    }
    *iters = it;
done:
    free(Dinv); free(r); free(p); free(v); free(y); free(s); free(z); free(t); free(rh);
    return status;
}

/* Direct solve (abd.py:637-654 factors the assembled matrix): dense
 * Cholesky when the Hessian is PSD-projected, else (or when a pivot is not
 * positive) LU with partial pivoting. */
static int dense_factor_solve(const AbdParams* P, const BSR* A, const double* b, double* x) {
    int nb = A->nb; long n = 12L * nb;
    double* M = (double*)calloc((size_t)(n * n), sizeof(double));
    for (int r = 0; r < nb; r++) for (int k = A->rowptr[r]; k < A->rowptr[r+1]; k++) {
        int c = A->col[k];
        for (int i = 0; i < 12; i++) for (int j = 0; j < 12; j++)
            M[(12L*r + i) * n + 12L*c + j] = A->val[144*k + 12*i + j];
    }
    memcpy(x, b, sizeof(double) * n);
    int ok = 0;
    if (P->hess_mode == ABD_HESS_PROJECTED) {
        double* L = (double*)malloc(sizeof(double) * n * n);
        memcpy(L, M, sizeof(double) * n * n);
        ok = 1;
        for (long j = 0; j < n && ok; j++) {
            double d = L[j*n + j];
            for (long k = 0; k < j; k++) d -= L[j*n + k] * L[j*n + k];
            if (!(d > 0)) { ok = 0; break; }
            d = sqrt(d); L[j*n + j] = d;
            #pragma omp parallel for num_threads(g_threads) schedule(static)
            for (long i = j + 1; i < n; i++) {
                double v = L[i*n + j];
                for (long k = 0; k < j; k++) v -= L[i*n + k] * L[j*n + k];
                L[i*n + j] = v / d;
            }
        }
        if (ok) {
            for (long i = 0; i < n; i++) { double v = x[i]; for (long k = 0; k < i; k++) v -= L[i*n + k] * x[k]; x[i] = v / L[i*n + i]; }
            for (long i = n - 1; i >= 0; i--) { double v = x[i]; for (long k = i + 1; k < n; k++) v -= L[k*n + i] * x[k]; x[i] = v / L[i*n + i]; }
        }
        free(L);
        memcpy(x, ok ? x : b, sizeof(double) * n);
        if (!ok) memcpy(x, b, sizeof(double) * n);
    }
    if (!ok) {
        int* piv = (int*)malloc(sizeof(int) * n);
        for (long j = 0; j < n; j++) {
            long p = j; for (long i = j + 1; i < n; i++) if (fabs(M[i*n + j]) > fabs(M[p*n + j])) p = i;
            piv[j] = (int)p;
            if (p != j) { for (long k = 0; k < n; k++) { double t = M[j*n + k]; M[j*n + k] = M[p*n + k]; M[p*n + k] = t; }
                          double t = x[j]; x[j] = x[p]; x[p] = t; }
            double d = M[j*n + j];
            if (d == 0.0) continue;
            #pragma omp parallel for num_threads(g_threads) schedule(static)
            for (long i = j + 1; i < n; i++) {
                double f = M[i*n + j] / d;
                M[i*n + j] = f;
                if (f != 0.0) for (long k = j + 1; k < n; k++) M[i*n + k] -= f * M[j*n + k];
            }
            for (long i = j + 1; i < n; i++) x[i] -= M[i*n + j] * x[j];
        }
        for (long i = n - 1; i >= 0; i--) { double v = x[i]; for (long k = i + 1; k < n; k++) v -= M[i*n + k] * x[k]; x[i] = M[i*n + i] != 0 ? v / M[i*n + i] : 0; }
        free(piv);
    }
    free(M);
    return 0;
}

static int use_direct(const OracleWorld* w) {
    int k = w->P.linear_solver;
    if (k == 2) return 1;
    if (k != 3) return 0;
    long long tot = 0;
    for (int i = 0; i < w->ns; i++) { long long n = 12LL * w->s[i].nb; tot += n * n; }
    return w->ns <= 64 && tot * 8 <= (4LL << 30);
}
static int solve_system(const OracleWorld* w, const BSR* A, const double* b, double* x, int* iters) {
    if (use_direct(w)) { *iters = 1; return dense_factor_solve(&w->P, A, b, x); }
    AbdParams P = w->P;
    if (P.linear_solver == 3) P.linear_solver = P.hess_mode == ABD_HESS_PROJECTED ? ABD_SOLVER_PCG : ABD_SOLVER_BICGSTAB;
    return krylov(&P, A, b, x, iters);
}

int oracle_solve(OracleWorld* w, double* du, int* iters) {
    int tot = 0;
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        Assembly as; assemble_scene(w, S, &as);
        int it = 0; solve_system(w, &as.A, as.g, du, &it);
        tot += it; du += 12 * S->nb;
        free(as.g); bsr_free(&as.A);
    }
    *iters = tot;
    return 0;
}

/* ------------------------------------------------------------------ */
/* CCD over a step x -> x + p for one scene                             */
/* ------------------------------------------------------------------ */
typedef struct { const OracleWorld* w; const OScene* S; const double* x; const double* p; double toi; } CcdCtx;
static void ccd_ee_cb(void* c, CandVec* out, int i, int j) {
    CcdCtx* d = (CcdCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* ea = S->edges + 2*i; const int* eb = S->edges + 2*j;
    if (ea[0] == eb[0] || ea[0] == eb[1] || ea[1] == eb[0] || ea[1] == eb[1]) return;
    if (!P->self_contact && S->vbody[ea[0]] == S->vbody[eb[0]]) return;
    int v[4] = {ea[0], ea[1], eb[0], eb[1]};
    double x[12], p[12];
    for (int k = 0; k < 4; k++) { memcpy(x + 3*k, d->x + 3*v[k], 24); memcpy(p + 3*k, d->p + 3*v[k], 24); }
    double t;
    if (oracle_accd(0, x, p, P->ccd_scale, 1.0, &t)) cv_push(out, 0, (int)(t * 1e9), 0);
}
static void ccd_pt_cb(void* c, CandVec* out, int pi, int ti) {
    CcdCtx* d = (CcdCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* tr = S->tris + 3*ti;
    if (pi == tr[0] || pi == tr[1] || pi == tr[2]) return;
    if (!P->self_contact && S->vbody[pi] == S->vbody[tr[0]]) return;
    int v[4] = {pi, tr[0], tr[1], tr[2]};
    double x[12], p[12];
    for (int k = 0; k < 4; k++) { memcpy(x + 3*k, d->x + 3*v[k], 24); memcpy(p + 3*k, d->p + 3*v[k], 24); }
    double t;
    if (oracle_accd(1, x, p, P->ccd_scale, 1.0, &t)) cv_push(out, 0, (int)(t * 1e9), 0);
}
/* returns the largest conservative step fraction in [0,1] */
static double scene_ccd(const OracleWorld* w, const OScene* S, const double* x, const double* p) {
    const AbdParams* P = &w->P;
    double toi = 1.0;
    CcdCtx ctx = {w, S, x, p, 1.0};
    CandVec hits = {0};
    if (P->contact_ee && S->ne > 1) {
        Box* bx = (Box*)xalloc(sizeof(Box) * S->ne);
        for (int e = 0; e < S->ne; e++) {
            int a = S->edges[2*e], b = S->edges[2*e+1];
            for (int k = 0; k < 3; k++) {
                double v0 = x[3*a+k], v1 = x[3*b+k], v2 = x[3*a+k] + p[3*a+k], v3 = x[3*b+k] + p[3*b+k];
                bx[e].lo[k] = fmin(fmin(v0, v1), fmin(v2, v3)) - 1e-9; bx[e].hi[k] = fmax(fmax(v0, v1), fmax(v2, v3)) + 1e-9;
            }
            bx[e].id = e; bx[e].set = 0;
        }
        sweep(bx, S->ne, 0, ccd_ee_cb, &ctx, &hits);
        free(bx);
    }
    if (P->contact_pt && S->nt > 0) {
        Box* bx = (Box*)xalloc(sizeof(Box) * (S->nv + S->nt));
        for (int v = 0; v < S->nv; v++) {
            for (int k = 0; k < 3; k++) {
                double a = x[3*v+k], b = a + p[3*v+k];
                bx[v].lo[k] = fmin(a, b) - 1e-9; bx[v].hi[k] = fmax(a, b) + 1e-9;
            }
            bx[v].id = v; bx[v].set = 0;
        }
        for (int t = 0; t < S->nt; t++) {
            Box* B = &bx[S->nv + t];
            for (int k = 0; k < 3; k++) {
                double lo = 1e300, hi = -1e300;
                for (int q = 0; q < 3; q++) { int v = S->tris[3*t+q]; double a = x[3*v+k], b = a + p[3*v+k]; lo = fmin(lo, fmin(a, b)); hi = fmax(hi, fmax(a, b)); }
                B->lo[k] = lo - 1e-9; B->hi[k] = hi + 1e-9;
            }
            B->id = t; B->set = 1;
        }
        sweep(bx, S->nv + S->nt, 1, ccd_pt_cb, &ctx, &hits);
        free(bx);
    }
    for (int k = 0; k < hits.n; k++) { double t = hits.v[k].a * 1e-9; if (t < toi) toi = t; }
    free(hits.v);
    for (int pl = 0; pl < S->np; pl++) {
        const double* n = S->planes + 4*pl;
        for (int v = 0; v < S->nv; v++) {
            double d = dot3(n, x + 3*v) - n[3], vn = dot3(n, p + 3*v);
            if (vn < 0) { double t = (1 - P->ccd_scale) * d / (-vn); if (t < toi) toi = t < 0 ? 0 : t; }
        }
    }
    return toi;
}

/* ------------------------------------------------------------------ */
/* Newton step (abd.py:674-702) with the reference line search          */
/* (gauss_newton.py:98-115)                                              */
/* ------------------------------------------------------------------ */
static void apply_du(OScene* S, const double* backup, const double* du, double alpha) {
    /* abd.py:768-785: nxt.c -= alpha du[4i]; nxt.q rows -= alpha du[4i+1..3] */
    for (int b = 0; b < S->nb; b++) {
        double* nx = S->st + 48*b + ST_NXT; const double* bk = backup + 48*b + ST_NXT;
        for (int k = 0; k < 12; k++) nx[k] = fma(-alpha, du[12*b + k], bk[k]);
    }
}
static void vertex_disp(const OScene* S, const double* du, double scale, double* p) {
    for (int v = 0; v < S->nv; v++) {
        const double* d = du + 12 * S->vbody[v]; const double* xb = S->xbar + 3*v;
        for (int k = 0; k < 3; k++) p[3*v+k] = scale * (d[k] + xb[0]*d[3+k] + xb[1]*d[6+k] + xb[2]*d[9+k]);
    }
}

static void prof_push(OScene* S, double res, double alpha) {
    if (S->prof_n == S->prof_cap) {
        S->prof_cap = S->prof_cap ? 2 * S->prof_cap : 256;
        S->prof_res = realloc(S->prof_res, sizeof(double) * S->prof_cap);
        S->prof_alpha = realloc(S->prof_alpha, sizeof(double) * S->prof_cap);
    }
    S->prof_res[S->prof_n] = res; S->prof_alpha[S->prof_n] = alpha; S->prof_n++;
}

/* ------------------------------------------------------------------ */
/* Contact groups of the line search (AbdParams.ls_groups; no reference */
/* counterpart).  Bodies whose boxes swept over x .. x + p, rounded      */
/* outward to float and padded by half the candidate distance, overlap  */
/* are joined (transitively); a group is named by its smallest body.    */
/* ------------------------------------------------------------------ */
static float f_rd(double d) { float f = (float)d; if ((double)f > d) f = nextafterf(f, -INFINITY); return f; }
static float f_ru(double d) { float f = (float)d; if ((double)f < d) f = nextafterf(f, INFINITY); return f; }
/* float a - b rounded down / a + b rounded up (the exact result is a double
 * when the exponents of a and b are within 28 of each other) */
static float fsub_rd(float a, float b) { return f_rd((double)a - (double)b); }
static float fadd_ru(float a, float b) { return f_ru((double)a + (double)b); }
static int grp_root(int* parent, int x) {
    int r = x;
    while (parent[r] != r) r = parent[r];
    while (parent[x] != r) { int n = parent[x]; parent[x] = r; x = n; }
    return r;
}
/* gid[b] = smallest body index of b's group */
static void contact_groups(const OracleWorld* w, const OScene* S, const double* x, const double* p, int* gid) {
    int nb = S->nb;
    double lim = w->P.cand_dist * (1.0 + 1e-6) + 1e-7;
    float pad = (float)(0.5 * lim);
    float* box = (float*)xalloc(sizeof(float) * 6 * nb);
    for (int b = 0; b < nb; b++) for (int k = 0; k < 3; k++) { box[6*b+k] = 3e38f; box[6*b+3+k] = -3e38f; }
    for (int v = 0; v < S->nv; v++) {
        int b = S->vbody[v];
        for (int k = 0; k < 3; k++) {
            double a = x[3*v+k], e = a + p[3*v+k];
            float lo = fsub_rd(f_rd(fmin(a, e)), pad), hi = fadd_ru(f_ru(fmax(a, e)), pad);
            box[6*b+k] = fminf(box[6*b+k], lo); box[6*b+3+k] = fmaxf(box[6*b+3+k], hi);
        }
    }
    for (int b = 0; b < nb; b++) gid[b] = b;
    for (int a = 0; a < nb; a++) {
        const float* A = box + 6*a;
        for (int b = a + 1; b < nb; b++) {
            const float* B = box + 6*b;
            if (A[0] > B[3] || A[3] < B[0] || A[1] > B[4] || A[4] < B[1] || A[2] > B[5] || A[5] < B[2]) continue;
            int ra = grp_root(gid, a), rb = grp_root(gid, b);
            if (ra == rb) continue;
            if (ra < rb) gid[rb] = ra; else gid[ra] = rb;
        }
    }
    for (int b = 0; b < nb; b++) gid[b] = grp_root(gid, b);
    free(box);
}
/* energy and its FP64 error scale per group (slot = group root) */
static void group_energy(const OracleWorld* w, OScene* S, const double* st, const int* gid, double* e, double* noise) {
    int nb = S->nb;
    for (int b = 0; b < nb; b++) { e[b] = 0; noise[b] = 0; }
    for (int b = 0; b < nb; b++) { double n_; e[gid[b]] += body_energy(w, S, st, b, &n_); noise[gid[b]] += n_; }
    transform(S, st, S->x);
    detect(w, S, S->x, w->P.cand_dist);
    double* ec = (double*)xalloc(sizeof(double) * 2 * (S->nc + 1));
    #pragma omp parallel for num_threads(g_threads) schedule(dynamic, 64)
    for (int c = 0; c < S->nc; c++) { CEval ce; eval_contact(w, S, S->x, &S->cand[c], 0, &ce); ec[2*c] = ce.e; ec[2*c+1] = ce.noise; }
    for (int c = 0; c < S->nc; c++) {
        const Cand* C = &S->cand[c];
        int v0 = C->kind == ABD_CONTACT_EE ? S->edges[2*C->a] : C->a;
        int g = gid[S->vbody[v0]];
        e[g] += ec[2*c]; noise[g] += ec[2*c+1];
    }
    free(ec);
}
/* CCD bound per group over x -> x + p */
typedef struct { const OracleWorld* w; const OScene* S; const double* x; const double* p; const int* gid; } GCcdCtx;
/* a hit is kept as (group, the bits of t) in the sweep's per-thread list */
static void gccd_pair(GCcdCtx* d, CandVec* out, int kind, const int v[4]) {
    const AbdParams* P = &d->w->P;
    double x[12], p[12];
    for (int k = 0; k < 4; k++) { memcpy(x + 3*k, d->x + 3*v[k], 24); memcpy(p + 3*k, d->p + 3*v[k], 24); }
    double t;
    if (oracle_accd(kind, x, p, P->ccd_scale, 1.0, &t)) {
        int bits[2]; memcpy(bits, &t, sizeof t);
        cv_push(out, d->gid[d->S->vbody[v[0]]], bits[0], bits[1]);
    }
}
static void gccd_ee_cb(void* c, CandVec* out, int i, int j) {
    GCcdCtx* d = (GCcdCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* ea = S->edges + 2*i; const int* eb = S->edges + 2*j;
    if (ea[0] == eb[0] || ea[0] == eb[1] || ea[1] == eb[0] || ea[1] == eb[1]) return;
    if (!P->self_contact && S->vbody[ea[0]] == S->vbody[eb[0]]) return;
    int v[4] = {ea[0], ea[1], eb[0], eb[1]};
    gccd_pair(d, out, 0, v);
}
static void gccd_pt_cb(void* c, CandVec* out, int pi, int ti) {
    GCcdCtx* d = (GCcdCtx*)c; const OScene* S = d->S; const AbdParams* P = &d->w->P;
    const int* tr = S->tris + 3*ti;
    if (pi == tr[0] || pi == tr[1] || pi == tr[2]) return;
    if (!P->self_contact && S->vbody[pi] == S->vbody[tr[0]]) return;
    int v[4] = {pi, tr[0], tr[1], tr[2]};
    gccd_pair(d, out, 1, v);
}
static void group_ccd(const OracleWorld* w, const OScene* S, const double* x, const double* p, const int* gid, double* toi) {
    const AbdParams* P = &w->P;
    for (int b = 0; b < S->nb; b++) toi[b] = 1.0;
    GCcdCtx ctx = {w, S, x, p, gid};
    CandVec hits = {0};
    if (P->contact_ee && S->ne > 1) {
        Box* bx = (Box*)xalloc(sizeof(Box) * S->ne);
        for (int e = 0; e < S->ne; e++) {
            int a = S->edges[2*e], b = S->edges[2*e+1];
            for (int k = 0; k < 3; k++) {
                double v0 = x[3*a+k], v1 = x[3*b+k], v2 = x[3*a+k] + p[3*a+k], v3 = x[3*b+k] + p[3*b+k];
                bx[e].lo[k] = fmin(fmin(v0, v1), fmin(v2, v3)) - 1e-9; bx[e].hi[k] = fmax(fmax(v0, v1), fmax(v2, v3)) + 1e-9;
            }
            bx[e].id = e; bx[e].set = 0;
        }
        sweep(bx, S->ne, 0, gccd_ee_cb, &ctx, &hits);
        free(bx);
    }
    if (P->contact_pt && S->nt > 0) {
        Box* bx = (Box*)xalloc(sizeof(Box) * (S->nv + S->nt));
        for (int v = 0; v < S->nv; v++) {
            for (int k = 0; k < 3; k++) {
                double a = x[3*v+k], b = a + p[3*v+k];
                bx[v].lo[k] = fmin(a, b) - 1e-9; bx[v].hi[k] = fmax(a, b) + 1e-9;
            }
            bx[v].id = v; bx[v].set = 0;
        }
        for (int t = 0; t < S->nt; t++) {
            Box* B = &bx[S->nv + t];
            for (int k = 0; k < 3; k++) {
                double lo = 1e300, hi = -1e300;
                for (int q = 0; q < 3; q++) { int v = S->tris[3*t+q]; double a = x[3*v+k], b = a + p[3*v+k]; lo = fmin(lo, fmin(a, b)); hi = fmax(hi, fmax(a, b)); }
                B->lo[k] = lo - 1e-9; B->hi[k] = hi + 1e-9;
            }
            B->id = t; B->set = 1;
        }
        sweep(bx, S->nv + S->nt, 1, gccd_pt_cb, &ctx, &hits);
        free(bx);
    }
    for (int k = 0; k < hits.n; k++) {
        double t; int bits[2] = {hits.v[k].a, hits.v[k].b}; memcpy(&t, bits, sizeof t);
        if (t < toi[hits.v[k].kind]) toi[hits.v[k].kind] = t;
    }
    free(hits.v);
    for (int pl = 0; pl < S->np; pl++) {
        const double* n = S->planes + 4*pl;
        for (int v = 0; v < S->nv; v++) {
            double d = dot3(n, x + 3*v) - n[3], vn = dot3(n, p + 3*v);
            if (vn < 0) {
                double t = (1 - P->ccd_scale) * d / (-vn);
                int g = gid[S->vbody[v]];
                if (t < toi[g]) toi[g] = t < 0 ? 0 : t;
            }
        }
    }
}
/* the line search with one step length per group: every group backs off
 * on its own energy (gauss_newton.py:98-115 per group); returns the
 * smallest accepted step, *stalled when every group gave up below
 * ABD_LS_STALL_ALPHA, *min_toi the smallest CCD bound */
static double group_line_search(const OracleWorld* w, OScene* S, const double* backup, const double* du, double* pv,
                                int* stalled, double* min_toi, int* trials) {
    const AbdParams* P = &w->P;
    int nb = S->nb;
    int* gid = (int*)xalloc(sizeof(int) * nb);
    double* d = (double*)xalloc(sizeof(double) * 6 * nb);
    double *E0 = d, *N0 = d + nb, *E1 = d + 2*nb, *N1 = d + 3*nb, *al = d + 4*nb, *toi = d + 5*nb;
    int* acc = (int*)xalloc(sizeof(int) * 2 * nb);
    int* stl = acc + nb;
    transform(S, S->st, S->x);
    vertex_disp(S, du, -1.0, pv);
    contact_groups(w, S, S->x, pv, gid);
    group_energy(w, S, S->st, gid, E0, N0);
    if (P->ccd) group_ccd(w, S, S->x, pv, gid, toi);
    *min_toi = 1.0;
    for (int g = 0; g < nb; g++) {
        acc[g] = gid[g] != g; stl[g] = 0;
        al[g] = P->ccd ? fmin(1.0, toi[g]) : 1.0;
        if (!acc[g] && P->ccd && toi[g] < *min_toi) *min_toi = toi[g];
    }
    for (;;) {
        for (int b = 0; b < nb; b++) {
            int g = gid[b];
            if (acc[g]) continue;
            double* nx = S->st + 48*b + ST_NXT; const double* bk = backup + 48*b + ST_NXT;
            for (int k = 0; k < 12; k++) nx[k] = fma(-al[g], du[12*b + k], bk[k]);
        }
        group_energy(w, S, S->st, gid, E1, N1);
        (*trials)++;
        int pending = 0;
        for (int g = 0; g < nb; g++) {
            if (acc[g]) continue;
            if (E1[g] < E0[g] || E1[g] - E0[g] <= N0[g] + N1[g]) acc[g] = 1;
            else if (al[g] * 0.5 < P->ls_min_alpha) { acc[g] = 1; stl[g] = al[g] < ABD_LS_STALL_ALPHA; }
            else { al[g] *= 0.5; pending++; }
        }
        if (!pending) break;
    }
    double amin = 1.0; int nact = 0, nst = 0;
    for (int g = 0; g < nb; g++) {
        if (gid[g] != g) continue;
        nact++; nst += stl[g];
        if (al[g] < amin) amin = al[g];
    }
    *stalled = nact > 0 && nst == nact;
    free(gid); free(d); free(acc);
    return amin;
}

static void scene_step(const OracleWorld* w, OScene* S, AbdStepStats* st) {
    const AbdParams* P = &w->P;
    int nb = S->nb;
    double dt = P->dt;
    double* backup = (double*)xalloc(sizeof(double) * 48 * nb);
    double* du = (double*)xalloc(sizeof(double) * 12 * nb);
    double* pv = (double*)xalloc(sizeof(double) * 3 * S->nv);
    if (P->warm_start == 2) {
        /* inertial prediction as the initial increment */
        for (int b = 0; b < nb; b++) {
            const double* now = S->st + 48*b + ST_NOW;
            for (int k = 0; k < 3; k++) S->ws[12*b + k] = dt * now[ST_V+k] + dt * dt * P->gravity[k];
            for (int k = 0; k < 9; k++) S->ws[12*b + 3 + k] = dt * now[ST_QD+k];
        }
        S->has_ws = 1;
    }
    if (S->has_ws) {
        memcpy(backup, S->st, sizeof(double) * 48 * nb);
        for (int i = 0; i < 12 * nb; i++) du[i] = -S->ws[i];
        for (int b = 0; b < nb; b++) if (!dynamic(S, b)) memset(du + 12*b, 0, 96);
        double a = 1.0;
        if (P->ccd) { transform(S, S->st, S->x); vertex_disp(S, du, -1.0, pv); a = scene_ccd(w, S, S->x, pv); }
        /* keep the start only where it lowers the energy below that of now
         * (nxt == now here): halve at most 7 times, else start from now */
        double E0 = scene_energy(w, S, S->st, NULL);
        int ok = 0;
        for (int t = 0; t < 8; t++) {
            apply_du(S, backup, du, a);
            double E1 = scene_energy(w, S, S->st, NULL);
            if (E1 < E0) { ok = 1; break; }
            a *= 0.5;
        }
        if (!ok) apply_du(S, backup, du, 0.0);
        S->has_ws = 0;
    }
    int it = 0;
    double res = 0;
    for (;;) {
        Assembly as; assemble_scene(w, S, &as);
        res = sqrt(vdot(12 * nb, as.g, as.g));
        int li = 0; solve_system(w, &as.A, as.g, du, &li);
        st->lin_iters += li; st->n_pairs = S->nc; st->n_active = as.n_active;
        free(as.g); bsr_free(&as.A);
        /* line search */
        memcpy(backup, S->st, sizeof(double) * 48 * nb);
        if (P->ls_groups) {
            int stalled = 0, trials = 0;
            double mt = 1.0;
            double alpha = group_line_search(w, S, backup, du, pv, &stalled, &mt, &trials);
            st->ls_trials += trials;
            if (mt < st->min_toi) st->min_toi = mt;
            it++;
            prof_push(S, res, alpha);
            if (res < P->newton_tol || it >= P->newton_max_iter || stalled) break;
            continue;
        }
        double N0, N1;
        double E0 = scene_energy(w, S, S->st, &N0);
        double alpha = 1.0;
        if (P->ccd) {
            transform(S, S->st, S->x);
            vertex_disp(S, du, -1.0, pv);
            double toi = scene_ccd(w, S, S->x, pv);
            if (toi < st->min_toi) st->min_toi = toi;
            if (toi < alpha) alpha = toi;
        }
        int stalled = 0;
        for (;;) {
            apply_du(S, backup, du, alpha);
            double E1 = scene_energy(w, S, S->st, &N1);
            st->ls_trials++;
            /* a change within the FP64 evaluation error of both energies is no increase */
            if (E1 < E0 || E1 - E0 <= N0 + N1) break;
            else if (alpha * 0.5 < P->ls_min_alpha) { stalled = alpha < ABD_LS_STALL_ALPHA; break; }
            else alpha *= 0.5;
        }
        it++;
        prof_push(S, res, alpha);
        /* a search that gave up at a negligible step left the state where it
         * was: the next iteration would find the same direction */
        if (res < P->newton_tol || it >= P->newton_max_iter || stalled) break;
    }
    if (!(res < P->newton_tol)) st->unconverged++;
    st->newton_iters += it;
    if (it > st->max_newton_iters) st->max_newton_iters = it;
    st->last_residual = fmax(st->last_residual, res);
    if (S->prof_steps % 256 == 0) S->prof_iters = realloc(S->prof_iters, sizeof(int) * (S->prof_steps + 256));
    S->prof_iters[S->prof_steps++] = it;
    /* abd.py:574-581 forward_states */
    for (int b = 0; b < nb; b++) {
        double* s = S->st + 48*b;
        for (int k = 0; k < 3; k++) s[ST_NXT+ST_V+k] = (s[ST_NXT+ST_C+k] - s[ST_NOW+ST_C+k]) / dt;
        for (int k = 0; k < 9; k++) s[ST_NXT+ST_QD+k] = (s[ST_NXT+ST_Q+k] - s[ST_NOW+ST_Q+k]) / dt;
        memcpy(s + ST_NOW, s + ST_NXT, sizeof(double) * 24);
    }
    free(backup); free(du); free(pv);
}

int oracle_step(OracleWorld* w, int n_steps, AbdStepStats* st) {
    AbdStepStats loc; memset(&loc, 0, sizeof loc); loc.min_toi = 1.0;
    for (int i = 0; i < w->ns; i++) { w->s[i].prof_n = 0; w->s[i].prof_steps = 0; }
    g_ccd_cap_hit = 0;
    for (int s = 0; s < n_steps; s++) {
        for (int i = 0; i < w->ns; i++) scene_step(w, &w->s[i], &loc);
        loc.steps++;
    }
    if (st) *st = loc;
    return g_ccd_cap_hit ? ABD_ERR_CCD_CAP : 0;
}

int oracle_get_profile(OracleWorld* w, int scene, double* res, double* alpha, int* ips, int cap, int* n) {
    if (scene < 0 || scene >= w->ns) return ABD_ERR_INVALID_ARG;
    OScene* S = &w->s[scene];
    int m = S->prof_n < cap ? S->prof_n : cap;
    memcpy(res, S->prof_res, sizeof(double) * m); memcpy(alpha, S->prof_alpha, sizeof(double) * m);
    if (ips) for (int i = 0; i < S->prof_steps && i < cap; i++) ips[i] = S->prof_iters[i];
    *n = m;
    return 0;
}

int oracle_set_warm_start(OracleWorld* w, const float* dq, int nb) {
    int off = 0;
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        if (off + S->nb > nb) return ABD_ERR_INVALID_ARG;
        for (int k = 0; k < 12 * S->nb; k++) S->ws[k] = dq[12*off + k];
        S->has_ws = 1; off += S->nb;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Edge-triangle intersections between different bodies (orientation   */
/* predicates in FP64).                                                   */
/* ------------------------------------------------------------------ */
static double orient3(const double* a, const double* b, const double* c, const double* d) {
    double u[3], v[3], wv[3], n[3]; sub3(b, a, u); sub3(c, a, v); sub3(d, a, wv); cross3(u, v, n); return dot3(n, wv);
}
static int seg_tri(const double* p, const double* q, const double* a, const double* b, const double* c) {
    double o1 = orient3(a, b, c, p), o2 = orient3(a, b, c, q);
    if ((o1 > 0 && o2 > 0) || (o1 < 0 && o2 < 0) || (o1 == 0 && o2 == 0)) return 0;
    double s1 = orient3(p, q, a, b), s2 = orient3(p, q, b, c), s3 = orient3(p, q, c, a);
    return (s1 > 0 && s2 > 0 && s3 > 0) || (s1 < 0 && s2 < 0 && s3 < 0);
}
typedef struct { const OScene* S; const double* x; } IxCtx;
static void ix_cb(void* c, CandVec* out, int e, int t) {
    IxCtx* d = (IxCtx*)c; const OScene* S = d->S;
    int a = S->edges[2*e], b = S->edges[2*e+1];
    const int* tr = S->tris + 3*t;
    if (S->vbody[a] == S->vbody[tr[0]]) return;
    if (seg_tri(d->x + 3*a, d->x + 3*b, d->x + 3*tr[0], d->x + 3*tr[1], d->x + 3*tr[2])) cv_push(out, 0, e, t);
}
int oracle_count_intersections(OracleWorld* w, int* count) {
    int tot = 0;
    for (int i = 0; i < w->ns; i++) {
        OScene* S = &w->s[i];
        if (S->nt == 0 || S->ne == 0) continue;
        transform(S, S->st, S->x);
        Box* bx = (Box*)xalloc(sizeof(Box) * (S->ne + S->nt));
        for (int e = 0; e < S->ne; e++) for (int k = 0; k < 3; k++) {
            double a = S->x[3*S->edges[2*e]+k], b = S->x[3*S->edges[2*e+1]+k];
            bx[e].lo[k] = fmin(a, b); bx[e].hi[k] = fmax(a, b); bx[e].id = e; bx[e].set = 0;
        }
        for (int t = 0; t < S->nt; t++) {
            Box* B = &bx[S->ne + t];
            for (int k = 0; k < 3; k++) {
                double a = S->x[3*S->tris[3*t]+k], b = S->x[3*S->tris[3*t+1]+k], c = S->x[3*S->tris[3*t+2]+k];
                B->lo[k] = fmin(a, fmin(b, c)); B->hi[k] = fmax(a, fmax(b, c));
            }
            B->id = t; B->set = 1;
        }
        CandVec hits = {0}; IxCtx ctx = {S, S->x};
        sweep(bx, S->ne + S->nt, 1, ix_cb, &ctx, &hits);
        tot += hits.n; free(hits.v); free(bx);
    }
    *count = tot;
    return 0;
}
