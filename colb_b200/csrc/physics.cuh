// physics.cuh — per-primitive device math of the ABD step.
//
//  barrier ............. barrier.py:6-65 (cubic / quadratic / log in x = d^2)
//  orthogonality ....... ortho.py:9-41
//  segment closest pts . Ericson, Real-Time Collision Detection §5.1.9, as
//                        called by contact.py:166 and abd.py:190 (float32)
//  squared distances ... IPC (Li et al. 2020) point-point, point-line,
//                        line-line and point-plane, with gradient and Hessian
//  PSD projection ...... cyclic Jacobi eigen-decomposition (abd.py:247)
//  triangle region ..... Ericson §5.1.5
//  additive CCD ........ Li, Kaufman, Jiang 2021 (C-IPC) Alg. 1
#pragma once
#include "common.cuh"

// ---------------------------------------------------------------- barrier
DV void barrier3(int kind, double x, double xh, double& b0, double& b1, double& b2) {
    b0 = b1 = b2 = 0.0;
    if (!(x < xh)) return;
    double t = x - xh;
    if (kind == ABD_BARRIER_CUBIC) {
        b0 = -t * t * t; b1 = -3.0 * t * t; b2 = -6.0 * t;
    } else if (kind == ABD_BARRIER_QUADRATIC) {
        b0 = t * t; b1 = 2.0 * t; b2 = 2.0;
    } else {
        double l = log(x / xh), ih = 1.0 / (xh * xh);
        b0 = -t * t * l * ih;
        b1 = (xh - x) * (2.0 * l + t / x) * ih;
        b2 = -(2.0 * l + t / x + t * (2.0 / x + xh / (x * x))) * ih;
    }
}

// ---------------------------------------------------------- orthogonality
// q: 9 doubles, rows a_i = q[3i..3i+2]
DV double ortho_energy(const double* q, double k) {
    double e = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double t = q[3*i] * q[3*j] + q[3*i+1] * q[3*j+1] + q[3*i+2] * q[3*j+2] - (i == j ? 1.0 : 0.0);
            e += t * t;
        }
    return e * k;
}
// Scale of the FP64 evaluation error of ortho_energy (in units of the
// rounding unit): k sum_ij (t_ij^2 + 4 |t_ij| |a_i| |a_j|), t_ij = a_i.a_j - delta_ij
DV double ortho_noise(const double* q, double k) {
    double na[3], e = 0;
#pragma unroll
    for (int i = 0; i < 3; i++) na[i] = sqrt(q[3*i] * q[3*i] + q[3*i+1] * q[3*i+1] + q[3*i+2] * q[3*i+2]);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double t = q[3*i] * q[3*j] + q[3*i+1] * q[3*j+1] + q[3*i+2] * q[3*j+2] - (i == j ? 1.0 : 0.0);
            e += t * t + 4.0 * fabs(t) * na[i] * na[j];
        }
    return e * k;
}
// Scale of the FP64 evaluation error of one barrier term sc*b(x), x = d^2,
// over a stencil whose coordinates are at most L in magnitude: the term
// itself plus the barrier slope times the error of x from rounded positions
// (mult scales FP32 distances)
DV double contact_noise(double sc, double b0, double b1, double x, double L, double mult) {
    return sc * (fabs(b0) + fabs(b1) * 8.0 * sqrt(fabs(x)) * L * mult);
}
DV void ortho_grad(const double* q, double k, double* g) {
#pragma unroll
    for (int i = 0; i < 3; i++) {
        double gi0 = -q[3*i], gi1 = -q[3*i+1], gi2 = -q[3*i+2];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double d = q[3*i] * q[3*j] + q[3*i+1] * q[3*j+1] + q[3*i+2] * q[3*j+2];
            gi0 += d * q[3*j]; gi1 += d * q[3*j+1]; gi2 += d * q[3*j+2];
        }
        g[3*i] = gi0 * 4.0 * k; g[3*i+1] = gi1 * 4.0 * k; g[3*i+2] = gi2 * 4.0 * k;
    }
}
// 3x3 block (i,j) of the ortho Hessian, entry (r,c)
DV double ortho_hess(const double* q, double k, int i, int j, int r, int c) {
    double v;
    if (i == j) {
        double d = q[3*i] * q[3*i] + q[3*i+1] * q[3*i+1] + q[3*i+2] * q[3*i+2] - 1.0;
        v = q[r] * q[c] + q[3+r] * q[3+c] + q[6+r] * q[6+c] + q[3*i+r] * q[3*i+c] + (r == c ? d : 0.0);
    } else {
        double d = q[3*j] * q[3*i] + q[3*j+1] * q[3*i+1] + q[3*j+2] * q[3*i+2];
        v = q[3*j+r] * q[3*i+c] + (r == c ? d : 0.0);
    }
    return v * 4.0 * k;
}

// Singular value decomposition A = U diag(s) V^T of a 3x3 matrix (row-major):
// cyclic Jacobi on A^T A (annihilated entries set to zero), u_i = A v_i / s_i,
// a vanishing singular value's u completed by a cross product.
DV void svd3(const double* A, double* U, double* s, double* V) {
    double S[9];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) S[3*i+j] = A[i] * A[j] + A[3+i] * A[3+j] + A[6+i] * A[6+j];
    for (int i = 0; i < 9; i++) V[i] = (i % 4 == 0) ? 1.0 : 0.0;
    const double tr = S[0] + S[4] + S[8];
    for (int sweep = 0; sweep < 16; sweep++) {
        double off = S[1] * S[1] + S[2] * S[2] + S[5] * S[5];
        if (!(off > 1e-34 * tr * tr)) break;
        for (int pq = 0; pq < 3; pq++) {
            int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            double apq = S[3*p+q];
            if (apq == 0.0) continue;
            double theta = (S[3*q+q] - S[3*p+p]) / (2 * apq);
            double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1));
            double c = 1.0 / sqrt(t * t + 1), sn = t * c;
            for (int k = 0; k < 3; k++) {          // S <- S R
                double skp = S[3*k+p], skq = S[3*k+q];
                S[3*k+p] = c * skp - sn * skq; S[3*k+q] = sn * skp + c * skq;
            }
            for (int k = 0; k < 3; k++) {          // S <- R^T S
                double spk = S[3*p+k], sqk = S[3*q+k];
                S[3*p+k] = c * spk - sn * sqk; S[3*q+k] = sn * spk + c * sqk;
            }
            S[3*p+q] = S[3*q+p] = 0.0;
            for (int k = 0; k < 3; k++) {          // V <- V R
                double vkp = V[3*k+p], vkq = V[3*k+q];
                V[3*k+p] = c * vkp - sn * vkq; V[3*k+q] = sn * vkp + c * vkq;
            }
        }
    }
    double smax = 0;
    for (int i = 0; i < 3; i++) { s[i] = sqrt(fmax(S[4*i], 0.0)); smax = fmax(smax, s[i]); }
    bool ok[3];
    for (int i = 0; i < 3; i++) {
        ok[i] = s[i] > 1e-12 * smax && s[i] > 0.0;
        for (int r = 0; r < 3; r++)
            U[3*r+i] = ok[i] ? (A[3*r] * V[i] + A[3*r+1] * V[3+i] + A[3*r+2] * V[6+i]) / s[i] : 0.0;
    }
    for (int i = 0; i < 3; i++) {
        if (ok[i]) continue;
        int j = (i + 1) % 3, k = (i + 2) % 3;
        d3 uj = mk3(U[j], U[3+j], U[6+j]), uk = mk3(U[k], U[3+k], U[6+k]);
        d3 w = cross(uj, uk);
        if (!(dot(w, w) > 0.5)) w = ok[j] ? (fabs(uj.x) < 0.9 ? cross(uj, mk3(1, 0, 0)) : cross(uj, mk3(0, 1, 0)))
                                          : mk3(i == 0, i == 1, i == 2);
        double n = sqrt(dot(w, w));
        U[i] = w.x / n; U[3+i] = w.y / n; U[6+i] = w.z / n;
        ok[i] = true;
    }
}

// PSD projection of the Hessian of k ||A A^T - I||_F^2 (A = q, entries in
// row-major order) from its analytic eigensystem: the energy is isotropic,
// psi(s) = sum (s_i^2 - 1)^2 of the singular values of A = U S V^T, and
// (Smith, de Goes, Kim 2019, "Analytic eigensystems for isotropic distortion
// energies") its nine eigenpairs are
//   U e_i e_i^T V^T                       12 s_i^2 - 4
//   U (e_i e_j^T + e_j e_i^T) V^T / sqrt2   4 (s_i^2 + s_i s_j + s_j^2 - 1)
//   U (e_i e_j^T - e_j e_i^T) V^T / sqrt2   4 (s_i^2 - s_i s_j + s_j^2 - 1)
// (times k).  Each lane of a warp writes its entries of out (ld 12) times
// scale; all 32 lanes call it.
DV void ortho_hess_psd_warp(const double* q, double scale, double* out, int lane) {
    double U[9], s[3], V[9];
    svd3(q, U, s, V);
    double lam[9], vec[9][9];
    int m = 0;
    const double r2 = 0.70710678118654752440;
    for (int i = 0; i < 3; i++, m++) {
        lam[m] = 12.0 * s[i] * s[i] - 4.0;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) vec[m][3*r+c] = U[3*r+i] * V[3*c+i];
    }
    for (int i = 0; i < 3; i++)
        for (int j = i + 1; j < 3; j++) {
            lam[m] = 4.0 * (s[i] * s[i] + s[i] * s[j] + s[j] * s[j] - 1.0);
            lam[m + 1] = 4.0 * (s[i] * s[i] - s[i] * s[j] + s[j] * s[j] - 1.0);
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    double a = U[3*r+i] * V[3*c+j], b = U[3*r+j] * V[3*c+i];
                    vec[m][3*r+c] = (a + b) * r2;
                    vec[m + 1][3*r+c] = (a - b) * r2;
                }
            m += 2;
        }
    for (int e = lane; e < 81; e += 32) {
        int a = e / 9, b = e % 9;
        double acc = 0;
        for (int k = 0; k < 9; k++) if (lam[k] > 0) acc += lam[k] * vec[k][a] * vec[k][b];
        out[a * 12 + b] = acc * scale;
    }
}

// ------------------------------------------------- segment closest points
// Every float operation is one IEEE round-to-nearest (no contraction), so
// the result is bit-identical to a C evaluation without FMA contraction.
DV float dotf_rn(const float* a, const float* b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}
DV float clampf01(float v) { return v < 0.f ? 0.f : (v > 1.f ? 1.f : v); }
DV void seg_seg_f32(const float* p1, const float* q1, const float* p2, const float* q2, float eps,
                    float& s, float& t, float& dist) {
    float d1[3], d2[3], r[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { d1[k] = __fsub_rn(q1[k], p1[k]); d2[k] = __fsub_rn(q2[k], p2[k]); r[k] = __fsub_rn(p1[k], p2[k]); }
    float a = dotf_rn(d1, d1), e = dotf_rn(d2, d2), f = dotf_rn(d2, r);
    if (a <= eps && e <= eps) { s = 0.f; t = 0.f; }
    else if (a <= eps) { s = 0.f; t = clampf01(__fdiv_rn(f, e)); }
    else {
        float c = dotf_rn(d1, r);
        if (e <= eps) { t = 0.f; s = clampf01(__fdiv_rn(-c, a)); }
        else {
            float b = dotf_rn(d1, d2);
            float denom = __fsub_rn(__fmul_rn(a, e), __fmul_rn(b, b));
            s = (denom != 0.f) ? clampf01(__fdiv_rn(__fsub_rn(__fmul_rn(b, f), __fmul_rn(c, e)), denom)) : 0.f;
            t = __fdiv_rn(__fadd_rn(__fmul_rn(b, s), f), e);
            if (t < 0.f) { t = 0.f; s = clampf01(__fdiv_rn(-c, a)); }
            else if (t > 1.f) { t = 1.f; s = clampf01(__fdiv_rn(__fsub_rn(b, c), a)); }
        }
    }
    float dv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) dv[k] = __fsub_rn(__fadd_rn(p1[k], __fmul_rn(d1[k], s)), __fadd_rn(p2[k], __fmul_rn(d2[k], t)));
    dist = __fsqrt_rn(dotf_rn(dv, dv));
}

DV double dotd_rn(const double* a, const double* b) {
    return __dadd_rn(__dadd_rn(__dmul_rn(a[0], b[0]), __dmul_rn(a[1], b[1])), __dmul_rn(a[2], b[2]));
}
DV double clampd01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }
DV void seg_seg_f64(const double* p1, const double* q1, const double* p2, const double* q2, double eps,
                    double& s, double& t, double& dist) {
    double d1[3], d2[3], r[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { d1[k] = __dsub_rn(q1[k], p1[k]); d2[k] = __dsub_rn(q2[k], p2[k]); r[k] = __dsub_rn(p1[k], p2[k]); }
    double a = dotd_rn(d1, d1), e = dotd_rn(d2, d2), f = dotd_rn(d2, r);
    if (a <= eps && e <= eps) { s = 0.0; t = 0.0; }
    else if (a <= eps) { s = 0.0; t = clampd01(__ddiv_rn(f, e)); }
    else {
        double c = dotd_rn(d1, r);
        if (e <= eps) { t = 0.0; s = clampd01(__ddiv_rn(-c, a)); }
        else {
            double b = dotd_rn(d1, d2);
            double denom = __dsub_rn(__dmul_rn(a, e), __dmul_rn(b, b));
            s = (denom != 0.0) ? clampd01(__ddiv_rn(__dsub_rn(__dmul_rn(b, f), __dmul_rn(c, e)), denom)) : 0.0;
            t = __ddiv_rn(__dadd_rn(__dmul_rn(b, s), f), e);
            if (t < 0.0) { t = 0.0; s = clampd01(__ddiv_rn(-c, a)); }
            else if (t > 1.0) { t = 1.0; s = clampd01(__ddiv_rn(__dsub_rn(b, c), a)); }
        }
    }
    double dv[3];
#pragma unroll
    for (int k = 0; k < 3; k++) dv[k] = __dsub_rn(__dadd_rn(p1[k], __dmul_rn(d1[k], s)), __dadd_rn(p2[k], __dmul_rn(d2[k], t)));
    dist = __dsqrt_rn(dotd_rn(dv, dv));
}

// ------------------------------------------- point-triangle region (f64)
// 0..2 vertex, 3 edge t0t1, 4 edge t1t2, 5 edge t2t0, 6 face; IEEE ops
// without contraction, bit-identical to the C oracle.
DV int pt_region(const double* p, const double* a, const double* b, const double* c) {
    double ab[3], ac[3], ap[3], bp[3], cp[3];
#pragma unroll
    for (int k = 0; k < 3; k++) { ab[k] = __dsub_rn(b[k], a[k]); ac[k] = __dsub_rn(c[k], a[k]); ap[k] = __dsub_rn(p[k], a[k]); }
    double d1 = dotd_rn(ab, ap), d2 = dotd_rn(ac, ap);
    if (d1 <= 0 && d2 <= 0) return 0;
#pragma unroll
    for (int k = 0; k < 3; k++) bp[k] = __dsub_rn(p[k], b[k]);
    double d3 = dotd_rn(ab, bp), d4 = dotd_rn(ac, bp);
    if (d3 >= 0 && d4 <= d3) return 1;
    double vc = __dsub_rn(__dmul_rn(d1, d4), __dmul_rn(d3, d2));
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return 3;
#pragma unroll
    for (int k = 0; k < 3; k++) cp[k] = __dsub_rn(p[k], c[k]);
    double d5 = dotd_rn(ab, cp), d6 = dotd_rn(ac, cp);
    if (d6 >= 0 && d5 <= d6) return 2;
    double vb = __dsub_rn(__dmul_rn(d5, d2), __dmul_rn(d1, d6));
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return 5;
    double va = __dsub_rn(__dmul_rn(d3, d6), __dmul_rn(d5, d4));
    if (va <= 0 && __dsub_rn(d4, d3) >= 0 && __dsub_rn(d5, d6) >= 0) return 4;
    return 6;
}

// ----------------------------------------------------- squared distances
// Values only (used by filters, energy and CCD).
DV double d2_pp_val(d3 a, d3 b) { d3 d = a - b; return dot(d, d); }
DV double d2_pe_val(d3 p, d3 e0, d3 e1) {
    d3 w = p - e0, e = e1 - e0; double c = dot(w, e), s = dot(e, e);
    return dot(w, w) - c * c / s;
}
DV double d2_wn_val(d3 w, d3 u, d3 v) { d3 n = cross(u, v); double a = dot(w, n); return a * a / dot(n, n); }
DV double d2_ee_line_val(d3 a0, d3 a1, d3 b0, d3 b1) { return d2_wn_val(a0 - b0, a1 - a0, b1 - b0); }
DV double d2_pt_plane_val(d3 p, d3 t0, d3 t1, d3 t2) { return d2_wn_val(p - t0, t1 - t0, t2 - t0); }

DV double pt_dist2(const double* p, const double* a, const double* b, const double* c) {
    int r = pt_region(p, a, b, c);
    d3 P = ld3(p), A = ld3(a), B = ld3(b), Cc = ld3(c);
    switch (r) {
        case 0: return d2_pp_val(P, A);
        case 1: return d2_pp_val(P, B);
        case 2: return d2_pp_val(P, Cc);
        case 3: return d2_pe_val(P, A, B);
        case 4: return d2_pe_val(P, B, Cc);
        case 5: return d2_pe_val(P, Cc, A);
        default: return d2_pt_plane_val(P, A, B, Cc);
    }
}

// With derivatives.  Outputs: g (3*np), H ((3np)^2 row-major, ld = 3np).
// Map from auxiliary vectors y to stencil points: C[point][aux] in {-1,0,1}.
template <int NP, int NA>
DV void map_aux(const signed char (&C)[NP][NA], const double* gy, const double* Hy, double* g, double* H) {
    constexpr int NY = 3 * NA, NX = 3 * NP;
#pragma unroll
    for (int i = 0; i < NP; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double s = 0;
#pragma unroll
            for (int a = 0; a < NA; a++) s += C[i][a] * gy[3*a+k];
            g[3*i+k] = s;
        }
#pragma unroll 1
    for (int i = 0; i < NP; i++)
#pragma unroll 1
        for (int j = 0; j < NP; j++)
#pragma unroll
            for (int r = 0; r < 3; r++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    double s = 0;
#pragma unroll
                    for (int a = 0; a < NA; a++)
#pragma unroll
                        for (int b = 0; b < NA; b++)
                            if (C[i][a] && C[j][b]) s += C[i][a] * C[j][b] * Hy[(3*a+r)*NY + 3*b+c];
                    H[(3*i+r)*NX + 3*j+c] = s;
                }
}

DV double d2_pp_full(d3 a, d3 b, double* g, double* H) {
    d3 d = a - b;
    g[0] = 2*d.x; g[1] = 2*d.y; g[2] = 2*d.z; g[3] = -2*d.x; g[4] = -2*d.y; g[5] = -2*d.z;
#pragma unroll
    for (int i = 0; i < 36; i++) H[i] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; k++) { H[k*6+k] = 2; H[(3+k)*6+3+k] = 2; H[k*6+3+k] = -2; H[(3+k)*6+k] = -2; }
    return dot(d, d);
}

DV double d2_pe_full(d3 p, d3 e0, d3 e1, double* g, double* H) {
    d3 w = p - e0, e = e1 - e0;
    double c = dot(w, e), s = dot(e, e), is = 1.0 / s;
    double f = dot(w, w) - c * c * is;
    double gy[6], Hy[36];
    double W[3] = {w.x, w.y, w.z}, E[3] = {e.x, e.y, e.z};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        gy[k] = 2*W[k] - 2*c*is*E[k];
        gy[3+k] = -2*c*is*W[k] + 2*c*c*is*is*E[k];
    }
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int q = 0; q < 3; q++) {
            double I = (r == q) ? 1.0 : 0.0;
            Hy[r*6+q] = 2*I - 2*is*E[r]*E[q];
            double we = -2*is*E[r]*W[q] - 2*c*is*I + 4*c*is*is*E[r]*E[q];
            Hy[r*6+3+q] = we;
            Hy[(3+q)*6+r] = we;
            Hy[(3+r)*6+3+q] = -2*is*W[r]*W[q] + 4*c*is*is*(W[r]*E[q] + E[r]*W[q])
                              - 8*c*c*is*is*is*E[r]*E[q] + 2*c*c*is*is*I;
        }
    const signed char C[3][2] = {{1, 0}, {-1, -1}, {0, 1}};
    map_aux<3, 2>(C, gy, Hy, g, H);
    return f;
}

DV void skew(d3 a, double* S) {
    S[0] = 0;    S[1] = -a.z; S[2] = a.y;
    S[3] = a.z;  S[4] = 0;    S[5] = -a.x;
    S[6] = -a.y; S[7] = a.x;  S[8] = 0;
}
// f = (w.n)^2/(n.n), n = u x v; derivatives w.r.t. (w, u, v)
DV double d2_wn_full(d3 w, d3 u, d3 v, double* gy, double* Hy) {
    d3 n = cross(u, v);
    double a = dot(w, n), b = dot(n, n), ib = 1.0 / b;
    double f = a * a * ib;
    d3 vw = cross(v, w), wu = cross(w, u), vn = cross(v, n), nu = cross(n, u);
    double ga[9] = {n.x, n.y, n.z, vw.x, vw.y, vw.z, wu.x, wu.y, wu.z};
    double gb[9] = {0, 0, 0, 2*vn.x, 2*vn.y, 2*vn.z, 2*nu.x, 2*nu.y, 2*nu.z};
    double Su[9], Sv[9], Sw[9], Sn[9];
    skew(u, Su); skew(v, Sv); skew(w, Sw); skew(n, Sn);
    // Ha and Hb only have off-diagonal (w,u), (w,v), (u,v) and (u,u), (u,v), (v,v) blocks
#pragma unroll
    for (int i = 0; i < 9; i++) gy[i] = 2*a*ib*ga[i] - a*a*ib*ib*gb[i];
    double c1 = 2*ib, c2 = 2*a*ib, c3 = 2*a*ib*ib, c4 = 2*a*a*ib*ib*ib, c5 = a*a*ib*ib;
#pragma unroll 1
    for (int i = 0; i < 9; i++)
#pragma unroll
        for (int j = 0; j < 9; j++) {
            int bi = i / 3, bj = j / 3, r = i % 3, c = j % 3;
            double ha = 0, hb = 0;
            if (bi == 0 && bj == 1) ha = -Sv[3*r+c];
            else if (bi == 1 && bj == 0) ha = -Sv[3*c+r];
            else if (bi == 0 && bj == 2) ha = Su[3*r+c];
            else if (bi == 2 && bj == 0) ha = Su[3*c+r];
            else if (bi == 1 && bj == 2) ha = -Sw[3*r+c];
            else if (bi == 2 && bj == 1) ha = -Sw[3*c+r];
            if (bi == 1 && bj == 1) {          // 2 [v]x^T [v]x
                double s = 0; for (int m = 0; m < 3; m++) s += Sv[3*m+r] * Sv[3*m+c]; hb = 2*s;
            } else if (bi == 1 && bj == 2) {   // 2 [v]x [u]x - 2 [n]x
                double s = 0; for (int m = 0; m < 3; m++) s += Sv[3*r+m] * Su[3*m+c]; hb = 2*s - 2*Sn[3*r+c];
            } else if (bi == 2 && bj == 1) {   // 2 [u]x [v]x + 2 [n]x
                double s = 0; for (int m = 0; m < 3; m++) s += Su[3*r+m] * Sv[3*m+c]; hb = 2*s + 2*Sn[3*r+c];
            } else if (bi == 2 && bj == 2) {   // 2 [u]x^T [u]x
                double s = 0; for (int m = 0; m < 3; m++) s += Su[3*m+r] * Su[3*m+c]; hb = 2*s;
            }
            Hy[i*9+j] = c1*ga[i]*ga[j] + c2*ha - c3*(ga[i]*gb[j] + gb[i]*ga[j]) + c4*gb[i]*gb[j] - c5*hb;
        }
    return f;
}
DV double d2_ee_line_full(d3 a0, d3 a1, d3 b0, d3 b1, double* g, double* H) {
    double gy[9], Hy[81];
    double f = d2_wn_full(a0 - b0, a1 - a0, b1 - b0, gy, Hy);
    const signed char C[4][3] = {{1, -1, 0}, {0, 1, 0}, {-1, 0, -1}, {0, 0, 1}};
    map_aux<4, 3>(C, gy, Hy, g, H);
    return f;
}
DV double d2_pt_plane_full(d3 p, d3 t0, d3 t1, d3 t2, double* g, double* H) {
    double gy[9], Hy[81];
    double f = d2_wn_full(p - t0, t1 - t0, t2 - t0, gy, Hy);
    const signed char C[4][3] = {{1, 0, 0}, {-1, -1, -1}, {0, 1, 0}, {0, 0, 1}};
    map_aux<4, 3>(C, gy, Hy, g, H);
    return f;
}


// ------------------------------------------------------------ additive CCD
// kind 0: edge-edge (x0 x1 | x2 x3), kind 1: point-triangle (x0 | x1 x2 x3).
// Returns 1 on a hit with *toi = conservative time; 0 if none in [0,tmax].
// The iteration count is capped at max_iter (AbdParams.ccd_max_iter, or
// ABD_CCD_MAX_ITER); on the cap the time reached so far is returned
// (conservative) and *capped is set.
DV double prim_dist2(int kind, const double* x) {
    if (kind == 0) { double s, t, d; seg_seg_f64(x, x + 3, x + 6, x + 9, 0.0, s, t, d); return d * d; }
    return pt_dist2(x, x + 3, x + 6, x + 9);
}
DV int accd(int kind, const double* x0, const double* p0, double s, double tmax, double* toi, int* capped,
            int max_iter) {
    double x[12], p[12], pm[3] = {0, 0, 0};
    for (int i = 0; i < 12; i++) { x[i] = x0[i]; p[i] = p0[i]; }
    for (int i = 0; i < 4; i++) for (int k = 0; k < 3; k++) pm[k] += p[3*i+k] * 0.25;
    for (int i = 0; i < 4; i++) for (int k = 0; k < 3; k++) p[3*i+k] -= pm[k];
    double n[4];
    for (int i = 0; i < 4; i++) n[i] = sqrt(p[3*i] * p[3*i] + p[3*i+1] * p[3*i+1] + p[3*i+2] * p[3*i+2]);
    double lp = (kind == 0) ? fmax(n[0], n[1]) + fmax(n[2], n[3]) : n[0] + fmax(n[1], fmax(n[2], n[3]));
    if (lp == 0.0) return 0;
    double d = sqrt(prim_dist2(kind, x));
    if (d == 0.0) { *toi = 0.0; return 1; }
    double g = s * d;
    double t = 0, tl = (1 - s) * d / lp;
    for (int it = 0; it < max_iter; it++) {
        for (int i = 0; i < 12; i++) x[i] += tl * p[i];
        d = sqrt(prim_dist2(kind, x));
        if (t > 0 && d < g) { *toi = t; return 1; }
        t += tl;
        if (t > tmax) return 0;
        tl = 0.9 * d / lp;
    }
    *capped = 1;
    *toi = t;
    return 1;
}
