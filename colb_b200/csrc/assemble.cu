// assemble.cu — gradient and block Hessian of the incremental potential.
//
//  inertia + orthogonality  abd.py:108-166, ortho.py:9-41 (one thread per body)
//  barrier contacts ....... abd.py:198-571: classify each candidate into a
//                           PP / PE / EE (or PT / PG) stencil, differentiate its
//                           squared distance, chain through the barrier and map
//                           vertex derivatives to body DoFs with
//                           J = [1, xbar^T] (x) I3.
//
// The reference writes 64 triplets per contact into a COO array (with the
// contact/inertia slot overlap at abd.py:111 vs :311) and converts the whole
// array to BSR every iteration (abd.py:634).  Here the body-pair pattern is
// built once per Newton iteration from the sorted contact list (radix sort +
// unique of 64-bit body-pair keys into CSR of 12x12 blocks), and each active
// contact adds its four body blocks into that structure with FP64/FP32
// atomics.
#include "contact.cuh"
#include "warp_eig.cuh"
#include <cub/cub.cuh>

Geo eng_geo(Engine* E);

DV int stencil_np(int type) { return type == T_PP ? 2 : (type == T_PE ? 3 : (type == T_PG ? 1 : 4)); }
DV int other_vertex(int type, int4 s) { return type == T_EE ? s.z : (type == T_PG ? s.x : s.y); }

// ---------------------------------------------------------- prepare + keys
// Contacts [0, n_total) (the device count); with nkey_pairs > n_total the key
// pairs of the slots up to nkey_pairs are sentinels (~0), so a sort sized
// before the count is known sees only real keys and sentinels.
__global__ void k_contact_prepare(const Counters* cnt, const int4* __restrict__ contacts, Geo G, int f32, double dhat,
                                  int nb, int4* cst, int* ctype, double* cxb, int2* cbody,
                                  unsigned long long* keys, int* n_active, int nkey_pairs) {
    int n = cnt->n_total;
    GS_LOOP(c, nkey_pairs) {
        if (c >= n) { keys[nb + 2*c] = ~0ull; keys[nb + 2*c + 1] = ~0ull; }
    }
    GS_LOOP(c, n) {
        int4 C = contacts[c];
        int4 stv; int type = -1; double xb = 0;
        bool act = classify(G, C.x, C.y, C.z, f32, dhat, stv, type, xb);
        unsigned long long k0 = ~0ull, k1 = ~0ull;
        if (act) {
            int b0 = G.vbody[stv.x];
            int b1 = G.vbody[other_vertex(type, stv)];
            cbody[c] = make_int2(b0, b1);
            if (b0 != b1 && G.mass[b0] > 0.0 && G.mass[b1] > 0.0) {
                k0 = (unsigned long long)b0 * nb + b1;
                k1 = (unsigned long long)b1 * nb + b0;
            }
            atomicAdd(n_active, 1);
        }
        cst[c] = stv; ctype[c] = act ? type : -1; cxb[c] = xb;
        keys[nb + 2*c] = k0; keys[nb + 2*c + 1] = k1;
    }
}
__global__ void k_diag_keys(int nb, unsigned long long* keys) {
    GS_LOOP(b, nb) keys[b] = (unsigned long long)b * nb + b;
}
__global__ void k_block_rows(int nb, const unsigned long long* __restrict__ ukeys, const int* n_unique,
                             int* row_ptr, int* bcol, Counters* cnt) {
    int m = *n_unique;
    if (m > 0 && ukeys[m-1] == ~0ull) m--;            // drop the sentinel
    GS_LOOP(i, m) {
        unsigned long long k = ukeys[i];
        int r = (int)(k / nb);
        bcol[i] = (int)(k % nb);
        if (i == 0 || (int)(ukeys[i-1] / nb) != r) row_ptr[r] = (int)i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { row_ptr[nb] = m; cnt->nnzb = m; }
}


template <class T>
__global__ void k_zero_vals(const Counters* cnt, T* vals) {
    long n = (long)cnt->nnzb * 144;
    GS_LOOP(i, n) vals[i] = (T)0;
}

// ---------------------------------------------------- inertia + ortho (abd.py:108-149)
// One warp per body: gradient by lanes 0..11, the 9x9 orthogonality Hessian
// (scaled by dt^2) built lane-parallel in shared memory, projected to PSD
// when requested, and written with the mass terms into the diagonal block.
#define BA_WARPS 4
template <class T>
__global__ void __launch_bounds__(32 * BA_WARPS) k_body_assemble(int nb, const double* __restrict__ st,
                                const double* __restrict__ mass, const double* __restrict__ J, double dt, double g0,
                                double g1, double g2, double k_ortho, int project, double pinned_diag,
                                const int* __restrict__ row_ptr, const int* __restrict__ bcol, T* vals, double* grad) {
    __shared__ WarpEigSmem sm[BA_WARPS];
    __shared__ double sq[BA_WARPS][9];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    WarpEigSmem& E = sm[w];
    for (int b = blockIdx.x * BA_WARPS + w; b < nb; b += gridDim.x * BA_WARPS) {
        int bi = find_block(row_ptr, bcol, b, b);
        if (bi < 0) continue;                              // every row holds its diagonal key
        T* V = vals + (long)bi * 144;
        double* g = grad + 12L * b;
        double m = mass[b];
        if (!(m > 0.0)) {
            if (lane < 12) g[lane] = 0.0;
            for (int e = lane; e < 144; e += 32) V[e] = (T)((e % 12 == e / 12) ? pinned_diag : 0.0);
            continue;
        }
        const double* now = st + ST_STRIDE * (long)b + ST_NOW; const double* nx = st + ST_STRIDE * (long)b + ST_NXT;
        if (lane < 9) sq[w][lane] = nx[ST_Q + lane];
        __syncwarp();
        const double* q = sq[w];
        double Jb = J[b];
        if (lane < 3) {
            double gv = lane == 0 ? g0 : (lane == 1 ? g1 : g2);
            double ct = now[ST_C + lane] + dt * now[ST_V + lane] + dt * dt * gv;
            g[lane] = (nx[ST_C + lane] - ct) * m;
        } else if (lane < 12) {
            int r = lane - 3, i = r / 3, c = r % 3;
            double gi = -q[3*i+c];
            for (int j = 0; j < 3; j++) gi += (q[3*i]*q[3*j] + q[3*i+1]*q[3*j+1] + q[3*i+2]*q[3*j+2]) * q[3*j+c];
            double qt = now[ST_Q + r] + dt * now[ST_QD + r];
            g[lane] = dt * dt * (gi * 4.0 * k_ortho) + (q[r] - qt) * Jb;
        }
        if (project) {
            ortho_hess_psd_warp(q, k_ortho * dt * dt, E.A, lane);    // analytic eigensystem
        } else {
            for (int e = lane; e < 81; e += 32) {
                int rr = e / 9, cc = e % 9;
                E.A[rr*12 + cc] = ortho_hess(q, k_ortho, rr / 3, cc / 3, rr % 3, cc % 3) * dt * dt;
            }
        }
        __syncwarp();
        for (int e = lane; e < 144; e += 32) {
            int row = e % 12, col = e / 12;
            double v;
            if (row < 3 || col < 3) v = (row == col) ? m : 0.0;
            else v = E.A[(row-3)*12 + (col-3)] + (row == col ? Jb : 0.0);
            V[e] = (T)v;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------- contacts (abd.py:198-571)
// One warp per active contact.  The stencil's squared-distance gradient and
// Hessian are built lane-parallel in shared memory (auxiliary vectors by
// lane 0, matrix entries by all lanes), chained through the barrier,
// projected to PSD by the warp Jacobi (warp_eig.cuh), and scattered into the
// body blocks: lanes own block entries, each summing the stencil vertices
// that map to it through J = [1, xbar^T] (x) I3.
struct ContactSmem {
    WarpEigSmem E;
    double x[12], g[12], gy[9], aux[48], J[4][4];
    double B0, B1, B2;
    int v[4], vb[4], np, type, bodies[2], nbd;
};

// C[point][aux] maps for the (w, u, v) and (w, e) parameterisations
__constant__ signed char c_map_ee[4][3] = {{1, -1, 0}, {0, 1, 0}, {-1, 0, -1}, {0, 0, 1}};
__constant__ signed char c_map_pt[4][3] = {{1, 0, 0}, {-1, -1, -1}, {0, 1, 0}, {0, 0, 1}};
__constant__ signed char c_map_pe[3][2] = {{1, 0}, {-1, -1}, {0, 1}};

DV void skew9(const double* a, double* S) {
    S[0] = 0; S[1] = -a[2]; S[2] = a[1]; S[3] = a[2]; S[4] = 0; S[5] = -a[0]; S[6] = -a[1]; S[7] = a[0]; S[8] = 0;
}
DV void cross3(const double* a, const double* b, double* o) {
    o[0] = a[1]*b[2] - a[2]*b[1]; o[1] = a[2]*b[0] - a[0]*b[2]; o[2] = a[0]*b[1] - a[1]*b[0];
}

// squared distance gradient (C.g) and Hessian (C.E.A, ld 12) of the stencil
DV void warp_distance_derivs(ContactSmem& C, const Geo& G) {
    const int lane = threadIdx.x & 31;
    const int m = 3 * C.np;
    double* A = C.E.A; double* Hy = C.E.T;
    if (C.type == T_PG) {
        if (lane == 0) {
            const double* nn = G.planes + 4 * C.v[1];
            double d = nn[0] * C.x[0] + nn[1] * C.x[1] + nn[2] * C.x[2] - nn[3];
            for (int k = 0; k < 3; k++) { C.g[k] = 2 * d * nn[k]; C.aux[k] = nn[k]; }
        }
        __syncwarp();
        if (lane < 9) A[(lane / 3) * 12 + lane % 3] = 2 * C.aux[lane / 3] * C.aux[lane % 3];
    } else if (C.type == T_PP) {
        if (lane < 6) { int k = lane % 3; double d = C.x[k] - C.x[3 + k]; C.g[lane] = lane < 3 ? 2 * d : -2 * d; }
        for (int e = lane; e < 36; e += 32) {
            int i = e / 6, j = e % 6;
            A[i*12+j] = (i % 3 == j % 3) ? ((i < 3) == (j < 3) ? 2.0 : -2.0) : 0.0;
        }
    } else if (C.type == T_PE) {
        // w = p - e0, e = e1 - e0, f = w.w - (w.e)^2/(e.e)
        if (lane == 0) {
            double w[3], e[3];
            for (int k = 0; k < 3; k++) { w[k] = C.x[k] - C.x[3+k]; e[k] = C.x[6+k] - C.x[3+k]; }
            double c = w[0]*e[0] + w[1]*e[1] + w[2]*e[2], s2 = e[0]*e[0] + e[1]*e[1] + e[2]*e[2], is = 1.0 / s2;
            for (int k = 0; k < 3; k++) {
                C.aux[k] = w[k]; C.aux[3+k] = e[k];
                C.gy[k] = 2*w[k] - 2*c*is*e[k];
                C.gy[3+k] = -2*c*is*w[k] + 2*c*c*is*is*e[k];
            }
            C.aux[6] = c; C.aux[7] = is;
        }
        __syncwarp();
        const double* W = C.aux; const double* Ev = C.aux + 3;
        double c = C.aux[6], is = C.aux[7];
        for (int e = lane; e < 36; e += 32) {
            int i = e / 6, j = e % 6, bi = i / 3, bj = j / 3, r = i % 3, q = j % 3;
            double I = (r == q) ? 1.0 : 0.0, h;
            if (bi == 0 && bj == 0) h = 2*I - 2*is*Ev[r]*Ev[q];
            else if (bi == 0 && bj == 1) h = -2*is*Ev[r]*W[q] - 2*c*is*I + 4*c*is*is*Ev[r]*Ev[q];
            else if (bi == 1 && bj == 0) h = -2*is*Ev[q]*W[r] - 2*c*is*I + 4*c*is*is*Ev[q]*Ev[r];
            else h = -2*is*W[r]*W[q] + 4*c*is*is*(W[r]*Ev[q] + Ev[r]*W[q]) - 8*c*c*is*is*is*Ev[r]*Ev[q] + 2*c*c*is*is*I;
            Hy[i*6+j] = h;
        }
        __syncwarp();
        if (lane < 9) {
            int pnt = lane / 3, k = lane % 3;
            C.g[lane] = c_map_pe[pnt][0] * C.gy[k] + c_map_pe[pnt][1] * C.gy[3+k];
        }
        for (int e = lane; e < 81; e += 32) {
            int i = e / 9, j = e % 9, pi = i / 3, pj = j / 3, r = i % 3, q = j % 3;
            double acc = 0;
            for (int a = 0; a < 2; a++) if (c_map_pe[pi][a])
                for (int b = 0; b < 2; b++) if (c_map_pe[pj][b])
                    acc += c_map_pe[pi][a] * c_map_pe[pj][b] * Hy[(3*a+r)*6 + 3*b+q];
            A[i*12+j] = acc;
        }
    } else {
        // f = (w.n)^2/(n.n), n = u x v; EE: w = a0-b0, u = a1-a0, v = b1-b0;
        // PT: w = p-t0, u = t1-t0, v = t2-t0
        if (lane == 0) {
            double w[3], u[3], v[3];
            for (int k = 0; k < 3; k++) {
                if (C.type == T_EE) { w[k] = C.x[k] - C.x[6+k]; u[k] = C.x[3+k] - C.x[k]; v[k] = C.x[9+k] - C.x[6+k]; }
                else { w[k] = C.x[k] - C.x[3+k]; u[k] = C.x[6+k] - C.x[3+k]; v[k] = C.x[9+k] - C.x[3+k]; }
            }
            double n[3]; cross3(u, v, n);
            double a = w[0]*n[0] + w[1]*n[1] + w[2]*n[2], b = n[0]*n[0] + n[1]*n[1] + n[2]*n[2], ib = 1.0 / b;
            double vw[3], wu[3], vn[3], nu[3];
            cross3(v, w, vw); cross3(w, u, wu); cross3(v, n, vn); cross3(n, u, nu);
            double* ga = C.aux; double* gb = C.aux + 9;
            for (int k = 0; k < 3; k++) {
                ga[k] = n[k]; ga[3+k] = vw[k]; ga[6+k] = wu[k];
                gb[k] = 0; gb[3+k] = 2*vn[k]; gb[6+k] = 2*nu[k];
            }
            skew9(u, C.aux + 18); skew9(v, C.aux + 27); skew9(w, C.aux + 36);
            double Sn[9]; skew9(n, Sn);
            // Sn is needed only in the (u,v) blocks: keep it in gy's slot after gy is consumed
            for (int i = 0; i < 9; i++) C.gy[i] = 2*a*ib*ga[i] - a*a*ib*ib*gb[i];
            C.aux[45] = a; C.aux[46] = ib;
            for (int i = 0; i < 9; i++) C.E.V[i] = Sn[i];          // V is free until the projection
        }
        __syncwarp();
        const double* ga = C.aux; const double* gb = C.aux + 9;
        const double* Su = C.aux + 18; const double* Sv = C.aux + 27; const double* Sw = C.aux + 36;
        const double* Sn = C.E.V;
        double a = C.aux[45], ib = C.aux[46];
        double c1 = 2*ib, c2 = 2*a*ib, c3 = 2*a*ib*ib, c4 = 2*a*a*ib*ib*ib, c5 = a*a*ib*ib;
        for (int e = lane; e < 81; e += 32) {
            int i = e / 9, j = e % 9, bi = i / 3, bj = j / 3, r = i % 3, c = j % 3;
            double ha = 0, hb = 0;
            if (bi == 0 && bj == 1) ha = -Sv[3*r+c];
            else if (bi == 1 && bj == 0) ha = -Sv[3*c+r];
            else if (bi == 0 && bj == 2) ha = Su[3*r+c];
            else if (bi == 2 && bj == 0) ha = Su[3*c+r];
            else if (bi == 1 && bj == 2) ha = -Sw[3*r+c];
            else if (bi == 2 && bj == 1) ha = -Sw[3*c+r];
            if (bi == 1 && bj == 1) { double t = 0; for (int q = 0; q < 3; q++) t += Sv[3*q+r] * Sv[3*q+c]; hb = 2*t; }
            else if (bi == 1 && bj == 2) { double t = 0; for (int q = 0; q < 3; q++) t += Sv[3*r+q] * Su[3*q+c]; hb = 2*t - 2*Sn[3*r+c]; }
            else if (bi == 2 && bj == 1) { double t = 0; for (int q = 0; q < 3; q++) t += Su[3*r+q] * Sv[3*q+c]; hb = 2*t + 2*Sn[3*r+c]; }
            else if (bi == 2 && bj == 2) { double t = 0; for (int q = 0; q < 3; q++) t += Su[3*q+r] * Su[3*q+c]; hb = 2*t; }
            Hy[i*9+j] = c1*ga[i]*ga[j] + c2*ha - c3*(ga[i]*gb[j] + gb[i]*ga[j]) + c4*gb[i]*gb[j] - c5*hb;
        }
        __syncwarp();
        const signed char (*Cm)[3] = C.type == T_EE ? c_map_ee : c_map_pt;
        if (lane < 12) {
            int pnt = lane / 3, k = lane % 3;
            double acc = 0;
            for (int q = 0; q < 3; q++) acc += Cm[pnt][q] * C.gy[3*q+k];
            C.g[lane] = acc;
        }
        for (int e = lane; e < 144; e += 32) {
            int i = e / 12, j = e % 12, pi = i / 3, pj = j / 3, r = i % 3, q = j % 3;
            double acc = 0;
            for (int aa = 0; aa < 3; aa++) if (Cm[pi][aa])
                for (int bb = 0; bb < 3; bb++) if (Cm[pj][bb])
                    acc += Cm[pi][aa] * Cm[pj][bb] * Hy[(3*aa+r)*9 + 3*bb+q];
            A[i*12+j] = acc;
        }
    }
    (void)m;
    __syncwarp();
}

template <class T, int CAW>
__global__ void __launch_bounds__(32 * CAW, 1) k_contact_assemble(const Counters* cnt, const int4* __restrict__ cst,
                                   const int* __restrict__ ctype, const double* __restrict__ cxb, Geo G, int barrier,
                                   double dhat, double sc, int hess_mode, const int* __restrict__ row_ptr,
                                   const int* __restrict__ bcol, T* vals, double* grad) {
    __shared__ ContactSmem sm[CAW];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    ContactSmem& C = sm[w];
    const int n = cnt->n_total;
    for (int c = blockIdx.x * CAW + w; c < n; c += gridDim.x * CAW) {
        int type = ctype[c];
        if (type < 0) continue;                       // warp-uniform
        if (lane == 0) {
            int4 s4 = cst[c];
            int sv[4] = {s4.x, s4.y, s4.z, s4.w};
            C.type = type;
            C.np = stencil_np(type);
            for (int i = 0; i < 4; i++) C.v[i] = sv[i];
            int nx = type == T_PG ? 1 : C.np;
            for (int i = 0; i < nx; i++) {
                int v = sv[i];
                for (int k = 0; k < 3; k++) C.x[3*i+k] = G.x[3*v+k];
                C.vb[i] = G.vbody[v];
                C.J[i][0] = 1.0; C.J[i][1] = G.xbar[3*v]; C.J[i][2] = G.xbar[3*v+1]; C.J[i][3] = G.xbar[3*v+2];
            }
            barrier3(barrier, cxb[c], dhat * dhat, C.B0, C.B1, C.B2);
            C.bodies[0] = C.vb[0]; C.nbd = 1;
            for (int i = 1; i < C.np; i++) if (C.vb[i] != C.bodies[0]) { C.bodies[1] = C.vb[i]; C.nbd = 2; break; }
        }
        __syncwarp();
        warp_distance_derivs(C, G);
        const int np = C.np, m = 3 * np;
        const double B1 = C.B1, B2 = C.B2;
        double* A = C.E.A;
        if (hess_mode == ABD_HESS_REFERENCE) {
            if (C.type == T_EE) team_psd_project_fast<32>(C.E, 12);      // abd.py:247
            for (int e = lane; e < m * m; e += 32) {
                int i = e / m, j = e % m;
                double h = (C.type == T_PP) ? 0.0 : B1 * A[i*12+j];       // abd.py:381-382
                A[i*12+j] = (h + B2 * C.g[i] * C.g[j]) * sc;
            }
            __syncwarp();
        } else if (C.type == T_PG || C.type == T_PP) {
            // analytic projection.  With d the separation (g = 2d on the first
            // point), B1 H + B2 g g^T is [M] (point-plane, d along the normal)
            // or [M -M; -M M] (point-point) with M = 2 B1 I + 4 B2 d d^T for
            // point-point and M = (2 B1 + 4 B2 d^2) n n^T for point-plane; the
            // projection clamps M's eigenvalues 2 B1 (across d) and
            // 2 B1 + 4 B2 |d|^2 (along d) at zero.
            const double dx = 0.5 * C.g[0], dy = 0.5 * C.g[1], dz = 0.5 * C.g[2];
            const double dd = dx * dx + dy * dy + dz * dz;
            const double lam_t = C.type == T_PP ? fmax(2.0 * B1, 0.0) : 0.0;
            const double lam_n = fmax(2.0 * B1 + 4.0 * B2 * dd, 0.0);
            const double dv[3] = {dx, dy, dz};
            for (int e = lane; e < m * m; e += 32) {
                int i = e / m, j = e % m, a = i % 3, b = j % 3;
                double nn = dd > 0.0 ? dv[a] * dv[b] / dd : 0.0;
                double Mab = lam_t * ((a == b ? 1.0 : 0.0) - nn) + lam_n * nn;
                A[i*12+j] = ((i / 3) == (j / 3) ? Mab : -Mab) * sc;
            }
            __syncwarp();
        } else {
            for (int e = lane; e < m * m; e += 32) {
                int i = e / m, j = e % m;
                A[i*12+j] = B1 * A[i*12+j] + B2 * C.g[i] * C.g[j];
            }
            __syncwarp();
            team_psd_project_fast<32>(C.E, m);
            for (int e = lane; e < m * m; e += 32) { int i = e / m, j = e % m; A[i*12+j] *= sc; }
            __syncwarp();
        }
        // gradient: G[b][3 al + k] += J_i[al] g_i[k] * B1 * sc for dynamic bodies
        for (int e = lane; e < np * 12; e += 32) {
            int i = e / 12, al = (e % 12) / 3, k = e % 3;
            int b = C.vb[i];
            if (G.mass[b] > 0.0) atomicAdd(grad + 12L * b + 3 * al + k, C.J[i][al] * C.g[3*i+k] * B1 * sc);
        }
        // Hessian blocks of the (at most two) bodies
        for (int pa = 0; pa < C.nbd; pa++)
            for (int pb = 0; pb < C.nbd; pb++) {
                int Ba = C.bodies[pa], Bb = C.bodies[pb];
                if (!(G.mass[Ba] > 0.0) || !(G.mass[Bb] > 0.0)) continue;
                int bi = find_block(row_ptr, bcol, Ba, Bb);
                if (bi < 0) continue;
                T* V = vals + (long)bi * 144;
                for (int e = lane; e < 144; e += 32) {
                    int row = e % 12, col = e / 12;          // column-major block entry (row, col)
                    int al = row / 3, r = row % 3, be = col / 3, q = col % 3;
                    double sum = 0;
                    for (int i = 0; i < np; i++) {
                        if (C.vb[i] != Ba) continue;
                        for (int j = 0; j < np; j++) {
                            if (C.vb[j] != Bb) continue;
                            sum += C.J[i][al] * C.J[j][be] * A[(3*i+r)*12 + 3*j+q];
                        }
                    }
                    if (sum != 0.0) atomicAdd(V + e, (T)sum);
                }
            }
        __syncwarp();
    }
}

// One block of NT threads per active contact: the same work as
// k_contact_assemble, with the PSD projection spread over the whole block.
template <class T, int NT>
__global__ void __launch_bounds__(NT, 1) k_contact_assemble_team(const Counters* cnt, const int4* __restrict__ cst,
                                   const int* __restrict__ ctype, const double* __restrict__ cxb, Geo G, int barrier,
                                   double dhat, double sc, int hess_mode, const int* __restrict__ row_ptr,
                                   const int* __restrict__ bcol, T* vals, double* grad) {
    __shared__ ContactSmem C;
    const int tid = threadIdx.x, warp = threadIdx.x >> 5;
    const int n = cnt->n_total;
    for (int c = blockIdx.x; c < n; c += gridDim.x) {
        int type = ctype[c];
        if (type < 0) continue;                       // block-uniform
        if (tid == 0) {
            int4 s4 = cst[c];
            int sv[4] = {s4.x, s4.y, s4.z, s4.w};
            C.type = type;
            C.np = stencil_np(type);
            for (int i = 0; i < 4; i++) C.v[i] = sv[i];
            int nx = type == T_PG ? 1 : C.np;
            for (int i = 0; i < nx; i++) {
                int v = sv[i];
                for (int k = 0; k < 3; k++) C.x[3*i+k] = G.x[3*v+k];
                C.vb[i] = G.vbody[v];
                C.J[i][0] = 1.0; C.J[i][1] = G.xbar[3*v]; C.J[i][2] = G.xbar[3*v+1]; C.J[i][3] = G.xbar[3*v+2];
            }
            barrier3(barrier, cxb[c], dhat * dhat, C.B0, C.B1, C.B2);
            C.bodies[0] = C.vb[0]; C.nbd = 1;
            for (int i = 1; i < C.np; i++) if (C.vb[i] != C.bodies[0]) { C.bodies[1] = C.vb[i]; C.nbd = 2; break; }
        }
        __syncthreads();
        if (warp == 0) warp_distance_derivs(C, G);
        __syncthreads();
        const int np = C.np, m = 3 * np;
        const double B1 = C.B1, B2 = C.B2;
        double* A = C.E.A;
        if (hess_mode == ABD_HESS_REFERENCE) {
            if (C.type == T_EE) team_psd_project_fast<NT>(C.E, 12);          // abd.py:247
            for (int e = tid; e < m * m; e += NT) {
                int i = e / m, j = e % m;
                double h = (C.type == T_PP) ? 0.0 : B1 * A[i*12+j];       // abd.py:381-382
                A[i*12+j] = (h + B2 * C.g[i] * C.g[j]) * sc;
            }
            __syncthreads();
        } else if (C.type == T_PG || C.type == T_PP) {
            // analytic projection.  With d the separation (g = 2d on the first
            // point), B1 H + B2 g g^T is [M] (point-plane, d along the normal)
            // or [M -M; -M M] (point-point) with M = 2 B1 I + 4 B2 d d^T for
            // point-point and M = (2 B1 + 4 B2 d^2) n n^T for point-plane; the
            // projection clamps M's eigenvalues 2 B1 (across d) and
            // 2 B1 + 4 B2 |d|^2 (along d) at zero.
            const double dx = 0.5 * C.g[0], dy = 0.5 * C.g[1], dz = 0.5 * C.g[2];
            const double dd = dx * dx + dy * dy + dz * dz;
            const double lam_t = C.type == T_PP ? fmax(2.0 * B1, 0.0) : 0.0;
            const double lam_n = fmax(2.0 * B1 + 4.0 * B2 * dd, 0.0);
            const double dv[3] = {dx, dy, dz};
            for (int e = tid; e < m * m; e += NT) {
                int i = e / m, j = e % m, a = i % 3, b = j % 3;
                double nn = dd > 0.0 ? dv[a] * dv[b] / dd : 0.0;
                double Mab = lam_t * ((a == b ? 1.0 : 0.0) - nn) + lam_n * nn;
                A[i*12+j] = ((i / 3) == (j / 3) ? Mab : -Mab) * sc;
            }
            __syncthreads();
        } else {
            for (int e = tid; e < m * m; e += NT) {
                int i = e / m, j = e % m;
                A[i*12+j] = B1 * A[i*12+j] + B2 * C.g[i] * C.g[j];
            }
            __syncthreads();
            team_psd_project_fast<NT>(C.E, m);
            for (int e = tid; e < m * m; e += NT) { int i = e / m, j = e % m; A[i*12+j] *= sc; }
            __syncthreads();
        }
        // gradient: G[b][3 al + k] += J_i[al] g_i[k] * B1 * sc for dynamic bodies
        for (int e = tid; e < np * 12; e += NT) {
            int i = e / 12, al = (e % 12) / 3, k = e % 3;
            int b = C.vb[i];
            if (G.mass[b] > 0.0) atomicAdd(grad + 12L * b + 3 * al + k, C.J[i][al] * C.g[3*i+k] * B1 * sc);
        }
        // Hessian blocks of the (at most two) bodies
        for (int pa = 0; pa < C.nbd; pa++)
            for (int pb = 0; pb < C.nbd; pb++) {
                int Ba = C.bodies[pa], Bb = C.bodies[pb];
                if (!(G.mass[Ba] > 0.0) || !(G.mass[Bb] > 0.0)) continue;
                int bi = find_block(row_ptr, bcol, Ba, Bb);
                if (bi < 0) continue;
                T* V = vals + (long)bi * 144;
                for (int e = tid; e < 144; e += NT) {
                    int row = e % 12, col = e / 12;          // column-major block entry (row, col)
                    int al = row / 3, r = row % 3, be = col / 3, q = col % 3;
                    double sum = 0;
                    for (int i = 0; i < np; i++) {
                        if (C.vb[i] != Ba) continue;
                        for (int j = 0; j < np; j++) {
                            if (C.vb[j] != Bb) continue;
                            sum += C.J[i][al] * C.J[j][be] * A[(3*i+r)*12 + 3*j+q];
                        }
                    }
                    if (sum != 0.0) atomicAdd(V + e, (T)sum);
                }
            }
        __syncthreads();
    }
}


// ---------------------------------------------------- block-Jacobi inverse
// One warp per body: Gauss-Jordan with partial pivoting on [D | I] in shared
// memory, lanes owning the 24 columns.  A singular block gives the identity.
#define BI_WARPS 4
template <class T>
__global__ void __launch_bounds__(32 * BI_WARPS) k_block_inverse(int nb, const int* __restrict__ row_ptr,
        const int* __restrict__ bcol, const T* __restrict__ vals, T* dinv) {
    __shared__ double sM[BI_WARPS][12][25];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double (*M)[25] = sM[w];
    for (int b = blockIdx.x * BI_WARPS + w; b < nb; b += gridDim.x * BI_WARPS) {
        int bi = find_block(row_ptr, bcol, b, b);
        if (bi < 0) continue;
        const T* V = vals + (long)bi * 144;
        for (int e = lane; e < 288; e += 32) {
            int r = e / 24, c = e % 24;
            M[r][c] = c < 12 ? (double)V[c*12 + r] : (c - 12 == r ? 1.0 : 0.0);
        }
        __syncwarp();
        bool ok = true;
        for (int c = 0; c < 12; c++) {
            // first row of largest magnitude in column c at or below the diagonal
            double best = lane >= c && lane < 12 ? fabs(M[lane][c]) : -1.0;
            int p = lane;
            for (int o = 16; o > 0; o >>= 1) {
                double ob = __shfl_xor_sync(0xffffffffu, best, o);
                int op = __shfl_xor_sync(0xffffffffu, p, o);
                if (ob > best || (ob == best && op < p)) { best = ob; p = op; }
            }
            if (M[p][c] == 0.0) { ok = false; break; }
            if (p != c && lane < 24) { double t = M[p][lane]; M[p][lane] = M[c][lane]; M[c][lane] = t; }
            __syncwarp();
            double iv = 1.0 / M[c][c];
            __syncwarp();
            if (lane < 24) M[c][lane] *= iv;
            __syncwarp();
            double f[12];
#pragma unroll
            for (int r = 0; r < 12; r++) f[r] = M[r][c];
            __syncwarp();
            if (lane < 24) {
                double mc = M[c][lane];
#pragma unroll
                for (int r = 0; r < 12; r++)
                    if (r != c && f[r] != 0.0) M[r][lane] -= f[r] * mc;
            }
            __syncwarp();
        }
        T* D = dinv + (long)b * 144;
        for (int e = lane; e < 144; e += 32) {
            int c = e / 12, r = e % 12;
            D[e] = (T)(ok ? M[r][12 + c] : (r == c ? 1.0 : 0.0));
        }
        __syncwarp();
    }
}

// per-scene ||g||^2
__global__ void k_grad_norm(int nb, const double* __restrict__ g, const int* __restrict__ bscene, double* gg) {
    long n = 12L * nb;
    for (long base = (long)blockIdx.x * blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        long i = base + threadIdx.x;
        bool valid = i < n;
        int s = valid ? bscene[i / 12] : 0;
        double v = valid ? g[i] * g[i] : 0.0;
        warp_reduce_add(gg, s, v, valid);
    }
}

// waits for the copy the last assembly queued (counters, block keys, done
// flags), not for the assembly kernels behind it
int eng_asm_wait(Engine* E) {
    if (!E->asm_pending) return ABD_OK;
    E->asm_pending = false;
    E->host_syncs++;
    CUDA_TRY(cudaEventSynchronize(E->ev_asm));
    E->keys_host = E->asm_direct;
    E->nnzb_host = E->hcnt->nkeys;   // may include the sentinel
    return ABD_OK;
}

int eng_sync_counters(Engine* E) {
    int rc = eng_asm_wait(E);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(E->hcnt, E->dcnt, sizeof(Counters), cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(eng_stream_sync(E));
    return ABD_OK;
}

int eng_grow_blocks(Engine* E, int need);

// the contact assembly with the autotuned launch shape: one warp per
// contact (2, 4 or 8 contacts per block) or one block of 64 / 128 threads per
// contact
template <class T>
static void launch_contact_assemble(Engine* E, int n, Geo G, double sc, T* V) {
    const AbdParams& P = E->P;
    cudaStream_t s = E->stream;
    int c = tune_begin(E, TK_CONTACT, 5, 1);
    const int threads = TUNE_CONTACT_THREADS[c], per_block = TUNE_CONTACT_PER_BLOCK[c];
    dim3 block(threads), grid(grid_for((long)n, per_block));
#define CA_ARGS E->dcnt, E->cst, E->ctype, E->cxb, G, P.barrier, P.dhat, sc, P.hess_mode, E->row_ptr, E->bcol, V, E->g
    if (c == 0) k_contact_assemble<T, 2><<<grid, block, 0, s>>>(CA_ARGS);
    else if (c == 2) k_contact_assemble<T, 8><<<grid, block, 0, s>>>(CA_ARGS);
    else if (c == 3) k_contact_assemble_team<T, 64><<<grid, block, 0, s>>>(CA_ARGS);
    else if (c == 4) k_contact_assemble_team<T, 128><<<grid, block, 0, s>>>(CA_ARGS);
    else k_contact_assemble<T, 4><<<grid, block, 0, s>>>(CA_ARGS);
#undef CA_ARGS
    tune_end(E, TK_CONTACT);
}

// Block keys: the diagonal and one pair per active contact, sorted and made
// unique, and for the direct solver their copy (with the done flags and the
// counters) to pinned host memory, where its component analysis reads them.
// Exact mode runs inside the assembly, sized by the contact count of the
// last sync, and records an event behind the copies (eng_asm_wait).  Ahead
// mode runs right after the next iterate's detection, before the
// end-of-iteration sync that then brings the keys back as well: the new
// count is not on the host yet, so the keys are sized for the current count
// plus a quarter and 256 (sentinels beyond the device count; a detection
// that found more contacts than that discards them, eng_keys_ahead_synced),
// and no event is needed.
static int asm_keys(Engine* E, bool ahead, long long& bound) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    Geo G = eng_geo(E);
    const int nb = E->nb;
    int rc;
    const int n_now = E->hcnt->n_total;
    const int n = ahead ? std::min(E->cap, n_now + n_now / 4 + 256) : n_now;
    if (ahead) E->keys_ahead_n = n;
    const int nkeys = nb + 2 * n;
    // room for every block before the count is known: the unique keys are
    // at most the nkeys written and at most every scene's dense pattern,
    // plus the sentinel
    bound = std::min<long long>(nkeys, E->dense_blocks) + 1;
    if (bound > E->blk_cap) { if ((rc = eng_grow_blocks(E, (int)bound))) return rc; }
    CUDA_TRY(cudaMemsetAsync(&E->dcnt->n_active, 0, sizeof(int), s));
    k_diag_keys<<<grid_for(nb), 256, 0, s>>>(nb, E->keys);
    k_contact_prepare<<<grid_for(n > 0 ? n : 1, 128), 128, 0, s>>>(E->dcnt, E->contacts, G, P.ee_f32, P.dhat, nb, E->cst,
                                                                   E->ctype, E->cxb, E->cbody, E->keys, &E->dcnt->n_active,
                                                                   ahead ? n : 0);
    int bits = 1;
    while (bits < 64 && ((unsigned long long)nb * nb) >> bits) bits++;
    size_t bytes = E->cub_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortKeys(E->cub_tmp, bytes, E->keys, E->keys_s, nkeys, 0, bits, s));
    bytes = E->cub_bytes;
    int* n_unique = &E->dcnt->nkeys;
    CUDA_TRY(cub::DeviceSelect::Unique(E->cub_tmp, bytes, E->keys_s, E->ukeys, n_unique, nkeys, s));
    E->launches += 4;
    E->keys_host = false;
    const int ls = E->P.linear_solver;
    const bool direct = ls == ABD_SOLVER_AUTO || ls == ABD_SOLVER_DIRECT;
    if (direct) {
        if (nkeys > E->h_ukeys_cap) {
            if (E->h_ukeys) cudaFreeHost(E->h_ukeys);
            E->h_ukeys = nullptr; E->h_ukeys_cap = 0;
            int cap = nkeys + nkeys / 2 + 1024;
            if (cudaMallocHost(&E->h_ukeys, sizeof(unsigned long long) * cap) != cudaSuccess)
                return E->fail(ABD_ERR_CUDA, "cudaMallocHost block keys");
            E->h_ukeys_cap = cap;
        }
        if (!E->h_done && cudaMallocHost(&E->h_done, sizeof(int) * E->ns) != cudaSuccess) {
            E->h_done = nullptr;
            return E->fail(ABD_ERR_CUDA, "cudaMallocHost done flags");
        }
        CUDA_TRY(cudaMemcpyAsync(E->h_ukeys, E->ukeys, sizeof(unsigned long long) * nkeys, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(E->h_done, E->sci + SI_DONE * E->ns, sizeof(int) * E->ns, cudaMemcpyDeviceToHost, s));
    }
    E->asm_direct = direct;
    if (!ahead) {
        CUDA_TRY(cudaMemcpyAsync(E->hcnt, E->dcnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaEventRecord(E->ev_asm, s));
        E->asm_pending = true;
    }
    return ABD_OK;
}

// the next iterate's block keys, queued before the end-of-iteration sync
int eng_assemble_keys_ahead(Engine* E) {
    long long bound = 0;
    int ph = phase_begin(E, PH_ASM_KEYS);
    int rc = asm_keys(E, true, bound);
    phase_end(E, ph, 0);
    if (rc) return rc;
    E->keys_ahead = true;
    E->keys_ahead_bound = bound;
    return ABD_OK;
}

// after the end-of-iteration sync: keys built ahead are on the host unless
// the detection they came from overflowed (then the assembly rebuilds them)
void eng_keys_ahead_synced(Engine* E) {
    if (!E->keys_ahead) return;
    if (E->hcnt->overflow || E->hcnt->n_total > E->keys_ahead_n) { E->keys_ahead = false; return; }
    E->keys_host = E->asm_direct;
    E->nnzb_host = E->hcnt->nkeys;   // may include the sentinel
}

int eng_assemble(Engine* E) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    Geo G = eng_geo(E);
    int nb = E->nb;
    int rc;
    // counters were synchronised by the caller after detection
    int n = E->hcnt->n_total;
    long long bound = 0;
    int ph = phase_begin(E, PH_ASM_KEYS);
    if (E->keys_ahead) {
        bound = E->keys_ahead_bound;      // keys, counters and host copies are there already
        E->keys_ahead = false;
    } else if ((rc = asm_keys(E, false, bound))) {
        return rc;
    }
    int* n_unique = &E->dcnt->nkeys;
    const long nnzb = bound;     // launch bound; the kernels read the count from the device
    k_block_rows<<<grid_for(nnzb), 256, 0, s>>>(nb, E->ukeys, n_unique, E->row_ptr, E->bcol, E->dcnt);
    phase_end(E, ph, 0);
    double sc = P.kappa * P.dt * P.dt;
    if (E->mixed) {
        float* V = (float*)E->vals;
        k_zero_vals<float><<<grid_for((long)nnzb * 144), 256, 0, s>>>(E->dcnt, V);
        k_body_assemble<float><<<grid_for(32L * nb, 32 * BA_WARPS), 32 * BA_WARPS, 0, s>>>(nb, E->st, E->mass, E->J, P.dt, P.gravity[0], P.gravity[1], P.gravity[2],
                                                               P.k_ortho, P.hess_mode == ABD_HESS_PROJECTED, P.pinned_diag,
                                                               E->row_ptr, E->bcol, V, E->g);
        if (n > 0)
            launch_contact_assemble<float>(E, n, G, sc, V);
        k_block_inverse<float><<<grid_for(32L * nb, 32 * BI_WARPS), 32 * BI_WARPS, 0, s>>>(nb, E->row_ptr, E->bcol, V, (float*)E->dinv);
    } else {
        double* V = (double*)E->vals;
        k_zero_vals<double><<<grid_for((long)nnzb * 144), 256, 0, s>>>(E->dcnt, V);
        int p1 = phase_begin(E, PH_ASM_BODY);
        k_body_assemble<double><<<grid_for(32L * nb, 32 * BA_WARPS), 32 * BA_WARPS, 0, s>>>(nb, E->st, E->mass, E->J, P.dt, P.gravity[0], P.gravity[1], P.gravity[2],
                                                                P.k_ortho, P.hess_mode == ABD_HESS_PROJECTED, P.pinned_diag,
                                                                E->row_ptr, E->bcol, V, E->g);
        phase_end(E, p1, 0);
        int p2 = phase_begin(E, PH_ASM_CONTACT);
        if (n > 0)
            launch_contact_assemble<double>(E, n, G, sc, V);
        if (E->timing && (rc = eng_asm_wait(E))) return rc;    // n_active for the phase's bytes
        // per candidate: type; per active contact: stencil, barrier argument,
        // 4 positions + 4 rest positions, 4 body blocks and the gradient rows
        phase_end(E, p2, 4.0 * n + E->hcnt->n_active * (16.0 + 8.0 + 96.0 + 96.0 + 4 * 1152.0 + 384.0));
        int p3 = phase_begin(E, PH_ASM_INV);
        k_block_inverse<double><<<grid_for(32L * nb, 32 * BI_WARPS), 32 * BI_WARPS, 0, s>>>(nb, E->row_ptr, E->bcol, V, (double*)E->dinv);
        phase_end(E, p3, 0);
    }
    double* gg = E->scd + SD_GG * E->ns;
    CUDA_TRY(cudaMemsetAsync(gg, 0, sizeof(double) * E->ns, s));
    k_grad_norm<<<grid_for(12L * nb), 256, 0, s>>>(nb, E->g, E->bscene, gg);
    E->launches += 6 + (n > 0);
    return ABD_OK;
}
