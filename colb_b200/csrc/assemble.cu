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
#include <cub/cub.cuh>

Geo eng_geo(Engine* E);

DV int stencil_np(int type) { return type == T_PP ? 2 : (type == T_PE ? 3 : (type == T_PG ? 1 : 4)); }
DV int other_vertex(int type, int4 s) { return type == T_EE ? s.z : (type == T_PG ? s.x : s.y); }

// ---------------------------------------------------------- prepare + keys
__global__ void k_contact_prepare(const Counters* cnt, const int4* __restrict__ contacts, Geo G, int f32, double dhat,
                                  int nb, int4* cst, int* ctype, double* cxb, int2* cbody,
                                  unsigned long long* keys, int* n_active) {
    int n = cnt->n_total;
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

DV int find_block(const int* row_ptr, const int* bcol, int r, int c) {
    int lo = row_ptr[r], hi = row_ptr[r+1] - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        int v = bcol[mid];
        if (v == c) return mid;
        if (v < c) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

template <class T>
__global__ void k_zero_vals(const Counters* cnt, T* vals) {
    long n = (long)cnt->nnzb * 144;
    GS_LOOP(i, n) vals[i] = (T)0;
}

// ---------------------------------------------------- inertia + ortho (abd.py:108-149)
template <class T>
__global__ void k_body_assemble(int nb, const double* __restrict__ st, const double* __restrict__ mass,
                                const double* __restrict__ J, double dt, double g0, double g1, double g2,
                                double k_ortho, int project, double pinned_diag, const int* __restrict__ row_ptr,
                                const int* __restrict__ bcol, T* vals, double* grad) {
    GS_LOOP(b, nb) {
        int bi = find_block(row_ptr, bcol, (int)b, (int)b);
        if (bi < 0) continue;                 // every row holds its diagonal key
        T* V = vals + (long)bi * 144;
        double* g = grad + 12 * b;
        double m = mass[b];
        if (m > 0.0) {
            const double* now = st + ST_STRIDE * b + ST_NOW; const double* nx = st + ST_STRIDE * b + ST_NXT;
            double q[9];
#pragma unroll
            for (int i = 0; i < 9; i++) q[i] = nx[ST_Q + i];
            double go[9]; ortho_grad(q, k_ortho, go);
            double gv[3] = {g0, g1, g2};
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double ct = now[ST_C+k] + dt * now[ST_V+k] + dt * dt * gv[k];
                g[k] = (nx[ST_C+k] - ct) * m;
            }
            double Jb = J[b];
#pragma unroll
            for (int r = 0; r < 9; r++) {
                double qt = now[ST_Q+r] + dt * now[ST_QD+r];
                g[3+r] = dt * dt * go[r] + (q[r] - qt) * Jb;
            }
            double H[81];
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
                for (int r = 0; r < 3; r++) for (int c = 0; c < 3; c++)
                    H[(3*i+r)*9 + 3*j+c] = ortho_hess(q, k_ortho, i, j, r, c) * dt * dt;
            if (project) psd_project(9, H);
            for (int c = 0; c < 12; c++)
                for (int r = 0; r < 12; r++) {
                    double v;
                    if (r < 3 || c < 3) v = (r == c) ? m : 0.0;
                    else v = H[(r-3)*9 + (c-3)] + (r == c ? Jb : 0.0);
                    V[c*12 + r] = (T)v;
                }
        } else {
            for (int k = 0; k < 12; k++) g[k] = 0.0;
            for (int c = 0; c < 12; c++) for (int r = 0; r < 12; r++) V[c*12 + r] = (T)(r == c ? pinned_diag : 0.0);
        }
    }
}

// ---------------------------------------------------- contacts (abd.py:198-571)
template <class T>
__global__ void k_contact_assemble(const Counters* cnt, const int4* __restrict__ cst, const int* __restrict__ ctype,
                                   const double* __restrict__ cxb, Geo G, int barrier, double dhat, double sc,
                                   int hess_mode, const int* __restrict__ row_ptr, const int* __restrict__ bcol,
                                   T* vals, double* grad) {
    int n = cnt->n_total;
    GS_LOOP(c, n) {
        int type = ctype[c];
        if (type < 0) continue;
        int4 s4 = cst[c];
        int sv[4] = {s4.x, s4.y, s4.z, s4.w};
        int np = stencil_np(type);
        int m = 3 * np;
        double g[12], H[144];
        if (type == T_PG) {
            const double* nrm = G.planes + 4 * s4.y;
            double d = nrm[0] * G.x[3*s4.x] + nrm[1] * G.x[3*s4.x+1] + nrm[2] * G.x[3*s4.x+2] - nrm[3];
            for (int r = 0; r < 3; r++) { g[r] = 2 * d * nrm[r]; for (int q = 0; q < 3; q++) H[r*3+q] = 2 * nrm[r] * nrm[q]; }
            sv[1] = -1;
        } else if (type == T_PP) {
            d2_pp_full(ld3(G.x + 3*sv[0]), ld3(G.x + 3*sv[1]), g, H);
        } else if (type == T_PE) {
            d2_pe_full(ld3(G.x + 3*sv[0]), ld3(G.x + 3*sv[1]), ld3(G.x + 3*sv[2]), g, H);
        } else if (type == T_EE) {
            d2_ee_line_full(ld3(G.x + 3*sv[0]), ld3(G.x + 3*sv[1]), ld3(G.x + 3*sv[2]), ld3(G.x + 3*sv[3]), g, H);
        } else {
            d2_pt_plane_full(ld3(G.x + 3*sv[0]), ld3(G.x + 3*sv[1]), ld3(G.x + 3*sv[2]), ld3(G.x + 3*sv[3]), g, H);
        }
        double B0, B1, B2;
        barrier3(barrier, cxb[c], dhat * dhat, B0, B1, B2);
        if (hess_mode == ABD_HESS_REFERENCE) {
            if (type == T_EE) psd_project(12, H);                     // abd.py:247
            for (int i = 0; i < m; i++)
                for (int j = 0; j < m; j++) {
                    double h = (type == T_PP) ? 0.0 : B1 * H[i*m+j];  // abd.py:381-382
                    H[i*m+j] = (h + B2 * g[i] * g[j]) * sc;
                }
        } else {
            for (int i = 0; i < m; i++)
                for (int j = 0; j < m; j++) H[i*m+j] = B1 * H[i*m+j] + B2 * g[i] * g[j];
            psd_project(m, H);
            for (int i = 0; i < m * m; i++) H[i] *= sc;
        }
        for (int i = 0; i < m; i++) g[i] *= B1 * sc;
        // gradient: G[b] += J_v^T g_v for dynamic bodies
        int vb[4]; double Jv[4][4];
        for (int i = 0; i < np; i++) {
            int v = sv[i];
            vb[i] = G.vbody[v];
            Jv[i][0] = 1.0; Jv[i][1] = G.xbar[3*v]; Jv[i][2] = G.xbar[3*v+1]; Jv[i][3] = G.xbar[3*v+2];
            if (!(G.mass[vb[i]] > 0.0)) continue;
            double* gb = grad + 12 * vb[i];
            for (int a = 0; a < 4; a++)
                for (int k = 0; k < 3; k++) atomicAdd(gb + 3*a + k, Jv[i][a] * g[3*i+k]);
        }
        // Hessian: distinct body pairs among the stencil (at most 2 bodies)
        int bodies[2] = {vb[0], vb[0]}; int nbd = 1;
        for (int i = 1; i < np; i++) if (vb[i] != bodies[0]) { bodies[1] = vb[i]; nbd = 2; break; }
        for (int pa = 0; pa < nbd; pa++)
            for (int pb = 0; pb < nbd; pb++) {
                int Ba = bodies[pa], Bb = bodies[pb];
                if (!(G.mass[Ba] > 0.0) || !(G.mass[Bb] > 0.0)) continue;
                int bi = find_block(row_ptr, bcol, Ba, Bb);
                if (bi < 0) continue;
                T* V = vals + (long)bi * 144;
                for (int al = 0; al < 4; al++)
                    for (int be = 0; be < 4; be++)
                        for (int r = 0; r < 3; r++)
                            for (int q = 0; q < 3; q++) {
                                double sum = 0;
                                for (int i = 0; i < np; i++) {
                                    if (vb[i] != Ba) continue;
                                    for (int j = 0; j < np; j++) {
                                        if (vb[j] != Bb) continue;
                                        sum += Jv[i][al] * Jv[j][be] * H[(3*i+r)*m + 3*j+q];
                                    }
                                }
                                if (sum != 0.0) atomicAdd(V + (3*be+q)*12 + 3*al+r, (T)sum);
                            }
            }
    }
}

// ---------------------------------------------------- block-Jacobi inverse
template <class T>
__global__ void k_block_inverse(int nb, const int* __restrict__ row_ptr, const int* __restrict__ bcol,
                                const T* __restrict__ vals, T* dinv) {
    GS_LOOP(b, nb) {
        int bi = find_block(row_ptr, bcol, (int)b, (int)b);
        if (bi < 0) continue;
        const T* V = vals + (long)bi * 144;
        double M[12][24];
        for (int r = 0; r < 12; r++)
            for (int c = 0; c < 24; c++) M[r][c] = c < 12 ? (double)V[c*12 + r] : (c - 12 == r ? 1.0 : 0.0);
        bool ok = true;
        for (int c = 0; c < 12 && ok; c++) {
            int p = c;
            for (int r = c + 1; r < 12; r++) if (fabs(M[r][c]) > fabs(M[p][c])) p = r;
            if (M[p][c] == 0.0) { ok = false; break; }
            if (p != c) for (int j = 0; j < 24; j++) { double t = M[p][j]; M[p][j] = M[c][j]; M[c][j] = t; }
            double iv = 1.0 / M[c][c];
            for (int j = 0; j < 24; j++) M[c][j] *= iv;
            for (int r = 0; r < 12; r++) if (r != c) {
                double f = M[r][c];
                if (f != 0.0) for (int j = 0; j < 24; j++) M[r][j] -= f * M[c][j];
            }
        }
        T* D = dinv + (long)b * 144;
        for (int c = 0; c < 12; c++)
            for (int r = 0; r < 12; r++) D[c*12 + r] = (T)(ok ? M[r][12 + c] : (r == c ? 1.0 : 0.0));
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

int eng_sync_counters(Engine* E) {
    CUDA_TRY(cudaMemcpyAsync(E->hcnt, E->dcnt, sizeof(Counters), cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    return ABD_OK;
}

int eng_grow_blocks(Engine* E, int need);

int eng_assemble(Engine* E) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    Geo G = eng_geo(E);
    int nb = E->nb;
    int rc;
    // counters were synchronised by the caller after detection
    int n = E->hcnt->n_total;
    int nkeys = nb + 2 * n;
    CUDA_TRY(cudaMemsetAsync(&E->dcnt->n_active, 0, sizeof(int), s));
    k_diag_keys<<<grid_for(nb), 256, 0, s>>>(nb, E->keys);
    k_contact_prepare<<<grid_for(n > 0 ? n : 1, 128), 128, 0, s>>>(E->dcnt, E->contacts, G, P.ee_f32, P.dhat, nb, E->cst,
                                                                   E->ctype, E->cxb, E->cbody, E->keys, &E->dcnt->n_active);
    int bits = 1;
    while (bits < 64 && ((unsigned long long)nb * nb) >> bits) bits++;
    size_t bytes = E->cub_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortKeys(E->cub_tmp, bytes, E->keys, E->keys_s, nkeys, 0, bits, s));
    bytes = E->cub_bytes;
    int* n_unique = &E->dcnt->nkeys;
    CUDA_TRY(cub::DeviceSelect::Unique(E->cub_tmp, bytes, E->keys_s, E->ukeys, n_unique, nkeys, s));
    E->launches += 4;
    if ((rc = eng_sync_counters(E))) return rc;
    int nnzb = E->hcnt->nkeys;   // may include the sentinel
    E->nnzb_host = nnzb;
    if (nnzb > E->blk_cap) { if ((rc = eng_grow_blocks(E, nnzb))) return rc; }
    k_block_rows<<<grid_for(nnzb), 256, 0, s>>>(nb, E->ukeys, n_unique, E->row_ptr, E->bcol, E->dcnt);
    double sc = P.kappa * P.dt * P.dt;
    if (E->mixed) {
        float* V = (float*)E->vals;
        k_zero_vals<float><<<grid_for((long)nnzb * 144), 256, 0, s>>>(E->dcnt, V);
        k_body_assemble<float><<<grid_for(nb, 64), 64, 0, s>>>(nb, E->st, E->mass, E->J, P.dt, P.gravity[0], P.gravity[1], P.gravity[2],
                                                               P.k_ortho, P.hess_mode == ABD_HESS_PROJECTED, P.pinned_diag,
                                                               E->row_ptr, E->bcol, V, E->g);
        if (n > 0)
            k_contact_assemble<float><<<grid_for(n, 64), 64, 0, s>>>(E->dcnt, E->cst, E->ctype, E->cxb, G, P.barrier, P.dhat, sc,
                                                                     P.hess_mode, E->row_ptr, E->bcol, V, E->g);
        k_block_inverse<float><<<grid_for(nb, 64), 64, 0, s>>>(nb, E->row_ptr, E->bcol, V, (float*)E->dinv);
    } else {
        double* V = (double*)E->vals;
        k_zero_vals<double><<<grid_for((long)nnzb * 144), 256, 0, s>>>(E->dcnt, V);
        k_body_assemble<double><<<grid_for(nb, 64), 64, 0, s>>>(nb, E->st, E->mass, E->J, P.dt, P.gravity[0], P.gravity[1], P.gravity[2],
                                                                P.k_ortho, P.hess_mode == ABD_HESS_PROJECTED, P.pinned_diag,
                                                                E->row_ptr, E->bcol, V, E->g);
        if (n > 0)
            k_contact_assemble<double><<<grid_for(n, 64), 64, 0, s>>>(E->dcnt, E->cst, E->ctype, E->cxb, G, P.barrier, P.dhat, sc,
                                                                      P.hess_mode, E->row_ptr, E->bcol, V, E->g);
        k_block_inverse<double><<<grid_for(nb, 64), 64, 0, s>>>(nb, E->row_ptr, E->bcol, V, (double*)E->dinv);
    }
    double* gg = E->scd + SD_GG * E->ns;
    CUDA_TRY(cudaMemsetAsync(gg, 0, sizeof(double) * E->ns, s));
    k_grad_norm<<<grid_for(12L * nb), 256, 0, s>>>(nb, E->g, E->bscene, gg);
    E->launches += 6 + (n > 0);
    return ABD_OK;
}
