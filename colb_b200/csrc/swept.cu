// swept.cu — one candidate list per Newton iteration for everything that
// looks at positions along the step.
//
// The reference re-runs full collision detection for every line-search
// trial (gauss_newton.py:98-115 -> abd.py:725-735 -> contact.py:270-279) and
// for the next Newton iteration.  Every one of those positions lies on the
// segment x(alpha) = x + alpha p, alpha in [0, 1], of the Newton step p.  So
// the library builds, once per step direction, the list of primitive pairs
// that can come within the candidate distance anywhere on that segment:
//   * boxes swept over [x, x + p], padded by half the candidate distance,
//     go through the hashed grid;
//   * a Lipschitz test drops pairs whose distance at alpha = 0 minus the
//     largest relative displacement already exceeds the candidate distance
//     (a point set moving by at most L changes its distance by at most L).
// CCD, every line-search energy, and the next iteration's candidate list are
// then evaluated over this list only.  The list is sorted by (kind, a, b),
// so filtering it yields the same sorted candidate list as a fresh
// detection.
#include "contact.cuh"
#include <cub/cub.cuh>

Geo eng_geo(Engine* E);
int eng_grow_swept(Engine* E, int need);

// displacement of each vertex for the step sign * dq; zero for pinned
// bodies and for scenes flagged done (they do not move in this step)
__global__ void k_vertex_disp2(int nv, const int* __restrict__ vbody, const double* __restrict__ xbar,
                               const double* __restrict__ dq, double sign, const double* __restrict__ mass,
                               const int* __restrict__ bscene, const int* __restrict__ done, double* p, float* pmag) {
    GS_LOOP(v, nv) {
        int b = vbody[v];
        const double* d = dq + 12 * b;
        double x0 = xbar[3*v], x1 = xbar[3*v+1], x2 = xbar[3*v+2];
        bool dyn = mass[b] > 0.0 && !done[bscene[b]];
        double q[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            q[k] = dyn ? sign * (d[k] + x0 * d[3+k] + x1 * d[6+k] + x2 * d[9+k]) : 0.0;
            p[3*v+k] = q[k];
        }
        pmag[v] = __double2float_ru(sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]));
    }
}

__global__ void k_sw_edge_boxes(int ne, const int2* __restrict__ edges, const double* __restrict__ x,
                                const double* __restrict__ p, const int* __restrict__ escene, float pad,
                                float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(e, ne) {
        int2 ed = edges[e];
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double a = x[3*ed.x+k], b = x[3*ed.y+k], a1 = a + p[3*ed.x+k], b1 = b + p[3*ed.y+k];
            l[k] = __fsub_rd(__double2float_rd(fmin(fmin(a, b), fmin(a1, b1))), pad);
            h[k] = __fadd_ru(__double2float_ru(fmax(fmax(a, b), fmax(a1, b1))), pad);
        }
        lo[e] = make_float4(l[0], l[1], l[2], 0.f); hi[e] = make_float4(h[0], h[1], h[2], 0.f); scene[e] = escene[e];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}
__global__ void k_sw_tri_boxes(int nt, const int* __restrict__ tris, const double* __restrict__ x,
                               const double* __restrict__ p, const int* __restrict__ tscene, float pad,
                               float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(t, nt) {
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double mn = 1e300, mx = -1e300;
            for (int q = 0; q < 3; q++) {
                int v = tris[3*t+q];
                double a = x[3*v+k], b = a + p[3*v+k];
                mn = fmin(mn, fmin(a, b)); mx = fmax(mx, fmax(a, b));
            }
            l[k] = __fsub_rd(__double2float_rd(mn), pad); h[k] = __fadd_ru(__double2float_ru(mx), pad);
        }
        lo[t] = make_float4(l[0], l[1], l[2], 0.f); hi[t] = make_float4(h[0], h[1], h[2], 0.f); scene[t] = tscene[t];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}
__global__ void k_sw_point_boxes(int nv, const double* __restrict__ x, const double* __restrict__ p,
                                 const int* __restrict__ vscene, float pad, float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(v, nv) {
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double a = x[3*v+k], b = a + p[3*v+k];
            l[k] = __fsub_rd(__double2float_rd(fmin(a, b)), pad); h[k] = __fadd_ru(__double2float_ru(fmax(a, b)), pad);
        }
        lo[v] = make_float4(l[0], l[1], l[2], 0.f); hi[v] = make_float4(h[0], h[1], h[2], 0.f); scene[v] = vscene[v];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}

// Lipschitz keep-test: distance at alpha = 0 minus the largest displacement
// of either primitive's points
DV bool ee_may_reach(const Geo& G, const float* pmag, int i, int j, double lim) {
    int2 a = G.edges[i], b = G.edges[j];
    double s, t, d;
    seg_seg_f64(G.x + 3*a.x, G.x + 3*a.y, G.x + 3*b.x, G.x + 3*b.y, 1e-12, s, t, d);
    double L = (double)fmaxf(pmag[a.x], pmag[a.y]) + (double)fmaxf(pmag[b.x], pmag[b.y]);
    return d - L < lim;
}
DV bool pt_may_reach(const Geo& G, const float* pmag, int p, int tr, double lim) {
    int a = G.tris[3*tr], b = G.tris[3*tr+1], c = G.tris[3*tr+2];
    double d = sqrt(pt_dist2(G.x + 3*p, G.x + 3*a, G.x + 3*b, G.x + 3*c));
    double L = (double)pmag[p] + (double)fmaxf(pmag[a], fmaxf(pmag[b], pmag[c]));
    return d - L < lim;
}

// mode 0 count, mode 1 write (sorted per query item)
__global__ void k_sw_ee(int ne, GridView GV, Geo G, const float* __restrict__ pmag, const float4* __restrict__ qlo,
                        const float4* __restrict__ qhi, const int* __restrict__ qscene, const int* __restrict__ skip,
                        int self_contact, double lim, int mode, int* qcount, const int* qoff, int cap, int4* out,
                        int* overflow) {
    GS_LOOP(i, ne) {
        int ii = (int)i, s = qscene[i];
        int c = 0;
        int base = mode == 1 ? qoff[i] : 0;
        if (!skip[s]) {
            grid_visit(GV, qlo[i], qhi[i], s, [&](int j) {
                if (j <= ii) return;
                int2 a = G.edges[ii], b = G.edges[j];
                if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return;
                if (!self_contact && G.vbody[a.x] == G.vbody[b.x]) return;
                if (!ee_may_reach(G, pmag, ii, j, lim)) return;
                if (mode == 1) { int at = base + c; if ((unsigned)at < (unsigned)cap) out[at] = make_int4(ABD_CONTACT_EE, ii, j, 0); else *overflow = 1; }
                c++;
            });
        }
        if (mode == 0) qcount[i] = c;
        else if (c > 1) {
            int lo = base, hi = min(base + c, cap);
            for (int k = lo + 1; k < hi; k++) { int4 v = out[k]; int m = k - 1; while (m >= lo && out[m].z > v.z) { out[m+1] = out[m]; m--; } out[m+1] = v; }
        }
    }
}
__global__ void k_sw_pt(int nv, GridView GV, Geo G, const float* __restrict__ pmag, const float4* __restrict__ qlo,
                        const float4* __restrict__ qhi, const int* __restrict__ qscene, const int* __restrict__ skip,
                        int self_contact, double lim, int mode, int* qcount, const int* qoff, const int* base_ee,
                        int cap, int4* out, int* overflow) {
    GS_LOOP(pi, nv) {
        int pp = (int)pi, s = qscene[pi];
        int c = 0;
        int base = mode == 1 ? *base_ee + qoff[pi] : 0;
        if (!skip[s]) {
            grid_visit(GV, qlo[pi], qhi[pi], s, [&](int t) {
                int a = G.tris[3*t];
                if (pp == a || pp == G.tris[3*t+1] || pp == G.tris[3*t+2]) return;
                if (!self_contact && G.vbody[pp] == G.vbody[a]) return;
                if (!pt_may_reach(G, pmag, pp, t, lim)) return;
                if (mode == 1) { int at = base + c; if ((unsigned)at < (unsigned)cap) out[at] = make_int4(ABD_CONTACT_PT, pp, t, 0); else *overflow = 1; }
                c++;
            });
        }
        if (mode == 0) qcount[pi] = c;
        else if (c > 1) {
            int lo = base, hi = min(base + c, cap);
            for (int k = lo + 1; k < hi; k++) { int4 v = out[k]; int m = k - 1; while (m >= lo && out[m].z > v.z) { out[m+1] = out[m]; m--; } out[m+1] = v; }
        }
    }
}
__global__ void k_sw_count(const int* off_ee, int ne, const int* off_pt, int npt, Counters* cnt, int cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int a = off_ee ? off_ee[ne] : 0, b = off_pt ? off_pt[npt] : 0;
        cnt->n_sw_ee = a; cnt->n_sw = a + b;
        // a scan whose sum passed the int range shows as a negative total
        if (a < 0 || b < 0 || (long long)a + b > cap) cnt->sw_overflow = 1;
    }
}

// Build the list for displacement p = sign * J dq from the current nxt state.
// Every scene is listed (scenes flagged `done` with zero displacement), so
// the list also covers the start of the next step.
int eng_swept(Engine* E, const double* dq, double sign, const int* done) {
    const int* skip = E->zero_ns;
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    int rc;
    double lim = P.cand_dist * (1.0 + 1e-6) + 1e-7;
    float pad = (float)(0.5 * lim);
    E->sw_scale = 1.0;
    if (eng_use_bp(E)) {
        if ((rc = eng_transform(E))) return rc;
        // a candidate list that does not fit even after growing (an increment
        // that sweeps most primitives into reach) is built for a quarter of
        // the step, then a sixteenth, ...; the line search then caps its step
        // length at that fraction (k_ls_init), so the list still covers every
        // position it visits
        for (double scale = 1.0;; scale *= 0.25) {
            k_vertex_disp2<<<grid_for(E->nv), 256, 0, s>>>(E->nv, E->vbody, E->xbar, dq, sign * scale, E->mass, E->bscene,
                                                            done, E->pv, E->pmag);
            E->launches++;
            if ((E->P.test_inject & ABD_INJECT_SWEPT_FULL) && !E->sw_inject_done && scale == 1.0) {
                E->sw_inject_done = true;        // test hook: the full step's list "does not fit"
                continue;
            }
            rc = eng_swept_bp(E, lim);
            if (rc == ABD_ERR_CONTACT_OVERFLOW && scale > 1e-6) { E->err.clear(); continue; }
            if (rc == ABD_OK) E->sw_scale = scale;
            return rc;
        }
    }
    for (;;) {
        if ((rc = eng_transform(E))) return rc;
        k_vertex_disp2<<<grid_for(E->nv), 256, 0, s>>>(E->nv, E->vbody, E->xbar, dq, sign, E->mass, E->bscene, done,
                                                        E->pv, E->pmag);
        E->launches++;
        CUDA_TRY(cudaMemsetAsync(&E->dcnt->n_sw, 0, sizeof(int) * 3, s));
        Geo G = eng_geo(E);
        int* off_ee = nullptr; int* off_pt = nullptr;
        if (P.contact_ee && E->ne > 1) {
            Grid& g = E->gee;
            CUDA_TRY(cudaMemsetAsync(g.cell, 0, sizeof(float), s));
            k_sw_edge_boxes<<<grid_for(g.n), 256, 0, s>>>(g.n, E->edges, E->x, E->pv, E->edge_scene, pad, g.lo, g.hi, g.scene, g.cell);
            E->launches++;
            if ((rc = eng_grid_build(E, g))) return rc;
            GridView v = eng_view(g);
            k_sw_ee<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, v, G, E->pmag, g.lo, g.hi, g.scene, skip, P.self_contact, lim, 0,
                                                          g.qcount, nullptr, E->sw_cap, E->sw, &E->dcnt->sw_overflow);
            CUDA_TRY(cudaMemsetAsync(g.qcount + E->ne, 0, sizeof(int), s));
            size_t bytes = E->cub_bytes;
            CUDA_TRY(cub::DeviceScan::ExclusiveSum(E->cub_tmp, bytes, g.qcount, g.qoff, E->ne + 1, s));
            k_sw_ee<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, v, G, E->pmag, g.lo, g.hi, g.scene, skip, P.self_contact, lim, 1,
                                                          g.qcount, g.qoff, E->sw_cap, E->sw, &E->dcnt->sw_overflow);
            E->launches += 3;
            off_ee = g.qoff;
        }
        if (P.contact_pt && E->nt > 0) {
            Grid& g = E->gpt;
            CUDA_TRY(cudaMemsetAsync(g.cell, 0, sizeof(float), s));
            k_sw_tri_boxes<<<grid_for(g.n), 256, 0, s>>>(g.n, E->tris, E->x, E->pv, E->tri_scene, pad, g.lo, g.hi, g.scene, g.cell);
            k_sw_point_boxes<<<grid_for(g.nq), 256, 0, s>>>(g.nq, E->x, E->pv, E->vscene, pad, g.qlo, g.qhi, g.qscene, g.cell);
            E->launches += 2;
            if ((rc = eng_grid_build(E, g))) return rc;
            GridView v = eng_view(g);
            const int* base_ee = off_ee ? off_ee + E->ne : E->zero_int;
            k_sw_pt<<<grid_for(E->nv, 128), 128, 0, s>>>(E->nv, v, G, E->pmag, g.qlo, g.qhi, g.qscene, skip, P.self_contact, lim, 0,
                                                          g.qcount, nullptr, base_ee, E->sw_cap, E->sw, &E->dcnt->sw_overflow);
            CUDA_TRY(cudaMemsetAsync(g.qcount + E->nv, 0, sizeof(int), s));
            size_t bytes = E->cub_bytes;
            CUDA_TRY(cub::DeviceScan::ExclusiveSum(E->cub_tmp, bytes, g.qcount, g.qoff, E->nv + 1, s));
            k_sw_pt<<<grid_for(E->nv, 128), 128, 0, s>>>(E->nv, v, G, E->pmag, g.qlo, g.qhi, g.qscene, skip, P.self_contact, lim, 1,
                                                          g.qcount, g.qoff, base_ee, E->sw_cap, E->sw, &E->dcnt->sw_overflow);
            E->launches += 3;
            off_pt = g.qoff;
        }
        k_sw_count<<<1, 32, 0, s>>>(off_ee, E->ne, off_pt, E->nv, E->dcnt, E->sw_cap);
        E->launches++;
        if ((rc = eng_sync_counters(E))) return rc;
        if (!E->hcnt->sw_overflow) break;
        if ((rc = eng_grow_swept(E, E->hcnt->n_sw))) return rc;
    }
    E->n_sw = E->hcnt->n_sw;
    E->n_sw_ee = E->hcnt->n_sw_ee;
    CUDA_TRY(cudaMemcpyAsync(E->sw_nee, &E->dcnt->n_sw_ee, sizeof(int), cudaMemcpyDeviceToDevice, s));
    E->sw_valid = true;
    return ABD_OK;
}

// ------------------------------------------------------------------ CCD over the list
__global__ void k_ccd_list(int n, const int4* __restrict__ list, Geo G, const double* __restrict__ p,
                           const int* __restrict__ bscene, const int* __restrict__ skip, double s_ccd, int ccd_it,
                           double* toi, int* capped) {
    GS_LOOP(c, n) {
        int4 C = list[c];
        int v[4];
        int kind;
        if (C.x == ABD_CONTACT_EE) { int2 a = G.edges[C.y], b = G.edges[C.z]; v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; kind = 0; }
        else { v[0] = C.y; v[1] = G.tris[3*C.z]; v[2] = G.tris[3*C.z+1]; v[3] = G.tris[3*C.z+2]; kind = 1; }
        int s = bscene[G.vbody[v[0]]];
        if (skip[s]) continue;
        double xx[12], pp[12];
        for (int k = 0; k < 4; k++) for (int q = 0; q < 3; q++) { xx[3*k+q] = G.x[3*v[k]+q]; pp[3*k+q] = p[3*v[k]+q]; }
        double t;
        if (accd(kind, xx, pp, s_ccd, 1.0, &t, capped, ccd_it)) atomic_min_pos(toi + s, t);
    }
}
// planes come from the vertex's scene; the bound goes to the unit of its body
__global__ void k_ccd_pg2(int nv, Geo G, const double* __restrict__ p, const int* __restrict__ vscene,
                          const int* __restrict__ bunit, double s_ccd, const int* skip, double* toi) {
    GS_LOOP(v, nv) {
        int s = vscene[v];
        int u = bunit[G.vbody[v]];
        if (skip[u]) continue;
        double best = 1.0;
        for (int pl = G.sc_plane_begin[s]; pl < G.sc_plane_begin[s+1]; pl++) {
            const double* n = G.planes + 4*pl;
            double d = n[0] * G.x[3*v] + n[1] * G.x[3*v+1] + n[2] * G.x[3*v+2] - n[3];
            double vn = n[0] * p[3*v] + n[1] * p[3*v+1] + n[2] * p[3*v+2];
            if (vn < 0) { double t = (1 - s_ccd) * d / (-vn); if (t < 0) t = 0; if (t < best) best = t; }
        }
        if (best < 1.0) atomic_min_pos(toi + u, best);
    }
}
__global__ void k_fill1(double* a, int n, double v) { GS_LOOP(i, n) a[i] = v; }

// per-unit (scene or contact group) largest conservative fraction of the
// listed displacement (E->pv) into U's SD_TOI slots
int eng_ccd_list(Engine* E, const LsUnits& U, const int* skip) {
    cudaStream_t s = E->stream;
    double* toi = U.d + SD_TOI * U.n;
    k_fill1<<<grid_for(U.n), 256, 0, s>>>(toi, U.n, 1.0);
    int rc = eng_transform(E);
    if (rc) return rc;
    Geo G = eng_geo(E);
    if (E->n_sw > 0)
        k_ccd_list<<<grid_for(E->n_sw, 64), 64, 0, s>>>(E->n_sw, E->sw, G, E->pv, U.bunit, skip, E->P.ccd_scale,
                                                        ccd_iters(E->P), toi, &E->dcnt->ccd_capped);
    if (E->npl > 0) k_ccd_pg2<<<grid_for(E->nv), 256, 0, s>>>(E->nv, G, E->pv, E->vscene, U.bunit, E->P.ccd_scale, skip, toi);
    E->launches += 1 + (E->n_sw > 0) + (E->npl > 0);
    return ABD_OK;
}

// ------------------------------------------------------------------ energy over the list
__global__ void k_list_energy(int n, const int* __restrict__ n_dev, const int4* __restrict__ list, Geo G,
                              const int* __restrict__ bscene, const int* __restrict__ skip, int f32, double dhat,
                              int barrier, double sc, double* Eo, double* En) {
    if (n_dev) n = *n_dev;
    for (long base = (long)blockIdx.x * blockDim.x; base < n; base += (long)gridDim.x * blockDim.x) {
        long c = base + threadIdx.x;
        bool valid = c < n;
        int s = 0;
        double e = 0, en = 0;
        if (valid) {
            int4 C = list[c];
            int v0 = C.x == ABD_CONTACT_EE ? G.edges[C.y].x : C.y;
            s = bscene[G.vbody[v0]];
            if (skip[s]) valid = false;
            else {
                int4 stv; int type; double xb;
                if (classify(G, C.x, C.y, C.z, f32, dhat, stv, type, xb)) {
                    double b0, b1, b2; barrier3(barrier, xb, dhat * dhat, b0, b1, b2);
                    e = b0 * sc;
                    int vs[4] = {stv.x, stv.y, stv.z, stv.w};
                    double L = 0;
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (vs[k] >= 0)
                            L = fmax(L, fmax(fabs(G.x[3*vs[k]]), fmax(fabs(G.x[3*vs[k]+1]), fabs(G.x[3*vs[k]+2]))));
                    // FP32 distances carry 2^29 times the FP64 rounding
                    en = contact_noise(sc, b0, b1, xb, L, (f32 && C.x == ABD_CONTACT_EE) ? 536870912.0 : 1.0) * DBL_EPSILON;
                }
            }
        }
        warp_reduce_add(Eo, s, e, valid);
        warp_reduce_add(En, s, en, valid);
    }
}

int eng_body_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip);
int eng_pg_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip);

// energy per unit (scene or contact group) into U's slot and the scale of
// its FP64 evaluation error into the noise slot (SD_E0 -> SD_E0N,
// SD_E1 -> SD_E1N)
int eng_energy_list(Engine* E, const LsUnits& U, int slot, const int* skip, bool dev_count) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    double* Eo = U.d + slot * U.n;
    double* En = U.d + (slot == SD_E0 ? SD_E0N : SD_E1N) * U.n;
    CUDA_TRY(cudaMemsetAsync(Eo, 0, sizeof(double) * U.n, s));
    CUDA_TRY(cudaMemsetAsync(En, 0, sizeof(double) * U.n, s));
    int rc = eng_transform(E);
    if (rc) return rc;
    if ((rc = eng_body_energy(E, U.bunit, Eo, En, skip))) return rc;
    if (E->n_sw > 0 || dev_count) {
        int ph = phase_begin(E, PH_ELIST);
        int tb = TUNE_THREADS[tune_begin(E, TK_LIST_ENERGY, 4, 1)];
        const int grid = dev_count ? NUM_SMS * 4 : grid_for(E->n_sw, tb);
        k_list_energy<<<grid, tb, 0, s>>>(E->n_sw, dev_count ? &E->dcnt->ls_nsw : nullptr, E->sw, eng_geo(E), U.bunit,
                                          skip, P.ee_f32, P.dhat, P.barrier, P.kappa * P.dt * P.dt, Eo, En);
        tune_end(E, TK_LIST_ENERGY);
        // per listed pair: the entry, its 2-4 vertex ids and positions
        phase_end(E, ph, E->n_sw * (16.0 + 16.0 + 4 * 24.0));
        E->launches++;
    }
    return eng_pg_energy(E, U.bunit, Eo, En, skip);
}

// ------------------------------------------------------------------ detection from the list
__global__ void k_list_flags(int n, const int4* __restrict__ list, Geo G, int f32, int self_contact, double cand,
                             int* flag) {
    GS_LOOP(c, n) {
        int4 C = list[c];
        bool keep;
        if (C.x == ABD_CONTACT_EE) { double s, t, d; keep = ee_test(G, C.y, C.z, f32, self_contact, cand, s, t, d); }
        else keep = pt_test(G, C.y, C.z, self_contact, cand);
        flag[c] = keep ? 1 : 0;
    }
}
__global__ void k_list_scatter(int n, const int4* __restrict__ list, const int* __restrict__ flag, const int* __restrict__ off,
                               int4* out, const int* __restrict__ n_ee_dev, Counters* cnt, int cap) {
    const int n_ee_list = *n_ee_dev;
    GS_LOOP(c, n) {
        if (flag[c]) { int at = off[c]; if ((unsigned)at < (unsigned)cap) out[at] = list[c]; }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        cnt->n_ee = off[n_ee_list];
        cnt->n_pt = off[n] - off[n_ee_list];
    }
}

int eng_pg_candidates(Engine* E, double filt);

// candidate list at the current nxt state from the swept list; the list
// must cover the current positions (built for the step that led here)
int eng_detect_list(Engine* E) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    int rc = eng_transform(E);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(E->dcnt, 0, DETECT_COUNTER_BYTES, s));
    int n = E->n_sw;
    if (n > 0) {
        Geo G = eng_geo(E);
        int* flag = E->sw_flag;
        int* off = E->sw_off;
        k_list_flags<<<grid_for(n), 256, 0, s>>>(n, E->sw, G, P.ee_f32, P.self_contact, P.cand_dist, flag);
        CUDA_TRY(cudaMemsetAsync(flag + n, 0, sizeof(int), s));
        size_t bytes = E->cub_bytes;
        CUDA_TRY(cub::DeviceScan::ExclusiveSum(E->cub_tmp, bytes, flag, off, n + 1, s));
        k_list_scatter<<<grid_for(n), 256, 0, s>>>(n, E->sw, flag, off, E->contacts, E->sw_nee, E->dcnt, E->cap);
        E->launches += 3;
    }
    return eng_pg_candidates(E, P.cand_dist);
}
