// detect.cu — vertex transform, uniform-grid broad phase, candidate pairs,
// contact energy, CCD and the intersection check.
//
//  transform ............ abd_simple.py:26-35
//  EE candidates ........ contact.py:25-32, :143-169 (float32 predicate, i<j,
//                         no shared vertex, distance < (thickness+buffer)*2)
//  PT / half-space ...... no reference counterpart
//  contact energy ....... abd.py:66-75
//
// The reference refits a Warp LBVH and appends pairs with an atomic counter
// (unordered, capacity 10000 with wrap-around).  Here every detection
// rebuilds a hashed uniform grid (one radix sort), counts pairs per query
// item, scans, and writes each item's pairs in index order, so the list is
// sorted and exact-size; overflow is reported instead of wrapping.
#include "contact.cuh"
#include <cub/cub.cuh>

// ------------------------------------------------------------------ transform
__global__ void k_transform(int nv, const double* __restrict__ xbar, const int* __restrict__ vbody,
                            const double* __restrict__ st, double* __restrict__ x, float4* __restrict__ xf) {
    GS_LOOP(v, nv) {
        const double* s = st + (long)ST_STRIDE * vbody[v] + ST_NXT;
        double xb0 = xbar[3*v], xb1 = xbar[3*v+1], xb2 = xbar[3*v+2];
        double o[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double t = s[ST_C + k];
            t = __fma_rn(s[ST_Q + 0 + k], xb0, t);
            t = __fma_rn(s[ST_Q + 3 + k], xb1, t);
            t = __fma_rn(s[ST_Q + 6 + k], xb2, t);
            o[k] = t;
        }
        x[3*v] = o[0]; x[3*v+1] = o[1]; x[3*v+2] = o[2];
        xf[v] = make_float4(__double2float_rn(o[0]), __double2float_rn(o[1]), __double2float_rn(o[2]), 0.f);
    }
}

int eng_body_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip);
int eng_pg_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip);
int eng_pg_candidates(Engine* E, double filt);

int eng_transform(Engine* E) {
    k_transform<<<grid_for(E->nv), 256, 0, E->stream>>>(E->nv, E->xbar, E->vbody, E->st, E->x, E->xf);
    E->launches++;
    return ABD_OK;
}

// ------------------------------------------------------------------ boxes
DV float f_rd(double v) { return __double2float_rd(v); }
DV float f_ru(double v) { return __double2float_ru(v); }

// Edge boxes, both stored and queried.  f32 mode boxes the float copies
// exactly; f64 mode rounds outward.  pad is added on every side.
__global__ void k_edge_boxes(int ne, const int2* __restrict__ edges, const double* __restrict__ x,
                             const float4* __restrict__ xf, const int* __restrict__ escene, float pad, int f32,
                             float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(e, ne) {
        int2 ed = edges[e];
        float l[3], h[3];
        if (f32) {
            float4 a = xf[ed.x], b = xf[ed.y];
            l[0] = fminf(a.x, b.x); l[1] = fminf(a.y, b.y); l[2] = fminf(a.z, b.z);
            h[0] = fmaxf(a.x, b.x); h[1] = fmaxf(a.y, b.y); h[2] = fmaxf(a.z, b.z);
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double a = x[3*ed.x+k], b = x[3*ed.y+k];
                l[k] = f_rd(fmin(a, b)); h[k] = f_ru(fmax(a, b));
            }
        }
        float4 L = make_float4(__fsub_rd(l[0], pad), __fsub_rd(l[1], pad), __fsub_rd(l[2], pad), 0.f);
        float4 Hh = make_float4(__fadd_ru(h[0], pad), __fadd_ru(h[1], pad), __fadd_ru(h[2], pad), 0.f);
        lo[e] = L; hi[e] = Hh; scene[e] = escene[e];
        ext = fmaxf(ext, fmaxf(Hh.x - L.x, fmaxf(Hh.y - L.y, Hh.z - L.z)));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}

__global__ void k_tri_boxes(int nt, const int* __restrict__ tris, const double* __restrict__ x,
                            const int* __restrict__ tscene, float pad, float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(t, nt) {
        int a = tris[3*t], b = tris[3*t+1], c = tris[3*t+2];
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double va = x[3*a+k], vb = x[3*b+k], vc = x[3*c+k];
            l[k] = __fsub_rd(f_rd(fmin(va, fmin(vb, vc))), pad);
            h[k] = __fadd_ru(f_ru(fmax(va, fmax(vb, vc))), pad);
        }
        lo[t] = make_float4(l[0], l[1], l[2], 0.f); hi[t] = make_float4(h[0], h[1], h[2], 0.f); scene[t] = tscene[t];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}

__global__ void k_point_boxes(int nv, const double* __restrict__ x, const int* __restrict__ vscene, float pad,
                              float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(v, nv) {
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) { l[k] = __fsub_rd(f_rd(x[3*v+k]), pad); h[k] = __fadd_ru(f_ru(x[3*v+k]), pad); }
        lo[v] = make_float4(l[0], l[1], l[2], 0.f); hi[v] = make_float4(h[0], h[1], h[2], 0.f); scene[v] = vscene[v];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}

// swept boxes of a displacement p (vertex array, 3 doubles each)
__global__ void k_swept_edge_boxes(int ne, const int2* __restrict__ edges, const double* __restrict__ x,
                                   const double* __restrict__ p, const int* __restrict__ escene,
                                   float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(e, ne) {
        int2 ed = edges[e];
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double a = x[3*ed.x+k], b = x[3*ed.y+k], a1 = a + p[3*ed.x+k], b1 = b + p[3*ed.y+k];
            l[k] = __fsub_rd(f_rd(fmin(fmin(a, b), fmin(a1, b1))), 1e-6f);
            h[k] = __fadd_ru(f_ru(fmax(fmax(a, b), fmax(a1, b1))), 1e-6f);
        }
        lo[e] = make_float4(l[0], l[1], l[2], 0.f); hi[e] = make_float4(h[0], h[1], h[2], 0.f); scene[e] = escene[e];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}
__global__ void k_swept_tri_boxes(int nt, const int* __restrict__ tris, const double* __restrict__ x,
                                  const double* __restrict__ p, const int* __restrict__ tscene,
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
            l[k] = __fsub_rd(f_rd(mn), 1e-6f); h[k] = __fadd_ru(f_ru(mx), 1e-6f);
        }
        lo[t] = make_float4(l[0], l[1], l[2], 0.f); hi[t] = make_float4(h[0], h[1], h[2], 0.f); scene[t] = tscene[t];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}
__global__ void k_swept_point_boxes(int nv, const double* __restrict__ x, const double* __restrict__ p,
                                    const int* __restrict__ vscene, float4* lo, float4* hi, int* scene, float* cell) {
    float ext = 0.f;
    GS_LOOP(v, nv) {
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double a = x[3*v+k], b = a + p[3*v+k];
            l[k] = __fsub_rd(f_rd(fmin(a, b)), 1e-6f); h[k] = __fadd_ru(f_ru(fmax(a, b)), 1e-6f);
        }
        lo[v] = make_float4(l[0], l[1], l[2], 0.f); hi[v] = make_float4(h[0], h[1], h[2], 0.f); scene[v] = vscene[v];
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}

// ------------------------------------------------------------------ grid build
__global__ void k_grid_keys(int n, const float4* __restrict__ lo, const int* __restrict__ scene, float* cell,
                            uint32_t mask, uint32_t* keys, int* vals) {
    float h = fmaxf(*cell, 1e-6f);
    GS_LOOP(i, n) {
        float4 l = lo[i];
        uint32_t key = cell_hash(scene[i], (int)floorf(l.x / h), (int)floorf(l.y / h), (int)floorf(l.z / h)) & mask;
        keys[i] = key; vals[i] = (int)i;
    }
}
__global__ void k_cell_floor(float* cell) { if (threadIdx.x == 0 && blockIdx.x == 0) *cell = fmaxf(*cell, 1e-6f); }
__global__ void k_grid_ranges(int n, const uint32_t* __restrict__ keys, int* bstart, int* bend) {
    GS_LOOP(i, n) {
        uint32_t k = keys[i];
        if (i == 0 || keys[i-1] != k) bstart[k] = (int)i;
        if (i == n - 1 || keys[i+1] != k) bend[k] = (int)i + 1;
    }
}

int eng_grid_build(Engine* E, Grid& G) {
    if (G.n == 0) return ABD_OK;
    cudaStream_t s = E->stream;
    k_cell_floor<<<1, 32, 0, s>>>(G.cell);
    k_grid_keys<<<grid_for(G.n), 256, 0, s>>>(G.n, G.lo, G.scene, G.cell, (uint32_t)(G.H - 1), G.keys, G.vals);
    size_t bytes = E->cub_bytes;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(E->cub_tmp, bytes, G.keys, G.keys_s, G.vals, G.vals_s, G.n, 0, G.bits, s));
    CUDA_TRY(cudaMemsetAsync(G.bstart, 0xFF, sizeof(int) * G.H, s));
    k_grid_ranges<<<grid_for(G.n), 256, 0, s>>>(G.n, G.keys_s, G.bstart, G.bend);
    E->launches += 4;
    return ABD_OK;
}
GridView eng_view(const Grid& G) {
    return GridView{G.lo, G.hi, G.scene, G.cell, G.vals_s, G.bstart, G.bend, (uint32_t)(G.H - 1)};
}

// ------------------------------------------------------------------ pair queries
// mode 0: count into qcount; mode 1: write sorted pairs at qoff + base
__global__ void k_ee_pairs(int ne, GridView GV, Geo G, const float4* __restrict__ qlo, const float4* __restrict__ qhi,
                           const int* __restrict__ qscene, int f32, int self_contact, double filt, int mode,
                           int* qcount, const int* qoff, int base_slot, const Counters* cnt, int cap,
                           int4* out, int* overflow) {
    GS_LOOP(i, ne) {
        int c = 0;
        int base = 0;
        if (mode == 1) {
            base = (base_slot == 0 ? 0 : cnt->n_ee) + qoff[i];
        }
        int ii = (int)i;
        grid_visit(GV, qlo[i], qhi[i], qscene[i], [&](int j) {
            if (j <= ii) return;
            double s, t, d;
            if (!ee_test(G, ii, j, f32, self_contact, filt, s, t, d)) return;
            if (mode == 1) {
                int at = base + c;
                if ((unsigned)at < (unsigned)cap) out[at] = make_int4(ABD_CONTACT_EE, ii, j, 0);
                else *overflow = 1;
            }
            c++;
        });
        if (mode == 0) qcount[i] = c;
        else if (c > 1) {
            // insertion sort of this item's segment by partner index
            int lo = base, hi = min(base + c, cap);
            for (int k = lo + 1; k < hi; k++) {
                int4 v = out[k]; int m = k - 1;
                while (m >= lo && out[m].z > v.z) { out[m+1] = out[m]; m--; }
                out[m+1] = v;
            }
        }
    }
}

__global__ void k_pt_pairs(int nv, GridView GV, Geo G, const float4* __restrict__ qlo, const float4* __restrict__ qhi,
                           const int* __restrict__ qscene, int self_contact, double filt, int mode,
                           int* qcount, const int* qoff, const Counters* cnt, int cap, int4* out, int* overflow) {
    GS_LOOP(p, nv) {
        int c = 0, base = 0;
        if (mode == 1) base = cnt->n_ee + qoff[p];
        int pp = (int)p;
        grid_visit(GV, qlo[p], qhi[p], qscene[p], [&](int t) {
            if (!pt_test(G, pp, t, self_contact, filt)) return;
            if (mode == 1) {
                int at = base + c;
                if ((unsigned)at < (unsigned)cap) out[at] = make_int4(ABD_CONTACT_PT, pp, t, 0);
                else *overflow = 1;
            }
            c++;
        });
        if (mode == 0) qcount[p] = c;
        else if (c > 1) {
            int lo = base, hi = min(base + c, cap);
            for (int k = lo + 1; k < hi; k++) {
                int4 v = out[k]; int m = k - 1;
                while (m >= lo && out[m].z > v.z) { out[m+1] = out[m]; m--; }
                out[m+1] = v;
            }
        }
    }
}

// half-space candidates: per vertex over its scene's planes
__global__ void k_pg_pairs(int nv, Geo G, const int* __restrict__ vscene, double filt, int mode,
                           int* qcount, const int* qoff, const Counters* cnt, int cap, int4* out, int* overflow) {
    GS_LOOP(v, nv) {
        int s = vscene[v];
        int p0 = G.sc_plane_begin[s], p1 = G.sc_plane_begin[s+1];
        int c = 0, base = 0;
        if (mode == 1) base = cnt->n_ee + cnt->n_pt + qoff[v];
        for (int pl = p0; pl < p1; pl++) {
            const double* n = G.planes + 4*pl;
            double d = n[0] * G.x[3*v] + n[1] * G.x[3*v+1] + n[2] * G.x[3*v+2] - n[3];
            if (!(d < filt)) continue;
            if (mode == 1) {
                int at = base + c;
                if ((unsigned)at < (unsigned)cap) out[at] = make_int4(ABD_CONTACT_PG, (int)v, pl, 0);
                else *overflow = 1;
            }
            c++;
        }
        if (mode == 0) qcount[v] = c;
    }
}

__global__ void k_store_count(const int* qoff, int n, int slot, Counters* cnt) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int v = qoff[n];
        if (slot == 0) cnt->n_ee = v;
        else if (slot == 1) cnt->n_pt = v;
        else cnt->n_pg = v;
    }
}
__global__ void k_finalize_counts(Counters* cnt, int cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int n = cnt->n_ee + cnt->n_pt + cnt->n_pg;
        cnt->n_total = n;
        if (n > cap) cnt->overflow = 1;
    }
}

static Geo geo(Engine* E) {
    return Geo{E->x, E->xf, E->edges, E->tris, E->vbody, E->bscene, E->planes, E->sc_plane_begin, E->mass, E->xbar};
}

static int scan_counts(Engine* E, int* qcount, int* qoff, int n) {
    size_t bytes = E->cub_bytes;
    CUDA_TRY(cub::DeviceScan::ExclusiveSum(E->cub_tmp, bytes, qcount, qoff, n + 1, E->stream));
    E->launches++;
    return ABD_OK;
}

// Build the EE grid (edges stored and queried) at the current positions.
static int build_ee_grid(Engine* E, double filt) {
    Grid& G = E->gee;
    if (G.n == 0) return ABD_OK;
    float pad = (float)(0.5 * filt * (1.0 + 1e-6) + 1e-7);
    CUDA_TRY(cudaMemsetAsync(G.cell, 0, sizeof(float), E->stream));
    k_edge_boxes<<<grid_for(G.n), 256, 0, E->stream>>>(G.n, E->edges, E->x, E->xf, E->edge_scene, pad, E->P.ee_f32,
                                                       G.lo, G.hi, G.scene, G.cell);
    E->launches++;
    return eng_grid_build(E, G);
}
static int build_pt_grid(Engine* E, double filt) {
    Grid& G = E->gpt;
    if (G.n == 0) return ABD_OK;
    float pad = (float)(0.5 * filt * (1.0 + 1e-6) + 1e-7);
    CUDA_TRY(cudaMemsetAsync(G.cell, 0, sizeof(float), E->stream));
    k_tri_boxes<<<grid_for(G.n), 256, 0, E->stream>>>(G.n, E->tris, E->x, E->tri_scene, pad, G.lo, G.hi, G.scene, G.cell);
    k_point_boxes<<<grid_for(G.nq), 256, 0, E->stream>>>(G.nq, E->x, E->vscene, pad, G.qlo, G.qhi, G.qscene, G.cell);
    E->launches += 2;
    return eng_grid_build(E, G);
}

int eng_detect(Engine* E, double filt) {
    int rc;
    cudaStream_t s = E->stream;
    if ((rc = eng_transform(E))) return rc;
    CUDA_TRY(cudaMemsetAsync(E->dcnt, 0, DETECT_COUNTER_BYTES, s));
    Geo G = geo(E);
    int f32 = E->P.ee_f32, sc = E->P.self_contact;
    if (E->P.contact_ee && E->ne > 1) {
        if ((rc = build_ee_grid(E, filt))) return rc;
        Grid& g = E->gee;
        k_ee_pairs<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, eng_view(g), G, g.lo, g.hi, g.scene, f32, sc, filt, 0,
                                                         g.qcount, nullptr, 0, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        CUDA_TRY(cudaMemsetAsync(g.qcount + E->ne, 0, sizeof(int), s));
        if ((rc = scan_counts(E, g.qcount, g.qoff, E->ne))) return rc;
        k_store_count<<<1, 32, 0, s>>>(g.qoff, E->ne, 0, E->dcnt);
        k_ee_pairs<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, eng_view(g), G, g.lo, g.hi, g.scene, f32, sc, filt, 1,
                                                         g.qcount, g.qoff, 0, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        E->launches += 3;
    }
    if (E->P.contact_pt && E->nt > 0) {
        if ((rc = build_pt_grid(E, filt))) return rc;
        Grid& g = E->gpt;
        k_pt_pairs<<<grid_for(E->nv, 128), 128, 0, s>>>(E->nv, eng_view(g), G, g.qlo, g.qhi, g.qscene, sc, filt, 0,
                                                         g.qcount, nullptr, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        CUDA_TRY(cudaMemsetAsync(g.qcount + E->nv, 0, sizeof(int), s));
        if ((rc = scan_counts(E, g.qcount, g.qoff, E->nv))) return rc;
        k_store_count<<<1, 32, 0, s>>>(g.qoff, E->nv, 1, E->dcnt);
        k_pt_pairs<<<grid_for(E->nv, 128), 128, 0, s>>>(E->nv, eng_view(g), G, g.qlo, g.qhi, g.qscene, sc, filt, 1,
                                                         g.qcount, g.qoff, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        E->launches += 3;
    }
    return eng_pg_candidates(E, filt);
}

// half-space candidates appended after EE and PT, then the total
int eng_pg_candidates(Engine* E, double filt) {
    cudaStream_t s = E->stream;
    int rc;
    if (E->npl > 0) {
        Geo G = geo(E);
        // reuse the PT query buffers for the per-vertex plane counts
        int* qc = E->gpt.qcount; int* qo = E->gpt.qoff;
        k_pg_pairs<<<grid_for(E->nv), 256, 0, s>>>(E->nv, G, E->vscene, filt, 0, qc, nullptr, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        CUDA_TRY(cudaMemsetAsync(qc + E->nv, 0, sizeof(int), s));
        if ((rc = scan_counts(E, qc, qo, E->nv))) return rc;
        k_store_count<<<1, 32, 0, s>>>(qo, E->nv, 2, E->dcnt);
        k_pg_pairs<<<grid_for(E->nv), 256, 0, s>>>(E->nv, G, E->vscene, filt, 1, qc, qo, E->dcnt, E->cap, E->contacts, &E->dcnt->overflow);
        E->launches += 3;
    }
    k_finalize_counts<<<1, 32, 0, s>>>(E->dcnt, E->cap);
    E->launches++;
    return ABD_OK;
}

// ------------------------------------------------------------------ energies
__global__ void k_body_energy(int nb, const double* __restrict__ st, const double* __restrict__ mass,
                              const double* __restrict__ J, const int* __restrict__ bscene, double dt,
                              double g0, double g1, double g2, double k_ortho, const int* done, double* E,
                              double* En) {
    for (long base = (long)blockIdx.x * blockDim.x; base < nb; base += (long)gridDim.x * blockDim.x) {
        long b = base + threadIdx.x;
        bool valid = b < nb;
        int s = valid ? bscene[b] : 0;
        double e = 0, en = 0;
        if (valid && !done[s]) {
            const double* now = st + ST_STRIDE * b + ST_NOW; const double* nx = st + ST_STRIDE * b + ST_NXT;
            double eo = ortho_energy(nx + ST_Q, k_ortho);
            double gv[3] = {g0, g1, g2};
            double n0 = 0, n1 = 0, s0 = 0, s1 = 0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                double ct = now[ST_C+k] + dt * now[ST_V+k] + dt * dt * gv[k];
                double d = nx[ST_C+k] - ct; n0 += d * d;
                s0 += fabs(d) * (fabs(nx[ST_C+k]) + fabs(ct));
            }
#pragma unroll
            for (int r = 0; r < 9; r++) {
                double qt = now[ST_Q+r] + dt * now[ST_QD+r];
                double d = nx[ST_Q+r] - qt; n1 += d * d;
                s1 += fabs(d) * (fabs(nx[ST_Q+r]) + fabs(qt));
            }
            e = eo * dt * dt + 0.5 * (n0 * mass[b] + n1 * J[b]);
            if (En) en = (e + s0 * fabs(mass[b]) + s1 * fabs(J[b]) + dt * dt * ortho_noise(nx + ST_Q, k_ortho)) * DBL_EPSILON;
        } else valid = false;
        warp_reduce_add(E, s, e, valid);
        if (En) warp_reduce_add(En, s, en, valid);
    }
}

// contact energy at the current positions: kappa dt^2 b(x) over active pairs
__global__ void k_ee_energy(int ne, GridView GV, Geo G, const float4* __restrict__ qlo, const float4* __restrict__ qhi,
                            const int* __restrict__ qscene, int f32, int self_contact, double dhat, int barrier,
                            double sc, const int* done, double* E) {
    for (long base = (long)blockIdx.x * blockDim.x; base < ne; base += (long)gridDim.x * blockDim.x) {
        long i = base + threadIdx.x;
        bool valid = i < ne;
        int s = valid ? qscene[i] : 0;
        double e = 0;
        if (valid && !done[s]) {
            int ii = (int)i;
            double xh = dhat * dhat;
            grid_visit(GV, qlo[i], qhi[i], s, [&](int j) {
                if (j <= ii) return;
                int2 ea = G.edges[ii], eb = G.edges[j];
                if (ea.x == eb.x || ea.x == eb.y || ea.y == eb.x || ea.y == eb.y) return;
                if (!self_contact && G.vbody[ea.x] == G.vbody[eb.x]) return;
                int4 stv; int type; double xb;
                if (!classify(G, ABD_CONTACT_EE, ii, j, f32, dhat, stv, type, xb)) return;
                double b0, b1, b2; barrier3(barrier, xb, xh, b0, b1, b2);
                e += b0 * sc;
            });
        } else valid = false;
        warp_reduce_add(E, s, e, valid);
    }
}
__global__ void k_pt_energy(int nv, GridView GV, Geo G, const float4* __restrict__ qlo, const float4* __restrict__ qhi,
                            const int* __restrict__ qscene, int self_contact, double dhat, int barrier, double sc,
                            const int* done, double* E) {
    for (long base = (long)blockIdx.x * blockDim.x; base < nv; base += (long)gridDim.x * blockDim.x) {
        long p = base + threadIdx.x;
        bool valid = p < nv;
        int s = valid ? qscene[p] : 0;
        double e = 0;
        if (valid && !done[s]) {
            int pp = (int)p;
            double xh = dhat * dhat;
            grid_visit(GV, qlo[p], qhi[p], s, [&](int t) {
                int ta = G.tris[3*t];
                if (pp == ta || pp == G.tris[3*t+1] || pp == G.tris[3*t+2]) return;
                if (!self_contact && G.vbody[pp] == G.vbody[ta]) return;
                int4 stv; int type; double xb;
                if (!classify(G, ABD_CONTACT_PT, pp, t, 0, dhat, stv, type, xb)) return;
                double b0, b1, b2; barrier3(barrier, xb, xh, b0, b1, b2);
                e += b0 * sc;
            });
        } else valid = false;
        warp_reduce_add(E, s, e, valid);
    }
}
// planes come from the vertex's scene; the energy goes to the unit of its body
__global__ void k_pg_energy(int nv, Geo G, const int* __restrict__ vscene, const int* __restrict__ bunit, double dhat,
                            int barrier, double sc, const int* done, double* E, double* En) {
    for (long base = (long)blockIdx.x * blockDim.x; base < nv; base += (long)gridDim.x * blockDim.x) {
        long v = base + threadIdx.x;
        bool valid = v < nv;
        int s = valid ? vscene[v] : 0;
        int u = valid ? bunit[G.vbody[v]] : 0;
        double e = 0, en = 0;
        if (valid && !done[u]) {
            double xh = dhat * dhat;
            double L = fmax(fabs(G.x[3*v]), fmax(fabs(G.x[3*v+1]), fabs(G.x[3*v+2])));
            for (int pl = G.sc_plane_begin[s]; pl < G.sc_plane_begin[s+1]; pl++) {
                const double* n = G.planes + 4*pl;
                double d = n[0] * G.x[3*v] + n[1] * G.x[3*v+1] + n[2] * G.x[3*v+2] - n[3];
                if (!(d < dhat)) continue;
                double b0, b1, b2; barrier3(barrier, d * d, xh, b0, b1, b2);
                e += b0 * sc;
                en += contact_noise(sc, b0, b1, d * d, fmax(L, fabs(n[3])), 1.0) * DBL_EPSILON;
            }
        } else valid = false;
        warp_reduce_add(E, u, e, valid);
        if (En) warp_reduce_add(En, u, en, valid);
    }
}

// energy per scene into scd[slot]; scenes flagged in sci[SI_ACC] (accepted)
// or sci[SI_DONE] are skipped via the `skip` array argument
static int energy_impl(Engine* E, int slot, const int* skip) {
    cudaStream_t s = E->stream;
    int rc;
    double* Eo = E->scd + slot * E->ns;
    CUDA_TRY(cudaMemsetAsync(Eo, 0, sizeof(double) * E->ns, s));
    if ((rc = eng_transform(E))) return rc;
    const AbdParams& P = E->P;
    if ((rc = eng_body_energy(E, E->bscene, Eo, nullptr, skip))) return rc;
    double sc = P.kappa * P.dt * P.dt;
    Geo G = geo(E);
    if (P.contact_ee && E->ne > 1) {
        if ((rc = build_ee_grid(E, P.dhat))) return rc;
        Grid& g = E->gee;
        int ph = phase_begin(E, PH_EQUERY);
        k_ee_energy<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, eng_view(g), G, g.lo, g.hi, g.scene, P.ee_f32, P.self_contact,
                                                          P.dhat, P.barrier, sc, skip, Eo);
        // edges, their boxes/scene, sorted values, bucket table, positions
        phase_end(E, ph, E->ne * (8.0 + 32.0 + 4.0 + 4.0) + g.H * 8.0 + E->nv * (P.ee_f32 ? 16.0 : 24.0));
        E->launches++;
    }
    if (P.contact_pt && E->nt > 0) {
        if ((rc = build_pt_grid(E, P.dhat))) return rc;
        Grid& g = E->gpt;
        int ph = phase_begin(E, PH_EQUERY);
        k_pt_energy<<<grid_for(E->nv, 128), 128, 0, s>>>(E->nv, eng_view(g), G, g.qlo, g.qhi, g.qscene, P.self_contact, P.dhat,
                                                          P.barrier, sc, skip, Eo);
        // points and their boxes, triangles, their boxes/scene, sorted values, buckets, positions
        phase_end(E, ph, E->nv * (32.0 + 4.0 + 24.0) + E->nt * (12.0 + 32.0 + 4.0 + 4.0) + g.H * 8.0);
        E->launches++;
    }
    return eng_pg_energy(E, E->bscene, Eo, nullptr, skip);
}
// En (may be null) accumulates the scale of the FP64 evaluation error
int eng_body_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip) {
    const AbdParams& P = E->P;
    int tb = TUNE_THREADS[tune_begin(E, TK_BODY_ENERGY, 4, 2)];
    k_body_energy<<<grid_for(E->nb, tb), tb, 0, E->stream>>>(E->nb, E->st, E->mass, E->J, bunit, P.dt, P.gravity[0],
                                                            P.gravity[1], P.gravity[2], P.k_ortho, skip, Eo, En);
    tune_end(E, TK_BODY_ENERGY);
    E->launches++;
    return ABD_OK;
}
int eng_pg_energy(Engine* E, const int* bunit, double* Eo, double* En, const int* skip) {
    const AbdParams& P = E->P;
    if (E->npl > 0) {
        k_pg_energy<<<grid_for(E->nv), 256, 0, E->stream>>>(E->nv, geo(E), E->vscene, bunit, P.dhat, P.barrier,
                                                            P.kappa * P.dt * P.dt, skip, Eo, En);
        E->launches++;
    }
    return ABD_OK;
}
int eng_energy(Engine* E, int slot) { return energy_impl(E, slot, E->sci + SI_DONE * E->ns); }
int eng_energy_masked(Engine* E, int slot, const int* skip) { return energy_impl(E, slot, skip); }

// ------------------------------------------------------------------ CCD
__global__ void k_vertex_disp(int nv, const int* __restrict__ vbody, const double* __restrict__ xbar,
                              const double* __restrict__ dq, double sign, const double* __restrict__ mass,
                              double* p) {
    GS_LOOP(v, nv) {
        int b = vbody[v];
        const double* d = dq + 12 * b;
        double x0 = xbar[3*v], x1 = xbar[3*v+1], x2 = xbar[3*v+2];
        bool dyn = mass[b] > 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++)
            p[3*v+k] = dyn ? sign * (d[k] + x0 * d[3+k] + x1 * d[6+k] + x2 * d[9+k]) : 0.0;
    }
}

__global__ void k_ccd_ee(int ne, GridView GV, Geo G, const double* __restrict__ p, const float4* __restrict__ qlo,
                         const float4* __restrict__ qhi, const int* __restrict__ qscene, int self_contact,
                         double s_ccd, int ccd_it, const int* done, double* toi, int* capped) {
    GS_LOOP(i, ne) {
        int s = qscene[i];
        if (done[s]) continue;
        int ii = (int)i;
        double best = 1.0;
        grid_visit(GV, qlo[i], qhi[i], s, [&](int j) {
            if (j <= ii) return;
            int2 a = G.edges[ii], b = G.edges[j];
            if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return;
            if (!self_contact && G.vbody[a.x] == G.vbody[b.x]) return;
            int v[4] = {a.x, a.y, b.x, b.y};
            double xx[12], pp[12];
            for (int k = 0; k < 4; k++) for (int c = 0; c < 3; c++) { xx[3*k+c] = G.x[3*v[k]+c]; pp[3*k+c] = p[3*v[k]+c]; }
            double t;
            if (accd(0, xx, pp, s_ccd, best, &t, capped, ccd_it) && t < best) best = t;
        });
        if (best < 1.0) atomic_min_pos(toi + s, best);
    }
}
__global__ void k_ccd_pt(int nv, GridView GV, Geo G, const double* __restrict__ p, const float4* __restrict__ qlo,
                         const float4* __restrict__ qhi, const int* __restrict__ qscene, int self_contact,
                         double s_ccd, int ccd_it, const int* done, double* toi, int* capped) {
    GS_LOOP(pi, nv) {
        int s = qscene[pi];
        if (done[s]) continue;
        int pp0 = (int)pi;
        double best = 1.0;
        grid_visit(GV, qlo[pi], qhi[pi], s, [&](int t) {
            int a = G.tris[3*t], b = G.tris[3*t+1], c = G.tris[3*t+2];
            if (pp0 == a || pp0 == b || pp0 == c) return;
            if (!self_contact && G.vbody[pp0] == G.vbody[a]) return;
            int v[4] = {pp0, a, b, c};
            double xx[12], pp[12];
            for (int k = 0; k < 4; k++) for (int q = 0; q < 3; q++) { xx[3*k+q] = G.x[3*v[k]+q]; pp[3*k+q] = p[3*v[k]+q]; }
            double tt;
            if (accd(1, xx, pp, s_ccd, best, &tt, capped, ccd_it) && tt < best) best = tt;
        });
        if (best < 1.0) atomic_min_pos(toi + s, best);
    }
}
__global__ void k_ccd_pg(int nv, Geo G, const double* __restrict__ p, const int* __restrict__ vscene, double s_ccd,
                         const int* done, double* toi) {
    GS_LOOP(v, nv) {
        int s = vscene[v];
        if (done[s]) continue;
        double best = 1.0;
        for (int pl = G.sc_plane_begin[s]; pl < G.sc_plane_begin[s+1]; pl++) {
            const double* n = G.planes + 4*pl;
            double d = n[0] * G.x[3*v] + n[1] * G.x[3*v+1] + n[2] * G.x[3*v+2] - n[3];
            double vn = n[0] * p[3*v] + n[1] * p[3*v+1] + n[2] * p[3*v+2];
            if (vn < 0) { double t = (1 - s_ccd) * d / (-vn); if (t < 0) t = 0; if (t < best) best = t; }
        }
        if (best < 1.0) atomic_min_pos(toi + s, best);
    }
}
__global__ void k_fill(double* a, int n, double v) { GS_LOOP(i, n) a[i] = v; }

// per-scene largest step fraction along x -> x + sign * J dq
int eng_ccd(Engine* E, const double* dq, double sign) {
    cudaStream_t s = E->stream;
    int rc;
    double* toi = E->scd + SD_TOI * E->ns;
    k_fill<<<grid_for(E->ns), 256, 0, s>>>(toi, E->ns, 1.0);
    if ((rc = eng_transform(E))) return rc;
    k_vertex_disp<<<grid_for(E->nv), 256, 0, s>>>(E->nv, E->vbody, E->xbar, dq, sign, E->mass, E->pv);
    E->launches += 2;
    const AbdParams& P = E->P;
    const int* done = E->sci + SI_DONE * E->ns;
    Geo G = geo(E);
    if (P.contact_ee && E->ne > 1) {
        Grid& g = E->gee;
        CUDA_TRY(cudaMemsetAsync(g.cell, 0, sizeof(float), s));
        k_swept_edge_boxes<<<grid_for(g.n), 256, 0, s>>>(g.n, E->edges, E->x, E->pv, E->edge_scene, g.lo, g.hi, g.scene, g.cell);
        E->launches++;
        if ((rc = eng_grid_build(E, g))) return rc;
        k_ccd_ee<<<grid_for(E->ne, 64), 64, 0, s>>>(E->ne, eng_view(g), G, E->pv, g.lo, g.hi, g.scene, P.self_contact, P.ccd_scale,
                                                    ccd_iters(P), done, toi, &E->dcnt->ccd_capped);
        E->launches++;
    }
    if (P.contact_pt && E->nt > 0) {
        Grid& g = E->gpt;
        CUDA_TRY(cudaMemsetAsync(g.cell, 0, sizeof(float), s));
        k_swept_tri_boxes<<<grid_for(g.n), 256, 0, s>>>(g.n, E->tris, E->x, E->pv, E->tri_scene, g.lo, g.hi, g.scene, g.cell);
        k_swept_point_boxes<<<grid_for(g.nq), 256, 0, s>>>(g.nq, E->x, E->pv, E->vscene, g.qlo, g.qhi, g.qscene, g.cell);
        E->launches += 2;
        if ((rc = eng_grid_build(E, g))) return rc;
        k_ccd_pt<<<grid_for(E->nv, 64), 64, 0, s>>>(E->nv, eng_view(g), G, E->pv, g.qlo, g.qhi, g.qscene, P.self_contact, P.ccd_scale,
                                                    ccd_iters(P), done, toi, &E->dcnt->ccd_capped);
        E->launches++;
    }
    if (E->npl > 0) {
        k_ccd_pg<<<grid_for(E->nv), 256, 0, s>>>(E->nv, G, E->pv, E->vscene, P.ccd_scale, done, toi);
        E->launches++;
    }
    return ABD_OK;
}

// ------------------------------------------------------------------ intersections
DV double orient3(d3 a, d3 b, d3 c, d3 d) { return dot(cross(b - a, c - a), d - a); }
__global__ void k_intersections(int ne, GridView GV, Geo G, const float4* __restrict__ qlo, const float4* __restrict__ qhi,
                                const int* __restrict__ qscene, int* count) {
    GS_LOOP(e, ne) {
        int2 ed = G.edges[e];
        d3 P = ld3(G.x + 3*ed.x), Q = ld3(G.x + 3*ed.y);
        int be = G.vbody[ed.x];
        int c = 0;
        grid_visit(GV, qlo[e], qhi[e], qscene[e], [&](int t) {
            int a = G.tris[3*t], b = G.tris[3*t+1], cc = G.tris[3*t+2];
            if (G.vbody[a] == be) return;
            d3 A = ld3(G.x + 3*a), B = ld3(G.x + 3*b), C = ld3(G.x + 3*cc);
            double o1 = orient3(A, B, C, P), o2 = orient3(A, B, C, Q);
            if ((o1 > 0 && o2 > 0) || (o1 < 0 && o2 < 0) || (o1 == 0 && o2 == 0)) return;
            double s1 = orient3(P, Q, A, B), s2 = orient3(P, Q, B, C), s3 = orient3(P, Q, C, A);
            if ((s1 > 0 && s2 > 0 && s3 > 0) || (s1 < 0 && s2 < 0 && s3 < 0)) c++;
        });
        if (c) atomicAdd(count, c);
    }
}
int eng_intersections(Engine* E, int* count) {
    *count = 0;
    if (E->nt == 0 || E->ne == 0) return ABD_OK;
    cudaStream_t s = E->stream;
    int rc;
    if ((rc = eng_transform(E))) return rc;
    Grid& g = E->gpt;   // triangles stored; edge boxes as queries (in the EE grid's box arrays)
    CUDA_TRY(cudaMemsetAsync(g.cell, 0, sizeof(float), s));
    CUDA_TRY(cudaMemsetAsync(&E->dcnt->nkeys, 0, sizeof(int), s));
    k_tri_boxes<<<grid_for(g.n), 256, 0, s>>>(g.n, E->tris, E->x, E->tri_scene, 0.f, g.lo, g.hi, g.scene, g.cell);
    Grid& q = E->gee;
    k_edge_boxes<<<grid_for(q.n), 256, 0, s>>>(q.n, E->edges, E->x, E->xf, E->edge_scene, 0.f, 0, q.lo, q.hi, q.scene, g.cell);
    if ((rc = eng_grid_build(E, g))) return rc;
    k_intersections<<<grid_for(E->ne, 128), 128, 0, s>>>(E->ne, eng_view(g), geo(E), q.lo, q.hi, q.scene, &E->dcnt->nkeys);
    E->launches += 3;
    CUDA_TRY(cudaMemcpyAsync(E->hcnt, E->dcnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CUDA_TRY(eng_stream_sync(E));
    *count = E->hcnt->nkeys;
    return ABD_OK;
}

// exported for assemble.cu
Geo eng_geo(Engine* E) { return geo(E); }
