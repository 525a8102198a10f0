// bpair.cu — two-level broad phase: bodies first, then primitives of each
// overlapping body pair staged in shared memory.
//
// Affine bodies are rigid-ish meshes whose primitives are mostly surrounded
// by primitives of the same body, which never pair with them when
// self-contact is off.  A uniform grid over primitives therefore spends its
// time rejecting same-body neighbours.  Here:
//   1. one warp per body reduces the body's swept, padded box;
//   2. one warp per body A tests A against every later body B of its scene
//      (and A against itself when self-contact is on) and appends the
//      overlapping pairs;
//   3. one CTA per body pair stages the primitives of A and of B whose boxes
//      touch the two bodies' box overlap into shared memory (block
//      compaction), tests all staged pairs, and appends hits;
//   4. hits are sorted by a 64-bit (kind, a, b) key, so the list comes out
//      in the same canonical order as the grid-based detection.
// Step 3 runs the reference's pair predicate (contact.py:158-168) in
// `detect` mode, or the Lipschitz reachability test along a step (see
// swept.cu) in `swept` mode.  Bodies must own contiguous vertex, edge and
// triangle ranges (as geometry.py:31-73 lays them out).
#include "contact.cuh"
#include <cub/cub.cuh>

Geo eng_geo(Engine* E);
int eng_grow_swept(Engine* E, int need);
int eng_grow_contacts(Engine* E, int need);
int eng_pg_candidates(Engine* E, double filt);

#define BP_CHUNK 1024
#define BP_THREADS 256

DV float4 fmin4(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.f); }
DV float4 fmax4(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), 0.f); }
DV bool overlap(float4 al, float4 ah, float4 bl, float4 bh) {
    return !(al.x > bh.x || ah.x < bl.x || al.y > bh.y || ah.y < bl.y || al.z > bh.z || ah.z < bl.z);
}

// swept (x .. x+p) padded box of one vertex, outward rounded
DV void vbox(const double* x, const double* p, int v, float pad, float4& lo, float4& hi) {
    double a0 = x[3*v], a1 = x[3*v+1], a2 = x[3*v+2];
    double b0 = a0, b1 = a1, b2 = a2;
    if (p) { b0 += p[3*v]; b1 += p[3*v+1]; b2 += p[3*v+2]; }
    lo = make_float4(__fsub_rd(__double2float_rd(fmin(a0, b0)), pad), __fsub_rd(__double2float_rd(fmin(a1, b1)), pad),
                     __fsub_rd(__double2float_rd(fmin(a2, b2)), pad), 0.f);
    hi = make_float4(__fadd_ru(__double2float_ru(fmax(a0, b0)), pad), __fadd_ru(__double2float_ru(fmax(a1, b1)), pad),
                     __fadd_ru(__double2float_ru(fmax(a2, b2)), pad), 0.f);
}

// 1. body boxes: one warp per body over its vertices; with vlo/vhi given,
// every vertex's box is kept too (the primitive boxes of the pair tests are
// the min/max over their vertices' boxes, exact in float)
__global__ void k_body_boxes(int nb, const int* __restrict__ vbeg, const double* __restrict__ x, const double* __restrict__ p,
                             float pad, float4* blo, float4* bhi, float4* vlo = nullptr, float4* vhi = nullptr) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    for (int b = warp; b < nb; b += (gridDim.x * blockDim.x) >> 5) {
        float4 lo = make_float4(3e38f, 3e38f, 3e38f, 0.f), hi = make_float4(-3e38f, -3e38f, -3e38f, 0.f);
        for (int v = vbeg[b] + lane; v < vbeg[b+1]; v += 32) {
            float4 l, h; vbox(x, p, v, pad, l, h);
            if (vlo) { vlo[v] = l; vhi[v] = h; }
            lo = fmin4(lo, l); hi = fmax4(hi, h);
        }
        for (int o = 16; o > 0; o >>= 1) {
            lo.x = fminf(lo.x, __shfl_xor_sync(0xffffffffu, lo.x, o)); lo.y = fminf(lo.y, __shfl_xor_sync(0xffffffffu, lo.y, o));
            lo.z = fminf(lo.z, __shfl_xor_sync(0xffffffffu, lo.z, o)); hi.x = fmaxf(hi.x, __shfl_xor_sync(0xffffffffu, hi.x, o));
            hi.y = fmaxf(hi.y, __shfl_xor_sync(0xffffffffu, hi.y, o)); hi.z = fmaxf(hi.z, __shfl_xor_sync(0xffffffffu, hi.z, o));
        }
        if (lane == 0) { blo[b] = lo; bhi[b] = hi; }
    }
}

// 2. body pairs (a <= b, same scene); a == b only with self-contact
__global__ void k_body_pairs(int nb, const int* __restrict__ bscene, const int* __restrict__ sc_body_begin,
                             const float4* __restrict__ blo, const float4* __restrict__ bhi, int self_contact,
                             int2* out, int cap, int* count) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    for (int a = warp; a < nb; a += (gridDim.x * blockDim.x) >> 5) {
        int s = bscene[a];
        int end = sc_body_begin[s + 1];
        float4 al = blo[a], ah = bhi[a];
        for (int b = a + (self_contact ? 0 : 1) + lane; b < end; b += 32) {
            if (!overlap(al, ah, blo[b], bhi[b])) continue;
            int at = atomicAdd(count, 1);
            if ((unsigned)at < (unsigned)cap) out[at] = make_int2(a, b);
        }
    }
}

// block-wide compaction of an index range into shared memory
template <class BoxFn>
DV int stage(int begin, int end, float4 rlo, float4 rhi, BoxFn box, int* idx, float4* lo, float4* hi, int* scount) {
    if (threadIdx.x == 0) *scount = 0;
    __syncthreads();
    for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
        float4 l, h; box(i, l, h);
        if (overlap(l, h, rlo, rhi)) {
            int at = atomicAdd(scount, 1);
            if (at < BP_CHUNK) { idx[at] = i; lo[at] = l; hi[at] = h; }
        }
    }
    __syncthreads();
    int n = min(*scount, BP_CHUNK);
    __syncthreads();     // everyone has read the count before it can be reset
    return n;
}

struct BpArgs {
    Geo G; const double* p; const float* pmag;
    const float4* vlo; const float4* vhi;          // per-vertex swept boxes of this build
    const int* ebeg; const int* tbeg; const int* vbeg;
    const float4* blo; const float4* bhi;
    float pad; double lim; double filt; int mode;   // mode 0 swept (Lipschitz, lim), 1 detect (predicate, filt)
    int f32; int self_contact; int do_ee; int do_pt;
    unsigned long long* out; int cap; int* count;
};

DV bool bp_ee_ok(const BpArgs& A, int i, int j) {
    const Geo& G = A.G;
    int2 a = G.edges[i], b = G.edges[j];
    if (a.x == b.x || a.x == b.y || a.y == b.x || a.y == b.y) return false;
    if (A.mode == 1) { double s, t, d; return ee_test(G, i, j, A.f32, 1, A.filt, s, t, d); }
    double s, t, d;
    seg_seg_f64(G.x + 3*a.x, G.x + 3*a.y, G.x + 3*b.x, G.x + 3*b.y, 1e-12, s, t, d);
    double L = (double)fmaxf(A.pmag[a.x], A.pmag[a.y]) + (double)fmaxf(A.pmag[b.x], A.pmag[b.y]);
    return d - L < A.lim;
}
DV bool bp_pt_ok(const BpArgs& A, int pv, int t) {
    const Geo& G = A.G;
    int a = G.tris[3*t], b = G.tris[3*t+1], c = G.tris[3*t+2];
    if (pv == a || pv == b || pv == c) return false;
    if (A.mode == 1) return pt_test(G, pv, t, 1, A.filt);
    double d = sqrt(pt_dist2(G.x + 3*pv, G.x + 3*a, G.x + 3*b, G.x + 3*c));
    double L = (double)A.pmag[pv] + (double)fmaxf(A.pmag[a], fmaxf(A.pmag[b], A.pmag[c]));
    return d - L < A.lim;
}
// the hit counter stops growing once it passes the capacity (by at most the
// threads in flight), so a pathological step (a displacement that makes every
// primitive pair reachable) cannot wrap it; the host then grows the buffer a
// bounded number of times and reports ABD_ERR_CONTACT_OVERFLOW
DV void bp_emit(const BpArgs& A, int kind, int a, int b) {
    if (*(volatile int*)A.count >= A.cap) return;
    int at = atomicAdd(A.count, 1);
    if ((unsigned)at < (unsigned)A.cap) A.out[at] = ((unsigned long long)kind << 62) | ((unsigned long long)a << 31) | (unsigned long long)b;
}

// 3. one CTA per body pair
__global__ void __launch_bounds__(BP_THREADS) k_bp_prims(const int2* __restrict__ bpairs, const int* __restrict__ npairs,
                                                        int bp_cap, BpArgs A) {
    extern __shared__ float4 smem[];
    float4* alo = smem;                  float4* ahi = alo + BP_CHUNK;
    float4* blo = ahi + BP_CHUNK;        float4* bhi = blo + BP_CHUNK;
    int* aidx = reinterpret_cast<int*>(bhi + BP_CHUNK);
    int* bidx = aidx + BP_CHUNK;
    __shared__ int sa, sb;
    const Geo& G = A.G;
    const float pad = A.pad;
    int n = min(*npairs, bp_cap);      // an overflowing pair list is rebuilt larger by the host
    for (int q = blockIdx.x; q < n; q += gridDim.x) {
        int2 bp = bpairs[q];
        int ba = bp.x, bb = bp.y;
        float4 rlo = fmax4(A.blo[ba], A.blo[bb]), rhi = fmin4(A.bhi[ba], A.bhi[bb]);
        const float4* __restrict__ vlo = A.vlo;
        const float4* __restrict__ vhi = A.vhi;
        auto ebox = [&](int e, float4& l, float4& h) {
            int2 ed = G.edges[e];
            l = fmin4(__ldg(vlo + ed.x), __ldg(vlo + ed.y)); h = fmax4(__ldg(vhi + ed.x), __ldg(vhi + ed.y));
        };
        auto tbox = [&](int t, float4& l, float4& h) {
            const int v0 = G.tris[3*t], v1 = G.tris[3*t+1], v2 = G.tris[3*t+2];
            l = fmin4(__ldg(vlo + v0), fmin4(__ldg(vlo + v1), __ldg(vlo + v2)));
            h = fmax4(__ldg(vhi + v0), fmax4(__ldg(vhi + v1), __ldg(vhi + v2)));
        };
        auto pbox = [&](int v, float4& l, float4& h) { l = __ldg(vlo + v); h = __ldg(vhi + v); };
        // ---- edge-edge
        if (A.do_ee) {
            for (int a0 = A.ebeg[ba]; a0 < A.ebeg[ba+1]; a0 += BP_CHUNK) {
                int na = stage(a0, min(a0 + BP_CHUNK, A.ebeg[ba+1]), rlo, rhi, ebox, aidx, alo, ahi, &sa);
                if (na == 0) continue;
                for (int b0 = A.ebeg[bb]; b0 < A.ebeg[bb+1]; b0 += BP_CHUNK) {
                    int nbb = stage(b0, min(b0 + BP_CHUNK, A.ebeg[bb+1]), rlo, rhi, ebox, bidx, blo, bhi, &sb);
                    // a staged box per warp row (in registers), the other side across the lanes
                    for (int ia = threadIdx.x >> 5; ia < na; ia += blockDim.x >> 5) {
                        const float4 al = alo[ia], ah = ahi[ia];
                        const int i = aidx[ia];
                        for (int ib = threadIdx.x & 31; ib < nbb; ib += 32) {
                            const int j = bidx[ib];
                            if (ba == bb && i >= j) continue;
                            if (!overlap(al, ah, blo[ib], bhi[ib])) continue;
                            int lo_ = min(i, j), hi_ = max(i, j);
                            if (bp_ee_ok(A, lo_, hi_)) bp_emit(A, ABD_CONTACT_EE, lo_, hi_);
                        }
                    }
                    __syncthreads();
                }
            }
        }
        // ---- point-triangle, both directions
        if (A.do_pt) {
            for (int dir = 0; dir < (ba == bb ? 1 : 2); dir++) {
                int pb = dir == 0 ? ba : bb, tb = dir == 0 ? bb : ba;
                for (int p0 = A.vbeg[pb]; p0 < A.vbeg[pb+1]; p0 += BP_CHUNK) {
                    int na = stage(p0, min(p0 + BP_CHUNK, A.vbeg[pb+1]), rlo, rhi, pbox, aidx, alo, ahi, &sa);
                    if (na == 0) continue;
                    for (int t0 = A.tbeg[tb]; t0 < A.tbeg[tb+1]; t0 += BP_CHUNK) {
                        int nt = stage(t0, min(t0 + BP_CHUNK, A.tbeg[tb+1]), rlo, rhi, tbox, bidx, blo, bhi, &sb);
                        for (int ia = threadIdx.x >> 5; ia < na; ia += blockDim.x >> 5) {
                            const float4 al = alo[ia], ah = ahi[ia];
                            const int pv = aidx[ia];
                            for (int ib = threadIdx.x & 31; ib < nt; ib += 32) {
                                if (!overlap(al, ah, blo[ib], bhi[ib])) continue;
                                const int tr = bidx[ib];
                                if (bp_pt_ok(A, pv, tr)) bp_emit(A, ABD_CONTACT_PT, pv, tr);
                            }
                        }
                        __syncthreads();
                    }
                }
            }
        }
    }
}

// 4. decode sorted keys into (kind, a, b) entries; count the EE prefix
__global__ void k_bp_decode(int n, const unsigned long long* __restrict__ keys, int4* out, int* n_ee) {
    GS_LOOP(i, n) {
        unsigned long long k = keys[i];
        int kind = (int)(k >> 62), a = (int)((k >> 31) & 0x7fffffffull), b = (int)(k & 0x7fffffffull);
        out[i] = make_int4(kind, a, b, 0);
        bool ee = kind == ABD_CONTACT_EE;
        bool next_ee = i + 1 < n && (int)(keys[i+1] >> 62) == ABD_CONTACT_EE;
        if (ee && !next_ee) *n_ee = (int)i + 1;
    }
}

struct BpScratch {
    float4* blo = nullptr; float4* bhi = nullptr;
    float4* vlo = nullptr; float4* vhi = nullptr;   // per-vertex boxes of the latest build
    int2* bpairs = nullptr; int bp_cap = 0;
    unsigned long long* keys = nullptr; unsigned long long* keys_s = nullptr; int key_cap = 0;
    int* cnt = nullptr;                     // [0] body pairs, [1] hits, [2] n_ee
    void* tmp = nullptr; size_t tmp_bytes = 0;
};
static BpScratch* bps(Engine* E) { return reinterpret_cast<BpScratch*>(E->bp_state); }

void eng_bp_free(Engine* E) {
    BpScratch* S = bps(E);
    if (!S) return;
    void* ps[] = {S->blo, S->bhi, S->vlo, S->vhi, S->bpairs, S->keys, S->keys_s, S->cnt, S->tmp};
    for (void* p : ps) if (p) cudaFree(p);
    delete S;
    E->bp_state = nullptr;
}

static int bp_reserve(Engine* E, int bp_need, int key_need) {
    BpScratch* S = bps(E);
    if (!S) {
        S = new BpScratch(); E->bp_state = S;
        if (cudaMalloc(&S->blo, sizeof(float4) * E->nb) != cudaSuccess || cudaMalloc(&S->bhi, sizeof(float4) * E->nb) != cudaSuccess ||
            cudaMalloc(&S->vlo, sizeof(float4) * std::max(E->nv, 1)) != cudaSuccess ||
            cudaMalloc(&S->vhi, sizeof(float4) * std::max(E->nv, 1)) != cudaSuccess ||
            cudaMalloc(&S->cnt, sizeof(int) * 4) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMalloc body boxes");
        cudaFuncSetAttribute(k_bp_prims, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(4 * BP_CHUNK * sizeof(float4) + 2 * BP_CHUNK * sizeof(int)));
    }
    // buffers in use by queued work are freed only after the stream drains
    if (bp_need > S->bp_cap || key_need > S->key_cap) eng_stream_sync(E);
    if (bp_need > S->bp_cap) {
        if (S->bpairs) cudaFree(S->bpairs);
        S->bp_cap = bp_need + bp_need / 2 + 1024;
        if (cudaMalloc(&S->bpairs, sizeof(int2) * S->bp_cap) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc body pairs");
    }
    if (key_need > S->key_cap) {
        if (S->keys) cudaFree(S->keys);
        if (S->keys_s) cudaFree(S->keys_s);
        if (S->tmp) cudaFree(S->tmp);
        S->key_cap = key_need + key_need / 2 + 4096;
        if (cudaMalloc(&S->keys, sizeof(unsigned long long) * S->key_cap) != cudaSuccess ||
            cudaMalloc(&S->keys_s, sizeof(unsigned long long) * S->key_cap) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMalloc pair keys");
        S->tmp_bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, S->tmp_bytes, S->keys, S->keys_s, S->key_cap);
        if (cudaMalloc(&S->tmp, S->tmp_bytes) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc sort scratch");
    }
    return ABD_OK;
}

// Build a sorted (kind, a, b) list of EE and PT candidates into `out`
// (capacity *cap, grown through `grow`).  p may be null (static positions).
// mode 0: swept list with limit lim; mode 1: detection with distance filt.
// The list length comes back to the host; its EE count stays on the device
// (copied to nee_dev when given; BpScratch::cnt[2] until the next build).
static int bp_build(Engine* E, const double* p, double lim, double filt, int mode, int4*& out, int& cap, int& n_out,
                    int* nee_dev, int (*grow)(Engine*, int)) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    int rc;
    if ((rc = bp_reserve(E, 4 * E->nb + 1024, std::max(cap, 4096)))) return rc;
    BpScratch* S = bps(E);
    float pad = (float)(0.5 * lim);
    for (int attempt = 0; attempt < 8; attempt++) {
        CUDA_TRY(cudaMemsetAsync(S->cnt, 0, sizeof(int) * 4, s));
        k_body_boxes<<<grid_for(32L * E->nb), 256, 0, s>>>(E->nb, E->bd_vbeg, E->x, p, pad, S->blo, S->bhi, S->vlo, S->vhi);
        k_body_pairs<<<grid_for(32L * E->nb), 256, 0, s>>>(E->nb, E->bscene, E->sc_body_begin, S->blo, S->bhi,
                                                            P.self_contact, S->bpairs, S->bp_cap, S->cnt);
        BpArgs A;
        A.G = eng_geo(E); A.p = p; A.pmag = E->pmag; A.ebeg = E->bd_ebeg; A.tbeg = E->bd_tbeg; A.vbeg = E->bd_vbeg;
        A.vlo = S->vlo; A.vhi = S->vhi;
        A.blo = S->blo; A.bhi = S->bhi; A.pad = pad; A.lim = lim; A.filt = filt; A.mode = mode; A.f32 = P.ee_f32;
        A.self_contact = P.self_contact; A.do_ee = P.contact_ee && E->ne > 0; A.do_pt = P.contact_pt && E->nt > 0;
        A.out = S->keys; A.cap = S->key_cap; A.count = S->cnt + 1;
        size_t smem = 4 * BP_CHUNK * sizeof(float4) + 2 * BP_CHUNK * sizeof(int);
        k_bp_prims<<<NUM_SMS * 2, BP_THREADS, smem, s>>>(S->bpairs, S->cnt, S->bp_cap, A);
        E->launches += 3;
        int h[2];
        CUDA_TRY(cudaMemcpyAsync(h, S->cnt, sizeof(int) * 2, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(eng_stream_sync(E));
        if (h[0] > S->bp_cap || h[1] > S->key_cap) {
            if ((rc = bp_reserve(E, h[0], h[1]))) return rc;
            continue;
        }
        int n = h[1];
        if (n > cap) { if ((rc = grow(E, n))) return rc; }
        if (n > 0) {
            size_t bytes = S->tmp_bytes;
            CUDA_TRY(cub::DeviceRadixSort::SortKeys(S->tmp, bytes, S->keys, S->keys_s, n, 0, 64, s));
            k_bp_decode<<<grid_for(n), 256, 0, s>>>(n, S->keys_s, out, S->cnt + 2);
            E->launches += 2;
        }
        if (nee_dev) CUDA_TRY(cudaMemcpyAsync(nee_dev, S->cnt + 2, sizeof(int), cudaMemcpyDeviceToDevice, s));
        n_out = n;
        return ABD_OK;
    }
    return E->fail(ABD_ERR_CONTACT_OVERFLOW, "body-pair broad phase did not fit after growing");
}

static int grow_sw(Engine* E, int need) { return eng_grow_swept(E, need); }
static int grow_ct(Engine* E, int need) { return eng_grow_contacts(E, need); }

// swept list along p = E->pv (computed by the caller), limit lim
int eng_swept_bp(Engine* E, double lim) {
    int n = 0;
    int rc = bp_build(E, E->pv, lim, lim, 0, E->sw, E->sw_cap, n, E->sw_nee, grow_sw);
    if (rc) return rc;
    E->n_sw = n; E->n_sw_ee = -1; E->sw_valid = true;   // EE count on the device only (E->sw_nee)
    return ABD_OK;
}

__global__ void k_bp_counts(Counters* cnt, const int* __restrict__ n_ee_dev, int n) {
    if (threadIdx.x == 0 && blockIdx.x == 0) { int n_ee = *n_ee_dev; cnt->n_ee = n_ee; cnt->n_pt = n - n_ee; cnt->overflow = 0; }
}

// full detection at the current positions with filter filt
int eng_detect_bp(Engine* E, double filt) {
    int rc = eng_transform(E);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(E->dcnt, 0, DETECT_COUNTER_BYTES, E->stream));
    double lim = filt * (1.0 + 1e-6) + 1e-7;
    int n = 0;
    if ((rc = bp_build(E, nullptr, lim, filt, 1, E->contacts, E->cap, n, nullptr, grow_ct))) return rc;
    k_bp_counts<<<1, 32, 0, E->stream>>>(E->dcnt, bps(E)->cnt + 2, n);
    E->launches++;
    return eng_pg_candidates(E, filt);
}

// ------------------------------------------------------------------ contact groups of the line search
//
// Two bodies belong to one group when their boxes swept over the listed
// step x .. x + p, padded by half the candidate distance on every side,
// overlap (transitively).  Bodies of different groups stay more than the
// candidate distance apart for any pair of step fractions in [0, 1], so no
// listed pair, barrier term or CCD bound couples them and each group can
// take its own step length.  The union-find hooks the larger root under the
// smaller with atomicCAS, so a group's root is its smallest body index.

DV int grp_find(const int* parent, int x, int limit) {
    for (int k = 0; k < limit; k++) {
        int p = __ldcg(parent + x);
        if (p == x) return x;
        x = p;
    }
    return x;
}

__global__ void k_grp_init(int nb, int* parent) { GS_LOOP(b, nb) parent[b] = (int)b; }

// one warp per body a: every later body b of the scene whose box overlaps
__global__ void k_grp_union(int nb, const int* __restrict__ bscene, const int* __restrict__ sc_body_begin,
                            const float4* __restrict__ blo, const float4* __restrict__ bhi, int* parent, Counters* cnt) {
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    for (int a = warp; a < nb; a += (gridDim.x * blockDim.x) >> 5) {
        int end = sc_body_begin[bscene[a] + 1];
        float4 al = blo[a], ah = bhi[a];
        for (int b = a + 1 + lane; b < end; b += 32) {
            if (!overlap(al, ah, blo[b], bhi[b])) continue;
            // every failed CAS means a root was hooked, which happens at
            // most nb - 1 times in total
            int ra = a, rb = b;
            bool ok = false;
            for (int k = 0; k <= nb; k++) {
                ra = grp_find(parent, ra, nb + 1); rb = grp_find(parent, rb, nb + 1);
                if (ra == rb) { ok = true; break; }
                if (ra < rb) { int t = ra; ra = rb; rb = t; }
                int old = atomicCAS(parent + ra, ra, rb);
                if (old == ra) { ok = true; break; }
                ra = old;
            }
            if (!ok) atomicExch(&cnt->grp_fail, 1);
        }
    }
}

// root per body; a unit (a root body) joins the line search when its scene
// is still iterating, every other slot is skipped
__global__ void k_grp_finish(int nb, int* parent, const int* __restrict__ bscene, const int* __restrict__ done,
                             int* udone) {
    GS_LOOP(b, nb) {
        int r = grp_find(parent, (int)b, nb + 1);
        parent[b] = r;
        udone[b] = (r != (int)b) || done[bscene[b]];
    }
}

void eng_groups_free(Engine* E) {
    void* ps[] = {E->grp, E->gscd, E->gsci, E->grp_lo, E->grp_hi};
    for (void* p : ps) if (p) cudaFree(p);
    E->grp = nullptr; E->gscd = nullptr; E->gsci = nullptr; E->grp_lo = nullptr; E->grp_hi = nullptr;
}

// groups of the step listed by the last eng_swept (positions E->x, step
// E->pv); needs contiguous per-body vertex ranges
int eng_groups(Engine* E, const int* done) {
    if (!E->bd_ok) return E->fail(ABD_ERR_INVALID_ARG, "ls_groups needs contiguous per-body vertex ranges");
    int nb = E->nb;
    cudaStream_t s = E->stream;
    if (!E->grp) {
        if (cudaMalloc(&E->grp, sizeof(int) * nb) != cudaSuccess ||
            cudaMalloc(&E->gscd, sizeof(double) * SD_COUNT * nb) != cudaSuccess ||
            cudaMalloc(&E->gsci, sizeof(int) * SI_COUNT * nb) != cudaSuccess ||
            cudaMalloc(&E->grp_lo, sizeof(float4) * nb) != cudaSuccess ||
            cudaMalloc(&E->grp_hi, sizeof(float4) * nb) != cudaSuccess) {
            eng_groups_free(E);
            return E->fail(ABD_ERR_CUDA, "cudaMalloc contact groups");
        }
        CUDA_TRY(cudaMemsetAsync(E->gscd, 0, sizeof(double) * SD_COUNT * nb, s));
        CUDA_TRY(cudaMemsetAsync(E->gsci, 0, sizeof(int) * SI_COUNT * nb, s));
    }
    double lim = E->P.cand_dist * (1.0 + 1e-6) + 1e-7;
    float pad = (float)(0.5 * lim);
    k_grp_init<<<grid_for(nb), 256, 0, s>>>(nb, E->grp);
    k_body_boxes<<<grid_for(32L * nb), 256, 0, s>>>(nb, E->bd_vbeg, E->x, E->pv, pad, E->grp_lo, E->grp_hi);
    k_grp_union<<<grid_for(32L * nb), 256, 0, s>>>(nb, E->bscene, E->sc_body_begin, E->grp_lo, E->grp_hi, E->grp, E->dcnt);
    k_grp_finish<<<grid_for(nb), 256, 0, s>>>(nb, E->grp, E->bscene, done, E->gsci + SI_DONE * nb);
    E->launches += 4;
    return ABD_OK;
}
