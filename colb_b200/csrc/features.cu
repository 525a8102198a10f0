// features.cu — per-body inputs of the learned warm start (no counterpart in
// the reference).
//
// At the current state (nxt == now between steps) the candidate pairs within
// ABD_FEAT_RADIUS_DHAT * dhat are detected with the solver's own broad and
// narrow phase.  Every pair gives each of its dynamic bodies one record: the
// primitive distance and the unit direction from the other primitive's
// closest point to this body's.  Records are sorted by (body, distance) and
// every body keeps its 8 nearest.  Everything is expressed in the body frame
// (directions d map to q d, q the body's 3x3 DoF rows):
//   f[0:3]   q (v + dt g)            inertial velocity of the centre
//   f[3:12]  q qdot^T (row-major)    affine velocity acting on rest positions
//   f[12:15] q g / |g|               gravity direction
//   f[15]    log(1 + pair count)
//   f[16+4k] distance_k / radius, f[17+4k..19+4k] direction_k  (k < 8;
//            missing entries are (1, 0, 0, 0))
#include "engine.cuh"
#include "contact.cuh"
#include <cub/cub.cuh>

Geo eng_geo(Engine* E);
int eng_detect_bp(Engine* E, double filt);
bool eng_use_bp(const Engine* E);
int eng_grow_contacts(Engine* E, int need);
int eng_sync_counters(Engine* E);

struct FeatState {
    unsigned long long* keys = nullptr; unsigned long long* keys_s = nullptr;
    int* vals = nullptr; int* vals_s = nullptr;
    float4* rec = nullptr;          // (direction xyz, distance) per record
    int cap = 0;
    int* bcount = nullptr;          // pairs per body
    void* tmp = nullptr; size_t tmp_bytes = 0;
};

void eng_features_free(Engine* E) {
    FeatState* F = reinterpret_cast<FeatState*>(E->feat_state);
    if (!F) return;
    void* ps[] = {F->keys, F->keys_s, F->vals, F->vals_s, F->rec, F->bcount, F->tmp};
    for (void* p : ps) if (p) cudaFree(p);
    delete F;
    E->feat_state = nullptr;
}

// closest point of p on triangle abc given its region (0..2 vertex, 3..5
// edge t0t1 / t1t2 / t2t0, 6 face)
DV d3 tri_closest(d3 p, d3 a, d3 b, d3 c, int r) {
    d3 T[3] = {a, b, c};
    if (r <= 2) return T[r];
    if (r <= 5) {
        d3 e0 = T[r - 3], e1 = T[(r - 3 + 1) % 3];
        d3 e = e1 - e0;
        double ee = dot(e, e);
        double t = ee > 0 ? dot(p - e0, e) / ee : 0.0;
        t = t < 0 ? 0 : (t > 1 ? 1 : t);
        return e0 + t * e;
    }
    d3 n = cross(b - a, c - a);
    double nn = dot(n, n);
    return nn > 0 ? p - (dot(p - a, n) / nn) * n : a;
}

__global__ void k_feat_records(const Counters* cnt, const int4* __restrict__ contacts, Geo G,
                               unsigned long long* keys, int* vals, float4* rec, int* bcount, int cap) {
    int n = min(cnt->n_total, cap / 2);
    GS_LOOP(c, n) {
        int4 C = contacts[c];
        d3 pa, pb;
        int ba, bb = -1;
        if (C.x == ABD_CONTACT_EE) {
            int2 ea = G.edges[C.y], eb = G.edges[C.z];
            double s, t, d;
            seg_seg_f64(G.x + 3*ea.x, G.x + 3*ea.y, G.x + 3*eb.x, G.x + 3*eb.y, 0.0, s, t, d);
            d3 a0 = ld3(G.x + 3*ea.x), a1 = ld3(G.x + 3*ea.y), b0 = ld3(G.x + 3*eb.x), b1 = ld3(G.x + 3*eb.y);
            pa = a0 + s * (a1 - a0); pb = b0 + t * (b1 - b0);
            ba = G.vbody[ea.x]; bb = G.vbody[eb.x];
        } else if (C.x == ABD_CONTACT_PT) {
            const int* tr = G.tris + 3*C.z;
            int r = pt_region(G.x + 3*C.y, G.x + 3*tr[0], G.x + 3*tr[1], G.x + 3*tr[2]);
            pa = ld3(G.x + 3*C.y);
            pb = tri_closest(pa, ld3(G.x + 3*tr[0]), ld3(G.x + 3*tr[1]), ld3(G.x + 3*tr[2]), r);
            ba = G.vbody[C.y]; bb = G.vbody[tr[0]];
        } else {
            const double* pl = G.planes + 4*C.z;
            pa = ld3(G.x + 3*C.y);
            double d = pl[0] * pa.x + pl[1] * pa.y + pl[2] * pa.z - pl[3];
            pb = pa - d * mk3(pl[0], pl[1], pl[2]);
            ba = G.vbody[C.y];
        }
        d3 dv = pa - pb;
        double d = sqrt(dot(dv, dv));
        d3 nrm = d > 0 ? (1.0 / d) * dv : mk3(0, 0, 0);
        if (C.x == ABD_CONTACT_PG) {
            const double* pl = G.planes + 4*C.z;
            nrm = mk3(pl[0], pl[1], pl[2]);
        }
        float df = (float)d;
        long r0 = 2 * c, r1 = 2 * c + 1;
        bool va = G.mass[ba] > 0.0, vb = bb >= 0 && G.mass[bb] > 0.0;
        keys[r0] = va ? (((unsigned long long)ba << 32) | __float_as_uint(df)) : ~0ull;
        keys[r1] = vb ? (((unsigned long long)bb << 32) | __float_as_uint(df)) : ~0ull;
        vals[r0] = (int)r0; vals[r1] = (int)r1;
        rec[r0] = make_float4((float)nrm.x, (float)nrm.y, (float)nrm.z, df);
        rec[r1] = make_float4(-(float)nrm.x, -(float)nrm.y, -(float)nrm.z, df);
        if (va) atomicAdd(bcount + ba, 1);
        if (vb) atomicAdd(bcount + bb, 1);
    }
}

// first position of body b in the sorted keys (keys of body b start at b << 32)
DV int lower_body(const unsigned long long* k, int n, int b) {
    unsigned long long key = (unsigned long long)b << 32;
    int lo = 0, hi = n;
    while (lo < hi) { int m = (lo + hi) >> 1; if (k[m] < key) lo = m + 1; else hi = m; }
    return lo;
}

__global__ void k_features(int nb, const double* __restrict__ st, const double* __restrict__ mass, double dt, double g0,
                           double g1, double g2, const Counters* cnt, int cap, const unsigned long long* __restrict__ keys,
                           const int* __restrict__ vals, const float4* __restrict__ rec, const int* __restrict__ bcount,
                           double radius, float* out) {
    int nrec = 2 * min(cnt->n_total, cap / 2);
    GS_LOOP(b, nb) {
        float* f = out + 48 * b;
        const double* now = st + ST_STRIDE * b + ST_NOW;
        const double* q = now + ST_Q;
        double vg[3] = {now[ST_V] + dt * g0, now[ST_V + 1] + dt * g1, now[ST_V + 2] + dt * g2};
        double gn = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
        double gd[3] = {gn > 0 ? g0 / gn : 0.0, gn > 0 ? g1 / gn : 0.0, gn > 0 ? g2 / gn : 0.0};
        for (int i = 0; i < 3; i++) {
            f[i] = (float)(q[3*i] * vg[0] + q[3*i+1] * vg[1] + q[3*i+2] * vg[2]);
            f[12 + i] = (float)(q[3*i] * gd[0] + q[3*i+1] * gd[1] + q[3*i+2] * gd[2]);
            for (int j = 0; j < 3; j++) {
                const double* qd = now + ST_QD;
                f[3 + 3*i + j] = (float)(q[3*i] * qd[3*j] + q[3*i+1] * qd[3*j+1] + q[3*i+2] * qd[3*j+2]);
            }
        }
        int count = bcount[b];
        f[15] = log1pf((float)count);
        int at = lower_body(keys, nrec, (int)b);
        for (int k = 0; k < 8; k++) {
            float* o = f + 16 + 4*k;
            if (k < count && at + k < nrec && (int)(keys[at + k] >> 32) == (int)b) {
                float4 r = rec[vals[at + k]];
                o[0] = (float)(r.w / radius);
                for (int i = 0; i < 3; i++) o[1 + i] = (float)(q[3*i] * r.x + q[3*i+1] * r.y + q[3*i+2] * r.z);
            } else {
                o[0] = 1.0f; o[1] = 0.0f; o[2] = 0.0f; o[3] = 0.0f;
            }
        }
        if (!(mass[b] > 0.0)) for (int i = 0; i < 48; i++) f[i] = 0.0f;
    }
}

// Features of every body at the current nxt state into feat_dev [nb][48].
int eng_features(Engine* E, float* feat_dev) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    const double radius = ABD_FEAT_RADIUS_DHAT * P.dhat;
    int rc;
    for (;;) {
        if ((rc = eng_use_bp(E) ? eng_detect_bp(E, radius) : eng_detect(E, radius))) return rc;
        if ((rc = eng_sync_counters(E))) return rc;
        if (!E->hcnt->overflow) break;
        if ((rc = eng_grow_contacts(E, E->hcnt->n_total))) return rc;
    }
    if (!E->feat_state) E->feat_state = new FeatState();
    FeatState* F = reinterpret_cast<FeatState*>(E->feat_state);
    int npairs = E->hcnt->n_total;
    int need = 2 * std::max(npairs, 1);
    if (need > F->cap) {
        void* ps[] = {F->keys, F->keys_s, F->vals, F->vals_s, F->rec, F->tmp};
        for (void* p : ps) if (p) cudaFree(p);
        F->tmp = nullptr; F->tmp_bytes = 0;
        F->cap = need + need / 2;
        if (cudaMalloc(&F->keys, sizeof(unsigned long long) * F->cap) != cudaSuccess ||
            cudaMalloc(&F->keys_s, sizeof(unsigned long long) * F->cap) != cudaSuccess ||
            cudaMalloc(&F->vals, sizeof(int) * F->cap) != cudaSuccess ||
            cudaMalloc(&F->vals_s, sizeof(int) * F->cap) != cudaSuccess ||
            cudaMalloc(&F->rec, sizeof(float4) * F->cap) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMalloc feature records");
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, F->keys, F->keys_s, F->vals, F->vals_s, F->cap, 0, 64, s);
        if (cudaMalloc(&F->tmp, bytes) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc feature sort");
        F->tmp_bytes = bytes;
    }
    if (!F->bcount && cudaMalloc(&F->bcount, sizeof(int) * E->nb) != cudaSuccess)
        return E->fail(ABD_ERR_CUDA, "cudaMalloc feature counts");
    CUDA_TRY(cudaMemsetAsync(F->bcount, 0, sizeof(int) * E->nb, s));
    Geo G = eng_geo(E);
    int nrec = 2 * npairs;
    if (npairs > 0) {
        k_feat_records<<<grid_for(npairs), 256, 0, s>>>(E->dcnt, E->contacts, G, F->keys, F->vals, F->rec, F->bcount, F->cap);
        size_t bytes = F->tmp_bytes;
        CUDA_TRY(cub::DeviceRadixSort::SortPairs(F->tmp, bytes, F->keys, F->keys_s, F->vals, F->vals_s, nrec, 0, 64, s));
        E->launches += 2;
    }
    k_features<<<grid_for(E->nb), 256, 0, s>>>(E->nb, E->st, E->mass, P.dt, P.gravity[0], P.gravity[1], P.gravity[2],
                                               E->dcnt, F->cap, F->keys_s, F->vals_s, F->rec, F->bcount, radius, feat_dev);
    E->launches++;
    return ABD_OK;
}

extern "C" int abd_get_features(AbdHandle* h, float* feat, int32_t n) {
    Engine* E = reinterpret_cast<Engine*>(h);
    if (!E) return ABD_ERR_INVALID_ARG;
    if (!feat || n != E->nb) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_features: n_bodies mismatch or null output");
    if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaSetDevice");
    float* d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * 48 * (size_t)E->nb) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc features");
    int rc = eng_features(E, d);
    if (!rc) {
        cudaError_t e = cudaMemcpyAsync(feat, d, sizeof(float) * 48 * (size_t)E->nb, cudaMemcpyDeviceToHost, E->stream);
        if (e == cudaSuccess) e = eng_stream_sync(E);
        if (e != cudaSuccess) rc = E->fail(ABD_ERR_CUDA, std::string("abd_get_features: ") + cudaGetErrorString(e));
    }
    cudaFree(d);
    return rc;
}
