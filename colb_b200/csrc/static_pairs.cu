// static_pairs.cu — edge-edge candidate detection that allocates nothing.
//
// Some callers cannot allocate device memory when they need the candidate
// pairs: a host application that has handed all device memory management to
// its own pool, a real-time loop that forbids allocation after start-up, or
// a plugin running inside a host that owns the CUDA context and bans
// cudaMalloc.  abd_ee_pairs_static serves them: the caller passes device
// buffers for its inputs and outputs, and every intermediate (boxes, grid
// keys, buckets, per-edge counts, radix-sort and scan scratch) lives in the
// file-scope __device__ arrays below, sized for ABD_STATIC_MAX_EDGES edges.
// Every GPU that loads the library holds these arrays until the process
// exits: boxes 2 MiB, grid keys and values 1 MiB, buckets 1 MiB, per-edge
// counts and offsets 0.5 MiB, sort and scan scratch 4 MiB, about 8.5 MiB in
// all.
//
// Host code must not pass the arrays' names to a kernel: in host code a
// __device__ symbol names a host-side stand-in, not device memory.  The
// first call on each device, with that device current, looks the device
// addresses up with cudaGetSymbolAddress and caches them; make that first
// call before any stream capture.  The cache is not refreshed: after a
// cudaDeviceReset of a device, this entry point must not be called on that
// device again in the same process.  Every call waits for its stream before
// it returns (it reads the pair count back).  All calls share the arrays:
// two calls whose work overlaps on the GPU (different streams, or the same
// arrays used by two threads at once) race and corrupt each other's results.
#include "engine.cuh"
#include "physics.cuh"
#include <cub/cub.cuh>
#include <mutex>

std::string& abd_global_error();   // capi.cu: the message abd_last_error(NULL) returns

#define ST_MAXE ABD_STATIC_MAX_EDGES
#define ST_H (2 * ST_MAXE)
#define ST_CUB_BYTES (4 << 20)

static __device__ __align__(256) float4 g_st_lo[ST_MAXE];
static __device__ __align__(256) float4 g_st_hi[ST_MAXE];
static __device__ __align__(256) uint32_t g_st_keys[2 * ST_MAXE];
static __device__ __align__(256) int g_st_vals[2 * ST_MAXE];
static __device__ __align__(256) int g_st_bucket[2 * ST_H];
static __device__ __align__(256) int g_st_count[2 * (ST_MAXE + 1) + 4];   // counts, offsets, bad-edge flag
static __device__ __align__(256) float g_st_cell[4];
static __device__ __align__(256) unsigned char g_st_cub[ST_CUB_BYTES];

struct StaticScratch {
    float4* lo; float4* hi; uint32_t* keys; int* vals; int* bucket; int* count; float* cell; void* cub;
    bool ready;
};
static StaticScratch g_scratch[64];
static std::mutex g_scratch_mu;

static int scratch_for_device(int dev, StaticScratch** out, std::string& err) {
    if (dev < 0 || dev >= 64) { err = "abd_ee_pairs_static: device index out of range"; return ABD_ERR_INVALID_ARG; }
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    StaticScratch& S = g_scratch[dev];
    if (!S.ready) {
        struct { void** p; const void* sym; } t[] = {
            {(void**)&S.lo, (const void*)&g_st_lo}, {(void**)&S.hi, (const void*)&g_st_hi},
            {(void**)&S.keys, (const void*)&g_st_keys}, {(void**)&S.vals, (const void*)&g_st_vals},
            {(void**)&S.bucket, (const void*)&g_st_bucket}, {(void**)&S.count, (const void*)&g_st_count},
            {(void**)&S.cell, (const void*)&g_st_cell}, {(void**)&S.cub, (const void*)&g_st_cub}};
        for (auto& e : t) {
            cudaError_t rc = cudaGetSymbolAddress(e.p, e.sym);
            if (rc != cudaSuccess) {
                err = std::string("abd_ee_pairs_static: cudaGetSymbolAddress: ") + cudaGetErrorString(rc);
                return ABD_ERR_CUDA;
            }
        }
        S.ready = true;
    }
    *out = &S;
    return ABD_OK;
}

// boxes of the float32 copies of the endpoints (contact.py:150-154), padded
__global__ void k_st_boxes(int ne, const double* __restrict__ x, const int* __restrict__ edges, float pad,
                           float4* lo, float4* hi, float* cell) {
    float ext = 0.f;
    GS_LOOP(e, ne) {
        int a = edges[2*e], b = edges[2*e+1];
        float l[3], h[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float fa = __double2float_rn(x[3*a+k]), fb = __double2float_rn(x[3*b+k]);
            l[k] = __fsub_rd(fminf(fa, fb), pad); h[k] = __fadd_ru(fmaxf(fa, fb), pad);
        }
        lo[e] = make_float4(l[0], l[1], l[2], 0.f); hi[e] = make_float4(h[0], h[1], h[2], 0.f);
        ext = fmaxf(ext, fmaxf(h[0] - l[0], fmaxf(h[1] - l[1], h[2] - l[2])));
    }
    for (int o = 16; o > 0; o >>= 1) ext = fmaxf(ext, __shfl_xor_sync(0xffffffffu, ext, o));
    if ((threadIdx.x & 31) == 0 && ext > 0.f) atomic_max_pos(cell, ext);
}
__global__ void k_st_keys(int n, const float4* __restrict__ lo, const float* cell, uint32_t mask, uint32_t* keys, int* vals) {
    float h = fmaxf(*cell, 1e-6f);
    GS_LOOP(i, n) {
        float4 l = lo[i];
        keys[i] = cell_hash(0, (int)floorf(l.x / h), (int)floorf(l.y / h), (int)floorf(l.z / h)) & mask;
        vals[i] = (int)i;
    }
}
__global__ void k_st_ranges(int n, const uint32_t* __restrict__ keys, int* bstart, int* bend) {
    GS_LOOP(i, n) {
        uint32_t k = keys[i];
        if (i == 0 || keys[i-1] != k) bstart[k] = (int)i;
        if (i == n - 1 || keys[i+1] != k) bend[k] = (int)i + 1;
    }
}
// mode 0: count per edge; mode 1: write vertex quadruples, sorted by
// partner, the rows that fit below cap (an edge whose rows cross cap keeps
// the ones it visited first, so on overflow the rows are not the first cap
// rows of the complete sorted list)
__global__ void k_st_pairs(int ne, GridView GV, const double* __restrict__ x, const int* __restrict__ edges,
                           const float4* __restrict__ qlo, const float4* __restrict__ qhi, double cand, int mode,
                           int* count, const int* off, int* out4, int cap) {
    float fc = __double2float_rn(cand);
    GS_LOOP(i, ne) {
        int ii = (int)i;
        int a0 = edges[2*i], a1 = edges[2*i+1];
        float p1[3], q1[3];
        for (int k = 0; k < 3; k++) { p1[k] = __double2float_rn(x[3*a0+k]); q1[k] = __double2float_rn(x[3*a1+k]); }
        int c = 0, base = mode == 1 ? off[i] : 0;
        grid_visit(GV, qlo[i], qhi[i], 0, [&](int j) {
            if (j <= ii) return;
            int b0 = edges[2*j], b1 = edges[2*j+1];
            if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return;
            float p2[3], q2[3];
            for (int k = 0; k < 3; k++) { p2[k] = __double2float_rn(x[3*b0+k]); q2[k] = __double2float_rn(x[3*b1+k]); }
            float s, t, d;
            seg_seg_f32(p1, q1, p2, q2, 1e-6f, s, t, d);
            if (!(d < fc)) return;
            if (mode == 1) {
                // the partner edge index goes in slot 2 until the segment is sorted
                int at = base + c;
                if ((unsigned)at < (unsigned)cap) { out4[4*at] = a0; out4[4*at+1] = a1; out4[4*at+2] = j; out4[4*at+3] = -1; }
            }
            c++;
        });
        if (mode == 0) { count[i] = c; continue; }
        // order this edge's pairs by partner edge index, as the handle-based
        // detection does, then expand partners to their vertex ids
        int lo = base, hi = min(base + c, cap);
        for (int k = lo + 1; k < hi; k++) {
            int v2 = out4[4*k+2];
            int m = k - 1;
            while (m >= lo && out4[4*m+2] > v2) { out4[4*(m+1)+2] = out4[4*m+2]; m--; }
            out4[4*(m+1)+2] = v2;
        }
        for (int k = lo; k < hi; k++) {
            int j = out4[4*k+2];
            out4[4*k+2] = edges[2*j]; out4[4*k+3] = edges[2*j+1];
        }
    }
}
// every edge index must name a vertex of x
__global__ void k_st_check(int ne, const int* __restrict__ edges, int nv, int* bad) {
    GS_LOOP(i, 2L * ne) { int v = edges[i]; if (v < 0 || v >= nv) *bad = 1; }
}
__global__ void k_st_total(const int* off, int ne, int* n_out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *n_out = off[ne];
}

extern "C" int abd_ee_pairs_static(const double* x_dev, const int32_t* edges_dev, int32_t n_verts, int32_t n_edges,
                                   double cand_dist, int32_t* pairs_dev, int32_t cap, int32_t* n_pairs_dev,
                                   void* stream_ptr) {
    std::string& err = abd_global_error();
    if (n_edges < 0 || n_verts < 0 || n_edges > ST_MAXE || cap < 0 || !(cand_dist > 0) ||
        (n_edges > 0 && (!x_dev || !edges_dev)) || !n_pairs_dev || (cap > 0 && !pairs_dev)) {
        err = "abd_ee_pairs_static: invalid arguments (n_edges must be in [0, " + std::to_string(ST_MAXE) +
              "], cand_dist > 0, device buffers non-null)";
        return ABD_ERR_INVALID_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { err = "abd_ee_pairs_static: no current device"; return ABD_ERR_NO_DEVICE; }
    StaticScratch* S = nullptr;
    int rc = scratch_for_device(dev, &S, err);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream_ptr;
    // clear what the previous call left behind
    float* cell = S->cell;
    int* bad_edge = S->count + 2 * (ST_MAXE + 1);
    if (cudaMemsetAsync(cell, 0, sizeof(float), s) != cudaSuccess ||
        cudaMemsetAsync(bad_edge, 0, sizeof(int), s) != cudaSuccess ||
        cudaMemsetAsync(n_pairs_dev, 0, sizeof(int32_t), s) != cudaSuccess) {
        err = "abd_ee_pairs_static: cudaMemsetAsync failed"; return ABD_ERR_CUDA;
    }
    if (n_edges < 2) return cudaStreamSynchronize(s) == cudaSuccess ? ABD_OK : ABD_ERR_CUDA;
    {
        int bad = 0;
        k_st_check<<<grid_for(2L * n_edges), 256, 0, s>>>(n_edges, edges_dev, n_verts, bad_edge);
        if (cudaMemcpyAsync(&bad, bad_edge, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) { err = "abd_ee_pairs_static: CUDA error"; return ABD_ERR_CUDA; }
        if (bad) { err = "abd_ee_pairs_static: an edge index is outside [0, n_verts)"; return ABD_ERR_INVALID_ARG; }
    }
    int H = 64; while (H < 2 * n_edges) H <<= 1;
    int bits = 0; while ((1 << bits) < H) bits++;
    float pad = (float)(0.5 * cand_dist * (1.0 + 1e-6) + 1e-7);
    uint32_t* keys = S->keys; uint32_t* keys_s = S->keys + ST_MAXE;
    int* vals = S->vals; int* vals_s = S->vals + ST_MAXE;
    int* bstart = S->bucket; int* bend = S->bucket + ST_H;
    int* count = S->count; int* off = S->count + (ST_MAXE + 1);
    k_st_boxes<<<grid_for(n_edges), 256, 0, s>>>(n_edges, x_dev, edges_dev, pad, S->lo, S->hi, cell);
    k_st_keys<<<grid_for(n_edges), 256, 0, s>>>(n_edges, S->lo, cell, (uint32_t)(H - 1), keys, vals);
    size_t need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, keys, keys_s, vals, vals_s, n_edges, 0, bits, s);
    size_t need2 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need2, count, off, n_edges + 1, s);
    if (need > ST_CUB_BYTES || need2 > ST_CUB_BYTES) { err = "abd_ee_pairs_static: sort scratch exceeds the static size"; return ABD_ERR_INVALID_ARG; }
    if (cub::DeviceRadixSort::SortPairs(S->cub, need, keys, keys_s, vals, vals_s, n_edges, 0, bits, s) != cudaSuccess) {
        err = "abd_ee_pairs_static: radix sort failed"; return ABD_ERR_CUDA;
    }
    if (cudaMemsetAsync(bstart, 0xFF, sizeof(int) * H, s) != cudaSuccess) { err = "abd_ee_pairs_static: memset"; return ABD_ERR_CUDA; }
    k_st_ranges<<<grid_for(n_edges), 256, 0, s>>>(n_edges, keys_s, bstart, bend);
    GridView GV{S->lo, S->hi, nullptr, cell, vals_s, bstart, bend, (uint32_t)(H - 1)};
    k_st_pairs<<<grid_for(n_edges, 128), 128, 0, s>>>(n_edges, GV, x_dev, edges_dev, S->lo, S->hi, cand_dist, 0, count,
                                                      nullptr, pairs_dev, cap);
    if (cudaMemsetAsync(count + n_edges, 0, sizeof(int), s) != cudaSuccess) { err = "abd_ee_pairs_static: memset"; return ABD_ERR_CUDA; }
    if (cub::DeviceScan::ExclusiveSum(S->cub, need2, count, off, n_edges + 1, s) != cudaSuccess) {
        err = "abd_ee_pairs_static: scan failed"; return ABD_ERR_CUDA;
    }
    k_st_pairs<<<grid_for(n_edges, 128), 128, 0, s>>>(n_edges, GV, x_dev, edges_dev, S->lo, S->hi, cand_dist, 1, count,
                                                      off, pairs_dev, cap);
    k_st_total<<<1, 32, 0, s>>>(off, n_edges, n_pairs_dev);
    int n = 0;
    if (cudaMemcpyAsync(&n, n_pairs_dev, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        err = std::string("abd_ee_pairs_static: ") + cudaGetErrorString(cudaGetLastError());
        return ABD_ERR_CUDA;
    }
    if (n > cap) { err = "abd_ee_pairs_static: more pairs than cap (the count is in *n_pairs_dev)"; return ABD_ERR_CONTACT_OVERFLOW; }
    return ABD_OK;
}
