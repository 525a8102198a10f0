// engine.cuh — device state of one ABD handle and the launch helpers.
//
// HBM layout (all scenes of a batch concatenated, body-major):
//   st      [nb][48]  f64  BDFAffine (the reference's layout)
//   xbar    [nv][3]   f64  rest positions in the body frame
//   x       [nv][3]   f64  current positions of the nxt state
//   xf      [nv]      f32x4 float copy used by the float32 EE predicate
//   edges   [ne]      i32x2, tris [nt][3] i32, vbody [nv] i32, bscene [nb] i32
//   g, du   [nb][12]  f64  gradient / Newton increment, DoF order [c q0 q1 q2]
//   blocks  [nnzb][144]  f64 or f32  12x12 body blocks, column-major inside a
//           block, rows in CSR order (row_ptr / bcol), both triangles stored
//   contacts[cap]     i32x4 {kind, a, b, 0} sorted by (kind, a, b)
#pragma once
#include "common.cuh"
#include <string>
#include <vector>

#define CUDA_TRY(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { \
    E->fail(ABD_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(_e)); return ABD_ERR_CUDA; } } while (0)

// Uniform-grid broad phase over axis-aligned boxes.  Items are stored in the
// cell of their box's lower corner, hashed into 2^k buckets; the cell edge is
// the largest box extent of the pass, so a query box covers at most 3 cells
// per axis.
struct Grid {
    int n = 0;                  // stored items
    int nq = 0;                 // query items
    int H = 0;                  // buckets (power of two)
    int bits = 0;
    float4* lo = nullptr;       // stored boxes (w unused)
    float4* hi = nullptr;
    int* scene = nullptr;       // scene of each stored item
    float4* qlo = nullptr;      // query boxes
    float4* qhi = nullptr;
    int* qscene = nullptr;
    float* cell = nullptr;      // device scalar, cell edge
    uint32_t* keys = nullptr; uint32_t* keys_s = nullptr;
    int* vals = nullptr; int* vals_s = nullptr;
    int* bstart = nullptr; int* bend = nullptr;
    int* qcount = nullptr;      // nq + 1
    int* qoff = nullptr;        // nq + 1
};

struct GridView {
    const float4* lo; const float4* hi; const int* scene;
    const float* cell; const int* vals; const int* bstart; const int* bend; uint32_t mask;
};

DV uint32_t cell_hash(int scene, int cx, int cy, int cz) {
    return ((uint32_t)cx * 73856093u) ^ ((uint32_t)cy * 19349663u) ^ ((uint32_t)cz * 83492791u) ^
           ((uint32_t)scene * 2654435761u);
}

// Visit every stored item whose box overlaps [qlo,qhi] in the same scene,
// each exactly once.
template <class F>
DV void grid_visit(const GridView& G, float4 qlo, float4 qhi, int scene, F&& visit) {
    float h = *G.cell;
    // non-finite boxes (a diverged state) visit nothing; the Newton loop's
    // NaN check reports them.  The cell edge bounds every box extent, so a
    // finite query spans at most 3 cells per axis.
    if (!(h > 0.f && h < 3.0e38f)) return;
    if (!(isfinite(qlo.x) && isfinite(qlo.y) && isfinite(qlo.z) && isfinite(qhi.x) && isfinite(qhi.y) && isfinite(qhi.z))) return;
    float fx0 = floorf((qlo.x - h) / h), fx1 = floorf(qhi.x / h);
    float fy0 = floorf((qlo.y - h) / h), fy1 = floorf(qhi.y / h);
    float fz0 = floorf((qlo.z - h) / h), fz1 = floorf(qhi.z / h);
    if (fx1 - fx0 > 4.f || fy1 - fy0 > 4.f || fz1 - fz0 > 4.f) return;
    if (fabsf(fx0) > 1.0e9f || fabsf(fy0) > 1.0e9f || fabsf(fz0) > 1.0e9f) return;
    int x0 = (int)fx0, x1 = (int)fx1, y0 = (int)fy0, y1 = (int)fy1, z0 = (int)fz0, z1 = (int)fz1;
    for (int cz = z0; cz <= z1; cz++)
        for (int cy = y0; cy <= y1; cy++)
            for (int cx = x0; cx <= x1; cx++) {
                uint32_t key = cell_hash(scene, cx, cy, cz) & G.mask;
                int b = G.bstart[key];
                if (b < 0) continue;
                int e = G.bend[key];
                for (int k = b; k < e; k++) {
                    int j = G.vals[k];
                    if (G.scene && G.scene[j] != scene) continue;
                    float4 lo = G.lo[j];
                    if ((int)floorf(lo.x / h) != cx || (int)floorf(lo.y / h) != cy || (int)floorf(lo.z / h) != cz) continue;
                    float4 hi = G.hi[j];
                    if (lo.x > qhi.x || hi.x < qlo.x || lo.y > qhi.y || hi.y < qlo.y || lo.z > qhi.z || hi.z < qlo.z) continue;
                    visit(j);
                }
            }
}

// device counters (one struct in device memory, mirrored in pinned memory)
struct Counters {
    int n_ee, n_pt, n_pg, n_total;
    int overflow, nnzb, n_active, scenes_done;
    int krylov_active, ccd_capped, nan_flag, ls_pending;
    int nkeys, grp_fail, ls_trials, ls_nsw;   // ls_*: trial count and list length of a graph line search
    int n_sw, n_sw_ee, sw_overflow, pos_changed;   // pos_changed: abd_set_state moved a body
    int du_guard;                                  // mixed-precision increments replaced (du_guard)
};
#define DETECT_COUNTER_BYTES (5 * sizeof(int))   // n_ee .. overflow

struct Engine {
    AbdParams P;
    int device = 0;
    cudaStream_t stream = nullptr;
    int ns = 0, nb = 0, nv = 0, ne = 0, nt = 0, npl = 0;
    bool mixed = false;
    std::string err;
    int launches = 0;
    int comp_band = 0, comp_small = 0, comp_large = 0, krylov_fallbacks = 0;   // direct-solver counters
    int solver_capped = 0;         // Krylov solves that ended at lin_max_iter above tolerance
    int du_guard_hits = 0;         // mixed-precision increments replaced by the block-Jacobi direction
    int host_syncs = 0;            // stream synchronisations of the current call
    struct Tuner {
        int chosen = -1, next = 0, running = -1;
        float sum[8] = {0}; int cnt[8] = {0};
        cudaEvent_t a = nullptr, b = nullptr;
    };
    Tuner tune[3];

    // host-side scene offsets
    std::vector<int> h_body_begin, h_vert_begin, h_edge_begin, h_tri_begin, h_plane_begin;
    std::vector<int> h_bscene;

    // geometry
    double* xbar = nullptr; int* vbody = nullptr; int* vscene = nullptr; int* bscene = nullptr;
    int2* edges = nullptr; int* tris = nullptr; double* mass = nullptr; double* J = nullptr;
    double* planes = nullptr; int* plane_scene = nullptr; int* sc_plane_begin = nullptr; int* sc_body_begin = nullptr;
    int* edge_scene = nullptr; int* tri_scene = nullptr;

    // state
    double* st = nullptr; double* backup = nullptr; double* du = nullptr; double* g = nullptr;
    double* x = nullptr; float4* xf = nullptr; double* pv = nullptr; double* ws = nullptr;
    int has_ws = 0;

    // broad phase
    Grid gee, gpt;                 // EE: edges vs edges; PT: triangles vs points
    int cap = 0;
    int4* contacts = nullptr;      // sorted candidate list
    int4* cst = nullptr;           // stencil vertex ids (-1 padded)
    int* ctype = nullptr;          // stencil type or -1 inactive
    double* cxb = nullptr;         // barrier argument
    int2* cbody = nullptr;         // bodies (b0, b1) of the stencil
    int4* cblk = nullptr;          // block indices (b0b0, b0b1, b1b0, b1b1)

    // swept candidate list (swept.cu)
    int4* sw = nullptr; int sw_cap = 0; int n_sw = 0, n_sw_ee = 0; bool sw_valid = false;
    // fraction of the increment the swept list covers (1 unless the full
    // step's list did not fit); the line search's step length is capped to it
    double sw_scale = 1.0;
    bool sw_inject_done = false;   // ABD_INJECT_SWEPT_FULL fired in this step
    int* sw_nee = nullptr;         // device copy of the list's EE count (the list filter reads it)
    // block keys and done flags of the last assembly, copied to pinned host
    // memory in the assembly's own sync for the direct solver's analysis
    unsigned long long* h_ukeys = nullptr; int h_ukeys_cap = 0; int* h_done = nullptr; bool keys_host = false;
    int* sw_flag = nullptr; int* sw_off = nullptr;
    float* pmag = nullptr;         // |displacement| per vertex of the listed step
    int* zero_int = nullptr;       // a device 0
    int* zero_ns = nullptr;        // ns device zeros (no scene skipped)

    // block matrix
    unsigned long long* keys = nullptr; unsigned long long* keys_s = nullptr; unsigned long long* ukeys = nullptr;
    int blk_cap = 0;
    int nnzb_host = 0;             // block count of the last assembly (host copy)
    long long dense_blocks = 0;    // sum over scenes of n_bodies^2: no assembly has more blocks
    // the assembly's counters and block keys travel to the host behind
    // ev_asm while its kernels keep running; eng_asm_wait collects them
    cudaEvent_t ev_asm = nullptr; bool asm_pending = false; bool asm_direct = false;
    // block keys of the next iterate built before the end-of-iteration sync
    bool keys_ahead = false; long long keys_ahead_bound = 0; int keys_ahead_n = 0;
    int* row_ptr = nullptr; int* bcol = nullptr;
    void* vals = nullptr;          // double or float [blk_cap*144]
    void* dinv = nullptr;          // [nb*144]

    // Krylov vectors (double or float) [12 nb] each
    void* kv[10] = {nullptr};
    // per-scene scalars
    double* scd = nullptr;         // [NSCD][ns]
    int* sci = nullptr;            // [NSCI][ns]
    // contact groups of the line search (ls_groups): group root body of
    // each body, the per-group scalars in the per-scene layout with nb
    // slots (a group's slot is its root body), and the swept body boxes
    int* grp = nullptr;            // [nb]
    double* gscd = nullptr;        // [NSCD][nb]
    int* gsci = nullptr;           // [NSCI][nb]
    float4* grp_lo = nullptr; float4* grp_hi = nullptr;   // [nb]
    void* ls_graph_state = nullptr;   // line-search graphs (ls_graph, step.cu)
    bool capturing = false;           // a graph body is being captured: the autotuner only reports its shape
    double* st_in = nullptr;          // [48 nb] abd_set_state staging (compared with st before it replaces it)

    // cub scratch
    void* cub_tmp = nullptr; size_t cub_bytes = 0;

    Counters* dcnt = nullptr; Counters* hcnt = nullptr;   // device / pinned host
    double* hscd = nullptr; int* hsci = nullptr;          // pinned mirrors of per-scene scalars

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    double* prof_d = nullptr;      // [2][ns][newton_max_iter] residual / alpha of the current step
    void* dense_state = nullptr;   // direct-solver state (dense.cu)
    void* feat_state = nullptr;    // feature records (features.cu)
    void* mlp = nullptr;           // learned warm start network (mlp.cu)
    void* bp_state = nullptr;      // body-pair broad phase scratch (bpair.cu)
    bool bd_ok = false;            // bodies own contiguous vertex / edge / triangle ranges
    int* bd_vbeg = nullptr; int* bd_ebeg = nullptr; int* bd_tbeg = nullptr;   // [nb+1]
    int krylov_kind = ABD_SOLVER_BICGSTAB;
    std::vector<int> h_edges, h_tris;  // host copies (global vertex ids) for abd_get_pairs

    // profile of the last abd_step call
    std::vector<std::vector<double>> prof_res, prof_alpha;
    std::vector<std::vector<int>> prof_iters;

    // phase timers
    bool timing = false;
    struct Rec { int phase; cudaEvent_t a, b; double bytes; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> ev_pool;
    double phase_ms[ABD_NUM_PHASES] = {0};
    long long phase_n[ABD_NUM_PHASES] = {0};
    double phase_bytes[ABD_NUM_PHASES] = {0};

    int fail(int code, const std::string& m) { err = m; return code; }
};

enum { PH_DETECT = 0, PH_ASSEMBLE, PH_SOLVE, PH_ENERGY, PH_CCD, PH_OTHER, PH_EQUERY, PH_SPMV,
       PH_ASM_KEYS, PH_ASM_BODY, PH_ASM_CONTACT, PH_ASM_INV, PH_DENSE, PH_SWEPT, PH_ELIST, PH_TRIALS, PH_BAND };

// Bracket device work with events when timing is on.  phase_begin returns a
// record index (or -1), phase_end closes it with the algorithmic bytes moved.
int phase_begin(Engine* E, int phase);
void phase_end(Engine* E, int rec, double bytes);
void phase_collect(Engine* E);   // after a stream sync: fold finished records into the totals

// per-scene double slots (scd[slot*ns + s])
enum {
    SD_RES = 0, SD_GG, SD_ALPHA, SD_E0, SD_E1, SD_E0N, SD_E1N, SD_TOI, SD_BB,
    // six Krylov dot-product rings of three slots each
    SD_K0, SD_K1 = SD_K0 + 3, SD_K2 = SD_K1 + 3, SD_K3 = SD_K2 + 3, SD_K4 = SD_K3 + 3, SD_K5 = SD_K4 + 3,
    SD_KS = SD_K5 + 3, SD_KA, SD_KW,   // BiCGSTAB running scalars rho, alpha, omega (even iterations)
    SD_KR, SD_KR1, SD_KR2,          // the same for odd iterations
    SD_PAD,
    SD_COUNT
};
// per-scene int slots
enum { SI_DONE = 0, SI_ITER, SI_ACC, SI_KDONE, SI_KITER, SI_NACT, SI_STALL, SI_GACT, SI_GSTALL, SI_DUBAD, SI_COUNT };

// The units the line search runs over: scenes (one step length per scene,
// the reference's line search) or contact groups (ls_groups).  bunit maps a
// body to its unit; d and i hold the unit scalars in the SD_* / SI_* layouts
// with n slots each.
struct LsUnits { int n; const int* bunit; double* d; int* i; };
inline LsUnits scene_units(Engine* E) { return LsUnits{E->ns, E->bscene, E->scd, E->sci}; }
inline LsUnits group_units(Engine* E) { return LsUnits{E->nb, E->grp, E->gscd, E->gsci}; }

// a host round trip on the handle's stream, counted for AbdStepStats.host_syncs
inline cudaError_t eng_stream_sync(Engine* E) { E->host_syncs++; return cudaStreamSynchronize(E->stream); }

// iteration cap of one additive-CCD query
inline int ccd_iters(const AbdParams& P) { return P.ccd_max_iter > 0 ? P.ccd_max_iter : ABD_CCD_MAX_ITER; }

// launch helpers
inline int grid_for(long n, int block = 256) {
    long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > NUM_SMS * 16) g = NUM_SMS * 16;
    return (int)g;
}
// index of block (r, c) in the block CSR, -1 when absent
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
#define GS_LOOP(i, n) for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < (long)(n); i += (long)gridDim.x * blockDim.x)

// implemented in the .cu files
// launch-shape autotuner (capi.cu): tune_begin returns the candidate index to
// launch (the chosen one once timed, the default when autotune is off) and
// brackets it with events until every candidate was timed TUNE_REPS times
enum { TK_CONTACT = 0, TK_LIST_ENERGY, TK_BODY_ENERGY, TK_COUNT };
// contact assembly: one warp per contact with 2, 4 (default) or 8 per block,
// or one block of 64 or 128 threads per contact
constexpr int TUNE_CONTACT_THREADS[5] = {64, 128, 256, 64, 128};
constexpr int TUNE_CONTACT_PER_BLOCK[5] = {2, 4, 8, 1, 1};
constexpr int TUNE_THREADS[4] = {64, 128, 256, 512};         // defaults 128 (list energy), 256 (body energy)
constexpr int TUNE_REPS = 3;
int tune_begin(Engine* E, int kernel, int ncand, int dflt);
void tune_end(Engine* E, int kernel);
int eng_alloc(Engine* E);
void eng_free(Engine* E);
int eng_transform(Engine* E);
int eng_detect(Engine* E, double filt);               // sorted candidate list at the nxt state
int eng_energy(Engine* E, int slot);                   // per-scene energy into scd[slot]
int eng_assemble(Engine* E);                           // g and blocks at the nxt state (uses the candidate list)
int eng_solve(Engine* E, int* iters, bool first_iter = false);   // du = A^-1 g for scenes not done
int eng_solve_direct(Engine* E, int* iters, int* fallback);   // dense factorization per connected component
void eng_dense_free(Engine* E);
void eng_features_free(Engine* E);
void eng_mlp_free(Engine* E);
int eng_features(Engine* E, float* feat_dev);     // per-body features at the nxt state
int eng_learned_ws(Engine* E);                     // network increment into ws
long long eng_dense_bytes(Engine* E);
int eng_ccd(Engine* E, const double* dq, double sign); // per-scene toi into scd[SD_TOI]
int eng_step(Engine* E, int n_steps, AbdStepStats* stats);
int eng_intersections(Engine* E, int* count);
int eng_sync_counters(Engine* E);
int eng_asm_wait(Engine* E);                           // counters and block keys of the last assembly on the host
int eng_assemble_keys_ahead(Engine* E);               // the next iterate's block keys, before the iteration's sync
void eng_keys_ahead_synced(Engine* E);                // after that sync: keys on the host unless the detection overflowed
int eng_grid_build(Engine* E, Grid& G);
GridView eng_view(const Grid& G);
int eng_swept(Engine* E, const double* dq, double sign, const int* done);
int eng_ccd_list(Engine* E, const LsUnits& U, const int* skip);
// dev_count: the listed-pair kernel reads the list length from
// dcnt->ls_nsw and runs a fixed grid (for a graph that outlives one list)
int eng_energy_list(Engine* E, const LsUnits& U, int slot, const int* skip, bool dev_count = false);
void eng_lsgraph_free(Engine* E);
int eng_groups(Engine* E, const int* done);   // contact groups of the listed step (after eng_swept)
void eng_groups_free(Engine* E);
int eng_detect_list(Engine* E);
int eng_swept_bp(Engine* E, double lim);
int eng_detect_bp(Engine* E, double filt);
void eng_bp_free(Engine* E);
bool eng_use_bp(const Engine* E);
