// capi.cu — the extern "C" entry points of libabd_b200.so (include/abd_b200.h)
// and the handle's device allocations.
#include "contact.cuh"
#include <cub/cub.cuh>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

static std::string g_err;
std::string& abd_global_error() { return g_err; }

int eng_energy_masked(Engine* E, int slot, const int* skip);
Geo eng_geo(Engine* E);

template <class T>
static int dalloc(Engine* E, T** p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) return E->fail(ABD_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    return ABD_OK;
}
#define DALLOC(p, n) do { int rc_ = dalloc(E, &(p), (size_t)(n)); if (rc_) return rc_; } while (0)

static int next_pow2(int n) { int h = 1; while (h < n) h <<= 1; return h; }
static int log2i(int h) { int b = 0; while ((1 << b) < h) b++; return b; }

static int grid_alloc(Engine* E, Grid& G, int n, int nq) {
    G.n = n; G.nq = nq;
    G.H = next_pow2(std::max(2 * n, 64)); G.bits = log2i(G.H);
    DALLOC(G.lo, n); DALLOC(G.hi, n); DALLOC(G.scene, n);
    DALLOC(G.qlo, nq); DALLOC(G.qhi, nq); DALLOC(G.qscene, nq);
    DALLOC(G.cell, 1);
    DALLOC(G.keys, n); DALLOC(G.keys_s, n); DALLOC(G.vals, n); DALLOC(G.vals_s, n);
    DALLOC(G.bstart, G.H); DALLOC(G.bend, G.H);
    DALLOC(G.qcount, std::max(nq, n) + 1); DALLOC(G.qoff, std::max(nq, n) + 1);
    return ABD_OK;
}
static void grid_free(Grid& G) {
    void* ps[] = {G.lo, G.hi, G.scene, G.qlo, G.qhi, G.qscene, G.cell, G.keys, G.keys_s, G.vals, G.vals_s,
                  G.bstart, G.bend, G.qcount, G.qoff};
    for (void* p : ps) if (p) cudaFree(p);
    G = Grid();
}

static size_t cub_need(Engine* E, int nkeys64) {
    size_t need = 0, b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, E->sw_cap + 1);
    need = std::max(need, b);
    int nmax = std::max(std::max(E->ne, E->nt), 1);
    cub::DeviceRadixSort::SortPairs(nullptr, b, (uint32_t*)nullptr, (uint32_t*)nullptr, (int*)nullptr, (int*)nullptr, nmax);
    need = std::max(need, b);
    cub::DeviceRadixSort::SortKeys(nullptr, b, (unsigned long long*)nullptr, (unsigned long long*)nullptr, nkeys64);
    need = std::max(need, b);
    cub::DeviceSelect::Unique(nullptr, b, (unsigned long long*)nullptr, (unsigned long long*)nullptr, (int*)nullptr, nkeys64);
    need = std::max(need, b);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (int*)nullptr, (int*)nullptr, std::max(E->ne, E->nv) + 1);
    need = std::max(need, b);
    return need;
}

int eng_grow_blocks(Engine* E, int need) {
    int cap = std::max(need, 2 * E->blk_cap);
    cudaStreamSynchronize(E->stream);
    if (E->bcol) cudaFree(E->bcol);
    if (E->vals) cudaFree(E->vals);
    E->bcol = nullptr; E->vals = nullptr;
    DALLOC(E->bcol, cap);
    size_t es = E->mixed ? sizeof(float) : sizeof(double);
    cudaError_t e = cudaMalloc(&E->vals, (size_t)cap * 144 * es);
    if (e != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc blocks");
    E->blk_cap = cap;
    return ABD_OK;
}

int eng_grow_contacts(Engine* E, int need) {
    int cap = std::max(need + need / 4 + 1024, 2 * E->cap);
    cudaStreamSynchronize(E->stream);
    void* ps[] = {E->contacts, E->cst, E->ctype, E->cxb, E->cbody, E->keys, E->keys_s, E->ukeys, E->cub_tmp};
    for (void* p : ps) if (p) cudaFree(p);
    E->cap = cap;
    int nkeys = E->nb + 2 * cap;
    DALLOC(E->contacts, cap); DALLOC(E->cst, cap); DALLOC(E->ctype, cap); DALLOC(E->cxb, cap); DALLOC(E->cbody, cap);
    DALLOC(E->keys, nkeys); DALLOC(E->keys_s, nkeys); DALLOC(E->ukeys, nkeys);
    E->cub_bytes = cub_need(E, nkeys);
    cudaError_t e = cudaMalloc(&E->cub_tmp, E->cub_bytes);
    if (e != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc cub scratch");
    return ABD_OK;
}

bool eng_use_bp(const Engine* E) {
    return E->bd_ok && (E->P.broadphase == 2 || E->P.broadphase == 0);
}

int eng_grow_swept(Engine* E, int need) {
    int cap = std::max(need + need / 4 + 1024, 2 * E->sw_cap);
    cudaStreamSynchronize(E->stream);
    void* ps[] = {E->sw, E->sw_flag, E->sw_off, E->cub_tmp};
    for (void* p : ps) if (p) cudaFree(p);
    E->sw = nullptr; E->sw_flag = nullptr; E->sw_off = nullptr; E->cub_tmp = nullptr;
    E->sw_cap = cap;
    DALLOC(E->sw, cap); DALLOC(E->sw_flag, cap + 1); DALLOC(E->sw_off, cap + 1);
    E->cub_bytes = cub_need(E, E->nb + 2 * E->cap);
    if (cudaMalloc(&E->cub_tmp, E->cub_bytes) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc cub scratch");
    E->sw_valid = false;
    return ABD_OK;
}

int eng_alloc(Engine* E) {
    int nb = E->nb, nv = E->nv, ns = E->ns;
    int rc;
    if ((rc = grid_alloc(E, E->gee, E->ne, E->ne))) return rc;
    if ((rc = grid_alloc(E, E->gpt, E->nt, nv))) return rc;
    DALLOC(E->st, 48L * nb); DALLOC(E->backup, 12L * nb); DALLOC(E->du, 12L * nb); DALLOC(E->g, 12L * nb);
    DALLOC(E->x, 3L * nv); DALLOC(E->xf, nv); DALLOC(E->pv, 3L * nv); DALLOC(E->ws, 12L * nb);
    E->cap = 0;
    E->sw_cap = std::max(E->P.contact_capacity, 1024);
    if ((rc = eng_grow_contacts(E, std::max(E->P.contact_capacity, 1024) * 4 / 5))) return rc;
    DALLOC(E->sw, E->sw_cap); DALLOC(E->sw_flag, E->sw_cap + 1); DALLOC(E->sw_off, E->sw_cap + 1);
    DALLOC(E->pmag, nv); DALLOC(E->zero_int, 1); DALLOC(E->zero_ns, ns); DALLOC(E->sw_nee, 1);
    cudaMemsetAsync(E->zero_int, 0, sizeof(int), E->stream);
    cudaMemsetAsync(E->sw_nee, 0, sizeof(int), E->stream);
    cudaMemsetAsync(E->zero_ns, 0, sizeof(int) * ns, E->stream);
    DALLOC(E->row_ptr, nb + 1);
    E->blk_cap = 0;
    if ((rc = eng_grow_blocks(E, nb + std::min(2 * E->cap, 8 * nb + 1024)))) return rc;
    size_t es = E->mixed ? sizeof(float) : sizeof(double);
    if (cudaMalloc(&E->dinv, (size_t)nb * 144 * es) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc dinv");
    for (int i = 0; i < 10; i++)
        if (cudaMalloc(&E->kv[i], (size_t)nb * 12 * es) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc krylov");
    DALLOC(E->scd, (size_t)SD_COUNT * ns); DALLOC(E->sci, (size_t)SI_COUNT * ns);
    DALLOC(E->prof_d, (size_t)2 * ns * std::max(E->P.newton_max_iter, 1));
    DALLOC(E->dcnt, 1);
    if (cudaMallocHost(&E->hcnt, sizeof(Counters)) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMallocHost");
    if (cudaMallocHost(&E->hscd, sizeof(double) * ns * SD_COUNT) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMallocHost");
    if (cudaMallocHost(&E->hsci, sizeof(int) * ns * SI_COUNT) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMallocHost");
    cudaMemsetAsync(E->scd, 0, sizeof(double) * SD_COUNT * ns, E->stream);
    cudaMemsetAsync(E->sci, 0, sizeof(int) * SI_COUNT * ns, E->stream);
    cudaMemsetAsync(E->dcnt, 0, sizeof(Counters), E->stream);
    cudaEventCreate(&E->ev0); cudaEventCreate(&E->ev1);
    cudaEventCreateWithFlags(&E->ev_asm, cudaEventDisableTiming);
    return ABD_OK;
}

void eng_free(Engine* E) {
    for (auto& t : E->tune) { if (t.a) cudaEventDestroy(t.a); if (t.b) cudaEventDestroy(t.b); }
    eng_dense_free(E);
    eng_features_free(E);
    eng_mlp_free(E);
    eng_bp_free(E);
    eng_groups_free(E);
    eng_lsgraph_free(E);
    void* bd[] = {E->bd_vbeg, E->bd_ebeg, E->bd_tbeg};
    for (void* p : bd) if (p) cudaFree(p);
    grid_free(E->gee); grid_free(E->gpt);
    if (E->st_in) cudaFree(E->st_in);
    if (E->h_ukeys) cudaFreeHost(E->h_ukeys);
    if (E->h_done) cudaFreeHost(E->h_done);
    void* ps[] = {E->xbar, E->vbody, E->vscene, E->bscene, E->edges, E->tris, E->mass, E->J, E->planes, E->plane_scene,
                  E->sc_plane_begin, E->sc_body_begin, E->edge_scene, E->tri_scene, E->st, E->backup, E->du, E->g, E->x,
                  E->xf, E->pv, E->ws, E->contacts, E->cst, E->ctype, E->cxb, E->cbody, E->cblk, E->keys, E->keys_s,
                  E->ukeys, E->row_ptr, E->bcol, E->vals, E->dinv, E->scd, E->sci, E->cub_tmp, E->dcnt, E->prof_d,
                  E->sw, E->sw_flag, E->sw_off, E->pmag, E->zero_int, E->zero_ns, E->sw_nee};
    for (void* p : ps) if (p) cudaFree(p);
    for (int i = 0; i < 10; i++) if (E->kv[i]) cudaFree(E->kv[i]);
    if (E->hcnt) cudaFreeHost(E->hcnt);
    if (E->hscd) cudaFreeHost(E->hscd);
    if (E->hsci) cudaFreeHost(E->hsci);
    if (E->ev0) cudaEventDestroy(E->ev0);
    if (E->ev1) cudaEventDestroy(E->ev1);
    if (E->ev_asm) cudaEventDestroy(E->ev_asm);
    if (E->stream) cudaStreamDestroy(E->stream);
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int abd_abi_version(void) { return ABD_ABI_VERSION; }

void abd_default_params(AbdParams* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->dt = 8e-3;                                 // links.py:16
    p->gravity[0] = 0.0; p->gravity[1] = -10.0; p->gravity[2] = 0.0;   // abd.py:28
    p->kappa = 4e8;                               // abd.py:30
    p->k_ortho = 1e5;                             // ortho.py:5
    p->dhat = 0.0475 * 2;                         // barrier.py:4
    p->cand_dist = (0.0475 + 0.0475) * 2.0;       // contact.py:7-9, :168
    p->barrier = ABD_BARRIER_CUBIC;               // barrier.py:47-65
    p->hess_mode = ABD_HESS_REFERENCE;
    p->contact_ee = 1; p->contact_pt = 0; p->self_contact = 1; p->ee_f32 = 1;
    p->linear_solver = ABD_SOLVER_BICGSTAB;       // abd.py:636
    p->lin_max_iter = 1000; p->lin_tol = 1e-5;
    p->newton_tol = 1e-5; p->newton_max_iter = 16;   // abd.py:679, :699
    p->ccd = 0; p->ccd_scale = 0.1;
    p->ls_min_alpha = 1e-2;                       // gauss_newton.py:110
    p->precision = ABD_PREC_FP64;
    p->contact_capacity = 1 << 16;
    p->pinned_diag = 100.0;                       // abd.py:146
    p->autotune = 1;
    p->ccd_max_iter = ABD_CCD_MAX_ITER;
}

const char* abd_last_error(AbdHandle* h) {
    if (!h) return g_err.c_str();
    return reinterpret_cast<Engine*>(h)->err.c_str();
}

#define HANDLE(h) Engine* E = reinterpret_cast<Engine*>(h); if (!E) { g_err = "null handle"; return ABD_ERR_INVALID_ARG; } \
    if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaSetDevice")

int abd_create(const AbdParams* params, const AbdSceneDesc* scenes, int32_t n_scenes, int32_t device, AbdHandle** out) {
    if (!params || !scenes || n_scenes <= 0 || !out) { g_err = "abd_create: invalid argument"; return ABD_ERR_INVALID_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { g_err = "abd_create: no CUDA device"; return ABD_ERR_NO_DEVICE; }
    if (device < 0 || device >= ndev) { g_err = "abd_create: bad device index"; return ABD_ERR_INVALID_ARG; }
    const AbdParams& P = *params;
    if (!(P.dt > 0) || !(P.dhat > 0) || !(P.cand_dist >= P.dhat) || P.newton_max_iter <= 0 || P.lin_max_iter <= 0 ||
        P.barrier < 0 || P.barrier > 2 || P.contact_capacity <= 0 || P.linear_solver < 0 || P.linear_solver > 3 || (P.ccd && !(P.ccd_scale > 0 && P.ccd_scale < 1)) ||
        P.ls_groups < 0 || P.ls_groups > 1 || P.ls_graph < 0 || P.ls_graph > 1 || P.ccd_max_iter < 0 ||
        (P.test_inject & ~(ABD_INJECT_DU_NONFINITE | ABD_INJECT_SWEPT_FULL))) {
        g_err = "abd_create: invalid parameters (dt, dhat <= cand_dist, iteration caps, barrier, capacity, ccd_scale, ls_groups, ls_graph)";
        return ABD_ERR_INVALID_ARG;
    }
    Engine* E = new (std::nothrow) Engine();
    if (!E) { g_err = "abd_create: out of host memory"; return ABD_ERR_INVALID_ARG; }
    E->P = P; E->device = device; E->ns = n_scenes; E->mixed = P.precision == ABD_PREC_MIXED;
    cudaSetDevice(device);
    // concatenate the scenes
    std::vector<double> xbar, mass, J, st, planes;
    std::vector<int> vbody, vscene, bscene, edges, tris, escene, tscene, pscene, sc_plane_begin, sc_body_begin;
    int nb = 0, nv = 0, npl = 0;
    sc_plane_begin.push_back(0); sc_body_begin.push_back(0);
    for (int s = 0; s < n_scenes; s++) {
        const AbdSceneDesc& D = scenes[s];
        if (D.n_bodies <= 0 || D.n_verts <= 0 || D.n_edges < 0 || D.n_tris < 0 || D.n_planes < 0 || !D.xbar ||
            !D.vert_body || !D.mass || !D.inertia_J || !D.state || (D.n_edges && !D.edges) || (D.n_tris && !D.tris) ||
            (D.n_planes && !D.planes)) {
            delete E; g_err = "abd_create: invalid scene descriptor " + std::to_string(s); return ABD_ERR_INVALID_ARG;
        }
        for (int v = 0; v < D.n_verts; v++) {
            int b = D.vert_body[v];
            if (b < 0 || b >= D.n_bodies) { delete E; g_err = "abd_create: vert_body out of range"; return ABD_ERR_INVALID_ARG; }
            for (int k = 0; k < 3; k++) xbar.push_back(D.xbar[3*v+k]);
            vbody.push_back(b + nb); vscene.push_back(s);
        }
        for (int e = 0; e < D.n_edges; e++) {
            int a = D.edges[2*e], b = D.edges[2*e+1];
            if (a < 0 || b < 0 || a >= D.n_verts || b >= D.n_verts || a == b) { delete E; g_err = "abd_create: bad edge"; return ABD_ERR_INVALID_ARG; }
            edges.push_back(a + nv); edges.push_back(b + nv); escene.push_back(s);
        }
        for (int t = 0; t < D.n_tris; t++) {
            for (int k = 0; k < 3; k++) {
                int a = D.tris[3*t+k];
                if (a < 0 || a >= D.n_verts) { delete E; g_err = "abd_create: bad triangle"; return ABD_ERR_INVALID_ARG; }
                tris.push_back(a + nv);
            }
            tscene.push_back(s);
        }
        for (int b = 0; b < D.n_bodies; b++) {
            mass.push_back(D.mass[b]); J.push_back(D.inertia_J[b]); bscene.push_back(s);
            for (int k = 0; k < 48; k++) st.push_back(D.state[48*b+k]);
        }
        for (int p = 0; p < D.n_planes; p++) { for (int k = 0; k < 4; k++) planes.push_back(D.planes[4*p+k]); pscene.push_back(s); }
        nb += D.n_bodies; nv += D.n_verts; npl += D.n_planes;
        sc_plane_begin.push_back(npl); sc_body_begin.push_back(nb);
    }
    E->nb = nb; E->nv = nv; E->ne = (int)escene.size(); E->nt = (int)tscene.size(); E->npl = npl;
    E->h_body_begin = sc_body_begin;
    for (int s = 0; s < n_scenes; s++) {
        long long m = sc_body_begin[s + 1] - sc_body_begin[s];
        E->dense_blocks += m * m;
    }
    E->h_bscene = bscene;
    E->h_edges = edges; E->h_tris = tris;
    if (cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking) != cudaSuccess) { delete E; g_err = "stream"; return ABD_ERR_CUDA; }
    if (P.broadphase < 0 || P.broadphase > 2) { delete E; g_err = "abd_create: broadphase must be 0, 1 or 2"; return ABD_ERR_INVALID_ARG; }
    if (P.warm_start < 0 || P.warm_start > 3) { delete E; g_err = "abd_create: warm_start must be 0..3"; return ABD_ERR_INVALID_ARG; }
    auto up = [&](auto*& dst, auto& src) -> int {
        using T = typename std::remove_reference<decltype(src)>::type::value_type;
        int rc = dalloc(E, (T**)&dst, src.size());
        if (rc) return rc;
        if (!src.empty() && cudaMemcpy((void*)dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMemcpy");
        return ABD_OK;
    };
    int rc = 0;
    int* edges_i = nullptr;
    if ((rc = up(E->xbar, xbar)) || (rc = up(E->vbody, vbody)) || (rc = up(E->vscene, vscene)) ||
        (rc = up(E->bscene, bscene)) || (rc = up(edges_i, edges)) || (rc = up(E->tris, tris)) ||
        (rc = up(E->mass, mass)) || (rc = up(E->J, J)) || (rc = up(E->planes, planes)) ||
        (rc = up(E->plane_scene, pscene)) || (rc = up(E->sc_plane_begin, sc_plane_begin)) ||
        (rc = up(E->sc_body_begin, sc_body_begin)) || (rc = up(E->edge_scene, escene)) ||
        (rc = up(E->tri_scene, tscene)) || (rc = eng_alloc(E))) {
        g_err = E->err; eng_free(E); delete E; return rc;
    }
    E->edges = reinterpret_cast<int2*>(edges_i);
    // per-body primitive ranges for the body-pair broad phase
    {
        std::vector<int> vb(nb + 1, 0), eb(nb + 1, 0), tb(nb + 1, 0);
        bool ok = true;
        auto ranges = [&](const std::vector<int>& owner, std::vector<int>& beg) {
            int cur = 0; beg[0] = 0;
            for (size_t i = 0; i < owner.size(); i++) {
                int b = owner[i];
                if (b < cur) { ok = false; return; }
                while (cur < b) { beg[++cur] = (int)i; }
            }
            while (cur < nb) beg[++cur] = (int)owner.size();
        };
        std::vector<int> eown(E->ne), town(E->nt);
        for (int e = 0; e < E->ne; e++) eown[e] = vbody[edges[2*e]];
        for (int t = 0; t < E->nt; t++) {
            int b0 = vbody[tris[3*t]];
            if (vbody[tris[3*t+1]] != b0 || vbody[tris[3*t+2]] != b0) ok = false;
            town[t] = b0;
        }
        for (int e = 0; e < E->ne; e++) if (vbody[edges[2*e+1]] != eown[e]) ok = false;
        ranges(vbody, vb); ranges(eown, eb); ranges(town, tb);
        E->bd_ok = ok;
        if (!ok && P.ls_groups) {
            g_err = "abd_create: ls_groups needs every body to own a contiguous vertex range"; eng_free(E); delete E;
            return ABD_ERR_INVALID_ARG;
        }
        if (ok && ((rc = up(E->bd_vbeg, vb)) || (rc = up(E->bd_ebeg, eb)) || (rc = up(E->bd_tbeg, tb)))) {
            g_err = E->err; eng_free(E); delete E; return rc;
        }
    }
    if (cudaMemcpy(E->st, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        g_err = "cudaMemcpy state"; eng_free(E); delete E; return ABD_ERR_CUDA;
    }
    if (cudaStreamSynchronize(E->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        g_err = "abd_create: CUDA error during set-up"; eng_free(E); delete E; return ABD_ERR_CUDA;
    }
    *out = reinterpret_cast<AbdHandle*>(E);
    return ABD_OK;
}

int abd_destroy(AbdHandle* h) {
    Engine* E = reinterpret_cast<Engine*>(h);
    if (!E) return ABD_OK;
    cudaSetDevice(E->device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    eng_free(E);
    delete E;
    return ABD_OK;
}

int abd_get_sizes(AbdHandle* h, int32_t* nb, int32_t* nv, int32_t* ne, int32_t* nt, int32_t* ns) {
    HANDLE(h);
    if (nb) *nb = E->nb; if (nv) *nv = E->nv; if (ne) *ne = E->ne; if (nt) *nt = E->nt; if (ns) *ns = E->ns;
    return ABD_OK;
}

// flags a body whose nxt position (c, q) differs bit for bit from the
// incoming state
__global__ void k_positions_differ(int nb, const double* __restrict__ cur, const double* __restrict__ in, int* flag) {
    GS_LOOP(i, 12L * nb) {
        long b = i / 12; int k = (int)(i % 12);
        long o = ST_STRIDE * b + ST_NXT + k;
        if (__double_as_longlong(cur[o]) != __double_as_longlong(in[o])) *flag = 1;
    }
}

int abd_set_state(AbdHandle* h, const double* st, int32_t n) {
    HANDLE(h);
    if (!st || n != E->nb) return E->fail(ABD_ERR_INVALID_ARG, "abd_set_state: n_bodies mismatch");
    for (long i = 0; i < 48L * n; i++)
        if (!std::isfinite(st[i]))
            return E->fail(ABD_ERR_NAN, "abd_set_state: non-finite value at body " + std::to_string(i / 48) +
                                        ", entry " + std::to_string(i % 48) + " (state left unchanged)");
    const size_t bytes = sizeof(double) * 48 * n;
    if (!E->st_in && cudaMalloc(&E->st_in, bytes) != cudaSuccess) { E->st_in = nullptr; return E->fail(ABD_ERR_CUDA, "cudaMalloc state staging"); }
    // the swept candidate list covers the current positions: it stays valid
    // when the caller hands back the positions it read (a host loop that
    // round-trips the state every step)
    CUDA_TRY(cudaMemcpyAsync(E->st_in, st, bytes, cudaMemcpyHostToDevice, E->stream));
    CUDA_TRY(cudaMemsetAsync(&E->dcnt->pos_changed, 0, sizeof(int), E->stream));
    k_positions_differ<<<grid_for(12L * n), 256, 0, E->stream>>>(n, E->st, E->st_in, &E->dcnt->pos_changed);
    CUDA_TRY(cudaMemcpyAsync(E->st, E->st_in, bytes, cudaMemcpyDeviceToDevice, E->stream));
    CUDA_TRY(cudaMemcpyAsync(&E->hcnt->pos_changed, &E->dcnt->pos_changed, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    if (E->hcnt->pos_changed) E->sw_valid = false;
    return ABD_OK;
}

int abd_get_state(AbdHandle* h, double* st) {
    HANDLE(h);
    if (!st) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_state: null");
    CUDA_TRY(cudaMemcpyAsync(st, E->st, sizeof(double) * 48 * E->nb, cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    return ABD_OK;
}

int abd_step(AbdHandle* h, int32_t n_steps, AbdStepStats* stats) {
    HANDLE(h);
    if (n_steps < 0) return E->fail(ABD_ERR_INVALID_ARG, "abd_step: n_steps < 0");
    int rc = eng_step(E, n_steps, stats);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return E->fail(ABD_ERR_CUDA, std::string("abd_step: ") + cudaGetErrorString(e));
    return rc;
}

int abd_get_profile(AbdHandle* h, int32_t scene, double* res, double* alpha, int32_t* ips, int32_t cap, int32_t* n) {
    HANDLE(h);
    if (scene < 0 || scene >= E->ns || !n) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_profile: bad scene");
    if (E->prof_res.size() != (size_t)E->ns) { *n = 0; return ABD_OK; }
    const auto& r = E->prof_res[scene]; const auto& a = E->prof_alpha[scene]; const auto& it = E->prof_iters[scene];
    int m = std::min<int>((int)r.size(), cap);
    for (int i = 0; i < m; i++) { if (res) res[i] = r[i]; if (alpha) alpha[i] = a[i]; }
    if (ips) for (int i = 0; i < (int)it.size() && i < cap; i++) ips[i] = it[i];
    *n = m;
    return ABD_OK;
}

int abd_get_vertices(AbdHandle* h, double* x) {
    HANDLE(h);
    if (!x) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_vertices: null");
    eng_transform(E);
    CUDA_TRY(cudaMemcpyAsync(x, E->x, sizeof(double) * 3 * E->nv, cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    return ABD_OK;
}

static int detect_full(Engine* E) {
    int rc;
    for (;;) {
        if ((rc = eng_use_bp(E) ? eng_detect_bp(E, E->P.cand_dist) : eng_detect(E, E->P.cand_dist))) return rc;
        if ((rc = eng_sync_counters(E))) return rc;
        if (!E->hcnt->overflow) return ABD_OK;
        if ((rc = eng_grow_contacts(E, E->hcnt->n_total))) return rc;
    }
}

int abd_get_pairs(AbdHandle* h, int32_t* out4, int32_t* kinds, int32_t cap, int32_t* n) {
    HANDLE(h);
    if (!n || (cap > 0 && !out4)) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_pairs: null");
    int rc = detect_full(E);
    if (rc) return rc;
    int tot = E->hcnt->n_total;
    std::vector<int4> c(tot);
    if (tot) CUDA_TRY(cudaMemcpy(c.data(), E->contacts, sizeof(int4) * tot, cudaMemcpyDeviceToHost));
    int m = std::min(tot, cap);
    for (int i = 0; i < m; i++) {
        int32_t* o = out4 + 4 * i;
        if (c[i].x == ABD_CONTACT_EE) {
            o[0] = E->h_edges[2*c[i].y]; o[1] = E->h_edges[2*c[i].y+1]; o[2] = E->h_edges[2*c[i].z]; o[3] = E->h_edges[2*c[i].z+1];
        } else if (c[i].x == ABD_CONTACT_PT) {
            o[0] = c[i].y; o[1] = E->h_tris[3*c[i].z]; o[2] = E->h_tris[3*c[i].z+1]; o[3] = E->h_tris[3*c[i].z+2];
        } else { o[0] = c[i].y; o[1] = c[i].z; o[2] = -1; o[3] = -1; }
        if (kinds) kinds[i] = c[i].x;
    }
    *n = tot;
    return tot > cap ? E->fail(ABD_ERR_CONTACT_OVERFLOW, "abd_get_pairs: cap smaller than the pair count") : ABD_OK;
}

// abd.py:759-766 get_contact_points: midpoint of the EE closest points and distance
__global__ void k_contact_points(const Counters* cnt, const int4* __restrict__ contacts, Geo G, int f32,
                                 double* pts, double* dists, int cap) {
    int n = min(cnt->n_total, cap);
    GS_LOOP(i, n) {
        int4 C = contacts[i];
        double px = 0, py = 0, pz = 0, d = 0;
        if (C.x == ABD_CONTACT_EE) {
            int2 a = G.edges[C.y], b = G.edges[C.z];
            double s, t;
            ee_test(G, C.y, C.z, f32, 1, 1e300, s, t, d);
            double v0[3], v1[3];
            for (int k = 0; k < 3; k++) {
                v0[k] = G.x[3*a.x+k] + s * (G.x[3*a.y+k] - G.x[3*a.x+k]);
                v1[k] = G.x[3*b.x+k] + t * (G.x[3*b.y+k] - G.x[3*b.x+k]);
            }
            px = 0.5 * (v0[0] + v1[0]); py = 0.5 * (v0[1] + v1[1]); pz = 0.5 * (v0[2] + v1[2]);
        } else if (C.x == ABD_CONTACT_PT) {
            int t0 = G.tris[3*C.z], t1 = G.tris[3*C.z+1], t2 = G.tris[3*C.z+2];
            d = sqrt(pt_dist2(G.x + 3*C.y, G.x + 3*t0, G.x + 3*t1, G.x + 3*t2));
            px = G.x[3*C.y]; py = G.x[3*C.y+1]; pz = G.x[3*C.y+2];
        } else {
            const double* nn = G.planes + 4*C.z;
            d = nn[0] * G.x[3*C.y] + nn[1] * G.x[3*C.y+1] + nn[2] * G.x[3*C.y+2] - nn[3];
            px = G.x[3*C.y]; py = G.x[3*C.y+1]; pz = G.x[3*C.y+2];
        }
        pts[3*i] = px; pts[3*i+1] = py; pts[3*i+2] = pz; dists[i] = d;
    }
}

int abd_get_contact_points(AbdHandle* h, double* pts, double* dists, int32_t cap, int32_t* n) {
    HANDLE(h);
    if (!n || (cap > 0 && (!pts || !dists))) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_contact_points: null");
    int rc = detect_full(E);
    if (rc) return rc;
    int tot = E->hcnt->n_total, m = std::min(tot, cap);
    double *dp = nullptr, *dd = nullptr;
    if (m > 0) {
        CUDA_TRY(cudaMalloc(&dp, sizeof(double) * 3 * m));
        CUDA_TRY(cudaMalloc(&dd, sizeof(double) * m));
        k_contact_points<<<grid_for(m), 256, 0, E->stream>>>(E->dcnt, E->contacts, eng_geo(E), E->P.ee_f32, dp, dd, m);
        CUDA_TRY(cudaMemcpyAsync(pts, dp, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, E->stream));
        CUDA_TRY(cudaMemcpyAsync(dists, dd, sizeof(double) * m, cudaMemcpyDeviceToHost, E->stream));
        CUDA_TRY(cudaStreamSynchronize(E->stream));
        cudaFree(dp); cudaFree(dd);
    }
    *n = tot;
    return ABD_OK;
}

int abd_energy(AbdHandle* h, double* e) {
    HANDLE(h);
    if (!e) return E->fail(ABD_ERR_INVALID_ARG, "abd_energy: null");
    int* skip = E->sci + SI_NACT * E->ns;
    CUDA_TRY(cudaMemsetAsync(skip, 0, sizeof(int) * E->ns, E->stream));
    int rc = eng_energy_masked(E, SD_E0, skip);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(e, E->scd + SD_E0 * E->ns, sizeof(double) * E->ns, cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    return ABD_OK;
}

static int assemble_full(Engine* E) {
    E->keys_ahead = false;           // block keys are built by this assembly itself
    CUDA_TRY(cudaMemsetAsync(E->sci + SI_DONE * E->ns, 0, sizeof(int) * E->ns, E->stream));
    int rc = detect_full(E);
    if (rc) return rc;
    if ((rc = eng_assemble(E))) return rc;
    return eng_asm_wait(E);
}

int abd_assemble(AbdHandle* h, double* grad, double* hess) {
    HANDLE(h);
    if (!grad) return E->fail(ABD_ERR_INVALID_ARG, "abd_assemble: null");
    if (hess && E->nb > 512) return E->fail(ABD_ERR_INVALID_ARG, "abd_assemble: dense Hessian only for n_bodies <= 512");
    int rc = assemble_full(E);
    if (rc) return rc;
    CUDA_TRY(cudaMemcpyAsync(grad, E->g, sizeof(double) * 12 * E->nb, cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    if (hess) {
        if ((rc = eng_sync_counters(E))) return rc;
        int nnzb;
        nnzb = E->hcnt->nnzb;
        std::vector<int> rp(E->nb + 1), col(nnzb);
        size_t es = E->mixed ? 4 : 8;
        std::vector<char> vals((size_t)nnzb * 144 * es);
        CUDA_TRY(cudaMemcpy(rp.data(), E->row_ptr, sizeof(int) * (E->nb + 1), cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(col.data(), E->bcol, sizeof(int) * nnzb, cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(vals.data(), E->vals, vals.size(), cudaMemcpyDeviceToHost));
        long n = 12L * E->nb;
        memset(hess, 0, sizeof(double) * n * n);
        for (int r = 0; r < E->nb; r++)
            for (int k = rp[r]; k < rp[r+1]; k++)
                for (int c = 0; c < 12; c++)
                    for (int rr = 0; rr < 12; rr++) {
                        double v = E->mixed ? (double)((float*)vals.data())[(size_t)k * 144 + c * 12 + rr]
                                            : ((double*)vals.data())[(size_t)k * 144 + c * 12 + rr];
                        hess[(12L * r + rr) * n + 12L * col[k] + c] = v;
                    }
    }
    return ABD_OK;
}

int abd_solve(AbdHandle* h, double* du, int32_t* iters) {
    HANDLE(h);
    if (!du) return E->fail(ABD_ERR_INVALID_ARG, "abd_solve: null");
    int rc = assemble_full(E);
    if (rc) return rc;
    int it = 0;
    E->solver_capped = 0;
    if ((rc = eng_solve(E, &it))) return rc;
    CUDA_TRY(cudaMemcpyAsync(du, E->du, sizeof(double) * 12 * E->nb, cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    if (iters) *iters = it;
    if (E->solver_capped) return E->fail(ABD_ERR_SOLVER_CAP, "abd_solve: Krylov iteration cap reached above tolerance");
    return ABD_OK;
}

int abd_set_warm_start(AbdHandle* h, const float* dq, int32_t n) {
    HANDLE(h);
    if (!dq || n != E->nb) return E->fail(ABD_ERR_INVALID_ARG, "abd_set_warm_start: n_bodies mismatch");
    std::vector<double> w(12L * n);
    for (long i = 0; i < 12L * n; i++) w[i] = dq[i];
    CUDA_TRY(cudaMemcpyAsync(E->ws, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, E->stream));
    CUDA_TRY(cudaStreamSynchronize(E->stream));
    E->has_ws = 1;
    return ABD_OK;
}

int abd_get_features(AbdHandle* h, float* feat, int32_t n);   // warmstart.cu

int abd_count_intersections(AbdHandle* h, int32_t* count) {
    HANDLE(h);
    if (!count) return E->fail(ABD_ERR_INVALID_ARG, "abd_count_intersections: null");
    int c = 0;
    int rc = eng_intersections(E, &c);
    *count = c;
    return rc;
}

}  // extern "C"

// ------------------------------------------------------------------ phase timers
static cudaEvent_t pool_get(Engine* E) {
    if (!E->ev_pool.empty()) { cudaEvent_t e = E->ev_pool.back(); E->ev_pool.pop_back(); return e; }
    cudaEvent_t e; cudaEventCreate(&e); return e;
}
int tune_begin(Engine* E, int k, int ncand, int dflt) {
    Engine::Tuner& t = E->tune[k];
    if (!E->P.autotune) return dflt;
    if (t.chosen >= 0) return t.chosen;
    if (E->capturing) return dflt;      // no timing inside a captured graph
    if (!t.a) { cudaEventCreate(&t.a); cudaEventCreate(&t.b); }
    if (t.running >= 0) {
        float ms = 0;
        if (cudaEventSynchronize(t.b) == cudaSuccess && cudaEventElapsedTime(&ms, t.a, t.b) == cudaSuccess) {
            t.sum[t.running] += ms; t.cnt[t.running]++;
        }
        t.running = -1;
    }
    int total = 0;
    for (int c = 0; c < ncand; c++) total += t.cnt[c];
    if (total >= ncand * TUNE_REPS) {
        int best = dflt;
        for (int c = 0; c < ncand; c++)
            if (t.cnt[c] && t.sum[c] / t.cnt[c] < t.sum[best] / std::max(1, t.cnt[best])) best = c;
        t.chosen = best;
        return best;
    }
    int c = t.next;
    t.next = (t.next + 1) % ncand;
    t.running = c;
    cudaEventRecord(t.a, E->stream);
    return c;
}
void tune_end(Engine* E, int k) {
    Engine::Tuner& t = E->tune[k];
    if (E->capturing) return;
    if (t.running >= 0) cudaEventRecord(t.b, E->stream);
}

int phase_begin(Engine* E, int phase) {
    if (!E->timing) return -1;
    Engine::Rec r; r.phase = phase; r.a = pool_get(E); r.b = pool_get(E); r.bytes = 0;
    cudaEventRecord(r.a, E->stream);
    E->recs.push_back(r);
    return (int)E->recs.size() - 1;
}
void phase_end(Engine* E, int rec, double bytes) {
    if (rec < 0 || !E->timing) return;
    E->recs[rec].bytes = bytes;
    cudaEventRecord(E->recs[rec].b, E->stream);
}
void phase_collect(Engine* E) {
    for (auto& r : E->recs) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            E->phase_ms[r.phase] += ms; E->phase_n[r.phase] += 1; E->phase_bytes[r.phase] += r.bytes;
        }
        E->ev_pool.push_back(r.a); E->ev_pool.push_back(r.b);
    }
    E->recs.clear();
}

extern "C" int abd_set_timing(AbdHandle* h, int32_t on, int32_t reset) {
    HANDLE(h);
    cudaStreamSynchronize(E->stream);
    phase_collect(E);
    E->timing = on != 0;
    if (reset) for (int i = 0; i < ABD_NUM_PHASES; i++) { E->phase_ms[i] = 0; E->phase_n[i] = 0; E->phase_bytes[i] = 0; }
    return ABD_OK;
}
extern "C" int abd_get_autotune(AbdHandle* h, int32_t* shapes, int32_t cap, int32_t* n) {
    HANDLE(h);
    if (!n || (cap > 0 && !shapes)) return E->fail(ABD_ERR_INVALID_ARG, "abd_get_autotune: null");
    int v[4];
    int cc = E->tune[TK_CONTACT].chosen;
    v[0] = cc < 0 ? -1 : TUNE_CONTACT_THREADS[cc];
    v[1] = cc < 0 ? -1 : TUNE_CONTACT_PER_BLOCK[cc];
    v[2] = E->tune[TK_LIST_ENERGY].chosen < 0 ? -1 : TUNE_THREADS[E->tune[TK_LIST_ENERGY].chosen];
    v[3] = E->tune[TK_BODY_ENERGY].chosen < 0 ? -1 : TUNE_THREADS[E->tune[TK_BODY_ENERGY].chosen];
    for (int i = 0; i < 4 && i < cap; i++) shapes[i] = v[i];
    *n = 4;
    return ABD_OK;
}

extern "C" int abd_get_timing(AbdHandle* h, double* ms, int64_t* launches, double* bytes) {
    HANDLE(h);
    cudaStreamSynchronize(E->stream);
    phase_collect(E);
    for (int i = 0; i < ABD_NUM_PHASES; i++) {
        if (ms) ms[i] = E->phase_ms[i];
        if (launches) launches[i] = E->phase_n[i];
        if (bytes) bytes[i] = E->phase_bytes[i];
    }
    return ABD_OK;
}
