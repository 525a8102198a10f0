// step.cu — the Newton step (abd.py:674-702) with the reference's
// back-off line search (gauss_newton.py:98-115) and forward_states
// (abd.py:574-581), run for all scenes of a batch at once.  Each scene keeps
// its own iteration count, residual, step length and done flag on the
// device; the host only reads "how many scenes are still iterating".
#include "engine.cuh"

int eng_energy_masked(Engine* E, int slot, const int* skip);

// nxt.c / nxt.q are 12 consecutive doubles in DoF order [c, q0, q1, q2]
__global__ void k_backup(int nb, const double* __restrict__ st, double* backup) {
    GS_LOOP(i, 12L * nb) backup[i] = st[ST_STRIDE * (i / 12) + ST_NXT + (i % 12)];
}
// abd.py:768-785: nxt = backup - alpha du, for scenes not yet accepted
__global__ void k_apply(int nb, const double* __restrict__ backup, const double* __restrict__ du,
                        const double* __restrict__ alpha, const int* __restrict__ skip, const int* __restrict__ bscene,
                        double* st) {
    GS_LOOP(i, 12L * nb) {
        long b = i / 12;
        int s = bscene[b];
        if (skip[s]) continue;
        st[ST_STRIDE * b + ST_NXT + (i % 12)] = __fma_rn(-alpha[s], du[i], backup[i]);
    }
}
// cap: the fraction of the increment the swept list covers (its CCD bound is a
// fraction of that shorter step)
__global__ void k_ls_init(int ns, const int* done, int* acc, double* alpha, const double* toi, int ccd, int* stall,
                          double cap) {
    GS_LOOP(s, ns) {
        acc[s] = done[s];
        alpha[s] = (ccd ? fmin(1.0, toi[s]) : 1.0) * cap;
        if (!done[s]) stall[s] = 0;
    }
}
// contact groups -> scenes: the smallest step length and CCD bound of the
// scene's groups (for the profile and the step statistics); the scene
// stalls when every group that searched gave up below ABD_LS_STALL_ALPHA
__global__ void k_grp_scene_init(int ns, const int* done, double* alpha, double* toi, int* gact, int* gstall) {
    GS_LOOP(s, ns) {
        if (done[s]) continue;
        alpha[s] = 1.0; toi[s] = 1.0; gact[s] = 0; gstall[s] = 0;
    }
}
__global__ void k_grp_to_scenes(int nb, const int* __restrict__ bscene, const int* __restrict__ udone,
                                const double* __restrict__ ualpha, const double* __restrict__ utoi,
                                const int* __restrict__ ustall, int ccd, double* alpha, double* toi, int* gact,
                                int* gstall) {
    GS_LOOP(u, nb) {
        if (udone[u]) continue;
        int s = bscene[u];
        atomic_min_pos(alpha + s, ualpha[u]);
        if (ccd) atomic_min_pos(toi + s, utoi[u]);
        atomicAdd(gact + s, 1);
        if (ustall[u]) atomicAdd(gstall + s, 1);
    }
}
__global__ void k_grp_scene_stall(int ns, const int* done, const int* gact, const int* gstall, int* stall) {
    GS_LOOP(s, ns) {
        if (done[s]) continue;
        stall[s] = gact[s] > 0 && gstall[s] == gact[s];
    }
}
// gauss_newton.py:107-113; an energy change within the FP64 evaluation
// error of the two energies (N0 + N1) is no increase
// one block: returns (to thread 0) the number of units still searching
DV int ls_decide_block(int ns, int* acc, double* alpha, const double* E0, const double* E1, const double* N0,
                       const double* N1, double min_alpha, int* stall) {
    __shared__ int pending;
    if (threadIdx.x == 0) pending = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        if (acc[s]) continue;
        if (E1[s] < E0[s] || E1[s] - E0[s] <= N0[s] + N1[s]) acc[s] = 1;
        else if (alpha[s] * 0.5 < min_alpha) { acc[s] = 1; if (alpha[s] < ABD_LS_STALL_ALPHA) stall[s] = 1; }
        else { alpha[s] *= 0.5; atomicAdd(&pending, 1); }
    }
    __syncthreads();
    return pending;
}
__global__ void k_ls_decide(int ns, int* acc, double* alpha, const double* E0, const double* E1, const double* N0,
                            const double* N1, double min_alpha, int* stall, Counters* cnt) {
    int pending = ls_decide_block(ns, acc, alpha, E0, E1, N0, N1, min_alpha, stall);
    if (threadIdx.x == 0) cnt->ls_pending = pending;
}
// the same decision inside the line-search graph: counts the trial and
// keeps the graph's while-node running while units are pending, for at most
// LS_MAX_TRIALS trials (the host loop's cap)
constexpr int LS_MAX_TRIALS = 64;
__global__ void k_ls_decide_graph(int ns, int* acc, double* alpha, const double* E0, const double* E1, const double* N0,
                                  const double* N1, double min_alpha, int* stall, Counters* cnt,
                                  cudaGraphConditionalHandle loop) {
    int pending = ls_decide_block(ns, acc, alpha, E0, E1, N0, N1, min_alpha, stall);
    if (threadIdx.x == 0) {
        cnt->ls_pending = pending;
        int t = cnt->ls_trials + 1;
        cnt->ls_trials = t;
        cudaGraphSetConditional(loop, (pending > 0 && t < LS_MAX_TRIALS) ? 1u : 0u);
    }
}
__global__ void k_ls_graph_prep(Counters* cnt, int n_sw) { cnt->ls_trials = 0; cnt->ls_nsw = n_sw; }

// Line-search graphs (ls_graph): one per unit kind (scenes, contact
// groups), each a while-node whose body is one trial: apply the step
// length, the energies of the listed step, the decision.  Every pointer in
// the body is fixed for the handle except the swept list, which can be
// reallocated when it grows: the graph is rebuilt then.
struct LsGraph {
    cudaGraph_t g = nullptr; cudaGraphExec_t x = nullptr;
    const void* sw = nullptr;       // swept list the body was captured with
    int shapes[2] = {-2, -2};       // autotuner choice (list, body energy) it was captured with
    int body_launches = 0;          // kernels per trial
};
struct LsGraphState { LsGraph gr[2]; bool failed = false; };
void eng_lsgraph_free(Engine* E) {
    auto* S = reinterpret_cast<LsGraphState*>(E->ls_graph_state);
    if (!S) return;
    for (auto& g : S->gr) { if (g.x) cudaGraphExecDestroy(g.x); if (g.g) cudaGraphDestroy(g.g); }
    delete S;
    E->ls_graph_state = nullptr;
}
static int ls_graph_build(Engine* E, LsGraph& G, const LsUnits& U, const int* uacc, double* ualpha, int* ustall) {
    cudaStream_t s = E->stream;
    if (G.x) { cudaGraphExecDestroy(G.x); G.x = nullptr; }
    if (G.g) { cudaGraphDestroy(G.g); G.g = nullptr; }
    CUDA_TRY(cudaGraphCreate(&G.g, 0));
    cudaGraphConditionalHandle h;
    CUDA_TRY(cudaGraphConditionalHandleCreate(&h, G.g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CUDA_TRY(cudaGraphAddNode(&node, G.g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    const int l0 = E->launches;
    CUDA_TRY(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const AbdParams& P = E->P;
    E->capturing = true;
    k_apply<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->backup, E->du, ualpha, uacc, U.bunit, E->st);
    int rc = eng_energy_list(E, U, SD_E1, uacc, true);
    k_ls_decide_graph<<<1, 256, 0, s>>>(U.n, const_cast<int*>(uacc), ualpha, U.d + SD_E0 * U.n, U.d + SD_E1 * U.n,
                                        U.d + SD_E0N * U.n, U.d + SD_E1N * U.n, P.ls_min_alpha, ustall, E->dcnt, h);
    E->capturing = false;
    cudaGraph_t captured = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &captured);
    G.body_launches = E->launches - l0 + 2;
    E->launches = l0;
    if (rc) return rc;
    CUDA_TRY(ce);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaGraphInstantiate(&G.x, G.g, 0));
    G.sw = E->sw;
    G.shapes[0] = E->tune[TK_LIST_ENERGY].chosen; G.shapes[1] = E->tune[TK_BODY_ENERGY].chosen;
    return ABD_OK;
}
// the line search of one Newton iteration as one graph launch, not waited
// for: the trial count (dcnt->ls_trials) is read at the Newton bookkeeping's
// host sync that follows; *body_launches gets the kernels per trial.
// Returns ABD_OK with *ran = 0 when the graph cannot be used (the caller then
// runs the host loop).
static int ls_graph_run(Engine* E, bool groups, const LsUnits& U, const int* uacc, double* ualpha, int* ustall,
                        int* body_launches, int* ran) {
    *ran = 0;
    if (!E->ls_graph_state) E->ls_graph_state = new LsGraphState();
    auto* S = reinterpret_cast<LsGraphState*>(E->ls_graph_state);
    if (S->failed || E->timing) return ABD_OK;
    LsGraph& G = S->gr[groups ? 1 : 0];
    // captured again when the swept list moved or the autotuner settled
    // on a launch shape after the capture
    if (!G.x || G.sw != E->sw || G.shapes[0] != E->tune[TK_LIST_ENERGY].chosen ||
        G.shapes[1] != E->tune[TK_BODY_ENERGY].chosen) {
        if (ls_graph_build(E, G, U, uacc, ualpha, ustall)) {
            // graphs unavailable: keep the host loop for this handle
            S->failed = true;
            cudaGetLastError();
            E->err.clear();
            return ABD_OK;
        }
    }
    k_ls_graph_prep<<<1, 1, 0, E->stream>>>(E->dcnt, E->n_sw);
    CUDA_TRY(cudaGraphLaunch(G.x, E->stream));
    E->launches += 1;
    *body_launches = G.body_launches;
    *ran = 1;
    return ABD_OK;
}
// abd.py:693-699 bookkeeping: record (residual, alpha), stop on tol or cap
__global__ void k_newton_book(int ns, int* done, int* iter, const int* stall, const double* gg, const double* alpha,
                              double* prof_res, double* prof_alpha, int max_iter, double tol, Counters* cnt) {
    __shared__ int ndone, nan;
    if (threadIdx.x == 0) { ndone = 0; nan = 0; }
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        if (!done[s]) {
            int it = iter[s];
            double res = sqrt(gg[s]);
            if (!(res == res)) atomicAdd(&nan, 1);
            prof_res[(long)s * max_iter + it] = res;
            prof_alpha[(long)s * max_iter + it] = alpha[s];
            iter[s] = it + 1;
            if (res < tol || it + 1 >= max_iter || !(res == res) || stall[s]) done[s] = 1;
        }
        if (done[s]) atomicAdd(&ndone, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) { cnt->scenes_done = ndone; if (nan) cnt->nan_flag = 1; }
}
// abd.py:574-581
__global__ void k_forward(int nb, double* st, double dt) {
    GS_LOOP(b, nb) {
        double* s = st + ST_STRIDE * b;
#pragma unroll
        for (int k = 0; k < 3; k++) s[ST_NXT + ST_V + k] = (s[ST_NXT + ST_C + k] - s[ST_NOW + ST_C + k]) / dt;
#pragma unroll
        for (int k = 0; k < 9; k++) s[ST_NXT + ST_QD + k] = (s[ST_NXT + ST_Q + k] - s[ST_NOW + ST_Q + k]) / dt;
#pragma unroll
        for (int k = 0; k < 24; k++) s[ST_NOW + k] = s[ST_NXT + k];
    }
}
// warm start as a line-search direction: du = -ws on dynamic bodies
__global__ void k_ws_to_du(int nb, const double* __restrict__ ws, const double* __restrict__ mass, double* du) {
    GS_LOOP(i, 12L * nb) du[i] = mass[i / 12] > 0.0 ? -ws[i] : 0.0;
}
// accept a warm start that lowers the energy below that of now; after the
// last trial the scene starts from now (alpha 0, applied once more)
__global__ void k_ws_decide(int ns, int* acc, double* alpha, const double* E0, const double* E1, int last, Counters* cnt) {
    __shared__ int pending;
    if (threadIdx.x == 0) pending = 0;
    __syncthreads();
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        if (acc[s]) continue;
        if (E1[s] < E0[s]) acc[s] = 1;
        else { alpha[s] = last ? 0.0 : alpha[s] * 0.5; atomicAdd(&pending, 1); }
    }
    __syncthreads();
    if (threadIdx.x == 0) cnt->ls_pending = pending;
}
// inertial prediction as an increment from now: ws = q_tilde - q_now
__global__ void k_ws_inertial(int nb, const double* __restrict__ st, double dt, double g0, double g1, double g2,
                              double* ws) {
    GS_LOOP(i, 12L * nb) {
        long b = i / 12; int k = (int)(i % 12);
        const double* now = st + ST_STRIDE * b + ST_NOW;
        double gv = k == 0 ? g0 : (k == 1 ? g1 : g2);
        ws[i] = k < 3 ? dt * now[ST_V + k] + dt * dt * gv : dt * now[ST_QD + (k - 3)];
    }
}
int eng_grow_contacts(Engine* E, int need);

// algorithmic bytes of one detection: positions in, float copy out, per
// edge/triangle/point the box, key, value, count and offset traffic, the
// bucket table, and the pair list written
static double detect_bytes(Engine* E) {
    double b = E->nv * (24.0 + 24.0 + 16.0);
    b += E->ne * (8.0 + 32.0 + 4.0 + 4.0 * 4 + 8.0) + E->gee.H * 8.0;
    if (E->P.contact_pt) b += E->nt * (12.0 + 32.0 + 16.0) + E->nv * (32.0 + 8.0) + E->gpt.H * 8.0;
    return b;
}

int eng_step(Engine* E, int n_steps, AbdStepStats* stats) {
    cudaStream_t s = E->stream;
    const AbdParams& P = E->P;
    int ns = E->ns, rc;
    int* done = E->sci + SI_DONE * ns;
    int* iter = E->sci + SI_ITER * ns;
    int* acc = E->sci + SI_ACC * ns;
    int* stall = E->sci + SI_STALL * ns;
    double* alpha = E->scd + SD_ALPHA * ns;
    int mi = P.newton_max_iter;
    double* prof_res = E->prof_d;
    double* prof_alpha = E->prof_d + (long)ns * mi;
    E->prof_res.assign(ns, {}); E->prof_alpha.assign(ns, {}); E->prof_iters.assign(ns, {});
    AbdStepStats st; memset(&st, 0, sizeof st); st.min_toi = 1.0;
    int launches0 = E->launches;
    E->comp_band = E->comp_small = E->comp_large = E->krylov_fallbacks = 0;
    E->solver_capped = 0; E->host_syncs = 0;
    int ccd_capped = 0;
    CUDA_TRY(cudaEventRecord(E->ev0, s));
    for (int step = 0; step < n_steps; step++) {
        CUDA_TRY(cudaMemsetAsync(done, 0, sizeof(int) * ns, s));
        CUDA_TRY(cudaMemsetAsync(iter, 0, sizeof(int) * ns, s));
        CUDA_TRY(cudaMemsetAsync(stall, 0, sizeof(int) * ns, s));
        CUDA_TRY(cudaMemsetAsync(E->dcnt, 0, sizeof(Counters), s));
        if (P.warm_start == 2) {
            k_ws_inertial<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->st, P.dt, P.gravity[0], P.gravity[1], P.gravity[2], E->ws);
            E->launches++;
            E->has_ws = 1;
        } else if (P.warm_start == 3) {
            if ((rc = eng_learned_ws(E))) return rc;
            E->has_ws = 1;
        }
        if (E->has_ws) {
            // warm start: list and CCD along now -> now + ws, then move to
            // now + a ws, a = min(1, toi) halved until the energy is below
            // that of now (at most 7 halvings, else a = 0)
            if ((rc = eng_swept(E, E->ws, 1.0, done))) return rc;
            if (P.ccd && (rc = eng_ccd_list(E, scene_units(E), done))) return rc;
            k_ws_to_du<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->ws, E->mass, E->du);
            k_backup<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->st, E->backup);
            k_ls_init<<<grid_for(ns), 256, 0, s>>>(ns, done, acc, alpha, E->scd + SD_TOI * ns, P.ccd, stall, E->sw_scale);
            E->launches += 3;
            if ((rc = eng_energy_list(E, scene_units(E), SD_E0, done))) return rc;
            for (int trial = 0;; trial++) {
                k_apply<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->backup, E->du, alpha, acc, E->bscene, E->st);
                E->launches++;
                if (trial == 8) break;
                if ((rc = eng_energy_list(E, scene_units(E), SD_E1, acc))) return rc;
                k_ws_decide<<<1, 256, 0, s>>>(ns, acc, alpha, E->scd + SD_E0 * ns, E->scd + SD_E1 * ns, trial == 7, E->dcnt);
                E->launches++;
                if ((rc = eng_sync_counters(E))) return rc;
                if (E->hcnt->ls_pending == 0) break;
            }
            E->has_ws = 0;
        }
        bool detected_ahead = false;      // this iteration's list filter ran before the last sync
        E->keys_ahead = false;
        E->sw_inject_done = false;
        for (int it = 0; it < mi; it++) {
            // contact.py:270-279 detection on the current iterate: filter the
            // swept list of the step that led here, or detect from scratch
            for (bool ahead = detected_ahead;; ahead = false) {
                if (!ahead) {
                    int ph = phase_begin(E, PH_DETECT);
                    rc = E->sw_valid ? eng_detect_list(E) : (eng_use_bp(E) ? eng_detect_bp(E, P.cand_dist) : eng_detect(E, P.cand_dist));
                    phase_end(E, ph, detect_bytes(E));
                    if (rc) return rc;
                    if ((rc = eng_sync_counters(E))) return rc;
                }
                if (!E->hcnt->overflow) break;
                if ((rc = eng_grow_contacts(E, E->hcnt->n_total))) return rc;
            }
            detected_ahead = false;
            st.n_pairs = E->hcnt->n_total;
            // abd.py:682-688 assembly
            { int ph = phase_begin(E, PH_ASSEMBLE); rc = eng_assemble(E); phase_end(E, ph, 0); if (rc) return rc; }
            // abd.py:690 / :631-658 solve
            int li = 0;
            { int ph = phase_begin(E, PH_SOLVE); rc = eng_solve(E, &li, it == 0); phase_end(E, ph, 0); if (rc) return rc; }
            st.lin_iters += li;
            st.n_active = E->hcnt->n_active;
            // candidates along x -> x - J du, shared by CCD, every energy
            // of the line search and the next detection
            {
                int ph = phase_begin(E, PH_SWEPT);
                rc = eng_swept(E, E->du, -1.0, done);
                // positions, rest positions, increments per vertex; topology; the listed pairs
                phase_end(E, ph, E->nv * (24.0 + 24.0 + 4.0) + E->nb * 96.0 + E->ne * 8.0 + E->nt * 12.0 + E->n_sw * 24.0);
                if (rc) return rc;
            }
            // the line search runs per scene, or per contact group of the
            // listed step (ls_groups): each unit has its own CCD bound,
            // energies, step length and back-off
            const bool groups = P.ls_groups && E->bd_ok;
            // eng_groups allocates the group slots on first use: take the
            // unit view only after it
            if (groups && (rc = eng_groups(E, done))) return rc;
            if (groups && !(E->grp && E->gscd && E->gsci)) return E->fail(ABD_ERR_CUDA, "contact groups not allocated");
            LsUnits U = groups ? group_units(E) : scene_units(E);
            const int* udone = U.i + SI_DONE * U.n;
            int* uacc = U.i + SI_ACC * U.n;
            int* ustall = U.i + SI_STALL * U.n;
            double* ualpha = U.d + SD_ALPHA * U.n;
            if (!groups) udone = done;
            if (P.ccd) {
                int ph = phase_begin(E, PH_CCD); rc = eng_ccd_list(E, U, udone); phase_end(E, ph, 0);
                if (rc) return rc;
            }
            // gauss_newton.py:98-115 line search
            { int ph = phase_begin(E, PH_ENERGY); rc = eng_energy_list(E, U, SD_E0, udone); phase_end(E, ph, 0); if (rc) return rc; }
            k_backup<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->st, E->backup);
            E->launches++;
            k_ls_init<<<grid_for(U.n), 256, 0, s>>>(U.n, udone, uacc, ualpha, U.d + SD_TOI * U.n, P.ccd, ustall,
                                                     E->sw_scale);
            E->launches++;
            int ph_tr = phase_begin(E, PH_TRIALS);
            int graph_ran = 0, graph_body = 0;
            if (P.ls_graph) {
                if ((rc = ls_graph_run(E, groups, U, uacc, ualpha, ustall, &graph_body, &graph_ran))) return rc;
                if (graph_ran) st.ls_graph_launches++;
            }
            for (int trial = 0; trial < LS_MAX_TRIALS && !graph_ran; trial++) {
                k_apply<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->backup, E->du, ualpha, uacc, U.bunit, E->st);
                { int ph = phase_begin(E, PH_ENERGY); rc = eng_energy_list(E, U, SD_E1, uacc); phase_end(E, ph, 0); if (rc) return rc; }
                k_ls_decide<<<1, 256, 0, s>>>(U.n, uacc, ualpha, U.d + SD_E0 * U.n, U.d + SD_E1 * U.n, U.d + SD_E0N * U.n,
                                              U.d + SD_E1N * U.n, P.ls_min_alpha, ustall, E->dcnt);
                E->launches += 2;
                st.ls_trials++;
                if ((rc = eng_sync_counters(E))) return rc;
                if (E->hcnt->grp_fail) return E->fail(ABD_ERR_CUDA, "contact groups: union-find did not settle");
                if (E->hcnt->ls_pending == 0) break;
            }
            phase_end(E, ph_tr, 0);
            if (groups) {
                int* gact = E->sci + SI_GACT * ns; int* gstall = E->sci + SI_GSTALL * ns;
                double* stoi = E->scd + SD_TOI * ns;
                k_grp_scene_init<<<grid_for(ns), 256, 0, s>>>(ns, done, alpha, stoi, gact, gstall);
                k_grp_to_scenes<<<grid_for(E->nb), 256, 0, s>>>(E->nb, E->bscene, udone, ualpha, U.d + SD_TOI * U.n, ustall,
                                                                P.ccd, alpha, stoi, gact, gstall);
                k_grp_scene_stall<<<grid_for(ns), 256, 0, s>>>(ns, done, gact, gstall, stall);
                E->launches += 3;
            }
            k_newton_book<<<1, 256, 0, s>>>(ns, done, iter, stall, E->scd + SD_GG * ns, alpha, prof_res, prof_alpha, mi,
                                            P.newton_tol, E->dcnt);
            E->launches++;
            // the next iteration's list filter (no host sync inside) is queued
            // before this sync, which then also brings back its counts; the
            // filter writes only the detection counters, not the bookkeeping's
            const bool ahead = E->sw_valid && it + 1 < mi;
            if (ahead) {
                int ph = phase_begin(E, PH_DETECT);
                rc = eng_detect_list(E);
                phase_end(E, ph, detect_bytes(E));
                if (rc) return rc;
                // and the next assembly's block keys, so that this sync
                // brings them to the direct solver too
                if ((rc = eng_assemble_keys_ahead(E))) return rc;
            }
            if ((rc = eng_sync_counters(E))) return rc;
            eng_keys_ahead_synced(E);
            detected_ahead = ahead;
            if (graph_ran) {
                // the graph's line search ended before the bookkeeping ran
                st.ls_trials += E->hcnt->ls_trials;
                E->launches += graph_body * E->hcnt->ls_trials;
                if (E->hcnt->grp_fail) return E->fail(ABD_ERR_CUDA, "contact groups: union-find did not settle");
            }
            if (E->hcnt->nan_flag) return E->fail(ABD_ERR_NAN, "non-finite gradient norm");
            if (E->hcnt->scenes_done == ns) break;
        }
        E->keys_ahead = false;           // keys built for an iteration that did not run
        // counters of this step (the last bookkeeping sync brought them back)
        st.du_guard_hits += E->hcnt->du_guard;
        ccd_capped |= E->hcnt->ccd_capped;
        if (P.ccd) {
            double* toi = E->scd + SD_TOI * ns;
            CUDA_TRY(cudaMemcpyAsync(E->hscd, toi, sizeof(double) * ns, cudaMemcpyDeviceToHost, s));
        }
        k_forward<<<grid_for(E->nb), 256, 0, s>>>(E->nb, E->st, P.dt);
        E->launches++;
        // profile
        std::vector<double> hr((size_t)ns * mi), ha((size_t)ns * mi);
        std::vector<int> hi(ns);
        CUDA_TRY(cudaMemcpyAsync(hr.data(), prof_res, sizeof(double) * ns * mi, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(ha.data(), prof_alpha, sizeof(double) * ns * mi, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaMemcpyAsync(hi.data(), iter, sizeof(int) * ns, cudaMemcpyDeviceToHost, s));
        CUDA_TRY(eng_stream_sync(E));
        for (int sc = 0; sc < ns; sc++) {
            int n = hi[sc];
            for (int k = 0; k < n; k++) {
                E->prof_res[sc].push_back(hr[(size_t)sc * mi + k]);
                E->prof_alpha[sc].push_back(ha[(size_t)sc * mi + k]);
            }
            E->prof_iters[sc].push_back(n);
            st.newton_iters += n;
            if (n > st.max_newton_iters) st.max_newton_iters = n;
            double last = n ? hr[(size_t)sc * mi + n - 1] : 0.0;
            if (!(last < P.newton_tol)) st.unconverged++;
            if (last > st.last_residual) st.last_residual = last;
            if (P.ccd && E->hscd[sc] < st.min_toi) st.min_toi = E->hscd[sc];
        }
        st.steps++;
    }
    CUDA_TRY(cudaEventRecord(E->ev1, s));
    CUDA_TRY(cudaEventSynchronize(E->ev1));
    phase_collect(E);
    float ms = 0;
    cudaEventElapsedTime(&ms, E->ev0, E->ev1);
    st.gpu_ms = ms;
    st.kernel_launches = E->launches - launches0;
    st.comp_band = E->comp_band; st.comp_small = E->comp_small; st.comp_large = E->comp_large;
    st.krylov_fallbacks = E->krylov_fallbacks;
    st.solver_capped = E->solver_capped;
    st.host_syncs = E->host_syncs + 1;      // + the closing event synchronisation
    if (stats) *stats = st;
    if (ccd_capped) return E->fail(ABD_ERR_CCD_CAP, "CCD iteration cap reached (step clamped conservatively)");
    if (E->solver_capped)
        return E->fail(ABD_ERR_SOLVER_CAP, "Krylov iteration cap reached above tolerance (step taken with that increment)");
    return ABD_OK;
}
