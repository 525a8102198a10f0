/*
 * abd_b200.h — C ABI of libabd_b200.so, the B200 (sm_100a) affine-body-dynamics
 * Newton step with IPC-style barrier contact.
 *
 * The reference exposes this path as the Python class `NewtonAbd`
 * (abd.py:583-757 of Luke-Skycrawler/colb) driven by `step()` from the viewer
 * (viewer.py:44-47).  Every entry point below names the reference interface
 * it replaces.  There is no plugin registry in the reference: a caller picks
 * the solver by constructing the class (links.py:17-22).
 *
 * Conventions
 *  - Plain C types only.  All arrays are host pointers unless stated.
 *  - Every call returns an int status (ABD_OK == 0, negative on error).  No
 *    exception crosses the ABI; abd_last_error() gives the message.
 *  - One handle per host thread.  All device work runs on the handle's own
 *    CUDA stream; calls return after that stream is synchronised.
 *  - Body state layout is the reference's BDFAffine (BDF1.py:11-14 with
 *    AffineState from quat_util.py:40-47): 48 doubles per body,
 *        now.c[3] now.q[9] now.v[3] now.qdot[9]  nxt.c[3] nxt.q[9] nxt.v[3] nxt.qdot[9]
 *    q is row-major with rows = affine DoFs (q = A^T), so a vertex maps as
 *    x = q^T xbar + c (abd_simple.py:26-35).
 *  - Per-body DoF vector (gradient, Newton increment): 12 doubles
 *    [c(3), q row0(3), q row1(3), q row2(3)], body-major (abd.py:595, :780-785).
 */
#ifndef ABD_B200_H
#define ABD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ABD_ABI_VERSION 2

/* ---- status codes ---------------------------------------------------- */
#define ABD_LS_STALL_ALPHA 1e-6

#define ABD_OK                   0
#define ABD_ERR_INVALID_ARG     -1
#define ABD_ERR_CUDA            -2
#define ABD_ERR_CONTACT_OVERFLOW -3  /* more candidate pairs than capacity (reference wraps silently, contact.py:137) */
#define ABD_ERR_NAN             -4  /* non-finite energy / gradient / state */
#define ABD_ERR_SOLVER_CAP      -5  /* Krylov iteration cap hit without reaching tolerance (non-fatal, reported) */
#define ABD_ERR_NEWTON_CAP      -6  /* Newton iteration cap hit (non-fatal, reported; abd.py:699 stops silently) */
#define ABD_ERR_CCD_CAP         -7  /* CCD iteration cap hit: step clamped conservatively */
#define ABD_ERR_NO_DEVICE       -8
#define ABD_ERR_NOT_BUILT       -9

/* ---- enums ----------------------------------------------------------- */
/* barrier.py:6-65 — the three barriers of barrier.py, all in x = d^2 */
#define ABD_BARRIER_CUBIC      0   /* b = -(x-xh)^3          (barrier.py:47-65, the active one) */
#define ABD_BARRIER_QUADRATIC  1   /* b = (x-xh)^2           (barrier.py:23-44) */
#define ABD_BARRIER_LOG        2   /* b = -(x-xh)^2 ln(x/xh)/xh^2 (barrier.py:6-21, derivatives as written) */

#define ABD_HESS_REFERENCE     0   /* abd.py:247-251: PSD-project the EE distance Hessian only, PE raw, PP drops B'H */
#define ABD_HESS_PROJECTED     1   /* project each contact's whole barrier Hessian and each body's ortho Hessian to PSD */

#define ABD_SOLVER_BICGSTAB    0   /* abd.py:636 uses bicgstab; here block-Jacobi preconditioned */
#define ABD_SOLVER_PCG         1   /* block-Jacobi PCG */
#define ABD_SOLVER_DIRECT      2   /* dense factorization per scene (the reference's solver_config="direct",
                                      abd.py:637-654): Cholesky for projected Hessians, else LU */
#define ABD_SOLVER_AUTO        3   /* DIRECT while the dense matrices fit (<= 64 scenes, <= 4 GiB), else PCG
                                      (projected Hessian) or BiCGSTAB (reference Hessian) */

#define ABD_PREC_FP64          0
#define ABD_PREC_MIXED         1   /* FP32 block matrix + Krylov vectors; FP64 distances, CCD, energy, residual */

/* contact kinds stored in the sorted contact list */
#define ABD_CONTACT_EE         0   /* edge-edge (contact.py:143-169) */
#define ABD_CONTACT_PT         1   /* point-triangle (no reference counterpart) */
#define ABD_CONTACT_PG         2   /* point-half-space (ground / box wall; no reference counterpart) */

/* ---- solver parameters (one set per handle, shared by all scenes) ---- */
typedef struct AbdParams {
    double dt;              /* links.py:16 (8e-3) */
    double gravity[3];      /* abd.py:28, :164-166 ((0,-10,0)) */
    double kappa;           /* contact stiffness, abd.py:30 (4e8) */
    double k_ortho;         /* orthogonality stiffness, ortho.py:5 (1e5) */
    double dhat;            /* barrier activation distance, barrier.py:4-5 (0.095) */
    double cand_dist;       /* EE candidate filter, contact.py:168 ((thickness+buffer)*2 = 0.19) */
    int32_t barrier;        /* ABD_BARRIER_* */
    int32_t hess_mode;      /* ABD_HESS_* */
    int32_t contact_ee;     /* enable edge-edge contacts */
    int32_t contact_pt;     /* enable point-triangle contacts */
    int32_t self_contact;   /* allow pairs within one body (reference: yes, contact.py:160) */
    int32_t ee_f32;         /* 1: EE filter/classification/barrier distance in FP32 exactly as
                               contact.py:166 / abd.py:190; 0: FP64 closest points */
    int32_t linear_solver;  /* ABD_SOLVER_* */
    int32_t lin_max_iter;   /* Krylov iteration cap per Newton iteration */
    double lin_tol;         /* relative residual tolerance, abd.py:636 (1e-5) */
    double newton_tol;      /* ||gradient||_2 tolerance, abd.py:699 (1e-5) */
    int32_t newton_max_iter;/* abd.py:679 (16) */
    int32_t ccd;            /* 1: additive-CCD time of impact bounds the line search */
    double ccd_scale;       /* ACCD conservative rescaling s in (0,1) (0.1 typical) */
    double ls_min_alpha;    /* gauss_newton.py:110: stop halving when alpha*0.5 < this (1e-2).
                             * A search that gives up below ABD_LS_STALL_ALPHA
                             * ends the scene's Newton loop (stalled: the next
                             * iteration would start from the same state). */
    int32_t precision;      /* ABD_PREC_* */
    int32_t contact_capacity;/* max candidate pairs per detection (reference: 10000, contact.py:8) */
    double pinned_diag;     /* diagonal of pinned bodies' blocks, abd.py:146 (100) */
    int32_t warm_start;     /* 0: start Newton from nxt = now (abd.py: history.nxt == now after
                               forward_states); 1: from now + the increment given to
                               abd_set_warm_start; 2: from the inertial prediction
                               (c + dt v + dt^2 g, q + dt qdot); 3: from the learned network
                               (abd_set_mlp); 1, 2 and 3 are clipped by CCD */
    int32_t broadphase;     /* 0 auto, 1 hashed grid over primitives, 2 body pairs then primitives
                               (needs contiguous per-body vertex/edge/triangle ranges) */
    int32_t autotune;       /* 1: time the launch-shape candidates of the tunable kernels during
                               the first Newton iterations of the handle and keep the fastest
                               (abd_get_autotune); 0: fixed launch shapes */
    int32_t ls_groups;      /* 0: one step length per scene, as gauss_newton.py:98-115 does for
                               its one scene; 1: one step length per contact group, the
                               connected components of the bodies whose swept, padded boxes
                               over the Newton step overlap (no contact can form between
                               groups along the step, so the energy is a sum of independent
                               group energies and each group takes its own CCD bound and
                               back-off).  Convergence stays per scene. */
    int32_t ls_graph;       /* 1: run the line-search trials of each Newton iteration as one CUDA
                               graph whose while-node repeats apply / energy / decide on the
                               device until every unit has accepted (at most 64 trials), with one
                               host round trip per search instead of one per trial; 0: the host
                               loop.  Same kernels and decisions either way. */
    int32_t ccd_max_iter;   /* iteration cap of one additive-CCD query (0: ABD_CCD_MAX_ITER); a
                               query that reaches it returns the time reached so far (a
                               conservative bound) and the step reports ABD_ERR_CCD_CAP */
    int32_t test_inject;    /* host-side failure injection for tests, 0 in production:
                               ABD_INJECT_DU_NONFINITE overwrites the first Newton increment of
                               every step of scene 0 with NaN before the mixed-precision guard
                               runs (the guard must replace it by the block-Jacobi direction);
                               ABD_INJECT_SWEPT_FULL makes the first swept candidate list of every
                               step report that it does not fit (the list must then be built for a
                               shorter step, and the step length capped to it) */
    int32_t reserved[1];
} AbdParams;

#define ABD_CCD_MAX_ITER 100000
#define ABD_INJECT_DU_NONFINITE 1
#define ABD_INJECT_SWEPT_FULL 2

/* ---- one scene: concatenated affine bodies (geometry.py:22-73) ------- */
typedef struct AbdSceneDesc {
    int32_t n_bodies;
    int32_t n_verts;
    int32_t n_edges;
    int32_t n_tris;
    const double*  xbar;       /* n_verts*3 rest positions in the body frame (Soup.xcs) */
    const int32_t* vert_body;  /* n_verts body index, 0-based within this scene (Soup.body) */
    const int32_t* edges;      /* n_edges*2 vertex indices (Soup.edges) */
    const int32_t* tris;       /* n_tris*3 vertex indices (Soup.triangles) */
    const double*  mass;       /* n_bodies, m<=0 pins the body (abd.py:115, rbd_simple.py:42-48) */
    const double*  inertia_J;  /* n_bodies scalar J of M = diag(m,J,J,J) (x) I3 (abd.py:77-85) */
    const double*  state;      /* n_bodies*48 initial BDFAffine (abd_simple.py:37-49) */
    int32_t n_planes;          /* static half-spaces n.x >= offset (ground, box walls) */
    const double*  planes;     /* n_planes*4 : nx ny nz offset (n unit) */
} AbdSceneDesc;

/* ---- per-step statistics -------------------------------------------- */
typedef struct AbdStepStats {
    int32_t steps;             /* steps taken by this call */
    int32_t newton_iters;      /* sum over steps and scenes of Newton iterations */
    int32_t max_newton_iters;  /* max over steps/scenes */
    int32_t lin_iters;         /* total Krylov iterations */
    int32_t n_pairs;           /* candidate pairs at the last detection */
    int32_t n_active;          /* active (d < dhat) contacts at the last assembly */
    int32_t unconverged;       /* (step,scene) pairs that hit the Newton cap */
    int32_t ls_trials;         /* total line-search energy evaluations */
    double  last_residual;     /* max over scenes of the last Newton iteration's ||g|| */
    double  min_toi;           /* smallest CCD time of impact seen (1 if none) */
    double  gpu_ms;            /* device time of the call (CUDA events) */
    int32_t kernel_launches;   /* kernels launched by the call */
    int32_t comp_band;         /* direct solver: components solved by the band kernel, */
    int32_t comp_small;        /*   by the shared-memory dense kernel, */
    int32_t comp_large;        /*   by cuSOLVER (summed over iterations), */
    int32_t krylov_fallbacks;  /*   and solves handed to the Krylov solver */
    int32_t ls_graph_launches; /* line searches run as one CUDA graph launch (ls_graph) */
    int32_t solver_capped;     /* Krylov solves that stopped at lin_max_iter above lin_tol
                                  (abd_step then returns ABD_ERR_SOLVER_CAP, non-fatal) */
    int32_t du_guard_hits;     /* mixed precision: scene solves whose increment had a non-finite
                                  entry and were replaced by the block-Jacobi direction */
    int32_t host_syncs;        /* host round trips (stream synchronisations) of the call */
    int32_t reserved_stats;
} AbdStepStats;

typedef struct AbdHandle AbdHandle;

/* Fills p with the reference's constants (abd.py:27-30, barrier.py:4-5,
 * contact.py:7-9, ortho.py:5, links.py:16, gauss_newton.py:110). */
void abd_default_params(AbdParams* p);

/* Replaces NewtonAbd.__init__ (abd.py:584-599) together with
 * ContactSolverBase.__init__ (contact.py:204-241) and AbdComplex/JSONComplex
 * scene set-up (abd_simple.py:53-69): copies the scene to the device and
 * allocates every buffer the step needs.  n_scenes > 1 builds a batch of
 * independent scenes stepped together (no reference counterpart). */
int abd_create(const AbdParams* params, const AbdSceneDesc* scenes, int32_t n_scenes,
               int32_t device, AbdHandle** out);

/* Frees all device memory of the handle. */
int abd_destroy(AbdHandle* h);

/* Size queries. */
int abd_get_sizes(AbdHandle* h, int32_t* n_bodies, int32_t* n_verts, int32_t* n_edges,
                  int32_t* n_tris, int32_t* n_scenes);

/* Replaces assigning NewtonAbd.history (abd_simple.py:14, :64-69). */
int abd_set_state(AbdHandle* h, const double* bdf_affine, int32_t n_bodies);
/* Replaces NewtonAbd.history.numpy() (BDFAffine array, 48 doubles/body). */
int abd_get_state(AbdHandle* h, double* bdf_affine_out);

/* Replaces NewtonAbd.step() (abd.py:674-702): n_steps full Newton steps with
 * collision detection, assembly, linear solve, line search and
 * forward_states.  stats may be NULL. */
int abd_step(AbdHandle* h, int32_t n_steps, AbdStepStats* stats);

/* Per-(step, Newton-iteration) profile of the last abd_step call for scene
 * `scene`: residual ||g|| and accepted alpha, like Profiller.convergence /
 * .alphas (abd.py:695-696, utils/data_collector.py:4-55).  Writes at most
 * cap entries; *n gets the number of iterations recorded. */
int abd_get_profile(AbdHandle* h, int32_t scene, double* residuals, double* alphas,
                    int32_t* iters_per_step, int32_t cap, int32_t* n);

/* Replaces compute_V(ret=True) (abd_simple.py:71-78): vertex positions of
 * the nxt state, n_verts*3 doubles. */
int abd_get_vertices(AbdHandle* h, double* x_out);

/* Runs detection on the current nxt state and returns the sorted candidate
 * list (replaces ContactSolverBase.detect_collision, contact.py:270-279).
 * Each entry is 4 vertex indices (XConstraint.a1a2b1b2, contact.py:46-51)
 * for EE; for PT (p, t0, t1, t2); for PG (p, plane, -1, -1).  kinds_out
 * (may be NULL) gets ABD_CONTACT_* per entry.  Order: kind, then first
 * primitive index, then second. */
int abd_get_pairs(AbdHandle* h, int32_t* out4, int32_t* kinds_out, int32_t cap, int32_t* n);

/* Replaces get_contact_points (abd.py:748-766): midpoint and distance per
 * candidate pair (EE closest points), cap entries. */
int abd_get_contact_points(AbdHandle* h, double* points_out, double* dists_out,
                           int32_t cap, int32_t* n);

/* Total incremental potential of the nxt state per scene (replaces
 * NewtonAbd.compute_g, abd.py:725-735). */
int abd_energy(AbdHandle* h, double* energy_per_scene);

/* Assembles gradient and Hessian at the nxt state (abd.py:686-688 with the
 * triplet overlap of the reference fixed) and copies them out: grad is
 * n_bodies*12; hess_dense (may be NULL) is (12 n_bodies)^2 row-major and
 * is only allowed for n_bodies <= 512. */
int abd_assemble(AbdHandle* h, double* grad, double* hess_dense);

/* Newton increment du = H^-1 g of the current assembly (abd.py:631-658);
 * du is n_bodies*12.  *iters gets the Krylov iteration count. */
int abd_solve(AbdHandle* h, double* du, int32_t* iters);

/* Warm start: per-body 12-DoF increment added to nxt = now at the start of
 * the next step (no reference counterpart; used by the learned warm start).
 * Values are in DoF order [c, q0, q1, q2]; the increment is clipped by CCD. */
int abd_set_warm_start(AbdHandle* h, const float* dq12, int32_t n_bodies);

/* Learned warm start (no reference counterpart).
 *
 * Features: 48 floats per body at the current state, in the body frame
 * (a direction d maps to q d, q the body's 3x3 DoF rows):
 *   [0:3]   q (v + dt g)          [3:12] q qdot^T (row-major)
 *   [12:15] q g / |g|             [15]   log(1 + number of nearby pairs)
 *   [16 + 4k] distance / radius, [17 + 4k : 20 + 4k] unit direction from the
 *   other primitive, for the 8 nearest pairs (missing ones: 1, 0, 0, 0);
 *   pairs are those within radius = ABD_FEAT_RADIUS_DHAT * dhat; pinned
 *   bodies get zeros.
 * Network: 48 -> 256 -> 256 -> 256 -> 12, GELU, BF16 weights and
 * activations, FP32 accumulation.  Parameters are ABD_MLP_NPARAM floats:
 * W1[256][48] b1[256] W2[256][256] b2[256] W3[256][256] b3[256] W4[12][256]
 * b4[12]; normalisation is ABD_MLP_NNORM floats: x mean[48], x std[48],
 * y mean[12], y std[12].  The output y (12) is the body-frame correction
 * to the inertial increment, per unit time:
 *   dc = dt v + dt^2 g + dt q^-1 y[0:3]
 *   dq = dt qdot + dt (q^-1 Y)^T, Y = y[3:12] as a row-major 3x3. */
#define ABD_FEAT_RADIUS_DHAT 50.0
#define ABD_MLP_IN 48
#define ABD_MLP_HIDDEN 256
#define ABD_MLP_OUT 12
#define ABD_MLP_NPARAM 147212
#define ABD_MLP_NNORM 120
int abd_get_features(AbdHandle* h, float* feat_out, int32_t n_bodies);

/* Sets the network used by warm_start 3 (copied and packed to BF16). */
int abd_set_mlp(AbdHandle* h, const float* params, const float* norm);

/* The network on n host rows of raw features -> n x 12 outputs (y above);
 * runs the same tensor-core kernel as warm_start 3. */
int abd_mlp_forward(AbdHandle* h, const float* x, int32_t n, float* y);

/* Trainer of the network on one GPU: FP32 master weights, Adam (0.9, 0.999,
 * 1e-8), mean-squared error on normalised targets, forward with BF16-rounded
 * weights and activations like inference. */
typedef struct AbdTrainer AbdTrainer;
int abd_trainer_create(int32_t device, const float* params, AbdTrainer** out);
int abd_trainer_destroy(AbdTrainer* t);
const char* abd_trainer_last_error(AbdTrainer* t);
/* x: n x 48 normalised features, y: n x 12 normalised targets (copied). */
int abd_trainer_set_data(AbdTrainer* t, const float* x, const float* y, int32_t n);
/* One pass over order[0..n) in mini-batches, one Adam step each. */
int abd_trainer_epoch(AbdTrainer* t, const int32_t* order, int32_t n, int32_t batch, float lr, float* mean_loss);
/* Loss and gradient (ABD_MLP_NPARAM floats) on the given rows, no update. */
int abd_trainer_grad(AbdTrainer* t, const float* x, const float* y, int32_t n, float* grad, float* loss);
int abd_trainer_params(AbdTrainer* t, float* params);

/* Launch shapes chosen by the autotuner (no reference counterpart): [0]
 * threads per block and [1] contacts per block of the contact assembly (one
 * warp per contact, or one block of 64 / 128 threads per contact), [2]
 * threads per block of the listed-pair energy, [3] of the body energy; -1
 * while still timing candidates.  *n gets the number of entries (4). */
int abd_get_autotune(AbdHandle* h, int32_t* shapes, int32_t cap, int32_t* n);

/* Number of edge-triangle intersections between different bodies at the
 * nxt state (FP64 exact predicate); 0 means intersection-free. */
int abd_count_intersections(AbdHandle* h, int32_t* count);

/* Device-side phase timers (no reference counterpart; the reference wraps
 * step() in wp.ScopedTimer, abd.py:676).  When on, every phase launch is
 * bracketed by CUDA events on the handle's stream and summed per phase:
 *   0 detect (pair list)        1 assemble (all of it)    2 solve
 *   3 line-search energy        4 CCD                     5 other
 *   6 contact-energy kernels    7 SpMV kernels            8 assembly: keys, sort, blocks
 *   9 assembly: bodies          10 assembly: contacts     11 assembly: block inverse
 *   12 dense factor + solve     13 swept candidate list   14 contact-energy list kernel
 *   15 line-search trials (apply + energy + decision)
 *   16 banded block-Cholesky kernel of the direct solver
 * abd_get_timing writes ms[17], launches[17] and the algorithmic bytes[17]
 * those phases moved (documented at each kernel); reset clears them. */
#define ABD_NUM_PHASES 17
int abd_set_timing(AbdHandle* h, int32_t on, int32_t reset);
int abd_get_timing(AbdHandle* h, double* ms, int64_t* launches, double* bytes);

/* Edge-edge candidate pairs that allocate no device memory.  This entry
 * point has no counterpart in the reference; it exists for callers that
 * cannot call cudaMalloc when they need the pairs (a host that manages all
 * device memory through its own pool, a real-time loop that forbids
 * allocation after start-up, a plugin whose host owns the CUDA context).
 * It computes the same sorted set as abd_get_pairs for an EE-only scene
 * under the reference predicate (contact.py:158-168: i < j, no shared
 * vertex, float32 segment distance < cand_dist), written as vertex
 * quadruples (a1, a2, b1, b2), but takes DEVICE pointers: x_dev (n_verts*3
 * doubles), edges_dev (n_edges*2 ints), pairs_dev (cap*4 ints) and
 * n_pairs_dev (one int).  All scratch lives in static device arrays of the
 * library (about 8.5 MiB per GPU, held until exit) sized for
 * ABD_STATIC_MAX_EDGES edges; larger inputs are rejected with
 * ABD_ERR_INVALID_ARG.  The first call on each device looks those arrays up
 * and caches their addresses (make it before any stream capture; after a
 * cudaDeviceReset of that device, do not call this entry point on it again
 * in the same process).  Calls share the arrays: calls whose GPU work
 * overlaps race.  Work runs on `stream` (a cudaStream_t, NULL for the
 * legacy default stream) and the call waits for that stream before it
 * returns.  ABD_ERR_CONTACT_OVERFLOW if more than cap pairs exist:
 * *n_pairs_dev holds the full count, nothing is written at or beyond row
 * cap, and which pairs the first cap rows hold is unspecified.
 * Errors: abd_last_error(NULL). */
#define ABD_STATIC_MAX_EDGES (1 << 16)
int abd_ee_pairs_static(const double* x_dev, const int32_t* edges_dev, int32_t n_verts, int32_t n_edges,
                        double cand_dist, int32_t* pairs_dev, int32_t cap, int32_t* n_pairs_dev, void* stream);

/* Message of the last failing call on this handle (or a global one for NULL). */
const char* abd_last_error(AbdHandle* h);

int abd_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ABD_B200_H */
