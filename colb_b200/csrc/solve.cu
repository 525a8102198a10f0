// solve.cu — block-Jacobi preconditioned Krylov solves on the 12x12 block
// system, one independent solve per scene (abd.py:631-658; the reference
// calls Warp's unpreconditioned bicgstab with tol 1e-5 on the whole BSR).
//
// Every scene runs its own CG / BiCGSTAB recurrences: dot products are
// reduced per scene, and each kernel recomputes the scene's scalars from
// those sums, so an iteration needs no host round trip.  Converged scenes
// stop updating.  The host checks the number of active scenes every
// CHECK_EVERY iterations.
//
// Thread mapping: 16 lanes per body row (lanes 0..11 own one DoF each), so
// a body's 12 entries live in one half-warp and the 12x12 preconditioner
// product uses width-16 shuffles.  Block values are column-major inside a
// block, so at fixed column the 12 lanes read 12 consecutive values.
#include "engine.cuh"

#define CHECK_EVERY 8

// resolved Krylov method for one solve
struct KrylovKind { KrylovKind(Engine* E, int k) { E->krylov_kind = k; } };
#define HALF 16

// kv slots
enum { KV_X = 0, KV_R, KV_Z, KV_P0, KV_P1, KV_V, KV_RH, KV_S, KV_T, KV_Y };

// per-scene dot ring: slot q of quantity K at scd[(SD_Kx + q) * ns + s]
#define RING(E_, K, q) ((E_)->scd + ((K) + (q)) * (E_)->ns)

template <class T>
struct KrylovArgs {
    int nb, ns;
    const int* row_ptr; const int* bcol; const T* vals; const T* dinv;
    const int* bscene; const int* ndone;   // Newton-done flag per scene
    const int* kdone;                      // Krylov breakdown flag per scene
    double tol2; int maxit;
    const double* bb;                      // ||b||^2 per scene
};

DV bool scene_active(const double* rr, const double* bb, double tol2, int s) {
    return rr[s] > tol2 * bb[s];
}

// y_l = sum_blocks V[c][l] * x[col][c]
template <class T>
DV double row_mv(const KrylovArgs<T>& A, int b, int l, const T* x) {
    double acc = 0;
    for (int k = A.row_ptr[b]; k < A.row_ptr[b+1]; k++) {
        const T* V = A.vals + (long)k * 144 + l;
        const T* xc = x + 12L * A.bcol[k];
#pragma unroll
        for (int c = 0; c < 12; c++) acc += (double)V[c * 12] * (double)xc[c];
    }
    return acc;
}
// z_l = sum_c Dinv[c][l] * r_c, r_c held by lane c of the half-warp
template <class T>
DV double precond_lane(const T* D, int l, double r_own, unsigned mask) {
    double acc = 0;
#pragma unroll
    for (int c = 0; c < 12; c++) {
        double rc = __shfl_sync(mask, r_own, c, HALF);
        if (l < 12) acc += (double)D[c * 12 + l] * rc;
    }
    return acc;
}

#define HALF_LOOP(nb) \
    for (long base_ = (long)blockIdx.x * blockDim.x; base_ < (long)(nb) * HALF; base_ += (long)gridDim.x * blockDim.x)

// ------------------------------------------------------------------ init
// x = 0, r = b = g (cast), z = M^-1 r; PCG: p0 = z, rz[0] = r.z;
// BiCGSTAB: rhat = r, p = v = 0, rho[0] = rhat.r.  rr[0] = bb = ||b||^2.
template <class T>
__global__ void k_kry_init(KrylovArgs<T> A, const double* __restrict__ g, T* x, T* r, T* z, T* p0, T* rh, T* v,
                           int bicg, double* rz0, double* rr0, double* bb) {
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        bool valid = b < A.nb && l < 12;
        int s = b < A.nb ? A.bscene[b] : 0;
        bool on = valid && !A.ndone[s];
        double rv = on ? g[12L * b + l] : 0.0;
        double zv = precond_lane(A.dinv + 144L * (b < A.nb ? b : 0), l, rv, 0xffffffffu);
        if (valid) {
            long i = 12L * b + l;
            x[i] = (T)0; r[i] = (T)rv;
            if (bicg) { rh[i] = (T)rv; p0[i] = (T)0; v[i] = (T)0; }
            else { z[i] = (T)zv; p0[i] = (T)zv; }
        }
        warp_reduce_add(bb, s, rv * rv, on);
        warp_reduce_add(rr0, s, rv * rv, on);
        warp_reduce_add(rz0, s, bicg ? rv * rv : rv * zv, on);
    }
}

// ------------------------------------------------------------------ PCG
// K1(k): p_k = z + beta p_{k-1} (on the fly), v = A p_k, pAp += p.v
template <class T>
__global__ void k_pcg_spmv(KrylovArgs<T> A, int k, const T* __restrict__ z, const T* __restrict__ pprev, T* pcur, T* v,
                           const double* rz_k, const double* rz_km1, const double* rr_k, const double* pAp_km1,
                           double* pAp_k, double* zero_a, double* zero_b) {
    if (blockIdx.x == 0) for (int s = threadIdx.x; s < A.ns; s += blockDim.x) { zero_a[s] = 0.0; zero_b[s] = 0.0; }
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        bool valid = b < A.nb && l < 12;
        int s = b < A.nb ? A.bscene[b] : 0;
        bool on = valid && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  (k == 0 || pAp_km1[s] > 0);
        double vv = 0, pv = 0;
        if (on) {
            double beta = (k == 0) ? 0.0 : rz_k[s] / rz_km1[s];
            double acc = 0;
            for (int q = A.row_ptr[b]; q < A.row_ptr[b+1]; q++) {
                const T* V = A.vals + (long)q * 144 + l;
                long cb = 12L * A.bcol[q];
#pragma unroll
                for (int c = 0; c < 12; c++) {
                    double pc = (k == 0) ? (double)pprev[cb + c] : (double)z[cb + c] + beta * (double)pprev[cb + c];
                    acc += (double)V[c * 12] * pc;
                }
            }
            long i = 12L * b + l;
            pv = (k == 0) ? (double)pprev[i] : (double)z[i] + beta * (double)pprev[i];
            pcur[i] = (T)pv;
            v[i] = (T)acc;
            vv = acc;
        }
        warp_reduce_add(pAp_k, s, pv * vv, on);
    }
}
// K2(k): x += a p, r -= a v, z = M^-1 r, rz_{k+1} += r.z, rr_{k+1} += r.r
template <class T>
__global__ void k_pcg_update(KrylovArgs<T> A, int k, T* x, T* r, T* z, const T* __restrict__ pcur, const T* __restrict__ v,
                             const double* rz_k, const double* pAp_k, const double* rr_k, const double* pAp_km1,
                             double* rz_k1, double* rr_k1, double* zero_pAp_next, int* kiter) {
    if (blockIdx.x == 0) for (int s = threadIdx.x; s < A.ns; s += blockDim.x) zero_pAp_next[s] = 0.0;
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        int bb = b < A.nb ? b : 0;
        bool valid = b < A.nb && l < 12;
        int s = A.bscene[bb];
        bool on = b < A.nb && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  (k == 0 || pAp_km1[s] > 0);
        // all 16 lanes of a body share `on`
        double rn = 0;
        long i = 12L * bb + (l < 12 ? l : 0);
        if (on && valid) {
            double pAp = pAp_k[s];
            double alpha = pAp > 0 ? rz_k[s] / pAp : 0.0;
            x[i] = (T)((double)x[i] + alpha * (double)pcur[i]);
            rn = (double)r[i] - alpha * (double)v[i];
            r[i] = (T)rn;
            // non-positive curvature (alpha = 0 here) stops the scene at the next iteration
        }
        double zv = precond_lane(A.dinv + 144L * bb, l, rn, 0xffffffffu);
        if (on && valid) z[i] = (T)zv;
        if (on && valid && l == 0) kiter[s] = k + 1;
        warp_reduce_add(rz_k1, s, rn * zv, on && valid);
        warp_reduce_add(rr_k1, s, rn * rn, on && valid);
    }
}

// ------------------------------------------------------------------ BiCGSTAB
// running scalars per scene: rho_prev, alpha, omega at SD_KS, SD_KA, SD_KW
// KA(k): beta = (rho_k/rho_prev)(alpha/omega); p = r + beta (p - omega v); y = M^-1 p
template <class T>
__global__ void k_bi_a(KrylovArgs<T> A, int k, const T* __restrict__ r, T* p, const T* __restrict__ v, T* y,
                       const double* rho_k, const double* rr_k, const double* run_rho, const double* run_al,
                       const double* run_om, double* z0, double* z1, double* z2, double* z3, double* z4) {
    if (blockIdx.x == 0) for (int s = threadIdx.x; s < A.ns; s += blockDim.x) { z0[s] = 0; z1[s] = 0; z2[s] = 0; z3[s] = 0; z4[s] = 0; }
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        int bb = b < A.nb ? b : 0;
        bool valid = b < A.nb && l < 12;
        int s = A.bscene[bb];
        bool on = b < A.nb && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  (k == 0 || (run_rho[s] != 0.0 && run_om[s] != 0.0));
        long i = 12L * bb + (l < 12 ? l : 0);
        double pn = 0;
        if (on && valid) {
            double beta = (k == 0) ? 0.0 : (rho_k[s] / run_rho[s]) * (run_al[s] / run_om[s]);
            pn = (double)r[i] + beta * ((double)p[i] - run_om[s] * (double)v[i]);
            p[i] = (T)pn;
        }
        double yv = precond_lane(A.dinv + 144L * bb, l, pn, 0xffffffffu);
        if (on && valid) y[i] = (T)yv;
    }
}
// KB / KD: out = A in; dot1 += w1.out, dot2 += out.out (optional)
DV bool bi_alive(int k, const double* run_rho, const double* run_om, int s) {
    return k == 0 || (run_rho[s] != 0.0 && run_om[s] != 0.0);
}
template <class T>
__global__ void k_bi_spmv(KrylovArgs<T> A, int k, const T* __restrict__ in, T* out, const T* __restrict__ w1,
                          double* dot1, double* dot2, const double* rr_k, const double* run_rho, const double* run_om) {
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        bool valid = b < A.nb && l < 12;
        int s = b < A.nb ? A.bscene[b] : 0;
        bool on = valid && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  bi_alive(k, run_rho, run_om, s);
        double o = 0, w = 0;
        if (on) {
            o = row_mv(A, b, l, in);
            long i = 12L * b + l;
            out[i] = (T)o;
            w = (double)w1[i];
        }
        warp_reduce_add(dot1, s, w * o, on);
        if (dot2) warp_reduce_add(dot2, s, o * o, on);
    }
}
// KC: alpha = rho_k / (rh.v); x += alpha y; s = r - alpha v; z = M^-1 s; ss += s.s
template <class T>
__global__ void k_bi_c(KrylovArgs<T> A, int k, T* x, const T* __restrict__ r, const T* __restrict__ v,
                       const T* __restrict__ y, T* sv, T* z, const double* rho_k, const double* rv, const double* rr_k,
                       double* ss, const double* run_rho, const double* run_om) {
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        int bb = b < A.nb ? b : 0;
        bool valid = b < A.nb && l < 12;
        int s = A.bscene[bb];
        bool on = b < A.nb && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  bi_alive(k, run_rho, run_om, s);
        long i = 12L * bb + (l < 12 ? l : 0);
        double sn = 0;
        if (on && valid) {
            double alpha = rv[s] != 0.0 ? rho_k[s] / rv[s] : 0.0;
            x[i] = (T)((double)x[i] + alpha * (double)y[i]);
            sn = (double)r[i] - alpha * (double)v[i];
            sv[i] = (T)sn;
        }
        double zv = precond_lane(A.dinv + 144L * bb, l, sn, 0xffffffffu);
        if (on && valid) z[i] = (T)zv;
        warp_reduce_add(ss, s, sn * sn, on && valid);
    }
}
// KE: omega = (t.s)/(t.t); x += omega z; r = s - omega t; rho_{k+1} += rh.r; rr_{k+1} += r.r
template <class T>
__global__ void k_bi_e(KrylovArgs<T> A, int k, T* x, T* r, const T* __restrict__ sv, const T* __restrict__ z,
                       const T* __restrict__ tv, const T* __restrict__ rh, const double* rho_k, const double* rv,
                       const double* ts, const double* tt, const double* ss, const double* rr_k, double* rho_k1,
                       double* rr_k1, const double* run_rho, const double* run_om, double* nrun_rho, double* nrun_al,
                       double* nrun_om, int* kiter) {
    HALF_LOOP(A.nb) {
        long t = base_ + threadIdx.x;
        int b = (int)(t / HALF), l = (int)(t % HALF);
        bool valid = b < A.nb && l < 12;
        int s = b < A.nb ? A.bscene[b] : 0;
        bool on = valid && !A.ndone[s] && !A.kdone[s] && scene_active(rr_k, A.bb, A.tol2, s) && k < A.maxit &&
                  bi_alive(k, run_rho, run_om, s);
        double rn = 0, rhv = 0;
        if (on) {
            bool s_conv = ss[s] <= A.tol2 * A.bb[s];
            double omega = (s_conv || !(tt[s] > 0)) ? 0.0 : ts[s] / tt[s];
            long i = 12L * b + l;
            x[i] = (T)((double)x[i] + omega * (double)z[i]);
            rn = (double)sv[i] - omega * (double)tv[i];
            r[i] = (T)rn;
            rhv = (double)rh[i];
            // the scene's first DoF keeps the running scalars
            if (l == 0 && (b == 0 || A.bscene[b-1] != s)) {
                // next iteration's scalars; omega == 0 or rho == 0 (breakdown or an
                // already converged s) ends this scene's iterations
                double alpha = rv[s] != 0.0 ? rho_k[s] / rv[s] : 0.0;
                nrun_rho[s] = rho_k[s]; nrun_al[s] = alpha; nrun_om[s] = omega;
                kiter[s] = k + 1;
            }
        }
        warp_reduce_add(rho_k1, s, rhv * rn, on);
        warp_reduce_add(rr_k1, s, rn * rn, on);
    }
}

// number of scenes still iterating
// PCG (bicg = 0): a scene stays alive while its last p.Ap > 0.
// BiCGSTAB (bicg = 1): while its running rho and omega are non-zero (rho may
// be negative).
__global__ void k_count_active(int ns, const int* ndone, const int* kdone, const double* rr, const double* bb,
                               double tol2, const double* alive1, const double* alive2, int bicg, int* out) {
    int c = 0;
    for (int s = threadIdx.x; s < ns; s += blockDim.x) {
        bool alive = bicg ? (alive1[s] != 0.0 && alive2[s] != 0.0) : (alive1[s] > 0.0);
        if (!ndone[s] && !kdone[s] && rr[s] > tol2 * bb[s] && alive) c++;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) { int t = 0; for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += sh[w]; *out = t; }
}

template <class T>
__global__ void k_copy_out(int n, const T* __restrict__ x, double* du) { GS_LOOP(i, n) du[i] = (double)x[i]; }

template <class T>
static int solve_t(Engine* E, int* iters) {
    int rc0 = eng_asm_wait(E);
    if (rc0) return rc0;
    cudaStream_t st = E->stream;
    int ns = E->ns, nb = E->nb;
    T* kv[10];
    for (int i = 0; i < 10; i++) kv[i] = (T*)E->kv[i];
    KrylovArgs<T> A;
    A.nb = nb; A.ns = ns; A.row_ptr = E->row_ptr; A.bcol = E->bcol; A.vals = (const T*)E->vals; A.dinv = (const T*)E->dinv;
    A.bscene = E->bscene; A.ndone = E->sci + SI_DONE * ns; A.kdone = E->sci + SI_KDONE * ns;
    A.tol2 = E->P.lin_tol * E->P.lin_tol; A.maxit = E->P.lin_max_iter; A.bb = E->scd + SD_BB * ns;
    int* kdone = E->sci + SI_KDONE * ns;
    int* kiter = E->sci + SI_KITER * ns;
    CUDA_TRY(cudaMemsetAsync(kdone, 0, sizeof(int) * ns, st));
    CUDA_TRY(cudaMemsetAsync(kiter, 0, sizeof(int) * ns, st));
    // zero all rings
    CUDA_TRY(cudaMemsetAsync(E->scd + SD_BB * ns, 0, sizeof(double) * ns * (SD_COUNT - SD_BB), st));
    int bicg = E->krylov_kind == ABD_SOLVER_BICGSTAB;
    int nthr = 256;
    int grid = grid_for((long)nb * HALF, nthr);
    double* rz = E->scd + SD_K0 * ns;   // ring of 3 (PCG rz / BiCGSTAB rho)
    double* rr = E->scd + SD_K1 * ns;   // ring of 3
    double* pa = E->scd + SD_K2 * ns;   // ring of 3 (PCG pAp / BiCGSTAB rh.v)
    double* s1 = E->scd + SD_K3 * ns;   // BiCGSTAB s.s (ring 3)
    double* s2 = E->scd + SD_K4 * ns;   // t.s
    double* s3 = E->scd + SD_K5 * ns;   // t.t
    auto R = [&](double* base, int q) { return base + (q % 3) * ns; };
    k_kry_init<T><<<grid, nthr, 0, st>>>(A, E->g, kv[KV_X], kv[KV_R], kv[KV_Z], kv[KV_P0], kv[KV_RH], kv[KV_V], bicg,
                                         R(rz, 0), R(rr, 0), E->scd + SD_BB * ns);
    E->launches++;
    // BiCGSTAB running scalars, double-buffered by iteration parity (the
    // SD_KS..SD_KR slots hold buffer 0, the K5 ring's spare slots buffer 1)
    double* runb[2][3] = {{E->scd + SD_KS * ns, E->scd + SD_KA * ns, E->scd + SD_KW * ns},
                          {E->scd + SD_KR * ns, E->scd + (SD_KR + 1) * ns, E->scd + (SD_KR + 2) * ns}};
    // algorithmic bytes of one SpMV: every block once, the input vector
    // (and for PCG the previous direction) once, two output vectors
    double spmv_bytes = (double)sizeof(T) * (144.0 * E->nnzb_host + 48.0 * nb);
    int k = 0;
    for (; k < A.maxit; k++) {
        if (!bicg) {
            T* pprev = kv[(k % 2) ? KV_P0 : KV_P1];
            T* pcur = kv[(k % 2) ? KV_P1 : KV_P0];
            if (k == 0) { pprev = kv[KV_P0]; pcur = kv[KV_P0]; }
            // K1 zeros rz/rr slot k+1; K2 zeros pAp slot k+1
            int ph = phase_begin(E, PH_SPMV);
            k_pcg_spmv<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_Z], pprev, pcur, kv[KV_V], R(rz, k), R(rz, k + 2), R(rr, k),
                                                 R(pa, k + 2), R(pa, k), R(rz, k + 1), R(rr, k + 1));
            phase_end(E, ph, spmv_bytes);
            k_pcg_update<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_X], kv[KV_R], kv[KV_Z], pcur, kv[KV_V], R(rz, k), R(pa, k),
                                                   R(rr, k), R(pa, k + 2), R(rz, k + 1), R(rr, k + 1), R(pa, k + 1), kiter);
            E->launches += 2;
        } else {
            double** rc_ = runb[k % 2];
            double** rn_ = runb[(k + 1) % 2];
            // KA zeros this iteration's accumulators (rh.v, s.s, t.s, t.t, rho_{k+1}, rr_{k+1})
            k_bi_a<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_R], kv[KV_P0], kv[KV_V], kv[KV_Y], R(rz, k), R(rr, k), rc_[0], rc_[1],
                                             rc_[2], R(pa, k), R(s1, k), R(s2, k), R(s3, k), R(rz, k + 1));
            CUDA_TRY(cudaMemsetAsync(R(rr, k + 1), 0, sizeof(double) * ns, st));
            int ph = phase_begin(E, PH_SPMV);
            k_bi_spmv<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_Y], kv[KV_V], kv[KV_RH], R(pa, k), nullptr, R(rr, k), rc_[0], rc_[2]);
            phase_end(E, ph, spmv_bytes);
            k_bi_c<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_X], kv[KV_R], kv[KV_V], kv[KV_Y], kv[KV_S], kv[KV_Z], R(rz, k),
                                             R(pa, k), R(rr, k), R(s1, k), rc_[0], rc_[2]);
            k_bi_spmv<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_Z], kv[KV_T], kv[KV_S], R(s2, k), R(s3, k), R(rr, k), rc_[0], rc_[2]);
            k_bi_e<T><<<grid, nthr, 0, st>>>(A, k, kv[KV_X], kv[KV_R], kv[KV_S], kv[KV_Z], kv[KV_T], kv[KV_RH], R(rz, k),
                                             R(pa, k), R(s2, k), R(s3, k), R(s1, k), R(rr, k), R(rz, k + 1), R(rr, k + 1),
                                             rc_[0], rc_[2], rn_[0], rn_[1], rn_[2], kiter);
            E->launches += 5;
        }
        if ((k + 1) % CHECK_EVERY == 0 || k + 1 == A.maxit) {
            if (bicg) k_count_active<<<1, 256, 0, st>>>(ns, A.ndone, kdone, R(rr, k + 1), A.bb, A.tol2, runb[(k + 1) % 2][0],
                                                        runb[(k + 1) % 2][2], 1, &E->dcnt->krylov_active);
            else k_count_active<<<1, 256, 0, st>>>(ns, A.ndone, kdone, R(rr, k + 1), A.bb, A.tol2, R(pa, k), nullptr, 0,
                                                   &E->dcnt->krylov_active);
            E->launches++;
            int rc = eng_sync_counters(E);
            if (rc) return rc;
            if (E->hcnt->krylov_active == 0) { k++; break; }
        }
    }
    // the cap ended the solve with scenes above tolerance: reported, not fatal
    if (k >= A.maxit && E->hcnt->krylov_active > 0) E->solver_capped++;
    k_copy_out<T><<<grid_for(12L * nb), 256, 0, st>>>(12 * nb, kv[KV_X], E->du);
    E->launches++;
    // iterations actually used by the slowest scene
    CUDA_TRY(cudaMemcpyAsync(E->hsci, kiter, sizeof(int) * ns, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(eng_stream_sync(E));
    int mx = 0;
    for (int s = 0; s < ns; s++) mx = E->hsci[s] > mx ? E->hsci[s] : mx;
    *iters = mx;
    return ABD_OK;
}

static int resolved_solver(const Engine* E) {
    int kind = E->P.linear_solver;
    // AUTO: the component-wise direct solve, which itself hands over to the
    // Krylov solver when a step has too many large components
    if (kind == ABD_SOLVER_AUTO) kind = ABD_SOLVER_DIRECT;
    return kind;
}

// an increment entry above this (scene units for positions, dimensionless for
// the affine rows) is no Newton step of a physical scene: it is taken as an
// FP32 breakdown like a non-finite one
constexpr double DU_GUARD_MAX = 1e6;
// Mixed precision: a scene whose FP32 solve left a non-finite entry in du
// takes the block-Jacobi direction du_b = D_b^-1 g_b instead (every body's
// inverse diagonal block is finite: a singular block inverts to the
// identity), so the line search gets a descent direction rather than NaN.
__global__ void k_du_nonfinite(int nb, const double* __restrict__ du, const int* __restrict__ bscene,
                               const int* __restrict__ done, int* bad) {
    GS_LOOP(i, 12L * nb) {
        int s = bscene[i / 12];
        if (!done[s] && !(fabs(du[i]) <= DU_GUARD_MAX)) bad[s] = 1;     // non-finite or absurd
    }
}
__global__ void k_du_jacobi(int nb, const float* __restrict__ dinv, const double* __restrict__ g,
                            const int* __restrict__ bscene, const int* __restrict__ bad, double* du) {
    GS_LOOP(i, 12L * nb) {
        long b = i / 12; int r = (int)(i % 12);
        if (!bad[bscene[b]]) continue;
        const float* D = dinv + 144 * b;
        double acc = 0;
#pragma unroll
        for (int c = 0; c < 12; c++) acc += (double)D[c * 12 + r] * g[12 * b + c];
        du[i] = acc;
    }
}
// counts the scenes whose increment the guard replaced (read with the
// step's statistics, no sync of its own)
__global__ void k_du_guard_count(int ns, const int* __restrict__ bad, Counters* cnt) {
    int n = 0;
    for (int s = threadIdx.x; s < ns; s += blockDim.x) n += bad[s];
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0 && n) atomicAdd(&cnt->du_guard, n);
}
// test hook (AbdParams.test_inject): a non-finite increment in scene 0,
// written over the solver's output on the host's request; no kernel reads
// outside du
__global__ void k_du_poison(const int* __restrict__ bscene, int nb, double* du) {
    GS_LOOP(i, 12L * nb) if (bscene[i / 12] == 0 && (i % 12) == 0) du[i] = __longlong_as_double(0x7ff8000000000000LL);
}
static int du_guard(Engine* E, bool inject) {
    cudaStream_t s = E->stream;
    int* bad = E->sci + SI_DUBAD * E->ns;
    if (inject) {
        k_du_poison<<<grid_for(12L * E->nb), 256, 0, s>>>(E->bscene, E->nb, E->du);
        E->launches++;
    }
    CUDA_TRY(cudaMemsetAsync(bad, 0, sizeof(int) * E->ns, s));
    k_du_nonfinite<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, E->du, E->bscene, E->sci + SI_DONE * E->ns, bad);
    k_du_jacobi<<<grid_for(12L * E->nb), 256, 0, s>>>(E->nb, (const float*)E->dinv, E->g, E->bscene, bad, E->du);
    k_du_guard_count<<<1, 256, 0, s>>>(E->ns, bad, E->dcnt);
    E->launches += 3;
    return ABD_OK;
}
static int solve_any(Engine* E, int* iters);
int eng_solve(Engine* E, int* iters, bool first_iter) {
    int rc = solve_any(E, iters);
    if (rc || !E->mixed) return rc;
    return du_guard(E, first_iter && (E->P.test_inject & ABD_INJECT_DU_NONFINITE));
}
static int solve_any(Engine* E, int* iters) {
    int kind = resolved_solver(E);
    if (kind == ABD_SOLVER_DIRECT) {
        int ph = phase_begin(E, PH_DENSE);
        int fallback = 0;
        int rc = eng_solve_direct(E, iters, &fallback);
        phase_end(E, ph, 0);
        if (rc || !fallback) return rc;
        // too many large components for one factorization each
        kind = E->P.hess_mode == ABD_HESS_PROJECTED ? ABD_SOLVER_PCG : ABD_SOLVER_BICGSTAB;
    }
    KrylovKind kk(E, kind);
    if (E->mixed) return solve_t<float>(E, iters);
    return solve_t<double>(E, iters);
}
