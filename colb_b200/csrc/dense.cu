// dense.cu — direct solve of the Newton system (the reference's
// solver_config != "cg" branch, abd.py:637-654, which factors the assembled
// matrix with a cuSOLVER wrapper).
//
// The system decouples into the connected components of the body graph whose
// edges are the off-diagonal 12x12 blocks (two dynamic bodies joined by an
// active contact).  A component is factored on its own:
//   - one body: the 12x12 block inverse written by the assembly;
//   - FP64, Hessian projected to PSD and, in reverse Cuthill-McKee order, a
//     body bandwidth of at most BAND_MAX: one CTA per component runs a banded
//     block Cholesky with a sliding window in shared memory, all such
//     components in one launch;
//   - otherwise up to SMALL_MAX_BODIES bodies: one CTA per component factors
//     it in shared memory (blocked Cholesky by 12-wide body columns; LU with
//     partial pivoting when a pivot is not positive), all in one launch;
//   - larger components: the 12x12 blocks are scattered into a dense
//     column-major matrix and factored with cuSOLVER (Cholesky, or LU when
//     Cholesky reports a non-positive pivot).
// Mixed precision factors in FP32.
#include "engine.cuh"
#include <cstring>
#include <cusolverDn.h>
#include <algorithm>

// Scatter the blocks of every body that belongs to a large component into
// that component's dense column-major matrix (16 lanes per body row).
template <class T>
__global__ void k_blocks_to_dense(int nb, const int* __restrict__ row_ptr, const int* __restrict__ bcol,
                                  const T* __restrict__ vals, const int* __restrict__ bcomp,
                                  const int* __restrict__ blocal, const long long* __restrict__ comp_off,
                                  const long long* __restrict__ comp_n, int only_c, T* dense) {
    for (long base = (long)blockIdx.x * blockDim.x; base < (long)nb * 16; base += (long)gridDim.x * blockDim.x) {
        long t = base + threadIdx.x;
        int b = (int)(t / 16), l = (int)(t % 16);
        if (b >= nb || l >= 12) continue;
        int c = bcomp[b];
        if (c < 0 || (only_c >= 0 && c != only_c)) continue;
        long n = comp_n[c];
        T* A = dense + comp_off[c];
        long row = 12L * blocal[b] + l;
        for (int k = row_ptr[b]; k < row_ptr[b + 1]; k++) {
            long colb = 12L * blocal[bcol[k]];
            const T* V = vals + (long)k * 144 + l;
#pragma unroll
            for (int j = 0; j < 12; j++) A[(colb + j) * n + row] = V[j * 12];
        }
    }
}
// right-hand sides of large components, gathered in component order
template <class T>
__global__ void k_rhs_gather(int nb, const double* __restrict__ g, const int* __restrict__ bcomp,
                             const int* __restrict__ blocal, const long long* __restrict__ comp_rhs, T* x) {
    GS_LOOP(i, 12L * nb) {
        int b = (int)(i / 12), c = bcomp[b];
        if (c >= 0) x[comp_rhs[c] + 12L * blocal[b] + i % 12] = (T)g[i];
    }
}
// du of every body: large components from their dense solution, single
// bodies from their 12x12 block inverse (column-major); bodies of small
// components (bcomp -2) and band components (-3) were written by
// k_small_solve / k_band_solve
template <class T>
__global__ void k_du_scatter(int nb, const double* __restrict__ g, const int* __restrict__ bcomp,
                             const int* __restrict__ blocal, const long long* __restrict__ comp_rhs,
                             const T* __restrict__ x, const T* __restrict__ dinv, const int* __restrict__ bscene,
                             const int* __restrict__ ndone, double* du) {
    GS_LOOP(i, 12L * nb) {
        int b = (int)(i / 12), r = (int)(i % 12);
        if (ndone[bscene[b]]) continue;
        int c = bcomp[b];
        if (c <= -2) continue;
        if (c >= 0) { du[i] = (double)x[comp_rhs[c] + 12L * blocal[b] + r]; continue; }
        const T* D = dinv + 144L * b;
        double acc = 0;
#pragma unroll
        for (int k = 0; k < 12; k++) acc += (double)D[k * 12 + r] * g[12L * b + k];
        du[i] = acc;
    }
}

constexpr int SMALL_MAX_BODIES = 12;
constexpr int SMALL_THREADS = 256;

// Load the blocks of the component's bodies (local order sb[0..nbod)) into
// the row-major n x n matrix A (leading dimension ld) and g into x.
template <class T>
__device__ void small_fill(int nbod, int n, int ld, const int* sb, const int* __restrict__ blocal,
                           const int* __restrict__ row_ptr, const int* __restrict__ bcol, const T* __restrict__ vals,
                           const double* __restrict__ g, T* A, T* x) {
    for (int e = threadIdx.x; e < n * ld; e += blockDim.x) A[e] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = warp; i < nbod; i += nw) {
        int b = sb[i];
        for (int k = row_ptr[b]; k < row_ptr[b + 1]; k++) {
            int j = blocal[bcol[k]];
            const T* V = vals + (long)k * 144;
            for (int e = lane; e < 144; e += 32) {
                int cc = e / 12, r = e % 12;        // blocks are column-major
                A[(12 * i + r) * ld + 12 * j + cc] = V[e];
            }
        }
        if (lane < 12) x[12 * i + lane] = (T)g[12L * b + lane];
    }
    __syncthreads();
}

// One CTA per small component: A du = g in shared memory.  status bit 0 is
// set when a component is singular (its du is zero).
template <class T>
__global__ void __launch_bounds__(SMALL_THREADS) k_small_solve(int nsmall, const int* __restrict__ sptr,
        const int* __restrict__ sbody, const int* __restrict__ blocal, const int* __restrict__ row_ptr,
        const int* __restrict__ bcol, const T* __restrict__ vals, const double* __restrict__ g, int try_chol,
        double* du, int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int flag, piv;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = blockIdx.x; c < nsmall; c += gridDim.x) {
        const int* sb = sbody + sptr[c];
        const int nbod = sptr[c + 1] - sptr[c], n = 12 * nbod, ld = n + 1;
        T* A = (T*)smem_raw;
        T* x = A + n * ld;
        small_fill<T>(nbod, n, ld, sb, blocal, row_ptr, bcol, vals, g, A, x);
        if (tid == 0) flag = try_chol ? 0 : 1;
        __syncthreads();
        // blocked right-looking Cholesky, lower triangle, 12-wide body columns;
        // flag is written by warp 0 in the diagonal step only and read right
        // after the barrier that follows it, so every thread takes the same branch
        for (int K = 0; try_chol && K < nbod; K++) {
            const int kb = 12 * K;
            if (warp == 0) {
                for (int j = 0; j < 12; j++) {
                    if (lane == 0) {
                        T d = A[(kb + j) * ld + kb + j];
                        if (!(d > (T)0)) flag = 1;
                        A[(kb + j) * ld + kb + j] = d > (T)0 ? sqrt(d) : (T)1;
                    }
                    __syncwarp();
                    T djj = A[(kb + j) * ld + kb + j];
                    if (lane > j && lane < 12) A[(kb + lane) * ld + kb + j] /= djj;
                    __syncwarp();
                    if (lane > j && lane < 12) {
                        T lij = A[(kb + lane) * ld + kb + j];
                        for (int cc = j + 1; cc <= lane; cc++) A[(kb + lane) * ld + kb + cc] -= lij * A[(kb + cc) * ld + kb + j];
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            if (flag) break;
            // panel: rows below solve L_ik D^T = A_ik
            for (int i = kb + 12 + tid; i < n; i += blockDim.x) {
                T* Ri = A + i * ld + kb;
                for (int j = 0; j < 12; j++) {
                    T a = Ri[j];
                    for (int t = 0; t < j; t++) a -= Ri[t] * A[(kb + j) * ld + kb + t];
                    Ri[j] = a / A[(kb + j) * ld + kb + j];
                }
            }
            __syncthreads();
            // trailing update of the lower triangle
            const int m = n - kb - 12;
            for (int e = tid; e < m * m; e += blockDim.x) {
                int i = kb + 12 + e / m, j = kb + 12 + e % m;
                if (j > i) continue;
                const T* Li = A + i * ld + kb;
                const T* Lj = A + j * ld + kb;
                T acc = 0;
#pragma unroll
                for (int t = 0; t < 12; t++) acc += Li[t] * Lj[t];
                A[i * ld + j] -= acc;
            }
            __syncthreads();
        }
        if (!flag) {
            // L y = g, then L^T du = y
            for (int K = 0; K < nbod; K++) {
                const int kb = 12 * K;
                if (tid == 0)
                    for (int j = 0; j < 12; j++) {
                        T a = x[kb + j];
                        for (int t = 0; t < j; t++) a -= A[(kb + j) * ld + kb + t] * x[kb + t];
                        x[kb + j] = a / A[(kb + j) * ld + kb + j];
                    }
                __syncthreads();
                for (int i = kb + 12 + tid; i < n; i += blockDim.x) {
                    T acc = 0;
                    for (int t = 0; t < 12; t++) acc += A[i * ld + kb + t] * x[kb + t];
                    x[i] -= acc;
                }
                __syncthreads();
            }
            for (int K = nbod - 1; K >= 0; K--) {
                const int kb = 12 * K;
                if (tid == 0)
                    for (int j = 11; j >= 0; j--) {
                        T a = x[kb + j];
                        for (int t = j + 1; t < 12; t++) a -= A[(kb + t) * ld + kb + j] * x[kb + t];
                        x[kb + j] = a / A[(kb + j) * ld + kb + j];
                    }
                __syncthreads();
                for (int i = tid; i < kb; i += blockDim.x) {
                    T acc = 0;
                    for (int t = 0; t < 12; t++) acc += A[(kb + t) * ld + i] * x[kb + t];
                    x[i] -= acc;
                }
                __syncthreads();
            }
        } else {
            // LU with partial pivoting on a fresh copy
            small_fill<T>(nbod, n, ld, sb, blocal, row_ptr, bcol, vals, g, A, x);
            bool singular = false;
            for (int k = 0; k < n; k++) {
                if (warp == 0) {
                    T best = -1; int bi = k;
                    for (int i = k + lane; i < n; i += 32) {
                        T v = fabs(A[i * ld + k]);
                        if (v > best) { best = v; bi = i; }
                    }
                    for (int o = 16; o > 0; o >>= 1) {
                        T ob = __shfl_xor_sync(0xffffffffu, best, o);
                        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
                    }
                    if (lane == 0) piv = bi;
                }
                __syncthreads();
                const int p = piv;
                if (p != k) {
                    for (int j = tid; j < n; j += blockDim.x) { T t = A[k * ld + j]; A[k * ld + j] = A[p * ld + j]; A[p * ld + j] = t; }
                    if (tid == 0) { T t = x[k]; x[k] = x[p]; x[p] = t; }
                }
                __syncthreads();
                const T pv = A[k * ld + k];
                if (pv == (T)0) { singular = true; break; }
                for (int i = k + 1 + tid; i < n; i += blockDim.x) A[i * ld + k] /= pv;
                __syncthreads();
                const int m = n - k - 1;
                for (int e = tid; e < m * m; e += blockDim.x) {
                    int i = k + 1 + e / m, j = k + 1 + e % m;
                    A[i * ld + j] -= A[i * ld + k] * A[k * ld + j];
                }
                __syncthreads();
            }
            if (singular) {
                for (int i = tid; i < n; i += blockDim.x) x[i] = 0;
                if (tid == 0) atomicOr(status, 1);
                __syncthreads();
            } else {
                for (int k = 0; k < n; k++) {
                    const T xk = x[k];
                    for (int i = k + 1 + tid; i < n; i += blockDim.x) x[i] -= A[i * ld + k] * xk;
                    __syncthreads();
                }
                for (int k = n - 1; k >= 0; k--) {
                    if (tid == 0) x[k] /= A[k * ld + k];
                    __syncthreads();
                    const T xk = x[k];
                    for (int i = tid; i < k; i += blockDim.x) x[i] -= A[i * ld + k] * xk;
                    __syncthreads();
                }
            }
        }
        for (int i = tid; i < n; i += blockDim.x) du[12L * sb[i / 12] + i % 12] = (double)x[i];
        __syncthreads();
    }
}


// ------------------------------------------------------------------ band components
// 16-byte asynchronous global -> shared copies (cp.async, L1 bypassed): the
// band kernel fetches the next block row, right-hand side and backward factor
// column while it computes, so no global load latency sits on its critical
// path.  Addresses are 16-byte aligned (blocks of 144 doubles, 12-double rows).
DV void band_cp16(void* sdst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"((uint32_t)__cvta_generic_to_shared(sdst)), "l"(gsrc)
                 : "memory");
}
DV void band_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
DV void band_cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
DV void band_cp_wait_but_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
// named CTA barrier `id` over `n` threads (counted per thread, so a warp
// may reach it diverged): arrive only, which publishes this thread's earlier
// shared-memory writes to the waiting threads, or arrive and wait
DV void band_bar_arrive(int id, int n) { asm volatile("barrier.arrive %0, %1;" :: "r"(id), "r"(n) : "memory"); }
DV void band_bar_sync(int id, int n) { asm volatile("barrier.sync %0, %1;" :: "r"(id), "r"(n) : "memory"); }
// cluster barrier in two halves: arrive (release: this thread's earlier
// writes, global memory included, become visible to the cluster) and wait
// (acquire); every thread of the cluster arrives once per phase
DV void band_cluster_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
DV void band_cluster_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }

// A component whose bodies, in reverse Cuthill-McKee order, couple only
// bodies at most BAND_MAX apart is a block band matrix: its Cholesky factor
// L has the same band.  One CTA factors it with a sliding window of
// (BAND_MAX + 1)^2 12x12 blocks in shared memory, all band components in
// one launch, with no host synchronisation.  The inverse diagonal factors
// Linv_k = L_kk^-1 are kept explicitly, so every panel entry is an
// independent dot product.  Block column k:
//   1. panel L_ik = A_ik Linv_k^T: warp 0 computes block row k + 1 and
//      signals it at a named barrier without waiting; warps 1..6 compute
//      the rows below, warp 7 the forward elimination y_k = Linv_k g_k;
//   2. warp 0 goes straight on: A_{k+1,k+1} - L_{k+1,k} L_{k+1,k}^T into
//      registers, then its Cholesky factor and inverse (Linv_{k+1}) in one
//      sweep of 12 pivots; warps 1..7, once the whole panel is there (named
//      barrier), apply column k to the rest of the window
//      (A_ij -= L_ik L_jk^T), eliminate the right-hand sides below, write
//      the factor column to global scratch and bring the next block row
//      into the window.
// One block barrier closes the column.  Warp 0's chain (one panel block
// row, the diagonal update, 12 pivots) is the critical path.  The backward
// solve, x_k = Linv_k^T (y_k - sum_d L_{k+d,k}^T x_{k+d}), is one short
// dependent chain per column and runs on warp 0 alone under warp-level
// synchronisation, each factor column prefetched two columns ahead.
// FP64 mode only: FP32 roundings of a stiff PSD-projected Hessian can leave
// the matrix indefinite (the rounded 12-body blocks of a chain mail in contact
// have negative eigenvalues), which a Cholesky factorization without pivoting
// cannot take, so mixed-precision components use the shared-memory and
// cuSOLVER paths, which fall back to LU.  A non-positive pivot, which a
// PSD-projected FP64 Hessian does not produce, is replaced by its magnitude.
constexpr int BAND_MAX = 8;
constexpr int BAND_W = BAND_MAX + 1;
constexpr int BAND_THREADS = 256;
// shared-memory stride of one 12x12 block: 146 doubles put the 81 block
// bases of the window on different banks (144 would start every block on
// bank 0, and tiles of different blocks read by one warp would conflict)
constexpr int BAND_BLK = 146;
constexpr int BAND_CREC = BAND_W * 144 + 12;   // backward record: factor column blocks, then y_k
constexpr int BAND_ORD_MAX = 1024;     // bodies of a band component (order kept in shared memory)
// dynamic shared memory of k_band_solve in doubles: window, staged block
// rows, inverse diagonal factors, right-hand sides, y_k, solution blocks,
// staged right-hand sides, backward records, then the body order (ints)
// and the block-pair tables (bytes)
constexpr int band_smem_doubles() {
    return BAND_W * BAND_W * BAND_BLK + 2 * BAND_W * 144 + 2 * 144 + BAND_W * 12 + 12 + BAND_W * 12 + 2 * 12 +
           3 * BAND_CREC + BAND_ORD_MAX / 2 + (BAND_MAX * (BAND_MAX + 1) + 7) / 8;
}
// a component of n bodies and body bandwidth wb is split between the two
// CTAs of its cluster at position m = (n - wb) / 2 when both halves keep at
// least wb / 2 + 6 block columns; -1 when it is factored by one CTA
inline int band_split_point(int n, int wb) { return n >= 2 * wb + 12 ? (n - wb) / 2 : -1; }


// Band blocks of every band component, contiguous and in FP64: A(i, i - d)
// of position i (component order), d = 0..BAND_MAX, row-major, at
// (loff + i BAND_W + d); blocks outside the band or absent are zero.  One
// warp per block.
template <class TV>
__global__ void k_band_gather(int npos, const int* __restrict__ pcomp, const int* __restrict__ cptr,
                              const int* __restrict__ order, const int* __restrict__ cbw, const long long* __restrict__ loff,
                              const int* __restrict__ row_ptr, const int* __restrict__ bcol, const TV* __restrict__ vals,
                              double* Ab) {
    const int lane = threadIdx.x & 31;
    for (long item = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; item < (long)npos * BAND_W;
         item += ((long)gridDim.x * blockDim.x) >> 5) {
        int p = (int)(item / BAND_W), d = (int)(item % BAND_W);
        int c = pcomp[p], i = p - cptr[c], j = i - d;
        int bi = -1;
        if (j >= 0 && d <= cbw[c]) bi = find_block(row_ptr, bcol, order[p], order[cptr[c] + j]);
        double* dst = Ab + (loff[c] + (long)i * BAND_W + d) * 144;
        for (int e = lane; e < 144; e += 32) {
            int r = e / 12, cc = e % 12;
            dst[e] = bi >= 0 ? (double)vals[(long)bi * 144 + cc * 12 + r] : 0.0;     // row-major from column-major
        }
    }
}

// Warp-wide Cholesky factorization and inversion of a 12x12 SPD block in
// one sweep of its 12 pivots.  On entry lane i < 12 holds row i of the
// (symmetric) block in a[]; on exit it holds row i of W = L^-1, zeros right
// of the diagonal, where L L^T is the block.  Step j: lane j owns the pivot
// d_j = a[j]; every lane i > j forms t = a_ij / d_j and subtracts t times
// lane j's row.  Right of column j that row is the remaining block row, so
// this is the Schur update a_ic -= a_ij a_jc / d_j; left of column j it is
// row j of the unscaled inverse w, so this is the forward substitution
// w_i -= (L_ij / L_jj) w_j of L w = I; slot j itself becomes w_ij = -t.
// Finally W_i = w_i / sqrt(d_i).  Lane j's row is final one step before it
// is needed, so each pivot costs one reciprocal square root and one
// broadcast on the dependent chain.  A non-positive pivot sets bit 1 of
// *status and is replaced by its magnitude.
DV void band_chol_inverse_rows(double (&a)[12], int* status) {
    const int lane = threadIdx.x & 31;
    double rown = 0.0;
#pragma unroll
    for (int j = 0; j < 12; j++) {
        double s = 0.0;
        if (lane == j) {
            double d = a[j];
            if (!(d > 0.0)) { atomicOr(status, 2); d = fabs(d) + 1e-30; }
            rown = rsqrt(d);        // the double-precision rsqrt: ~76 cycles of latency on sm_100
            s = rown * rown;
        }
        if (j < 11) {
            s = __shfl_sync(0xffffffffu, s, j);
            const bool upd = lane > j && lane < 12;
            const double t = a[j] * s;
#pragma unroll
            for (int c = 0; c < 12; c++) {
                if (c == j) continue;
                const double v = __shfl_sync(0xffffffffu, a[c], j);
                if (upd) a[c] = fma(-t, v, a[c]);
            }
            if (upd) a[j] = -t;
        }
        if (lane == j) {
            a[j] = 1.0;
#pragma unroll
            for (int c = j + 1; c < 12; c++) a[c] = 0.0;
        }
    }
#pragma unroll
    for (int c = 0; c < 12; c++) a[c] *= rown;
}

// Panel rows in place: R (one row of a block below the diagonal) becomes
// R Linv^T, i.e. entry c = sum_{s <= c} R[s] Linv[c][s].  Two lanes (adjacent
// or 12 apart) share a row and write six entries each; every lane of the
// warp must call it, `act` says whether this lane has a row.
DV void band_panel_row(double* R, const double* Li, int half, bool act) {
    double v[12];
    if (act) {
#pragma unroll
        for (int s = 0; s < 12; s++) v[s] = R[s];
    }
    __syncwarp();
    if (act) {
#pragma unroll
        for (int c6 = 0; c6 < 6; c6++) {
            const int c = half * 6 + c6;
            double acc = 0.0;
#pragma unroll
            for (int s = 0; s < 12; s++) if (s <= c) acc += v[s] * Li[c * 12 + s];
            R[c] = acc;
        }
    }
    __syncwarp();
}

// One job per cluster of two CTAs.  A job is a band component (sub-component
// ct) factored by CTA 0 alone, or a large one split in two: ct holds its
// bodies [0, m + wb) in order, cb the bodies [m, N) in reverse order, and
// S = [m, m + wb) separates [0, m) from [m + wb, N) (the band couples bodies
// at most wb apart).  CTA 0 eliminates [0, m) while CTA 1 eliminates
// [m + wb, N) from the far end; each leaves S in its window with its own
// Schur update applied.  After a cluster barrier CTA 0 adds CTA 1's update
// (S = W0 + W1 - A_SS, right-hand sides likewise), factors and solves S,
// and signals the solution at a second cluster barrier; then both CTAs run
// their backward halves.  The dependent chain shrinks from N block columns
// each way to about (N - wb) / 2 + wb.  jobs holds (ct, cb, m) per job,
// cb = -1 for an unsplit component (m is then its size).
// one CTA per SM (its shared memory allows no second), so the register cap is set for one
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(BAND_THREADS, 1)
k_band_solve(int njobs, const int* __restrict__ jobs, const int* __restrict__ cptr,
        const int* __restrict__ order, const int* __restrict__ cbw, const long long* __restrict__ loff,
        const double* __restrict__ Ab, long long ltot, const double* __restrict__ g, double* Lg, double* du,
        int* status) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* win = (double*)smem_raw;                          // [BAND_W][BAND_W] row-major 12x12 blocks, BAND_BLK apart
    double* stage = win + BAND_W * BAND_W * BAND_BLK;         // [2][BAND_W][144]: next block row
    double* linv = stage + 2 * BAND_W * 144;                  // [2][144] inverse diagonal factors
    double* rhs = linv + 2 * 144;                             // [BAND_W][12]
    double* ybuf = rhs + BAND_W * 12;                         // [12] y_k of the current column
    double* xs = ybuf + 12;                                   // [BAND_W][12] latest solution blocks (backward)
    double* gst = xs + BAND_W * 12;                           // [2][12] right-hand side of each staged block row
    double* cst = gst + 2 * 12;                               // [3][BAND_CREC] backward factor columns and y_k
    int* ord = (int*)(cst + 3 * BAND_CREC);                   // [BAND_ORD_MAX] bodies of the sub-component
    unsigned char* tri_a = (unsigned char*)(ord + BAND_ORD_MAX);   // block pair p -> (a, b), b <= a
    unsigned char* tri_b = tri_a + BAND_MAX * (BAND_MAX + 1) / 2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int t1 = tid - 32, n1 = blockDim.x - 32;            // thread index among warps 1..7
    const int crank = blockIdx.x & 1;                         // rank in the cluster
    if (tid < BAND_MAX * (BAND_MAX + 1) / 2) {
        int a = 0; while ((a + 1) * (a + 2) / 2 <= tid) a++;
        tri_a[tid] = (unsigned char)a; tri_b[tid] = (unsigned char)(tid - a * (a + 1) / 2);
    }
    for (int jb = blockIdx.x >> 1; jb < njobs; jb += gridDim.x >> 1) {
        const int ct = jobs[3 * jb], cb = jobs[3 * jb + 1], msplit = jobs[3 * jb + 2];
        const bool split = cb >= 0;
        if (crank == 1 && !split) {
            // nothing to factor: keep the cluster barriers in step with CTA 0
            band_cluster_arrive(); band_cluster_wait();
            band_cluster_arrive(); band_cluster_wait();
            continue;
        }
        const int cc = crank == 0 ? ct : cb;
        const int N = cptr[cc + 1] - cptr[cc], wb = cbw[cc];
        // columns this CTA eliminates before the merge
        const int ncol1 = !split ? N : (crank == 0 ? msplit : N - wb);
        for (int e = tid; e < N; e += blockDim.x) ord[e] = order[cptr[cc] + e];
        double* L = Lg + loff[cc] * 144;                      // Linv_k at (k BAND_W), L(k + d, k) at (k BAND_W + d)
        double* Y = Lg + ltot * 144 + (loff[cc] / BAND_W) * 12;   // y_k at k * 12
        const double* A = Ab + loff[cc] * 144;                // block A(i, i - d) at (i BAND_W + d)
        __syncthreads();
        auto slot = [&](int i, int j) { return win + ((i % BAND_W) * BAND_W + (j % BAND_W)) * BAND_BLK; };
        // window rows 0..min(wb, N - 1), their right-hand sides, and block
        // row wb + 1 fetched ahead into its staging buffer
        const int r0 = min(wb, N - 1);
        for (int e = tid; e < (r0 + 1) * BAND_W * 144; e += blockDim.x) {
            int i = e / (BAND_W * 144), d = (e / 144) % BAND_W, q = e % 144;
            if (d <= i) slot(i, i - d)[q] = A[(long)e];
        }
        for (int e = tid; e < (r0 + 1) * 12; e += blockDim.x) rhs[(e / 12) * 12 + e % 12] = g[12L * ord[e / 12] + e % 12];
        // block row m and its right-hand side into staging buffer m & 1 by
        // warps 1..7; the stored row holds A(m, m - d) at block d, staged at
        // block wb - d (column m - wb + (wb - d)); the same threads wait for
        // it before the named barrier of the next column
        auto fetch_row = [&](int m) {
            double* dst = stage + (m & 1) * BAND_W * 144;
            const double* src = A + (long)m * BAND_W * 144;
            for (int e = t1; e < (wb + 1) * 72 + 6; e += n1) {
                if (e < (wb + 1) * 72) {
                    const int d = e / 72, c = e % 72;
                    band_cp16(dst + (wb - d) * 144 + 2 * c, src + d * 144 + 2 * c);
                } else {
                    const int c = e - (wb + 1) * 72;
                    band_cp16(gst + (m & 1) * 12 + 2 * c, g + 12L * ord[m] + 2 * c);
                }
            }
            band_cp_commit();
        };
        // warp 0: factor and invert the diagonal block in slot(k, k) into linv[k & 1]
        auto factor_diag = [&](int k) {
            const double* D = slot(k, k);
            double a[12];
#pragma unroll
            for (int c = 0; c < 12; c++) a[c] = lane < 12 ? D[lane * 12 + c] : 0.0;
            band_chol_inverse_rows(a, status);
            if (lane < 12) {
#pragma unroll
                for (int c = 0; c < 12; c++) linv[(k & 1) * 144 + lane * 12 + c] = a[c];
            }
        };
        // block columns k0..k1-1; Linv_k0 is in linv[k0 & 1].  When k1 < N
        // the last column leaves the next diagonal block unfactored, its
        // update applied by warps 1..7 like every other block pair.
        auto columns = [&](int k0, int k1) {
            for (int k = k0; k < k1; k++) {
                const int nk = min(wb, N - 1 - k);               // blocks below the diagonal in this column
                const bool factor_next = k + 1 < k1;
                const double* Li = linv + (k & 1) * 144;
                if (warp == 0) {
                    // panel block row k + 1 (lanes r and r + 12 share row r), signalled to warps 1..7
                    const int r = lane % 12, half = lane / 12;
                    double* P = slot(k + 1, k);
                    if (nk > 0) band_panel_row(P + r * 12, Li, half, lane < 24);
                    band_bar_arrive(1, blockDim.x);
                    if (nk > 0 && factor_next) {
                        // row r of A_{k+1,k+1} - L_{k+1,k} L_{k+1,k}^T: lane r forms entries 0..5,
                        // lane r + 12 entries 6..11 and passes them to lane r
                        const double* Dk = slot(k + 1, k + 1);
                        double h[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                        if (lane < 24) {
                            double lr[12];
#pragma unroll
                            for (int s = 0; s < 12; s++) lr[s] = P[r * 12 + s];
#pragma unroll
                            for (int c6 = 0; c6 < 6; c6++) {
                                const int c = half * 6 + c6;
                                double acc0 = Dk[r * 12 + c], acc1 = 0.0;
#pragma unroll
                                for (int s = 0; s < 12; s += 2) {
                                    acc0 = fma(-lr[s], P[c * 12 + s], acc0);
                                    acc1 = fma(-lr[s + 1], P[c * 12 + s + 1], acc1);
                                }
                                h[c6] = acc0 + acc1;
                            }
                        }
                        double a[12];
#pragma unroll
                        for (int c6 = 0; c6 < 6; c6++) {
                            const double o = __shfl_sync(0xffffffffu, h[c6], (lane + 12) & 31);
                            a[c6] = lane < 12 ? h[c6] : 0.0;
                            a[6 + c6] = lane < 12 ? o : 0.0;
                        }
                        band_chol_inverse_rows(a, status);
                        if (lane < 12) {
                            double* Ln = linv + ((k + 1) & 1) * 144;
#pragma unroll
                            for (int c = 0; c < 12; c++) Ln[lane * 12 + c] = a[c];
                        }
                    }
                } else {
                    if (warp < 7) {
                        // panel rows of blocks k + 2 .. k + nk, two adjacent lanes per row
                        const int q = 12 + (t1 >> 1);
                        const bool act = q < 12 * nk;
                        band_panel_row(act ? slot(k + 1 + q / 12, k) + (q % 12) * 12 : win, Li, t1 & 1, act);
                    } else if (lane < 12) {
                        const double* rk = rhs + (k % BAND_W) * 12;
                        double y = 0.0;
#pragma unroll
                        for (int s = 0; s < 12; s++) if (s <= lane) y += Li[lane * 12 + s] * rk[s];
                        ybuf[lane] = y;
                        Y[(long)k * 12 + lane] = y;
                    }
                    band_cp_wait_all();              // this thread's copies of the staged block row
                    band_bar_sync(1, blockDim.x);    // panel (warp 0's row included), y_k and the staged row are there
                    // A_ij -= L_ik L_jk^T over the window in 3 x 4 tiles (12 per
                    // block pair); pair 0, (k+1, k+1), is warp 0's unless it stays unfactored
                    const int npair = nk * (nk + 1) / 2;
                    for (int e = t1 + (factor_next ? 12 : 0); e < npair * 12; e += n1) {
                        int p = e / 12, tile = e % 12;
                        int i = k + 1 + tri_a[p], j = k + 1 + tri_b[p];
                        int r0t = (tile / 3) * 3, c0t = (tile % 3) * 4;
                        const double* Lia = slot(i, k) + r0t * 12;
                        const double* Ljb = slot(j, k) + c0t * 12;
                        // rows 0, 4 and 8 of a block share a bank (12 doubles per
                        // row): the lanes of the three column groups walk the 12
                        // columns rotated by 0, 1 and 2, so the rows they read at
                        // once lie on different banks
                        const int rot = c0t >> 2;
                        double acc[3][4] = {};
#pragma unroll
                        for (int s0 = 0; s0 < 12; s0++) {
                            const int s = s0 + rot < 12 ? s0 + rot : s0 + rot - 12;
                            double li[3], lj[4];
#pragma unroll
                            for (int a2 = 0; a2 < 3; a2++) li[a2] = Lia[a2 * 12 + s];
#pragma unroll
                            for (int b2 = 0; b2 < 4; b2++) lj[b2] = Ljb[b2 * 12 + s];
#pragma unroll
                            for (int a2 = 0; a2 < 3; a2++)
#pragma unroll
                                for (int b2 = 0; b2 < 4; b2++) acc[a2][b2] += li[a2] * lj[b2];
                        }
                        double* Aij = slot(i, j);
#pragma unroll
                        for (int a2 = 0; a2 < 3; a2++)
#pragma unroll
                            for (int b2 = 0; b2 < 4; b2++) Aij[(r0t + a2) * 12 + c0t + b2] -= acc[a2][b2];
                    }
                    // rhs_i -= L_ik y_k
                    for (int t = t1; t < 12 * nk; t += n1) {
                        int i = k + 1 + t / 12, r = t % 12;
                        const double* R = slot(i, k) + r * 12;
                        double acc = 0.0;
#pragma unroll
                        for (int c = 0; c < 12; c++) acc += R[c] * ybuf[c];
                        rhs[(i % BAND_W) * 12 + r] -= acc;
                    }
                    // factor column k to global: Linv_k, then L(k + d, k)
                    for (int e = t1; e < (nk + 1) * 144; e += n1) {
                        int d = e / 144, q = e % 144;
                        L[((long)k * BAND_W + d) * 144 + q] = d == 0 ? Li[q] : slot(k + d, k)[q];
                    }
                    // block row k + 1 + wb enters the window (staged during the
                    // previous column; its ring row is that of row k, free now),
                    // and row k + 2 + wb is fetched
                    const int m1 = k + 1 + wb, m2 = k + 2 + wb;
                    if (m1 < N) {
                        const double* src = stage + (m1 & 1) * BAND_W * 144;
                        for (int e = t1; e < (wb + 1) * 144; e += n1) {
                            int q = e / 144, x = e % 144;             // block q: column k + 1 + q
                            slot(m1, k + 1 + q)[x] = src[e];
                        }
                        if (t1 < 12) rhs[(m1 % BAND_W) * 12 + t1] = gst[(m1 & 1) * 12 + t1];
                    }
                    if (m2 < N) fetch_row(m2);
                }
                __syncthreads();
            }
        };
        // warp 0: x_k = Linv_k^T (y_k - sum_d L_{k+d,k}^T x_{k+d}) for
        // k = kfirst down to 0, the solution blocks above kfirst already in
        // xs.  The record of column k (its factor blocks, then y_k) sits in
        // ring buffer k % 3 of cst, fetched two columns ahead.  After column
        // kcall the callback runs (once).
        auto backward = [&](int kfirst, int kcall, auto&& callback) {
            auto fetch_col = [&](int kk) {
                const int nkk = min(wb, N - 1 - kk);
                double* dst = cst + (kk % 3) * BAND_CREC;
                const double* src = L + (long)kk * BAND_W * 144;
                for (int e = lane; e < (nkk + 1) * 72 + 6; e += 32) {
                    if (e < (nkk + 1) * 72) band_cp16(dst + 2 * e, src + 2 * e);
                    else band_cp16(dst + BAND_W * 144 + 2 * (e - (nkk + 1) * 72), Y + (long)kk * 12 + 2 * (e - (nkk + 1) * 72));
                }
                band_cp_commit();
            };
            fetch_col(kfirst);
            if (kfirst >= 1) { fetch_col(kfirst - 1); band_cp_wait_but_one(); } else band_cp_wait_all();
            __syncwarp();
            const int r = lane % 12, half = lane / 12;
            for (int k = kfirst; k >= 0; k--) {
                const int nk = min(wb, N - 1 - k);
                const double* col = cst + (k % 3) * BAND_CREC;
                if (k >= 2) fetch_col(k - 2);        // into the buffer column k + 1 used
                // t_r = y_k[r] - sum_d (L_{k+d,k}^T x_{k+d})[r]: lanes r and r + 12 take alternate blocks d
                double t = 0.0;
                if (lane < 24) {
                    double acc0 = half == 0 ? col[BAND_W * 144 + r] : 0.0, acc1 = 0.0;
                    for (int d = 1 + half; d <= nk; d += 2) {
                        const double* B = col + d * 144;
                        const double* xi = xs + ((k + d) % BAND_W) * 12;
#pragma unroll
                        for (int c = 0; c < 12; c += 2) {
                            acc0 = fma(-B[c * 12 + r], xi[c], acc0);
                            acc1 = fma(-B[(c + 1) * 12 + r], xi[c + 1], acc1);
                        }
                    }
                    t = acc0 + acc1;
                }
                t += __shfl_sync(0xffffffffu, t, (lane + 12) & 31);
                // x_k[lane] = sum_{c >= lane} Linv[c][lane] t_c
                double x = 0.0;
#pragma unroll
                for (int c = 0; c < 12; c++) {
                    const double tc = __shfl_sync(0xffffffffu, t, c);
                    if (lane < 12 && c >= lane) x += col[c * 12 + lane] * tc;
                }
                if (lane < 12) { du[12L * ord[k] + lane] = x; xs[(k % BAND_W) * 12 + lane] = x; }
                if (k == kcall) callback();
                // column k - 1 (fetched during column k + 1) must have landed; the
                // fetch issued in this column may still be in flight
                if (k >= 2) band_cp_wait_but_one(); else band_cp_wait_all();
                __syncwarp();
            }
        };
        auto nothing = [] {};

        if (warp > 0 && wb + 1 < N) fetch_row(wb + 1);
        __syncthreads();
        if (warp == 0) factor_diag(0);
        __syncthreads();
        // with a body bandwidth wb >= 1 (a connected component of two or more
        // bodies), every column but the last has nk >= 1 blocks below the diagonal
        columns(0, ncol1);
        if (!split) {
            if (warp == 0) backward(N - 1, -1, nothing);
            band_cluster_arrive(); band_cluster_wait();
            band_cluster_arrive(); band_cluster_wait();
        } else if (crank == 1) {
            // hand S (positions ncol1..N-1, the separator in reverse order)
            // to CTA 0 in this sub-component's unused factor slots: block
            // (p, q) at (p BAND_W + p - q), its right-hand side at Y + 12 p
            for (int e = tid; e < wb * BAND_W * 144; e += blockDim.x) {
                const int p = ncol1 + e / (BAND_W * 144), d = (e / 144) % BAND_W, x = e % 144;
                if (p - d >= ncol1) L[((long)p * BAND_W + d) * 144 + x] = slot(p, p - d)[x];
            }
            for (int e = tid; e < wb * 12; e += blockDim.x) Y[(long)(ncol1 + e / 12) * 12 + e % 12] = rhs[((ncol1 + e / 12) % BAND_W) * 12 + e % 12];
            __threadfence();
            band_cluster_arrive(); band_cluster_wait();       // S handed over
            band_cluster_arrive(); band_cluster_wait();       // S solved by CTA 0
            if (warp == 0) {
                // x of the separator from du, then the backward half
                for (int e = lane; e < wb * 12; e += 32) {
                    const int p = ncol1 + e / 12;
                    xs[(p % BAND_W) * 12 + e % 12] = __ldcg(du + 12L * ord[p] + e % 12);
                }
                __syncwarp();
                backward(ncol1 - 1, -1, nothing);
            }
        } else {
            band_cluster_arrive(); band_cluster_wait();       // CTA 1's half of S is in global memory
            // S = W0 + W1 - A_SS: window row i (forward position) takes block
            // (i, j) of CTA 1 as its transposed reverse block (pj, pi),
            // pi = Nt - 1 - i with Nt = m + N1 the component size
            const int ncb = cptr[cb + 1] - cptr[cb];
            const double* L1 = Lg + loff[cb] * 144;
            const double* Y1 = Lg + ltot * 144 + (loff[cb] / BAND_W) * 12;
            const int nt1 = msplit + ncb - 1;                 // forward position i <-> reverse position nt1 - i
            for (int e = tid; e < wb * wb * 144; e += blockDim.x) {
                const int i = msplit + e / (wb * 144), j = msplit + (e / 144) % wb, x = e % 144;
                if (j > i) continue;
                const int rr = x / 12, c = x % 12, pi = nt1 - i, pj = nt1 - j;
                const double w1 = __ldcg(L1 + ((long)pj * BAND_W + (pj - pi)) * 144 + c * 12 + rr);
                slot(i, j)[x] += w1 - A[((long)i * BAND_W + (i - j)) * 144 + x];
            }
            for (int e = tid; e < wb * 12; e += blockDim.x) {
                const int i = msplit + e / 12, rr = e % 12;
                rhs[(i % BAND_W) * 12 + rr] += __ldcg(Y1 + (long)(nt1 - i) * 12 + rr) - g[12L * ord[i] + rr];
            }
            __syncthreads();
            if (warp == 0) factor_diag(msplit);
            __syncthreads();
            columns(msplit, N);
            if (warp == 0) {
                backward(N - 1, msplit, [&] { __threadfence(); band_cluster_arrive(); });
            } else {
                band_cluster_arrive();
            }
            band_cluster_wait();
        }
        __syncthreads();
    }
}

struct DenseState {
    cusolverDnHandle_t h = nullptr;
    void* A = nullptr; size_t A_bytes = 0;
    void* rhs = nullptr; size_t rhs_bytes = 0;
    void* work = nullptr; size_t work_bytes = 0; int work_n = 0;
    int* ipiv = nullptr;
    int* info = nullptr;                             // [0] small-component status, then 2 per large component
    long long* comp_d = nullptr;                     // per large component: offset | rhs offset | n
    int* imap_d = nullptr; int* imap_h = nullptr;    // bmap | blocal | sptr | sbody | band cptr | bw | order
    long long* loff_d = nullptr; long long* loff_h = nullptr;   // band factor offsets (blocks)
    void* Lg = nullptr; size_t Lg_bytes = 0;         // band factors
    void* Ab = nullptr;                              // band blocks gathered in component order (Lg_bytes)
    std::vector<unsigned long long> keys;
    std::vector<int> done, parent, size, root, bmap, fill;
    std::vector<int> adj_ptr, adj, pos, deg, members, mptr, bfs;
    bool smem_set[2] = {false, false};
    bool band_smem_set = false;
};
static DenseState* ds_of(Engine* E) { return reinterpret_cast<DenseState*>(E->dense_state); }

constexpr int MAX_LARGE_COMPONENTS = 16;

void eng_dense_free(Engine* E) {
    DenseState* D = ds_of(E);
    if (!D) return;
    if (D->h) cusolverDnDestroy(D->h);
    void* ps[] = {D->A, D->rhs, D->work, D->ipiv, D->info, D->comp_d, D->imap_d, D->loff_d, D->Lg, D->Ab};
    for (void* p : ps) if (p) cudaFree(p);
    if (D->imap_h) cudaFreeHost(D->imap_h);
    if (D->loff_h) cudaFreeHost(D->loff_h);
    delete D;
    E->dense_state = nullptr;
}

// bytes of the dense matrices if every scene were one component
long long eng_dense_bytes(Engine* E) {
    long long tot = 0;
    for (int s = 0; s < E->ns; s++) {
        long long n = 12LL * (E->h_body_begin[s + 1] - E->h_body_begin[s]);
        tot += n * n;
    }
    return tot * (E->mixed ? 4 : 8);
}

static int dense_init(Engine* E) {
    if (E->dense_state) return ABD_OK;
    DenseState* D = new DenseState();
    E->dense_state = D;
    if (cusolverDnCreate(&D->h) != CUSOLVER_STATUS_SUCCESS) return E->fail(ABD_ERR_CUDA, "cusolverDnCreate");
    cusolverDnSetStream(D->h, E->stream);
    // component maps, small-component lists, band sub-components (a split
    // component's separator appears in both halves) and band jobs
    size_t ni = 10 * (size_t)E->nb + 16;
    if (cudaMalloc(&D->imap_d, sizeof(int) * ni) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc maps");
    if (cudaMallocHost(&D->imap_h, sizeof(int) * ni) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMallocHost maps");
    if (cudaMalloc(&D->loff_d, sizeof(long long) * (E->nb + 1)) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc band offsets");
    if (cudaMallocHost(&D->loff_h, sizeof(long long) * (E->nb + 1)) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMallocHost band offsets");
    if (cudaMalloc(&D->info, sizeof(int) * (2 * MAX_LARGE_COMPONENTS + 2)) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc info");
    if (cudaMalloc(&D->comp_d, sizeof(long long) * 3 * MAX_LARGE_COMPONENTS) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc comps");
    return ABD_OK;
}

template <class T>
static int dense_reserve(Engine* E, DenseState* D, size_t a_elems, size_t rhs_elems, int nmax) {
    size_t es = sizeof(T);
    if (a_elems * es > D->A_bytes) {
        if (D->A) cudaFree(D->A);
        D->A_bytes = std::max(a_elems * es * 2, (size_t)1 << 20);
        if (cudaMalloc(&D->A, D->A_bytes) != cudaSuccess) { D->A = nullptr; D->A_bytes = 0; return E->fail(ABD_ERR_CUDA, "cudaMalloc dense matrices"); }
    }
    if (rhs_elems * es > D->rhs_bytes) {
        if (D->rhs) cudaFree(D->rhs);
        D->rhs_bytes = rhs_elems * es + 4096;
        if (cudaMalloc(&D->rhs, D->rhs_bytes) != cudaSuccess) { D->rhs = nullptr; D->rhs_bytes = 0; return E->fail(ABD_ERR_CUDA, "cudaMalloc dense rhs"); }
    }
    if (nmax > D->work_n || D->work_bytes % es) {
        // room for components up to twice this size (at most the whole handle)
        nmax = std::min(std::max(2 * nmax, 384), std::max(12 * E->nb, nmax));
        if (D->work) cudaFree(D->work);
        if (D->ipiv) cudaFree(D->ipiv);
        D->work = nullptr; D->ipiv = nullptr;
        int lw1 = 0, lw2 = 0;
        if constexpr (sizeof(T) == 4) {
            cusolverDnSpotrf_bufferSize(D->h, CUBLAS_FILL_MODE_LOWER, nmax, (float*)D->A, nmax, &lw1);
            cusolverDnSgetrf_bufferSize(D->h, nmax, nmax, (float*)D->A, nmax, &lw2);
        } else {
            cusolverDnDpotrf_bufferSize(D->h, CUBLAS_FILL_MODE_LOWER, nmax, (double*)D->A, nmax, &lw1);
            cusolverDnDgetrf_bufferSize(D->h, nmax, nmax, (double*)D->A, nmax, &lw2);
        }
        D->work_bytes = ((size_t)std::max(lw1, lw2) + 32) * es;
        D->work_n = nmax;
        if (cudaMalloc(&D->work, D->work_bytes) != cudaSuccess || cudaMalloc(&D->ipiv, sizeof(int) * nmax) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMalloc cusolver work");
    }
    return ABD_OK;
}

template <class T>
static cusolverStatus_t potrf(DenseState* D, int n, T* A, T* work, int lwork, int* info) {
    if constexpr (sizeof(T) == 8) return cusolverDnDpotrf(D->h, CUBLAS_FILL_MODE_LOWER, n, A, n, work, lwork, info);
    else return cusolverDnSpotrf(D->h, CUBLAS_FILL_MODE_LOWER, n, A, n, work, lwork, info);
}
template <class T>
static cusolverStatus_t potrs(DenseState* D, int n, T* A, T* x, int* info) {
    if constexpr (sizeof(T) == 8) return cusolverDnDpotrs(D->h, CUBLAS_FILL_MODE_LOWER, n, 1, A, n, x, n, info);
    else return cusolverDnSpotrs(D->h, CUBLAS_FILL_MODE_LOWER, n, 1, A, n, x, n, info);
}
template <class T>
static cusolverStatus_t lu_solve(DenseState* D, int n, T* A, T* x, T* work, int* info) {
    cusolverStatus_t cs;
    if constexpr (sizeof(T) == 8) {
        cs = cusolverDnDgetrf(D->h, n, n, A, n, work, D->ipiv, info);
        if (cs == CUSOLVER_STATUS_SUCCESS) cs = cusolverDnDgetrs(D->h, CUBLAS_OP_N, n, 1, A, n, D->ipiv, x, n, info + 1);
    } else {
        cs = cusolverDnSgetrf(D->h, n, n, A, n, work, D->ipiv, info);
        if (cs == CUSOLVER_STATUS_SUCCESS) cs = cusolverDnSgetrs(D->h, CUBLAS_OP_N, n, 1, A, n, D->ipiv, x, n, info + 1);
    }
    return cs;
}

// Returns 1 in *fallback when there are more large components than
// MAX_LARGE_COMPONENTS or their matrices would exceed 4 GiB (the caller then
// runs the Krylov solver).
template <class T>
static int dense_solve_t(Engine* E, int* iters, int* fallback) {
    *fallback = 0;
    int rc = eng_asm_wait(E);
    if (rc) return rc;
    if ((rc = dense_init(E))) return rc;
    DenseState* D = ds_of(E);
    cudaStream_t st = E->stream;
    const int* ndone = E->sci + SI_DONE * E->ns;
    const int nb = E->nb;
    // block pattern and done flags to the host (already there when the
    // assembly copied them within its sync)
    const int nk = E->nnzb_host;
    D->keys.resize(std::max(nk, 1));
    D->done.resize(E->ns);
    if (E->keys_host && nk <= E->h_ukeys_cap) {
        if (nk > 0) memcpy(D->keys.data(), E->h_ukeys, sizeof(unsigned long long) * nk);
        memcpy(D->done.data(), E->h_done, sizeof(int) * E->ns);
    } else {
        if (nk > 0) CUDA_TRY(cudaMemcpyAsync(D->keys.data(), E->ukeys, sizeof(unsigned long long) * nk, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaMemcpyAsync(D->done.data(), ndone, sizeof(int) * E->ns, cudaMemcpyDeviceToHost, st));
        CUDA_TRY(eng_stream_sync(E));
    }
    E->keys_host = false;
    // union-find over bodies, joined by off-diagonal blocks
    std::vector<int>& parent = D->parent;
    parent.resize(nb);
    for (int b = 0; b < nb; b++) parent[b] = b;
    auto find = [&](int x) { while (parent[x] != x) { parent[x] = parent[parent[x]]; x = parent[x]; } return x; };
    for (int k = 0; k < nk; k++) {
        unsigned long long key = D->keys[k];
        if (key == ~0ull) continue;
        int r = (int)(key / nb), c = (int)(key % nb);
        if (r == c) continue;
        int a = find(r), b2 = find(c);
        if (a != b2) { if (a < b2) parent[b2] = a; else parent[a] = b2; }
    }
    D->size.assign(nb, 0);
    for (int b = 0; b < nb; b++) D->size[find(b)]++;
    const bool projected = E->P.hess_mode == ABD_HESS_PROJECTED;
    // body adjacency (off-diagonal blocks, both directions are stored)
    D->adj_ptr.assign(nb + 1, 0);
    for (int k = 0; k < nk; k++) {
        unsigned long long key = D->keys[k];
        if (key == ~0ull) continue;
        int r = (int)(key / nb), c = (int)(key % nb);
        if (r != c) D->adj_ptr[r + 1]++;
    }
    for (int b = 0; b < nb; b++) D->adj_ptr[b + 1] += D->adj_ptr[b];
    D->adj.resize(std::max(D->adj_ptr[nb], 1));
    {
        std::vector<int> at(D->adj_ptr.begin(), D->adj_ptr.end() - 1);
        for (int k = 0; k < nk; k++) {           // keys are sorted: neighbours ascending
            unsigned long long key = D->keys[k];
            if (key == ~0ull) continue;
            int r = (int)(key / nb), c = (int)(key % nb);
            if (r != c) D->adj[at[r]++] = c;
        }
    }
    // members of every multi-body component of a scene still iterating
    D->mptr.assign(nb + 1, 0);
    for (int b = 0; b < nb; b++) { int r = find(b); if (D->size[r] >= 2 && !D->done[E->h_bscene[b]]) D->mptr[r + 1]++; }
    for (int b = 0; b < nb; b++) D->mptr[b + 1] += D->mptr[b];
    D->members.resize(std::max(D->mptr[nb], 1));
    {
        std::vector<int> at(D->mptr.begin(), D->mptr.end() - 1);
        for (int b = 0; b < nb; b++) { int r = find(b); if (D->size[r] >= 2 && !D->done[E->h_bscene[b]]) D->members[at[r]++] = b; }
    }
    // reverse Cuthill-McKee order of a component (BFS from a minimum-degree
    // body, neighbours by ascending degree, reversed) and its body bandwidth
    D->pos.assign(nb, -1);
    auto rcm = [&](int r, std::vector<int>& out) {
        const int* m = D->members.data() + D->mptr[r];
        int n = D->mptr[r + 1] - D->mptr[r];
        auto degree = [&](int b) { return D->adj_ptr[b + 1] - D->adj_ptr[b]; };
        int start = m[0];
        for (int i = 1; i < n; i++) if (degree(m[i]) < degree(start)) start = m[i];
        out.clear(); out.push_back(start); D->pos[start] = 0;
        std::vector<int> nb_;
        for (size_t h = 0; h < out.size(); h++) {
            int u = out[h];
            nb_.clear();
            for (int e = D->adj_ptr[u]; e < D->adj_ptr[u + 1]; e++) if (D->pos[D->adj[e]] < 0) nb_.push_back(D->adj[e]);
            std::sort(nb_.begin(), nb_.end(), [&](int a, int b) { return degree(a) != degree(b) ? degree(a) < degree(b) : a < b; });
            for (int v : nb_) if (D->pos[v] < 0) { D->pos[v] = 0; out.push_back(v); }
        }
        std::reverse(out.begin(), out.end());
        for (int i = 0; i < (int)out.size(); i++) D->pos[out[i]] = i;
        int bw = 0;
        for (int u : out)
            for (int e = D->adj_ptr[u]; e < D->adj_ptr[u + 1]; e++) bw = std::max(bw, std::abs(D->pos[u] - D->pos[D->adj[e]]));
        return bw;
    };
    // components of scenes still iterating: band components (one CTA each,
    // Cholesky), small ones (one CTA each, dense in shared memory) and large
    // ones (cuSOLVER)
    D->root.assign(nb, -1);
    D->bmap.assign(nb, -1);
    std::vector<int> small_root, large_n, band_cptr(1, 0), band_bw, band_order, ord, band_jobs;
    std::vector<long long> large_off, large_rhs;
    long long aoff = 0, roff = 0, lblocks = 0;
    int nmax_large = 0, nmax_small = 0, small_bodies = 0, nband = 0, ncomp_band = 0;
    // a band sub-component: bodies in factor order, body bandwidth
    auto band_sub = [&](const int* bodies, int len, int bw) {
        D->loff_h[nband] = lblocks;
        lblocks += (long long)len * BAND_W;
        band_order.insert(band_order.end(), bodies, bodies + len);
        band_cptr.push_back((int)band_order.size());
        band_bw.push_back(bw);
        return nband++;
    };
    for (int b = 0; b < nb; b++) {
        int r = find(b), sz = D->size[r];
        if (sz < 2 || D->done[E->h_bscene[b]]) continue;
        // FP32 roundings of a stiff projected Hessian can make it indefinite
        // (the band Cholesky has no pivoting), so the band path runs in FP64
        // mode only; there it takes every component of body bandwidth <= 8,
        // large ones split between the two CTAs of a cluster, and cuSOLVER
        // only the components of wider bandwidth
        if (D->root[r] == -1 && projected && !E->mixed) {
            int bw = rcm(r, ord);
            if (bw >= 1 && bw <= BAND_MAX && sz <= BAND_ORD_MAX) {
                D->root[r] = -10 - ncomp_band++;          // marks a band component
                const int m = band_split_point(sz, bw);
                if (m > 0) {
                    // bodies [0, m + bw) forward, [m, sz) from the far end
                    const int ct = band_sub(ord.data(), m + bw, bw);
                    std::vector<int> rev(ord.rbegin(), ord.rend() - m);
                    const int cb = band_sub(rev.data(), sz - m, bw);
                    band_jobs.insert(band_jobs.end(), {ct, cb, m});
                } else {
                    const int ct = band_sub(ord.data(), sz, bw);
                    band_jobs.insert(band_jobs.end(), {ct, -1, sz});
                }
            }
        }
        if (D->root[r] <= -10) { D->bmap[b] = -3; continue; }
        if (D->root[r] < 0) {
            if (sz <= SMALL_MAX_BODIES) {
                D->root[r] = (int)small_root.size();
                small_root.push_back(r);
                nmax_small = std::max(nmax_small, 12 * sz);
            } else {
                if ((int)large_n.size() >= MAX_LARGE_COMPONENTS) { *fallback = 1; E->krylov_fallbacks++; return ABD_OK; }
                D->root[r] = (int)large_n.size();
                int n = 12 * sz;
                large_n.push_back(n); large_off.push_back(aoff); large_rhs.push_back(roff);
                aoff += (long long)n * n; roff += n;
                nmax_large = std::max(nmax_large, n);
            }
        }
        if (sz <= SMALL_MAX_BODIES) { D->bmap[b] = -2; small_bodies++; }
        else D->bmap[b] = D->root[r];
    }
    const int nsmall = (int)small_root.size(), nlarge = (int)large_n.size();
    E->comp_band += ncomp_band; E->comp_small += nsmall; E->comp_large += nlarge;

    if (aoff * (long long)sizeof(T) > (4LL << 30)) { *fallback = 1; E->krylov_fallbacks++; return ABD_OK; }
    // local body index inside its component (body order) and the small
    // components' body lists, packed into one upload
    int* h = D->imap_h;
    int* h_bmap = h; int* h_blocal = h + nb; int* h_sptr = h + 2 * nb; int* h_sbody = h_sptr + nsmall + 1;
    D->fill.assign(nsmall + nlarge, 0);
    h_sptr[0] = 0;
    for (int c = 0; c < nsmall; c++) h_sptr[c + 1] = h_sptr[c] + D->size[small_root[c]];
    for (int b = 0; b < nb; b++) {
        int m = D->bmap[b];
        h_bmap[b] = m;
        h_blocal[b] = 0;
        if (m == -2) {
            int c = D->root[find(b)];
            int l = D->fill[c]++;
            h_blocal[b] = l;
            h_sbody[h_sptr[c] + l] = b;
        } else if (m >= 0) {
            h_blocal[b] = D->fill[nsmall + m]++;
        }
    }
    // band components: cptr | bandwidth | bodies in order
    int* h_bcptr = h_sbody + small_bodies;
    int* h_bbw = h_bcptr + nband + 1;
    int* h_bord = h_bbw + nband;
    for (int c = 0; c <= nband; c++) h_bcptr[c] = band_cptr[c];
    for (int c = 0; c < nband; c++) h_bbw[c] = band_bw[c];
    for (size_t i = 0; i < band_order.size(); i++) h_bord[i] = band_order[i];
    int* h_pcomp = h_bord + band_order.size();
    for (int c = 0; c < nband; c++)
        for (int q = band_cptr[c]; q < band_cptr[c + 1]; q++) h_pcomp[q] = c;
    int* h_jobs = h_pcomp + band_order.size();
    for (size_t i = 0; i < band_jobs.size(); i++) h_jobs[i] = band_jobs[i];
    const size_t nints = 2 * (size_t)nb + nsmall + 1 + small_bodies + 2 * (size_t)nband + 1 + 2 * band_order.size() +
                         band_jobs.size();
    CUDA_TRY(cudaMemcpyAsync(D->imap_d, h, sizeof(int) * nints, cudaMemcpyHostToDevice, st));
    const int* d_bmap = D->imap_d; const int* d_blocal = D->imap_d + nb;
    const int* d_sptr = D->imap_d + 2 * nb; const int* d_sbody = d_sptr + nsmall + 1;
    CUDA_TRY(cudaMemsetAsync(D->info, 0, sizeof(int), st));      // status of the band and small kernels
    if (nband > 0) {
        const int* d_bcptr = d_sbody + small_bodies;
        const int* d_bbw = d_bcptr + nband + 1;
        const int* d_bord = d_bbw + nband;
        size_t need = ((size_t)lblocks * 144 + 12 * band_order.size()) * sizeof(double);
        if (need > D->Lg_bytes) {
            if (D->Lg) cudaFree(D->Lg);
            if (D->Ab) cudaFree(D->Ab);
            D->Ab = nullptr;
            D->Lg_bytes = std::max(2 * need, (size_t)1 << 20);
            if (cudaMalloc(&D->Lg, D->Lg_bytes) != cudaSuccess || cudaMalloc(&D->Ab, D->Lg_bytes) != cudaSuccess) {
                D->Lg_bytes = 0;
                return E->fail(ABD_ERR_CUDA, "cudaMalloc band factors");
            }
        }
        CUDA_TRY(cudaMemcpyAsync(D->loff_d, D->loff_h, sizeof(long long) * nband, cudaMemcpyHostToDevice, st));
        const size_t smem = (size_t)band_smem_doubles() * sizeof(double);
        if (!D->band_smem_set) {
            CUDA_TRY(cudaFuncSetAttribute(k_band_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            D->band_smem_set = true;
        }
        const int* d_pcomp = d_bord + band_order.size();
        const int* d_jobs = d_pcomp + band_order.size();
        const int npos = (int)band_order.size(), njobs = (int)band_jobs.size() / 3;
        k_band_gather<T><<<grid_for(32L * npos * BAND_W), 256, 0, st>>>(npos, d_pcomp, d_bcptr, d_bord, d_bbw, D->loff_d,
                                                                       E->row_ptr, E->bcol, (const T*)E->vals, (double*)D->Ab);
        E->launches++;
        int ph = phase_begin(E, PH_BAND);
        // one cluster of two CTAs per job
        k_band_solve<<<2 * njobs, BAND_THREADS, smem, st>>>(njobs, d_jobs, d_bcptr, d_bord, d_bbw, D->loff_d,
                                                            (const double*)D->Ab, lblocks, E->g, (double*)D->Lg, E->du,
                                                            D->info);
        // per component: band blocks read, factor written and read back,
        // g read, y and du written and read
        double bytes = 0;
        for (int c = 0; c < nband; c++)
            bytes += (band_cptr[c + 1] - band_cptr[c]) * ((band_bw[c] + 1) * 144.0 * sizeof(double) * 3 + 96.0 * 4);
        phase_end(E, ph, bytes);
        E->launches++;
    }
    if (nsmall > 0) {
        size_t smem = ((size_t)nmax_small * (nmax_small + 1) + nmax_small) * sizeof(T);
        if (!D->smem_set[sizeof(T) == 8]) {
            const size_t nm = 12 * SMALL_MAX_BODIES;
            CUDA_TRY(cudaFuncSetAttribute(k_small_solve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)((nm * (nm + 1) + nm) * sizeof(T))));
            D->smem_set[sizeof(T) == 8] = true;
        }
        k_small_solve<T><<<nsmall, SMALL_THREADS, smem, st>>>(nsmall, d_sptr, d_sbody, d_blocal, E->row_ptr, E->bcol,
                                                              (const T*)E->vals, E->g, projected ? 1 : 0, E->du, D->info);
        E->launches++;
    }
    T* x = nullptr;
    if (nlarge > 0) {
        if ((rc = dense_reserve<T>(E, D, (size_t)aoff, (size_t)roff, nmax_large))) return rc;
        std::vector<long long> comp(3 * nlarge);
        for (int c = 0; c < nlarge; c++) { comp[c] = large_off[c]; comp[nlarge + c] = large_rhs[c]; comp[2 * nlarge + c] = large_n[c]; }
        CUDA_TRY(cudaMemcpyAsync(D->comp_d, comp.data(), sizeof(long long) * 3 * nlarge, cudaMemcpyHostToDevice, st));
        const long long* d_off = D->comp_d; const long long* d_rhs = D->comp_d + nlarge; const long long* d_n = D->comp_d + 2 * nlarge;
        T* A = (T*)D->A;
        x = (T*)D->rhs;
        CUDA_TRY(cudaMemsetAsync(A, 0, sizeof(T) * (size_t)aoff, st));
        k_blocks_to_dense<T><<<grid_for(16L * nb), 256, 0, st>>>(nb, E->row_ptr, E->bcol, (const T*)E->vals, d_bmap,
                                                                d_blocal, d_off, d_n, -1, A);
        k_rhs_gather<T><<<grid_for(12L * nb), 256, 0, st>>>(nb, E->g, d_bmap, d_blocal, d_rhs, x);
        E->launches += 2;
        T* work = (T*)D->work;
        int lwork = (int)(D->work_bytes / sizeof(T));
        std::vector<char> use_lu(nlarge, projected ? 0 : 1);
        if (projected) {
            for (int c = 0; c < nlarge; c++)
                if (potrf<T>(D, large_n[c], A + large_off[c], work, lwork, D->info + 2 + 2 * c) != CUSOLVER_STATUS_SUCCESS)
                    return E->fail(ABD_ERR_CUDA, "cusolver potrf");
            std::vector<int> info(2 * nlarge);
            CUDA_TRY(cudaMemcpyAsync(info.data(), D->info + 2, sizeof(int) * 2 * nlarge, cudaMemcpyDeviceToHost, st));
            CUDA_TRY(eng_stream_sync(E));
            for (int c = 0; c < nlarge; c++) {
                if (info[2 * c] != 0) {
                    // not positive definite after all: rebuild this component for LU
                    use_lu[c] = 1;
                    CUDA_TRY(cudaMemsetAsync(A + large_off[c], 0, sizeof(T) * (size_t)large_n[c] * large_n[c], st));
                    k_blocks_to_dense<T><<<grid_for(16L * nb), 256, 0, st>>>(nb, E->row_ptr, E->bcol, (const T*)E->vals, d_bmap,
                                                                            d_blocal, d_off, d_n, c, A);
                    E->launches++;
                } else if (potrs<T>(D, large_n[c], A + large_off[c], x + large_rhs[c], D->info + 3 + 2 * c) != CUSOLVER_STATUS_SUCCESS) {
                    return E->fail(ABD_ERR_CUDA, "cusolver potrs");
                }
            }
        }
        for (int c = 0; c < nlarge; c++)
            if (use_lu[c] && lu_solve<T>(D, large_n[c], A + large_off[c], x + large_rhs[c], work, D->info + 2 + 2 * c) != CUSOLVER_STATUS_SUCCESS)
                return E->fail(ABD_ERR_CUDA, "cusolver getrf/getrs");
    }
    k_du_scatter<T><<<grid_for(12L * nb), 256, 0, st>>>(nb, E->g, d_bmap, d_blocal, nlarge ? D->comp_d + nlarge : nullptr, x,
                                                       (const T*)E->dinv, E->bscene, ndone, E->du);
    E->launches++;
    *iters = 1;
    return ABD_OK;
}

int eng_solve_direct(Engine* E, int* iters, int* fallback) {
    if (E->mixed) return dense_solve_t<float>(E, iters, fallback);
    return dense_solve_t<double>(E, iters, fallback);
}
