// dense.cu — direct solve of the Newton system, one dense factorization per
// scene (the reference's solver_config != "cg" branch, abd.py:637-654, which
// factors the assembled matrix with a cuSOLVER wrapper).
//
// The 12x12 body blocks of each scene are scattered into a dense
// column-major matrix (16 lanes per body row, the Krylov kernels' mapping),
// then factored with cuSOLVER: Cholesky when the Hessian is PSD-projected,
// LU with partial pivoting for the reference's indefinite Hessian (or when
// Cholesky reports a non-positive pivot).  Mixed precision factors in FP32.
#include "engine.cuh"
#include <cusolverDn.h>
#include <algorithm>

template <class T>
__global__ void k_blocks_to_dense(int nb, const int* __restrict__ row_ptr, const int* __restrict__ bcol,
                                  const T* __restrict__ vals, const int* __restrict__ bscene,
                                  const int* __restrict__ sc_body_begin, const long long* __restrict__ dense_off,
                                  const int* __restrict__ ndone, T* dense) {
    for (long base = (long)blockIdx.x * blockDim.x; base < (long)nb * 16; base += (long)gridDim.x * blockDim.x) {
        long t = base + threadIdx.x;
        int b = (int)(t / 16), l = (int)(t % 16);
        if (b >= nb || l >= 12) continue;
        int s = bscene[b];
        if (ndone[s]) continue;
        int b0 = sc_body_begin[s];
        long n = 12L * (sc_body_begin[s + 1] - b0);
        T* A = dense + dense_off[s];
        long row = 12L * (b - b0) + l;
        for (int k = row_ptr[b]; k < row_ptr[b + 1]; k++) {
            long colb = 12L * (bcol[k] - b0);
            const T* V = vals + (long)k * 144 + l;
#pragma unroll
            for (int j = 0; j < 12; j++) A[(colb + j) * n + row] = V[j * 12];
        }
    }
}
template <class T>
__global__ void k_rhs_cast(int n, const double* __restrict__ g, T* x) { GS_LOOP(i, n) x[i] = (T)g[i]; }
template <class T>
__global__ void k_rhs_back(int n, const T* __restrict__ x, const int* __restrict__ bscene, const int* __restrict__ ndone,
                           double* du) {
    GS_LOOP(i, n) { if (!ndone[bscene[i / 12]]) du[i] = (double)x[i]; }
}

struct DenseState {
    cusolverDnHandle_t h = nullptr;
    void* A = nullptr; size_t A_bytes = 0;
    void* work = nullptr; size_t work_bytes = 0;
    int* ipiv = nullptr; int ipiv_n = 0;
    int* info = nullptr;
    long long* off_d = nullptr;
    std::vector<long long> off;
    std::vector<int> n;
    void* rhs = nullptr;
};
static DenseState* ds_of(Engine* E) { return reinterpret_cast<DenseState*>(E->dense_state); }

void eng_dense_free(Engine* E) {
    DenseState* D = ds_of(E);
    if (!D) return;
    if (D->h) cusolverDnDestroy(D->h);
    void* ps[] = {D->A, D->work, D->ipiv, D->info, D->off_d, D->rhs};
    for (void* p : ps) if (p) cudaFree(p);
    delete D;
    E->dense_state = nullptr;
}

// bytes the dense path needs (matrices only)
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
    long long tot = 0;
    int nmax = 0;
    for (int s = 0; s < E->ns; s++) {
        int n = 12 * (E->h_body_begin[s + 1] - E->h_body_begin[s]);
        D->off.push_back(tot); D->n.push_back(n);
        tot += (long long)n * n;
        nmax = std::max(nmax, n);
    }
    size_t es = E->mixed ? 4 : 8;
    D->A_bytes = (size_t)tot * es;
    if (cudaMalloc(&D->A, D->A_bytes) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc dense matrices");
    if (cudaMalloc(&D->off_d, sizeof(long long) * E->ns) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc");
    cudaMemcpy(D->off_d, D->off.data(), sizeof(long long) * E->ns, cudaMemcpyHostToDevice);
    if (cudaMalloc(&D->ipiv, sizeof(int) * nmax) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc ipiv");
    D->ipiv_n = nmax;
    if (cudaMalloc(&D->info, sizeof(int) * 2) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc info");
    if (cudaMalloc(&D->rhs, es * 12 * (size_t)E->nb) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc rhs");
    // workspace for the largest scene, both factorizations
    int lw1 = 0, lw2 = 0;
    if (E->mixed) {
        cusolverDnSpotrf_bufferSize(D->h, CUBLAS_FILL_MODE_LOWER, nmax, (float*)D->A, std::max(nmax, 1), &lw1);
        cusolverDnSgetrf_bufferSize(D->h, nmax, nmax, (float*)D->A, std::max(nmax, 1), &lw2);
    } else {
        cusolverDnDpotrf_bufferSize(D->h, CUBLAS_FILL_MODE_LOWER, nmax, (double*)D->A, std::max(nmax, 1), &lw1);
        cusolverDnDgetrf_bufferSize(D->h, nmax, nmax, (double*)D->A, std::max(nmax, 1), &lw2);
    }
    D->work_bytes = (size_t)std::max(lw1, lw2) * es + 256;
    if (cudaMalloc(&D->work, D->work_bytes) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc cusolver work");
    return ABD_OK;
}

template <class T>
static int dense_solve_t(Engine* E, int* iters) {
    int rc = dense_init(E);
    if (rc) return rc;
    DenseState* D = ds_of(E);
    cudaStream_t st = E->stream;
    const int* ndone = E->sci + SI_DONE * E->ns;
    // which scenes still iterate (host copy of the done flags)
    std::vector<int> done(E->ns);
    CUDA_TRY(cudaMemcpyAsync(done.data(), ndone, sizeof(int) * E->ns, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    CUDA_TRY(cudaMemsetAsync(D->A, 0, D->A_bytes, st));
    T* A = (T*)D->A;
    k_blocks_to_dense<T><<<grid_for(16L * E->nb), 256, 0, st>>>(E->nb, E->row_ptr, E->bcol, (const T*)E->vals, E->bscene,
                                                               E->sc_body_begin, D->off_d, ndone, A);
    T* x = (T*)D->rhs;
    k_rhs_cast<T><<<grid_for(12L * E->nb), 256, 0, st>>>(12 * E->nb, E->g, x);
    E->launches += 2;
    bool projected = E->P.hess_mode == ABD_HESS_PROJECTED;
    std::vector<int> use_lu(E->ns, projected ? 0 : 1);
    T* work = (T*)D->work;
    int lwork = (int)(D->work_bytes / sizeof(T));
    for (int pass = 0; pass < 2; pass++) {
        bool any = false;
        for (int s = 0; s < E->ns; s++) {
            if (done[s] || D->n[s] == 0) continue;
            if (pass == 1 && !use_lu[s]) continue;
            any = true;
            int n = D->n[s];
            T* As = A + D->off[s];
            T* xs = x + 12L * E->h_body_begin[s];
            cusolverStatus_t cs;
            if (!use_lu[s]) {
                if constexpr (sizeof(T) == 8) {
                    cs = cusolverDnDpotrf(D->h, CUBLAS_FILL_MODE_LOWER, n, (double*)As, n, (double*)work, lwork, D->info);
                    if (cs == CUSOLVER_STATUS_SUCCESS)
                        cs = cusolverDnDpotrs(D->h, CUBLAS_FILL_MODE_LOWER, n, 1, (double*)As, n, (double*)xs, n, D->info + 1);
                } else {
                    cs = cusolverDnSpotrf(D->h, CUBLAS_FILL_MODE_LOWER, n, (float*)As, n, (float*)work, lwork, D->info);
                    if (cs == CUSOLVER_STATUS_SUCCESS)
                        cs = cusolverDnSpotrs(D->h, CUBLAS_FILL_MODE_LOWER, n, 1, (float*)As, n, (float*)xs, n, D->info + 1);
                }
                if (cs != CUSOLVER_STATUS_SUCCESS) return E->fail(ABD_ERR_CUDA, "cusolver potrf/potrs");
                int info = 0;
                CUDA_TRY(cudaMemcpyAsync(&info, D->info, sizeof(int), cudaMemcpyDeviceToHost, st));
                CUDA_TRY(cudaStreamSynchronize(st));
                if (info != 0) use_lu[s] = 1;     // not positive definite: redo with LU in pass 1
            } else {
                if constexpr (sizeof(T) == 8) {
                    cs = cusolverDnDgetrf(D->h, n, n, (double*)As, n, (double*)work, D->ipiv, D->info);
                    if (cs == CUSOLVER_STATUS_SUCCESS)
                        cs = cusolverDnDgetrs(D->h, CUBLAS_OP_N, n, 1, (double*)As, n, D->ipiv, (double*)xs, n, D->info + 1);
                } else {
                    cs = cusolverDnSgetrf(D->h, n, n, (float*)As, n, (float*)work, D->ipiv, D->info);
                    if (cs == CUSOLVER_STATUS_SUCCESS)
                        cs = cusolverDnSgetrs(D->h, CUBLAS_OP_N, n, 1, (float*)As, n, D->ipiv, (float*)xs, n, D->info + 1);
                }
                if (cs != CUSOLVER_STATUS_SUCCESS) return E->fail(ABD_ERR_CUDA, "cusolver getrf/getrs");
            }
        }
        if (pass == 0) {
            // scenes that fell back to LU need their matrix and right-hand side again
            bool redo = false;
            for (int s = 0; s < E->ns; s++) if (projected && use_lu[s] && !done[s]) redo = true;
            if (!redo) break;
            std::vector<int> mask(E->ns, 1);
            for (int s = 0; s < E->ns; s++) if (use_lu[s] && !done[s]) mask[s] = 0;
            int* dmask = E->sci + SI_NACT * E->ns;
            CUDA_TRY(cudaMemcpyAsync(dmask, mask.data(), sizeof(int) * E->ns, cudaMemcpyHostToDevice, st));
            // right-hand sides of the redone scenes only
            for (int s = 0; s < E->ns; s++) if (!mask[s]) {
                int n = D->n[s];
                CUDA_TRY(cudaMemsetAsync(A + D->off[s], 0, sizeof(T) * (size_t)n * n, st));
            }
            k_blocks_to_dense<T><<<grid_for(16L * E->nb), 256, 0, st>>>(E->nb, E->row_ptr, E->bcol, (const T*)E->vals,
                                                                       E->bscene, E->sc_body_begin, D->off_d, dmask, A);
            for (int s = 0; s < E->ns; s++) if (!mask[s]) {
                int n = D->n[s];
                k_rhs_cast<T><<<grid_for(n), 256, 0, st>>>(n, E->g + 12L * E->h_body_begin[s], x + 12L * E->h_body_begin[s]);
            }
            (void)any;
        }
    }
    k_rhs_back<T><<<grid_for(12L * E->nb), 256, 0, st>>>(12 * E->nb, x, E->bscene, ndone, E->du);
    E->launches++;
    *iters = 1;
    return ABD_OK;
}

int eng_solve_direct(Engine* E, int* iters) {
    if (E->mixed) return dense_solve_t<float>(E, iters);
    return dense_solve_t<double>(E, iters);
}
