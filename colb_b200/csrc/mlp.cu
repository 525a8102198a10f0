// mlp.cu — the learned warm start's network (no counterpart in the
// reference): 48 -> 256 -> 256 -> 256 -> 12, GELU, BF16 weights and
// activations, FP32 accumulation.
//
// Inference (every step of warm_start 3): one CTA of 4 warps runs 128 bodies
// through all four layers.  Layer weights are stored once in the UMMA
// canonical K-major layout (8x8 core matrices, no swizzle) and copied into
// shared memory with one bulk asynchronous copy per layer; the activations
// stay in shared memory in the same layout.  One elected thread issues
// tcgen05.mma (kind::f16, M = 128, N = 256 or 16, K = 16 per instruction)
// with the FP32 accumulator in tensor memory; the four warps read their 32
// accumulator lanes back with tcgen05.ld, add the bias, apply GELU and write
// the next layer's BF16 operand.  Every wait is bounded and reports through
// an error flag; tensor memory is freed on every path.
//
// Training: FP32 master weights, Adam; every GEMM of the forward and backward
// pass (Z = H W^T, dW = dZ^T H, dH = dZ W) on the tensor cores (tcgen05,
// BF16 operands, FP32 accumulation in tensor memory), the forward with
// BF16-rounded weights and activations like inference, MSE loss, backward
// with straight-through rounding.
#include "engine.cuh"
#include <cuda_bf16.h>

namespace {

constexpr int MI = ABD_MLP_IN, MH = ABD_MLP_HIDDEN, MO = ABD_MLP_OUT;
constexpr int K1 = 64;            // input width padded to a multiple of 16
constexpr int NO = 16;            // output width padded to the MMA's N step
// parameter blob offsets (FP32, W[out][in] row-major then bias)
constexpr int OW1 = 0, OB1 = OW1 + MH * MI, OW2 = OB1 + MH, OB2 = OW2 + MH * MH, OW3 = OB2 + MH, OB3 = OW3 + MH * MH,
              OW4 = OB3 + MH, OB4 = OW4 + MO * MH, NPARAM = OB4 + MO;
static_assert(NPARAM == ABD_MLP_NPARAM, "parameter count");
// packed BF16 weights (canonical layout), byte offsets
constexpr int PW1 = 0, PW2 = PW1 + MH * K1 * 2, PW3 = PW2 + MH * MH * 2, PW4 = PW3 + MH * MH * 2, PTOT = PW4 + NO * MH * 2;
// shared memory of the inference kernel
constexpr int S_A = 0, S_W = S_A + 128 * MH * 2, S_BAR = S_W + MH * MH * 2, S_TM = S_BAR + 16, S_TOT = S_TM + 16;
constexpr int NTHR = 128;
constexpr long WAIT_LIMIT = 1L << 22;

// element index of (r, k) in a K-major canonical tile with K columns
HD int canon(int r, int k, int K) { return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7); }

DV float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
DV float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}
DV float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

DV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor: no swizzle, K-major; lbo = byte distance of
// the two 8-column halves of a K = 16 slice, sbo = byte distance of 8-row groups
DV uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((addr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                       // descriptor version of sm_100
    return d;                                     // base offset 0, no swizzle
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128
HD uint32_t idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

DV void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
DV bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (long i = 0; i < WAIT_LIMIT; i++) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
// one bulk copy of `bytes` (multiple of 16) from global into shared memory,
// completing on `bar`
DV void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
    for (uint32_t off = 0; off < bytes; off += 32768) {
        uint32_t n = bytes - off < 32768 ? bytes - off : 32768;
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     :: "r"(dst + off), "l"((const char*)src + off), "r"(n), "r"(bar) : "memory");
    }
}
DV void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id, uint32_t acc) {
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "setp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0) : "memory");
}
DV void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}
DV void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}
DV void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Y[n][12] = net((X - mean) / std) * ystd + ymean, 128 rows per CTA.
__global__ void __launch_bounds__(NTHR, 1) k_mlp_infer(int n, const float* __restrict__ X, const float* __restrict__ norm,
                                                      const uint8_t* __restrict__ wpack, const float* __restrict__ bias,
                                                      float* __restrict__ Y, int* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(smem + S_A);
    const uint32_t aA = smem_u32(smem + S_A), aW = smem_u32(smem + S_W);
    const uint32_t bar_w = smem_u32(smem + S_BAR), bar_m = bar_w + 8;
    uint32_t* tm_holder = reinterpret_cast<uint32_t*>(smem + S_TM);
    __shared__ int status;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row0 = blockIdx.x * 128;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tm_holder)), "r"(256) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        status = 0;
        mbar_init(bar_w, 1);
        mbar_init(bar_m, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tm_holder;
    if (tid == 0) bulk_load(aW, wpack + PW1, MH * K1 * 2, bar_w);

    // layer-1 operand: normalised inputs of this CTA's rows, BF16, K = 64
    {
        int r = tid, gr = row0 + r;
        for (int k0 = 0; k0 < K1; k0 += 8) {
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                int k = k0 + j;
                float x = 0.0f;
                if (gr < n && k < MI) x = (X[(long)gr * MI + k] - norm[k]) / norm[MI + k];
                v[j] = __float2bfloat16_rn(x);
            }
            *reinterpret_cast<uint4*>(sA + canon(r, k0, K1)) = *reinterpret_cast<const uint4*>(v);
        }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    const int Ks[4] = {K1, MH, MH, MH};
    const int Ns[4] = {MH, MH, MH, NO};
    const int Poff[4] = {PW1, PW2, PW3, PW4};
    const int Boff[4] = {0, MH, 2 * MH, 3 * MH};
    for (int l = 0; l < 4; l++) {
        const int K = Ks[l], N = Ns[l];
        if (tid == 0) {
            bool ok = mbar_wait(bar_w, l & 1);
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t id = idesc(N), sbo = (uint32_t)K * 16;
                for (int kk = 0; kk < K / 16; kk++)
                    mma_bf16(tmem, sdesc(aA + kk * 256, 128, sbo), sdesc(aW + kk * 256, 128, sbo), id, kk > 0);
                mma_commit(bar_m);
                ok = mbar_wait(bar_m, l & 1);
            }
            if (!ok) { status = 1; atomicExch(err, 1); }
            else if (l < 3) {
                // the MMAs of this layer are done with the weights: fetch the next layer's
                int bytes = (l + 1 < 3) ? MH * MH * 2 : NO * MH * 2;
                bulk_load(aW, wpack + Poff[l + 1], bytes, bar_w);
            }
        }
        __syncthreads();
        if (status) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int r = warp * 32 + lane, gr = row0 + r;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        if (l < 3) {
            for (int c0 = 0; c0 < N; c0 += 32) {
                float v[32];
                tmem_ld32(trow + c0, v);
#pragma unroll
                for (int j0 = 0; j0 < 32; j0 += 8) {
                    __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                    for (int j = 0; j < 8; j++) h[j] = __float2bfloat16_rn(gelu(v[j0 + j] + bias[Boff[l] + c0 + j0 + j]));
                    *reinterpret_cast<uint4*>(sA + canon(r, c0 + j0, MH)) = *reinterpret_cast<const uint4*>(h);
                }
            }
        } else {
            float v[16];
            tmem_ld16(trow, v);
            if (gr < n) {
                const float* ym = norm + 2 * MI;
                const float* ys = norm + 2 * MI + MO;
#pragma unroll
                for (int j = 0; j < MO; j++) Y[(long)gr * MO + j] = (v[j] + bias[Boff[3] + j]) * ys[j] + ym[j];
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
    }
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(256) : "memory");
    }
}

// FP32 parameter blob -> BF16 canonical tiles + FP32 biases (output padded to 16)
__global__ void k_mlp_pack(const float* __restrict__ P, __nv_bfloat16* pack, float* bias) {
    GS_LOOP(i, (long)MH * K1 + 2L * MH * MH + (long)NO * MH) {
        long j = i;
        if (j < (long)MH * K1) {
            int r = (int)(j / K1), k = (int)(j % K1);
            pack[PW1 / 2 + canon(r, k, K1)] = __float2bfloat16_rn(k < MI ? P[OW1 + r * MI + k] : 0.0f);
            continue;
        }
        j -= (long)MH * K1;
        if (j < 2L * MH * MH) {
            int layer = (int)(j / (MH * MH)), e = (int)(j % (MH * MH));
            int r = e / MH, k = e % MH;
            int src = layer == 0 ? OW2 : OW3, dst = layer == 0 ? PW2 : PW3;
            pack[dst / 2 + canon(r, k, MH)] = __float2bfloat16_rn(P[src + r * MH + k]);
            continue;
        }
        j -= 2L * MH * MH;
        int r = (int)(j / MH), k = (int)(j % MH);
        pack[PW4 / 2 + canon(r, k, MH)] = __float2bfloat16_rn(r < MO ? P[OW4 + r * MH + k] : 0.0f);
    }
    GS_LOOP(i, 4 * MH) {
        int l = (int)(i / MH), c = (int)(i % MH);
        float b = 0.0f;
        if (l == 0) b = P[OB1 + c];
        else if (l == 1) b = P[OB2 + c];
        else if (l == 2) b = P[OB3 + c];
        else b = c < MO ? P[OB4 + c] : 0.0f;
        bias[i] = b;
    }
}

// ------------------------------------------------------------------ training kernels
// Training GEMMs on the tensor cores:
//   C[m][n] = sum_k A(m,k) B(k,n) (+ bias[n]),
//   A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn]
// (the strides express the transposes of the backward pass).  One CTA of 4
// warps computes a 128 x 64 tile of C: the operands are staged 64 k at a time
// into shared memory, rounded to BF16, in the UMMA canonical K-major layout
// (8x8 core matrices, no swizzle; the staging writes any transpose into that
// layout), one elected thread issues tcgen05.mma (kind::f16, M = 128,
// N = 64, K = 16 per instruction) into a 64-column FP32 accumulator in tensor
// memory, and the warps read their 32 lanes back with tcgen05.ld.  Waits are
// bounded and report through *err; tensor memory is freed on every path.
constexpr int TG_M = 128, TG_N = 64, TG_K = 64, TG_THR = 128;
constexpr int TG_SA = 0, TG_SB = TG_SA + TG_M * TG_K * 2, TG_BAR = TG_SB + TG_N * TG_K * 2, TG_TM = TG_BAR + 8,
              TG_TOT = TG_TM + 8;
__global__ void __launch_bounds__(TG_THR) k_tc_gemm(int M, int N, int K, const float* __restrict__ A, long sam, long sak,
                                                    const float* __restrict__ B, long sbk, long sbn, float* __restrict__ C,
                                                    int ldc, const float* __restrict__ bias, int* err) {
    __shared__ __align__(1024) uint8_t smem[TG_TOT];
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(smem + TG_SA);
    __nv_bfloat16* sB = reinterpret_cast<__nv_bfloat16*>(smem + TG_SB);
    const uint32_t aA = smem_u32(smem + TG_SA), aB = smem_u32(smem + TG_SB), bar = smem_u32(smem + TG_BAR);
    uint32_t* tm_holder = reinterpret_cast<uint32_t*>(smem + TG_TM);
    __shared__ int status;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TG_M, n0 = blockIdx.x * TG_N;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tm_holder)), "r"(TG_N) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        status = 0;
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tm_holder;
    int chunk = 0;
    for (int k0 = 0; k0 < K; k0 += TG_K, chunk++) {
        // operands of this k range, zero outside the matrices
        for (int e = tid; e < (TG_M + TG_N) * (TG_K / 8); e += TG_THR) {
            const bool isA = e < TG_M * (TG_K / 8);
            const int f = isA ? e : e - TG_M * (TG_K / 8);
            const int r = f / (TG_K / 8), kg = (f % (TG_K / 8)) * 8;
            __align__(16) __nv_bfloat16 v[8];
#pragma unroll
            for (int j = 0; j < 8; j++) {
                const int k = k0 + kg + j;
                float x = 0.0f;
                if (isA) { const int m = m0 + r; if (m < M && k < K) x = A[(long)m * sam + (long)k * sak]; }
                else { const int n = n0 + r; if (n < N && k < K) x = B[(long)k * sbk + (long)n * sbn]; }
                v[j] = __float2bfloat16_rn(x);
            }
            __nv_bfloat16* dst = (isA ? sA : sB) + canon(r, kg, TG_K);
            *reinterpret_cast<uint4*>(dst) = *reinterpret_cast<const uint4*>(v);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t id = idesc(TG_N), sbo = (uint32_t)TG_K * 16;
#pragma unroll
            for (int kk = 0; kk < TG_K / 16; kk++)
                mma_bf16(tmem, sdesc(aA + kk * 256, 128, sbo), sdesc(aB + kk * 256, 128, sbo), id, (chunk > 0 || kk > 0) ? 1u : 0u);
            mma_commit(bar);
            // the next chunk overwrites the operands: wait for these MMAs
            if (!mbar_wait(bar, chunk & 1)) { status = 1; atomicExch(err, 1); }
        }
        __syncthreads();
        if (status) break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!status && K > 0) {
        const int m = m0 + warp * 32 + lane;
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < TG_N; c0 += 32) {
            float v[32];
            tmem_ld32(trow + c0, v);
            if (m < M) {
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    const int n = n0 + c0 + j;
                    if (n < N) C[(long)m * ldc + n] = v[j] + (bias ? bias[n] : 0.0f);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TG_N) : "memory");
    }
}
__global__ void k_round(long n, const float* __restrict__ a, float* b) { GS_LOOP(i, n) b[i] = bf16r(a[i]); }
__global__ void k_gelu_round(long n, const float* __restrict__ z, float* h) { GS_LOOP(i, n) h[i] = bf16r(gelu(z[i])); }
__global__ void k_gelu_back(long n, const float* __restrict__ z, float* d) { GS_LOOP(i, n) d[i] *= gelu_grad(z[i]); }
__global__ void k_gather(int b, const int* __restrict__ idx, const float* __restrict__ X, const float* __restrict__ T,
                         float* Xb, float* Tb) {
    GS_LOOP(i, (long)b * (MI + MO)) {
        int r = (int)(i / (MI + MO)), c = (int)(i % (MI + MO));
        long src = idx[r];
        if (c < MI) Xb[(long)r * MI + c] = bf16r(X[src * MI + c]);
        else Tb[(long)r * MO + c - MI] = T[src * MO + c - MI];
    }
}
// dY = 2 (Y - T) / (b * 12), loss += sum (Y - T)^2 / (b * 12)
__global__ void k_mse(int b, const float* __restrict__ Y, const float* __restrict__ T, float* dY, float* loss) {
    float l = 0.0f;
    const float s = 1.0f / ((float)b * MO);
    GS_LOOP(i, (long)b * MO) {
        float e = Y[i] - T[i];
        dY[i] = 2.0f * e * s;
        l += e * e * s;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}
// db[c] = sum_r d[r][c]
__global__ void k_colsum(int rows, int cols, const float* __restrict__ d, float* db) {
    GS_LOOP(c, cols) {
        float s = 0.0f;
        for (int r = 0; r < rows; r++) s += d[(long)r * cols + c];
        db[c] = s;
    }
}
__global__ void k_adam(long n, float* P, const float* __restrict__ G, float* m, float* v, float lr, float b1t, float b2t) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    GS_LOOP(i, n) {
        float g = G[i];
        float mi = b1 * m[i] + (1.0f - b1) * g, vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi; v[i] = vi;
        P[i] -= lr * (mi / (1.0f - b1t)) / (sqrtf(vi / (1.0f - b2t)) + eps);
    }
}

} // namespace

// ------------------------------------------------------------------ inference state per handle
struct MlpDev {
    uint8_t* pack = nullptr;   // PTOT bytes
    float* bias = nullptr;     // 4 * 256
    float* norm = nullptr;     // ABD_MLP_NNORM
    float* y = nullptr; int ycap = 0;
    float* feat = nullptr;
    int* err = nullptr;
};

void eng_mlp_free(Engine* E) {
    MlpDev* M = reinterpret_cast<MlpDev*>(E->mlp);
    if (!M) return;
    void* ps[] = {M->pack, M->bias, M->norm, M->y, M->feat, M->err};
    for (void* p : ps) if (p) cudaFree(p);
    delete M;
    E->mlp = nullptr;
}

static int mlp_infer(Engine* E, const float* X, int n, float* Y) {
    MlpDev* M = reinterpret_cast<MlpDev*>(E->mlp);
    static bool attr_set[64] = {false};
    int dev = E->device;
    if (dev < 64 && !attr_set[dev]) {
        CUDA_TRY(cudaFuncSetAttribute(k_mlp_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, S_TOT));
        attr_set[dev] = true;
    }
    if (n <= 0) return ABD_OK;
    CUDA_TRY(cudaMemsetAsync(M->err, 0, sizeof(int), E->stream));
    k_mlp_infer<<<(n + 127) / 128, NTHR, S_TOT, E->stream>>>(n, X, M->norm, M->pack, M->bias, Y, M->err);
    E->launches++;
    return ABD_OK;
}
static int mlp_check(Engine* E) {
    MlpDev* M = reinterpret_cast<MlpDev*>(E->mlp);
    int h = 0;
    CUDA_TRY(cudaMemcpyAsync(&h, M->err, sizeof(int), cudaMemcpyDeviceToHost, E->stream));
    CUDA_TRY(eng_stream_sync(E));
    if (h) return E->fail(ABD_ERR_CUDA, "mlp inference: a wait ran out");
    return ABD_OK;
}

// learned increment: ws = inertial increment + dt * (body frame -> world) y
__global__ void k_ws_learned(int nb, const double* __restrict__ st, const float* __restrict__ y,
                             const double* __restrict__ mass, double dt, double g0, double g1, double g2, double* ws) {
    GS_LOOP(b, nb) {
        double* w = ws + 12 * b;
        if (!(mass[b] > 0.0)) { for (int i = 0; i < 12; i++) w[i] = 0.0; continue; }
        const double* now = st + ST_STRIDE * b + ST_NOW;
        const double* q = now + ST_Q;
        // inverse of q by the adjugate
        double c00 = q[4] * q[8] - q[5] * q[7], c01 = q[5] * q[6] - q[3] * q[8], c02 = q[3] * q[7] - q[4] * q[6];
        double det = q[0] * c00 + q[1] * c01 + q[2] * c02;
        double id = det != 0.0 ? 1.0 / det : 0.0;
        double qi[9] = {c00 * id, (q[2] * q[7] - q[1] * q[8]) * id, (q[1] * q[5] - q[2] * q[4]) * id,
                        c01 * id, (q[0] * q[8] - q[2] * q[6]) * id, (q[2] * q[3] - q[0] * q[5]) * id,
                        c02 * id, (q[1] * q[6] - q[0] * q[7]) * id, (q[0] * q[4] - q[1] * q[3]) * id};
        const float* r = y + 12 * b;
        double gv[3] = {g0, g1, g2};
        for (int i = 0; i < 3; i++) {
            double s = 0;
            for (int k = 0; k < 3; k++) s += qi[3 * i + k] * r[k];
            w[i] = dt * now[ST_V + i] + dt * dt * gv[i] + dt * s;
        }
        // dq = (q^-1 M)^T: row i of dq, column j = (q^-1 M)[j][i]
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double s = 0;
                for (int k = 0; k < 3; k++) s += qi[3 * j + k] * r[3 + 3 * k + i];
                w[3 + 3 * i + j] = dt * now[ST_QD + 3 * i + j] + dt * s;
            }
    }
}

int eng_features(Engine* E, float* feat_dev);

// warm start of the next step from the network (warm_start 3)
int eng_learned_ws(Engine* E) {
    MlpDev* M = reinterpret_cast<MlpDev*>(E->mlp);
    if (!M) return E->fail(ABD_ERR_INVALID_ARG, "warm_start 3 needs abd_set_mlp first");
    int rc;
    if ((rc = eng_features(E, M->feat))) return rc;
    if ((rc = mlp_infer(E, M->feat, E->nb, M->y))) return rc;
    const AbdParams& P = E->P;
    k_ws_learned<<<grid_for(E->nb), 256, 0, E->stream>>>(E->nb, E->st, M->y, E->mass, P.dt, P.gravity[0], P.gravity[1],
                                                         P.gravity[2], E->ws);
    E->launches++;
    return ABD_OK;
}

extern "C" int abd_set_mlp(AbdHandle* h, const float* params, const float* norm) {
    Engine* E = reinterpret_cast<Engine*>(h);
    if (!E) return ABD_ERR_INVALID_ARG;
    if (!params || !norm) return E->fail(ABD_ERR_INVALID_ARG, "abd_set_mlp: null");
    if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaSetDevice");
    if (!E->mlp) {
        MlpDev* M = new MlpDev();
        E->mlp = M;
        if (cudaMalloc(&M->pack, PTOT) != cudaSuccess || cudaMalloc(&M->bias, sizeof(float) * 4 * MH) != cudaSuccess ||
            cudaMalloc(&M->norm, sizeof(float) * ABD_MLP_NNORM) != cudaSuccess ||
            cudaMalloc(&M->y, sizeof(float) * MO * (size_t)E->nb) != cudaSuccess ||
            cudaMalloc(&M->feat, sizeof(float) * MI * (size_t)E->nb) != cudaSuccess ||
            cudaMalloc(&M->err, sizeof(int)) != cudaSuccess)
            return E->fail(ABD_ERR_CUDA, "cudaMalloc mlp");
    }
    MlpDev* M = reinterpret_cast<MlpDev*>(E->mlp);
    float* P = nullptr;
    if (cudaMalloc(&P, sizeof(float) * NPARAM) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaMalloc params");
    cudaError_t e = cudaMemcpyAsync(P, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(M->norm, norm, sizeof(float) * ABD_MLP_NNORM, cudaMemcpyHostToDevice, E->stream);
    if (e == cudaSuccess) {
        k_mlp_pack<<<grid_for((long)MH * MH), 256, 0, E->stream>>>(P, reinterpret_cast<__nv_bfloat16*>(M->pack), M->bias);
        e = eng_stream_sync(E);
    }
    cudaFree(P);
    if (e != cudaSuccess) return E->fail(ABD_ERR_CUDA, std::string("abd_set_mlp: ") + cudaGetErrorString(e));
    return ABD_OK;
}

extern "C" int abd_mlp_forward(AbdHandle* h, const float* x, int32_t n, float* y) {
    Engine* E = reinterpret_cast<Engine*>(h);
    if (!E) return ABD_ERR_INVALID_ARG;
    if (!E->mlp) return E->fail(ABD_ERR_INVALID_ARG, "abd_mlp_forward: no network set");
    if (n < 0 || (n > 0 && (!x || !y))) return E->fail(ABD_ERR_INVALID_ARG, "abd_mlp_forward: bad arguments");
    if (n == 0) return ABD_OK;
    if (cudaSetDevice(E->device) != cudaSuccess) return E->fail(ABD_ERR_CUDA, "cudaSetDevice");
    float *dx = nullptr, *dy = nullptr;
    if (cudaMalloc(&dx, sizeof(float) * MI * (size_t)n) != cudaSuccess || cudaMalloc(&dy, sizeof(float) * MO * (size_t)n) != cudaSuccess) {
        cudaFree(dx);
        return E->fail(ABD_ERR_CUDA, "cudaMalloc mlp io");
    }
    int rc = ABD_OK;
    cudaError_t e = cudaMemcpyAsync(dx, x, sizeof(float) * MI * (size_t)n, cudaMemcpyHostToDevice, E->stream);
    if (e != cudaSuccess) rc = E->fail(ABD_ERR_CUDA, "abd_mlp_forward: copy in");
    if (!rc) rc = mlp_infer(E, dx, n, dy);
    if (!rc) rc = mlp_check(E);
    if (!rc) {
        e = cudaMemcpyAsync(y, dy, sizeof(float) * MO * (size_t)n, cudaMemcpyDeviceToHost, E->stream);
        if (e == cudaSuccess) e = eng_stream_sync(E);
        if (e != cudaSuccess) rc = E->fail(ABD_ERR_CUDA, "abd_mlp_forward: copy out");
    }
    cudaFree(dx); cudaFree(dy);
    return rc;
}

// ------------------------------------------------------------------ trainer
struct AbdTrainer {
    int device = 0;
    cudaStream_t s = nullptr;
    float *P = nullptr, *Pq = nullptr, *G = nullptr, *m = nullptr, *v = nullptr;
    long t = 0;
    float *X = nullptr, *T = nullptr; int n = 0;
    int bcap = 0;
    float *Xb = nullptr, *Tb = nullptr, *Z[3] = {}, *H[3] = {}, *Y = nullptr, *dY = nullptr, *dA = nullptr, *dB = nullptr;
    int* idx = nullptr;
    float* loss = nullptr;
    int* dflag = nullptr;              // set by a tensor-core GEMM whose wait gave up
    std::string err;
};

static void tr_free_batch(AbdTrainer* T) {
    float* ps[] = {T->Xb, T->Tb, T->Z[0], T->Z[1], T->Z[2], T->H[0], T->H[1], T->H[2], T->Y, T->dY, T->dA, T->dB};
    for (float* p : ps) if (p) cudaFree(p);
    if (T->idx) cudaFree(T->idx);
    T->Xb = T->Tb = T->Y = T->dY = T->dA = T->dB = nullptr;
    for (int i = 0; i < 3; i++) { T->Z[i] = nullptr; T->H[i] = nullptr; }
    T->idx = nullptr; T->bcap = 0;
}
static bool tr_reserve(AbdTrainer* T, int b) {
    if (b <= T->bcap) return true;
    tr_free_batch(T);
    bool ok = cudaMalloc(&T->Xb, sizeof(float) * MI * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->Tb, sizeof(float) * MO * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->Y, sizeof(float) * MO * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->dY, sizeof(float) * MO * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->dA, sizeof(float) * MH * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->dB, sizeof(float) * MH * (size_t)b) == cudaSuccess &&
              cudaMalloc(&T->idx, sizeof(int) * (size_t)b) == cudaSuccess;
    for (int i = 0; i < 3 && ok; i++)
        ok = cudaMalloc(&T->Z[i], sizeof(float) * MH * (size_t)b) == cudaSuccess &&
             cudaMalloc(&T->H[i], sizeof(float) * MH * (size_t)b) == cudaSuccess;
    if (ok) T->bcap = b;
    return ok;
}
static dim3 gemm_grid(int M, int N) { return dim3((N + TG_N - 1) / TG_N, (M + TG_M - 1) / TG_M); }

// loss and gradient (into T->G) of the batch in Xb / Tb (b rows)
static void tr_forward_backward(AbdTrainer* T, int b) {
    cudaStream_t s = T->s;
    const float* W[4] = {T->Pq + OW1, T->Pq + OW2, T->Pq + OW3, T->Pq + OW4};
    const float* Bs[4] = {T->P + OB1, T->P + OB2, T->P + OB3, T->P + OB4};
    const int in[4] = {MI, MH, MH, MH}, out[4] = {MH, MH, MH, MO};
    const int gW[4] = {OW1, OW2, OW3, OW4}, gB[4] = {OB1, OB2, OB3, OB4};
    const float* Hin[4] = {T->Xb, T->H[0], T->H[1], T->H[2]};
    // forward: Z = Hin W^T + b
    for (int l = 0; l < 4; l++) {
        float* Zl = l < 3 ? T->Z[l] : T->Y;
        k_tc_gemm<<<gemm_grid(b, out[l]), TG_THR, 0, s>>>(b, out[l], in[l], Hin[l], in[l], 1, W[l], 1, in[l], Zl, out[l], Bs[l],
                                                         T->dflag);
        if (l < 3) k_gelu_round<<<grid_for((long)b * MH), 256, 0, s>>>((long)b * MH, Zl, T->H[l]);
    }
    cudaMemsetAsync(T->loss, 0, sizeof(float), s);
    k_mse<<<grid_for((long)b * MO), 256, 0, s>>>(b, T->Y, T->Tb, T->dY, T->loss);
    // backward: dW = dZ^T Hin, db = colsum dZ, dHin = dZ W
    float* dZ = T->dY;
    for (int l = 3; l >= 0; l--) {
        k_tc_gemm<<<gemm_grid(out[l], in[l]), TG_THR, 0, s>>>(out[l], in[l], b, dZ, 1, out[l], Hin[l], in[l], 1,
                                                              T->G + gW[l], in[l], nullptr, T->dflag);
        k_colsum<<<grid_for(out[l]), 256, 0, s>>>(b, out[l], dZ, T->G + gB[l]);
        if (l > 0) {
            float* dH = (dZ == T->dA) ? T->dB : T->dA;
            k_tc_gemm<<<gemm_grid(b, in[l]), TG_THR, 0, s>>>(b, in[l], out[l], dZ, out[l], 1, W[l], in[l], 1, dH, in[l], nullptr,
                                                             T->dflag);
            k_gelu_back<<<grid_for((long)b * MH), 256, 0, s>>>((long)b * MH, T->Z[l - 1], dH);
            dZ = dH;
        }
    }
}

#define TR_TRY(x) do { cudaError_t _e = (x); if (_e != cudaSuccess) { T->err = std::string(#x) + ": " + cudaGetErrorString(_e); return ABD_ERR_CUDA; } } while (0)

extern "C" int abd_trainer_create(int32_t device, const float* params, AbdTrainer** out) {
    if (!params || !out) return ABD_ERR_INVALID_ARG;
    AbdTrainer* T = new AbdTrainer();
    T->device = device;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&T->s, cudaStreamNonBlocking) != cudaSuccess) {
        delete T;
        return ABD_ERR_NO_DEVICE;
    }
    size_t nb = sizeof(float) * NPARAM;
    if (cudaMalloc(&T->P, nb) != cudaSuccess || cudaMalloc(&T->Pq, nb) != cudaSuccess || cudaMalloc(&T->G, nb) != cudaSuccess ||
        cudaMalloc(&T->m, nb) != cudaSuccess || cudaMalloc(&T->v, nb) != cudaSuccess || cudaMalloc(&T->loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&T->dflag, sizeof(int)) != cudaSuccess) {
        *out = T;
        T->err = "cudaMalloc trainer";
        return ABD_ERR_CUDA;
    }
    *out = T;
    TR_TRY(cudaMemcpyAsync(T->P, params, nb, cudaMemcpyHostToDevice, T->s));
    TR_TRY(cudaMemsetAsync(T->m, 0, nb, T->s));
    TR_TRY(cudaMemsetAsync(T->v, 0, nb, T->s));
    TR_TRY(cudaMemsetAsync(T->dflag, 0, sizeof(int), T->s));
    k_round<<<grid_for(NPARAM), 256, 0, T->s>>>(NPARAM, T->P, T->Pq);
    TR_TRY(cudaStreamSynchronize(T->s));
    return ABD_OK;
}

extern "C" int abd_trainer_destroy(AbdTrainer* T) {
    if (!T) return ABD_ERR_INVALID_ARG;
    cudaSetDevice(T->device);
    tr_free_batch(T);
    float* ps[] = {T->P, T->Pq, T->G, T->m, T->v, T->X, T->T, T->loss};
    for (float* p : ps) if (p) cudaFree(p);
    if (T->dflag) cudaFree(T->dflag);
    if (T->s) cudaStreamDestroy(T->s);
    delete T;
    return ABD_OK;
}

extern "C" const char* abd_trainer_last_error(AbdTrainer* T) { return T ? T->err.c_str() : "null trainer"; }

extern "C" int abd_trainer_set_data(AbdTrainer* T, const float* x, const float* y, int32_t n) {
    if (!T || n <= 0 || !x || !y) return ABD_ERR_INVALID_ARG;
    if (cudaSetDevice(T->device) != cudaSuccess) return ABD_ERR_CUDA;
    if (T->X) cudaFree(T->X);
    if (T->T) cudaFree(T->T);
    T->X = T->T = nullptr;
    TR_TRY(cudaMalloc(&T->X, sizeof(float) * MI * (size_t)n));
    TR_TRY(cudaMalloc(&T->T, sizeof(float) * MO * (size_t)n));
    TR_TRY(cudaMemcpyAsync(T->X, x, sizeof(float) * MI * (size_t)n, cudaMemcpyHostToDevice, T->s));
    TR_TRY(cudaMemcpyAsync(T->T, y, sizeof(float) * MO * (size_t)n, cudaMemcpyHostToDevice, T->s));
    TR_TRY(cudaStreamSynchronize(T->s));
    T->n = n;
    return ABD_OK;
}

// One pass over `order` (n row indices into the data set) in mini-batches of
// `batch` rows, one Adam step per mini-batch; *mean_loss gets the mean of
// the mini-batch losses.
extern "C" int abd_trainer_epoch(AbdTrainer* T, const int32_t* order, int32_t n, int32_t batch, float lr, float* mean_loss) {
    if (!T || !order || n <= 0 || batch <= 0 || !T->X) return ABD_ERR_INVALID_ARG;
    for (int i = 0; i < n; i++) if (order[i] < 0 || order[i] >= T->n) { T->err = "abd_trainer_epoch: index out of range"; return ABD_ERR_INVALID_ARG; }
    if (cudaSetDevice(T->device) != cudaSuccess) return ABD_ERR_CUDA;
    if (!tr_reserve(T, batch)) { T->err = "cudaMalloc batch"; return ABD_ERR_CUDA; }
    int* didx = nullptr;
    TR_TRY(cudaMalloc(&didx, sizeof(int) * (size_t)n));
    TR_TRY(cudaMemcpyAsync(didx, order, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, T->s));
    float* dl = nullptr;
    int nbat = (n + batch - 1) / batch;
    TR_TRY(cudaMalloc(&dl, sizeof(float) * nbat));
    for (int k = 0; k < nbat; k++) {
        int b = std::min(batch, n - k * batch);
        k_gather<<<grid_for((long)b * (MI + MO)), 256, 0, T->s>>>(b, didx + (long)k * batch, T->X, T->T, T->Xb, T->Tb);
        tr_forward_backward(T, b);
        cudaMemcpyAsync(dl + k, T->loss, sizeof(float), cudaMemcpyDeviceToDevice, T->s);
        T->t++;
        float b1t = powf(0.9f, (float)T->t), b2t = powf(0.999f, (float)T->t);
        k_adam<<<grid_for(NPARAM), 256, 0, T->s>>>(NPARAM, T->P, T->G, T->m, T->v, lr, b1t, b2t);
        k_round<<<grid_for(NPARAM), 256, 0, T->s>>>(NPARAM, T->P, T->Pq);
    }
    std::vector<float> hl(nbat);
    TR_TRY(cudaMemcpyAsync(hl.data(), dl, sizeof(float) * nbat, cudaMemcpyDeviceToHost, T->s));
    int flag = 0;
    TR_TRY(cudaMemcpyAsync(&flag, T->dflag, sizeof(int), cudaMemcpyDeviceToHost, T->s));
    TR_TRY(cudaStreamSynchronize(T->s));
    cudaFree(dl); cudaFree(didx);
    if (flag) { T->err = "tensor-core GEMM: an mbarrier wait gave up"; return ABD_ERR_CUDA; }
    double s = 0;
    for (float v : hl) s += v;
    if (mean_loss) *mean_loss = (float)(s / nbat);
    return ABD_OK;
}

// Loss and gradient of the current parameters on the given rows (no update).
extern "C" int abd_trainer_grad(AbdTrainer* T, const float* x, const float* y, int32_t n, float* grad, float* loss) {
    if (!T || !x || !y || n <= 0 || !grad) return ABD_ERR_INVALID_ARG;
    if (cudaSetDevice(T->device) != cudaSuccess) return ABD_ERR_CUDA;
    if (!tr_reserve(T, n)) { T->err = "cudaMalloc batch"; return ABD_ERR_CUDA; }
    std::vector<float> xr((size_t)n * MI);
    for (size_t i = 0; i < xr.size(); i++) xr[i] = __bfloat162float(__float2bfloat16_rn(x[i]));
    TR_TRY(cudaMemcpyAsync(T->Xb, xr.data(), sizeof(float) * MI * (size_t)n, cudaMemcpyHostToDevice, T->s));
    TR_TRY(cudaMemcpyAsync(T->Tb, y, sizeof(float) * MO * (size_t)n, cudaMemcpyHostToDevice, T->s));
    tr_forward_backward(T, n);
    TR_TRY(cudaMemcpyAsync(grad, T->G, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, T->s));
    float l = 0;
    int flag = 0;
    TR_TRY(cudaMemcpyAsync(&l, T->loss, sizeof(float), cudaMemcpyDeviceToHost, T->s));
    TR_TRY(cudaMemcpyAsync(&flag, T->dflag, sizeof(int), cudaMemcpyDeviceToHost, T->s));
    TR_TRY(cudaStreamSynchronize(T->s));
    if (flag) { T->err = "tensor-core GEMM: an mbarrier wait gave up"; return ABD_ERR_CUDA; }
    if (loss) *loss = l;
    return ABD_OK;
}

extern "C" int abd_trainer_params(AbdTrainer* T, float* params) {
    if (!T || !params) return ABD_ERR_INVALID_ARG;
    if (cudaSetDevice(T->device) != cudaSuccess) return ABD_ERR_CUDA;
    TR_TRY(cudaMemcpyAsync(params, T->P, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, T->s));
    TR_TRY(cudaStreamSynchronize(T->s));
    return ABD_OK;
}
