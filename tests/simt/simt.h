// Host-side emulation of the CUDA execution model for testing kernel source
// on a machine without a GPU: every thread of a block runs as a std::thread,
// __syncthreads and __syncwarp are std::barriers, __shfl_sync exchanges
// through a per-warp array between two warp barriers, and each block's
// dynamic shared memory is one host buffer.  The blocks of a cluster run
// at the same time (a cluster barrier is a std::barrier over all of their
// threads, split into arrive and wait); clusters run one after the other.
// It covers what the direct solver's band kernel and the warp-level PSD
// projection of the contact Hessians use.  The band kernel's cp.async
// helpers are plain copies here, so the emulation checks indexing and
// barriers, not the timing of asynchronous copies; its named barrier 1 is a
// std::barrier over the whole block that producers arrive at without
// waiting; warp votes and shuffles go through the per-warp array.  A kernel
// that needs anything else (tensor cores, atomics on shared memory,
// distributed shared memory) does not compile against it.
#pragma once
#include <barrier>
#include <thread>
#include <vector>
#include <memory>
#include <optional>
#include <cmath>
#include <atomic>
#include <algorithm>
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
struct dim3 { unsigned x = 1, y = 1, z = 1; };
inline thread_local dim3 threadIdx, blockIdx;
inline dim3 blockDim, gridDim;
struct SimtBlock {
    std::unique_ptr<std::barrier<>> block, named;
    std::vector<std::unique_ptr<std::barrier<>>> warps;
    double xd[64][32];
    std::vector<unsigned char> smem;
};
inline thread_local SimtBlock* g_blk = nullptr;
inline thread_local unsigned char* g_dyn_smem = nullptr;
inline std::barrier<>* g_cluster_bar = nullptr;
inline thread_local std::optional<std::barrier<>::arrival_token> g_cluster_tok;
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__
#define __launch_bounds__(...)
#define __cluster_dims__(...)
#define __align__(x) alignas(x)
#define DV inline
#define HD inline
using std::min; using std::max;
// the device rsqrtf is an approximation (2 ulp); this one is off by a relative
// 2.3e-7 (close to 2^-22), so that kernel code refining it is tested from a
// start as coarse (the kernels run here take the double-precision rsqrt)
inline float rsqrtf(float x) { return (float)((1.0 / std::sqrt((double)x)) * (1.0 + 2.3e-7)); }
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
inline void __syncthreads() { g_blk->block->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { g_blk->warps[threadIdx.x / 32]->arrive_and_wait(); }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }
inline double __ldcg(const double* p) { return *p; }
inline double __shfl_sync(unsigned, double v, int src) {
    int w = threadIdx.x / 32, l = threadIdx.x % 32;
    g_blk->xd[w][l] = v;
    g_blk->warps[w]->arrive_and_wait();
    double r = g_blk->xd[w][src & 31];
    g_blk->warps[w]->arrive_and_wait();
    return r;
}
inline double __shfl_xor_sync(unsigned m, double v, int o) { return __shfl_sync(m, v, (int)(threadIdx.x % 32) ^ o); }
inline bool __any_sync(unsigned, bool pred) {
    int w = threadIdx.x / 32, l = threadIdx.x % 32;
    g_blk->xd[w][l] = pred ? 1.0 : 0.0;
    g_blk->warps[w]->arrive_and_wait();
    bool any = false;
    for (int i = 0; i < 32; i++) any = any || g_blk->xd[w][i] != 0.0;
    g_blk->warps[w]->arrive_and_wait();
    return any;
}
inline float __shfl_sync(unsigned m, float v, int src) { return (float)__shfl_sync(m, (double)v, src); }
inline int __shfl_sync(unsigned m, int v, int src) { return (int)__shfl_sync(m, (double)v, src); }
inline int atomicOr(int* p, int v) { return std::atomic_ref<int>(*p).fetch_or(v); }
// cp.async stand-ins: the copy happens at once, so the waits have nothing to wait for
inline void band_cp16(void* sdst, const void* gsrc) { std::memcpy(sdst, gsrc, 16); }
inline void band_cp_commit() {}
inline void band_cp_wait_all() {}
inline void band_cp_wait_but_one() {}
// named barrier: the kernel uses id 1 over the whole block only
inline void band_bar_sync(int id, int n) {
    if (id != 1 || n != (int)blockDim.x) { std::fprintf(stderr, "named barrier %d/%d unsupported\n", id, n); std::abort(); }
    g_blk->named->arrive_and_wait();
}
inline void band_bar_arrive(int id, int n) {
    if (id != 1 || n != (int)blockDim.x) { std::fprintf(stderr, "named barrier %d/%d unsupported\n", id, n); std::abort(); }
    auto token = g_blk->named->arrive();
    (void)token;
}
inline void band_cluster_arrive() {
    if (g_cluster_tok) { std::fprintf(stderr, "cluster barrier: arrive twice in one phase\n"); std::abort(); }
    g_cluster_tok.emplace(g_cluster_bar->arrive());
}
inline void band_cluster_wait() {
    if (!g_cluster_tok) { std::fprintf(stderr, "cluster barrier: wait without arrive\n"); std::abort(); }
    g_cluster_bar->wait(std::move(*g_cluster_tok));
    g_cluster_tok.reset();
}
// grid blocks of `block` threads in clusters of `cluster` blocks
template <class F> void launch(int grid, int block, size_t smem, F f, int cluster = 1) {
    gridDim.x = grid; blockDim.x = block;
    for (int c0 = 0; c0 < grid; c0 += cluster) {
        std::barrier<> cb(cluster * block);
        g_cluster_bar = &cb;
        std::vector<std::unique_ptr<SimtBlock>> blks;
        for (int b = 0; b < cluster; b++) {
            auto B = std::make_unique<SimtBlock>();
            B->block = std::make_unique<std::barrier<>>(block);
            B->named = std::make_unique<std::barrier<>>(block);
            for (int w = 0; w < (block + 31) / 32; w++) B->warps.push_back(std::make_unique<std::barrier<>>(32));
            B->smem.assign(smem, 0);
            blks.push_back(std::move(B));
        }
        std::vector<std::thread> ts;
        for (int b = 0; b < cluster; b++)
            for (int t = 0; t < block; t++)
                ts.emplace_back([&, t, b] {
                    threadIdx.x = t; blockIdx.x = c0 + b;
                    g_blk = blks[b].get(); g_dyn_smem = blks[b]->smem.data();
                    f();
                    if (g_cluster_tok) { std::fprintf(stderr, "cluster barrier: thread exits after arrive without wait\n"); std::abort(); }
                });
        for (auto& th : ts) th.join();
    }
}
