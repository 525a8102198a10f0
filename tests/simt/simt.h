// Host-side emulation of the CUDA execution model for testing kernel source
// on a machine without a GPU: every thread of a block runs as a std::thread,
// __syncthreads and __syncwarp are std::barriers, __shfl_sync exchanges
// through a per-warp array between two warp barriers, and the dynamic shared
// memory is one host buffer.  Blocks of a grid run one after the other.  It
// covers what the direct solver's band kernel uses (its cp.async helpers are
// plain copies here, so the emulation checks indexing and barriers, not the
// timing of asynchronous copies; its named barrier 1 is a std::barrier over
// the whole block that producers arrive at without waiting); a kernel that
// needs anything else (tensor cores, atomics on shared memory, clusters)
// does not compile against it.
#pragma once
#include <barrier>
#include <thread>
#include <vector>
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
inline std::barrier<>* g_block_bar = nullptr;
inline std::vector<std::barrier<>*> g_warp_bar;
inline std::barrier<>* g_named_bar = nullptr;
inline double g_xd[64][32];
inline unsigned char* g_dyn_smem = nullptr;
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __restrict__
#define __launch_bounds__(...)
#define __align__(x) alignas(x)
#define DV inline
#define HD inline
using std::min; using std::max;
// the device rsqrtf is an approximation (2 ulp); this one is off by a relative
// 2.3e-7 (close to 2^-22) so that refinements of it are tested from a start as coarse
inline float rsqrtf(float x) { return (float)((1.0 / std::sqrt((double)x)) * (1.0 + 2.3e-7)); }
inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
inline void __syncthreads() { g_block_bar->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { g_warp_bar[threadIdx.x / 32]->arrive_and_wait(); }
inline double __shfl_sync(unsigned, double v, int src) {
    int w = threadIdx.x / 32, l = threadIdx.x % 32;
    g_xd[w][l] = v;
    g_warp_bar[w]->arrive_and_wait();
    double r = g_xd[w][src & 31];
    g_warp_bar[w]->arrive_and_wait();
    return r;
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
    g_named_bar->arrive_and_wait();
}
inline void band_bar_arrive(int id, int n) {
    if (id != 1 || n != (int)blockDim.x) { std::fprintf(stderr, "named barrier %d/%d unsupported\n", id, n); std::abort(); }
    auto token = g_named_bar->arrive();
    (void)token;
}
template <class F> void launch(int grid, int block, size_t smem, F f) {
    gridDim.x = grid; blockDim.x = block;
    std::vector<unsigned char> dyn(smem);
    g_dyn_smem = dyn.data();
    for (int b = 0; b < grid; b++) {
        std::barrier<> bb(block), nb(block);
        g_block_bar = &bb;
        g_named_bar = &nb;
        std::vector<std::barrier<>*> wb;
        for (int w = 0; w < (block + 31) / 32; w++) wb.push_back(new std::barrier<>(32));
        g_warp_bar = wb;
        std::vector<std::thread> ts;
        for (int t = 0; t < block; t++)
            ts.emplace_back([&, t, b] { threadIdx.x = t; blockIdx.x = b; f(); });
        for (auto& th : ts) th.join();
        for (auto* p : wb) delete p;
    }
}
