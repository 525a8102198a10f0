// common.cuh — shared definitions of the sm_100a ABD library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <float.h>
#include "../../include/abd_b200.h"

// BDFAffine layout (BDF1.py:11-14, quat_util.py:40-47): 48 doubles per body.
#define ST_STRIDE 48
#define ST_NOW 0
#define ST_NXT 24
#define ST_C 0
#define ST_Q 3
#define ST_V 12
#define ST_QD 15

// stencil types of an active contact
#define T_PP 0
#define T_PE 1
#define T_EE 2
#define T_PT 3
#define T_PG 4

#define HD __host__ __device__ __forceinline__
#define DV __device__ __forceinline__

// Grid sizing: B200 has 148 SMs.  Grid-stride kernels launch a multiple of
// the SM count and read their item count from device memory, so they can be
// captured in a CUDA graph before that count is known on the host.
#define NUM_SMS 148

struct d3 { double x, y, z; };
HD d3 mk3(double x, double y, double z) { return d3{x, y, z}; }
HD d3 operator+(d3 a, d3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
HD d3 operator-(d3 a, d3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
HD d3 operator*(double s, d3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
HD double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
HD d3 cross(d3 a, d3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
HD double comp(d3 a, int k) { return k == 0 ? a.x : (k == 1 ? a.y : a.z); }
DV d3 ld3(const double* p) { return mk3(p[0], p[1], p[2]); }

// Full-warp keyed reduction: every lane of the warp must call it.
DV void warp_reduce_add(double* acc, int key, double v, bool valid) {
    int k = valid ? key : -1;
    int k0 = __shfl_sync(0xffffffffu, k, 0);
    bool same = __all_sync(0xffffffffu, k == k0 || k < 0);
    if (same) {
        double s = valid ? v : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        // lane 0 may itself be invalid: pick the first valid lane's key
        unsigned vm = __ballot_sync(0xffffffffu, valid);
        if (vm && (threadIdx.x & 31) == (unsigned)(__ffs(vm) - 1)) atomicAdd(acc + key, s);
        return;
    }
    if (valid) atomicAdd(acc + key, v);
}

// atomic min of a non-negative double (bit pattern order == value order)
DV void atomic_min_pos(double* addr, double v) {
    if (!(v >= 0.0)) v = 0.0;
    atomicMin(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// atomic max of a non-negative float
DV void atomic_max_pos(float* addr, float v) {
    atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}
