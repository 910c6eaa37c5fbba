// device_common.cuh — device helpers shared by the kernel files.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "yao_internal.h"

namespace yao {

// Complex arithmetic with the exact operation structure of num_complex
// (ac - bd, ad + bc) and no FMA contraction: the double-precision kernels
// reproduce the CPU path's roundings bit for bit.
__device__ __forceinline__ double2 cmul_x(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cadd_x(double2 a, double2 b) {
    return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
// MulAssign of num_complex: re = re*b.re - im*b.im; im = im*b.re + re_old*b.im
__device__ __forceinline__ double2 cmulassign_x(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.y, b.x), __dmul_rn(a.x, b.y)));
}

// float2 counterparts (single precision forms; FMA allowed).
__device__ __forceinline__ float2 cmul_x(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd_x(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cmulassign_x(float2 a, float2 b) { return cmul_x(a, b); }

template <typename V>
struct VecT;
template <>
struct VecT<double2> {
    typedef double R;
    static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
};
template <>
struct VecT<float2> {
    typedef float R;
    static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
};

// Insert a zero bit at each of the sorted positions pos[0] < pos[1] < ...
__device__ __forceinline__ uint64_t insert_zeros(uint64_t g, const int8_t* pos, int n) {
    for (int j = 0; j < n; j++) {
        int p = pos[j];
        uint64_t low = g & ((1ull << p) - 1);
        g = ((g >> p) << (p + 1)) | low;
    }
    return g;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum `nv` per-thread values over the block in a fixed order; thread 0
// writes them to out[0..nv).  smem must hold nv * (blockDim/32) doubles.
__device__ __forceinline__ void block_sum_write(double* vals, int nv, double* smem, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int i = 0; i < nv; i++) {
        double v = warp_sum(vals[i]);
        if (lane == 0) smem[i * nw + warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < nv; i++) {
            double s = 0.0;
            for (int w = 0; w < nw; w++) s += smem[i * nw + w];
            out[i] = s;
        }
    }
    __syncthreads();
}

// Grid used by the streaming kernels.
inline unsigned grid_for(uint64_t work, unsigned threads, int num_sms, int per_sm = 8) {
    uint64_t b = (work + threads - 1) / threads;
    uint64_t cap = (uint64_t)num_sms * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace yao
