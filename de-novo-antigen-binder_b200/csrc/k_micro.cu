// k_micro.cu — FP32 peak microbenchmark: the roofline denominator for the FP32
// kernels (the measured-peaks file of this pool carries HBM and bf16 figures only).
//
// Every thread runs 8 independent FMA chains (enough to cover the FMA latency);
// a full-occupancy grid of 148 x k CTAs keeps every SM sub-partition issuing.  The
// packed variant uses Blackwell's fma.rn.f32x2 (two FP32 FMAs per instruction).
#include "kernels.h"

namespace binder {

__global__ void __launch_bounds__(256) k_ffma(float* out, int iters, float b, float c) {
    float a0 = threadIdx.x * 1e-3f, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f, a4 = a0 + 4.f, a5 = a0 + 5.f,
          a6 = a0 + 6.f, a7 = a0 + 7.f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            a0 = fmaf(a0, b, c); a1 = fmaf(a1, b, c); a2 = fmaf(a2, b, c); a3 = fmaf(a3, b, c);
            a4 = fmaf(a4, b, c); a5 = fmaf(a5, b, c); a6 = fmaf(a6, b, c); a7 = fmaf(a7, b, c);
        }
    }
    const float s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    if (s == 1234.5f) out[blockIdx.x] = s;  // never true for the chosen b, c; keeps the chains live
}

__device__ __forceinline__ unsigned long long fma2(unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
    unsigned long long d;
    asm volatile("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

__global__ void __launch_bounds__(256) k_ffma2(float* out, int iters, float b, float c) {
    const float a = threadIdx.x * 1e-3f;
    unsigned long long bb, cc, x[8];
    asm("mov.b64 %0, {%1, %1};" : "=l"(bb) : "f"(b));
    asm("mov.b64 %0, {%1, %1};" : "=l"(cc) : "f"(c));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float lo = a + 2 * k, hi = a + 2 * k + 1;
        asm("mov.b64 %0, {%1, %2};" : "=l"(x[k]) : "f"(lo), "f"(hi));
    }
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) x[k] = fma2(x[k], bb, cc);
        }
    }
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo, hi;
        asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(x[k]));
        s += lo + hi;
    }
    if (s == 1234.5f) out[blockIdx.x] = s;
}

// Returns FMA flops executed (2 per FMA) for the launch.
double launch_ffma(cudaStream_t s, float* scratch, int ctas, int iters, bool packed) {
    if (packed) k_ffma2<<<ctas, 256, 0, s>>>(scratch, iters, 0.999999f, 1e-7f);
    else k_ffma<<<ctas, 256, 0, s>>>(scratch, iters, 0.999999f, 1e-7f);
    const double fmas_per_thread = (double)iters * 16.0 * 8.0 * (packed ? 2.0 : 1.0);
    return 2.0 * fmas_per_thread * 256.0 * ctas;
}

}  // namespace binder
