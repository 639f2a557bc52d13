// mlp_tile.cuh — the proposal network evaluated inside a Metropolis CTA on one
// tile of at most 16 residues (the residues of one candidate that drew a move in
// a step: a handful of rows, below the 64/128-row tiles of tcgen05.mma, so the
// CTA's eight warps use the warp-level BF16 MMA, m16n8k16 with FP32 accumulators).
// Weights are read from global memory (L2-resident, 240 KB) in fragment order with
// 16-byte loads, double-buffered in registers; activations stay in shared memory as
// BF16, the output as FP32.  Same arithmetic as the batched
// tensor-core path up to the order of the FP32 sums.
#pragma once

#include <cuda_bf16.h>

#include "mlp.cuh"

namespace binder {

constexpr int MT_ROWS = 16;
constexpr int MT_XS = 200;  // X row stride (BF16): 100 words, rows land on distinct banks
constexpr int MT_HS = 264;  // H row stride (BF16): 132 words
constexpr int MT_YS = MLP_OUT_PAD;
// shared-memory bytes of a tile: X, H1, H2 (BF16), Y (FP32), environment counts (int)
constexpr int MT_X_BYTES = MT_ROWS * MT_XS * 2;
constexpr int MT_H_BYTES = MT_ROWS * MT_HS * 2;
constexpr int MT_Y_BYTES = MT_ROWS * MT_YS * 4;
constexpr int MT_CNT_BYTES = MT_ROWS * MLP_SHELLS * N_AA * 4;
constexpr int MT_BYTES = MT_X_BYTES + 2 * MT_H_BYTES + MT_Y_BYTES + MT_CNT_BYTES;

struct MlpTile {
    __nv_bfloat16* x;   // [16][MT_XS]
    __nv_bfloat16* h1;  // [16][MT_HS]
    __nv_bfloat16* h2;  // [16][MT_HS]
    float* y;           // [16][32]
    int* cnt;           // [16][160]
};
__device__ __forceinline__ MlpTile mlp_tile_carve(unsigned char* p) {
    MlpTile t;
    t.x = (__nv_bfloat16*)p;
    t.h1 = (__nv_bfloat16*)(p + MT_X_BYTES);
    t.h2 = (__nv_bfloat16*)(p + MT_X_BYTES + MT_H_BYTES);
    t.y = (float*)(p + MT_X_BYTES + 2 * MT_H_BYTES);
    t.cnt = (int*)(p + MT_X_BYTES + 2 * MT_H_BYTES + MT_Y_BYTES);
    return t;
}

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld_s32(const __nv_bfloat16* p) { return *(const uint32_t*)p; }
__device__ __forceinline__ uint4 ld_g128(const uint4* p) { return __ldg(p); }
__device__ __forceinline__ float silu_f(float z) { return z / (1.0f + expf(-z)); }

// One dense layer on the tile: out[16][cols of the warp] = act(in[16][K] W^T + b).
// Warp w computes the n-tiles n_tile0 .. n_tile0+NT-1 (8 columns each); ACT = SiLU to
// BF16 (out_h) or identity to FP32 (out_f).  The warp's weights (fragment order,
// 16 bytes per lane per pair of k-steps) stream through registers in batches of
// two pairs, the next batch in flight while the current one is multiplied.
template <int K, int NT, bool ACT>
__device__ __forceinline__ void mlp_tile_layer(const __nv_bfloat16* in, int in_stride, const uint4* Wf,
                                               const float* bias, __nv_bfloat16* out_h, int out_stride,
                                               float* out_f, int n_tile0) {
    constexpr int SP = K / 32;   // pairs of k-steps
    constexpr int PB = 2;        // pairs per batch
    constexpr int NB = SP / PB;  // batches
    static_assert(SP % PB == 0, "K must be a multiple of 64");
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
    float acc[NT][4];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0f;
    uint4 buf[2][PB][NT];
#pragma unroll
    for (int p = 0; p < PB; ++p)
#pragma unroll
        for (int t = 0; t < NT; ++t) buf[0][p][t] = ld_g128(Wf + frag_index(n_tile0 + t, p, lane, K));
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
        if (bi + 1 < NB) {
#pragma unroll
            for (int p = 0; p < PB; ++p)
#pragma unroll
                for (int t = 0; t < NT; ++t)
                    buf[(bi + 1) & 1][p][t] = ld_g128(Wf + frag_index(n_tile0 + t, (bi + 1) * PB + p, lane, K));
        }
#pragma unroll
        for (int p = 0; p < PB; ++p)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k0 = ((bi * PB + p) * 2 + h) * 16;
                uint32_t a[4];
                a[0] = ld_s32(in + g * in_stride + k0 + 2 * tg);
                a[1] = ld_s32(in + (g + 8) * in_stride + k0 + 2 * tg);
                a[2] = ld_s32(in + g * in_stride + k0 + 8 + 2 * tg);
                a[3] = ld_s32(in + (g + 8) * in_stride + k0 + 8 + 2 * tg);
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    const uint4 v = buf[bi & 1][p][t];
                    mma_bf16_16816(acc[t], a, h ? v.z : v.x, h ? v.w : v.y);
                }
            }
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int c = (n_tile0 + t) * 8 + 2 * tg;
        const float b0 = bias[c], b1 = bias[c + 1];
        if (ACT) {
            out_h[g * out_stride + c] = __float2bfloat16_rn(silu_f(acc[t][0] + b0));
            out_h[g * out_stride + c + 1] = __float2bfloat16_rn(silu_f(acc[t][1] + b1));
            out_h[(g + 8) * out_stride + c] = __float2bfloat16_rn(silu_f(acc[t][2] + b0));
            out_h[(g + 8) * out_stride + c + 1] = __float2bfloat16_rn(silu_f(acc[t][3] + b1));
        } else {
            out_f[g * MT_YS + c] = acc[t][0] + b0;
            out_f[g * MT_YS + c + 1] = acc[t][1] + b1;
            out_f[(g + 8) * MT_YS + c] = acc[t][2] + b0;
            out_f[(g + 8) * MT_YS + c + 1] = acc[t][3] + b1;
        }
    }
}

// Network outputs of the 16 rows of T.x into T.y, by the 8 warps of the CTA
// (all threads call; barriers inside).
__device__ __forceinline__ void mlp_tile_forward(const MlpDev& M, const MlpTile& T) {
    const int warp = threadIdx.x >> 5;
    mlp_tile_layer<MLP_K1, 4, true>(T.x, MT_XS, M.f1, M.b1, T.h1, MT_HS, nullptr, warp * 4);
    __syncthreads();
    mlp_tile_layer<MLP_H, 4, true>(T.h1, MT_HS, M.f2, M.b2, T.h2, MT_HS, nullptr, warp * 4);
    __syncthreads();
    if (warp < MLP_OUT_PAD / 8) mlp_tile_layer<MLP_H, 1, false>(T.h2, MT_HS, M.f3, M.b3, nullptr, 0, T.y, warp);
    __syncthreads();
}

}  // namespace binder
