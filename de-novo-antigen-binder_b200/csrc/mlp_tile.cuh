// mlp_tile.cuh — the proposal network evaluated inside a Metropolis CTA on one
// tile of at most 16 residues (the residues of one candidate that drew a move in
// a step: a handful of rows, below the 64/128-row tiles of tcgen05.mma, so the
// CTA's eight warps use the warp-level BF16 MMA, m16n8k16 with FP32 accumulators).
// Weights are read from global memory (L2-resident, 240 KB, not cached in L1) in
// fragment order with 16-byte loads, in a few large register batches per layer; activations stay in
// shared memory as BF16, the output as FP32.  Same arithmetic as the batched
// tensor-core path up to the order of the FP32 sums.
#pragma once

#include <cuda_bf16.h>

#include "mlp.cuh"

namespace binder {

constexpr int MT_ROWS = 16;
constexpr int MT_XS = 200;  // X row stride (BF16): 100 words, rows land on distinct banks
constexpr int MT_HS = MLP_H + 8;  // H row stride (BF16): 4 words mod 32, rows land on distinct banks
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
// weights are cached in L2 only: streamed through L1 they would evict the antigen
// atoms that the CTA's energy evaluations read from it
__device__ __forceinline__ uint4 ld_g128(const uint4* p) { return __ldcg(p); }
// SiLU as the batched GEMM epilogue computes it: z * sigmoid, sigmoid = 1 / (1 + e^-z)
// with the fast exponential and a correctly rounded reciprocal
__device__ __forceinline__ float silu_f(float z) { return z * __frcp_rn(1.0f + __expf(-z)); }

// Weight registers of a lane: one batch of a layer's fragments (16 bytes per n-tile
// per pair of k-steps), at most MT_WREGS of them.
constexpr int MT_WREGS = 12;

// Batch bi of a layer's weights for the warp's n-tiles n_tile0 .. n_tile0+NT-1:
// pairs of k-steps bi*PB .. bi*PB+PB-1.
template <int K, int NT, int PB>
__device__ __forceinline__ void mlp_tile_fetch(uint4 (&w)[MT_WREGS], const uint4* __restrict__ Wf, int n_tile0,
                                               int bi) {
    static_assert(NT * PB <= MT_WREGS, "weight batch larger than the registers");
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int p = 0; p < PB; ++p)
#pragma unroll
        for (int t = 0; t < NT; ++t) w[p * NT + t] = ld_g128(Wf + frag_index(n_tile0 + t, bi * PB + p, lane, K));
}

// One dense layer on the tile: out[16][cols of the warp] = act(in[16][K] W^T + b).
// Warp w computes the n-tiles n_tile0 .. n_tile0+NT-1 (8 columns each); ACT = SiLU to
// BF16 (out_h) or identity to FP32 (out_f).  The weights (fragment order, L2-resident)
// come in batches of PB pairs of k-steps: w holds batch 0 on entry; each batch is
// multiplied, then the registers are refilled with the next one -- after the last
// batch with batch 0 of the next layer (Wn: K2 / NT2 / PB2 at n-tile n_next; none
// when null), so that its latency hides behind this layer's epilogue and barrier.
// Rows >= rows hold no move: the epilogue writes them as zeros without evaluating
// the activation (the MMA rows are independent of each other).
template <int K, int NT, int PB, bool ACT, int K2, int NT2, int PB2>
__device__ __forceinline__ void mlp_tile_layer(uint4 (&w)[MT_WREGS], const __nv_bfloat16* in, int in_stride,
                                               const uint4* __restrict__ Wf, int n_tile0, const float* bias,
                                               __nv_bfloat16* out_h, int out_stride, float* out_f,
                                               const uint4* __restrict__ Wn, int n_next, int rows) {
    constexpr int SP = K / 32;   // pairs of k-steps
    constexpr int NB = SP / PB;  // batches
    static_assert(SP % PB == 0, "batches must split the k-step pairs evenly");
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
    float acc[NT][4];
#pragma unroll
    for (int t = 0; t < NT; ++t) acc[t][0] = acc[t][1] = acc[t][2] = acc[t][3] = 0.0f;
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
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
                    const uint4 v = w[p * NT + t];
                    mma_bf16_16816(acc[t], a, h ? v.z : v.x, h ? v.w : v.y);
                }
            }
        if (bi + 1 < NB) mlp_tile_fetch<K, NT, PB>(w, Wf, n_tile0, bi + 1);
        else if (Wn) mlp_tile_fetch<K2, NT2, PB2>(w, Wn, n_next, 0);
    }
    const bool lo = g < rows, hi = g + 8 < rows;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int c = (n_tile0 + t) * 8 + 2 * tg;
        const float b0 = bias[c], b1 = bias[c + 1];
        if (ACT) {
            __nv_bfloat162 v0 = __floats2bfloat162_rn(0.0f, 0.0f), v1 = v0;
            if (lo) v0 = __floats2bfloat162_rn(silu_f(acc[t][0] + b0), silu_f(acc[t][1] + b1));
            if (hi) v1 = __floats2bfloat162_rn(silu_f(acc[t][2] + b0), silu_f(acc[t][3] + b1));
            *(__nv_bfloat162*)(out_h + g * out_stride + c) = v0;
            *(__nv_bfloat162*)(out_h + (g + 8) * out_stride + c) = v1;
        } else {
            if (lo) {
                out_f[g * MT_YS + c] = acc[t][0] + b0;
                out_f[g * MT_YS + c + 1] = acc[t][1] + b1;
            }
            if (hi) {
                out_f[(g + 8) * MT_YS + c] = acc[t][2] + b0;
                out_f[(g + 8) * MT_YS + c + 1] = acc[t][3] + b1;
            }
        }
    }
}

// Shapes: layers 1 and 2 over MT_NT n-tiles of 8 columns per warp (the 8 warps
// cover the hidden width), their k-step pairs in batches that fill the weight
// registers (hidden width 256: layer 1's 6 pairs x 4 n-tiles in two batches of 3,
// layer 2's 8 pairs x 4 n-tiles in four batches of 2); layer 3 (32 outputs) on
// warps 0-3, one n-tile and all its pairs in one batch.
constexpr int MT_NT = MLP_H / 64;
constexpr int MT_PB1 = MT_WREGS / MT_NT < MLP_K1 / 32 ? MT_WREGS / MT_NT : MLP_K1 / 32;
constexpr int MT_PB2 = MLP_H / 32 <= MT_WREGS / MT_NT ? MLP_H / 32 : 2;
constexpr int MT_PB3 = MLP_H / 32;
static_assert(MT_NT * MT_PB1 <= MT_WREGS && MT_NT * MT_PB2 <= MT_WREGS && MT_PB3 <= MT_WREGS,
              "weight batches must fit the registers");

// Batch 0 of layer 1 into w: issue it before the tile's inputs are ready.
__device__ __forceinline__ void mlp_tile_prefetch(const MlpDev& M, uint4 (&w)[MT_WREGS]) {
    mlp_tile_fetch<MLP_K1, MT_NT, MT_PB1>(w, M.f1, (int)(threadIdx.x >> 5) * MT_NT, 0);
}

// Network outputs of rows 0 .. rows-1 of T.x into T.y, by the 8 warps of the CTA
// (all threads call; barriers inside).  w holds layer 1's batch 0 (mlp_tile_prefetch).
__device__ __forceinline__ void mlp_tile_forward(const MlpDev& M, const MlpTile& T, uint4 (&w)[MT_WREGS],
                                                 int rows) {
    const int warp = threadIdx.x >> 5;
    const bool out_warp = warp < MLP_OUT_PAD / 8;
    mlp_tile_layer<MLP_K1, MT_NT, MT_PB1, true, MLP_H, MT_NT, MT_PB2>(w, T.x, MT_XS, M.f1, warp * MT_NT, M.b1, T.h1,
                                                                       MT_HS, nullptr, M.f2, warp * MT_NT, rows);
    __syncthreads();
    mlp_tile_layer<MLP_H, MT_NT, MT_PB2, true, MLP_H, 1, MT_PB3>(w, T.h1, MT_HS, M.f2, warp * MT_NT, M.b2, T.h2,
                                                                  MT_HS, nullptr, out_warp ? M.f3 : nullptr, warp,
                                                                  rows);
    __syncthreads();
    if (out_warp)
        mlp_tile_layer<MLP_H, 1, MT_PB3, false, MLP_H, 1, MT_PB3>(w, T.h2, MT_HS, M.f3, warp, M.b3, nullptr, 0, T.y,
                                                                  nullptr, 0, rows);
    __syncthreads();
}

}  // namespace binder
