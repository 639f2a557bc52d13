// mlp_tile.cuh — the proposal network evaluated inside a Metropolis CTA on one
// tile of at most 8 rows (the residues of one candidate that drew a move in a
// step: about two on average, far below the 64/128-row tiles of tcgen05.mma), by
// the CTA's eight warps with the warp-level BF16 MMA (m16n8k16, FP32 accumulators).
// The weights are the MMA's A operand (16 outputs x 16 k) and the tile's rows its
// N = 8 columns, so one MMA covers every row of the tile: a layer of N outputs over
// K inputs is (N / 16) x (K / 16) MMAs per CTA, whatever the number of rows.
// Weights are read from global memory (L2-resident, 240 KB, not cached in L1) in
// fragment order with 16-byte loads, in a few large register batches per layer;
// activations stay in shared memory as BF16, the output as FP32.  Same arithmetic
// as the batched tensor-core path up to the order of the FP32 sums.
#pragma once

#include <cuda_bf16.h>

#include "mlp.cuh"

namespace binder {

constexpr int MT_ROWS = 8;
constexpr int MT_XS = 200;  // X row stride (BF16): 100 words, rows land on distinct banks
constexpr int MT_HS = MLP_H + 8;  // H row stride (BF16): 4 words mod 32, rows land on distinct banks
constexpr int MT_YS = MLP_OUT_PAD;
constexpr int MT_KQ = 4;    // layer 3: its 16 k-steps split over 4 warps per output tile
constexpr int MT_PS = MT_YS + 1;  // row stride of layer 3's partial sums (FP32; no bank conflicts)
// shared-memory bytes of a tile: X, H1, H2 (BF16), Y (FP32), environment counts
// (int); layer 3's partial sums (FP32 [MT_KQ][8][MT_PS]) reuse H1
constexpr int MT_X_BYTES = MT_ROWS * MT_XS * 2;
constexpr int MT_H_BYTES = MT_ROWS * MT_HS * 2;
constexpr int MT_Y_BYTES = MT_ROWS * MT_YS * 4;
constexpr int MT_CNT_BYTES = MT_ROWS * MLP_SHELLS * N_AA * 4;
constexpr int MT_BYTES = MT_X_BYTES + 2 * MT_H_BYTES + MT_Y_BYTES + MT_CNT_BYTES;
static_assert(MT_KQ * MT_ROWS * MT_PS * 4 <= MT_H_BYTES, "layer 3 partial sums must fit H1");
static_assert(MT_ROWS * MT_YS == 256, "the final sums take one thread of the 256 per output");

struct MlpTile {
    __nv_bfloat16* x;   // [8][MT_XS]
    __nv_bfloat16* h1;  // [8][MT_HS]
    __nv_bfloat16* h2;  // [8][MT_HS]
    float* y;           // [8][32]
    int* cnt;           // [8][160]
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

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], const uint4& a, uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a.x), "r"(a.y), "r"(a.z), "r"(a.w), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld_s32(const __nv_bfloat16* p) { return *(const uint32_t*)p; }
// weights are cached in L2 only: streamed through L1 they would evict the antigen
// atoms that the CTA's energy evaluations read from it
__device__ __forceinline__ uint4 ld_g128(const uint4* p) { return __ldcg(p); }
// SiLU as the batched GEMM epilogue computes it: z * sigmoid, sigmoid = 1 / (1 + e^-z)
// with the fast exponential and the approximate reciprocal
__device__ __forceinline__ float silu_f(float z) { return z * rcp_approx(1.0f + __expf(-z)); }

// Weight registers of a lane: one batch of a layer's fragments (16 bytes per output
// tile per k-step), at most MT_WREGS of them.
constexpr int MT_WREGS = 16;

// k-steps s0 .. s0+SB-1 of the warp's output tiles mt0 .. mt0+MT-1 into w.
template <int K, int MT, int SB>
__device__ __forceinline__ void mlp_tile_fetch(uint4 (&w)[MT_WREGS], const uint4* __restrict__ Wf, int mt0, int s0) {
    static_assert(MT * SB <= MT_WREGS, "weight batch larger than the registers");
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < SB; ++s)
#pragma unroll
        for (int m = 0; m < MT; ++m) w[s * MT + m] = ld_g128(Wf + frag_index(mt0 + m, s0 + s, lane, K));
}

// Sums of in[8][K] W^T over the k-steps s0 .. s0+NB*SB-1 for the warp's output
// tiles mt0 .. mt0+MT-1: acc[m] holds (lane g = lane / 4, c = 2 (lane % 4)) the
// outputs 16 (mt0+m) + g (entries 0, 1: rows c, c+1) and 16 (mt0+m) + g + 8 (2, 3).
// The weights come in NB batches of SB k-steps: w holds the first batch on entry;
// each batch is multiplied, then the registers are refilled with the next one --
// after the last batch by next() (the next layer's first batch), so that its
// latency hides behind this layer's epilogue and barrier.
template <int K, int MT, int SB, int NB, class Next>
__device__ __forceinline__ void mlp_tile_sums(uint4 (&w)[MT_WREGS], const __nv_bfloat16* in, int in_stride,
                                              const uint4* __restrict__ Wf, int mt0, int s0, float (&acc)[MT][4],
                                              Next next) {
    const int lane = threadIdx.x & 31, g = lane >> 2, tg = lane & 3;
#pragma unroll
    for (int m = 0; m < MT; ++m) acc[m][0] = acc[m][1] = acc[m][2] = acc[m][3] = 0.0f;
    const __nv_bfloat16* xr = in + g * in_stride + 2 * tg;  // B operand: row g of the input
#pragma unroll
    for (int bi = 0; bi < NB; ++bi) {
#pragma unroll
        for (int s = 0; s < SB; ++s) {
            const int k0 = (s0 + bi * SB + s) * 16;
            const uint32_t b0 = ld_s32(xr + k0), b1 = ld_s32(xr + k0 + 8);
#pragma unroll
            for (int m = 0; m < MT; ++m) mma_bf16_16816(acc[m], w[s * MT + m], b0, b1);
        }
        if (bi + 1 < NB) mlp_tile_fetch<K, MT, SB>(w, Wf, mt0, s0 + (bi + 1) * SB);
        else next();
    }
}

// SiLU epilogue of a hidden layer: out[row][col] = silu(acc + bias) as BF16 for the
// rows < rows, zero for the others.
template <int MT>
__device__ __forceinline__ void mlp_tile_silu(const float (&acc)[MT][4], int mt0, const float* bias,
                                              __nv_bfloat16* out, int rows) {
    const int lane = threadIdx.x & 31, g = lane >> 2, r0 = 2 * (lane & 3);
#pragma unroll
    for (int m = 0; m < MT; ++m) {
        const int c = 16 * (mt0 + m) + g;
        const float b_lo = bias[c], b_hi = bias[c + 8];
        const __nv_bfloat16 z = __float2bfloat16_rn(0.0f);
        out[r0 * MT_HS + c] = r0 < rows ? __float2bfloat16_rn(silu_f(acc[m][0] + b_lo)) : z;
        out[(r0 + 1) * MT_HS + c] = r0 + 1 < rows ? __float2bfloat16_rn(silu_f(acc[m][1] + b_lo)) : z;
        out[r0 * MT_HS + c + 8] = r0 < rows ? __float2bfloat16_rn(silu_f(acc[m][2] + b_hi)) : z;
        out[(r0 + 1) * MT_HS + c + 8] = r0 + 1 < rows ? __float2bfloat16_rn(silu_f(acc[m][3] + b_hi)) : z;
    }
}

// Shapes: layers 1 and 2 over MT_MT = 2 output tiles of 16 per warp (the 8 warps
// cover the hidden width), layer 1's 12 k-steps in two batches of 6, layer 2's 16
// in two batches of 8; layer 3 (32 outputs, 2 tiles) splits its 16 k-steps over
// MT_KQ = 4 warps per tile, one batch of 4 each, and adds the four partial sums in
// a fixed order.
constexpr int MT_MT = MLP_H / 16 / 8;
constexpr int MT_SB1 = MLP_K1 / 16 / 2;
constexpr int MT_SB2 = MLP_H / 16 / 2;
constexpr int MT_SB3 = MLP_H / 16 / MT_KQ;
static_assert(MT_MT * MT_SB1 <= MT_WREGS && MT_MT * MT_SB2 <= MT_WREGS && MT_SB3 <= MT_WREGS,
              "weight batches must fit the registers");
static_assert(MLP_OUT_PAD / 16 * MT_KQ == 8, "layer 3 takes the 8 warps");

// The first batch of layer 1 into w: issue it before the tile's inputs are ready.
__device__ __forceinline__ void mlp_tile_prefetch(const MlpDev& M, uint4 (&w)[MT_WREGS]) {
    mlp_tile_fetch<MLP_K1, MT_MT, MT_SB1>(w, M.f1, (int)(threadIdx.x >> 5) * MT_MT, 0);
}

// Network outputs of rows 0 .. rows-1 of T.x into T.y, by the 8 warps of the CTA
// (all threads call; barriers inside).  w holds layer 1's first batch
// (mlp_tile_prefetch).  Rows rows .. 7 of T.x must be finite (zero).
__device__ __forceinline__ void mlp_tile_forward(const MlpDev& M, const MlpTile& T, uint4 (&w)[MT_WREGS],
                                                 int rows) {
    const int warp = threadIdx.x >> 5;
    const int mt0 = warp * MT_MT;
    const int mt3 = warp & 1, kq = warp >> 1;  // layer 3: output tile, quarter of K
    float acc[MT_MT][4];
    mlp_tile_sums<MLP_K1, MT_MT, MT_SB1, 2>(w, T.x, MT_XS, M.f1, mt0, 0, acc, [&] {
        mlp_tile_fetch<MLP_H, MT_MT, MT_SB2>(w, M.f2, mt0, 0);
    });
    mlp_tile_silu<MT_MT>(acc, mt0, M.b1, T.h1, rows);
    __syncthreads();
    mlp_tile_sums<MLP_H, MT_MT, MT_SB2, 2>(w, T.h1, MT_HS, M.f2, mt0, 0, acc, [&] {
        mlp_tile_fetch<MLP_H, 1, MT_SB3>(w, M.f3, mt3, kq * MT_SB3);
    });
    mlp_tile_silu<MT_MT>(acc, mt0, M.b2, T.h2, rows);
    __syncthreads();
    float a3[1][4];
    mlp_tile_sums<MLP_H, 1, MT_SB3, 1>(w, T.h2, MT_HS, M.f3, mt3, kq * MT_SB3, a3, [] {});
    {  // partial sums of this quarter of K: part[kq][row][col] (H1 is free now)
        float* part = (float*)T.h1 + kq * (MT_ROWS * MT_PS);
        const int lane = threadIdx.x & 31, c = 16 * mt3 + (lane >> 2), r0 = 2 * (lane & 3);
        part[r0 * MT_PS + c] = a3[0][0];
        part[(r0 + 1) * MT_PS + c] = a3[0][1];
        part[r0 * MT_PS + c + 8] = a3[0][2];
        part[(r0 + 1) * MT_PS + c + 8] = a3[0][3];
    }
    __syncthreads();
    {
        const float* part = (const float*)T.h1;
        const int i = threadIdx.x;  // 256 threads = 8 rows x 32 outputs
        const int r = i / MT_YS, c = i % MT_YS;
        if (r < rows) {
            float v = part[r * MT_PS + c];
#pragma unroll
            for (int q = 1; q < MT_KQ; ++q) v += part[q * (MT_ROWS * MT_PS) + r * MT_PS + c];
            T.y[r * MT_YS + c] = v + M.b3[c];
        }
    }
    __syncthreads();
}

}  // namespace binder
