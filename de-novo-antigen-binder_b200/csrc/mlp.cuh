// mlp.cuh — sizes, parameter layout and device views of the learned proposal
// network (k_mlp.cu), and the environment count shared by the feature kernel and
// the Metropolis kernel.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace binder {

constexpr int MLP_IN = 180;       // 20 one-hot + 8 shells x 20 amino acids
constexpr int MLP_K1 = 192;       // first-layer K padded to the MMA K step
constexpr int MLP_H = 256;        // hidden width
constexpr int MLP_OUT = 25;       // 20 mutation targets + 5 rotamers
constexpr int MLP_OUT_PAD = 32;   // output rows of W3 (rows >= 25 stay zero)
constexpr int MLP_SHELLS = 8;     // radial shells of 1.25 A out to 10 A
constexpr int MLP_COUNT_CAP = 255;
constexpr int MLP_NO_AA = 255;    // amino-acid input of a mutation query: none (no one-hot)

// flat FP32 parameter vector: W1 [256][192], b1 [256], W2 [256][256], b2 [256],
// W3 [32][256], b3 [32]
constexpr int MLP_OFF_W1 = 0;
constexpr int MLP_OFF_B1 = MLP_OFF_W1 + MLP_H * MLP_K1;
constexpr int MLP_OFF_W2 = MLP_OFF_B1 + MLP_H;
constexpr int MLP_OFF_B2 = MLP_OFF_W2 + MLP_H * MLP_H;
constexpr int MLP_OFF_W3 = MLP_OFF_B2 + MLP_H;
constexpr int MLP_OFF_B3 = MLP_OFF_W3 + MLP_OUT_PAD * MLP_H;
constexpr int MLP_N_PARAMS = MLP_OFF_B3 + MLP_OUT_PAD;
constexpr int MLP_BIASES = 2 * MLP_H + MLP_OUT_PAD;  // b1, b2, b3

// Shell of a squared distance r2 < 100: the number of squared shell radii
// (1.25 k)^2, k = 1..7, that r2 reaches.  Every radius square is exact in f32.
__host__ __device__ __forceinline__ int mlp_shell(float r2) {
    return (r2 >= 1.5625f) + (r2 >= 6.25f) + (r2 >= 14.0625f) + (r2 >= 25.0f) + (r2 >= 39.0625f) +
           (r2 >= 56.25f) + (r2 >= 76.5625f);
}

// Approximate reciprocal (PTX rcp.approx.ftz.f32: within 1 ulp; 1 / inf = 0), for
// the sigmoid of the network's SiLU, whose results are rounded to BF16.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Counts of antigen Calphas by (shell, amino acid) around (x, y, z), by one warp:
// cnt[shell * 20 + aa] += 1 for every antigen Calpha with r^2 < 100 (the
// reference's f32 rounding of r^2).  cnt is zeroed by the caller.  Each lane reads
// and tests four Calphas before its first count, so that their loads overlap.
__device__ __forceinline__ void mlp_count_env(const float4* __restrict__ ag_ca, const uint8_t* __restrict__ ag_aa,
                                              int n, float x, float y, float z, int* cnt) {
    constexpr int U = 4;
    for (int i0 = (threadIdx.x & 31); i0 < n; i0 += 32 * U) {
        float r2[U];
        int a[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + 32 * u;
            r2[u] = 1e30f;
            a[u] = 0;
            if (i < n) {
                const float4 q = ag_ca[i];
                r2[u] = xdist2(xsub(x, q.x), xsub(y, q.y), xsub(z, q.z));
                a[u] = ag_aa[i];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (r2[u] < 100.0f) atomicAdd(&cnt[mlp_shell(r2[u]) * N_AA + a[u]], 1);
    }
}

enum : int { EPI_F32 = 0, EPI_PARTIAL = 1, EPI_SILU = 2, EPI_DSILU = 3 };

// Epilogue of k_gemm_tc.
//  EPI_F32:     c[row][col] = acc + bias[col]                (cols < n_valid, rows < m_valid)
//  EPI_PARTIAL: the same without bias at c + blockIdx.y * part_stride (split-K partials)
//  EPI_SILU:    z = acc + bias; h = silu(z) as BF16 to h[row][col] (rows < h_rows) and
//               ht[col][row] (rows < ht_rows); silu'(z) as BF16 to sp[row][col] (if sp);
//               rows >= m_valid store 0
//  EPI_DSILU:   h = acc * sp[row][col] (the saved BF16 silu'(z)) as BF16 to h / ht likewise
struct GemmEpi {
    int mode = EPI_F32;
    const float* bias = nullptr;
    float* c = nullptr;
    int ldc = 0;
    long long part_stride = 0;
    __nv_bfloat16* h = nullptr;
    int ldh = 0, h_rows = 0;
    __nv_bfloat16* ht = nullptr;
    int ldht = 0, ht_rows = 0;
    __nv_bfloat16* sp = nullptr;  // silu'(z), BF16 [rows][ldsp]
    int ldsp = 0;
    int n_valid = 0, m_valid = 0;
};

// C = A * B^T: A [m][k] (row stride lda), B [n][k] (row stride ldb), BF16, K-major.
// k and k_split multiples of 16 and 64; n in 16..256, multiple of 16.
struct GemmArgs {
    const __nv_bfloat16* a = nullptr;
    int lda = 0, m = 0;
    const __nv_bfloat16* b = nullptr;
    int ldb = 0, n = 0;
    int k = 0, k_split = 0;
    GemmEpi e;
};

// Fragment order of a BF16 weight matrix W [N][K] for the warp-level MMA with the
// weights as the A operand (m16n8k16, A row-major: 16 outputs x 16 k; the rows of
// the network's input are the N = 8 columns): element (mt, s, l) (mt = tile of 16
// outputs, s = 16-wide k-step, l = lane; g = l / 4, c = 2 (l % 4), k0 = 16 s) is 16
// bytes holding {W[16mt+g][k0+c], W[16mt+g][k0+c+1]}, {W[16mt+g+8][k0+c], ..+1},
// {W[16mt+g][k0+8+c], ..+1}, {W[16mt+g+8][k0+8+c], ..+1} -- the lane's a0..a3
// registers of one MMA in one 16-byte load; a warp's loads are 512 contiguous bytes.
__host__ __device__ constexpr int frag_index(int mt, int s, int lane, int K) { return (mt * (K / 16) + s) * 32 + lane; }

// BF16 weight copies used by the GEMMs and the Metropolis kernel's network tile
struct MlpBf16 {
    __nv_bfloat16* w1;   // [H][192]
    __nv_bfloat16* w2;   // [H][H]
    __nv_bfloat16* w2t;  // [H][H] transposed
    __nv_bfloat16* w3;   // [32][H]
    __nv_bfloat16* w3t;  // [H][32] transposed
    uint4* f1;           // W1 in fragment order (H/16 output tiles x 12 k-steps x 32 lanes)
    uint4* f2;           // W2 in fragment order (H/16 x H/16 x 32)
    uint4* f3;           // W3 in fragment order (2 x H/16 x 32)
};

// One logged Metropolis proposal (binder_mc_tuple of the C ABI, 32 bytes).
struct MlpTuple {
    float x, y, z;      // Calpha when the move was proposed
    float delta_e;      // exact Metropolis energy change of the move
    int32_t cand;
    float log_ratio;    // log q(reverse) - log q(forward) of the proposal (0 when uniform)
    int16_t residue;
    uint8_t aa, action, antigen, accepted;
    uint8_t pad[2];
};

// The network as the Metropolis kernel sees it (BF16 weights in fragment order,
// FP32 biases).
struct MlpDev {
    const uint4* f1;
    const uint4* f2;
    const uint4* f3;
    const float* b1;
    const float* b2;
    const float* b3;
    float t_prop_min;         // proposal temperature = max(T, t_prop_min)
    float t_max;              // steps at temperatures above t_max use the uniform proposal
};
static_assert(sizeof(MlpTuple) == 32, "tuple layout");

}  // namespace binder
