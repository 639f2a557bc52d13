// k_mlp.cu — the learned mutation / rotamer proposal network on sm_100a.
//
// Network: 180 environment features -> 128 (SiLU) -> 128 (SiLU) -> 25 outputs
// (predicted Metropolis energy change of a mutation to each of the 20 amino acids
// and of each of the 5 rotamers).  Weights and activations are BF16, every sum is
// FP32.  The dense layers of training and of batched inference run on the 5th-gen
// tensor cores: one kernel, k_gemm_tc, computes C = A * B^T for K-major BF16
// operands with tcgen05.mma (one elected thread issues, the FP32 accumulator
// lives in tensor memory), operands staged in shared memory in the canonical
// no-swizzle core-matrix layout by 16-byte cp.async copies through a two-stage
// ring, and the epilogue (bias, SiLU, SiLU', BF16 packing, transposed copies for
// the weight-gradient GEMMs, split-K partials) fused on the tcgen05.ld path.
//
// Features of a residue (one warp per residue): a 20-way one-hot of its amino
// acid (none for a mutation query, amino acid MLP_NO_AA), then for each of 8
// radial shells of 1.25 A around its Calpha (0..10 A) the number of antigen
// Calphas of each of the 20 amino acids, log1p-scaled.
// Shell membership compares r^2 (the reference's f32 rounding) with the exact
// f32 squares of the shell radii, and log1p comes from a table filled on the
// host, so the features are bit-identical wherever they are computed.
#include <algorithm>

#include <cuda_bf16.h>

#include "kernels.h"
#include "mlp.cuh"

namespace binder {

__constant__ float c_log1p[MLP_COUNT_CAP + 1];

cudaError_t mlp_init_tables(const float* log1p_table) {
    return cudaMemcpyToSymbol(c_log1p, log1p_table, sizeof(float) * (MLP_COUNT_CAP + 1));
}

__device__ float mlp_log1p_count(int n) { return c_log1p[n < MLP_COUNT_CAP ? n : MLP_COUNT_CAP]; }

// ---- features ---------------------------------------------------------------------
// One warp per row: rows r = warp index; Calpha ca[r], amino acid aa[r], antigen
// ag[r] (index into ags).  X is BF16 [n_pad][MLP_K1] (columns >= MLP_IN zero);
// rows n..n_pad-1 are written as zeros.
__global__ void k_features(int n, int n_pad, const float* __restrict__ ca, const uint8_t* __restrict__ aa,
                           const int* __restrict__ ag, const AgView* __restrict__ ags, __nv_bfloat16* __restrict__ X) {
    __shared__ int s_cnt[8][MLP_SHELLS * N_AA];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = blockIdx.x * 8 + warp;
    if (r >= n_pad) return;
    int* cnt = s_cnt[warp];
    __nv_bfloat16* row = X + (size_t)r * MLP_K1;
    if (r >= n) {
        for (int j = lane; j < MLP_K1; j += 32) row[j] = __float2bfloat16_rn(0.0f);
        return;
    }
    for (int j = lane; j < MLP_SHELLS * N_AA; j += 32) cnt[j] = 0;
    __syncwarp();
    const AgView& A = ags[ag ? ag[r] : 0];
    mlp_count_env(A.ca_atom, A.res_aa, A.n_res, ca[3 * r], ca[3 * r + 1], ca[3 * r + 2], cnt);
    __syncwarp();
    const int a = aa[r];
    for (int j = lane; j < MLP_K1; j += 32) {
        float v = 0.0f;
        if (j < N_AA) v = j == a ? 1.0f : 0.0f;
        else if (j < MLP_IN) v = mlp_log1p_count(cnt[j - N_AA]);
        row[j] = __float2bfloat16_rn(v);
    }
}

// host f32 features [n][MLP_IN] -> BF16 [n_pad][MLP_K1]
__global__ void k_pack_features(int n, int n_pad, const float* __restrict__ f, __nv_bfloat16* __restrict__ X) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_pad * MLP_K1) return;
    const int r = (int)(t / MLP_K1), j = (int)(t % MLP_K1);
    X[t] = __float2bfloat16_rn(r < n && j < MLP_IN ? f[(size_t)r * MLP_IN + j] : 0.0f);
}

// out[c][r] = in[r][c], 32 x 32 tiles through shared memory
__global__ void k_transpose_bf16(int rows, int cols, const __nv_bfloat16* __restrict__ in,
                                 __nv_bfloat16* __restrict__ out) {
    __shared__ __nv_bfloat16 t[32][33];
    const int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y)
        if (r0 + i < rows && c < cols) t[i][threadIdx.x] = in[(size_t)(r0 + i) * cols + c];
    __syncthreads();
    const int r = r0 + threadIdx.x, c0 = blockIdx.x * 32;
    for (int i = threadIdx.y; i < 32; i += blockDim.y)
        if (c0 + i < cols && r < rows) out[(size_t)(c0 + i) * rows + r] = t[threadIdx.x][i];
}

// ---- tcgen05 helpers (PTX ISA 8.7, sm_100a) ---------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
    const int n = valid ? 16 : 0;  // 0 bytes read: the 16 destination bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// generic-proxy writes of shared memory made visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of barrier b; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, uint32_t max_polls = 1u << 22) {
    for (uint32_t i = 0; i < max_polls; ++i) {
        if (mbar_try_wait(b, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::f16 (BF16 inputs, FP32 accumulator)
__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// arrive on b once every tcgen05.mma this thread issued so far has completed
__device__ __forceinline__ void tc_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(b))
                 : "memory");
}
// 32 lanes x 8 consecutive FP32 columns: thread t of the warp gets lane (base lane + t)
__device__ __forceinline__ void tc_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8 rows x
// 16 bytes; lbo = byte distance between the two 8-element K halves of an MMA,
// sbo = byte distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;                // base offset 0, absolute LBO mode, layout type 0 = no swizzle
}
// Instruction descriptor of kind::f16: FP32 D, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// logistic sigmoid with the fast exponential and the approximate reciprocal (the
// results are rounded to BF16); the network tile of the Metropolis kernel uses the same
__device__ __forceinline__ float sigmoid_fast(float z) { return rcp_approx(1.0f + __expf(-z)); }

// ---- C[M x N] = A[M x K] * B[N x K]^T on the tensor cores ----------------------------
// One CTA of 256 threads per 128-row tile of A (blockIdx.x) and K slice (blockIdx.y,
// split-K); the whole N (16..256, multiple of 16) in one tensor-memory accumulator.
// A rows >= m and K beyond the slice are zero-filled in shared memory.  Warps w and
// w + 4 read the accumulator lanes 32 (w % 4) .. +31 and split its columns.
constexpr int G_M = 128, G_K = 64, G_THREADS = 256;
constexpr int G_STAGE_A = G_M * G_K * 2;                       // 16 KB
__host__ __device__ constexpr int gemm_stage_bytes(int n) { return G_STAGE_A + n * G_K * 2; }
__host__ __device__ constexpr int gemm_smem_bytes(int n) { return 2 * gemm_stage_bytes(n) + 1024; }

// core-matrix offset of (row r, 8-element K group kg) inside a stage operand
__device__ __forceinline__ uint32_t cm_off(int r, int kg) { return (uint32_t)((r >> 3) * 1024 + kg * 128 + (r & 7) * 16); }

__global__ void __launch_bounds__(G_THREADS) k_gemm_tc(GemmArgs g, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char g_smem[];
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * G_M;
    const int k_begin = blockIdx.y * g.k_split;
    const int k_end = min(g.k, k_begin + g.k_split);
    const int n_chunks = (k_end - k_begin + G_K - 1) / G_K;
    const uint32_t base = (smem_u32(g_smem) + 1023u) & ~1023u;
    const int stage_bytes = gemm_stage_bytes(g.n);
    const uint32_t ncols = g.n <= 32 ? 32u : (g.n <= 64 ? 64u : (g.n <= 128 ? 128u : 256u));

    if (warp == 0) {
        tmem_alloc(&s_tmem, ncols);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s_tmem;
    const uint32_t idesc = idesc_bf16(G_M, g.n);

    auto load_chunk = [&](int c, int st) {
        const int k0 = k_begin + c * G_K;
        const uint32_t sa = base + st * stage_bytes, sb = sa + G_STAGE_A;
        for (int p = tid; p < G_M * 8; p += G_THREADS) {
            const int r = p >> 3, kg = p & 7, k = k0 + kg * 8;
            const bool ok = m0 + r < g.m && k < k_end;
            const __nv_bfloat16* src = ok ? g.a + (size_t)(m0 + r) * g.lda + k : g.a;
            cp_async16(sa + cm_off(r, kg), src, ok);
        }
        for (int p = tid; p < g.n * 8; p += G_THREADS) {
            const int r = p >> 3, kg = p & 7, k = k0 + kg * 8;
            const bool ok = k < k_end;
            const __nv_bfloat16* src = ok ? g.b + (size_t)r * g.ldb + k : g.b;
            cp_async16(sb + cm_off(r, kg), src, ok);
        }
        cp_async_commit();
    };

    bool ok = true;
    if (n_chunks > 0) load_chunk(0, 0);
    for (int c = 0; c < n_chunks && ok; ++c) {
        const int st = c & 1;
        if (c + 1 < n_chunks) {
            // stage st^1 was read by the MMAs of chunk c-1: wait for them before refilling it
            if (c >= 1) ok = mbar_wait(&s_bar[st ^ 1], ((c - 1) >> 1) & 1);
            if (!ok) break;
            load_chunk(c + 1, st ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t sa = base + st * stage_bytes, sb = sa + G_STAGE_A;
            const int kc = min(G_K, k_end - (k_begin + c * G_K));
            for (int j = 0; j < kc / 16; ++j)
                tc_mma(tmem, smem_desc(sa + 256 * j, 128, 1024), smem_desc(sb + 256 * j, 128, 1024), idesc,
                       (c > 0 || j > 0) ? 1u : 0u);
            tc_commit(&s_bar[st]);
        }
    }
    if (ok && n_chunks > 0) ok = mbar_wait(&s_bar[(n_chunks - 1) & 1], ((n_chunks - 1) >> 1) & 1);
    // every thread saw the same waits; a thread that gave up raises the flag
    if (!ok && err) atomicOr(err, ERRF_TIMEOUT);
    tc_fence_after();

    // ---- epilogue: warp w owns accumulator lanes (rows) 32 (w % 4) .. +31, columns
    //      [n/2 * (w / 4), n/2 * (w / 4 + 1)) (multiples of 8) ----
    const int wl = warp & 3, half = warp >> 2;
    const int row = m0 + wl * 32 + lane;
    const bool row_ok = row < g.e.m_valid;
    const GemmEpi& e = g.e;
    const int n8 = g.n / 8;                        // column groups of 8
    const int cg0 = (n8 * half) / 2, cg1 = (n8 * (half + 1)) / 2;
    for (int cgi = cg0; cgi < cg1 && ok; ++cgi) {
        const int c0 = cgi * 8;
        float v[8];
        if (n_chunks > 0) tc_ld8(tmem + ((uint32_t)(wl * 32) << 16) + (uint32_t)c0, v);
        else {
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = 0.0f;
        }
        if (e.mode == EPI_F32 || e.mode == EPI_PARTIAL) {
            if (row_ok) {
                float* out = e.c + (e.mode == EPI_PARTIAL ? (size_t)blockIdx.y * e.part_stride : 0) +
                             (size_t)row * e.ldc;
#pragma unroll
                for (int i = 0; i < 8; ++i)
                    if (c0 + i < e.n_valid) out[c0 + i] = v[i] + (e.bias ? e.bias[c0 + i] : 0.0f);
            }
        } else {
            __align__(16) __nv_bfloat16 h[8];
            __align__(16) __nv_bfloat16 dz[8];
            if (e.mode == EPI_DSILU && row_ok) *(uint4*)dz = *(const uint4*)(e.sp + (size_t)row * e.ldsp + c0);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                float o = 0.0f, d = 0.0f;
                if (row_ok) {
                    if (e.mode == EPI_SILU) {
                        const float z = v[i] + (e.bias ? e.bias[c0 + i] : 0.0f);
                        const float sg = sigmoid_fast(z);
                        o = z * sg;
                        d = sg * (1.0f + z * (1.0f - sg));
                    } else {  // EPI_DSILU
                        o = v[i] * __bfloat162float(dz[i]);
                    }
                }
                h[i] = __float2bfloat16_rn(o);
                dz[i] = __float2bfloat16_rn(d);
                if (e.ht && row < e.ht_rows) e.ht[(size_t)(c0 + i) * e.ldht + row] = h[i];
            }
            if (e.h && row < e.h_rows) *(uint4*)(e.h + (size_t)row * e.ldh + c0) = *(const uint4*)h;
            if (e.mode == EPI_SILU && e.sp && row < e.h_rows)
                *(uint4*)(e.sp + (size_t)row * e.ldsp + c0) = *(const uint4*)dz;
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, ncols);
    }
}

// The bounded wait on a barrier nothing arrives on: raises ERRF_TIMEOUT after
// max_polls polls and returns (the error path of every tcgen05 wait, exercised
// without a fault).
__global__ void k_wait_selftest(uint32_t max_polls, uint32_t* __restrict__ err) {
    __shared__ __align__(8) uint64_t bar;
    mbar_init(&bar, 1);
    __syncwarp();
    if (!mbar_wait(&bar, 0, max_polls) && err) atomicOr(err, ERRF_TIMEOUT);
}

cudaError_t launch_wait_selftest(cudaStream_t s, uint32_t max_polls, uint32_t* err) {
    k_wait_selftest<<<1, 1, 0, s>>>(max_polls, err);
    return cudaGetLastError();
}

cudaError_t launch_gemm_tc(cudaStream_t s, const GemmArgs& g, uint32_t* err) {
    if (g.n < 16 || g.n > 256 || g.n % 16 || g.k % 16 || g.lda % 8 || g.ldb % 8 || g.k_split % G_K)
        return cudaErrorInvalidValue;
    const int smem = gemm_smem_bytes(g.n);
    cudaError_t e = cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e) return e;
    const int m_tiles = (g.m + G_M - 1) / G_M;
    const int k_slices = (g.k + g.k_split - 1) / g.k_split;
    if (m_tiles <= 0 || k_slices <= 0) return cudaSuccess;
    k_gemm_tc<<<dim3(m_tiles, k_slices), G_THREADS, smem, s>>>(g, err);
    return cudaGetLastError();
}

// ---- training kernels -------------------------------------------------------------
// Huber loss of the predicted energy change against the logged one; writes the
// output gradient dY (BF16 [m_pad][32] and its transpose [32][m_pad]) and adds the
// batch loss.  Prediction: y[action] - y[ref] with a reference output (ref >= 0:
// a mutation query, ref = the amino acid before the move; a row with ref == action
// carries nothing), else y[action].  Rows >= m get zero gradients.
__global__ void k_mlp_loss(int m, int m_pad, const float* __restrict__ Y, const int* __restrict__ action,
                           const int* __restrict__ ref, const float* __restrict__ target, float delta,
                           __nv_bfloat16* __restrict__ dY, __nv_bfloat16* __restrict__ dYt, double* __restrict__ loss) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m_pad) return;
    int a = -1, b = -1;
    float g = 0.0f, l = 0.0f;
    if (r < m) {
        a = action[r];
        b = ref ? ref[r] : -1;
        if (b == a) {
            a = b = -1;
        } else {
            const float* y = Y + (size_t)r * MLP_OUT_PAD;
            const float d = (b >= 0 ? y[a] - y[b] : y[a]) - target[r];
            const float ad = fabsf(d);
            l = ad <= delta ? 0.5f * d * d : delta * (ad - 0.5f * delta);
            g = fminf(fmaxf(d, -delta), delta) / (float)m;
        }
    }
    for (int j = 0; j < MLP_OUT_PAD; ++j) {
        const __nv_bfloat16 v = __float2bfloat16_rn(j == a ? g : (j == b ? -g : 0.0f));
        dY[(size_t)r * MLP_OUT_PAD + j] = v;
        dYt[(size_t)j * m_pad + r] = v;
    }
    // warp sum in fixed order, one atomic per warp
    for (int o = 16; o; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, (double)l / (double)m);
}

// out[j] = sum over k < m of G[j][k] (BF16 rows), one warp per j, fixed order
__global__ void k_rowsum_bf16(int rows, int m, int ld, const __nv_bfloat16* __restrict__ G, float* __restrict__ out) {
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= rows) return;
    float s = 0.0f;
    for (int k = lane; k < m; k += 32) s += __bfloat162float(G[(size_t)j * ld + k]);
    for (int o = 16; o; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = s;
}

// out[i] = sum over s < n_part of part[s * stride + i], fixed order
__global__ void k_reduce_partials(int n, int n_part, long long stride, const float* __restrict__ part,
                                  float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float s = 0.0f;
    for (int p = 0; p < n_part; ++p) s += part[(size_t)p * stride + i];
    out[i] = s;
}

// Adam (Kingma & Ba 2015) on the flat FP32 parameter vector
__global__ void k_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
}

// 16-byte fragment-order element (mt, s, lane) of W [N][K] at w (FP32 master copy)
__device__ __forceinline__ uint4 pack_frag(const float* __restrict__ w, int K, int mt, int s, int lane) {
    const int g = lane / 4, c = 2 * (lane % 4), k0 = 16 * s;
    const float* r0 = w + (size_t)(16 * mt + g) * K + k0;
    const float* r1 = w + (size_t)(16 * mt + g + 8) * K + k0;
    const __nv_bfloat162 a0 = __floats2bfloat162_rn(r0[c], r0[c + 1]);
    const __nv_bfloat162 a1 = __floats2bfloat162_rn(r1[c], r1[c + 1]);
    const __nv_bfloat162 a2 = __floats2bfloat162_rn(r0[8 + c], r0[9 + c]);
    const __nv_bfloat162 a3 = __floats2bfloat162_rn(r1[8 + c], r1[9 + c]);
    return make_uint4(*(const uint32_t*)&a0, *(const uint32_t*)&a1, *(const uint32_t*)&a2, *(const uint32_t*)&a3);
}

// BF16 copies of the weights: W1 [H][192], W2 [H][H] and W2^T, W3 [32][H] and W3^T,
// and the fragment-order copies of W1, W2, W3 (one thread per element of the
// largest of them)
__global__ void k_pack_weights(const float* __restrict__ p, MlpBf16 o) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (MLP_H / 16) * (MLP_K1 / 16) * 32) {
        const int lane = t % 32, ks = (t / 32) % (MLP_K1 / 16), mt = t / (32 * (MLP_K1 / 16));
        o.f1[t] = pack_frag(p + MLP_OFF_W1, MLP_K1, mt, ks, lane);
    }
    if (t < (MLP_H / 16) * (MLP_H / 16) * 32) {
        const int lane = t % 32, ks = (t / 32) % (MLP_H / 16), mt = t / (32 * (MLP_H / 16));
        o.f2[t] = pack_frag(p + MLP_OFF_W2, MLP_H, mt, ks, lane);
    }
    if (t < (MLP_OUT_PAD / 16) * (MLP_H / 16) * 32) {
        const int lane = t % 32, ks = (t / 32) % (MLP_H / 16), mt = t / (32 * (MLP_H / 16));
        o.f3[t] = pack_frag(p + MLP_OFF_W3, MLP_H, mt, ks, lane);
    }
    if (t < MLP_H * MLP_K1) o.w1[t] = __float2bfloat16_rn(p[MLP_OFF_W1 + t]);
    if (t < MLP_H * MLP_H) {
        const int n = t / MLP_H, k = t % MLP_H;
        const __nv_bfloat16 v = __float2bfloat16_rn(p[MLP_OFF_W2 + t]);
        o.w2[t] = v;
        o.w2t[(size_t)k * MLP_H + n] = v;
    }
    if (t < MLP_OUT_PAD * MLP_H) {
        const int n = t / MLP_H, k = t % MLP_H;
        const __nv_bfloat16 v = __float2bfloat16_rn(p[MLP_OFF_W3 + t]);
        o.w3[t] = v;
        o.w3t[(size_t)k * MLP_OUT_PAD + n] = v;
    }
}

// Gather a minibatch of logged tuples: features input rows, action, reference
// output, target.  A mutation is a query without amino acid (MLP_NO_AA) whose
// energy change is predicted as y[new] - y[old]; a rotamer move queries with its
// amino acid and is predicted by y[20 + rotamer].
__global__ void k_gather_tuples(int m, const int* __restrict__ idx, const MlpTuple* __restrict__ tup,
                                float* __restrict__ ca, uint8_t* __restrict__ aa, int* __restrict__ ag,
                                int* __restrict__ action, int* __restrict__ ref, float* __restrict__ target) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const MlpTuple t = tup[idx[r]];
    const bool mut = t.action < N_AA;
    ca[3 * r] = t.x;
    ca[3 * r + 1] = t.y;
    ca[3 * r + 2] = t.z;
    aa[r] = mut ? (uint8_t)MLP_NO_AA : t.aa;
    ag[r] = t.antigen;
    action[r] = t.action;
    ref[r] = mut ? (int)t.aa : -1;
    target[r] = t.delta_e;
}
// minibatch indices drawn with the Philox generator: idx[r] = uniform in [0, n_tuples)
__global__ void k_draw_batch(int m, int n_tuples, uint64_t seed, uint32_t step, int* __restrict__ idx) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    const U4 u = philox((uint32_t)r, step, 0xB47Cu, 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
    idx[r] = (int)(((uint64_t)u.x * (uint32_t)n_tuples) >> 32);
}

// ---- launchers ----------------------------------------------------------------------
void launch_features(cudaStream_t s, int n, int n_pad, const float* ca, const uint8_t* aa, const int* ag,
                     const AgView* ags, __nv_bfloat16* X) {
    if (n_pad > 0) k_features<<<(n_pad + 7) / 8, 256, 0, s>>>(n, n_pad, ca, aa, ag, ags, X);
}
void launch_pack_features(cudaStream_t s, int n, int n_pad, const float* f, __nv_bfloat16* X) {
    const long long t = (long long)n_pad * MLP_K1;
    if (t > 0) k_pack_features<<<(unsigned)((t + 255) / 256), 256, 0, s>>>(n, n_pad, f, X);
}
void launch_transpose_bf16(cudaStream_t s, int rows, int cols, const __nv_bfloat16* in, __nv_bfloat16* out) {
    if (rows > 0 && cols > 0) k_transpose_bf16<<<dim3((cols + 31) / 32, (rows + 31) / 32), dim3(32, 8), 0, s>>>(rows, cols, in, out);
}
void launch_mlp_loss(cudaStream_t s, int m, int m_pad, const float* Y, const int* action, const int* ref,
                     const float* target, float delta, __nv_bfloat16* dY, __nv_bfloat16* dYt, double* loss) {
    if (m_pad > 0)
        k_mlp_loss<<<(m_pad + 255) / 256, 256, 0, s>>>(m, m_pad, Y, action, ref, target, delta, dY, dYt, loss);
}
void launch_rowsum_bf16(cudaStream_t s, int rows, int m, int ld, const __nv_bfloat16* G, float* out) {
    if (rows > 0) k_rowsum_bf16<<<(rows + 7) / 8, 256, 0, s>>>(rows, m, ld, G, out);
}
void launch_reduce_partials(cudaStream_t s, int n, int n_part, long long stride, const float* part, float* out) {
    if (n > 0) k_reduce_partials<<<(n + 255) / 256, 256, 0, s>>>(n, n_part, stride, part, out);
}
void launch_adam(cudaStream_t s, int n, float* w, const float* g, float* m1, float* m2, float lr, float b1, float b2,
                 float eps, float bc1, float bc2) {
    if (n > 0) k_adam<<<(n + 255) / 256, 256, 0, s>>>(n, w, g, m1, m2, lr, b1, b2, eps, bc1, bc2);
}
void launch_pack_weights(cudaStream_t s, const float* p, const MlpBf16& o) {
    const int n = std::max(MLP_H * MLP_K1, std::max(MLP_H * MLP_H, MLP_OUT_PAD * MLP_H));
    k_pack_weights<<<(n + 255) / 256, 256, 0, s>>>(p, o);
}
void launch_gather_tuples(cudaStream_t s, int m, const int* idx, const MlpTuple* tup, float* ca, uint8_t* aa, int* ag,
                          int* action, int* ref, float* target) {
    if (m > 0) k_gather_tuples<<<(m + 255) / 256, 256, 0, s>>>(m, idx, tup, ca, aa, ag, action, ref, target);
}
void launch_draw_batch(cudaStream_t s, int m, int n_tuples, uint64_t seed, uint32_t step, int* idx) {
    if (m > 0) k_draw_batch<<<(m + 255) / 256, 256, 0, s>>>(m, n_tuples, seed, step, idx);
}

}  // namespace binder
