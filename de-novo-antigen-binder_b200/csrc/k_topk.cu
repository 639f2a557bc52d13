// k_topk.cu — survivor selection: the k lowest energies of each segment in
// stable ascending order (diffusion.rs:1042-1057 sorts with a stable sort and
// truncates to the population).
//
// One CTA per segment.  k <= 64: warps keep sorted best-64 lists in registers and a
// merge tree joins them (k_topk64).  Larger k: energies are mapped to order-preserving 64-bit keys
// (-0.0 folded onto +0.0, NaN after every number) and paired with their index,
// so a plain lexicographic (key, index) order is exactly the stable sort.  The
// CTA keeps a running best-k list in shared memory and merges the segment in
// chunks with a bitonic sort of (chunk + best-k) elements, its short-stride stages
// in registers.
#include "kernels.h"
#include "topk.cuh"

namespace binder {

constexpr int TOPK_SORT = 4096;   // elements per bitonic pass (pow2)
constexpr int TOPK_MAX_K = 1024;  // best-k kept between passes
constexpr int TOPK_THREADS = 1024;

// Bitonic stages with stride < 32 for sizes size_lo..size_hi (powers of two): every
// position p < N (N a multiple of 32, so whole warps take part or none) is held by
// lane p % 32 of a warp, whose partner p ^ stride is a lane of the same warp.  The
// lower position of a pair keeps the smaller (key, index) when the pair sorts
// ascending (bit `size` of p clear), the larger otherwise.
__device__ __forceinline__ void register_stages(unsigned long long* key, int* idx, int N, int size_lo, int size_hi) {
    for (int p = threadIdx.x; p < N; p += blockDim.x) {
        unsigned long long k = key[p];
        int i = idx[p];
        for (int size = size_lo; size <= size_hi; size <<= 1) {
            for (int stride = min(size >> 1, 16); stride > 0; stride >>= 1) {
                const unsigned long long ko = __shfl_xor_sync(0xffffffffu, k, stride);
                const int io = __shfl_xor_sync(0xffffffffu, i, stride);
                const bool lower = (p & stride) == 0, up = (p & size) == 0;
                const bool other_less = (ko < k) || (ko == k && io < i);
                if (other_less == (lower == up)) {  // take the partner's element
                    k = ko;
                    i = io;
                }
            }
        }
        key[p] = k;
        idx[p] = i;
    }
}

__global__ void __launch_bounds__(TOPK_THREADS) k_topk(const double* __restrict__ e,
                                                        const int* __restrict__ idx_list,
                                                        const long long* __restrict__ seg_off, int k,
                                                        int* __restrict__ out_idx) {
    extern __shared__ unsigned char smem_raw[];
    unsigned long long* key = reinterpret_cast<unsigned long long*>(smem_raw);
    int* idx = reinterpret_cast<int*>(key + TOPK_SORT);
    const int seg = blockIdx.x;
    const long long b0 = seg_off[seg], b1 = seg_off[seg + 1];
    const long long n = b1 - b0;
    const int chunk = TOPK_SORT - k;  // new elements per pass
    int kept = 0;                     // valid entries at the front of key/idx
    for (long long base = 0; base < n || base == 0; base += chunk) {
        const long long take = min((long long)chunk, n - base);
        // bitonic size: the next power of two holding the kept list and the chunk
        int N = 64;
        while (N < kept + take) N <<= 1;
        // slots [kept, N): new chunk, padded with +inf keys
        for (int t = threadIdx.x; t < N; t += blockDim.x) {
            if (t < kept) continue;
            const long long j = base + (t - kept);
            if (t - kept < take) {
                const int g = idx_list ? idx_list[b0 + j] : (int)(b0 + j);
                key[t] = order_key(e[g]);
                idx[t] = g;
            } else {
                key[t] = 0xFFFFFFFFFFFFFFFFull;
                idx[t] = INT32_MAX;
            }
        }
        __syncthreads();
        // bitonic sort of [0, N): the stages with stride >= 32 exchange through shared
        // memory (a barrier each); those with stride < 32 pair lanes of one warp and run
        // in registers with shuffles -- sizes 2..32 entirely, then the five last
        // strides of every larger size
        register_stages(key, idx, N, 2, 32);
        __syncthreads();
        for (int size = 64; size <= N; size <<= 1) {
            for (int stride = size >> 1; stride >= 32; stride >>= 1) {
                for (int t = threadIdx.x; t < N / 2; t += blockDim.x) {
                    const int lo = 2 * t - (t & (stride - 1));
                    const int hi = lo + stride;
                    const bool up = ((lo & size) == 0);
                    const unsigned long long kl = key[lo], kh = key[hi];
                    const int il = idx[lo], ih = idx[hi];
                    const bool gt = (kl > kh) || (kl == kh && il > ih);
                    if (gt == up) {
                        key[lo] = kh; key[hi] = kl;
                        idx[lo] = ih; idx[hi] = il;
                    }
                }
                __syncthreads();
            }
            register_stages(key, idx, N, size, size);
            __syncthreads();
        }
        kept = (int)min((long long)k, (long long)kept + take);
        if (take <= 0) break;
    }
    for (int t = threadIdx.x; t < k; t += blockDim.x)
        out_idx[(long long)seg * k + t] = (t < kept && idx[t] != INT32_MAX) ? idx[t] : -1;
}

// ---- k <= 64: warp sorts and a merge tree (topk.cuh) ---------------------------------
constexpr int TOPK64_WARPS = 32;
__global__ void __launch_bounds__(TOPK64_WARPS * 32) k_topk64(const double* __restrict__ e,
                                                               const int* __restrict__ idx_list,
                                                               const long long* __restrict__ seg_off, int k,
                                                               int* __restrict__ out_idx) {
    __shared__ unsigned long long s_k[TOPK64_WARPS][64];
    __shared__ int s_i[TOPK64_WARPS][64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = blockIdx.x;
    const long long b0 = seg_off[seg], n = seg_off[seg + 1] - b0;
    const KI inf = {0xFFFFFFFFFFFFFFFFull, INT32_MAX};
    KI a = inf, b = inf;  // this warp's best 64, sorted
    for (long long base = (long long)warp * 32; base < n; base += TOPK64_WARPS * 32) {
        KI v = inf;
        if (base + lane < n) {
            const int g = idx_list ? idx_list[b0 + base + lane] : (int)(b0 + base + lane);
            v = KI{order_key(e[g]), g};
        }
        v = warp_sort32(v, lane);
        warp_merge64(a, b, v, inf, lane);
    }
    // merge tree over the warps' lists
    for (int level = 1; level < TOPK64_WARPS; level <<= 1) {
        if ((warp & (2 * level - 1)) == level) {
            s_k[warp][lane] = a.k; s_i[warp][lane] = a.i;
            s_k[warp][lane + 32] = b.k; s_i[warp][lane + 32] = b.i;
        }
        __syncthreads();
        if ((warp & (2 * level - 1)) == 0) {
            const int o = warp + level;
            const KI c = {s_k[o][lane], s_i[o][lane]}, d = {s_k[o][lane + 32], s_i[o][lane + 32]};
            warp_merge64(a, b, c, d, lane);
        }
        __syncthreads();
    }
    if (warp == 0) {
        if (lane < k) out_idx[(long long)seg * k + lane] = a.i != INT32_MAX ? a.i : -1;
        if (lane + 32 < k) out_idx[(long long)seg * k + lane + 32] = b.i != INT32_MAX ? b.i : -1;
    }
}

int launch_topk_segments(cudaStream_t s, const double* energies, const int* idx_list, const long long* seg_off,
                         int n_seg, int k, int* out_idx) {
    if (n_seg <= 0 || k <= 0) return 0;
    if (k > TOPK_MAX_K) return -1;
    if (k <= 64) {
        k_topk64<<<n_seg, TOPK64_WARPS * 32, 0, s>>>(energies, idx_list, seg_off, k, out_idx);
        return 1;
    }
    const size_t smem = (size_t)TOPK_SORT * (sizeof(unsigned long long) + sizeof(int));
    cudaFuncSetAttribute(k_topk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_topk<<<n_seg, TOPK_THREADS, smem, s>>>(energies, idx_list, seg_off, k, out_idx);
    return 1;
}

}  // namespace binder
