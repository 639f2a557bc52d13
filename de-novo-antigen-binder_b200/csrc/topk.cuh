// topk.cuh — order-preserving keys of FP64 energies and the warp-level sorted
// best-64 lists of the survivor selection (k_topk.cu), also used by the fused
// candidate-sum + selection kernel of the scoring path (k_score.cu).
#pragma once

#include "kernels.h"

namespace binder {

// (key, index) in lexicographic order is the stable ascending sort of the energies:
// -0.0 is folded onto +0.0, NaN sorts after every number.
__device__ __forceinline__ unsigned long long order_key(double e) {
    if (e != e) return 0xFFFFFFFFFFFFFFFFull;  // NaN last
    e = e + 0.0;                               // -0.0 -> +0.0
    unsigned long long b = (unsigned long long)__double_as_longlong(e);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}


// Each warp keeps the 64 smallest (key, index) pairs it has seen as a sorted list, two
// per lane (positions lane and lane + 32).  A chunk of 32 new elements is sorted in
// registers and merged in: the 64 smallest of the list and the chunk are
// min(list[i], chunk[63 - i]) (the chunk padded with +inf), a bitonic sequence that six
// compare-exchange stages sort.  The warps' lists are then merged pairwise in shared
// memory, five levels for 32 warps.  (key, index) order is the stable sort's, so the
// first k of the final list are the stable top-k.
struct KI {
    unsigned long long k;
    int i;
};
__device__ __forceinline__ bool ki_less(const KI& a, const KI& b) { return a.k < b.k || (a.k == b.k && a.i < b.i); }
__device__ __forceinline__ KI ki_shfl_xor(const KI& v, int m) {
    return KI{__shfl_xor_sync(0xffffffffu, v.k, m), __shfl_xor_sync(0xffffffffu, v.i, m)};
}
__device__ __forceinline__ KI ki_shfl(const KI& v, int src) {
    return KI{__shfl_sync(0xffffffffu, v.k, src), __shfl_sync(0xffffffffu, v.i, src)};
}
__device__ __forceinline__ KI ki_min(const KI& a, const KI& b) { return ki_less(b, a) ? b : a; }
__device__ __forceinline__ KI ki_max(const KI& a, const KI& b) { return ki_less(b, a) ? a : b; }

// ascending bitonic sort of one element per lane
__device__ __forceinline__ KI warp_sort32(KI v, int lane) {
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            const KI o = ki_shfl_xor(v, stride);
            const bool lower = (lane & stride) == 0, up = (lane & size) == 0 || size == 32;
            const bool take = lower == up ? ki_less(o, v) : ki_less(v, o);
            if (take) v = o;
        }
    return v;
}

// (a, b) = positions lane and lane + 32 of a bitonic 64-sequence -> sorted ascending
__device__ __forceinline__ void warp_bitonic64(KI& a, KI& b, int lane) {
    const KI lo = ki_min(a, b), hi = ki_max(a, b);
    a = lo;
    b = hi;
#pragma unroll
    for (int stride = 16; stride > 0; stride >>= 1) {
        const bool lower = (lane & stride) == 0;
        const KI oa = ki_shfl_xor(a, stride), ob = ki_shfl_xor(b, stride);
        a = lower ? ki_min(a, oa) : ki_max(a, oa);
        b = lower ? ki_min(b, ob) : ki_max(b, ob);
    }
}

// the 64 smallest of the sorted list (a, b) and the sorted 64-list (c, d), sorted
__device__ __forceinline__ void warp_merge64(KI& a, KI& b, KI c, KI d, int lane) {
    // reversed second list: position i holds element 63 - i
    const KI rc = ki_shfl(d, 31 - lane), rd = ki_shfl(c, 31 - lane);
    a = ki_min(a, rc);
    b = ki_min(b, rd);
    warp_bitonic64(a, b, lane);
}


// the sorted 64-list (a, b) of this warp into shared memory
__device__ __forceinline__ void ki_store64(unsigned long long* sk, int* si, const KI& a, const KI& b, int lane) {
    sk[lane] = a.k; si[lane] = a.i;
    sk[lane + 32] = b.k; si[lane + 32] = b.i;
}

}  // namespace binder
