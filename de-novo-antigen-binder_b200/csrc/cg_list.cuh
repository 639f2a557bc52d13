// cg_list.cuh — per-residue Verlet lists of antigen Calphas for the coarse-grained
// force of compute_forces_with_grid (energy.rs:322-398), shared by the gradient-step
// kernel (k_search.cu) and the Langevin part of the Metropolis kernel (k_anneal.cu).
//
// The reference sums the pair terms in its probe order: cells (cx+dx, cy+dy, cz+dz)
// for dx, dy, dz = -1..1 (dz fastest), atoms ascending within a cell.  The antigen
// Calphas are stored sorted by cell in the same lexicographic order (ascending
// original index within a cell), so that probe order is ascending position in the
// sorted array.  A list holds, ascending, the positions of the Calphas within
// cutoff + skin of a list centre: while the residue's Calpha stays within the skin of
// the centre it holds every in-cutoff Calpha, and its entries that pass the
// reference's tests, taken in list order, are the reference's pairs in the
// reference's order.
#pragma once

#include "geom.cuh"

namespace binder {

constexpr int CG_LIST_MAX = CG_LIST_CAP;
constexpr float CG_SKIN = 2.0f;      // list radius = 10 A cutoff + skin; a residue's first skin
constexpr float CG_SKIN_MAX = 5.0f;  // a residue that outruns its list gets twice the skin, up to this


__device__ __forceinline__ bool cell_far(int cx, int cy, int cz) {
    return abs(cx) > (1 << 29) || abs(cy) > (1 << 29) || abs(cz) > (1 << 29);
}

// Verlet list of the residue whose group of G lanes calls this (gl = lane in group):
// positions (ascending) of the antigen Calphas within skin + 10 A (+ 10 mA for
// rounding) of p, found by a walk over the (2K+1)^3 cells around p's cell, K =
// ceil(radius / cell), culled by slab distance.  The lanes split the (2K+1)^2
// (dx, dy) columns into contiguous runs (for fixed (dx, dy) the cells along z are
// one contiguous range of the sorted array), count, take offsets by a prefix sum
// and write.  Returns the list length (all lanes); a length above CG_LIST_MAX (or a
// grid finer than radius / 8) leaves the list unusable.
template <int G>
__device__ __noinline__ int build_cg_list(const GridView& g, const float4* __restrict__ ca_pq, F3 p, int gl,
                                          unsigned gmask, int* list, float skin) {
    const float R = 10.0f + skin + 0.01f, R2 = R * R;
    const int c[3] = {cell_coord(p.x, g.inv), cell_coord(p.y, g.inv), cell_coord(p.z, g.inv)};
    if (cell_far(c[0], c[1], c[2]) || !(R <= 8.0f * g.cell)) return CG_LIST_MAX + 1;
    const int K = (int)ceilf(R / g.cell), W = 2 * K + 1, ncol = W * W;
    const float pp[3] = {p.x, p.y, p.z};
    auto slab2 = [&](int d, int o) {  // squared distance from p to the cell slab c[d] + o along d
        const float lo = (float)(c[d] + o) * g.cell, hi = lo + g.cell;
        const float dd = fmaxf(fmaxf(lo - pp[d], pp[d] - hi), 0.0f);
        return dd * dd;
    };
    const int col0 = (ncol * gl) / G, col1 = (ncol * (gl + 1)) / G;
    int n_mine = 0, off = 0, total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        int w = off;
        for (int col = col0; col < col1; ++col) {
            const int ox = col / W - K, oy = col % W - K;
            const float dxy = slab2(0, ox) + slab2(1, oy);
            if (dxy > R2) continue;
            const int X = c[0] + ox - g.ox, Y = c[1] + oy - g.oy;
            if (X < 0 || Y < 0 || X >= g.nx || Y >= g.ny) continue;
            int zl = -K, zh = K;
            while (zl <= K && dxy + slab2(2, zl) > R2) ++zl;
            while (zh >= zl && dxy + slab2(2, zh) > R2) --zh;
            if (zl > zh) continue;
            const int Z0 = max(c[2] + zl - g.oz, 0), Z1 = min(c[2] + zh - g.oz, g.nz - 1);
            if (Z0 > Z1) continue;
            const int base = (X * g.ny + Y) * g.nz;
            const int a1 = g.cell_start[base + Z1 + 1];
            for (int i = g.cell_start[base + Z0]; i < a1; ++i) {
                const float4 a = ca_pq[i];
                const float dx = p.x - a.x, dy = p.y - a.y, dz = p.z - a.z;
                if (dx * dx + dy * dy + dz * dz > R2) continue;
                if (pass == 0) ++n_mine;
                else list[w++] = i;
            }
        }
        if (pass == 0) {
            int incl = n_mine;
#pragma unroll
            for (int d = 1; d < G; d <<= 1) {
                const int v = __shfl_up_sync(gmask, incl, d, G);
                if (gl >= d) incl += v;
            }
            total = __shfl_sync(gmask, incl, G - 1, G);
            off = incl - n_mine;
            if (total > CG_LIST_MAX) return total;
        }
    }
    __syncwarp(gmask);
    return total;
}


// The same list built by a whole warp in one pass (positions as T: 16-bit for
// antigens of at most 65536 Calphas, or int): the lanes find the atom ranges of 32
// (dx, dy) columns at a time, a warp prefix sum over the range lengths concatenates
// them in column order (ascending positions), and the warp tests 32 consecutive
// atoms of the concatenation per round, each lane finding its column by a binary
// search over the prefix; a ballot orders the hits.  Writes at most CG_LIST_MAX
// entries to out and returns the length (all lanes; above CG_LIST_MAX: unusable).
template <typename T>
__device__ __noinline__ int build_cg_list_warp(const GridView& g, const float4* __restrict__ ca_pq, F3 p, int lane,
                                               T* out, float skin) {
    const float R = 10.0f + skin + 0.01f, R2 = R * R;
    const int c[3] = {cell_coord(p.x, g.inv), cell_coord(p.y, g.inv), cell_coord(p.z, g.inv)};
    if (cell_far(c[0], c[1], c[2]) || !(R <= 8.0f * g.cell)) return CG_LIST_MAX + 1;
    const int K = (int)ceilf(R / g.cell), W = 2 * K + 1, ncol = W * W;
    const float pp[3] = {p.x, p.y, p.z};
    auto slab2 = [&](int d, int o) {
        const float lo = (float)(c[d] + o) * g.cell, hi = lo + g.cell;
        const float dd = fmaxf(fmaxf(lo - pp[d], pp[d] - hi), 0.0f);
        return dd * dd;
    };
    const unsigned lt = (1u << lane) - 1u;
    int n = 0;
    for (int col0 = 0; col0 < ncol; col0 += 32) {
        // this lane's column: its z-run of cells within R, as a range of sorted positions
        int a0 = 0, len = 0;
        const int col = col0 + lane;
        if (col < ncol) {
            const int ox = col / W - K, oy = col % W - K;
            const float dxy = slab2(0, ox) + slab2(1, oy);
            const int X = c[0] + ox - g.ox, Y = c[1] + oy - g.oy;
            if (dxy <= R2 && X >= 0 && Y >= 0 && X < g.nx && Y < g.ny) {
                int zl = -K, zh = K;
                while (zl <= K && dxy + slab2(2, zl) > R2) ++zl;
                while (zh >= zl && dxy + slab2(2, zh) > R2) --zh;
                const int Z0 = max(c[2] + zl - g.oz, 0), Z1 = min(c[2] + zh - g.oz, g.nz - 1);
                if (zl <= zh && Z0 <= Z1) {
                    const int base = (X * g.ny + Y) * g.nz;
                    a0 = g.cell_start[base + Z0];
                    len = g.cell_start[base + Z1 + 1] - a0;
                }
            }
        }
        int incl = len;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        const int tot = __shfl_sync(0xffffffffu, incl, 31);
        for (int f0 = 0; f0 < tot; f0 += 32) {
            const int f = f0 + lane;
            const int fq = min(f, tot - 1);
            // the first column whose inclusive prefix exceeds fq (every lane searches)
            int lo = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1) {
                const int v = __shfl_sync(0xffffffffu, incl, lo + step - 1);
                if (v <= fq) lo += step;
            }
            const int v_lo = __shfl_sync(0xffffffffu, incl, lo);
            const int len_lo = __shfl_sync(0xffffffffu, len, lo);
            const int a_lo = __shfl_sync(0xffffffffu, a0, lo);
            const int i = a_lo + (fq - (v_lo - len_lo));
            bool hit = false;
            if (f < tot) {
                const float4 a = ca_pq[i];
                const float dx = p.x - a.x, dy = p.y - a.y, dz = p.z - a.z;
                hit = dx * dx + dy * dy + dz * dz <= R2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            const int w = n + __popc(m & lt);
            if (hit && w < CG_LIST_MAX) out[w] = (T)i;
            n += __popc(m);
        }
    }
    __syncwarp();
    return n;
}

constexpr int CG_IN_MAX = 48;      // in-cutoff list entries a residue holds per step
constexpr float CG_NEAR_SQ = 99.0f;  // r^2 below which a pair is in adjacent 10 A cells

}  // namespace binder
