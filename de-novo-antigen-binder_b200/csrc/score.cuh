// score.cuh — the all-atom pair energy of one group of candidate atoms (a residue,
// or a few consecutive GpuAtoms) against a resident antigen, warp-wide: the device
// code shared by the scoring kernels (k_score.cu) and the post-search kernels
// (k_post.cu).  Pair math: the LJ/Coulomb/hydrophobic part of
// interaction_energy_atoms_breakdown (energy.rs:261-301), with H-bond
// (energy.rs:303-307, 32-39) and EEF1 solvation (solvation.rs:34-84) when FULL.
// f32 pair terms with rsqrt, per-lane compensated (Kahan) sums.
//
// Each translation unit that includes this header owns a copy of the constant
// tables and fills it with score_tables_init() (no relocatable device code).
#pragma once

#include "kernels.h"

namespace binder {

static __constant__ float4 c_slot_prm[N_AA][SLOT_STRIDE];  // q*sqrt(332), r_min_half, sqrt(eps), hydrophobic
static __constant__ int c_slot_type[N_AA][SLOT_STRIDE];
static __constant__ int c_topo_n[N_AA];
static __constant__ float4 c_eef1[16];  // dg_ref, vol, lambda, 1/(PI32*lambda^3)
static __constant__ int c_hb[16];       // bit0 donor, bit1 acceptor

static const float SQRT_COULOMB_K = 18.220867f;  // sqrt(332) in f32

// Fills this translation unit's copy of the tables.
static cudaError_t score_tables_init() {
    float4 slot[N_AA][SLOT_STRIDE];
    int stype[N_AA][SLOT_STRIDE];
    for (int a = 0; a < N_AA; ++a)
        for (int k = 0; k < SLOT_STRIDE; ++k) {
            if (k < BT_TOPO_N[a]) {
                int t = BT_SLOT_TYPE[a][k];
                slot[a][k] = make_float4(BT_SLOT_Q[a][k] * SQRT_COULOMB_K, BT_NB[t][0], sqrtf(BT_NB[t][1]),
                                         BT_SLOT_HYD[a][k] == 1 ? 1.0f : 0.0f);
                stype[a][k] = t;
            } else {
                slot[a][k] = make_float4(0.f, 0.f, 0.f, 0.f);
                stype[a][k] = 0;
            }
        }
    float4 eef[16];
    int hb[16];
    for (int t = 0; t < 16; ++t) {
        float lam = BT_EEF1[t][2];
        eef[t] = make_float4(BT_EEF1[t][0], BT_EEF1[t][1], lam, 1.0f / (PI32 * (lam * lam * lam)));
        hb[t] = BT_HB[t];
    }
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(c_slot_prm, slot, sizeof(slot))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_slot_type, stype, sizeof(stype))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_topo_n, BT_TOPO_N, sizeof(BT_TOPO_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_eef1, eef, sizeof(eef))) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_hb, hb, sizeof(hb));
}

struct AtomIn {
    float x, y, z, qs, rmh, se, h;
    int type;
};

struct Acc {
    float s, c;      // Kahan sum and compensation
    float abs_s;     // sum of |pair terms| (condition number), plain f32
    float fx, fy, fz;
    int pairs;
};

template <bool KAHAN>
__device__ __forceinline__ void acc_add(Acc& a, float v) {
    if (KAHAN) {
        float y = v - a.c;
        float t = a.s + y;
        a.c = (t - a.s) - y;
        a.s = t;
    } else {
        a.s += v;
    }
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ bool finite3(float x, float y, float z) { return isfinite(x) && isfinite(y) && isfinite(z); }

// Fixed-order CTA reduction of one double per warp; thread 0 gets the total.
template <int NW>
__device__ __forceinline__ double cta_sum(double v, double* sm, int lane, int warp) {
    v = warp_sum_d(v);
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NW; ++w) t += sm[w];
    __syncthreads();
    return t;
}

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// ---- grouped scoring: one warp per group of <= 16 nearby candidate atoms ----------
// A group (a residue of the resident state, or 8 consecutive GpuAtoms) sits in
// shared memory.  The warp walks the grid columns within 10 A + group radius of
// the group centre (warp-uniform loop, lanes stride a column's contiguous atom
// range), keeps the antigen atoms that pass a sphere test in a per-warp queue, and
// evaluates full batches of 32 queued atoms against every group atom — so the
// pair math never runs on idle lanes.  Every lane visits its antigen atoms in
// increasing grid order, which keeps the sums deterministic.
constexpr int GMAX = 16;
constexpr int FLAT_GROUP = 8;

// Group atom coordinates also as separate x / y / z arrays, so that the pair test
// reads two atoms' coordinates as one 8-byte word; entries n..GMAX-1 hold GROUP_PAD.
constexpr float GROUP_PAD = 1e30f;  // its squared distance to any atom overflows to +inf

struct GroupSmem {
    float4 pos[GMAX];  // x, y, z, q*sqrt(332)
    float4 prm[GMAX];  // r_min_half, sqrt(epsilon), hydrophobic, AMBER type
    __align__(8) float sx[GMAX];
    __align__(8) float sy[GMAX];
    __align__(8) float sz[GMAX];
    // charge * sqrt(332), r_min_half, sqrt(epsilon), hydrophobic as separate arrays too,
    // so that the pair terms read two atoms' parameters as one 8-byte word
    __align__(8) float sqs[GMAX];
    __align__(8) float srm[GMAX];
    __align__(8) float sse[GMAX];
    __align__(8) float shy[GMAX];
    int q[64];         // queued antigen atom indices
};

__device__ __forceinline__ void group_xyz(GroupSmem& s, int lane, int n, float x, float y, float z) {
    if (lane < n) {
        s.sx[lane] = x;
        s.sy[lane] = y;
        s.sz[lane] = z;
    } else if (lane < GMAX) {
        s.sx[lane] = s.sy[lane] = s.sz[lane] = GROUP_PAD;
    }
}
// the parameter arrays of group atom `lane` (pads: zeros, finite terms never added)
__device__ __forceinline__ void group_prm(GroupSmem& s, int lane, int n, float qs, float rmh, float se, float hy) {
    if (lane < n) {
        s.sqs[lane] = qs;
        s.srm[lane] = rmh;
        s.sse[lane] = se;
        s.shy[lane] = hy;
    } else if (lane < GMAX) {
        s.sqs[lane] = s.srm[lane] = s.sse[lane] = s.shy[lane] = 0.0f;
    }
}

// Energy of one pair within the cutoff (r2: the reference's rounding of r^2):
// candidate atom b / bp, antigen atom a / ap, each (x, y, z, q sqrt(332)) and
// (r_min_half, sqrt(epsilon), hydrophobic, AMBER type).  LJ + Coulomb + hydrophobic
// (energy.rs:269-301), with FULL the H-bond (energy.rs:303-307) and EEF1 solvation
// (solvation.rs:34-50: ei the antigen atom's, ej the candidate atom's) terms; the
// first three are returned in lj, coul, hyd as well.
template <bool FULL>
__device__ __forceinline__ float pair_energy(const float4& b, const float4& bp, const float4& a, const float4& ap,
                                             float r2, float& lj, float& coul, float& hyd) {
    const float ir = rsqrtf(r2);
    const float ir2 = ir * ir;
    const float R = bp.x + ap.x;
    const float s2 = R * R * ir2;
    const float s6 = s2 * s2 * s2;
    lj = (bp.y * ap.y) * (s6 * (s6 - 2.0f));
    coul = (b.w * a.w) * ir;
    hyd = (r2 < HYDRO_CUTOFF_SQ) ? HYDRO_BONUS * (bp.z * ap.z) : 0.0f;
    float e = lj + coul + hyd;
    if (FULL) {
        const int bt = (int)bp.w, at = (int)ap.w;
        if ((((c_hb[bt] & 1) && (c_hb[at] & 2)) || ((c_hb[bt] & 2) && (c_hb[at] & 1))) && r2 <= HB_CUTOFF_SQ) {
            const float z = (r2 * ir - HB_R0) / HB_SIGMA;
            e += -HB_DEPTH * expf(-0.5f * z * z);
        }
        const float4 ej = c_eef1[bt];
        if (r2 < SOLV_CUTOFF_SQ && !(ej.y == 0.0f && ej.x == 0.0f)) {
            const float4 ei = c_eef1[at];
            const float r = r2 * ir;
            const float xi = r / ei.z, xj = r / ej.z;
            e += -(ei.x * ej.y * expf(-(xi * xi)) * ei.w + ej.x * ei.y * expf(-(xj * xj)) * ej.w);
        }
    }
    return e;
}

// One antigen atom (this lane's) against the n group atoms in shared memory, two
// group atoms per step: dx = b - a in packed f32x2 arithmetic, r^2 = (dx*dx + dy*dy)
// + dz*dz with the reference's roundings (scalar, never fused), hence its pair set;
// the terms of the pairs within the cutoff (packed) are added in group-atom order.
template <bool KAHAN, bool FULL, bool ABS, bool COUNT>
__device__ __forceinline__ void group_pairs(const float4* __restrict__ pq, const float4* __restrict__ prm,
                                            const GroupSmem& s, int n, int idx, Acc& acc) {
    const float4 a = __ldg(&pq[idx]);
    const float4 ap = __ldg(&prm[idx]);
    float part = 0.0f, pabs = 0.0f;
    int np = 0;
    auto term = [&](int j, float r2) {
        float lj, coul, hyd;
        const float e = pair_energy<FULL>(s.pos[j], s.prm[j], a, ap, r2, lj, coul, hyd);
        part += e;
        if (ABS) pabs += fabsf(lj) + fabsf(coul) + fabsf(hyd);
        if (COUNT) ++np;
    };
    const uint64_t ax = f2_pack(a.x, a.x), ay = f2_pack(a.y, a.y), az = f2_pack(a.z, a.z);
    const uint64_t aq = f2_pack(a.w, a.w), arm = f2_pack(ap.x, ap.x), ase = f2_pack(ap.y, ap.y);
    const uint64_t ahy = f2_pack(HYDRO_BONUS * ap.z, HYDRO_BONUS * ap.z), two = f2_pack(2.0f, 2.0f);
#pragma unroll 1
    for (int j = 0; j < n; j += 2) {
        const uint64_t dx = f2_sub(*(const uint64_t*)&s.sx[j], ax);
        const uint64_t dy = f2_sub(*(const uint64_t*)&s.sy[j], ay);
        const uint64_t dz = f2_sub(*(const uint64_t*)&s.sz[j], az);
        float r2a, r2b;
        f2_dist2(dx, dy, dz, r2a, r2b);
        const bool ina = r2a <= CUTOFF_SQ && r2a >= MIN_R_SQ;
        const bool inb = r2b <= CUTOFF_SQ && r2b >= MIN_R_SQ;  // j + 1 = n: a pad, +inf
        if (FULL) {
            if (ina) term(j, r2a);
            if (inb) term(j + 1, r2b);
        } else if (ina || inb) {
            // both pairs' terms in packed f32x2 arithmetic; an out-of-range element is
            // computed but never added
            const uint64_t ir = f2_pack(rsqrtf(r2a), rsqrtf(r2b));
            const uint64_t ir2 = f2_mul(ir, ir);
            const uint64_t R = f2_add(*(const uint64_t*)&s.srm[j], arm);
            const uint64_t s2 = f2_mul(f2_mul(R, R), ir2);
            const uint64_t s6 = f2_mul(f2_mul(s2, s2), s2);
            const uint64_t lj = f2_mul(f2_mul(*(const uint64_t*)&s.sse[j], ase), f2_mul(s6, f2_sub(s6, two)));
            const uint64_t coul = f2_mul(f2_mul(*(const uint64_t*)&s.sqs[j], aq), ir);
            const uint64_t hy = f2_mul(*(const uint64_t*)&s.shy[j], ahy);
            const float hya = r2a < HYDRO_CUTOFF_SQ ? f2_lo(hy) : 0.0f;
            const float hyb = r2b < HYDRO_CUTOFF_SQ ? f2_hi(hy) : 0.0f;
            const uint64_t e = f2_add(f2_add(lj, coul), f2_pack(hya, hyb));
            if (ina) part += f2_lo(e);
            if (inb) part += f2_hi(e);
            if (ABS) {
                if (ina) pabs += fabsf(f2_lo(lj)) + fabsf(f2_lo(coul)) + fabsf(hya);
                if (inb) pabs += fabsf(f2_hi(lj)) + fabsf(f2_hi(coul)) + fabsf(hyb);
            }
            if (COUNT) np += (int)ina + (int)inb;
        }
    }
    acc_add<KAHAN>(acc, part);
    if (ABS) acc.abs_s += pabs;
    if (COUNT) acc.pairs += np;
}

// Everything one warp does for one group already in shared memory (n atoms): centre
// and radius, warp-uniform walk over the culled grid columns, sphere prefilter into
// the queue, batched pair evaluation.  Accumulates into the lane's acc.
template <bool KAHAN, bool FULL, bool ABS, bool COUNT>
__device__ __forceinline__ void score_group(const AgView* __restrict__ Ap, GroupSmem& s, int n, int lane,
                                            unsigned lt, Acc& acc) {
    const float4* __restrict__ pq = Ap->pq;
    const float4* __restrict__ prm = Ap->prm;
    const int* __restrict__ cell_start = Ap->grid.cell_start;
    const float inv = Ap->grid.inv;
    const int ox = Ap->grid.ox, oy = Ap->grid.oy, oz = Ap->grid.oz;
    const int gnx = Ap->grid.nx, gny = Ap->grid.ny, gnz = Ap->grid.nz;
    // group centre and radius
    float px = 0.f, py = 0.f, pz = 0.f;
    if (lane < n) {
        const float4 p = s.pos[lane];
        px = p.x; py = p.y; pz = p.z;
    }
    const float inv_n = 1.0f / (float)n;
    const float cx = warp_sum_f(px) * inv_n, cy = warp_sum_f(py) * inv_n, cz = warp_sum_f(pz) * inv_n;
    const float dgx = px - cx, dgy = py - cy, dgz = pz - cz;
    const float rad2 = warp_max_f(lane < n ? dgx * dgx + dgy * dgy + dgz * dgz : 0.0f);
    const float reach = 10.01f + sqrtf(rad2) * 1.0001f + 1e-3f;
    const float reach2 = reach * reach;
    // grid columns within reach of the centre (cell units)
    const float ux = cx * inv - (float)ox, uy = cy * inv - (float)oy, uz = cz * inv - (float)oz;
    const float rc = reach * inv, rc2 = rc * rc;
    const int i0 = max(0, (int)floorf(ux - rc)), i1 = min(gnx - 1, (int)floorf(ux + rc));
    const int j0 = max(0, (int)floorf(uy - rc)), j1 = min(gny - 1, (int)floorf(uy + rc));
    // the columns (i, j) in x-major order, 32 at a time: each lane finds one column's
    // atom range (z-run of cells within reach) in parallel, then the warp takes the
    // non-empty ranges in column order
    const int nj = j1 - j0 + 1;
    const int ncol = (i1 >= i0 && j1 >= j0) ? (i1 - i0 + 1) * nj : 0;
    int qn = 0;
    for (int c0 = 0; c0 < ncol; c0 += 32) {
        int ra0 = 0, ra1 = 0;
        if (c0 + lane < ncol) {
            const int i = i0 + (c0 + lane) / nj, j = j0 + (c0 + lane) % nj;
            const float ddx = fmaxf(fmaxf((float)i - ux, ux - (float)(i + 1)), 0.0f);
            const float ddy = fmaxf(fmaxf((float)j - uy, uy - (float)(j + 1)), 0.0f);
            const float rem2 = rc2 - ddx * ddx - ddy * ddy;
            if (rem2 >= 0.0f) {
                const float rem = sqrtf(rem2);
                const int k0 = max(0, (int)floorf(uz - rem)), k1 = min(gnz - 1, (int)floorf(uz + rem));
                if (k0 <= k1) {
                    const int base = (i * gny + j) * gnz;
                    ra0 = __ldg(&cell_start[base + k0]);
                    ra1 = __ldg(&cell_start[base + k1 + 1]);
                }
            }
        }
        unsigned live = __ballot_sync(0xffffffffu, ra1 > ra0);
        while (live) {
            const int src = __ffs(live) - 1;
            live &= live - 1;
            const int a0 = __shfl_sync(0xffffffffu, ra0, src), a1 = __shfl_sync(0xffffffffu, ra1, src);
            for (int t0 = a0; t0 < a1; t0 += 32) {
                const int t = t0 + lane;
                bool pass = false;
                if (t < a1) {
                    const float4 a = __ldg(&pq[t]);
                    const float ex = a.x - cx, ey = a.y - cy, ez = a.z - cz;
                    pass = ex * ex + ey * ey + ez * ez <= reach2;
                }
                const unsigned m = __ballot_sync(0xffffffffu, pass);
                if (pass) s.q[qn + __popc(m & lt)] = t;
                qn += __popc(m);
                __syncwarp();
                if (qn >= 32) {
                    group_pairs<KAHAN, FULL, ABS, COUNT>(pq, prm, s, n, s.q[lane], acc);
                    __syncwarp();
                    if (lane < qn - 32) s.q[lane] = s.q[32 + lane];
                    qn -= 32;
                    __syncwarp();
                }
            }
        }
    }
    if (lane < qn) group_pairs<KAHAN, FULL, ABS, COUNT>(pq, prm, s, n, s.q[lane], acc);
    __syncwarp();
}


}  // namespace binder
