// k_score.cu — all-atom AMBER LJ + Coulomb + hydrophobic pair energy (and force)
// of candidates against a resident antigen, on the FP32 pipes with rsqrt.
//
// Replaces GpuContext::score_batch (gpu.rs:166-267) and its shader
// (energy.wgsl:47-118), whose pair math is the LJ/Coulomb/hydrophobic part of
// interaction_energy_atoms_breakdown (energy.rs:261-314).  The shader is brute
// force over every antigen atom; here each candidate atom visits only the grid
// columns whose cells can hold an antigen atom within the 10 A cutoff, so the
// pair set is exactly the reference's (0.25 <= r^2 <= 100 with the reference's
// f32 rounding of r^2) at a fraction of the pair tests.
//
// Work decomposition: a persistent grid of CTAs strides over candidates; inside
// a CTA each warp takes one candidate atom at a time and its 32 lanes stride over
// the antigen atoms of each culled column (antigen sorted by cell, so a column's
// z-run of cells is one contiguous range).  Precision: f32 pair terms, per-lane
// compensated (Kahan) sums, FP64 warp-shuffle and cross-warp reductions in a
// fixed order (deterministic).
#include "kernels.h"

namespace binder {

__constant__ float4 c_slot_prm[N_AA][SLOT_STRIDE];  // q*sqrt(332), r_min_half, sqrt(eps), hydrophobic
__constant__ int c_slot_type[N_AA][SLOT_STRIDE];
__constant__ int c_topo_n[N_AA];
__constant__ float4 c_eef1[16];  // dg_ref, vol, lambda, 1/(PI32*lambda^3)
__constant__ int c_hb[16];       // bit0 donor, bit1 acceptor

static const float SQRT_COULOMB_K = 18.220867f;  // sqrt(332) in f32

cudaError_t score_init_tables() {
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

// One candidate atom against every antigen atom within the cutoff; lane-strided.
template <bool KAHAN, bool FULL, bool ABS, bool FORCE, bool COUNT>
__device__ __forceinline__ void atom_vs_antigen(const AgView& A, const AtomIn& b, Acc& acc, int lane) {
    const GridView& g = A.grid;
    const float inv = g.inv;
    const float ux = b.x * inv - (float)g.ox;
    const float uy = b.y * inv - (float)g.oy;
    const float uz = b.z * inv - (float)g.oz;
    const float reach = 10.01f * inv;  // cutoff + margin, in cell units
    const float reach2 = reach * reach;
    const int i0 = max(0, (int)floorf(ux - reach)), i1 = min(g.nx - 1, (int)floorf(ux + reach));
    const int j0 = max(0, (int)floorf(uy - reach)), j1 = min(g.ny - 1, (int)floorf(uy + reach));
    for (int i = i0; i <= i1; ++i) {
        const float ddx = fmaxf(fmaxf((float)i - ux, ux - (float)(i + 1)), 0.0f);
        for (int j = j0; j <= j1; ++j) {
            const float ddy = fmaxf(fmaxf((float)j - uy, uy - (float)(j + 1)), 0.0f);
            const float rem2 = reach2 - ddx * ddx - ddy * ddy;
            if (rem2 < 0.0f) continue;
            const float rem = sqrtf(rem2);
            const int k0 = max(0, (int)floorf(uz - rem)), k1 = min(g.nz - 1, (int)floorf(uz + rem));
            if (k0 > k1) continue;
            const int base = (i * g.ny + j) * g.nz;
            const int a0 = __ldg(&g.cell_start[base + k0]);
            const int a1 = __ldg(&g.cell_start[base + k1 + 1]);
            for (int t = a0 + lane; t < a1; t += 32) {
                const float4 apq = __ldg(&A.pq[t]);
                const float4 aprm = __ldg(&A.prm[t]);
                const float dx = b.x - apq.x, dy = b.y - apq.y, dz = b.z - apq.z;
                const float r2 = xdist2(dx, dy, dz);  // reference rounding: same pair set
                if (r2 <= CUTOFF_SQ && r2 >= MIN_R_SQ) {
                    const float ir = rsqrtf(r2);
                    const float ir2 = ir * ir;
                    const float R = b.rmh + aprm.x;
                    const float s2 = R * R * ir2;
                    const float s6 = s2 * s2 * s2;
                    const float eps = b.se * aprm.y;
                    const float lj = eps * (s6 * (s6 - 2.0f));
                    const float qq = b.qs * apq.w;
                    const float coul = qq * ir;
                    float e = lj + coul;
                    const float hyd = (r2 < HYDRO_CUTOFF_SQ) ? HYDRO_BONUS * (b.h * aprm.z) : 0.0f;
                    e += hyd;
                    if (FULL) {
                        const int at = (int)aprm.w;
                        if (((c_hb[b.type] & 1) && (c_hb[at] & 2)) || ((c_hb[b.type] & 2) && (c_hb[at] & 1))) {
                            if (r2 <= HB_CUTOFF_SQ) {
                                const float r = r2 * ir;
                                const float z = (r - HB_R0) / HB_SIGMA;
                                e += -HB_DEPTH * __expf(-0.5f * z * z);
                            }
                        }
                        const float4 ej = c_eef1[b.type];
                        if (r2 < SOLV_CUTOFF_SQ && !(ej.y == 0.0f && ej.x == 0.0f)) {
                            const float4 ei = c_eef1[at];
                            const float r = r2 * ir;
                            const float xi = r / ei.z, xj = r / ej.z;
                            const float fi = __expf(-(xi * xi)) * ei.w;
                            const float fj = __expf(-(xj * xj)) * ej.w;
                            e += -(ei.x * ej.y * fi + ej.x * ei.y * fj);
                        }
                    }
                    acc_add<KAHAN>(acc, e);
                    if (ABS) acc.abs_s += fabsf(lj) + fabsf(coul) + fabsf(hyd);
                    if (FORCE) {
                        // -dE/dr * r_hat / r : 12 eps (s12 - s6)/r^2 + qq/r^3
                        const float sc = 12.0f * eps * (s6 * (s6 - 1.0f)) * ir2 + coul * ir2;
                        acc.fx += sc * dx;
                        acc.fy += sc * dy;
                        acc.fz += sc * dz;
                    }
                    if (COUNT) acc.pairs++;
                }
            }
        }
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

// ---- flat GpuAtom candidates (binder_gpu_atom = 2 x float4) -------------------------
template <int NW, bool KAHAN, bool ABS, bool FORCE, bool COUNT>
__global__ void __launch_bounds__(NW * 32) k_score_flat(const float4* __restrict__ atoms,
                                                         const long long* __restrict__ off, int n_cand,
                                                         const AgView* __restrict__ ags,
                                                         const int* __restrict__ cand_ag, double* __restrict__ out,
                                                         double* __restrict__ out_abs, float* __restrict__ force,
                                                         long long* __restrict__ pair_count,
                                                         uint32_t* __restrict__ err) {
    __shared__ double sm[NW];
    __shared__ double sm2[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int my_pairs = 0;
    for (int c = blockIdx.x; c < n_cand; c += gridDim.x) {
        const AgView A = ags[cand_ag ? cand_ag[c] : 0];
        const long long a_begin = off[c], a_end = off[c + 1];
        Acc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
        for (long long j = a_begin + warp; j < a_end; j += NW) {
            const float4 p0 = __ldg(&atoms[2 * j]);
            const float4 p1 = __ldg(&atoms[2 * j + 1]);
            if (!finite3(p0.x, p0.y, p0.z)) {
                if (lane == 0) atomicOr(err, ERRF_NAN);
                continue;
            }
            AtomIn b;
            b.x = p0.x; b.y = p0.y; b.z = p0.z;
            b.qs = p0.w * SQRT_COULOMB_K;
            b.rmh = p1.x;
            b.se = sqrtf(p1.y);
            b.h = p1.z > 0.5f ? 1.0f : 0.0f;
            b.type = 0;
            if (FORCE) { acc.fx = 0.f; acc.fy = 0.f; acc.fz = 0.f; }
            atom_vs_antigen<KAHAN, false, ABS, FORCE, COUNT>(A, b, acc, lane);
            if (FORCE) {
                const float fx = warp_sum_f(acc.fx), fy = warp_sum_f(acc.fy), fz = warp_sum_f(acc.fz);
                if (lane == 0) { force[3 * j] = fx; force[3 * j + 1] = fy; force[3 * j + 2] = fz; }
            }
        }
        const double lane_e = KAHAN ? ((double)acc.s - (double)acc.c) : (double)acc.s;
        const double e = cta_sum<NW>(lane_e, sm, lane, warp);
        double ea = 0.0;
        if (ABS) ea = cta_sum<NW>((double)acc.abs_s, sm2, lane, warp);
        if (threadIdx.x == 0) {
            if (out) out[c] = e;
            if (ABS) out_abs[c] = ea;
        }
        if (COUNT) my_pairs += acc.pairs;
    }
    if (COUNT) {
        int p = my_pairs;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0 && p) atomicAdd((unsigned long long*)pair_count, (unsigned long long)p);
    }
}

// ---- resident state (slot layout) -------------------------------------------------
template <int NW, bool KAHAN, bool FULL, bool ABS, bool COUNT>
__global__ void __launch_bounds__(NW * 32) k_score_state(StateView st, const AgView* __restrict__ ags,
                                                          double* __restrict__ out, double* __restrict__ out_abs,
                                                          long long* __restrict__ pair_count,
                                                          uint32_t* __restrict__ err) {
    __shared__ double sm[NW];
    __shared__ double sm2[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int my_pairs = 0;
    for (int c = blockIdx.x; c < st.n_cand; c += gridDim.x) {
        const AgView A = ags[st.cand_ag[c]];
        const int r0 = st.cand_res_off[c], r1 = st.cand_res_off[c + 1];
        const int n_work = (r1 - r0) * SLOT_STRIDE;
        Acc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
        for (int w = warp; w < n_work; w += NW) {
            const int r = r0 + (w >> 4), k = w & (SLOT_STRIDE - 1);
            const int aa = st.res_aa[r];
            if (k >= c_topo_n[aa]) continue;
            const float4 p = st.res_pos[(size_t)r * SLOT_STRIDE + k];
            if (!finite3(p.x, p.y, p.z)) {
                if (lane == 0) atomicOr(err, ERRF_NAN);
                continue;
            }
            const float4 prm = c_slot_prm[aa][k];
            AtomIn b;
            b.x = p.x; b.y = p.y; b.z = p.z;
            b.qs = prm.x; b.rmh = prm.y; b.se = prm.z; b.h = prm.w;
            b.type = c_slot_type[aa][k];
            atom_vs_antigen<KAHAN, FULL, ABS, false, COUNT>(A, b, acc, lane);
        }
        const double lane_e = KAHAN ? ((double)acc.s - (double)acc.c) : (double)acc.s;
        double e = cta_sum<NW>(lane_e, sm, lane, warp);
        double ea = 0.0;
        if (ABS) ea = cta_sum<NW>((double)acc.abs_s, sm2, lane, warp);
        if (FULL) {
            // disulfide_energy (allatom.rs:155-180): Gaussian well between Cys SG atoms
            if (threadIdx.x == 0) {
                float ds = 0.0f;
                for (int ri = r0; ri < r1; ++ri) {
                    if (st.res_aa[ri] != CYS) continue;
                    const float4 pi = st.res_pos[(size_t)ri * SLOT_STRIDE + 5];
                    for (int rj = ri + 1; rj < r1; ++rj) {
                        if (st.res_aa[rj] != CYS) continue;
                        const float4 pj = st.res_pos[(size_t)rj * SLOT_STRIDE + 5];
                        const float d = xsqrt(xdist2(xsub(pi.x, pj.x), xsub(pi.y, pj.y), xsub(pi.z, pj.z)));
                        if (d > 4.0f) continue;
                        const float z = xdiv(xsub(d, 2.05f), 0.4f);
                        ds = xsub(ds, xmul(4.0f, expf(xmul(xmul(-0.5f, z), z))));
                    }
                }
                e += (double)ds;
            }
        }
        if (threadIdx.x == 0) {
            if (out) out[c] = e;
            if (ABS) out_abs[c] = ea;
        }
        if (COUNT) my_pairs += acc.pairs;
    }
    if (COUNT) {
        int p = my_pairs;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0 && p) atomicAdd((unsigned long long*)pair_count, (unsigned long long)p);
    }
}

// ---- launchers ----------------------------------------------------------------------
constexpr int NW_SCORE = 8;

int launch_score_flat(cudaStream_t s, const float* atoms, const long long* offsets, int n_cand, const AgView* ags,
                      const int* cand_ag, int accumulate, const ScoreOut& o, int grid_ctas, int block) {
    (void)block;
    if (n_cand <= 0) return 0;
    const float4* a4 = reinterpret_cast<const float4*>(atoms);
    const int g = grid_ctas > 0 ? min(grid_ctas, n_cand) : n_cand;
    const bool kahan = accumulate == 0;
#define BINDER_FLAT(K, A, F, C)                                                                                 \
    k_score_flat<NW_SCORE, K, A, F, C><<<g, NW_SCORE * 32, 0, s>>>(a4, offsets, n_cand, ags, cand_ag, o.energy, \
                                                                   o.abs_sum, o.force, o.pairs, o.err)
    if (o.force) {
        if (kahan) BINDER_FLAT(true, false, true, false); else BINDER_FLAT(false, false, true, false);
    } else if (o.pairs) {
        BINDER_FLAT(true, false, false, true);
    } else if (o.abs_sum) {
        if (kahan) BINDER_FLAT(true, true, false, false); else BINDER_FLAT(false, true, false, false);
    } else {
        if (kahan) BINDER_FLAT(true, false, false, false); else BINDER_FLAT(false, false, false, false);
    }
#undef BINDER_FLAT
    return 1;
}

int launch_score_state(cudaStream_t s, const StateView& st, const AgView* ags, int accumulate, int full,
                       const ScoreOut& o, int grid_ctas, int block) {
    (void)block;
    if (st.n_cand <= 0) return 0;
    const int g = grid_ctas > 0 ? min(grid_ctas, st.n_cand) : st.n_cand;
    const bool kahan = accumulate == 0;
#define BINDER_STATE(K, FU, A, C) \
    k_score_state<NW_SCORE, K, FU, A, C><<<g, NW_SCORE * 32, 0, s>>>(st, ags, o.energy, o.abs_sum, o.pairs, o.err)
    if (o.pairs) {
        BINDER_STATE(true, false, false, true);
    } else if (full) {
        BINDER_STATE(true, true, false, false);
    } else if (o.abs_sum) {
        if (kahan) BINDER_STATE(true, false, true, false); else BINDER_STATE(false, false, true, false);
    } else {
        if (kahan) BINDER_STATE(true, false, false, false); else BINDER_STATE(false, false, false, false);
    }
#undef BINDER_STATE
    return 1;
}

void launch_score_state_count(cudaStream_t s, const StateView& st, const AgView* ags, long long* pairs,
                              uint32_t* err, int grid_ctas) {
    if (st.n_cand <= 0) return;
    const int g = grid_ctas > 0 ? min(grid_ctas, st.n_cand) : st.n_cand;
    k_score_state<NW_SCORE, true, false, false, true>
        <<<g, NW_SCORE * 32, 0, s>>>(st, ags, nullptr, nullptr, pairs, err);
}

}  // namespace binder

namespace binder {

__global__ void k_uniform_offsets(long long* __restrict__ off, int n_cand, long long n_ab) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c <= n_cand) off[c] = (long long)c * n_ab;
}
void launch_uniform_offsets(cudaStream_t s, long long* off, int n_cand, long long n_ab) {
    k_uniform_offsets<<<(n_cand + 1 + 255) / 256, 256, 0, s>>>(off, n_cand, n_ab);
}

}  // namespace binder
