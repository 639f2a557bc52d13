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
#include "score.cuh"
#include "topk.cuh"

namespace binder {

cudaError_t score_init_tables() { return score_tables_init(); }

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
                                e += -HB_DEPTH * expf(-0.5f * z * z);
                            }
                        }
                        const float4 ej = c_eef1[b.type];
                        if (r2 < SOLV_CUTOFF_SQ && !(ej.y == 0.0f && ej.x == 0.0f)) {
                            const float4 ei = c_eef1[at];
                            const float r = r2 * ir;
                            const float xi = r / ei.z, xj = r / ej.z;
                            const float fi = expf(-(xi * xi)) * ei.w;
                            const float fj = expf(-(xj * xj)) * ej.w;
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

struct SrcStateG {
    StateView st;
    __device__ int ag(int c) const { return st.cand_ag[c]; }
    __device__ int n_groups(int c) const { return st.cand_res_off[c + 1] - st.cand_res_off[c]; }
    __device__ int load(int c, int g, int lane, GroupSmem& s, bool& bad) const {
        const int r = st.cand_res_off[c] + g;
        const int aa = st.res_aa[r];
        const int n = c_topo_n[aa];
        if (lane < n) {
            const float4 p = st.res_pos[(size_t)r * SLOT_STRIDE + lane];
            const float4 m = c_slot_prm[aa][lane];
            bad = !finite3(p.x, p.y, p.z);
            s.pos[lane] = make_float4(p.x, p.y, p.z, m.x);
            s.prm[lane] = make_float4(m.y, m.z, m.w, (float)c_slot_type[aa][lane]);
            group_xyz(s, lane, n, p.x, p.y, p.z);
            group_prm(s, lane, n, m.x, m.y, m.z, m.w);
        } else {
            group_xyz(s, lane, n, 0.f, 0.f, 0.f);
            group_prm(s, lane, n, 0.f, 0.f, 0.f, 0.f);
        }
        return n;
    }
};

struct SrcFlatG {
    const float4* atoms;  // binder_gpu_atom = 2 x float4
    const long long* off;
    const int* cand_ag;
    __device__ int ag(int c) const { return cand_ag ? cand_ag[c] : 0; }
    __device__ int n_groups(int c) const {
        return (int)((off[c + 1] - off[c] + FLAT_GROUP - 1) / FLAT_GROUP);
    }
    __device__ int load(int c, int g, int lane, GroupSmem& s, bool& bad) const {
        const long long j0 = off[c] + (long long)g * FLAT_GROUP;
        const int n = (int)min((long long)FLAT_GROUP, off[c + 1] - j0);
        if (lane < n) {
            const float4 p0 = __ldg(&atoms[2 * (j0 + lane)]);
            const float4 p1 = __ldg(&atoms[2 * (j0 + lane) + 1]);
            bad = !finite3(p0.x, p0.y, p0.z);
            s.pos[lane] = make_float4(p0.x, p0.y, p0.z, p0.w * SQRT_COULOMB_K);
            s.prm[lane] = make_float4(p1.x, sqrtf(p1.y), p1.z > 0.5f ? 1.0f : 0.0f, 0.0f);
            group_xyz(s, lane, n, p0.x, p0.y, p0.z);
            group_prm(s, lane, n, s.pos[lane].w, s.prm[lane].x, s.prm[lane].y, s.prm[lane].z);
        } else {
            group_xyz(s, lane, n, 0.f, 0.f, 0.f);
            group_prm(s, lane, n, 0.f, 0.f, 0.f, 0.f);
        }
        return n;
    }
};

// Resident state: persistent warps take residues from a work queue (an atomic
// counter; residues in index order, or in Calpha-cell order so that neighbouring
// warps share antigen atoms in L1 -- whichever the autotuner timed faster) and
// write one FP64 energy per residue; k_sum_residues adds a candidate's residues in
// index order.  No CTA barrier: warps never wait for each other.
template <int NW, bool KAHAN, bool FULL, bool ABS, bool COUNT>
__global__ void __launch_bounds__(NW * 32) k_score_residues(StateView st, const AgView* __restrict__ ags,
                                                             const int* __restrict__ order, int* __restrict__ queue,
                                                             double* __restrict__ res_e, double* __restrict__ res_abs,
                                                             long long* __restrict__ pair_count,
                                                             uint32_t* __restrict__ err) {
    __shared__ GroupSmem gs[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    GroupSmem& s = gs[warp];
    SrcStateG src{st};
    int my_pairs = 0;
    for (;;) {
        int gi = 0;
        if (lane == 0) gi = atomicAdd(queue, 1);
        gi = __shfl_sync(0xffffffffu, gi, 0);
        if (gi >= st.total_res) break;
        const int r = order ? order[gi] : gi;
        const int c = st.res_cand[r];
        bool bad = false;
        const int n = src.load(c, r - st.cand_res_off[c], lane, s, bad);
        Acc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
        if (__any_sync(0xffffffffu, bad)) {
            if (lane == 0) atomicOr(err, ERRF_NAN);
        } else if (n > 0) {
            __syncwarp();
            score_group<KAHAN, FULL, ABS, COUNT>(&ags[st.cand_ag[c]], s, n, lane, lt, acc);
        }
        __syncwarp();
        const double e = warp_sum_d(KAHAN ? ((double)acc.s - (double)acc.c) : (double)acc.s);
        const double ea = ABS ? warp_sum_d((double)acc.abs_s) : 0.0;
        if (lane == 0) {
            if (res_e) res_e[r] = e;
            if (ABS) res_abs[r] = ea;
        }
        if (COUNT) my_pairs += acc.pairs;
    }
    if (COUNT) {
        int p = my_pairs;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0 && p) atomicAdd((unsigned long long*)pair_count, (unsigned long long)p);
    }
    queue_retire(queue);
}

template <class Src, int NW, bool KAHAN, bool FULL, bool ABS, bool COUNT>
__global__ void __launch_bounds__(NW * 32) k_score_grouped(Src src, int n_cand, const AgView* __restrict__ ags,
                                                            double* __restrict__ out, double* __restrict__ out_abs,
                                                            long long* __restrict__ pair_count,
                                                            uint32_t* __restrict__ err) {
    __shared__ GroupSmem gs[NW];
    __shared__ double sm[NW];
    __shared__ double sm2[NW];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    GroupSmem& s = gs[warp];
    int my_pairs = 0;
    for (int c = blockIdx.x; c < n_cand; c += gridDim.x) {
        const AgView* Ap = &ags[src.ag(c)];
        Acc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
        const int ng = src.n_groups(c);
        for (int gi = warp; gi < ng; gi += NW) {
            bool bad = false;
            const int n = src.load(c, gi, lane, s, bad);
            if (__any_sync(0xffffffffu, bad)) {
                if (lane == 0) atomicOr(err, ERRF_NAN);
                __syncwarp();
                continue;
            }
            if (n == 0) continue;
            __syncwarp();
            score_group<KAHAN, FULL, ABS, COUNT>(Ap, s, n, lane, lt, acc);
        }
        const double lane_e = KAHAN ? ((double)acc.s - (double)acc.c) : (double)acc.s;
        const double e = cta_sum<NW>(lane_e, sm, lane, warp);
        double ea = 0.0;
        if (ABS) ea = cta_sum<NW>((double)acc.abs_s, sm2, lane, warp);
        if (COUNT) my_pairs += acc.pairs;
        if (threadIdx.x == 0) {
            if (out) out[c] = e;
            if (ABS) out_abs[c] = ea;
        }
    }
    if (COUNT) {
        int p = my_pairs;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0 && p) atomicAdd((unsigned long long*)pair_count, (unsigned long long)p);
    }
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

// ---- launchers ----------------------------------------------------------------------
constexpr int NW_SCORE = 8;

// disulfide_energy (allatom.rs:155-180) of candidate c of the resident state: Gaussian
// well between every pair of Cys SG atoms (topology atom 5), reference f32 order.
__device__ float disulfide_energy(const StateView& st, int c) {
    const int r0 = st.cand_res_off[c], r1 = st.cand_res_off[c + 1];
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
            ds = xsub(ds, xmul(4.0f, mc_exp(xmul(xmul(-0.5f, z), z))));
        }
    }
    return ds;
}

__global__ void k_add_disulfide(StateView st, double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < st.n_cand) out[c] += (double)disulfide_energy(st, c);
}

template <class Src>
static void grouped(cudaStream_t s, const Src& src, int n_cand, const AgView* ags, bool kahan, bool full, bool abs_,
                    bool count, const ScoreOut& o, int g) {
#define BINDER_G(K, FU, A, C) \
    k_score_grouped<Src, NW_SCORE, K, FU, A, C><<<g, NW_SCORE * 32, 0, s>>>(src, n_cand, ags, o.energy, o.abs_sum, \
                                                                          o.pairs, o.err)
    if (count) BINDER_G(true, false, false, true);
    else if (full) BINDER_G(true, true, false, false);
    else if (abs_) { if (kahan) BINDER_G(true, false, true, false); else BINDER_G(false, false, true, false); }
    else { if (kahan) BINDER_G(true, false, false, false); else BINDER_G(false, false, false, false); }
#undef BINDER_G
}

int launch_score_flat(cudaStream_t s, const float* atoms, const long long* offsets, int n_cand, const AgView* ags,
                      const int* cand_ag, int accumulate, const ScoreOut& o, int grid_ctas, int block) {
    (void)block;
    if (n_cand <= 0) return 0;
    const float4* a4 = reinterpret_cast<const float4*>(atoms);
    const int g = grid_ctas > 0 ? min(grid_ctas, n_cand) : n_cand;
    const bool kahan = accumulate == 0;
    if (o.force) {  // per-atom warps: each warp owns one candidate atom's force
        if (kahan)
            k_score_flat<NW_SCORE, true, false, true, false><<<g, NW_SCORE * 32, 0, s>>>(
                a4, offsets, n_cand, ags, cand_ag, o.energy, o.abs_sum, o.force, o.pairs, o.err);
        else
            k_score_flat<NW_SCORE, false, false, true, false><<<g, NW_SCORE * 32, 0, s>>>(
                a4, offsets, n_cand, ags, cand_ag, o.energy, o.abs_sum, o.force, o.pairs, o.err);
        return 1;
    }
    SrcFlatG src{a4, offsets, cand_ag};
    grouped(s, src, n_cand, ags, kahan, false, o.abs_sum != nullptr, o.pairs != nullptr, o, g);
    return 1;
}

// candidate energy = its residues' energies added in index order (+ disulfide when full)
__global__ void k_sum_residues(StateView st, const double* __restrict__ res_e, const double* __restrict__ res_abs,
                               int full, double* __restrict__ out, double* __restrict__ out_abs) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= st.n_cand) return;
    double e = 0.0, ea = 0.0;
    for (int r = st.cand_res_off[c]; r < st.cand_res_off[c + 1]; ++r) {
        e += res_e[r];
        if (res_abs) ea += res_abs[r];
    }
    if (full) e += (double)disulfide_energy(st, c);
    out[c] = e;
    if (out_abs) out_abs[c] = ea;
}

// Candidate sums and survivor selection in one launch (k <= 64, segments of at most
// SS_MAX candidates): one CTA per segment.  Thread t adds the residue energies of the
// segment's entries t, t + 1024, ... in residue order (the k_sum_residues sums, loads
// issued ahead of the additions) and keeps their order-preserving keys.  A radix select, 8 bits
// of the 64-bit key per pass from the top, finds the bucket that holds the k-th
// smallest key: every key below it is a survivor, and of the keys in it (all equal
// after the last pass) the ones earliest in the segment, which is candidate-index
// order.  One warp sorts the k survivors by (key, index): the stable top-k of the
// segment, as k_topk64 computes it.  A pass costs three barriers; it ends early
// once the bucket holds exactly the survivors still missing (typically after the
// third pass, when the bucket holds a single key).
constexpr int SS_THREADS = 1024;
constexpr int SS_PER = 4;
constexpr int SS_MAX = SS_THREADS * SS_PER;

__global__ void __launch_bounds__(SS_THREADS) k_sum_select(StateView st, const double* __restrict__ res_e, int full,
                                                           double* __restrict__ out, const int* __restrict__ idx_list,
                                                           const long long* __restrict__ seg_off, int k,
                                                           int* __restrict__ out_idx) {
    __shared__ int s_hist[256];
    __shared__ unsigned long long s_sel_k[64];
    __shared__ int s_sel_i[64];
    __shared__ unsigned long long s_prefix;
    __shared__ int s_need, s_cnt, s_nsel;
    __shared__ unsigned long long s_prefix_tot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int seg = blockIdx.x;
    const long long b0 = seg_off[seg];
    const int n = (int)(seg_off[seg + 1] - b0);
    const int kk = min(k, n);
    // this thread's candidates: segment entries t + SS_THREADS * q
    unsigned long long key[SS_PER];
    int cid[SS_PER];
#pragma unroll
    for (int q = 0; q < SS_PER; ++q) {
        const int j = (int)threadIdx.x + SS_THREADS * q;
        key[q] = 0xFFFFFFFFFFFFFFFFull;
        cid[q] = -1;
        if (j < n) {
            const int c = idx_list ? idx_list[b0 + j] : (int)(b0 + j);
            const int r0 = st.cand_res_off[c], r1 = st.cand_res_off[c + 1];
            double e = 0.0;
            int r = r0;
            for (; r + 4 <= r1; r += 4) {
                const double v0 = res_e[r], v1 = res_e[r + 1], v2 = res_e[r + 2], v3 = res_e[r + 3];
                e += v0;
                e += v1;
                e += v2;
                e += v3;
            }
            for (; r < r1; ++r) e += res_e[r];
            if (full) e += (double)disulfide_energy(st, c);
            out[c] = e;
            key[q] = order_key(e);
            cid[q] = c;
        }
    }
    if (threadIdx.x == 0) {
        s_prefix = 0ull;
        s_need = kk;
        s_cnt = 0;
        s_nsel = 0;
    }
    // ---- radix select of the kk-th smallest key ----
    unsigned long long mask = 0ull;
    bool all_in = false;  // the final bucket holds exactly the survivors still missing
    for (int shift = 56; shift >= 0 && kk > 0; shift -= 8) {
        for (int t = threadIdx.x; t < 256; t += SS_THREADS) s_hist[t] = 0;
        __syncthreads();
        const unsigned long long prefix = s_prefix;
#pragma unroll
        for (int q = 0; q < SS_PER; ++q) {
            if (q * SS_THREADS >= n) break;  // no thread holds entry q
            // one shared atomic per distinct digit of the warp: the lowest lane still
            // pending takes every lane with its digit
            const bool in = cid[q] >= 0 && (key[q] & mask) == prefix;
            const int dg = in ? (int)((key[q] >> shift) & 255ull) : -1;
            unsigned pend = __ballot_sync(0xffffffffu, in);
            while (pend) {
                const int leader = __ffs(pend) - 1;
                const int d = __shfl_sync(0xffffffffu, dg, leader);
                const unsigned same = __ballot_sync(0xffffffffu, in && dg == d);
                if (lane == leader) atomicAdd(&s_hist[d], __popc(same));
                pend &= ~same;
            }
        }
        __syncthreads();
        if (warp == 0) {  // the digit whose bucket holds the s_need-th key
            const int need = s_need;
            int h[8], loc = 0;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                h[i] = s_hist[lane * 8 + i];
                loc += h[i];
            }
            int inc = loc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += v;
            }
            const int exc = inc - loc;
            if (exc < need && need <= inc) {
                int cum = exc;
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    if (cum + h[i] >= need) {
                        s_prefix = prefix | ((unsigned long long)(lane * 8 + i) << shift);
                        s_need = need - cum;
                        s_cnt = h[i];
                        break;
                    }
                    cum += h[i];
                }
            }
        }
        __syncthreads();
        mask |= 0xFFull << shift;
        if (s_cnt == s_need) {
            all_in = true;
            break;
        }
    }
    __syncthreads();
    // ---- the survivors: keys below the bucket, and the bucket's first s_need ----
    const unsigned long long prefix = s_prefix;
    const int need = s_need;
    // rank of each bucket member in segment order (entry t + 1024 q: q major), from a
    // block scan of the per-q membership flags packed 16 bits per q (only needed when
    // the bucket holds more keys than survivors missing)
    int rank[SS_PER] = {0, 0, 0, 0};
    if (!all_in && kk > 0) {
        unsigned long long mine = 0ull;
#pragma unroll
        for (int q = 0; q < SS_PER; ++q)
            if (cid[q] >= 0 && (key[q] & mask) == prefix) mine |= 1ull << (16 * q);
        unsigned long long inc = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long v = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += v;
        }
        __shared__ unsigned long long s_wsum[32];
        if (lane == 31) s_wsum[warp] = inc;
        __syncthreads();
        if (warp == 0) {
            const unsigned long long w = s_wsum[lane];
            unsigned long long wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long v = __shfl_up_sync(0xffffffffu, wi, o);
                if (lane >= o) wi += v;
            }
            s_wsum[lane] = wi - w;
            if (lane == 31) s_prefix_tot = wi;  // per-q totals of the bucket
        }
        __syncthreads();
        const unsigned long long before = s_wsum[warp] + inc - mine;  // earlier threads, per q
        const unsigned long long tot = s_prefix_tot;
        int base = 0;
#pragma unroll
        for (int q = 0; q < SS_PER; ++q) {
            rank[q] = base + (int)((before >> (16 * q)) & 0xFFFFull);
            base += (int)((tot >> (16 * q)) & 0xFFFFull);
        }
    }
#pragma unroll
    for (int q = 0; q < SS_PER; ++q) {
        if (cid[q] < 0 || kk == 0) continue;
        const bool below = key[q] < prefix;  // prefix has zeros under the mask
        bool take = below;
        if (!below && (key[q] & mask) == prefix) take = all_in || rank[q] < need;
        if (take) {
            const int p = atomicAdd(&s_nsel, 1);
            if (p < 64) {
                s_sel_k[p] = key[q];
                s_sel_i[p] = cid[q];
            }
        }
    }
    __syncthreads();
    if (warp == 0) {  // sort the kk survivors by (key, index)
        const KI inf = {0xFFFFFFFFFFFFFFFFull, INT32_MAX};
        KI a = lane < kk ? KI{s_sel_k[lane], s_sel_i[lane]} : inf;
        KI b = lane + 32 < kk ? KI{s_sel_k[lane + 32], s_sel_i[lane + 32]} : inf;
        a = warp_sort32(a, lane);
        b = warp_sort32(b, lane);
        KI hi = inf;
        warp_merge64(a, hi, b, inf, lane);
        int* oi = out_idx + (long long)seg * k;
        if (lane < k) oi[lane] = a.i != INT32_MAX ? a.i : -1;
        if (lane + 32 < k) oi[lane + 32] = hi.i != INT32_MAX ? hi.i : -1;
    }
}

bool sum_topk_fits(int k, long long max_segment) { return k > 0 && k <= 64 && max_segment <= SS_MAX; }

void launch_sum_select(cudaStream_t s, const StateView& st, const double* res_e, int full, double* energy,
                       const SumTopk& tk) {
    if (st.n_cand <= 0 || tk.n_seg <= 0) return;
    k_sum_select<<<tk.n_seg, SS_THREADS, 0, s>>>(st, res_e, full, energy, tk.idx_list, tk.seg_off, tk.k, tk.out_idx);
}

template <int NW>
static void score_residues_nw(cudaStream_t s, int g, const StateView& st, const AgView* ags, bool kahan, bool full,
                              bool abs_, bool count, const ScoreOut& o, const StateScoreScratch& scr) {
#define BINDER_R(K, FU, A, C)                                                                                    \
    k_score_residues<NW, K, FU, A, C><<<g, NW * 32, 0, s>>>(st, ags, scr.order, scr.queue,                      \
                                                            count ? nullptr : scr.res_e, scr.res_abs, o.pairs,  \
                                                            o.err)
    if (count) BINDER_R(true, false, false, true);
    else if (full) BINDER_R(true, true, false, false);
    else if (abs_) { if (kahan) BINDER_R(true, false, true, false); else BINDER_R(false, false, true, false); }
    else { if (kahan) BINDER_R(true, false, false, false); else BINDER_R(false, false, false, false); }
#undef BINDER_R
}

int launch_score_state(cudaStream_t s, const StateView& st, const AgView* ags, int accumulate, int full,
                       const ScoreOut& o, const StateScoreScratch& scr, int grid_ctas, int warps_per_cta,
                       const SumTopk* tk) {
    if (st.n_cand <= 0) return 0;
    const bool kahan = accumulate == 0, abs_ = o.abs_sum != nullptr, count = o.pairs != nullptr;
    const int g = grid_ctas > 0 ? grid_ctas : 148 * 4;
    switch (warps_per_cta) {
        case 4: score_residues_nw<4>(s, g, st, ags, kahan, full, abs_, count, o, scr); break;
        case 16: score_residues_nw<16>(s, g, st, ags, kahan, full, abs_, count, o, scr); break;
        default: score_residues_nw<8>(s, g, st, ags, kahan, full, abs_, count, o, scr); break;
    }
    if (!count && tk && !abs_) {
        if (tk->defer) return 1;  // the sums and the selection come later (launch_sum_select)
        if (tk->mid) cudaEventRecord(tk->mid, s);
        launch_sum_select(s, st, scr.res_e, full, o.energy, *tk);
    } else if (!count) {
        k_sum_residues<<<(st.n_cand + 127) / 128, 128, 0, s>>>(st, scr.res_e, abs_ ? scr.res_abs : nullptr, full,
                                                               o.energy, o.abs_sum);
    }
    return count ? 1 : 2;  // launches issued
}

void launch_score_state_count(cudaStream_t s, const StateView& st, const AgView* ags, long long* pairs,
                              uint32_t* err, const StateScoreScratch& scr, int grid_ctas) {
    if (st.n_cand <= 0) return;
    ScoreOut o{nullptr, nullptr, nullptr, pairs, err};
    launch_score_state(s, st, ags, 0, 0, o, scr, grid_ctas, NW_SCORE);
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
