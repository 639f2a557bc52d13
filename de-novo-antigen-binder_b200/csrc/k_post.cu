// k_post.cu — the post-search refinement of the reference's all-atom results on
// the GPU, batched over every resident candidate (main.rs:336-346).
//
//  * minimize (diffusion.rs:854-916) against the candidate's antigen: steepest
//    descent on the Calpha-level grid force (compute_forces_with_grid,
//    energy.rs:322-398) with a step decaying linearly to zero (MIN_STEP 0.04,
//    every component clamped to MIN_MAX_DISP 0.5, diffusion.rs:63-64), the side
//    chains rebuilt from the moved backbone (allatom.rs:244-270), and a step kept
//    only when the all-atom energy (allatom_energy: interaction_energy_atoms +
//    disulfide_energy, diffusion.rs:281-283, 835-840) drops.  Three launches per
//    step: the move of every residue into a trial copy of the positions, the full
//    score of the trial copy, the per-candidate keep-or-restore.
//  * affinity_maturation_allatom (diffusion.rs:924-961) over the interface
//    residues (filters.rs:96-105, main.rs:342-344): one CTA per candidate walks its
//    mutable positions in order; at a position the 19 other amino acids (ALL_AA
//    order, atom.rs:29, each at its top rotamer) and the mutation back to the old
//    amino acid and chi are built at once (mutate_residue, allatom.rs:299-384),
//    their residue energies computed by the warps of the CTA, and the first
//    amino acid whose total is strictly below the best is kept -- the reference's
//    scan, whose candidates differ only in the one residue.
//
// Residue geometry keeps the reference's f32 operation order (bit-identical to
// the CPU restatement); energies are f32 pair terms with compensated sums and
// FP64 totals, so every keep / reject decision is the f64 energy's.
#include <algorithm>
#include <vector>

#include "geom.cuh"
#include "score.cuh"

namespace binder {

cudaError_t post_init_tables() {
    cudaError_t e = geom_init_tables();
    if (e != cudaSuccess) return e;
    return score_tables_init();
}

// ---- minimize -----------------------------------------------------------------------
// One thread per residue: the grid force on the pre-step Calpha (pos_in), the
// clamped move, the translated residue and its rebuilt side chain (pos_out).
__global__ void k_min_move(StateView st, const AgView* __restrict__ ags, const float4* __restrict__ pos_in,
                           float4* __restrict__ pos_out, float step_size) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= st.total_res) return;
    const int aa = st.res_aa[r];
    const AgView& A = ags[st.cand_ag[st.res_cand[r]]];
    const float4* in = pos_in + (size_t)r * SLOT_STRIDE;
    const int n_at = s_topo_n[aa];
    const float4 c4 = in[1];  // Calpha = topology atom 1
    const F3 ca = {c4.x, c4.y, c4.z};
    float fx, fy, fz;
    cg_force(A, cg_body(ca.x, ca.y, ca.z, aa), fx, fy, fz);
    // fx_buf (zeroed) += the one partner's force, then the clamped step (f32 clamp)
    constexpr float MAXD = 0.5f;
    auto clampf = [](float v) { return v < -MAXD ? -MAXD : (v > MAXD ? MAXD : v); };
    const float dx = clampf(xmul(step_size, xadd(0.0f, fx)));
    const float dy = clampf(xmul(step_size, xadd(0.0f, fy)));
    const float dz = clampf(xmul(step_size, xadd(0.0f, fz)));
    const F3 new_ca = {xadd(ca.x, dx), xadd(ca.y, dy), xadd(ca.z, dz)};
    const F3 dl = sub3(new_ca, ca);  // set_ca_pos: every atom += new - old
    F3 atoms[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
        const float4 v = in[k];
        atoms[k] = k < n_at ? F3{xadd(v.x, dl.x), xadd(v.y, dl.y), xadd(v.z, dl.z)} : F3{v.x, v.y, v.z};
    }
    // rebuild_side_chain: the side chain from the moved backbone at the residue's chi
    const int n_bb = aa == GLY ? 4 : 5;
    const ChiTrig ct = unpack_trig(st.res_trig[2 * r], st.res_trig[2 * r + 1]);
    build_side_chain(aa, atoms, n_bb, ct);
    float4* out = pos_out + (size_t)r * SLOT_STRIDE;
#pragma unroll
    for (int k = 0; k < SLOT_STRIDE; ++k)
        out[k] = k < n_at ? make_float4(atoms[k].x, atoms[k].y, atoms[k].z, 0.f) : in[k];
}

// Keep the trial positions of candidate c when its energy is strictly lower.
__global__ void k_min_accept(StateView st, const float4* __restrict__ trial, const double* __restrict__ e_trial,
                             double* __restrict__ best, int* __restrict__ kept) {
    const int c = blockIdx.x;
    __shared__ int s_take;
    if (threadIdx.x == 0) {
        const double e = e_trial[c];
        s_take = e < best[c];
        if (s_take) {
            best[c] = e;
            if (kept) kept[c] += 1;
        }
    }
    __syncthreads();
    if (!s_take) return;
    const size_t s0 = (size_t)st.cand_res_off[c] * SLOT_STRIDE, s1 = (size_t)st.cand_res_off[c + 1] * SLOT_STRIDE;
    for (size_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) st.res_pos[i] = trial[i];
}

void launch_min_move(cudaStream_t s, const StateView& st, const AgView* ags, const float4* pos_in, float4* pos_out,
                     float step_size) {
    if (st.total_res > 0) k_min_move<<<(st.total_res + 127) / 128, 128, 0, s>>>(st, ags, pos_in, pos_out, step_size);
}
void launch_min_accept(cudaStream_t s, const StateView& st, const float4* trial, const double* e_trial, double* best,
                       int* kept) {
    if (st.n_cand > 0) k_min_accept<<<st.n_cand, 128, 0, s>>>(st, trial, e_trial, best, kept);
}

// ---- affinity maturation ------------------------------------------------------------
constexpr int MAT_TRIALS = 20;  // 19 other amino acids + the mutation back
constexpr int MAT_WARPS = 10;

// disulfide_energy (allatom.rs:155-180) of candidate c with residue `rr` replaced by
// (aa_r, sg_r): Gaussian well between every pair of Cys SG atoms (topology atom 5),
// pairs in the reference's order, f32.
__device__ float disulfide_with(const StateView& st, int c, int rr, int aa_r, float4 sg_r) {
    const int r0 = st.cand_res_off[c], r1 = st.cand_res_off[c + 1];
    float ds = 0.0f;
    for (int ri = r0; ri < r1; ++ri) {
        const int ai = ri == rr ? aa_r : st.res_aa[ri];
        if (ai != CYS) continue;
        const float4 pi = ri == rr ? sg_r : st.res_pos[(size_t)ri * SLOT_STRIDE + 5];
        for (int rj = ri + 1; rj < r1; ++rj) {
            const int aj = rj == rr ? aa_r : st.res_aa[rj];
            if (aj != CYS) continue;
            const float4 pj = rj == rr ? sg_r : st.res_pos[(size_t)rj * SLOT_STRIDE + 5];
            const float d = xsqrt(xdist2(xsub(pi.x, pj.x), xsub(pi.y, pj.y), xsub(pi.z, pj.z)));
            if (d > 4.0f) continue;
            const float z = xdiv(xsub(d, 2.05f), 0.4f);
            ds = xsub(ds, xmul(4.0f, mc_exp(xmul(xmul(-0.5f, z), z))));
        }
    }
    return ds;
}

// One CTA per candidate.  res_e: the per-residue full energies of the state (kept
// current); out_best: the final score (the reference's `best`); out_kept:
// mutations kept.
__global__ void __launch_bounds__(MAT_WARPS * 32) k_mature(StateView st, const AgView* __restrict__ ags,
                                                            double* __restrict__ res_e, double* __restrict__ out_best,
                                                            int* __restrict__ out_kept, uint32_t* __restrict__ err) {
    const int c = blockIdx.x;
    const int r0 = st.cand_res_off[c], r1 = st.cand_res_off[c + 1], n = r1 - r0;
    const AgView& A = ags[st.cand_ag[c]];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ GroupSmem gs[MAT_WARPS];
    __shared__ float4 s_pos[MAT_TRIALS][SLOTS];
    __shared__ int s_aa[MAT_TRIALS];
    __shared__ float4 s_chi[MAT_TRIALS], s_trig[MAT_TRIALS][2];
    __shared__ double s_e[MAT_TRIALS];
    __shared__ float s_ds[MAT_TRIALS];
    __shared__ unsigned char s_mut[ANNEAL_MAX_RES];
    __shared__ double s_best;
    __shared__ int s_pick, s_kept;
    if (n > ANNEAL_MAX_RES) {
        if (threadIdx.x == 0) atomicOr(err, ERRF_RANGE);
        return;
    }
    // mutable = interface residues (filters.rs:96-105): an antigen Calpha closer than 8 A
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 p = st.res_pos[(size_t)(r0 + i) * SLOT_STRIDE + 1];
        bool any = false;
        for (int j = 0; j < A.n_res && !any; ++j) {
            const float4 q = A.ca_atom[j];
            any = xdist2(xsub(p.x, q.x), xsub(p.y, q.y), xsub(p.z, q.z)) < 64.0f;
        }
        s_mut[i] = any;
    }
    if (threadIdx.x == 0) {
        double e = 0.0;
        for (int r = r0; r < r1; ++r) e += res_e[r];
        s_best = e + (double)disulfide_with(st, c, -1, 0, make_float4(0.f, 0.f, 0.f, 0.f));
        s_kept = 0;
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
        if (!s_mut[i]) continue;  // CTA-uniform
        const int r = r0 + i;
        const int old_aa = st.res_aa[r];
        // build the trials: t < 19 the t-th other amino acid at its top rotamer, 19 the old one at its chi
        if (threadIdx.x < MAT_TRIALS) {
            const int t = threadIdx.x;
            const float4 c4 = st.res_pos[(size_t)r * SLOT_STRIDE + 1];
            int aa;
            ChiTrig ct;
            float4 chi, tr0, tr1;
            if (t < MAT_TRIALS - 1) {
                aa = t < old_aa ? t : t + 1;
                if (s_rot_n[aa] > 0) {
                    ct = rot_trig(aa, 0);
                    chi = s_rot_chi[aa][0];
                } else {
                    ct = zero_trig();
                    chi = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                tr0 = make_float4(ct.t[0].x, ct.t[0].y, ct.t[1].x, ct.t[1].y);
                tr1 = make_float4(ct.t[2].x, ct.t[2].y, ct.t[3].x, ct.t[3].y);
            } else {
                aa = old_aa;
                tr0 = st.res_trig[2 * r];
                tr1 = st.res_trig[2 * r + 1];
                ct = unpack_trig(tr0, tr1);
                chi = st.res_chi[r];
            }
            F3 atoms[SLOTS];
            const int n_bb = ideal_backbone(F3{c4.x, c4.y, c4.z}, aa, atoms);
            build_side_chain(aa, atoms, n_bb, ct);
            const int n_at = s_topo_n[aa];
            for (int k = 0; k < SLOTS; ++k)
                s_pos[t][k] = k < n_at ? make_float4(atoms[k].x, atoms[k].y, atoms[k].z, 0.f)
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
            s_aa[t] = aa;
            s_chi[t] = chi;
            s_trig[t][0] = tr0;
            s_trig[t][1] = tr1;
            s_ds[t] = disulfide_with(st, c, r, aa, s_pos[t][5]);
        }
        __syncthreads();
        // residue energy of every trial: one warp per trial
        GroupSmem& g = gs[warp];
        for (int t = warp; t < MAT_TRIALS; t += MAT_WARPS) {
            const int aa = s_aa[t];
            const int na = c_topo_n[aa];
            if (lane < na) {
                const float4 p = s_pos[t][lane];
                const float4 m = c_slot_prm[aa][lane];
                g.pos[lane] = make_float4(p.x, p.y, p.z, m.x);
                g.prm[lane] = make_float4(m.y, m.z, m.w, (float)c_slot_type[aa][lane]);
                group_xyz(g, lane, na, p.x, p.y, p.z);
                group_prm(g, lane, na, m.x, m.y, m.z, m.w);
            } else {
                group_xyz(g, lane, na, 0.f, 0.f, 0.f);
                group_prm(g, lane, na, 0.f, 0.f, 0.f, 0.f);
            }
            __syncwarp();
            Acc acc = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0};
            score_group<true, true, false, false>(&A, g, na, lane, lt, acc);
            const double e = warp_sum_d((double)acc.s - (double)acc.c);
            if (lane == 0) s_e[t] = e;
            __syncwarp();
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double others = 0.0;
            for (int q = r0; q < r1; ++q)
                if (q != r) others += res_e[q];
            int pick = MAT_TRIALS - 1;
            for (int t = 0; t < MAT_TRIALS - 1; ++t) {
                const double tot = (others + s_e[t]) + (double)s_ds[t];
                if (tot < s_best) {
                    s_best = tot;
                    pick = t;
                    ++s_kept;
                    break;
                }
            }
            s_pick = pick;
            res_e[r] = s_e[pick];
            st.res_aa[r] = (uint8_t)s_aa[pick];
            st.res_chi[r] = s_chi[pick];
            st.res_trig[2 * r] = s_trig[pick][0];
            st.res_trig[2 * r + 1] = s_trig[pick][1];
        }
        __syncthreads();
        if (threadIdx.x < SLOT_STRIDE)
            st.res_pos[(size_t)r * SLOT_STRIDE + threadIdx.x] =
                threadIdx.x < SLOTS ? s_pos[s_pick][threadIdx.x] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out_best[c] = s_best;
        if (out_kept) out_kept[c] = s_kept;
    }
}

void launch_mature(cudaStream_t s, const StateView& st, const AgView* ags, double* res_e, double* out_best,
                   int* out_kept, uint32_t* err) {
    if (st.n_cand > 0) k_mature<<<st.n_cand, MAT_WARPS * 32, 0, s>>>(st, ags, res_e, out_best, out_kept, err);
}

// ---- Fv two-chain engine (diffusion.rs:477-827) -----------------------------------------
// The resident state interleaves the heavy (2i) and light (2i + 1) chain of each Fv
// candidate i.
constexpr int FVP_THREADS = 256;
constexpr int FVP_MAX_RES = 160;  // residues of a chain the pair kernel stages

// interaction_energy_atoms (energy.rs:256-314, solvation.rs:52-84) between the two chains
// of candidate i (heavy as energy.rs's "antigen", light as its "antibody"), all five
// terms, FP64 total; residue pairs whose bounding spheres are further apart than the
// cutoff are skipped (they hold no pair within 10 A).
__global__ void __launch_bounds__(FVP_THREADS) k_fv_pair(StateView st, double* __restrict__ out) {
    const int i = blockIdx.x;
    const int h0 = st.cand_res_off[2 * i], nh = st.cand_res_off[2 * i + 1] - h0;
    const int l0 = st.cand_res_off[2 * i + 1], nl = st.cand_res_off[2 * i + 2] - l0;
    __shared__ float4 s_c[2][FVP_MAX_RES];  // residue centroid, radius
    __shared__ double s_sum[FVP_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (nh > FVP_MAX_RES || nl > FVP_MAX_RES) {
        if (threadIdx.x == 0) out[i] = nan("");
        return;
    }
    for (int t = threadIdx.x; t < nh + nl; t += blockDim.x) {
        const int r = t < nh ? h0 + t : l0 + (t - nh);
        const int na = c_topo_n[st.res_aa[r]];
        const float4* p = st.res_pos + (size_t)r * SLOT_STRIDE;
        float cx = 0.f, cy = 0.f, cz = 0.f;
        for (int k = 0; k < na; ++k) {
            cx += p[k].x; cy += p[k].y; cz += p[k].z;
        }
        cx /= na; cy /= na; cz /= na;
        float rad = 0.f;
        for (int k = 0; k < na; ++k) {
            const float dx = p[k].x - cx, dy = p[k].y - cy, dz = p[k].z - cz;
            rad = fmaxf(rad, sqrtf(dx * dx + dy * dy + dz * dz));
        }
        s_c[t < nh ? 0 : 1][t < nh ? t : t - nh] = make_float4(cx, cy, cz, rad * 1.0001f + 1e-3f);
    }
    __syncthreads();
    float s = 0.f, comp = 0.f;  // compensated sum of this thread's pair terms
    for (int t = threadIdx.x; t < nh * nl; t += blockDim.x) {
        const int a = t / nl, b = t - a * nl;
        const float4 ca = s_c[0][a], cb = s_c[1][b];
        const float dx = ca.x - cb.x, dy = ca.y - cb.y, dz = ca.z - cb.z;
        const float reach = 10.01f + ca.w + cb.w;
        if (dx * dx + dy * dy + dz * dz > reach * reach) continue;
        const int aa_a = st.res_aa[h0 + a], aa_b = st.res_aa[l0 + b];
        const int na = c_topo_n[aa_a], nb = c_topo_n[aa_b];
        const float4* pa = st.res_pos + (size_t)(h0 + a) * SLOT_STRIDE;
        const float4* pb = st.res_pos + (size_t)(l0 + b) * SLOT_STRIDE;
        for (int kb = 0; kb < nb; ++kb) {
            const float4 m = c_slot_prm[aa_b][kb];
            const float4 B = make_float4(pb[kb].x, pb[kb].y, pb[kb].z, m.x);
            const float4 Bp = make_float4(m.y, m.z, m.w, (float)c_slot_type[aa_b][kb]);
            for (int ka = 0; ka < na; ++ka) {
                const float4 n = c_slot_prm[aa_a][ka];
                const float4 A = make_float4(pa[ka].x, pa[ka].y, pa[ka].z, n.x);
                const float r2 = xdist2(B.x - A.x, B.y - A.y, B.z - A.z);
                if (r2 > CUTOFF_SQ || r2 < MIN_R_SQ) continue;
                const float4 Ap = make_float4(n.y, n.z, n.w, (float)c_slot_type[aa_a][ka]);
                float lj, coul, hyd;
                const float e = pair_energy<true>(B, Bp, A, Ap, r2, lj, coul, hyd);
                const float y = e - comp, tt = s + y;
                comp = (tt - s) - y;
                s = tt;
            }
        }
    }
    const double v = warp_sum_d((double)s - (double)comp);
    if (lane == 0) s_sum[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double e = 0.0;
        for (int w = 0; w < FVP_THREADS / 32; ++w) e += s_sum[w];
        out[i] = e;
    }
}

// fv_energy = both chains' energies against the antigen (each with its disulfide
// term) + the pair energy; elitist keep (diffusion.rs:800-810): a lower energy
// becomes the best pair, a higher one is replaced by the best pair.  mode 1: put the
// best pair back whatever the energy (the result of run_fv is the best); mode 2: the
// pair as it is becomes the best (the start of the run, diffusion.rs:788-790).
__global__ void k_fv_keep(StateView st, const double* __restrict__ e_chain, const double* __restrict__ e_pair,
                          double* __restrict__ best, float4* __restrict__ b_pos, uint8_t* __restrict__ b_aa,
                          float4* __restrict__ b_chi, float4* __restrict__ b_trig, int restore) {
    const int i = blockIdx.x;
    __shared__ int s_dec;
    if (threadIdx.x == 0) {
        const double e = e_chain[2 * i] + e_chain[2 * i + 1] + e_pair[i];
        int dec = 0;
        if (restore == 1) dec = -1;
        else if (restore == 2 || e < best[i]) dec = 1;
        else if (e > best[i]) dec = -1;
        if (dec == 1) best[i] = e;
        s_dec = dec;
    }
    __syncthreads();
    const int dec = s_dec;
    if (dec == 0) return;
    const int r0 = st.cand_res_off[2 * i], r1 = st.cand_res_off[2 * i + 2];
    for (int t = r0 * SLOT_STRIDE + (int)threadIdx.x; t < r1 * SLOT_STRIDE; t += blockDim.x) {
        if (dec > 0) b_pos[t] = st.res_pos[t];
        else st.res_pos[t] = b_pos[t];
    }
    for (int r = r0 + (int)threadIdx.x; r < r1; r += blockDim.x) {
        if (dec > 0) {
            b_aa[r] = st.res_aa[r];
            b_chi[r] = st.res_chi[r];
            b_trig[2 * r] = st.res_trig[2 * r];
            b_trig[2 * r + 1] = st.res_trig[2 * r + 1];
        } else {
            st.res_aa[r] = b_aa[r];
            st.res_chi[r] = b_chi[r];
            st.res_trig[2 * r] = b_trig[2 * r];
            st.res_trig[2 * r + 1] = b_trig[2 * r + 1];
        }
    }
}

void launch_fv_pair(cudaStream_t s, const StateView& st, double* out) {
    if (st.n_cand >= 2) k_fv_pair<<<st.n_cand / 2, FVP_THREADS, 0, s>>>(st, out);
}
void launch_fv_keep(cudaStream_t s, const StateView& st, const double* e_chain, const double* e_pair, double* best,
                    float4* b_pos, uint8_t* b_aa, float4* b_chi, float4* b_trig, int restore) {
    if (st.n_cand >= 2)
        k_fv_keep<<<st.n_cand / 2, 256, 0, s>>>(st, e_chain, e_pair, best, b_pos, b_aa, b_chi, b_trig, restore);
}

// ---- structure validation (validate.rs) ------------------------------------------------
// Clash test of one atom pair (validate.rs:52-59): d^2 < (0.7 (rmh_i + rmh_j))^2, f32.
__device__ __forceinline__ bool clash(float4 a, float4 b) {
    const float d_sq = xdist2(xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z));
    const float thresh = xmul(0.7f, xadd(a.w, b.w));
    return d_sq < xmul(thresh, thresh);
}

// dihedral (validate.rs:72-86) in degrees (f32::to_degrees); atan2 evaluated in
// double and rounded once to f32, as the CPU restatement does
__device__ float dihedral_deg(F3 p0, F3 p1, F3 p2, F3 p3) {
    const F3 b1 = sub3(p1, p0), b2 = sub3(p2, p1), b3 = sub3(p3, p2);
    const F3 n1 = norm3(cross3(b1, b2));
    const F3 n2 = norm3(cross3(b2, b3));
    const F3 m1 = cross3(n1, norm3(b2));
    const float x = xadd(xadd(xmul(n1.x, n2.x), xmul(n1.y, n2.y)), xmul(n1.z, n2.z));
    const float y = xadd(xadd(xmul(m1.x, n2.x), xmul(m1.y, n2.y)), xmul(m1.z, n2.z));
    return xmul((float)atan2((double)y, (double)x), 57.2957795130823208767981548141051703f);
}

// in_allowed_basin (validate.rs:101-108), inclusive ranges
__device__ __forceinline__ bool allowed_basin(float phi, float psi) {
    const bool alpha_r = phi >= -100.0f && phi <= -30.0f && psi >= -80.0f && psi <= -5.0f;
    const bool beta = (phi >= -170.0f && phi <= -60.0f && psi >= 90.0f && psi <= 180.0f) ||
                      (phi >= -170.0f && phi <= -60.0f && psi >= -180.0f && psi <= -150.0f);
    const bool alpha_l = phi >= 30.0f && phi <= 100.0f && psi >= -10.0f && psi <= 80.0f;
    return alpha_r || beta || alpha_l;
}

// One CTA per candidate: its atoms (x, y, z, r_min_half) and residue index in shared
// memory, the atom pairs split over the threads, then the backbone torsions.
constexpr int VAL_THREADS = 256;
constexpr int VAL_MAX_RES = 640;  // a candidate's atoms fit the shared memory of one CTA
__global__ void __launch_bounds__(VAL_THREADS) k_validate(StateView st, int* __restrict__ clashes,
                                                           int* __restrict__ rama) {
    const int c = blockIdx.x;
    const int r0 = st.cand_res_off[c], n = st.cand_res_off[c + 1] - r0;
    extern __shared__ __align__(16) unsigned char v_dyn[];
    float4* at = reinterpret_cast<float4*>(v_dyn);
    int* res = reinterpret_cast<int*>(at + (size_t)n * SLOTS);
    __shared__ int s_n, s_count[VAL_THREADS / 32];
    if (threadIdx.x == 0) {
        int m = 0;
        for (int i = 0; i < n; ++i) m += s_topo_n[st.res_aa[r0 + i]];
        s_n = m;
    }
    __syncthreads();
    // the flattened atoms, residue after residue in topology order
    if (threadIdx.x < 32) {
        int base = 0;
        for (int i = 0; i < n; ++i) {
            const int aa = st.res_aa[r0 + i], na = s_topo_n[aa];
            if ((int)threadIdx.x < na) {
                const float4 p = st.res_pos[(size_t)(r0 + i) * SLOT_STRIDE + threadIdx.x];
                at[base + threadIdx.x] = make_float4(p.x, p.y, p.z, c_slot_prm[aa][threadIdx.x].y);
                res[base + threadIdx.x] = i;
            }
            base += na;
        }
    }
    __syncthreads();
    const int m = s_n;
    const long long pairs = (long long)m * (m - 1) / 2;
    int cnt = 0;
    for (long long t = threadIdx.x; t < pairs; t += blockDim.x) {
        // pair t -> (i, j), i < j: row i holds m - 1 - i pairs
        int i = (int)((2.0 * m - 1.0 - sqrt((2.0 * m - 1.0) * (2.0 * m - 1.0) - 8.0 * (double)t)) * 0.5);
        i = max(0, min(i, m - 2));
        while (i > 0 && (long long)i * (2 * m - i - 1) / 2 > t) --i;
        while ((long long)(i + 1) * (2 * m - i - 2) / 2 <= t) ++i;
        const int j = (int)(t - (long long)i * (2 * m - i - 1) / 2) + i + 1;
        if (abs(res[i] - res[j]) <= 1) continue;
        cnt += clash(at[i], at[j]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) s_count[threadIdx.x >> 5] = cnt;
    // ramachandran_outliers: residues 1..n-2 (both torsions defined)
    int out = 0;
    for (int r = (int)threadIdx.x + 1; r + 1 < n; r += blockDim.x) {
        const float4* p = st.res_pos + (size_t)(r0 + r) * SLOT_STRIDE;
        const float4 cp = st.res_pos[(size_t)(r0 + r - 1) * SLOT_STRIDE + 2];
        const float4 nn = st.res_pos[(size_t)(r0 + r + 1) * SLOT_STRIDE + 0];
        const float phi = dihedral_deg(f3(cp), f3(p[0]), f3(p[1]), f3(p[2]));
        const float psi = dihedral_deg(f3(p[0]), f3(p[1]), f3(p[2]), f3(nn));
        out += !allowed_basin(phi, psi);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) out += __shfl_xor_sync(0xffffffffu, out, o);
    __shared__ int s_rama[VAL_THREADS / 32];
    if ((threadIdx.x & 31) == 0) s_rama[threadIdx.x >> 5] = out;
    __syncthreads();
    if (threadIdx.x == 0) {
        int a = 0, b = 0;
        for (int w = 0; w < VAL_THREADS / 32; ++w) {
            a += s_count[w];
            b += s_rama[w];
        }
        clashes[c] = a;
        rama[c] = b;
    }
}

cudaError_t launch_validate(cudaStream_t s, const StateView& st, int* clashes, int* rama) {
    if (st.n_cand <= 0) return cudaSuccess;
    int max_res = 0;  // the launch reserves the largest candidate's atoms
    std::vector<int> off(st.n_cand + 1);
    cudaMemcpyAsync(off.data(), st.cand_res_off, off.size() * sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    for (int c = 0; c < st.n_cand; ++c) max_res = std::max(max_res, off[c + 1] - off[c]);
    const size_t smem = (size_t)max_res * SLOTS * (sizeof(float4) + sizeof(int));
    if (max_res > VAL_MAX_RES) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) cudaFuncSetAttribute(k_validate, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_validate<<<st.n_cand, VAL_THREADS, smem, s>>>(st, clashes, rama);
    return cudaGetLastError();
}

}  // namespace binder
