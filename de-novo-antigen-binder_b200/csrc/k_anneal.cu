// k_anneal.cu — allatom_diffusion_step with its Metropolis moves (diffusion.rs:290-463)
// on the GPU: one CTA per candidate, the candidate's residues resident in shared
// memory for all n_steps of the launch.
//
// Per step, in the reference's order:
//  1. Langevin: coarse-grained force (the 27-cell walk in the reference's order),
//     restraint, noise, 2 A clamp, rigid translation (diffusion.rs:306-339).
//  2. Interface mask: any antigen Calpha within sqrt(iface_cutoff_sq) (:343-351).
//  3. Mutation / rotamer sweep (:354-399).  A move at residue r changes only
//     residue r's atoms, and the Calpha-level energy of r depends only on r's
//     Calpha and amino acid; residues interact only through the disulfide term.
//     So every residue's proposal, its rejection rebuild and both Calpha energies
//     are computed in parallel, and one thread then takes the decisions in
//     residue order, updating the disulfide energy wherever a Cys is involved —
//     the reference's sequential sweep, exactly.
//  4. Backbone phi/psi sweep (:403-418): sequential over the attempted moves;
//     per move the Calpha energies of residues r..n are evaluated by warps over
//     the antigen Calphas, the downstream atoms rotated by all threads (Rodrigues,
//     allatom.rs:397-479), and the decision broadcast; a rejected move is undone
//     by the opposite rotation, as in the reference.
// Calpha energies are cached per residue and recomputed whenever the Calpha moved.
//
// Accumulation: ACC = float reproduces the reference's f32 sums bit for bit; ACC =
// double sums the same f32 pair terms in double and takes the Metropolis test on
// the double energy difference.
#include "geom.cuh"
#include "kernels.h"

namespace binder {

cudaError_t anneal_init_tables() { return geom_init_tables(); }

constexpr int AN_WARPS = 8;
constexpr int AN_THREADS = AN_WARPS * 32;
enum : int { MV_NONE = 0, MV_ROT = 1, MV_MUT = 2 };
enum : int { SEL_KEEP = 0, SEL_PROP = 1, SEL_REJ = 2 };

// Shared-memory carve of one CTA for candidates of up to R residues.
struct AnSmem {
    float4 *pos, *prop, *rej;  // R * SLOT_STRIDE each: state, proposal, rejection rebuild
    float4* trig;              // 2R: sin/cos of chi1..4
    float4* chi;               // R (degrees)
    float4* ldelta;            // R: Langevin translation
    float4* stage;             // AN_WARPS * 32: in-cutoff pair terms of one warp chunk
    double *c_cur, *c_old, *c_new;  // R: Calpha energies (exact f32 values when ACC = float)
    float *u_acc, *bb_delta, *bb_u;  // R
    int *aa, *kind, *new_aa, *new_rot, *sel, *valid, *bb_att, *bb_phi, *iface;  // R
    double* dscal;  // [0] disulfide energy of the current state
    int* iscal;     // [0] disulfide valid, [1] decision
};
__host__ __device__ inline size_t anneal_smem_bytes(int R) {
    return (size_t)R * SLOT_STRIDE * 16 * 3 + (size_t)R * 16 * 4 + (size_t)AN_WARPS * 32 * 16 + (size_t)R * 8 * 3 +
           (size_t)R * 4 * 3 + (size_t)R * 4 * 9 + 16 + 16;
}
__device__ inline AnSmem carve(unsigned char* b, int R) {
    AnSmem s;
    auto take = [&](size_t bytes) { unsigned char* p = b; b += bytes; return p; };
    s.pos = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.prop = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.rej = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.trig = (float4*)take((size_t)R * 32);
    s.chi = (float4*)take((size_t)R * 16);
    s.ldelta = (float4*)take((size_t)R * 16);
    s.stage = (float4*)take((size_t)AN_WARPS * 32 * 16);
    s.c_cur = (double*)take((size_t)R * 8);
    s.c_old = (double*)take((size_t)R * 8);
    s.c_new = (double*)take((size_t)R * 8);
    s.dscal = (double*)take(16);
    s.u_acc = (float*)take((size_t)R * 4);
    s.bb_delta = (float*)take((size_t)R * 4);
    s.bb_u = (float*)take((size_t)R * 4);
    s.aa = (int*)take((size_t)R * 4);
    s.kind = (int*)take((size_t)R * 4);
    s.new_aa = (int*)take((size_t)R * 4);
    s.new_rot = (int*)take((size_t)R * 4);
    s.sel = (int*)take((size_t)R * 4);
    s.valid = (int*)take((size_t)R * 4);
    s.bb_att = (int*)take((size_t)R * 4);
    s.bb_phi = (int*)take((size_t)R * 4);
    s.iface = (int*)take((size_t)R * 4);
    s.iscal = (int*)take(16);
    return s;
}

// hbond_energy (energy.rs:32-39) with the Metropolis-path exponential
__device__ __forceinline__ float hbond_mc(float r_sq) {
    if (r_sq > HB_CUTOFF_SQ) return 0.0f;
    const float r = xsqrt(r_sq);
    const float z = xdiv(xsub(r, HB_R0), HB_SIGMA);
    return xmul(-HB_DEPTH, mc_exp(xmul(xmul(-0.5f, z), z)));
}

// residue_contribution_allatom (diffusion.rs:425-463) of a Calpha at `ca` of amino
// acid `aa`, by one warp: lanes evaluate 32 antigen Calphas at a time (in index
// order); the in-cutoff terms are staged in shared memory and lane 0 adds them in
// the reference's order.  Result valid in lane 0.
template <class ACC>
__device__ ACC warp_contribution(const AgView& A, F3 ca, int aa, float4* stage) {
    const int lane = threadIdx.x & 31;
    const float4 b = s_ca_atom[aa];  // q, r_min_half, epsilon, hydrophobic
    const int bt = s_ca_type[aa];
    const int bhb = s_hb_role[bt];
    ACC e = 0;
    for (int base = 0; base < A.n_res; base += 32) {
        const int i = base + lane;
        bool in = false;
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < A.n_res) {
            const float4 a = A.ca_atom[i];
            const float4 ap = A.ca_atom_prm[i];
            const float r_sq = xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z));
            in = !(r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ);
            if (in) {
                unsigned fl = 0;
                const float r_ij = xadd(b.y, ap.x);
                const float eps = xsqrt(xmul(b.z, ap.y));
                const float r2 = xdiv(xmul(r_ij, r_ij), r_sq);
                const float r6 = xmul(xmul(r2, r2), r2);
                t.x = xmul(eps, xsub(xmul(r6, r6), xmul(2.0f, r6)));
                if (b.x != 0.0f && a.w != 0.0f) {
                    t.y = xdiv(xmul(xmul(COULOMB_K, b.x), a.w), xsqrt(r_sq));
                    fl |= 1u;
                }
                if (b.w == 1.0f && ap.z == 1.0f && r_sq < HYDRO_CUTOFF_SQ) fl |= 2u;
                const int ahb = s_hb_role[(int)ap.w];
                if (((bhb & 1) && (ahb & 2)) || ((bhb & 2) && (ahb & 1))) {
                    t.z = hbond_mc(r_sq);
                    fl |= 4u;
                }
                t.w = __uint_as_float(fl);
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) stage[__popc(m & ((1u << lane) - 1u))] = t;
        __syncwarp();
        if (lane == 0) {
            const int cnt = __popc(m);
            for (int j = 0; j < cnt; ++j) {
                const float4 v = stage[j];
                const unsigned fl = __float_as_uint(v.w);
                e += (ACC)v.x;
                if (fl & 1u) e += (ACC)v.y;
                if (fl & 2u) e -= (ACC)0.5f;
                if (fl & 4u) e += (ACC)v.z;
            }
        }
        __syncwarp();
    }
    return e;
}

// Slots of residue j as the sweep currently sees them: its proposal when accepted
// this sweep, its rejection rebuild when rejected, else the state.
__device__ __forceinline__ const float4* cur_slots(const AnSmem& S, int j) {
    const int s = S.sel[j];
    return (s == SEL_PROP ? S.prop : (s == SEL_REJ ? S.rej : S.pos)) + (size_t)j * SLOT_STRIDE;
}

// disulfide_energy (allatom.rs:155-180) over the SG atoms (topology atom 5 of Cys)
// in residue order; residue `sub` (>= 0) is taken from `sub_slots` with amino
// acid `sub_aa` instead.
template <class ACC>
__device__ ACC disulfide_sweep(const AnSmem& S, int n, int sub, const float4* sub_slots, int sub_aa) {
    ACC e = 0;
    for (int i = 0; i < n; ++i) {
        const int ai = i == sub ? sub_aa : S.aa[i];
        if (ai != CYS) continue;
        const float4 pi = (i == sub ? sub_slots : cur_slots(S, i))[5];
        for (int j = i + 1; j < n; ++j) {
            const int aj = j == sub ? sub_aa : S.aa[j];
            if (aj != CYS) continue;
            const float4 pj = (j == sub ? sub_slots : cur_slots(S, j))[5];
            const float d = xsqrt(xdist2(xsub(pi.x, pj.x), xsub(pi.y, pj.y), xsub(pi.z, pj.z)));
            if (d > 4.0f) continue;
            const float z = xdiv(xsub(d, 2.05f), 0.4f);
            e -= (ACC)xmul(4.0f, mc_exp(xmul(xmul(-0.5f, z), z)));
        }
    }
    return e;
}

// Metropolis criterion (diffusion.rs:368, 385, 414-415)
__device__ __forceinline__ bool metropolis(float de, float temp, float u) {
    return de <= 0.0f || u < mc_exp(xdiv(-de, temp));
}
__device__ __forceinline__ bool metropolis(double de, float temp, float u) {
    return de <= 0.0 || (double)u < exp(-de / (double)temp);
}

// The residue a move leaves: which = SEL_PROP builds the proposal, SEL_REJ the state
// after a rejection (rebuild_side_chain with the old chi, or mutate_residue back to
// the old amino acid around the same Calpha; allatom.rs:244-384).
__device__ void build_move(const AnSmem& S, int r, int which) {
    const int oa = S.aa[r];
    const int kind = S.kind[r];
    const int na = kind == MV_MUT ? S.new_aa[r] : oa;
    const float4* cur = S.pos + (size_t)r * SLOT_STRIDE;
    float4* out = (which == SEL_PROP ? S.prop : S.rej) + (size_t)r * SLOT_STRIDE;
    const ChiTrig old_t = unpack_trig(S.trig[2 * r], S.trig[2 * r + 1]);
    F3 atoms[SLOTS];
    if (kind == MV_ROT || na == oa) {
        // side chain rebuilt on the current backbone (N, CA, C, O[, CB])
        ChiTrig t = old_t;
        if (which == SEL_PROP) {
            if (kind == MV_ROT) t = rot_trig(oa, S.new_rot[r]);
            else t = s_rot_n[oa] > 0 ? rot_trig(oa, 0) : zero_trig();
        }
        const int n_bb = 4 + (oa != GLY ? 1 : 0);
        for (int k = 0; k < n_bb; ++k) atoms[k] = f3(cur[k]);
        build_side_chain(oa, atoms, n_bb, t);
        const int n_at = s_topo_n[oa];
        for (int k = 0; k < SLOT_STRIDE; ++k)
            out[k] = (k >= n_bb && k < n_at) ? make_float4(atoms[k].x, atoms[k].y, atoms[k].z, 0.f) : cur[k];
    } else {
        // ideal backbone around the Calpha with the new (or, rejected, the old) residue
        const int a = which == SEL_PROP ? na : oa;
        const ChiTrig t = which == SEL_PROP ? (s_rot_n[na] > 0 ? rot_trig(na, 0) : zero_trig()) : old_t;
        const int n_bb = ideal_backbone(f3(cur[1]), a, atoms);
        build_side_chain(a, atoms, n_bb, t);
        store_residue(out, atoms, s_topo_n[a]);
    }
}

// rodrigues (allatom.rs:467-479)
__device__ __forceinline__ float4 rodrigues(float4 p, F3 o, F3 ax, float ca, float sa) {
    const F3 v = {xsub(p.x, o.x), xsub(p.y, o.y), xsub(p.z, o.z)};
    const float dot = xadd(xadd(xmul(v.x, ax.x), xmul(v.y, ax.y)), xmul(v.z, ax.z));
    const F3 cx = cross3(ax, v);
    const float omc = xsub(1.0f, ca);
    const float rx = xadd(xadd(xmul(v.x, ca), xmul(cx.x, sa)), xmul(xmul(ax.x, dot), omc));
    const float ry = xadd(xadd(xmul(v.y, ca), xmul(cx.y, sa)), xmul(xmul(ax.y, dot), omc));
    const float rz = xadd(xadd(xmul(v.z, ca), xmul(cx.z, sa)), xmul(xmul(ax.z, dot), omc));
    return make_float4(xadd(rx, o.x), xadd(ry, o.y), xadd(rz, o.z), p.w);
}

// Rotate the atoms a phi (about N-CA through CA: residue r's atoms after CA and all
// later residues) or psi move (about CA-C through C: residue r's O and all later
// residues) moves; allatom.rs:397-455.
__device__ void rotate_downstream(const AnSmem& S, int n, int r, bool phi, float angle) {
    const float4* rs = S.pos + (size_t)r * SLOT_STRIDE;
    const F3 a0 = f3(rs[phi ? 0 : 1]), a1 = f3(rs[phi ? 1 : 2]);
    const F3 axis = norm3(sub3(a1, a0));
    const F3 origin = a1;
    const float ca = mc_cos(angle), sa = mc_sin(angle);
    const int n_at_r = s_topo_n[S.aa[r]];
    for (int idx = threadIdx.x; idx < (n - r) * SLOT_STRIDE; idx += AN_THREADS) {
        const int q = r + idx / SLOT_STRIDE, k = idx % SLOT_STRIDE;
        const bool mv = q == r ? (phi ? (k >= 2 && k < n_at_r) : k == 3) : k < s_topo_n[S.aa[q]];
        if (mv) {
            float4* p = S.pos + (size_t)q * SLOT_STRIDE + k;
            *p = rodrigues(*p, origin, axis, ca, sa);
        }
    }
}

template <class ACC>
__global__ void __launch_bounds__(AN_THREADS) k_anneal(StateView st, const AgView* __restrict__ ags, StepParams p,
                                                       int n_steps, uint32_t step0, int with_noise,
                                                       const float* __restrict__ temps, int R,
                                                       uint32_t* __restrict__ err, long long* __restrict__ stats) {
    extern __shared__ __align__(16) unsigned char an_smem[];
    const AnSmem S = carve(an_smem, R);
    const int c = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = st.cand_res_off[c];
    const int n = st.cand_res_off[c + 1] - r0;
    if (n <= 0 || n > R) return;
    const uint32_t cid = st.cand_id[c];
    const AgView A = ags[st.cand_ag[c]];
    float4* stage = S.stage + warp * 32;

    for (int i = tid; i < n * SLOT_STRIDE; i += AN_THREADS) S.pos[i] = st.res_pos[(size_t)r0 * SLOT_STRIDE + i];
    for (int r = tid; r < n; r += AN_THREADS) {
        S.aa[r] = st.res_aa[r0 + r];
        S.chi[r] = st.res_chi[r0 + r];
        S.trig[2 * r] = st.res_trig[2 * (r0 + r)];
        S.trig[2 * r + 1] = st.res_trig[2 * (r0 + r) + 1];
        S.sel[r] = SEL_KEEP;
    }
    long long n_mc = 0, n_mc_acc = 0, n_bb = 0, n_bb_acc = 0;
    __syncthreads();

    for (int s = 0; s < n_steps; ++s) {
        const uint32_t step = step0 + (uint32_t)s;
        const float temp = temps ? temps[s] : p.t_hot;
        // ---- 1. Langevin (diffusion.rs:306-339) ----
        for (int r = tid; r < n; r += AN_THREADS) {
            const F3 ca = f3(S.pos[r * SLOT_STRIDE + 1]);
            if (err && (!isfinite(ca.x) || !isfinite(ca.y) || !isfinite(ca.z))) atomicOr(err, ERRF_NAN);
            float fx, fy, fz;
            cg_force(A, cg_body(ca.x, ca.y, ca.z, S.aa[r]), fx, fy, fz);
            const float dx_c = xsub(ca.x, A.cx), dy_c = xsub(ca.y, A.cy), dz_c = xsub(ca.z, A.cz);
            const float d = fmaxf(xsqrt(xdist2(dx_c, dy_c, dz_c)), 0.001f);
            const float f_r = xdiv(xmul(-p.restraint_k, xsub(d, p.shell_radius)), d);
            fx = xadd(fx, xmul(f_r, dx_c));
            fy = xadd(fy, xmul(f_r, dy_c));
            fz = xadd(fz, xmul(f_r, dz_c));
            float nx = 0.f, ny = 0.f, nz = 0.f;
            if (with_noise) {
                const float sigma = xmul(p.noise_base, xsqrt(temp));
                const U4 u = rng_draw(p.seed, cid, step, STREAM_NOISE, (uint32_t)r);
                nx = frange(u.x, -sigma, sigma);
                ny = frange(u.y, -sigma, sigma);
                nz = frange(u.z, -sigma, sigma);
            }
            const float md = p.max_disp;
            const F3 nca = {xadd(xadd(ca.x, fminf(fmaxf(xmul(p.step, fx), -md), md)), nx),
                            xadd(xadd(ca.y, fminf(fmaxf(xmul(p.step, fy), -md), md)), ny),
                            xadd(xadd(ca.z, fminf(fmaxf(xmul(p.step, fz), -md), md)), nz)};
            const F3 dl = sub3(nca, ca);
            S.ldelta[r] = make_float4(dl.x, dl.y, dl.z, 0.f);
            S.valid[r] = 0;
        }
        if (tid == 0) S.iscal[0] = 0;  // disulfide energy stale
        __syncthreads();
        for (int i = tid; i < n * SLOT_STRIDE; i += AN_THREADS) {
            const int r = i / SLOT_STRIDE, k = i % SLOT_STRIDE;
            if (k < s_topo_n[S.aa[r]]) {
                const float4 d = S.ldelta[r];
                float4 v = S.pos[i];
                v.x = xadd(v.x, d.x); v.y = xadd(v.y, d.y); v.z = xadd(v.z, d.z);
                S.pos[i] = v;
            }
        }
        __syncthreads();

        // ---- 2. interface mask (diffusion.rs:343-351) + backbone draws ----
        for (int r = warp; r < n; r += AN_WARPS) {
            const F3 ca = f3(S.pos[r * SLOT_STRIDE + 1]);
            bool hit = false;
            for (int base = 0; base < A.n_res && !hit; base += 32) {
                const int i = base + lane;
                bool h = false;
                if (i < A.n_res) {
                    const float4 a = A.ca_atom[i];
                    h = xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z)) < p.iface_cutoff_sq;
                }
                hit = __any_sync(0xffffffffu, h);
            }
            if (lane == 0) S.iface[r] = hit;
        }
        for (int r = tid; r < n; r += AN_THREADS) {
            const U4 d = rng_draw(p.seed, cid, step, STREAM_BACKBONE, (uint32_t)r);
            S.bb_att[r] = u01(d.x) < p.backbone_move_p;
            S.bb_delta[r] = xmul(frange(d.y, -p.max_torsion_deg, p.max_torsion_deg), RADS_PER_DEG);
            S.bb_phi[r] = (int)((d.z >> 31) & 1u);
            S.bb_u[r] = u01(d.w);
        }
        __syncthreads();

        // ---- 3. mutation / rotamer proposals (diffusion.rs:354-399) ----
        for (int r = tid; r < n; r += AN_THREADS) {
            const bool itf = S.iface[r] != 0;
            const float eff_mut_p = itf ? xmul(p.mutation_p, 3.0f) : xmul(p.mutation_p, 0.4f);
            const float eff_rot_p = itf ? xmul(p.rotamer_move_p, 2.0f) : p.rotamer_move_p;
            const U4 d = rng_draw(p.seed, cid, step, STREAM_MC, (uint32_t)r);
            int kind = MV_NONE;
            if (u01(d.x) < eff_mut_p) {
                const int aa = S.aa[r];
                if (u01(d.y) < eff_rot_p) {
                    if (s_rot_n[aa] > 0) {
                        kind = MV_ROT;
                        S.new_rot[r] = (int)urange(d.z, (uint32_t)s_rot_n[aa]);
                        S.new_aa[r] = aa;
                    }
                } else {
                    kind = MV_MUT;
                    S.new_aa[r] = (int)urange(d.z, (uint32_t)N_AA);
                    S.new_rot[r] = 0;
                }
            }
            S.kind[r] = kind;
            S.u_acc[r] = u01(d.w);
        }
        __syncthreads();
        // proposals and rejection rebuilds (two threads per residue), then the Calpha
        // energies before / after each move (one warp per energy)
        for (int t = tid; t < 2 * n; t += AN_THREADS) {
            const int r = t >> 1;
            if (S.kind[r] != MV_NONE) build_move(S, r, (t & 1) ? SEL_REJ : SEL_PROP);
        }
        for (int t = warp; t < 2 * n; t += AN_WARPS) {
            const int r = t >> 1, which = t & 1;
            const int kind = S.kind[r];
            if (kind == MV_NONE) continue;
            const bool same = kind == MV_ROT || S.new_aa[r] == S.aa[r];
            if (which == 1 && same) continue;  // same Calpha, same amino acid: same energy
            const int a = which ? S.new_aa[r] : S.aa[r];
            const ACC e = warp_contribution<ACC>(A, f3(S.pos[r * SLOT_STRIDE + 1]), a, stage);
            if (lane == 0) {
                if (which == 0) {
                    S.c_old[r] = (double)e;
                    if (same) S.c_new[r] = (double)e;
                } else {
                    S.c_new[r] = (double)e;
                }
            }
        }
        __syncthreads();
        // the sweep's decisions, in residue order
        if (tid == 0) {
            bool have_d = false;
            ACC D = 0;
            for (int r = 0; r < n; ++r) {
                const int kind = S.kind[r];
                if (kind == MV_NONE) continue;
                if (!have_d) {
                    D = disulfide_sweep<ACC>(S, n, -1, nullptr, 0);
                    have_d = true;
                }
                const int oa = S.aa[r];
                const int na = kind == MV_MUT ? S.new_aa[r] : oa;
                const bool cys = oa == CYS || na == CYS;
                const ACC Dn = cys ? disulfide_sweep<ACC>(S, n, r, S.prop + (size_t)r * SLOT_STRIDE, na) : D;
                const ACC old_e = (ACC)S.c_old[r] + D;
                const ACC new_e = (ACC)S.c_new[r] + Dn;
                const bool acc = metropolis(new_e - old_e, temp, S.u_acc[r]);
                ++n_mc;
                n_mc_acc += acc;
                if (acc) {
                    S.sel[r] = SEL_PROP;
                    S.aa[r] = na;
                    const int rot = S.new_rot[r];
                    const bool has = s_rot_n[na] > 0;
                    S.chi[r] = has ? s_rot_chi[na][rot] : make_float4(0.f, 0.f, 0.f, 0.f);
                    const ChiTrig t = has ? rot_trig(na, rot) : zero_trig();
                    S.trig[2 * r] = make_float4(t.t[0].x, t.t[0].y, t.t[1].x, t.t[1].y);
                    S.trig[2 * r + 1] = make_float4(t.t[2].x, t.t[2].y, t.t[3].x, t.t[3].y);
                    S.c_cur[r] = S.c_new[r];
                    D = Dn;
                } else {
                    S.sel[r] = SEL_REJ;
                    S.c_cur[r] = S.c_old[r];
                    if (oa == CYS) D = disulfide_sweep<ACC>(S, n, -1, nullptr, 0);  // SG rebuilt
                }
                S.valid[r] = 1;
            }
            if (have_d) {
                S.dscal[0] = (double)D;
                S.iscal[0] = 1;
            }
        }
        __syncthreads();
        for (int i = tid; i < n * SLOT_STRIDE; i += AN_THREADS) {
            const int r = i / SLOT_STRIDE;
            const int sl = S.sel[r];
            if (sl == SEL_PROP) S.pos[i] = S.prop[i];
            else if (sl == SEL_REJ) S.pos[i] = S.rej[i];
        }
        __syncthreads();
        for (int r = tid; r < n; r += AN_THREADS) S.sel[r] = SEL_KEEP;
        __syncthreads();

        // ---- 4. backbone phi/psi moves (diffusion.rs:403-418) ----
        for (int r = 0; r < n; ++r) {
            if (!S.bb_att[r]) continue;
            const bool phi = S.bb_phi[r] != 0;
            // Calpha energies of residues r..n at the current positions, and the
            // disulfide energy
            if (tid == 0 && !S.iscal[0]) {
                S.dscal[0] = (double)disulfide_sweep<ACC>(S, n, -1, nullptr, 0);
                S.iscal[0] = 1;
            }
            for (int i = r + warp; i < n; i += AN_WARPS) {
                if (S.valid[i]) continue;
                const ACC e = warp_contribution<ACC>(A, f3(S.pos[i * SLOT_STRIDE + 1]), S.aa[i], stage);
                if (lane == 0) {
                    S.c_cur[i] = (double)e;
                    S.valid[i] = 1;
                }
            }
            __syncthreads();
            ACC old_e = 0;
            if (tid == 0) {
                for (int i = r; i < n; ++i) old_e += (ACC)S.c_cur[i];
                old_e += (ACC)S.dscal[0];
            }
            bool cys_down = false;  // a Cys at or after r: the disulfide term can change
            for (int i = r; i < n; ++i) cys_down |= S.aa[i] == CYS;
            rotate_downstream(S, n, r, phi, S.bb_delta[r]);
            __syncthreads();
            for (int i = r + 1 + warp; i < n; i += AN_WARPS) {
                const ACC e = warp_contribution<ACC>(A, f3(S.pos[i * SLOT_STRIDE + 1]), S.aa[i], stage);
                if (lane == 0) S.c_new[i] = (double)e;
            }
            __syncthreads();
            if (tid == 0) {
                const ACC Dn = cys_down ? disulfide_sweep<ACC>(S, n, -1, nullptr, 0) : (ACC)S.dscal[0];
                ACC new_e = 0;
                new_e += (ACC)S.c_cur[r];
                for (int i = r + 1; i < n; ++i) new_e += (ACC)S.c_new[i];
                new_e += Dn;
                const bool acc = metropolis(new_e - old_e, temp, S.bb_u[r]);
                ++n_bb;
                n_bb_acc += acc;
                if (acc) {
                    for (int i = r + 1; i < n; ++i) S.c_cur[i] = S.c_new[i];
                    S.dscal[0] = (double)Dn;
                } else {
                    for (int i = r + 1; i < n; ++i) S.valid[i] = 0;
                    if (cys_down) S.iscal[0] = 0;
                }
                S.iscal[1] = acc;
            }
            __syncthreads();
            if (!S.iscal[1]) {
                rotate_downstream(S, n, r, phi, -S.bb_delta[r]);
                __syncthreads();
            }
        }
    }

    for (int i = tid; i < n * SLOT_STRIDE; i += AN_THREADS) st.res_pos[(size_t)r0 * SLOT_STRIDE + i] = S.pos[i];
    for (int r = tid; r < n; r += AN_THREADS) {
        st.res_aa[r0 + r] = (uint8_t)S.aa[r];
        st.res_chi[r0 + r] = S.chi[r];
        st.res_trig[2 * (r0 + r)] = S.trig[2 * r];
        st.res_trig[2 * (r0 + r) + 1] = S.trig[2 * r + 1];
    }
    if (tid == 0 && stats) {
        stats[4 * c] += n_mc;
        stats[4 * c + 1] += n_mc_acc;
        stats[4 * c + 2] += n_bb;
        stats[4 * c + 3] += n_bb_acc;
    }
}

size_t anneal_smem(int max_res) { return anneal_smem_bytes(max_res); }

cudaError_t launch_anneal(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          uint32_t step0, int with_noise, const float* temps, int accumulate, int max_res,
                          uint32_t* err, long long* stats) {
    if (st.n_cand <= 0 || n_steps <= 0 || max_res <= 0) return cudaSuccess;
    const size_t smem = anneal_smem_bytes(max_res);
    cudaError_t e;
    if (accumulate == 1) {
        if ((e = cudaFuncSetAttribute(k_anneal<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
            return e;
        k_anneal<float><<<st.n_cand, AN_THREADS, smem, s>>>(st, ags, p, n_steps, step0, with_noise, temps, max_res,
                                                           err, stats);
    } else {
        if ((e = cudaFuncSetAttribute(k_anneal<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)))
            return e;
        k_anneal<double><<<st.n_cand, AN_THREADS, smem, s>>>(st, ags, p, n_steps, step0, with_noise, temps, max_res,
                                                            err, stats);
    }
    return cudaGetLastError();
}

}  // namespace binder
