// k_search.cu — residue construction and the gradient-phase search step on the GPU.
//
//  * protein_from_ca_trace (allatom.rs:523-541): ideal backbone + NERF side chain
//    per residue, one thread each.
//  * compute_forces_with_grid (energy.rs:322-398) for a batch of bodies.
//  * The Langevin part of allatom_diffusion_step (diffusion.rs:306-339) without
//    Metropolis moves: per-residue Verlet lists of antigen Calphas in the
//    reference's probe order, four or eight lanes per residue evaluate the pair
//    terms, lane 0 folds them in that order, and n_steps are fused per launch
//    since in this phase every residue moves independently.
//  * The residue visiting order by Calpha cell (one of the autotuned orders of the
//    gradient-step and scoring kernels) and the slot packing kernels.
#include <algorithm>

#include "cg_list.cuh"
#include "geom.cuh"
#include "kernels.h"

namespace binder {

cudaError_t search_init_tables() { return geom_init_tables(); }

// protein_from_ca_trace (allatom.rs:523-541): one thread per residue.  chi_trig
// (8 floats per residue: sin/cos of chi1..4) overrides the top rotamer when given.
__global__ void k_build_residues(int n, const float* __restrict__ ca_xyz, const uint8_t* __restrict__ aa_in,
                                 const float4* __restrict__ chi_trig, const float* __restrict__ chi_deg,
                                 float4* __restrict__ out_pos, float4* __restrict__ out_chi) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    const int aa = aa_in[r];
    F3 atoms[SLOTS];
    const F3 ca = {ca_xyz[3 * r], ca_xyz[3 * r + 1], ca_xyz[3 * r + 2]};
    const int n_bb = ideal_backbone(ca, aa, atoms);
    ChiTrig ct;
    float4 chi;
    if (chi_trig) {
        const float4 a = chi_trig[2 * r], b = chi_trig[2 * r + 1];
        ct.t[0] = make_float2(a.x, a.y); ct.t[1] = make_float2(a.z, a.w);
        ct.t[2] = make_float2(b.x, b.y); ct.t[3] = make_float2(b.z, b.w);
        chi = make_float4(chi_deg[4 * r], chi_deg[4 * r + 1], chi_deg[4 * r + 2], chi_deg[4 * r + 3]);
    } else if (s_rot_n[aa] > 0) {
        ct = rot_trig(aa, 0);
        chi = s_rot_chi[aa][0];
    } else {
        for (int i = 0; i < 4; ++i) ct.t[i] = make_float2(0.f, 1.f);
        chi = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    build_side_chain(aa, atoms, n_bb, ct);
    store_residue(out_pos + (size_t)r * SLOT_STRIDE, atoms, s_topo_n[aa]);
    out_chi[r] = chi;
}


// compute_forces_with_grid (energy.rs:322-398) for a batch of residue-level atoms
__global__ void k_cg_forces(const AgView* __restrict__ ag, const float* __restrict__ bx, const float* __restrict__ by,
                            const float* __restrict__ bz, const uint8_t* __restrict__ baa, int n,
                            float* __restrict__ fx, float* __restrict__ fy, float* __restrict__ fz) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const AgView A = *ag;
    float a, b, c;
    cg_force(A, cg_body(bx[j], by[j], bz[j], baa[j]), a, b, c);
    fx[j] = a; fy[j] = b; fz[j] = c;
}

// ---- Langevin steps without Metropolis moves (diffusion.rs:306-339) ----------------
// The reference sums the pair terms of compute_forces_with_grid in its probe order:
// cells (cx+dx, cy+dy, cz+dz) for dx, dy, dz = -1..1 (dz fastest), atoms ascending
// within a cell.  The antigen Calphas are stored sorted by cell in the same
// lexicographic order (ascending original index within a cell), so that probe order
// is ascending position in the sorted array.  Each residue therefore keeps a Verlet
// list: the positions, ascending, of the antigen Calphas within cutoff + skin of a
// list centre.  While the Calpha stays within the skin of the centre the list holds
// every in-cutoff Calpha; a step evaluates the list entries whose cell is adjacent
// to the Calpha's current cell and whose r^2 passes the reference's cutoff test,
// and sums their terms in list order -- the reference's pair set in the reference's
// order, hence the same f32 sum.  A Calpha leaving the skin rebuilds its list.
//
// G lanes per residue (G = 4 or 8; residue order and schedule autotuned, see
// res_of_slot and the work description below): the lanes split
// the list entries, write their terms to shared memory, and lane 0 folds them in
// order.  A list longer than CG_LIST_MAX, or a cell index near the i32 limits (where
// the reference's cell arithmetic wraps), sends the residue to the one-lane 27-cell
// walk (same sum).  The residue's atoms live in registers, atom k on lane k % G, and
// take every step's translation as set_ca_pos does (allatom.rs:279-293).
// COUNT: count the in-cutoff pairs of the same trajectory, leave the state as is.
// The one-lane walk over all 27 cells, out of line: it is rarely taken and must
// not take registers from the list path.
template <bool COUNT>
__device__ __noinline__ void cg_force_walk(const AgView* __restrict__ ag, float x, float y, float z, int aa,
                                           float3* out, int* n_pairs) {
    float sx, sy, sz;
    cg_force<COUNT>(*ag, cg_body(x, y, z, aa), sx, sy, sz, n_pairs);
    *out = make_float3(sx, sy, sz);
}


// Residue of a lane group's slot: the cell-sorted permutation (order_mode 0), the
// state's own order (1: candidate after candidate), a stride through it (2:
// slot * CG_STRIDE mod total, a bijection when total is coprime to the prime
// CG_STRIDE) that spreads each warp's residues over unrelated candidates, so the
// costly residues in contact are shared out evenly; the flat kernel's order 3
// (work-balanced tasks) is its own (slot_res).  Results never depend on it.
constexpr long long CG_STRIDE = 1000003;
__device__ __forceinline__ int res_of_slot(const int* __restrict__ order, int mode, int slot, int total) {
    if (mode == 2) return (int)(((long long)slot * CG_STRIDE) % total);
    if (mode == 1 || !order) return slot;
    return order[slot];
}

// Dynamic shared memory of the antigen staging: Calphas (pq, prm, cell) and the
// grid's cell starts of an antigen with n Calphas and ncell cells.
__host__ __device__ inline size_t cg_stage_bytes(int n, int ncell) {
    return (size_t)n * 48 + ((size_t)(ncell + 1) * 4 + 15) / 16 * 16;
}

// The antigen Calphas a CTA's residues probe (their pq / prm / cell arrays and the
// CG grid's cell starts) are copied to shared memory at the start of the launch
// when that antigen fits the dynamic shared memory the launch reserved; residues
// of other antigens read theirs from global memory.  Same values either way.
//
// Work: a warp takes NG = 32 / G residue slots at a time.  Static grid (queue
// null): one task per warp, as many CTAs as tasks need.  Persistent grid: the
// resident CTAs only, each warp taking tasks from the queue counter (zeroed before
// the launch) until none is left, so that warps with residues out of contact pick
// up the slack of those in contact.
// register budget: 24 resident warps per SM (80 registers a thread; a 64-register
// budget spills more than the extra occupancy gains)
template <bool COUNT, int CG_WARPS, int G>
__global__ void __launch_bounds__(CG_WARPS * 32, 24 / CG_WARPS) k_langevin(StateView st, const AgView* __restrict__ ags,
                                                             StepParams p, int n_steps, uint32_t step0,
                                                             int with_noise, const float* __restrict__ temps,
                                                             uint32_t* __restrict__ err,
                                                             long long* __restrict__ pair_count,
                                                             const int* __restrict__ order, int order_mode,
                                                             int stage_cap, int stage_ag, int* __restrict__ queue) {
    constexpr int RPC = CG_WARPS * 32 / G;  // residues per CTA
    constexpr int NG = 32 / G;              // residues (lane groups) per warp
    constexpr int NA = (SLOTS + G - 1) / G; // atoms per lane
    static_assert(RPC <= 32, "list storage is sized for 32 residues per CTA");
    __shared__ int s_list[RPC][CG_LIST_MAX];
    __shared__ int s_in[RPC][CG_IN_MAX];
    __shared__ float3 s_term[RPC][CG_IN_MAX];
    const int lane = threadIdx.x & 31;
    const int gl = lane & (G - 1);
    const int gshift = lane & ~(G - 1);
    const unsigned gmask = ((1u << G) - 1u) << gshift;
    const int rl = threadIdx.x / G;                  // this group's residue slot in the CTA
    const int rl0 = (threadIdx.x & ~31) / G;         // the warp's first residue slot
    extern __shared__ __align__(16) unsigned char cg_dyn[];
    __shared__ int s_stage_ag;
    // stage one antigen: stage_ag when every residue of the state probes it, else
    // (static grid) the antigen of the CTA's residues when its first and last share it
    if (threadIdx.x == 0) {
        int a0 = stage_ag, a1 = stage_ag;
        if (a0 < 0 && !queue) {
            const int first = blockIdx.x * RPC;
            const int last = min(first + RPC, st.total_res) - 1;
            // the first and last residue's antigen (order 2: every residue's); a residue of
            // another antigen reads its antigen from global memory all the same
            a0 = st.cand_ag[st.res_cand[res_of_slot(order, order_mode, first, st.total_res)]];
            a1 = st.cand_ag[st.res_cand[res_of_slot(order, order_mode, last, st.total_res)]];
            if (order_mode == 2)
                for (int q = first; q <= last && a1 == a0; ++q)
                    a1 = st.cand_ag[st.res_cand[res_of_slot(order, order_mode, q, st.total_res)]];
        }
        bool fits = a0 >= 0 && a0 == a1;
        if (fits) {
            const GridView& gv = ags[a0].ca_grid;
            fits = cg_stage_bytes(ags[a0].n_res, gv.nx * gv.ny * gv.nz) <= (size_t)stage_cap;
        }
        s_stage_ag = fits ? a0 : -1;
    }
    __syncthreads();
    const int sa = s_stage_ag;
    float4* spq = (float4*)cg_dyn;
    float4* sprm = spq;
    int4* scell = (int4*)cg_dyn;
    int* sstart = (int*)cg_dyn;
    if (sa >= 0) {
        const AgView& S = ags[sa];
        const int n = S.n_res, ncell = S.ca_grid.nx * S.ca_grid.ny * S.ca_grid.nz;
        sprm = spq + n;
        scell = (int4*)(sprm + n);
        sstart = (int*)(scell + n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            spq[i] = S.ca_pq[i];
            sprm[i] = S.ca_prm[i];
            scell[i] = S.ca_cell[i];
        }
        for (int i = threadIdx.x; i <= ncell; i += blockDim.x) sstart[i] = S.ca_grid.cell_start[i];
        __syncthreads();
    }
    // one task: the residue of this lane group's slot, n_steps gradient steps
    auto residue_task = [&](const int slot_id) {
        // every lane of a warp stays to the end: the pair evaluation is warp-wide
        const bool valid = slot_id < st.total_res;
        int* list = s_list[rl];
        int* in = s_in[rl];
        float3* terms = s_term[rl];
        const int r = valid ? res_of_slot(order, order_mode, slot_id, st.total_res) : 0;
        const int c = valid ? st.res_cand[r] : 0;
        const int r_local = valid ? r - st.cand_res_off[c] : 0;
        const uint32_t cid = valid ? st.cand_id[c] : 0u;
        const AgView* __restrict__ Ap = ags + (valid ? st.cand_ag[c] : 0);
        GridView g = Ap->ca_grid;
        const float4* __restrict__ ca_pq = Ap->ca_pq;
        const float4* __restrict__ ca_prm = Ap->ca_prm;
        const int4* __restrict__ ca_cell = Ap->ca_cell;
        const float ag_cx = Ap->cx, ag_cy = Ap->cy, ag_cz = Ap->cz;
        if (valid && st.cand_ag[c] == sa) {  // the staged antigen
            ca_pq = spq;
            ca_prm = sprm;
            ca_cell = scell;
            g.cell_start = sstart;
        }
        const int aa = valid ? st.res_aa[r] : 0;
        const int n_at = valid ? s_topo_n[aa] : 0;
        const float4 res = s_res[aa];
        float4* slot = st.res_pos + (size_t)r * SLOT_STRIDE;
        F3 ca = {0.f, 0.f, 0.f};
        if (valid) {
            const float4 v1 = slot[1];  // Calpha = topology atom 1 of every residue (amber.rs:358-377)
            ca = {v1.x, v1.y, v1.z};
            if (gl == 0 && err && (!isfinite(ca.x) || !isfinite(ca.y) || !isfinite(ca.z))) atomicOr(err, ERRF_NAN);
        }
        float4 at[NA];
#pragma unroll
        for (int j = 0; j < NA; ++j) {
            const int k = gl + G * j;
            at[j] = (!COUNT && k < n_at) ? slot[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        // the residue's list from the previous launch when it was built for this antigen
        // set and antigen and still covers the Calpha, else a new one
        F3 centre = ca;
        int nl = 0;
        bool dirty = false;
        float skin = CG_SKIN;
        if (valid) {
            const int ep = st.ag_epoch ? *st.ag_epoch : -2;
            const int4 meta = st.cg_meta ? st.cg_meta[r] : make_int4(-1, -1, -1, -1);
            bool reuse = false;
            float4 cc = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ep >= 0 && meta.z == ep && meta.y == st.cand_ag[c] && meta.x >= 0 && meta.x <= CG_LIST_MAX) {
                cc = st.cg_centre[r];
                skin = fminf(fmaxf(cc.w, CG_SKIN), CG_SKIN_MAX);
                const float mx = ca.x - cc.x, my = ca.y - cc.y, mz = ca.z - cc.z;
                reuse = mx * mx + my * my + mz * mz <= (skin - 0.01f) * (skin - 0.01f);
                if (!reuse) skin = fminf(2.0f * skin, CG_SKIN_MAX);  // it outran the list
            }
            if (reuse) {
                centre = {cc.x, cc.y, cc.z};
                nl = meta.x;
                for (int j = gl; j < nl; j += G) list[j] = st.cg_list[(size_t)r * CG_LIST_MAX + j];
                __syncwarp(gmask);
            } else {
                nl = build_cg_list<G>(g, ca_pq, centre, gl, gmask, list, skin);
                dirty = true;
            }
        }
        int n_pairs = 0;
        for (int s = 0; s < n_steps; ++s) {
            const int cx = cell_coord(ca.x, g.inv), cy = cell_coord(ca.y, g.inv), cz = cell_coord(ca.z, g.inv);
            bool use_list = valid && nl <= CG_LIST_MAX && !cell_far(cx, cy, cz);
            // Cells at least as wide as the cutoff and coordinates below 1e4 A: a pair
            // whose r^2 (reference rounding) is <= CG_NEAR_SQ is then in adjacent cells
            // (distance <= 9.95 A, under 0.995 cell edges however x * inv rounds), so the
            // reference's cell test only decides the entries closer to the cutoff.
            const bool near_adjacent = g.cell >= 10.0f && fabsf(ca.x) < 1e4f && fabsf(ca.y) < 1e4f &&
                                       fabsf(ca.z) < 1e4f;
            // A-C in rounds: each round a group compacts its next in-cutoff list entries
            // (r^2 passing the reference's cutoff test, adjacent cell; list order) up to
            // CG_IN_MAX, the warp evaluates every group's compacted pairs one pair per lane,
            // and lane 0 of each group continues its sum in order -- the reference's sum,
            // however many rounds a residue needs.
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            int from = 0;  // next list entry of this group
            bool more = use_list;
            while (__any_sync(0xffffffffu, more)) {
                int n_in = 0;
                if (more) {
                    while (from < nl && n_in + G <= CG_IN_MAX) {
                        const int j = from + gl;
                        bool ok = false;
                        int i = 0;
                        if (j < nl) {
                            i = list[j];
                            const float4 a = ca_pq[i];
                            const float r_sq = xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z));
                            ok = !(r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ);
                            if (ok && !(near_adjacent && r_sq <= CG_NEAR_SQ)) {  // the reference's cell test
                                const int4 ce = ca_cell[i];
                                ok = abs((long long)ce.x - cx) <= 1 && abs((long long)ce.y - cy) <= 1 &&
                                     abs((long long)ce.z - cz) <= 1;
                            }
                        }
                        const unsigned m = (__ballot_sync(gmask, ok) >> gshift) & ((1u << G) - 1u);
                        if (ok) in[n_in + __popc(m & ((1u << gl) - 1u))] = i;
                        n_in += __popc(m);
                        from += G;
                    }
                    if (COUNT && gl == 0) n_pairs += n_in;
                }
                // B. the round's pair terms of every residue of the warp, one pair per lane
                int pre[NG + 1];
                pre[0] = 0;
#pragma unroll
                for (int q = 0; q < NG; ++q) pre[q + 1] = pre[q] + __shfl_sync(0xffffffffu, n_in, q * G);
                const int total = pre[NG];
                for (int base = 0; base < total; base += 32) {
                    const int pidx = base + lane;
                    int q = 0;
#pragma unroll
                    for (int t = 1; t < NG; ++t) q += pidx >= pre[t] ? 1 : 0;
                    const int src = q * G;
                    const CgB body{__shfl_sync(0xffffffffu, ca.x, src), __shfl_sync(0xffffffffu, ca.y, src),
                                   __shfl_sync(0xffffffffu, ca.z, src), __shfl_sync(0xffffffffu, res.x, src),
                                   __shfl_sync(0xffffffffu, res.y, src), __shfl_sync(0xffffffffu, res.z, src),
                                   __shfl_sync(0xffffffffu, res.w, src)};
                    // the antigen Calphas of the pair's own residue: the groups of a warp
                    // may probe different antigens
                    const float4* q_pq = reinterpret_cast<const float4*>(
                        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(ca_pq), src));
                    const float4* q_prm = reinterpret_cast<const float4*>(
                        __shfl_sync(0xffffffffu, reinterpret_cast<unsigned long long>(ca_prm), src));
                    if (pidx < total) {
                        const int k = pidx - pre[q];
                        const int i = s_in[rl0 + q][k];
                        float tx, ty, tz;
                        cg_term_parts(body, q_pq[i], q_prm[i], tx, ty, tz);
                        s_term[rl0 + q][k] = make_float3(tx, ty, tz);
                    }
                }
                __syncwarp();
                // C. lane 0 of each group continues its sum in order
                if (gl == 0)
                    for (int k = 0; k < n_in; ++k) {
                        const float3 t = terms[k];
                        sx = xadd(sx, t.x);
                        sy = xadd(sy, t.y);
                        sz = xadd(sz, t.z);
                    }
                __syncwarp();  // term slots are rewritten next round
                more = more && from < nl;
            }
            if (gl == 0 && valid && !use_list) {  // list overflow or cells near the i32 limits
                int np = 0;
                float3 f;
                cg_force_walk<COUNT>(Ap, ca.x, ca.y, ca.z, aa, &f, &np);
                sx = f.x; sy = f.y; sz = f.z;
                if (COUNT) n_pairs += np;
            }
            float fx = __shfl_sync(0xffffffffu, sx, gshift), fy = __shfl_sync(0xffffffffu, sy, gshift),
                  fz = __shfl_sync(0xffffffffu, sz, gshift);
            if (!valid) continue;  // uniform per group; the warp-wide shuffles above were all taken
            // harmonic restraint toward the shell (diffusion.rs:317-327)
            const float dx_c = xsub(ca.x, ag_cx), dy_c = xsub(ca.y, ag_cy), dz_c = xsub(ca.z, ag_cz);
            const float d = fmaxf(xsqrt(xdist2(dx_c, dy_c, dz_c)), 0.001f);
            const float excess = xsub(d, p.shell_radius);
            const float f_r = xdiv(xmul(-p.restraint_k, excess), d);
            fx = xadd(fx, xmul(f_r, dx_c));
            fy = xadd(fy, xmul(f_r, dy_c));
            fz = xadd(fz, xmul(f_r, dz_c));
            float nx = 0.0f, ny = 0.0f, nz = 0.0f;
            if (with_noise) {
                const float temp = temps ? temps[s] : p.t_hot;
                const float sigma = xmul(p.noise_base, xsqrt(temp));
                const U4 u = rng_draw(p.seed, cid, step0 + (uint32_t)s, STREAM_NOISE, (uint32_t)r_local);
                nx = frange(u.x, -sigma, sigma);
                ny = frange(u.y, -sigma, sigma);
                nz = frange(u.z, -sigma, sigma);
            }
            const float md = p.max_disp;
            const F3 new_ca = {xadd(xadd(ca.x, fminf(fmaxf(xmul(p.step, fx), -md), md)), nx),
                               xadd(xadd(ca.y, fminf(fmaxf(xmul(p.step, fy), -md), md)), ny),
                               xadd(xadd(ca.z, fminf(fmaxf(xmul(p.step, fz), -md), md)), nz)};
            // set_ca_pos: delta = new - old; every atom (the Calpha included) += delta
            const F3 dl = sub3(new_ca, ca);
            if (!COUNT) {
#pragma unroll
                for (int j = 0; j < NA; ++j) {
                    at[j].x = xadd(at[j].x, dl.x);
                    at[j].y = xadd(at[j].y, dl.y);
                    at[j].z = xadd(at[j].z, dl.z);
                }
            }
            ca = {xadd(ca.x, dl.x), xadd(ca.y, dl.y), xadd(ca.z, dl.z)};
            if (s + 1 < n_steps) {
                const float mx = ca.x - centre.x, my = ca.y - centre.y, mz = ca.z - centre.z;
                if (!(mx * mx + my * my + mz * mz <= (skin - 0.01f) * (skin - 0.01f))) {
                    // left the skin (or NaN): a new list with twice the skin
                    skin = fminf(2.0f * skin, CG_SKIN_MAX);
                    centre = ca;
                    nl = build_cg_list<G>(g, ca_pq, centre, gl, gmask, list, skin);
                    dirty = true;
                }
            }
        }
        if (!valid) return;  // ends this task
        if (!COUNT && dirty && st.cg_meta) {  // keep the list for the next launch
            for (int j = gl; j < min(nl, CG_LIST_MAX); j += G) st.cg_list[(size_t)r * CG_LIST_MAX + j] = list[j];
            if (gl == 0) {
                st.cg_centre[r] = make_float4(centre.x, centre.y, centre.z, skin);
                st.cg_meta[r] = make_int4(nl, st.cand_ag[c], st.ag_epoch ? *st.ag_epoch : -2, 0);
            }
        }
        if (COUNT) {
            if (gl == 0 && n_pairs) atomicAdd((unsigned long long*)pair_count, (unsigned long long)n_pairs);
            return;
        }
#pragma unroll
        for (int j = 0; j < NA; ++j) {
            const int k = gl + G * j;
            if (k < n_at) slot[k] = at[j];
        }
    };
    // tasks of NG residue slots, one per warp: the warp's own (static grid) or taken
    // from the work queue until it runs dry (persistent grid); warp-uniform
    int task = blockIdx.x * CG_WARPS + (int)(threadIdx.x >> 5);
    for (;;) {
        if (queue) {
            __syncwarp();  // the last task's list reads are done before the next writes
            int t = 0;
            if (lane == 0) t = atomicAdd(queue, 1);
            task = __shfl_sync(0xffffffffu, t, 0);
        }
        if ((long long)task * NG >= st.total_res) break;
        const int slot_id = task * NG + lane / G;
        residue_task(slot_id);
        if (!queue) break;
    }
    if (queue) queue_retire(queue);
}

// ---- gradient steps, flat form -------------------------------------------------------
// The same steps and sums as k_langevin with the work laid out differently.  A warp
// takes R residues (lane q < R owns residue q: its Calpha, list, force sum and
// update).  Each step the warp scans the concatenation of its R residues' Verlet
// lists 32 entries at a time, one entry per lane, whatever list an entry belongs
// to, and compacts the entries that pass the reference's tests into a hit buffer
// in concatenation order -- residue after residue, list order within a residue;
// the hits are then evaluated one pair per lane, and lane q adds its residue's
// terms in that order: the reference's pair set in the reference's order.  Long
// and short lists thereby share the warp's lanes instead of leaving them idle.
// The residue's atoms are not carried through the steps: each step's translation
// (set_ca_pos, allatom.rs:289-293) is recorded and the atoms take the recorded
// translations one after another, in step order, when the record is full and at
// the end -- the same additions in the same order as translating them every step.
// A task's lists live in shared memory (16-bit positions) for the launch and the
// state's list storage carries them between launches; a residue that leaves its
// skin gets a new list built by the whole warp in one pass.  A list that overflows, or a
// cell index near the i32 limits, sends the residue to the one-lane 27-cell walk.
constexpr int FLAT_HCAP = 128;   // hits a warp holds per round
constexpr int FLAT_DSTEPS = 10;  // step translations recorded before the atoms take them
template <int R>
struct FlatWarp {
    float4 body[R];             // Calpha x, y, z of the current step
    float4 prm[R];              // residue-level charge, epsilon, sigma, hydrophobic
    int4 cell[R];               // CG cell of the Calpha, w = cell test needed only beyond CG_NEAR_SQ
    const float4* pq[R];        // the residue's antigen Calphas (shared memory when staged)
    const float4* aprm[R];
    const int4* acell[R];
    int pref[R + 1];            // exclusive prefix of the list lengths scanned this step
    int rid[R];                 // residue index (-1: no residue)
    int nat[R];                 // atoms of the residue
    int hit[FLAT_HCAP];         // residue slot << 26 | antigen Calpha position
    float3 term[FLAT_HCAP];
    float3 dl[FLAT_DSTEPS][R];  // recorded translations
    uint16_t sl[R][CG_LIST_MAX];  // the residues' Verlet lists for the launch (positions)
};

// Apply the recorded translations 0..nd-1 to every atom of the warp's residues.
template <int R>
__device__ __forceinline__ void flat_flush(const StateView& st, FlatWarp<R>& fw, int nd, int lane) {
    __syncwarp();
    for (int t = lane; t < R * SLOTS; t += 32) {
        const int q = t / SLOTS, k = t - q * SLOTS;
        const int r = fw.rid[q];
        if (r < 0 || k >= fw.nat[q]) continue;
        float4* at = st.res_pos + (size_t)r * SLOT_STRIDE + k;
        float4 v = *at;
        for (int d = 0; d < nd; ++d) {
            const float3 u = fw.dl[d][q];
            v.x = xadd(v.x, u.x);
            v.y = xadd(v.y, u.y);
            v.z = xadd(v.z, u.z);
        }
        *at = v;
    }
    __syncwarp();
}

template <int W, int R>
__global__ void __launch_bounds__(W * 32, (R <= 4 ? 32 : 24) / W) k_langevin_flat(StateView st, const AgView* __restrict__ ags, StepParams p,
                                                           int n_steps, uint32_t step0, int with_noise,
                                                           const float* __restrict__ temps, uint32_t* __restrict__ err,
                                                           const int* __restrict__ order, int order_mode,
                                                           int stage_cap, int stage_ag, int* __restrict__ queue) {
    static_assert(R == 4 || R == 8 || R == 16 || R == 32, "residues per warp");
    constexpr int RPC = W * R;  // residues per CTA
    __shared__ int s_stage_ag;
    // dynamic shared memory: the warps' FlatWarp records, then the antigen staging
    extern __shared__ __align__(16) unsigned char cg_dyn_all[];
    FlatWarp<R>* s_fw = reinterpret_cast<FlatWarp<R>*>(cg_dyn_all);
    unsigned char* cg_dyn = cg_dyn_all + W * sizeof(FlatWarp<R>);
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    FlatWarp<R>& fw = s_fw[threadIdx.x >> 5];
    // order 3: the ranks of this launch are the buckets the previous launch filled
    // (cg_bal_* in common.cuh); identity while they do not hold every residue
    __shared__ int s_bpre[CG_BAL_BINS + 1];
    __shared__ int s_bpar, s_bvalid;
    const bool bal = order_mode == 3 && st.cg_bal;
    if (bal) {
        if (threadIdx.x == 0) {
            const int par = st.cg_bal[0] & 1;
            const int* cnt = cg_bal_count(st.cg_bal, par);
            int run = 0;
            for (int b = 0; b < CG_BAL_BINS; ++b) {
                s_bpre[b] = run;
                run += cnt[b];
            }
            s_bpre[CG_BAL_BINS] = run;
            s_bpar = par;
            s_bvalid = run == st.total_res;
        }
        __syncthreads();
    }
    const int bal_T = st.total_res / R, bal_full = bal_T * R;
    auto slot_res = [&](int slot) -> int {
        if (!bal) return res_of_slot(order, order_mode, slot, st.total_res);
        if (!s_bvalid) return slot;
        int rank = slot;
        if (slot < bal_full) {  // snake deal: task t takes ranks j*T + t (j even), j*T + T-1-t (j odd)
            const int t = slot / R, j = slot - t * R;
            rank = j * bal_T + ((j & 1) ? bal_T - 1 - t : t);
        }
        int b = 0;
        while (b + 1 < CG_BAL_BINS && s_bpre[b + 1] <= rank) ++b;
        return cg_bal_bucket(st.cg_bal, st.total_res, s_bpar, b)[rank - s_bpre[b]];
    };
    // antigen staging, as k_langevin does it
    if (threadIdx.x == 0) {
        int a0 = stage_ag, a1 = stage_ag;
        if (a0 < 0 && !queue) {
            const int first = blockIdx.x * RPC;
            const int last = min(first + RPC, st.total_res) - 1;
            a0 = st.cand_ag[st.res_cand[slot_res(first)]];
            a1 = st.cand_ag[st.res_cand[slot_res(last)]];
            if (order_mode >= 2)
                for (int q = first; q <= last && a1 == a0; ++q) a1 = st.cand_ag[st.res_cand[slot_res(q)]];
        }
        bool fits = a0 >= 0 && a0 == a1;
        if (fits) {
            const GridView& gv = ags[a0].ca_grid;
            fits = cg_stage_bytes(ags[a0].n_res, gv.nx * gv.ny * gv.nz) <= (size_t)stage_cap;
        }
        s_stage_ag = fits ? a0 : -1;
    }
    __syncthreads();
    const int sa = s_stage_ag;
    float4* spq = (float4*)cg_dyn;
    float4* sprm = spq;
    int4* scell = (int4*)cg_dyn;
    int* sstart = (int*)cg_dyn;
    if (sa >= 0) {
        const AgView& S = ags[sa];
        const int n = S.n_res, ncell = S.ca_grid.nx * S.ca_grid.ny * S.ca_grid.nz;
        sprm = spq + n;
        scell = (int4*)(sprm + n);
        sstart = (int*)(scell + n);
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            spq[i] = S.ca_pq[i];
            sprm[i] = S.ca_prm[i];
            scell[i] = S.ca_cell[i];
        }
        for (int i = threadIdx.x; i <= ncell; i += blockDim.x) sstart[i] = S.ca_grid.cell_start[i];
        __syncthreads();
    }
    const int epoch = st.ag_epoch ? *st.ag_epoch : -2;

    // Build residue q's list into shared memory with the whole warp (all lanes call;
    // q's antigen, centre and skin are taken from lane q).  Returns the length on
    // every lane.
    auto warp_build = [&](int q, int a, F3 centre, float skin) -> int {
        a = __shfl_sync(0xffffffffu, a, q);
        centre.x = __shfl_sync(0xffffffffu, centre.x, q);
        centre.y = __shfl_sync(0xffffffffu, centre.y, q);
        centre.z = __shfl_sync(0xffffffffu, centre.z, q);
        skin = __shfl_sync(0xffffffffu, skin, q);
        GridView g = ags[a].ca_grid;
        const float4* pq = ags[a].ca_pq;
        if (a == sa) {
            g.cell_start = sstart;
            pq = spq;
        }
        return build_cg_list_warp<uint16_t>(g, pq, centre, lane, fw.sl[q], skin);
    };

    int task = blockIdx.x * W + (int)(threadIdx.x >> 5);
    for (;;) {
        if (queue) {
            __syncwarp();
            int t = 0;
            if (lane == 0) t = atomicAdd(queue, 1);
            task = __shfl_sync(0xffffffffu, t, 0);
        }
        if ((long long)task * R >= st.total_res) break;
        // ---- this lane's residue (lanes >= R own none) ----
        const int slot_id = task * R + lane;
        const bool valid = lane < R && slot_id < st.total_res;
        const int r = valid ? slot_res(slot_id) : 0;
        const int c = valid ? st.res_cand[r] : 0;
        const int r_local = valid ? r - st.cand_res_off[c] : 0;
        const uint32_t cid = valid ? st.cand_id[c] : 0u;
        const int a = valid ? st.cand_ag[c] : 0;
        const AgView* __restrict__ Ap = ags + a;
        const float ginv = Ap->ca_grid.inv, gcell = Ap->ca_grid.cell;
        const float ag_cx = Ap->cx, ag_cy = Ap->cy, ag_cz = Ap->cz;
        const int aa = valid ? st.res_aa[r] : 0;
        F3 ca = {0.f, 0.f, 0.f};
        if (valid) {
            const float4 v1 = st.res_pos[(size_t)r * SLOT_STRIDE + 1];
            ca = {v1.x, v1.y, v1.z};
            if (err && (!isfinite(ca.x) || !isfinite(ca.y) || !isfinite(ca.z))) atomicOr(err, ERRF_NAN);
        }
        if (lane < R) {
            fw.rid[lane] = valid ? r : -1;
            fw.nat[lane] = valid ? s_topo_n[aa] : 0;
            fw.prm[lane] = s_res[aa];
            const bool staged = valid && a == sa;
            fw.pq[lane] = staged ? spq : Ap->ca_pq;
            fw.aprm[lane] = staged ? sprm : Ap->ca_prm;
            fw.acell[lane] = staged ? scell : Ap->ca_cell;
        }
        // the list of the previous launch when it was built for this antigen set and
        // antigen and still covers the Calpha, else a new one
        F3 centre = ca;
        int nl = 0;
        int nreb = 0;  // lists this residue builds in the launch
        bool dirty = false;
        float skin = CG_SKIN;
        bool need = false;
        if (valid) {
            const int4 meta = st.cg_meta[r];
            bool reuse = false;
            if (epoch >= 0 && meta.z == epoch && meta.y == a && meta.x >= 0 && meta.x <= CG_LIST_MAX) {
                const float4 cc = st.cg_centre[r];
                skin = fminf(fmaxf(cc.w, CG_SKIN), CG_SKIN_MAX);
                const float mx = ca.x - cc.x, my = ca.y - cc.y, mz = ca.z - cc.z;
                reuse = mx * mx + my * my + mz * mz <= (skin - 0.01f) * (skin - 0.01f);
                if (reuse) {
                    centre = {cc.x, cc.y, cc.z};
                    nl = meta.x;
                } else {
                    skin = fminf(2.0f * skin, CG_SKIN_MAX);  // it outran the list
                }
            }
            need = !reuse;
        }
        {  // the carried lists into shared memory: all residues' entries, 32 per round
            const int nc = (valid && !need) ? nl : 0;
            int inc = nc;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += v;
            }
            const int tot = __shfl_sync(0xffffffffu, inc, 31);
            if (lane < R) fw.pref[lane + 1] = inc;
            if (lane == 0) fw.pref[0] = 0;
            __syncwarp();
            int q = 0;
            for (int f = lane; f < tot; f += 32) {
                while (fw.pref[q + 1] <= f) ++q;
                const int k = f - fw.pref[q];
                fw.sl[q][k] = (uint16_t)__ldg(st.cg_list + (size_t)fw.rid[q] * CG_LIST_MAX + k);
            }
        }
        __syncwarp();
        for (unsigned m = __ballot_sync(0xffffffffu, need); m; m &= m - 1) {
            const int q = __ffs(m) - 1;
            const int n = warp_build(q, a, centre, skin);
            if (lane == q) {
                nl = n;
                dirty = true;
                ++nreb;
            }
        }
        int nd = 0;  // recorded translations
        for (int s = 0; s < n_steps; ++s) {
            const int cx = cell_coord(ca.x, ginv), cy = cell_coord(ca.y, ginv), cz = cell_coord(ca.z, ginv);
            const bool use_list = valid && nl <= CG_LIST_MAX && !cell_far(cx, cy, cz);
            // cells at least as wide as the cutoff and coordinates below 1e4 A: pairs with
            // r^2 <= CG_NEAR_SQ are in adjacent cells (see k_langevin)
            const bool near_adjacent = gcell >= 10.0f && fabsf(ca.x) < 1e4f && fabsf(ca.y) < 1e4f && fabsf(ca.z) < 1e4f;
            const int nle = use_list ? nl : 0;
            int incl = nle;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += v;
            }
            const int total = __shfl_sync(0xffffffffu, incl, 31);
            const int my_lo = incl - nle;  // this residue's entries: [my_lo, incl)
            if (lane < R) {
                fw.body[lane] = make_float4(ca.x, ca.y, ca.z, 0.f);
                fw.cell[lane] = make_int4(cx, cy, cz, near_adjacent ? 1 : 0);
                fw.pref[lane + 1] = incl;
                if (lane == 0) fw.pref[0] = 0;
            }
            __syncwarp();
            float sx = 0.0f, sy = 0.0f, sz = 0.0f;
            int f0 = 0, rq = 0;
            while (f0 < total) {  // rounds: scan until the hit buffer could overflow
                int nh = 0, my_cnt = 0, my_first = -1;
                while (f0 < total && nh + 32 <= FLAT_HCAP) {
                    const int f = f0 + lane;
                    bool hit = false;
                    int code = 0;
                    if (f < total) {
                        while (fw.pref[rq + 1] <= f) ++rq;
                        const int i = fw.sl[rq][f - fw.pref[rq]];
                        const float4 b = fw.body[rq];
                        const float4 ap = fw.pq[rq][i];
                        const float r_sq = xdist2(xsub(b.x, ap.x), xsub(b.y, ap.y), xsub(b.z, ap.z));
                        hit = !(r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ);
                        const int4 cc = fw.cell[rq];
                        if (hit && !(cc.w && r_sq <= CG_NEAR_SQ)) {  // the reference's cell test
                            const int4 ce = fw.acell[rq][i];
                            hit = abs((long long)ce.x - cc.x) <= 1 && abs((long long)ce.y - cc.y) <= 1 &&
                                  abs((long long)ce.z - cc.z) <= 1;
                        }
                        code = (rq << 26) | i;
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (hit) fw.hit[nh + __popc(m & lt)] = code;
                    // this lane's residue: its hits of the chunk are the ballot bits of its entries
                    const int lo = max(my_lo - f0, 0), hi = min(incl - f0, 32);
                    if (lane < R && hi > lo) {
                        const unsigned mask = (hi == 32 ? 0xffffffffu : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
                        const unsigned mine = m & mask;
                        if (mine && my_first < 0) my_first = nh + __popc(m & ((1u << lo) - 1u));
                        my_cnt += __popc(mine);
                    }
                    nh += __popc(m);
                    f0 += 32;
                }
                __syncwarp();
                for (int h = lane; h < nh; h += 32) {  // the round's pair terms, one pair per lane
                    const int code = fw.hit[h];
                    const int q = code >> 26, i = code & ((1 << 26) - 1);
                    const float4 b = fw.body[q], bp = fw.prm[q];
                    const CgB body{b.x, b.y, b.z, bp.x, bp.y, bp.z, bp.w};
                    float tx, ty, tz;
                    cg_term_parts(body, fw.pq[q][i], fw.aprm[q][i], tx, ty, tz);
                    fw.term[h] = make_float3(tx, ty, tz);
                }
                __syncwarp();
                for (int k = 0; k < my_cnt; ++k) {  // this residue's terms, in order
                    const float3 t = fw.term[my_first + k];
                    sx = xadd(sx, t.x);
                    sy = xadd(sy, t.y);
                    sz = xadd(sz, t.z);
                }
                __syncwarp();  // hit and term slots are rewritten next round
            }
            if (valid && !use_list) {  // list overflow or cells near the i32 limits
                int np = 0;
                float3 f;
                cg_force_walk<false>(Ap, ca.x, ca.y, ca.z, aa, &f, &np);
                sx = f.x; sy = f.y; sz = f.z;
            }
            bool rebuild = false;
            if (valid) {
                float fx = sx, fy = sy, fz = sz;
                // harmonic restraint toward the shell (diffusion.rs:317-327)
                const float dx_c = xsub(ca.x, ag_cx), dy_c = xsub(ca.y, ag_cy), dz_c = xsub(ca.z, ag_cz);
                const float d = fmaxf(xsqrt(xdist2(dx_c, dy_c, dz_c)), 0.001f);
                const float excess = xsub(d, p.shell_radius);
                const float f_r = xdiv(xmul(-p.restraint_k, excess), d);
                fx = xadd(fx, xmul(f_r, dx_c));
                fy = xadd(fy, xmul(f_r, dy_c));
                fz = xadd(fz, xmul(f_r, dz_c));
                float nx = 0.0f, ny = 0.0f, nz = 0.0f;
                if (with_noise) {
                    const float temp = temps ? temps[s] : p.t_hot;
                    const float sigma = xmul(p.noise_base, xsqrt(temp));
                    const U4 u = rng_draw(p.seed, cid, step0 + (uint32_t)s, STREAM_NOISE, (uint32_t)r_local);
                    nx = frange(u.x, -sigma, sigma);
                    ny = frange(u.y, -sigma, sigma);
                    nz = frange(u.z, -sigma, sigma);
                }
                const float md = p.max_disp;
                const F3 new_ca = {xadd(xadd(ca.x, fminf(fmaxf(xmul(p.step, fx), -md), md)), nx),
                                   xadd(xadd(ca.y, fminf(fmaxf(xmul(p.step, fy), -md), md)), ny),
                                   xadd(xadd(ca.z, fminf(fmaxf(xmul(p.step, fz), -md), md)), nz)};
                // set_ca_pos: delta = new - old; every atom (the Calpha included) += delta
                const F3 dl = sub3(new_ca, ca);
                fw.dl[nd][lane] = make_float3(dl.x, dl.y, dl.z);
                ca = {xadd(ca.x, dl.x), xadd(ca.y, dl.y), xadd(ca.z, dl.z)};
                if (s + 1 < n_steps) {
                    const float mx = ca.x - centre.x, my = ca.y - centre.y, mz = ca.z - centre.z;
                    if (!(mx * mx + my * my + mz * mz <= (skin - 0.01f) * (skin - 0.01f))) {
                        // left the skin (or NaN): a new list with twice the skin
                        skin = fminf(2.0f * skin, CG_SKIN_MAX);
                        centre = ca;
                        rebuild = true;
                    }
                }
            }
            if (++nd == FLAT_DSTEPS || s + 1 == n_steps) {
                flat_flush<R>(st, fw, nd, lane);
                nd = 0;
            }
            for (unsigned m = __ballot_sync(0xffffffffu, rebuild); m; m &= m - 1) {
                const int q = __ffs(m) - 1;
                const int n = warp_build(q, a, centre, skin);
                if (lane == q) {
                    nl = n;
                    dirty = true;
                    ++nreb;
                }
            }
        }
        if (valid && dirty) {  // keep the list for the next launch
            st.cg_centre[r] = make_float4(centre.x, centre.y, centre.z, skin);
            st.cg_meta[r] = make_int4(nl, a, epoch, 0);
        }
        if (bal && valid) {  // the next launch's ranks: this residue into its work band
            const int w = min(255, (nl <= CG_LIST_MAX ? nl : 200) + 32 * nreb);
            const int band = (255 - w) >> 4;
            const int k = atomicAdd(cg_bal_count(st.cg_bal, s_bpar ^ 1) + band, 1);
            if (k < st.total_res) cg_bal_bucket(st.cg_bal, st.total_res, s_bpar ^ 1, band)[k] = r;
        }
        {  // rebuilt lists back to the state's list storage, all residues' entries at once
            const int nc = (valid && dirty && nl <= CG_LIST_MAX) ? nl : 0;
            int inc = nc;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, inc, d);
                if (lane >= d) inc += v;
            }
            const int tot = __shfl_sync(0xffffffffu, inc, 31);
            __syncwarp();
            if (lane < R) fw.pref[lane + 1] = inc;
            if (lane == 0) fw.pref[0] = 0;
            __syncwarp();
            int q = 0;
            for (int f = lane; f < tot; f += 32) {
                while (fw.pref[q + 1] <= f) ++q;
                const int k = f - fw.pref[q];
                st.cg_list[(size_t)fw.rid[q] * CG_LIST_MAX + k] = fw.sl[q][k];
            }
            __syncwarp();
        }
        if (!queue) break;
    }
    if (queue) queue_retire(queue);
    if (bal) {  // the last CTA empties the buckets it read and hands the new ones over
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(st.cg_bal + 1, 1) == (int)gridDim.x - 1) {
                int* cnt = cg_bal_count(st.cg_bal, s_bpar);
                for (int b = 0; b < CG_BAL_BINS; ++b) cnt[b] = 0;
                st.cg_bal[1] = 0;
                __threadfence();
                atomicAdd(st.cg_bal, 1);
            }
        }
    }
}

// ---- launchers ----------------------------------------------------------------------
void launch_build_residues(cudaStream_t s, int n, const float* ca_xyz, const uint8_t* aa, const float4* chi_trig,
                           const float* chi_deg, float4* out_pos, float4* out_chi) {
    if (n > 0) k_build_residues<<<(n + 127) / 128, 128, 0, s>>>(n, ca_xyz, aa, chi_trig, chi_deg, out_pos, out_chi);
}

void launch_cg_forces(cudaStream_t s, const AgView* ag, const float* bx, const float* by, const float* bz,
                      const uint8_t* baa, int n, float* fx, float* fy, float* fz) {
    if (n > 0) k_cg_forces<<<(n + 127) / 128, 128, 0, s>>>(ag, bx, by, bz, baa, n, fx, fy, fz);
}

// ---- residue order by Calpha cell (counting sort with atomic slots) ----------------
// Key = the antigen's cell base + the clamped Calpha cell in that antigen's CG box.
// The order inside a cell is arbitrary: every residue is still computed by exactly
// one thread with the same arithmetic, so the results do not depend on it.
__device__ __forceinline__ int res_key(const StateView& st, const AgView* ags, const int* key_base, int r) {
    const int c = st.res_cand[r];
    const int a = st.cand_ag[c];
    const GridView& g = ags[a].ca_grid;
    const float4 ca = st.res_pos[(size_t)r * SLOT_STRIDE + 1];
    // the antigen's CG box widened by RES_KEY_MARGIN cells on every side (antibody
    // residues sit around the antigen); positions further out share the edge keys
    const int M = RES_KEY_MARGIN;
    const int kx = g.nx + 2 * M, ky = g.ny + 2 * M, kz = g.nz + 2 * M;
    const int ix = min(max(cell_coord(ca.x, g.inv) - g.ox + M, 0), kx - 1);
    const int iy = min(max(cell_coord(ca.y, g.inv) - g.oy + M, 0), ky - 1);
    const int iz = min(max(cell_coord(ca.z, g.inv) - g.oz + M, 0), kz - 1);
    return key_base[a] + (ix * ky + iy) * kz + iz;
}
__global__ void k_res_key_hist(StateView st, const AgView* __restrict__ ags, const int* __restrict__ key_base,
                               int* __restrict__ keys, int* __restrict__ counts) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= st.total_res) return;
    const int k = res_key(st, ags, key_base, r);
    keys[r] = k;
    atomicAdd(&counts[k], 1);
}
__global__ void k_res_scatter(int n, const int* __restrict__ keys, int* __restrict__ cursor, int* __restrict__ order) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    order[atomicAdd(&cursor[keys[r]], 1)] = r;
}

void launch_residue_order(cudaStream_t s, const StateView& st, const AgView* ags, const int* key_base, int n_keys,
                          int* keys, int* counts, int* cursor, int* order) {
    if (st.total_res <= 0) return;
    cudaMemsetAsync(counts, 0, (size_t)n_keys * sizeof(int), s);
    k_res_key_hist<<<(st.total_res + 255) / 256, 256, 0, s>>>(st, ags, key_base, keys, counts);
    launch_exclusive_scan(s, counts, n_keys, cursor);
    k_res_scatter<<<(st.total_res + 255) / 256, 256, 0, s>>>(st.total_res, keys, cursor, order);
}

template <int W, int G>
static void diffuse_w(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                      uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order,
                      int order_mode, int stage_bytes, int stage_ag, int* queue) {
    const int threads = W * 32;
    const long long total = (long long)st.total_res * G;
    long long ctas = (total + threads - 1) / threads;
    auto kern = k_langevin<false, W, G>;
    if (stage_bytes > 0) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, stage_bytes);
    if (queue) {  // persistent: the CTAs that are resident at once
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, stage_bytes);
        ctas = std::min(ctas, (long long)std::max(1, sms * std::max(per_sm, 1)));
    }
    kern<<<(int)ctas, threads, stage_bytes, s>>>(st, ags, p, n_steps, step0, with_noise, temps, err, nullptr, order,
                                                 order_mode, stage_bytes, stage_ag, queue);
}

template <int W, int R>
static void diffuse_flat(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                         uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order,
                         int order_mode, int stage_bytes, int stage_ag, int* queue) {
    const int threads = W * 32;
    const long long tasks = ((long long)st.total_res + R - 1) / R;
    long long ctas = (tasks + W - 1) / W;
    auto kern = k_langevin_flat<W, R>;
    const int dyn = (int)(W * sizeof(FlatWarp<R>)) + stage_bytes;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
    if (queue) {  // persistent: the CTAs that are resident at once
        int dev = 0, sms = 0, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, dyn);
        ctas = std::min(ctas, (long long)std::max(1, sms * std::max(per_sm, 1)));
    }
    kern<<<(int)ctas, threads, dyn, s>>>(st, ags, p, n_steps, step0, with_noise, temps, err, order, order_mode,
                                         stage_bytes, stage_ag, queue);
}

void launch_diffuse(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                    uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order,
                    int warps_per_cta, int lanes_per_res, int order_mode, int max_ag_res, int max_ag_cells,
                    int stage_ag, int* queue, int flat_res) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    if (order_mode == 2 && st.total_res % CG_STRIDE == 0) order_mode = 1;  // stride not a bijection
    // antigen staging: up to 96 KB of dynamic shared memory per CTA
    const size_t sb = cg_stage_bytes(max_ag_res, max_ag_cells);
    const int stage = sb <= 96 * 1024 ? (int)sb : 0;
    // the flat form keeps 16-bit list positions: antigens of at most 65536 Calphas
    if (flat_res && st.cg_list && st.cg_meta && st.cg_centre && max_ag_res <= 65536) {
#define BINDER_FLAT(W, R)                                                                                    \
    diffuse_flat<W, R>(s, st, ags, p, n_steps, step0, with_noise, temps, err, order, order_mode, stage,          \
                       stage ? stage_ag : -1, queue)
        if (flat_res == 32) BINDER_FLAT(4, 32);
        else if (flat_res == 16) {
            if (warps_per_cta <= 4) BINDER_FLAT(4, 16);
            else BINDER_FLAT(8, 16);
        } else if (flat_res == 4) {
            if (warps_per_cta <= 4) BINDER_FLAT(4, 4);
            else BINDER_FLAT(8, 4);
        } else {
            if (warps_per_cta <= 4) BINDER_FLAT(4, 8);
            else BINDER_FLAT(8, 8);
        }
#undef BINDER_FLAT
        return;
    }
#define BINDER_DIFFUSE(W, G)                                                                                 \
    diffuse_w<W, G>(s, st, ags, p, n_steps, step0, with_noise, temps, err, order, order_mode, stage,               \
                    stage ? stage_ag : -1, queue)
    if (lanes_per_res == 8) {
        switch (warps_per_cta) {
            case 2: BINDER_DIFFUSE(2, 8); break;
            case 8: BINDER_DIFFUSE(8, 8); break;
            default: BINDER_DIFFUSE(4, 8); break;
        }
    } else {  // four lanes: at most four warps per CTA (list storage)
        if (warps_per_cta == 2) BINDER_DIFFUSE(2, 4);
        else BINDER_DIFFUSE(4, 4);
    }
#undef BINDER_DIFFUSE
}

void launch_diffuse_count(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          long long* pairs) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    const int threads = 4 * 32;
    const long long total = (long long)st.total_res * 4;
    k_langevin<true, 4, 4><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(
        st, ags, p, n_steps, 0, 0, nullptr, nullptr, pairs, nullptr, 1, 0, -1, nullptr);
}

}  // namespace binder

namespace binder {

// ---- slot-layout packing: host float[n][14][3] <-> device float4[n][16] ------------
__global__ void k_pack_slots(int n_res, const float* __restrict__ in, float4* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_res * SLOT_STRIDE) return;
    const int r = t / SLOT_STRIDE, k = t % SLOT_STRIDE;
    out[t] = k < SLOTS ? make_float4(in[(r * SLOTS + k) * 3], in[(r * SLOTS + k) * 3 + 1], in[(r * SLOTS + k) * 3 + 2], 0.f)
                       : make_float4(0.f, 0.f, 0.f, 0.f);
}
__global__ void k_unpack_slots(int n_res, const float4* __restrict__ in, float* __restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_res * SLOTS) return;
    const int r = t / SLOTS, k = t % SLOTS;
    const float4 v = in[r * SLOT_STRIDE + k];
    out[3 * t] = v.x; out[3 * t + 1] = v.y; out[3 * t + 2] = v.z;
}

// ---- resident-state gather (survivor selection) -------------------------------------
__global__ void k_gather_state(int total, const int* __restrict__ map, const uint8_t* __restrict__ aa,
                               const float4* __restrict__ chi, const float4* __restrict__ trig,
                               const float4* __restrict__ pos, uint8_t* __restrict__ o_aa, float4* __restrict__ o_chi,
                               float4* __restrict__ o_trig, float4* __restrict__ o_pos, int n_cand,
                               const int* __restrict__ cidx, const long long* __restrict__ stats,
                               long long* __restrict__ o_stats) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < (long long)total * SLOT_STRIDE) {
        const int r = (int)(t / SLOT_STRIDE), k = (int)(t % SLOT_STRIDE);
        const int src = map[r];
        o_pos[t] = pos[(size_t)src * SLOT_STRIDE + k];
        if (k == 0) {
            o_aa[r] = aa[src];
            o_chi[r] = chi[src];
        }
        if (k < 2 && trig) o_trig[2 * r + k] = trig[2 * src + k];
    }
    if (t < 4ll * n_cand) o_stats[t] = stats[4 * cidx[t / 4] + t % 4];
}
void launch_gather_state(cudaStream_t s, int total, const int* map, const uint8_t* aa, const float4* chi,
                         const float4* trig, const float4* pos, uint8_t* o_aa, float4* o_chi, float4* o_trig,
                         float4* o_pos, int n_cand, const int* cidx, const long long* stats, long long* o_stats) {
    const long long n = std::max((long long)total * SLOT_STRIDE, 4ll * n_cand);
    if (n > 0)
        k_gather_state<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(total, map, aa, chi, trig, pos, o_aa, o_chi, o_trig,
                                                                   o_pos, n_cand, cidx, stats, o_stats);
}

void launch_pack_slots(cudaStream_t s, int n_res, const float* in, float4* out) {
    if (n_res > 0) k_pack_slots<<<(n_res * SLOT_STRIDE + 255) / 256, 256, 0, s>>>(n_res, in, out);
}
void launch_unpack_slots(cudaStream_t s, int n_res, const float4* in, float* out) {
    if (n_res > 0) k_unpack_slots<<<(n_res * SLOTS + 255) / 256, 256, 0, s>>>(n_res, in, out);
}

}  // namespace binder
