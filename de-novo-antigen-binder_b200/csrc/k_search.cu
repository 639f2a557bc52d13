// k_search.cu — residue construction and the gradient-phase search step on the GPU.
//
//  * protein_from_ca_trace (allatom.rs:523-541): ideal backbone + NERF side chain
//    per residue, one thread each.
//  * compute_forces_with_grid (energy.rs:322-398) for a batch of bodies.
//  * The Langevin part of allatom_diffusion_step (diffusion.rs:306-339) without
//    Metropolis moves: four lanes per residue probe the Calpha grid, the pair
//    terms are folded in the reference's order, and n_steps are fused per launch
//    since in this phase every residue moves independently.
//  * The residue visiting order by Calpha cell and the slot packing kernels.
#include <algorithm>

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
// Four lanes per residue (eight residues per warp, residues in Calpha-cell order).
// The 27 probe cells, in the reference's order, are split into four contiguous
// runs, one per lane; each lane tests its cells' atoms and evaluates the in-cutoff
// pair terms of its run into shared memory.  The accumulator then passes lane 0 ->
// 1 -> 2 -> 3 and each lane folds its own terms in order: exactly the reference's
// sequential sum, with the probing and the IEEE-exact pair math spread over four
// lanes.  A lane whose run holds more than CG_TERMS in-cutoff pairs sends the
// residue to the one-lane walk over all 27 cells (same sum).  Per-step translations
// are recorded and applied to the residue's atoms at the end, atom k on lane k % 4
// (the same sequence of roundings as set_ca_pos, allatom.rs:279-293).
// COUNT: count the in-cutoff pairs of the same trajectory, leave the state as is.
constexpr int CG_GROUP = 4;
// in-cutoff terms a lane holds per step (static shared memory stays under 48 KB)
template <int CG_WARPS>
constexpr int cg_terms() { return CG_WARPS >= 8 ? 15 : 24; }
constexpr int CG_MAX_STEPS = 32;  // steps per launch (the host splits longer runs)

template <bool COUNT, int CG_WARPS>
__global__ void __launch_bounds__(CG_WARPS * 32) k_langevin(StateView st, const AgView* __restrict__ ags,
                                                             StepParams p, int n_steps, uint32_t step0,
                                                             int with_noise, const float* __restrict__ temps,
                                                             uint32_t* __restrict__ err,
                                                             long long* __restrict__ pair_count,
                                                             const int* __restrict__ order) {
    constexpr int CG_TERMS = cg_terms<CG_WARPS>();
    __shared__ float3 s_terms[CG_WARPS * 32][CG_TERMS];
    const int lane = threadIdx.x & 31;
    const int gl = lane & (CG_GROUP - 1);
    const int gshift = lane & ~(CG_GROUP - 1);
    const unsigned gmask = ((1u << CG_GROUP) - 1u) << gshift;
    const int slot_id = (blockIdx.x * blockDim.x + threadIdx.x) / CG_GROUP;
    if (slot_id >= st.total_res) return;  // the whole group leaves together
    const int r = order ? order[slot_id] : slot_id;
    const int c = st.res_cand[r];
    const int r_local = r - st.cand_res_off[c];
    const uint32_t cid = st.cand_id[c];
    const AgView A = ags[st.cand_ag[c]];  // by value: the fields live in registers
    const int aa = st.res_aa[r];
    const int n_at = s_topo_n[aa];
    const float4 res = s_res[aa];
    float4* slot = st.res_pos + (size_t)r * SLOT_STRIDE;
    const float4 v1 = slot[1];  // Calpha = topology atom 1 of every residue (amber.rs:358-377)
    F3 ca = {v1.x, v1.y, v1.z};
    if (gl == 0 && err && (!isfinite(ca.x) || !isfinite(ca.y) || !isfinite(ca.z))) atomicOr(err, ERRF_NAN);
    float3* my_terms = s_terms[threadIdx.x];
    const GridView& g = A.ca_grid;
    // this lane's run of the 9 probe columns (dx, dy), in the reference's order
    const int c0 = gl == 0 ? 0 : 1 + 2 * gl, c1 = gl == 0 ? 3 : 3 + 2 * gl;
    F3 delta[CG_MAX_STEPS];
    int n_pairs = 0;
    for (int s = 0; s < n_steps; ++s) {
        const CgB body{ca.x, ca.y, ca.z, res.x, res.y, res.z, res.w};
        const int cx = cell_coord(ca.x, g.inv), cy = cell_coord(ca.y, g.inv), cz = cell_coord(ca.z, g.inv);
        // Squared distances from the Calpha to the lower / upper neighbour slab in each
        // dimension; a cell beyond the cutoff (+1 mA, above the f32 rounding of r^2
        // and of the slab bounds) holds no in-cutoff atom, so skipping it changes
        // nothing.  For fixed (dx, dy) the three cells dz = -1..1 are one contiguous
        // range of the sorted array, visited in the reference's order.
        const float reach = 10.001f + 4e-7f * (fabsf(ca.x) + fabsf(ca.y) + fabsf(ca.z));
        const float reach2 = reach * reach;
        const float xm = fmaxf(ca.x - (float)cx * g.cell, 0.f), xp = fmaxf((float)(cx + 1) * g.cell - ca.x, 0.f);
        const float ym = fmaxf(ca.y - (float)cy * g.cell, 0.f), yp = fmaxf((float)(cy + 1) * g.cell - ca.y, 0.f);
        const float zm = fmaxf(ca.z - (float)cz * g.cell, 0.f), zp = fmaxf((float)(cz + 1) * g.cell - ca.z, 0.f);
        // cell indices near the i32 limits: the one-lane walk reproduces the wrapping
        const bool far = abs(cx) > (1 << 29) || abs(cy) > (1 << 29) || abs(cz) > (1 << 29);
        int nt = 0;
        if (!far) {
            for (int col = c0; col < c1; ++col) {
                const int dx = col >= 6 ? 1 : (col >= 3 ? 0 : -1);
                const int dy = col - 3 * (dx + 1) - 1;
                const float ddx = dx < 0 ? xm : (dx > 0 ? xp : 0.f);
                const float ddy = dy < 0 ? ym : (dy > 0 ? yp : 0.f);
                const float dxy = ddx * ddx + ddy * ddy;
                if (dxy > reach2) continue;
                const long long X = (long long)cx + dx - g.ox, Y = (long long)cy + dy - g.oy;
                if (X < 0 || Y < 0 || X >= g.nx || Y >= g.ny) continue;
                long long zl = (dxy + zm * zm > reach2) ? cz : (long long)cz - 1;
                long long zh = (dxy + zp * zp > reach2) ? cz : (long long)cz + 1;
                zl = max(zl - g.oz, 0ll);
                zh = min(zh - g.oz, (long long)g.nz - 1);
                if (zl > zh) continue;
                const int base = ((int)X * g.ny + (int)Y) * g.nz;
                const int a1 = g.cell_start[base + (int)zh + 1];
                for (int i = g.cell_start[base + (int)zl]; i < a1; ++i) {
                    float tx, ty, tz;
                    if (!cg_term_parts(body, A.ca_pq[i], A.ca_prm[i], tx, ty, tz)) continue;
                    if (nt < CG_TERMS) my_terms[nt] = make_float3(tx, ty, tz);
                    ++nt;
                }
            }
            if (COUNT) n_pairs += nt;
        }
        const bool overflow = (__ballot_sync(gmask, far || nt > CG_TERMS) & gmask) != 0u;
        float sx = 0.0f, sy = 0.0f, sz = 0.0f;
        if (!overflow) {
#pragma unroll
            for (int L = 0; L < CG_GROUP; ++L) {
                if (gl == L)
                    for (int k = 0; k < nt; ++k) {
                        const float3 t = my_terms[k];
                        sx = xadd(sx, t.x);
                        sy = xadd(sy, t.y);
                        sz = xadd(sz, t.z);
                    }
                sx = __shfl_sync(gmask, sx, L, CG_GROUP);
                sy = __shfl_sync(gmask, sy, L, CG_GROUP);
                sz = __shfl_sync(gmask, sz, L, CG_GROUP);
            }
        } else {
            int np = 0;
            if (gl == 0) cg_force<COUNT>(A, body, sx, sy, sz, &np);
            if (COUNT && far) n_pairs += np;  // lanes did not count when far
            sx = __shfl_sync(gmask, sx, 0, CG_GROUP);
            sy = __shfl_sync(gmask, sy, 0, CG_GROUP);
            sz = __shfl_sync(gmask, sz, 0, CG_GROUP);
        }
        float fx = sx, fy = sy, fz = sz;
        // harmonic restraint toward the shell (diffusion.rs:317-327)
        const float dx_c = xsub(ca.x, A.cx), dy_c = xsub(ca.y, A.cy), dz_c = xsub(ca.z, A.cz);
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
        delta[s] = dl;
        ca = {xadd(ca.x, dl.x), xadd(ca.y, dl.y), xadd(ca.z, dl.z)};
    }
    if (COUNT) {
        if (n_pairs) atomicAdd((unsigned long long*)pair_count, (unsigned long long)n_pairs);
        return;
    }
    for (int k = gl; k < n_at; k += CG_GROUP) {
        float4 v = slot[k];
        for (int s = 0; s < n_steps; ++s) {
            v.x = xadd(v.x, delta[s].x);
            v.y = xadd(v.y, delta[s].y);
            v.z = xadd(v.z, delta[s].z);
        }
        slot[k] = v;
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

template <int W>
static void diffuse_w(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                      uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order) {
    const int threads = W * 32;
    const long long total = (long long)st.total_res * CG_GROUP;
    for (int s0 = 0; s0 < n_steps; s0 += CG_MAX_STEPS) {
        const int ns = min(CG_MAX_STEPS, n_steps - s0);
        k_langevin<false, W><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(
            st, ags, p, ns, step0 + (uint32_t)s0, with_noise, temps ? temps + s0 : nullptr, err, nullptr, order);
    }
}

void launch_diffuse(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                    uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order,
                    int warps_per_cta) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    switch (warps_per_cta) {
        case 2: diffuse_w<2>(s, st, ags, p, n_steps, step0, with_noise, temps, err, order); break;
        case 8: diffuse_w<8>(s, st, ags, p, n_steps, step0, with_noise, temps, err, order); break;
        default: diffuse_w<4>(s, st, ags, p, n_steps, step0, with_noise, temps, err, order); break;
    }
}

void launch_diffuse_count(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          long long* pairs) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    const int threads = 4 * 32;
    const long long total = (long long)st.total_res * CG_GROUP;
    k_langevin<true, 4><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(
        st, ags, p, min(n_steps, CG_MAX_STEPS), 0, 0, nullptr, nullptr, pairs, nullptr);
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
        if (k < 2) o_trig[2 * r + k] = trig[2 * src + k];
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
