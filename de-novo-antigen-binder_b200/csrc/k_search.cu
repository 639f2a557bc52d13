// k_search.cu — residue geometry and the search step on the GPU.
//
//  * NERF side-chain placement (rotamer.rs:198-232, 439-462) and residue
//    construction around a Calpha (allatom.rs:502-541) in the slot layout.
//  * The coarse-grained force of compute_forces_with_grid (energy.rs:322-398),
//    bit-exact with the reference's f32 order: one thread per antibody residue
//    walks the 27 cells in the reference's order and accumulates sequentially
//    with separately rounded operations.
//  * The Langevin part of allatom_diffusion_step (diffusion.rs:315-339):
//    restraint toward the shell, 2 A clamp, uniform noise, rigid translation of
//    the residue (set_ca_pos, allatom.rs:279-293) — fused over n_steps in one
//    launch, since in the gradient phase every residue moves independently.
//
// All sin/cos values of the NERF programs are of table angles (bond angles, fixed
// dihedrals, rotamer chis); they are evaluated once on the host with the C
// library's sinf/cosf and read from constant memory, so residue geometry is
// bit-identical to the CPU restatement of the reference.
#include <cmath>

#include "kernels.h"

namespace binder {

__constant__ int s_topo_n[N_AA];
__constant__ int s_sc_n[N_AA];
__constant__ uchar4 s_sc_ref[N_AA][9];     // ref a, b, c, chi index (255 = fixed)
__constant__ float4 s_sc_geom[N_AA][9];    // bond, sin(angle), cos(angle), unused
__constant__ float2 s_sc_fix[N_AA][9];     // sin, cos of the fixed dihedral
__constant__ int s_rot_n[N_AA];
__constant__ float4 s_rot_chi[N_AA][5];    // chi1..chi4 in degrees
__constant__ float2 s_rot_trig[N_AA][5][4];// sin, cos of each rotamer chi
__constant__ float4 s_res[N_AA];           // residue-level charge, epsilon, sigma, hydrophobic (atom.rs:55-104)

// Rust's f32::to_radians multiplies by the f32 constant PI/180.
static const float RADS_PER_DEG = 3.14159265358979323846f / 180.0f;

cudaError_t search_init_tables() {
    uchar4 ref[N_AA][9];
    float4 geom[N_AA][9];
    float2 fix[N_AA][9];
    float4 rchi[N_AA][5];
    float2 rtrig[N_AA][5][4];
    float4 res[N_AA];
    for (int a = 0; a < N_AA; ++a) {
        for (int k = 0; k < 9; ++k) {
            ref[a][k] = make_uchar4(BT_SC_REF[a][k][0], BT_SC_REF[a][k][1], BT_SC_REF[a][k][2], BT_SC_REF[a][k][3]);
            const float ang = BT_SC_GEOM[a][k][1] * RADS_PER_DEG;
            const float dih = BT_SC_GEOM[a][k][2] * RADS_PER_DEG;
            geom[a][k] = make_float4(BT_SC_GEOM[a][k][0], std::sin(ang), std::cos(ang), 0.f);
            fix[a][k] = make_float2(std::sin(dih), std::cos(dih));
        }
        for (int r = 0; r < 5; ++r) {
            rchi[a][r] = make_float4(BT_ROT_CHI[a][r][0], BT_ROT_CHI[a][r][1], BT_ROT_CHI[a][r][2], BT_ROT_CHI[a][r][3]);
            for (int c = 0; c < 4; ++c) {
                const float x = BT_ROT_CHI[a][r][c] * RADS_PER_DEG;
                rtrig[a][r][c] = make_float2(std::sin(x), std::cos(x));
            }
        }
        res[a] = make_float4(BT_RES[a][0], BT_RES[a][1], BT_RES[a][2], BT_RES[a][3]);
    }
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(s_topo_n, BT_TOPO_N, sizeof(BT_TOPO_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_n, BT_SC_N, sizeof(BT_SC_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_ref, ref, sizeof(ref))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_geom, geom, sizeof(geom))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_fix, fix, sizeof(fix))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_n, BT_ROT_N, sizeof(BT_ROT_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_chi, rchi, sizeof(rchi))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_trig, rtrig, sizeof(rtrig))) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(s_res, res, sizeof(res));
}

// ---- exact vector helpers (allatom.rs:481-489, rotamer.rs:234-252) ----------------
struct F3 { float x, y, z; };
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)}; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
            xsub(xmul(a.x, b.y), xmul(a.y, b.x))};
}
__device__ __forceinline__ F3 norm3(F3 v) {
    const float len = fmaxf(xsqrt(xdist2(v.x, v.y, v.z)), 1e-8f);
    return {xdiv(v.x, len), xdiv(v.y, len), xdiv(v.z, len)};
}

// place_atom (rotamer.rs:198-232) with precomputed sin/cos of angle and dihedral.
__device__ __forceinline__ F3 place_atom(F3 a, F3 b, F3 c, float bond, float sa, float ca, float sd, float cd) {
    const F3 bc = norm3(sub3(b, c));
    const F3 ba = sub3(b, a);
    const F3 n = norm3(cross3(ba, bc));
    const F3 m = cross3(bc, n);
    const float sacd = xmul(sa, cd), sasd = xmul(sa, sd), nca = -ca;
    return {xadd(c.x, xmul(bond, xadd(xadd(xmul(nca, bc.x), xmul(sacd, m.x)), xmul(sasd, n.x)))),
            xadd(c.y, xmul(bond, xadd(xadd(xmul(nca, bc.y), xmul(sacd, m.y)), xmul(sasd, n.y)))),
            xadd(c.z, xmul(bond, xadd(xadd(xmul(nca, bc.z), xmul(sacd, m.z)), xmul(sasd, n.z))))};
}

// Side-chain trigonometry of one residue: sin/cos of chi1..chi4.
struct ChiTrig { float2 t[4]; };
__device__ __forceinline__ ChiTrig rot_trig(int aa, int rot) {
    ChiTrig c;
#pragma unroll
    for (int i = 0; i < 4; ++i) c.t[i] = s_rot_trig[aa][rot][i];
    return c;
}

// build_side_chain (rotamer.rs:439-462): atoms[0..n_bb) hold the backbone; side-chain
// atoms are appended at n_bb.. in program order (= topology order).
__device__ __forceinline__ void build_side_chain(int aa, F3* atoms, int n_bb, const ChiTrig& chi) {
    const int n = s_sc_n[aa];
    for (int k = 0; k < n; ++k) {
        const uchar4 r = s_sc_ref[aa][k];
        const float4 g = s_sc_geom[aa][k];
        float2 d;
        if (r.w == 255) d = s_sc_fix[aa][k];
        else d = chi.t[r.w];
        atoms[n_bb + k] = place_atom(atoms[r.x], atoms[r.y], atoms[r.z], g.x, g.y, g.z, d.x, d.y);
    }
}

// build_ideal_backbone_around_ca (allatom.rs:502-517); returns the backbone length
__device__ __forceinline__ int ideal_backbone(F3 ca, int aa, F3* out) {
    const F3 c = {xadd(ca.x, CA_C_BOND), ca.y, ca.z};
    out[0] = {xsub(ca.x, N_CA_BOND), ca.y, ca.z};
    out[1] = ca;
    out[2] = c;
    out[3] = {xadd(c.x, 0.5f), xadd(c.y, xmul(C_O_BOND, 0.9f)), c.z};
    out[4] = {ca.x, xsub(ca.y, CA_CB_BOND), ca.z};
    return aa == GLY ? 4 : 5;
}

__device__ __forceinline__ void store_residue(float4* slot, const F3* atoms, int n) {
#pragma unroll
    for (int k = 0; k < SLOT_STRIDE; ++k)
        slot[k] = k < n ? make_float4(atoms[k].x, atoms[k].y, atoms[k].z, 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
}

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

// ---- coarse-grained force (energy.rs:322-398), reference f32 order ---------------
struct CgB { float x, y, z, q, eps, sig; float hyd; };

// The three products f_total*dx, f_total*dy, f_total*dz of one pair term of
// compute_forces_with_grid (energy.rs:362-391); false outside 0.25 <= r^2 <= 100.
__device__ __forceinline__ bool cg_term_parts(const CgB& b, const float4 apq, const float4 aprm, float& tx, float& ty,
                                              float& tz) {
    const float ddx = xsub(b.x, apq.x), ddy = xsub(b.y, apq.y), ddz = xsub(b.z, apq.z);
    const float r_sq = xdist2(ddx, ddy, ddz);
    if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) return false;
    const float eps_ij = xsqrt(xmul(b.eps, aprm.x));
    const float sig_ij = xmul(0.5f, xadd(b.sig, aprm.y));
    const float sigma_sq = xmul(sig_ij, sig_ij);
    const float s2 = xdiv(sigma_sq, r_sq);
    const float s6 = xmul(xmul(s2, s2), s2);
    const float s12 = xmul(s6, s6);
    const float f_lj = xmul(xdiv(xmul(24.0f, eps_ij), r_sq), xsub(xmul(2.0f, s12), s6));
    float f_coul = 0.0f;
    if (b.q != 0.0f && apq.w != 0.0f) f_coul = xdiv(xmul(xmul(COULOMB_K, b.q), apq.w), xmul(r_sq, xsqrt(r_sq)));
    const float f_hydro =
        (b.hyd == 1.0f && aprm.z == 1.0f && r_sq < HYDRO_CUTOFF_SQ) ? xdiv(-0.1f, xsqrt(r_sq)) : 0.0f;
    const float f_total = xadd(xadd(f_lj, f_coul), f_hydro);
    tx = xmul(f_total, ddx);
    ty = xmul(f_total, ddy);
    tz = xmul(f_total, ddz);
    return true;
}

// One pair term of compute_forces_with_grid (energy.rs:353-391), accumulated in the
// reference's order; false when the pair is outside 0.25 <= r^2 <= 100.
__device__ __forceinline__ bool cg_term(const CgB& b, const float4 apq, const float4 aprm, float& sx, float& sy,
                                        float& sz) {
    const float ddx = xsub(b.x, apq.x), ddy = xsub(b.y, apq.y), ddz = xsub(b.z, apq.z);
    const float r_sq = xdist2(ddx, ddy, ddz);
    if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) return false;
    const float eps_ij = xsqrt(xmul(b.eps, aprm.x));
    const float sig_ij = xmul(0.5f, xadd(b.sig, aprm.y));
    const float sigma_sq = xmul(sig_ij, sig_ij);
    const float s2 = xdiv(sigma_sq, r_sq);
    const float s6 = xmul(xmul(s2, s2), s2);
    const float s12 = xmul(s6, s6);
    const float f_lj = xmul(xdiv(xmul(24.0f, eps_ij), r_sq), xsub(xmul(2.0f, s12), s6));
    float f_coul = 0.0f;
    if (b.q != 0.0f && apq.w != 0.0f) f_coul = xdiv(xmul(xmul(COULOMB_K, b.q), apq.w), xmul(r_sq, xsqrt(r_sq)));
    const float f_hydro =
        (b.hyd == 1.0f && aprm.z == 1.0f && r_sq < HYDRO_CUTOFF_SQ) ? xdiv(-0.1f, xsqrt(r_sq)) : 0.0f;
    const float f_total = xadd(xadd(f_lj, f_coul), f_hydro);
    sx = xadd(sx, xmul(f_total, ddx));
    sy = xadd(sy, xmul(f_total, ddy));
    sz = xadd(sz, xmul(f_total, ddz));
    return true;
}

template <bool COUNT = false>
__device__ __forceinline__ void cg_force(const AgView& A, const CgB& b, float& fx, float& fy, float& fz,
                                         int* n_pairs = nullptr) {
    const GridView& g = A.ca_grid;
    const int cx = cell_coord(b.x, g.inv), cy = cell_coord(b.y, g.inv), cz = cell_coord(b.z, g.inv);
    // Squared distance from the point to each neighbour slab; a cell whose box lies
    // beyond the cutoff (+1 mA margin, far above f32 rounding of r^2) holds no
    // in-cutoff atom, so skipping it leaves the reference's callback sequence of
    // in-cutoff pairs, and hence the sums, unchanged.
    float sl[3][3];
    {
        const float p[3] = {b.x, b.y, b.z};
        const int c[3] = {cx, cy, cz};
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int o = 0; o < 3; ++o) {
                const float lo = (float)(c[d] + o - 1) * g.cell, hi = lo + g.cell;
                const float dd = fmaxf(fmaxf(lo - p[d], p[d] - hi), 0.0f);
                sl[d][o] = dd * dd;
            }
    }
    // margin covers the f32 rounding of x*inv and of the slab bounds at large |x|
    const float reach = 10.001f + 4e-7f * (fabsf(b.x) + fabsf(b.y) + fabsf(b.z));
    const float reach2 = reach * reach;
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                if (sl[0][dx + 1] + sl[1][dy + 1] + sl[2][dz + 1] > reach2) continue;
                int a0, a1;
                if (!probe_cell(g, cx, cy, cz, dx, dy, dz, a0, a1)) continue;
                for (int i = a0; i < a1; ++i) {
                    if (cg_term(b, A.ca_pq[i], A.ca_prm[i], sx, sy, sz) && COUNT) ++*n_pairs;
                }
            }
    fx = sx; fy = sy; fz = sz;
}

__device__ __forceinline__ CgB cg_body(float x, float y, float z, int aa) {
    const float4 t = s_res[aa];
    return CgB{x, y, z, t.x, t.y, t.z, t.w};
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
constexpr int CG_TERMS = 24;      // in-cutoff terms a lane holds per step
constexpr int CG_WARPS = 4;       // warps per CTA
constexpr int CG_MAX_STEPS = 32;  // steps per launch (the host splits longer runs)

template <bool COUNT>
__global__ void __launch_bounds__(CG_WARPS * 32) k_langevin(StateView st, const AgView* __restrict__ ags,
                                                             StepParams p, int n_steps, uint32_t step0,
                                                             int with_noise, const float* __restrict__ temps,
                                                             uint32_t* __restrict__ err,
                                                             long long* __restrict__ pair_count,
                                                             const int* __restrict__ order) {
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

void launch_diffuse(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                    uint32_t step0, int with_noise, int with_mc, const float* temps, uint32_t* err,
                    const int* order) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    (void)with_mc;
    const int threads = CG_WARPS * 32;
    const long long total = (long long)st.total_res * CG_GROUP;
    for (int s0 = 0; s0 < n_steps; s0 += CG_MAX_STEPS) {
        const int ns = min(CG_MAX_STEPS, n_steps - s0);
        k_langevin<false><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(
            st, ags, p, ns, step0 + (uint32_t)s0, with_noise, temps ? temps + s0 : nullptr, err, nullptr, order);
    }
}

void launch_diffuse_count(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          long long* pairs) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    const int threads = CG_WARPS * 32;
    const long long total = (long long)st.total_res * CG_GROUP;
    k_langevin<true><<<(int)((total + threads - 1) / threads), threads, 0, s>>>(
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
void launch_pack_slots(cudaStream_t s, int n_res, const float* in, float4* out) {
    if (n_res > 0) k_pack_slots<<<(n_res * SLOT_STRIDE + 255) / 256, 256, 0, s>>>(n_res, in, out);
}
void launch_unpack_slots(cudaStream_t s, int n_res, const float4* in, float* out) {
    if (n_res > 0) k_unpack_slots<<<(n_res * SLOTS + 255) / 256, 256, 0, s>>>(n_res, in, out);
}

}  // namespace binder
