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

template <bool COUNT = false>
__device__ __forceinline__ void cg_force(const AgView& A, const CgB& b, float& fx, float& fy, float& fz,
                                         int* n_pairs = nullptr) {
    const GridView& g = A.ca_grid;
    const int cx = cell_coord(b.x, g.inv), cy = cell_coord(b.y, g.inv), cz = cell_coord(b.z, g.inv);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                int a0, a1;
                if (!probe_cell(g, cx, cy, cz, dx, dy, dz, a0, a1)) continue;
                for (int i = a0; i < a1; ++i) {
                    const float4 apq = A.ca_pq[i];
                    const float4 aprm = A.ca_prm[i];
                    const float ddx = xsub(b.x, apq.x), ddy = xsub(b.y, apq.y), ddz = xsub(b.z, apq.z);
                    const float r_sq = xdist2(ddx, ddy, ddz);
                    if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) continue;
                    if (COUNT) ++*n_pairs;
                    const float eps_ij = xsqrt(xmul(b.eps, aprm.x));
                    const float sig_ij = xmul(0.5f, xadd(b.sig, aprm.y));
                    const float sigma_sq = xmul(sig_ij, sig_ij);
                    const float s2 = xdiv(sigma_sq, r_sq);
                    const float s6 = xmul(xmul(s2, s2), s2);
                    const float s12 = xmul(s6, s6);
                    const float f_lj = xmul(xdiv(xmul(24.0f, eps_ij), r_sq), xsub(xmul(2.0f, s12), s6));
                    float f_coul = 0.0f;
                    if (b.q != 0.0f && apq.w != 0.0f)
                        f_coul = xdiv(xmul(xmul(COULOMB_K, b.q), apq.w), xmul(r_sq, xsqrt(r_sq)));
                    const float f_hydro =
                        (b.hyd == 1.0f && aprm.z == 1.0f && r_sq < HYDRO_CUTOFF_SQ) ? xdiv(-0.1f, xsqrt(r_sq)) : 0.0f;
                    const float f_total = xadd(xadd(f_lj, f_coul), f_hydro);
                    sx = xadd(sx, xmul(f_total, ddx));
                    sy = xadd(sy, xmul(f_total, ddy));
                    sz = xadd(sz, xmul(f_total, ddz));
                }
            }
    fx = sx; fy = sy; fz = sz;
}

__device__ __forceinline__ CgB cg_body(float x, float y, float z, int aa) {
    const float4 t = s_res[aa];
    return CgB{x, y, z, t.x, t.y, t.z, t.w};
}

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
// One thread per residue; the residue's atoms stay in registers for n_steps.
// COUNT: count the in-cutoff CG pairs of the same trajectory, leave the state as is.
template <bool COUNT>
__global__ void __launch_bounds__(128) k_langevin(StateView st, const AgView* __restrict__ ags, StepParams p,
                                                   int n_steps, uint32_t step0, int with_noise,
                                                   const float* __restrict__ temps, uint32_t* __restrict__ err,
                                                   long long* __restrict__ pair_count) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= st.total_res) return;
    const int c = st.res_cand[r];
    const int r_local = r - st.cand_res_off[c];
    const uint32_t cid = st.cand_id[c];
    const AgView A = ags[st.cand_ag[c]];
    const int aa = st.res_aa[r];
    const int n_at = s_topo_n[aa];
    float4* slot = st.res_pos + (size_t)r * SLOT_STRIDE;
    F3 at[SLOTS];
#pragma unroll
    for (int k = 0; k < SLOTS; ++k) {
        const float4 v = k < n_at ? slot[k] : make_float4(0.f, 0.f, 0.f, 0.f);
        at[k] = {v.x, v.y, v.z};
    }
    if (err && (!isfinite(at[1].x) || !isfinite(at[1].y) || !isfinite(at[1].z))) atomicOr(err, ERRF_NAN);
    const float4 res = s_res[aa];
    int n_pairs = 0;
    for (int s = 0; s < n_steps; ++s) {
        const F3 ca = at[1];  // Calpha is topology atom 1 of every residue (amber.rs:358-377)
        float fx, fy, fz;
        cg_force<COUNT>(A, CgB{ca.x, ca.y, ca.z, res.x, res.y, res.z, res.w}, fx, fy, fz, &n_pairs);
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
        // set_ca_pos: delta = new - old, every atom of the residue += delta
        const F3 delta = sub3(new_ca, ca);
#pragma unroll
        for (int k = 0; k < SLOTS; ++k) {
            if (k < n_at) at[k] = {xadd(at[k].x, delta.x), xadd(at[k].y, delta.y), xadd(at[k].z, delta.z)};
        }
    }
    if (COUNT) {
        atomicAdd((unsigned long long*)pair_count, (unsigned long long)n_pairs);
        return;
    }
#pragma unroll
    for (int k = 0; k < SLOTS; ++k)
        if (k < n_at) slot[k] = make_float4(at[k].x, at[k].y, at[k].z, 0.f);
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

void launch_diffuse(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                    uint32_t step0, int with_noise, int with_mc, const float* temps, uint32_t* err) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    (void)with_mc;
    k_langevin<false>
        <<<(st.total_res + 127) / 128, 128, 0, s>>>(st, ags, p, n_steps, step0, with_noise, temps, err, nullptr);
}

void launch_diffuse_count(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          long long* pairs) {
    if (st.total_res <= 0 || n_steps <= 0) return;
    k_langevin<true><<<(st.total_res + 127) / 128, 128, 0, s>>>(st, ags, p, n_steps, 0, 0, nullptr, nullptr, pairs);
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
