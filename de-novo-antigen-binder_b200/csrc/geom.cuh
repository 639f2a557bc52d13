// geom.cuh — residue geometry and coarse-grained force device code shared by the
// search kernels (k_search.cu, k_anneal.cu).
//
//  * NERF side-chain placement (rotamer.rs:198-232, 439-462) and residue
//    construction around a Calpha (allatom.rs:502-541) in the slot layout.
//  * The coarse-grained pair force of compute_forces_with_grid (energy.rs:322-398)
//    with separately rounded operations in the reference's order.
//
// Each translation unit that includes this header owns a copy of the constant
// tables and fills it with geom_init_tables() (no relocatable device code).
// All sin/cos values of the NERF programs are of table angles (bond angles, fixed
// dihedrals, rotamer chis); they are evaluated once on the host with the C
// library's sinf/cosf and read from constant memory, so residue geometry is
// bit-identical to the CPU restatement of the reference.
#pragma once

#include <cmath>

#include "common.cuh"

namespace binder {

static __constant__ int s_topo_n[N_AA];
static __constant__ int s_sc_n[N_AA];
static __constant__ uchar4 s_sc_ref[N_AA][9];     // ref a, b, c, chi index (255 = fixed)
static __constant__ float4 s_sc_geom[N_AA][9];    // bond, sin(angle), cos(angle), unused
static __constant__ float2 s_sc_fix[N_AA][9];     // sin, cos of the fixed dihedral
static __constant__ int s_rot_n[N_AA];
static __constant__ float4 s_rot_chi[N_AA][5];    // chi1..chi4 in degrees
static __constant__ float2 s_rot_trig[N_AA][5][4];// sin, cos of each rotamer chi
static __constant__ float4 s_res[N_AA];           // residue-level charge, epsilon, sigma, hydrophobic (atom.rs:55-104)
// AMBER parameters of each amino acid's Calpha (topology atom 1, amber.rs:126-351):
// partial charge, r_min_half, epsilon, hydrophobic; its atom type; H-bond role of
// every atom type (bit 0 donor, bit 1 acceptor; amber.rs:398-431)
static __constant__ float4 s_ca_atom[N_AA];
static __constant__ int s_ca_type[N_AA];
static __constant__ int s_hb_role[16];

// Rust's f32::to_radians multiplies by the f32 constant PI/180.
static const float RADS_PER_DEG = 3.14159265358979323846f / 180.0f;

static cudaError_t geom_init_tables() {
    uchar4 ref[N_AA][9];
    float4 geom[N_AA][9];
    float2 fix[N_AA][9];
    float4 rchi[N_AA][5];
    float2 rtrig[N_AA][5][4];
    float4 res[N_AA], ca_atom[N_AA];
    int ca_type[N_AA], hb[16];
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
        const int t = BT_SLOT_TYPE[a][1];
        ca_atom[a] = make_float4(BT_SLOT_Q[a][1], BT_NB[t][0], BT_NB[t][1], (float)BT_SLOT_HYD[a][1]);
        ca_type[a] = t;
    }
    for (int t = 0; t < 16; ++t) hb[t] = BT_HB[t];
    cudaError_t e;
    if ((e = cudaMemcpyToSymbol(s_topo_n, BT_TOPO_N, sizeof(BT_TOPO_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_n, BT_SC_N, sizeof(BT_SC_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_ref, ref, sizeof(ref))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_geom, geom, sizeof(geom))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_sc_fix, fix, sizeof(fix))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_n, BT_ROT_N, sizeof(BT_ROT_N))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_chi, rchi, sizeof(rchi))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_rot_trig, rtrig, sizeof(rtrig))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_ca_atom, ca_atom, sizeof(ca_atom))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_ca_type, ca_type, sizeof(ca_type))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(s_hb_role, hb, sizeof(hb))) != cudaSuccess) return e;
    return cudaMemcpyToSymbol(s_res, res, sizeof(res));
}

// ---- exact vector helpers (allatom.rs:481-489, rotamer.rs:234-252) ----------------
struct F3 { float x, y, z; };
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return {xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)}; }
__device__ __forceinline__ F3 add3(F3 a, F3 b) { return {xadd(a.x, b.x), xadd(a.y, b.y), xadd(a.z, b.z)}; }
__device__ __forceinline__ F3 cross3(F3 a, F3 b) {
    return {xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
            xsub(xmul(a.x, b.y), xmul(a.y, b.x))};
}
__device__ __forceinline__ F3 norm3(F3 v) {
    const float len = fmaxf(xsqrt(xdist2(v.x, v.y, v.z)), 1e-8f);
    return {xdiv(v.x, len), xdiv(v.y, len), xdiv(v.z, len)};
}
__device__ __forceinline__ F3 f3(float4 v) { return {v.x, v.y, v.z}; }

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
// chi = 0 (residues without rotamers): sin 0 = 0, cos 0 = 1 exactly
__device__ __forceinline__ ChiTrig zero_trig() {
    ChiTrig c;
#pragma unroll
    for (int i = 0; i < 4; ++i) c.t[i] = make_float2(0.f, 1.f);
    return c;
}
// packed per-residue form: two float4 {sin chi1, cos chi1, sin chi2, cos chi2}, {..chi3, ..chi4}
__device__ __forceinline__ ChiTrig unpack_trig(float4 a, float4 b) {
    ChiTrig c;
    c.t[0] = make_float2(a.x, a.y); c.t[1] = make_float2(a.z, a.w);
    c.t[2] = make_float2(b.x, b.y); c.t[3] = make_float2(b.z, b.w);
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
    float tx, ty, tz;
    if (!cg_term_parts(b, apq, aprm, tx, ty, tz)) return false;
    sx = xadd(sx, tx);
    sy = xadd(sy, ty);
    sz = xadd(sz, tz);
    return true;
}

// compute_forces_with_grid for one body: the 27 cells in the reference's order,
// one sequential f32 sum.
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

}  // namespace binder
