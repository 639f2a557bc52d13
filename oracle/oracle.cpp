// oracle.cpp — CPU restatement of the reference's all-atom scoring + search path.
//
// TEST INFRASTRUCTURE ONLY (the checker for the CUDA library; see oracle.h).
// Every function cites the reference file:line it restates.  f32 functions keep
// the reference's operation order; this file must be compiled with
// -ffp-contract=off so that no a*b+c is fused (Rust never contracts).
#include "oracle.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstring>
#include <map>
#include <numeric>
#include <thread>
#include <tuple>
#include <vector>

namespace {

#include "oracle_tables.inc"

// energy.rs:13-27
const float COULOMB_K = 332.0f;
const float CUTOFF_SQ = 100.0f;
const float MIN_R_SQ = 0.25f;
const float HYDRO_CUTOFF_SQ = 36.0f;
const float HYDRO_BONUS = -0.5f;
const float HB_R0 = 2.9f;
const float HB_SIGMA = 0.35f;
const float HB_DEPTH = 1.5f;
const float HB_CUTOFF_SQ = 25.0f;
// solvation.rs:23-27
const float PI32 = 5.568328f;
const float SOLV_CUTOFF_SQ = 9.0f * 9.0f;
// allatom.rs:494-497
const float N_CA_BOND = 1.46f;
const float CA_C_BOND = 1.52f;
const float C_O_BOND = 1.23f;
const float CA_CB_BOND = 1.52f;
// Rust f32::to_radians multiplies by the f32 constant PI/180.
const float RADS_PER_DEG = 3.14159265358979323846f / 180.0f;
const int GLY = 7;
const int CYS = 4;
const int SLOTS = ORC_MAX_SLOTS;

typedef std::array<float, 3> V3;

inline V3 sub3(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 add3(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 cross3(const V3& a, const V3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
// rotamer.rs:249-252 / allatom.rs:486-489
inline V3 norm3(const V3& v) {
    float len = std::fmax(std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]), 1e-8f);
    return {v[0] / len, v[1] / len, v[2] / len};
}

// rotamer.rs:198-232 (NERF)
V3 place_atom(const V3& a, const V3& b, const V3& c, float bond_len, float angle_deg, float dihedral_deg) {
    float angle = angle_deg * RADS_PER_DEG;
    float dihedral = dihedral_deg * RADS_PER_DEG;
    V3 bc = norm3(sub3(b, c));
    V3 ba = sub3(b, a);
    V3 n = norm3(cross3(ba, bc));
    V3 m = cross3(bc, n);
    float sa = std::sin(angle);
    float ca = std::cos(angle);
    float sd = std::sin(dihedral);
    float cd = std::cos(dihedral);
    V3 d;
    for (int k = 0; k < 3; ++k) d[k] = c[k] + bond_len * (-ca * bc[k] + sa * cd * m[k] + sa * sd * n[k]);
    return d;
}

// allatom.rs:502-517
int ideal_backbone(const V3& ca, int aa, V3 out[5]) {
    V3 n = {ca[0] - N_CA_BOND, ca[1], ca[2]};
    V3 c = {ca[0] + CA_C_BOND, ca[1], ca[2]};
    V3 o = {c[0] + 0.5f, c[1] + C_O_BOND * 0.9f, c[2]};
    V3 cb = {ca[0], ca[1] - CA_CB_BOND, ca[2]};
    out[0] = n; out[1] = ca; out[2] = c; out[3] = o; out[4] = cb;
    return aa == GLY ? 4 : 5;
}

// rotamer.rs:439-462: side-chain atoms appended after `backbone`
int build_side_chain(int aa, const V3* backbone, int n_backbone, const float chi[4], V3* out) {
    V3 atoms[SLOTS];
    for (int k = 0; k < n_backbone; ++k) atoms[k] = backbone[k];
    int n = n_backbone;
    for (int k = 0; k < T_SC_N[aa]; ++k) {
        const TScDef& bd = T_SC[aa][k];
        float dih = bd.chi == 255 ? bd.dih : chi[bd.chi];
        V3 pos = place_atom(atoms[bd.a], atoms[bd.b], atoms[bd.c], bd.bond, bd.angle, dih);
        atoms[n++] = pos;
        out[k] = pos;
    }
    return T_SC_N[aa];
}

// Slot-layout protein (one candidate).  Slot k of residue r holds topology atom k,
// which is exactly the order push_residue appends them (allatom.rs:201-240).
struct Prot {
    int n;
    uint8_t* aa;
    float* chi;  // n*4
    float* pos;  // n*14*3
    V3 at(int r, int k) const { const float* p = pos + ((size_t)r * SLOTS + k) * 3; return {p[0], p[1], p[2]}; }
    void set(int r, int k, const V3& v) { float* p = pos + ((size_t)r * SLOTS + k) * 3; p[0] = v[0]; p[1] = v[1]; p[2] = v[2]; }
    int natoms(int r) const { return T_TOPO_N[aa[r]]; }
};

// push_residue (allatom.rs:201-240) into slot layout
void place_residue(Prot& P, int r, int aa, const V3* backbone, int n_bb, const float chi[4]) {
    int n_topo = T_TOPO_N[aa];
    int nb = std::min(n_bb, n_topo);
    for (int k = 0; k < nb; ++k) P.set(r, k, backbone[k]);
    V3 sc[SLOTS];
    int n_sc = build_side_chain(aa, backbone, n_bb, chi, sc);
    int n_sc_topo = n_topo - nb;
    for (int k = 0; k < n_sc && k < n_sc_topo; ++k) P.set(r, nb + k, sc[k]);
    for (int k = n_topo; k < SLOTS; ++k) P.set(r, k, V3{0.f, 0.f, 0.f});
    P.aa[r] = (uint8_t)aa;
    for (int c = 0; c < 4; ++c) P.chi[r * 4 + c] = chi[c];
}

// rebuild_side_chain (allatom.rs:244-270)
void rebuild_side_chain(Prot& P, int r) {
    int aa = P.aa[r];
    int n_bb = 4 + (aa != GLY ? 1 : 0);
    V3 bb[5];
    for (int k = 0; k < n_bb; ++k) bb[k] = P.at(r, k);
    V3 sc[SLOTS];
    int n_sc = build_side_chain(aa, bb, n_bb, &P.chi[r * 4], sc);
    int n_sc_topo = std::max(T_TOPO_N[aa] - n_bb, 0);
    for (int k = 0; k < n_sc && k < n_sc_topo; ++k) P.set(r, n_bb + k, sc[k]);
}

// mutate_residue (allatom.rs:299-384)
void mutate_residue(Prot& P, int r, int new_aa, const float chi[4]) {
    int old_aa = P.aa[r];
    if (old_aa == new_aa) {
        for (int c = 0; c < 4; ++c) P.chi[r * 4 + c] = chi[c];
        rebuild_side_chain(P, r);
        return;
    }
    V3 ca = P.at(r, T_TOPO_CA[old_aa]);
    V3 bb[5];
    int n_bb = ideal_backbone(ca, new_aa, bb);
    V3 sc[SLOTS];
    int n_sc = build_side_chain(new_aa, bb, n_bb, chi, sc);
    int n_new = T_TOPO_N[new_aa];
    for (int k = 0; k < n_new; ++k) {
        V3 pos = k < n_bb ? bb[k] : ((k - n_bb) < n_sc ? sc[k - n_bb] : ca);
        P.set(r, k, pos);
    }
    for (int k = n_new; k < SLOTS; ++k) P.set(r, k, V3{0.f, 0.f, 0.f});
    P.aa[r] = (uint8_t)new_aa;
    for (int c = 0; c < 4; ++c) P.chi[r * 4 + c] = chi[c];
}

// set_ca_pos / translate_residue (allatom.rs:279-293)
void set_ca_pos(Prot& P, int r, const V3& new_pos) {
    V3 old = P.at(r, T_TOPO_CA[P.aa[r]]);
    V3 delta = {new_pos[0] - old[0], new_pos[1] - old[1], new_pos[2] - old[2]};
    for (int k = 0; k < P.natoms(r); ++k) {
        float* p = P.pos + ((size_t)r * SLOTS + k) * 3;
        p[0] += delta[0]; p[1] += delta[1]; p[2] += delta[2];
    }
}

// Transcendentals of the Metropolis path (acceptance exp, H-bond and disulfide
// Gaussians, rotation by a random torsion): evaluated in double and rounded once
// to f32, as the CUDA kernels do.  Both double functions are within 1 ulp of the
// exact value, so the two f32 results agree unless the exact value lies within
// about 2^-29 (relative) of an f32 rounding boundary.  Rust's f32 exp/sin/cos
// (libm) are within 1 ulp of these values.
inline float mc_exp(float x) { return (float)std::exp((double)x); }
inline float mc_sin(float x) { return (float)std::sin((double)x); }
inline float mc_cos(float x) { return (float)std::cos((double)x); }

// rodrigues (allatom.rs:467-479)
V3 rodrigues(const V3& point, const V3& origin, const V3& axis, float angle) {
    V3 v = sub3(point, origin);
    float ca = mc_cos(angle);
    float sa = mc_sin(angle);
    float dot = v[0] * axis[0] + v[1] * axis[1] + v[2] * axis[2];
    V3 cx = cross3(axis, v);
    V3 rotd = {v[0] * ca + cx[0] * sa + axis[0] * dot * (1.0f - ca),
               v[1] * ca + cx[1] * sa + axis[1] * dot * (1.0f - ca),
               v[2] * ca + cx[2] * sa + axis[2] * dot * (1.0f - ca)};
    return add3(rotd, origin);
}

// perturb_phi (allatom.rs:397-424)
void perturb_phi(Prot& P, int r, float delta) {
    if (P.natoms(r) < 3) return;
    V3 n = P.at(r, 0), ca = P.at(r, 1);
    V3 axis = norm3(sub3(ca, n));
    for (int k = 2; k < P.natoms(r); ++k) P.set(r, k, rodrigues(P.at(r, k), ca, axis, delta));
    for (int q = r + 1; q < P.n; ++q)
        for (int k = 0; k < P.natoms(q); ++k) P.set(q, k, rodrigues(P.at(q, k), ca, axis, delta));
}

// perturb_psi (allatom.rs:429-455)
void perturb_psi(Prot& P, int r, float delta) {
    if (P.natoms(r) < 4) return;
    V3 ca = P.at(r, 1), c = P.at(r, 2);
    V3 axis = norm3(sub3(c, ca));
    P.set(r, 3, rodrigues(P.at(r, 3), c, axis, delta));
    for (int q = r + 1; q < P.n; ++q)
        for (int k = 0; k < P.natoms(q); ++k) P.set(q, k, rodrigues(P.at(q, k), c, axis, delta));
}

// disulfide_energy (allatom.rs:155-180); SG is topology atom 5 of CYS (sg_pos, :139-150).
// Acc = float: the reference's f32 sum; Acc = double: the same f32 pair terms
// summed in double.
template <class Acc>
Acc disulfide_t(const Prot& P) {
    const float D0 = 2.05f, SIGMA = 0.4f, DEPTH = 4.0f, CUT = 4.0f;
    std::vector<V3> sg;
    for (int r = 0; r < P.n; ++r)
        if (P.aa[r] == CYS && P.natoms(r) > 5) sg.push_back(P.at(r, 5));
    Acc e = 0;
    for (size_t i = 0; i < sg.size(); ++i)
        for (size_t j = i + 1; j < sg.size(); ++j) {
            float dx = sg[i][0] - sg[j][0], dy = sg[i][1] - sg[j][1], dz = sg[i][2] - sg[j][2];
            float d = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (d > CUT) continue;
            float z = (d - D0) / SIGMA;
            e -= (Acc)(DEPTH * mc_exp(-0.5f * z * z));
        }
    return e;
}
float disulfide(const Prot& P) { return disulfide_t<float>(P); }

// hbond_energy (energy.rs:32-39)
inline float hbond_energy(float r_sq) {
    if (r_sq > HB_CUTOFF_SQ) return 0.0f;
    float r = std::sqrt(r_sq);
    float z = (r - HB_R0) / HB_SIGMA;
    return -HB_DEPTH * std::exp(-0.5f * z * z);
}
inline float hbond_energy_mc(float r_sq) {
    if (r_sq > HB_CUTOFF_SQ) return 0.0f;
    float r = std::sqrt(r_sq);
    float z = (r - HB_R0) / HB_SIGMA;
    return -HB_DEPTH * mc_exp(-0.5f * z * z);
}
inline double hbond_energy64(double r_sq) {
    if (r_sq > (double)HB_CUTOFF_SQ) return 0.0;
    double r = std::sqrt(r_sq);
    double z = (r - (double)HB_R0) / (double)HB_SIGMA;
    return -(double)HB_DEPTH * std::exp(-0.5 * z * z);
}
inline bool hb_pair(int bt, int at) {
    return (T_HB_DONOR[bt] && T_HB_ACC[at]) || (T_HB_ACC[bt] && T_HB_DONOR[at]);
}

// Rust `f32 as i32` saturates and maps NaN to 0.
inline int32_t sat_i32(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return INT32_MAX;
    if (v < -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}

// SpatialHashGrid (spatial.rs:12-67).  A std::map replaces the HashMap: the probe
// visits cells in a fixed (dx,dy,dz) order and atoms in insertion order, so the
// container type does not change the callback sequence.
struct Grid {
    float inv;
    std::map<std::tuple<int32_t, int32_t, int32_t>, std::vector<uint32_t>> cells;
    explicit Grid(float cell) : inv(1.0f / cell) {}
    std::tuple<int32_t, int32_t, int32_t> cell_of(float x, float y, float z) const {
        return std::make_tuple(sat_i32(std::floor(x * inv)), sat_i32(std::floor(y * inv)), sat_i32(std::floor(z * inv)));
    }
    void build(const float* x, const float* y, const float* z, int64_t n) {
        cells.clear();
        for (int64_t i = 0; i < n; ++i) cells[cell_of(x[i], y[i], z[i])].push_back((uint32_t)i);
    }
    template <class F> void query(float px, float py, float pz, F&& cb) const {
        int32_t cx, cy, cz;
        std::tie(cx, cy, cz) = cell_of(px, py, pz);
        for (int dx = -1; dx <= 1; ++dx)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dz = -1; dz <= 1; ++dz) {
                    // i32 addition wraps in the reference's release build
                    auto key = std::make_tuple((int32_t)((uint32_t)cx + (uint32_t)dx),
                                               (int32_t)((uint32_t)cy + (uint32_t)dy),
                                               (int32_t)((uint32_t)cz + (uint32_t)dz));
                    auto it = cells.find(key);
                    if (it == cells.end()) continue;
                    for (uint32_t idx : it->second) cb(idx);
                }
    }
};

// One CG pair force term of compute_forces_with_grid (energy.rs:353-391).
struct CgAtom { float x, y, z, q, eps, sig; uint8_t hyd; };
inline CgAtom cg_atom(float x, float y, float z, int aa) {
    return {x, y, z, T_RES_Q[aa], T_RES_EPS[aa], T_RES_SIG[aa], T_RES_HYD[aa]};
}
inline bool cg_pair(const CgAtom& b, const CgAtom& a, float& fx, float& fy, float& fz) {
    float dx = b.x - a.x, dy = b.y - a.y, dz = b.z - a.z;
    float r_sq = dx * dx + dy * dy + dz * dz;
    if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) return false;
    float eps_ij = std::sqrt(b.eps * a.eps);
    float sig_ij = 0.5f * (b.sig + a.sig);
    float sigma_sq_ij = sig_ij * sig_ij;
    float s2 = sigma_sq_ij / r_sq;
    float s6 = s2 * s2 * s2;
    float s12 = s6 * s6;
    float f_lj = (24.0f * eps_ij / r_sq) * (2.0f * s12 - s6);
    float f_coul = 0.0f;
    if (b.q != 0.0f && a.q != 0.0f) {
        float r = std::sqrt(r_sq);
        f_coul = COULOMB_K * b.q * a.q / (r_sq * r);
    }
    float f_hydro = (b.hyd == 1 && a.hyd == 1 && r_sq < HYDRO_CUTOFF_SQ) ? -0.1f / std::sqrt(r_sq) : 0.0f;
    float f_total = f_lj + f_coul + f_hydro;
    fx += f_total * dx;
    fy += f_total * dy;
    fz += f_total * dz;
    return true;
}
inline void cg_pair64(const CgAtom& b, const CgAtom& a, double& fx, double& fy, double& fz) {
    double dx = (double)b.x - a.x, dy = (double)b.y - a.y, dz = (double)b.z - a.z;
    double r_sq = dx * dx + dy * dy + dz * dz;
    // the cutoff decision is taken in f32 exactly as the reference does, so both
    // variants sum over the same pair set
    float dxf = b.x - a.x, dyf = b.y - a.y, dzf = b.z - a.z;
    float r_sq_f = dxf * dxf + dyf * dyf + dzf * dzf;
    if (r_sq_f > CUTOFF_SQ || r_sq_f < MIN_R_SQ) return;
    double eps_ij = std::sqrt((double)b.eps * a.eps);
    double sig_ij = 0.5 * ((double)b.sig + a.sig);
    double s2 = sig_ij * sig_ij / r_sq;
    double s6 = s2 * s2 * s2;
    double f_lj = (24.0 * eps_ij / r_sq) * (2.0 * s6 * s6 - s6);
    double f_coul = (b.q != 0.0f && a.q != 0.0f) ? (double)COULOMB_K * b.q * a.q / (r_sq * std::sqrt(r_sq)) : 0.0;
    double f_hydro = (b.hyd == 1 && a.hyd == 1 && r_sq_f < HYDRO_CUTOFF_SQ) ? -0.1 / std::sqrt(r_sq) : 0.0;
    double f = f_lj + f_coul + f_hydro;
    fx += f * dx; fy += f * dy; fz += f * dz;
}

template <class F> void parallel_for(int64_t n, int n_threads, F&& fn) {
    if (n_threads <= 1 || n < 2) {
        for (int64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    int nt = (int)std::min<int64_t>(n_threads, n);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t]() {
            for (int64_t i = t; i < n; i += nt) fn(i);
        });
    for (auto& x : th) x.join();
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy
// as 1, 2, 3", SC'11).  Multipliers and Weyl key increments from that paper.
inline void philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Draw conventions shared with the CUDA library (its binder_rng.h states them):
// uniform float in [0,1) from the top 24 bits; integer range by multiply-shift;
// float range lo + u*(hi-lo) with separate rounding of each operation.
inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }
inline uint32_t urange(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }
inline float frange(uint32_t x, float lo, float hi) {
    float t = hi - lo;
    float s = u01(x) * t;
    return lo + s;
}
enum { STREAM_NOISE = 0, STREAM_MC = 1, STREAM_BACKBONE = 2 };
inline void draw(uint64_t seed, uint32_t cand, uint32_t step, uint32_t stream, uint32_t r, uint32_t out[4]) {
    uint32_t ctr[4] = {cand, step, (stream << 16) | (r & 0xFFFFu), 0u};
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    philox(ctr, key, out);
}

}  // namespace

// ---------------------------------------------------------------------------
// antigen
struct orc_antigen {
    int n_res;
    std::vector<uint8_t> aa;
    std::vector<float> pos;  // slots
    // Calpha cloud (run_allatom ag_ca, diffusion.rs:994-1002)
    std::vector<float> cx, cy, cz;
    std::vector<CgAtom> cg;
    Grid grid{10.0f};
    float center[3];
    // all-atom cloud (flattened)
    std::vector<float> x, y, z, q, rmh, eps;
    std::vector<uint8_t> hyd, type;
};

extern "C" {

int orc_topology_size(int aa) { return (aa >= 0 && aa < 20) ? T_TOPO_N[aa] : 0; }
int orc_topology_atom(int aa, int k, float* charge, int* type, int* hydrophobic) {
    if (aa < 0 || aa >= 20 || k < 0 || k >= T_TOPO_N[aa]) return -1;
    *charge = T_TOPO_Q[aa][k];
    *type = T_TOPO_TYPE[aa][k];
    *hydrophobic = T_TOPO_HYD[aa][k];
    return 0;
}
void orc_amber_nb(int type, float* rmh, float* eps) { *rmh = T_NB[type][0]; *eps = T_NB[type][1]; }
int orc_hbond_flags(int type) { return (T_HB_DONOR[type] ? 1 : 0) | (T_HB_ACC[type] ? 2 : 0); }
void orc_eef1(int type, float* dg, float* vol, float* lam) { *dg = T_EEF1[type][0]; *vol = T_EEF1[type][1]; *lam = T_EEF1[type][2]; }
int orc_rotamer_count(int aa) { return T_ROT_N[aa]; }
void orc_rotamer(int aa, int idx, float chi[4], float* prob) {
    for (int c = 0; c < 4; ++c) chi[c] = T_ROT[aa][idx][c];
    *prob = T_ROT[aa][idx][4];
}
int orc_sidechain_def_count(int aa) { return T_SC_N[aa]; }
void orc_sidechain_def(int aa, int k, int ref[3], float* bond, float* angle, float* dih, int* chi_idx) {
    const TScDef& d = T_SC[aa][k];
    ref[0] = d.a; ref[1] = d.b; ref[2] = d.c;
    *bond = d.bond; *angle = d.angle; *dih = d.dih; *chi_idx = d.chi;
}
void orc_residue_level(int aa, float* q, float* eps, float* sig, int* hyd) {
    *q = T_RES_Q[aa]; *eps = T_RES_EPS[aa]; *sig = T_RES_SIG[aa]; *hyd = T_RES_HYD[aa];
}

void orc_place_atom(const float a[3], const float b[3], const float c[3], float bond, float ang, float dih, float out[3]) {
    V3 d = place_atom(V3{a[0], a[1], a[2]}, V3{b[0], b[1], b[2]}, V3{c[0], c[1], c[2]}, bond, ang, dih);
    out[0] = d[0]; out[1] = d[1]; out[2] = d[2];
}

// protein_from_ca_trace (allatom.rs:523-541)
void orc_build_residues(int n, const float* ca_xyz, const uint8_t* aa, const float* chi_or_null, float* out_pos, float* out_chi) {
    std::vector<uint8_t> aa_buf(aa, aa + n);
    std::vector<float> chi_buf((size_t)n * 4);
    Prot P{n, aa_buf.data(), chi_buf.data(), out_pos};
    for (int r = 0; r < n; ++r) {
        V3 ca = {ca_xyz[r * 3], ca_xyz[r * 3 + 1], ca_xyz[r * 3 + 2]};
        V3 bb[5];
        int n_bb = ideal_backbone(ca, aa[r], bb);
        float chi[4] = {0.f, 0.f, 0.f, 0.f};
        if (chi_or_null) {
            for (int c = 0; c < 4; ++c) chi[c] = chi_or_null[r * 4 + c];
        } else if (T_ROT_N[aa[r]] > 0) {
            for (int c = 0; c < 4; ++c) chi[c] = T_ROT[aa[r]][0][c];
        }
        place_residue(P, r, aa[r], bb, n_bb, chi);
    }
    if (out_chi) std::memcpy(out_chi, chi_buf.data(), chi_buf.size() * sizeof(float));
}

int orc_flatten(int n, const uint8_t* aa, const float* pos, float* x, float* y, float* z, float* q, float* rmh,
                float* eps, uint8_t* hyd, uint8_t* type, uint32_t* resi) {
    int m = 0;
    for (int r = 0; r < n; ++r)
        for (int k = 0; k < T_TOPO_N[aa[r]]; ++k) {
            const float* p = pos + ((size_t)r * SLOTS + k) * 3;
            int t = T_TOPO_TYPE[aa[r]][k];
            if (x) { x[m] = p[0]; y[m] = p[1]; z[m] = p[2]; }
            if (q) q[m] = T_TOPO_Q[aa[r]][k];
            if (rmh) rmh[m] = T_NB[t][0];
            if (eps) eps[m] = T_NB[t][1];
            if (hyd) hyd[m] = T_TOPO_HYD[aa[r]][k];
            if (type) type[m] = (uint8_t)t;
            if (resi) resi[m] = (uint32_t)r;
            ++m;
        }
    return m;
}

// ca_center_of_mass (allatom.rs:183-195): CA is slot 1 for every residue
void orc_ca_center(int n, const float* pos, float out[3]) {
    if (n == 0) { out[0] = out[1] = out[2] = 0.f; return; }
    float cx = 0.f, cy = 0.f, cz = 0.f;
    for (int r = 0; r < n; ++r) {
        const float* p = pos + ((size_t)r * SLOTS + 1) * 3;
        cx += p[0]; cy += p[1]; cz += p[2];
    }
    float nf = (float)n;
    out[0] = cx / nf; out[1] = cy / nf; out[2] = cz / nf;
}

void orc_grid_cell(float cell, float x, float y, float z, int32_t out[3]) {
    Grid g(cell);
    auto c = g.cell_of(x, y, z);
    out[0] = std::get<0>(c); out[1] = std::get<1>(c); out[2] = std::get<2>(c);
}

int64_t orc_grid_neighbors(float cell, const float* ax, const float* ay, const float* az, int64_t n_ag,
                           const float* px, const float* py, const float* pz, int64_t n_q,
                           int64_t* out_offsets, uint32_t* out_idx, int64_t cap) {
    Grid g(cell);
    g.build(ax, ay, az, n_ag);
    int64_t m = 0;
    bool overflow = false;
    for (int64_t q = 0; q < n_q; ++q) {
        out_offsets[q] = m;
        g.query(px[q], py[q], pz[q], [&](uint32_t i) {
            if (m < cap) out_idx[m] = i; else overflow = true;
            ++m;
        });
    }
    out_offsets[n_q] = m;
    return overflow ? -1 : m;
}

// compute_forces (energy.rs:154-234)
void orc_forces_cg_brute(const float* ax, const float* ay, const float* az, const uint8_t* aaa, int n_ag,
                         const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                         float* fx, float* fy, float* fz) {
    for (int j = 0; j < n_ab; ++j) {
        CgAtom b = cg_atom(bx[j], by[j], bz[j], baa[j]);
        float ax_ = 0.f, ay_ = 0.f, az_ = 0.f;
        for (int i = 0; i < n_ag; ++i) cg_pair(b, cg_atom(ax[i], ay[i], az[i], aaa[i]), ax_, ay_, az_);
        fx[j] = ax_; fy[j] = ay_; fz[j] = az_;
    }
}

// compute_forces_with_grid (energy.rs:322-398)
void orc_forces_cg_grid(float cell, const float* ax, const float* ay, const float* az, const uint8_t* aaa, int n_ag,
                        const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                        float* fx, float* fy, float* fz) {
    Grid g(cell);
    g.build(ax, ay, az, n_ag);
    for (int j = 0; j < n_ab; ++j) {
        CgAtom b = cg_atom(bx[j], by[j], bz[j], baa[j]);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        g.query(b.x, b.y, b.z, [&](uint32_t i) { cg_pair(b, cg_atom(ax[i], ay[i], az[i], aaa[i]), sx, sy, sz); });
        fx[j] = sx; fy[j] = sy; fz[j] = sz;
    }
}

void orc_forces_cg64(float cell, int use_grid, const float* ax, const float* ay, const float* az, const uint8_t* aaa,
                     int n_ag, const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                     double* fx, double* fy, double* fz) {
    Grid g(cell);
    if (use_grid) g.build(ax, ay, az, n_ag);
    for (int j = 0; j < n_ab; ++j) {
        CgAtom b = cg_atom(bx[j], by[j], bz[j], baa[j]);
        double sx = 0, sy = 0, sz = 0;
        if (use_grid)
            g.query(b.x, b.y, b.z, [&](uint32_t i) { cg_pair64(b, cg_atom(ax[i], ay[i], az[i], aaa[i]), sx, sy, sz); });
        else
            for (int i = 0; i < n_ag; ++i) cg_pair64(b, cg_atom(ax[i], ay[i], az[i], aaa[i]), sx, sy, sz);
        fx[j] = sx; fy[j] = sy; fz[j] = sz;
    }
}

// interaction_energy_atoms_breakdown (energy.rs:261-314) + solvation_interaction
// (solvation.rs:52-84).  The reference sums the solvation term over a Rayon tree;
// here it is summed sequentially over antibody atoms.
void orc_energy_atoms32(const orc_cloud* ag, const orc_cloud* ab, float out[5]) {
    float lj = 0.f, coul = 0.f, hydro = 0.f, hb = 0.f, solv = 0.f;
    for (int64_t j = 0; j < ab->n; ++j) {
        float bx = ab->x[j], by = ab->y[j], bz = ab->z[j], bq = ab->q[j], brm = ab->rmh[j], be = ab->eps[j];
        uint8_t bh = ab->hyd[j];
        for (int64_t i = 0; i < ag->n; ++i) {
            float dx = bx - ag->x[i], dy = by - ag->y[i], dz = bz - ag->z[i];
            float r_sq = dx * dx + dy * dy + dz * dz;
            if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) continue;
            float r_ij = brm + ag->rmh[i];
            float eps = std::sqrt(be * ag->eps[i]);
            float r2 = (r_ij * r_ij) / r_sq;
            float r6 = r2 * r2 * r2;
            float r12 = r6 * r6;
            lj += eps * (r12 - 2.0f * r6);
            float q1 = bq, q2 = ag->q[i];
            if (q1 != 0.0f && q2 != 0.0f) coul += COULOMB_K * q1 * q2 / std::sqrt(r_sq);
            if (bh == 1 && ag->hyd[i] == 1 && r_sq < HYDRO_CUTOFF_SQ) hydro += HYDRO_BONUS;
            if (hb_pair(ab->type[j], ag->type[i])) hb += hbond_energy(r_sq);
        }
    }
    for (int64_t j = 0; j < ab->n; ++j) {
        const float* ej = T_EEF1[ab->type[j]];
        if (ej[1] == 0.0f && ej[0] == 0.0f) continue;
        float local = 0.f;
        for (int64_t i = 0; i < ag->n; ++i) {
            float dx = ab->x[j] - ag->x[i], dy = ab->y[j] - ag->y[i], dz = ab->z[j] - ag->z[i];
            float r_sq = dx * dx + dy * dy + dz * dz;
            if (r_sq >= SOLV_CUTOFF_SQ || r_sq < 0.25f) continue;
            const float* ei = T_EEF1[ag->type[i]];
            float r = std::sqrt(r_sq);
            float ri = r / ei[2], rj = r / ej[2];
            float fi = std::exp(-(ri * ri)) / (PI32 * (ei[2] * ei[2] * ei[2]));
            float fj = std::exp(-(rj * rj)) / (PI32 * (ej[2] * ej[2] * ej[2]));
            local += -(ei[0] * ej[1] * fi + ej[0] * ei[1] * fj);
        }
        solv += local;
    }
    out[0] = lj; out[1] = coul; out[2] = hydro; out[3] = hb; out[4] = solv;
}

void orc_energy_atoms64(const orc_cloud* ag, const orc_cloud* ab, double out[5], double out_abs[5]) {
    double s[5] = {0, 0, 0, 0, 0}, a[5] = {0, 0, 0, 0, 0};
    for (int64_t j = 0; j < ab->n; ++j) {
        for (int64_t i = 0; i < ag->n; ++i) {
            float dxf = ab->x[j] - ag->x[i], dyf = ab->y[j] - ag->y[i], dzf = ab->z[j] - ag->z[i];
            float r_sq_f = dxf * dxf + dyf * dyf + dzf * dzf;
            double dx = (double)ab->x[j] - ag->x[i], dy = (double)ab->y[j] - ag->y[i], dz = (double)ab->z[j] - ag->z[i];
            double r_sq = dx * dx + dy * dy + dz * dz;
            if (r_sq_f <= CUTOFF_SQ && r_sq_f >= MIN_R_SQ) {
                double r_ij = (double)ab->rmh[j] + ag->rmh[i];
                double eps = std::sqrt((double)ab->eps[j] * ag->eps[i]);
                double r2 = r_ij * r_ij / r_sq;
                double r6 = r2 * r2 * r2;
                double lj = eps * (r6 * r6 - 2.0 * r6);
                s[0] += lj; a[0] += std::fabs(lj);
                if (ab->q[j] != 0.0f && ag->q[i] != 0.0f) {
                    double c = (double)COULOMB_K * ab->q[j] * ag->q[i] / std::sqrt(r_sq);
                    s[1] += c; a[1] += std::fabs(c);
                }
                if (ab->hyd[j] == 1 && ag->hyd[i] == 1 && r_sq_f < HYDRO_CUTOFF_SQ) { s[2] += HYDRO_BONUS; a[2] += 0.5; }
                if (hb_pair(ab->type[j], ag->type[i])) {
                    double h = hbond_energy64(r_sq);
                    s[3] += h; a[3] += std::fabs(h);
                }
            }
            const float* ej = T_EEF1[ab->type[j]];
            if (ej[1] == 0.0f && ej[0] == 0.0f) continue;
            if (r_sq_f >= SOLV_CUTOFF_SQ || r_sq_f < 0.25f) continue;
            const float* ei = T_EEF1[ag->type[i]];
            double r = std::sqrt(r_sq);
            double li = ei[2], lj_ = ej[2];
            double fi = std::exp(-(r / li) * (r / li)) / ((double)PI32 * li * li * li);
            double fj = std::exp(-(r / lj_) * (r / lj_)) / ((double)PI32 * lj_ * lj_ * lj_);
            double sv = -((double)ei[0] * ej[1] * fi + (double)ej[0] * ei[1] * fj);
            s[4] += sv; a[4] += std::fabs(sv);
        }
    }
    for (int k = 0; k < 5; ++k) { out[k] = s[k]; if (out_abs) out_abs[k] = a[k]; }
}

// score_batch (gpu.rs:166-267): per candidate LJ + Coulomb + hydrophobic with the
// shader's pair math (energy.wgsl:67-94); f32 accumulated in the CPU breakdown's
// loop order (energy.rs:269-301), three component sums added as in total().
void orc_score_batch32(const float* ag, int64_t n_ag, const float* cand, const int64_t* off, int64_t n_cand,
                       float* out, int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        float lj = 0.f, coul = 0.f, hydro = 0.f;
        for (int64_t j = off[c]; j < off[c + 1]; ++j) {
            const float* b = cand + j * 8;
            for (int64_t i = 0; i < n_ag; ++i) {
                const float* a = ag + i * 8;
                float dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
                float r_sq = dx * dx + dy * dy + dz * dz;
                if (r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ) continue;
                float r_ij = b[4] + a[4];
                float eps = std::sqrt(b[5] * a[5]);
                float r2 = (r_ij * r_ij) / r_sq;
                float r6 = r2 * r2 * r2;
                lj += eps * (r6 * r6 - 2.0f * r6);
                if (b[3] != 0.0f && a[3] != 0.0f) coul += COULOMB_K * b[3] * a[3] / std::sqrt(r_sq);
                if (b[6] > 0.5f && a[6] > 0.5f && r_sq < HYDRO_CUTOFF_SQ) hydro += HYDRO_BONUS;
            }
        }
        out[c] = lj + coul + hydro;
    });
}

void orc_score_batch64(const float* ag, int64_t n_ag, const float* cand, const int64_t* off, int64_t n_cand,
                       double* out, double* out_abs, int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        double s = 0, sa = 0;
        for (int64_t j = off[c]; j < off[c + 1]; ++j) {
            const float* b = cand + j * 8;
            for (int64_t i = 0; i < n_ag; ++i) {
                const float* a = ag + i * 8;
                float dxf = b[0] - a[0], dyf = b[1] - a[1], dzf = b[2] - a[2];
                float r_sq_f = dxf * dxf + dyf * dyf + dzf * dzf;
                if (r_sq_f > CUTOFF_SQ || r_sq_f < MIN_R_SQ) continue;
                double dx = (double)b[0] - a[0], dy = (double)b[1] - a[1], dz = (double)b[2] - a[2];
                double r_sq = dx * dx + dy * dy + dz * dz;
                double r_ij = (double)b[4] + a[4];
                double eps = std::sqrt((double)b[5] * a[5]);
                double r2 = r_ij * r_ij / r_sq;
                double r6 = r2 * r2 * r2;
                double lj = eps * (r6 * r6 - 2.0 * r6);
                s += lj; sa += std::fabs(lj);
                if (b[3] != 0.0f && a[3] != 0.0f) {
                    double cc = (double)COULOMB_K * b[3] * a[3] / std::sqrt(r_sq);
                    s += cc; sa += std::fabs(cc);
                }
                if (b[6] > 0.5f && a[6] > 0.5f && r_sq_f < HYDRO_CUTOFF_SQ) { s += HYDRO_BONUS; sa += 0.5; }
            }
        }
        out[c] = s;
        if (out_abs) out_abs[c] = sa;
    });
}

// -grad of the score's LJ + Coulomb terms with respect to each candidate atom
// (no reference counterpart: the reference moves residues by the CG force only).
void orc_forces_allatom64(const float* ag, int64_t n_ag, const float* cand, const int64_t* off, int64_t n_cand,
                          double* out_f, double* out_e, int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        double e = 0;
        for (int64_t j = off[c]; j < off[c + 1]; ++j) {
            const float* b = cand + j * 8;
            double fx = 0, fy = 0, fz = 0;
            for (int64_t i = 0; i < n_ag; ++i) {
                const float* a = ag + i * 8;
                float dxf = b[0] - a[0], dyf = b[1] - a[1], dzf = b[2] - a[2];
                float r_sq_f = dxf * dxf + dyf * dyf + dzf * dzf;
                if (r_sq_f > CUTOFF_SQ || r_sq_f < MIN_R_SQ) continue;
                double dx = (double)b[0] - a[0], dy = (double)b[1] - a[1], dz = (double)b[2] - a[2];
                double u = dx * dx + dy * dy + dz * dz;
                double R = (double)b[4] + a[4];
                double eps = std::sqrt((double)b[5] * a[5]);
                double s = R * R / u;
                double s3 = s * s * s;
                e += eps * (s3 * s3 - 2.0 * s3);
                double scale = 12.0 * eps * (s3 * s3 - s3) / u;
                if (b[3] != 0.0f && a[3] != 0.0f) {
                    double r = std::sqrt(u);
                    double kqq = (double)COULOMB_K * b[3] * a[3];
                    e += kqq / r;
                    scale += kqq / (u * r);
                }
                if (b[6] > 0.5f && a[6] > 0.5f && r_sq_f < HYDRO_CUTOFF_SQ) e += HYDRO_BONUS;
                fx += scale * dx; fy += scale * dy; fz += scale * dz;
            }
            out_f[j * 3] = fx; out_f[j * 3 + 1] = fy; out_f[j * 3 + 2] = fz;
        }
        if (out_e) out_e[c] = e;
    });
}

int64_t orc_count_pairs(const float* ag, int64_t n_ag, const float* cand, int64_t n_cand_atoms, int n_threads) {
    int nt = std::max(1, n_threads);
    std::vector<int64_t> cnt(nt, 0);
    parallel_for(nt, nt, [&](int64_t t) {
        int64_t m = 0;
        for (int64_t j = t; j < n_cand_atoms; j += nt) {
            const float* b = cand + j * 8;
            for (int64_t i = 0; i < n_ag; ++i) {
                const float* a = ag + i * 8;
                float dx = b[0] - a[0], dy = b[1] - a[1], dz = b[2] - a[2];
                float r_sq = dx * dx + dy * dy + dz * dz;
                m += (r_sq <= CUTOFF_SQ && r_sq >= MIN_R_SQ);
            }
        }
        cnt[t] = m;
    });
    return std::accumulate(cnt.begin(), cnt.end(), (int64_t)0);
}

void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) { philox(ctr, key, out); }

// diffusion.rs:65-83 constants; shell_radius replaces INIT_RADIUS as restraint radius
void orc_default_params(orc_params* p) {
    p->step = 0.08f; p->noise_base = 0.25f; p->t_hot = 3.0f; p->t_cold = 0.02f;
    p->mutation_p = 0.08f; p->rotamer_move_p = 0.12f; p->backbone_move_p = 0.04f;
    p->max_torsion_deg = 15.0f; p->iface_cutoff_sq = 64.0f; p->shell_radius = 20.0f;
    p->max_disp = 2.0f; p->restraint_k = 0.02f; p->ca_cell = 10.0f; p->accumulate = 0; p->seed = 0;
}

// temperature (diffusion.rs:102-104)
float orc_temperature(int iter, int total) {
    const float T_HOT = 3.0f, T_COLD = 0.02f;
    return T_HOT * std::pow(T_COLD / T_HOT, (float)iter / (float)total);
}

orc_antigen* orc_antigen_new(int n_res, const uint8_t* aa, const float* pos, float ca_cell) {
    orc_antigen* A = new orc_antigen();
    A->n_res = n_res;
    A->aa.assign(aa, aa + n_res);
    A->pos.assign(pos, pos + (size_t)n_res * SLOTS * 3);
    A->grid = Grid(ca_cell);
    for (int r = 0; r < n_res; ++r) {
        const float* p = pos + ((size_t)r * SLOTS + 1) * 3;
        A->cx.push_back(p[0]); A->cy.push_back(p[1]); A->cz.push_back(p[2]);
        A->cg.push_back(cg_atom(p[0], p[1], p[2], aa[r]));
    }
    A->grid.build(A->cx.data(), A->cy.data(), A->cz.data(), n_res);
    orc_ca_center(n_res, pos, A->center);
    int m = 0;
    for (int r = 0; r < n_res; ++r) m += T_TOPO_N[aa[r]];
    A->x.resize(m); A->y.resize(m); A->z.resize(m); A->q.resize(m); A->rmh.resize(m); A->eps.resize(m);
    A->hyd.resize(m); A->type.resize(m);
    orc_flatten(n_res, aa, pos, A->x.data(), A->y.data(), A->z.data(), A->q.data(), A->rmh.data(), A->eps.data(),
                A->hyd.data(), A->type.data(), nullptr);
    return A;
}
void orc_antigen_free(orc_antigen* A) { delete A; }
void orc_antigen_center(const orc_antigen* A, float out[3]) { out[0] = A->center[0]; out[1] = A->center[1]; out[2] = A->center[2]; }

}  // extern "C"

namespace {
// residue_contribution_allatom (diffusion.rs:425-463): Calpha of residue r against
// every antigen Calpha, AMBER LJ + Coulomb + hydrophobic + H-bond.  Acc = float:
// the reference's f32 sum; Acc = double: the same f32 terms summed in double.
template <class Acc>
Acc residue_contribution_t(const orc_antigen* A, const Prot& P, int r) {
    int baa = P.aa[r];
    int bca = T_TOPO_CA[baa];
    V3 p = P.at(r, bca);
    int bt = T_TOPO_TYPE[baa][bca];
    float brm = T_NB[bt][0], be = T_NB[bt][1], bq = T_TOPO_Q[baa][bca];
    uint8_t bh = T_TOPO_HYD[baa][bca];
    Acc e = 0;
    for (int i = 0; i < A->n_res; ++i) {
        int aaa = A->aa[i];
        int aca = T_TOPO_CA[aaa];
        const float* pa = &A->pos[((size_t)i * SLOTS + aca) * 3];
        float dx = p[0] - pa[0], dy = p[1] - pa[1], dz = p[2] - pa[2];
        float r_sq = dx * dx + dy * dy + dz * dz;
        if (r_sq > CUTOFF_SQ || r_sq < 0.25f) continue;
        int at = T_TOPO_TYPE[aaa][aca];
        float arm = T_NB[at][0], ae = T_NB[at][1], aq = T_TOPO_Q[aaa][aca];
        uint8_t ah = T_TOPO_HYD[aaa][aca];
        float r_ij = brm + arm;
        float eps = std::sqrt(be * ae);
        float r2 = (r_ij * r_ij) / r_sq;
        float r6 = r2 * r2 * r2;
        e += (Acc)(eps * (r6 * r6 - 2.0f * r6));
        if (bq != 0.0f && aq != 0.0f) e += (Acc)(332.0f * bq * aq / std::sqrt(r_sq));
        if (bh == 1 && ah == 1 && r_sq < 36.0f) e -= (Acc)0.5f;
        if (hb_pair(bt, at)) e += (Acc)hbond_energy_mc(r_sq);
    }
    return e;
}
float residue_contribution(const orc_antigen* A, const Prot& P, int r) {
    return residue_contribution_t<float>(A, P, r);
}

// Metropolis criterion (diffusion.rs:368, 385, 414-415): accept downhill moves, else
// with probability exp(-dE/T).  f32: the reference's arithmetic; double: the
// difference of the double energies and a double exponential.
inline bool metropolis(float delta_e, float temp, float u) {
    return delta_e <= 0.0f || u < mc_exp(-delta_e / temp);
}
inline bool metropolis(double delta_e, float temp, float u) {
    return delta_e <= 0.0 || (double)u < std::exp(-delta_e / (double)temp);
}

// allatom_diffusion_step (diffusion.rs:290-419) for one candidate; Acc is the
// accumulation type of the Metropolis energies.
template <class Acc>
void step_one(const orc_antigen* A, const orc_params* prm, Prot& P, uint32_t cand, uint32_t step, float temp,
              bool with_noise, bool with_mc, int64_t* stats) {
    const int n = P.n;
    std::vector<float> fx(n), fy(n), fz(n);
    // Calpha cloud + compute_forces_with_grid (diffusion.rs:306-313)
    for (int r = 0; r < n; ++r) {
        V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
        CgAtom b = cg_atom(ca[0], ca[1], ca[2], P.aa[r]);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        A->grid.query(b.x, b.y, b.z, [&](uint32_t i) { cg_pair(b, A->cg[i], sx, sy, sz); });
        fx[r] = sx; fy[r] = sy; fz[r] = sz;
    }
    float noise_sigma = with_noise ? prm->noise_base * std::sqrt(temp) : 0.0f;
    const float* c = A->center;
    for (int r = 0; r < n; ++r) {  // diffusion.rs:317-339
        V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
        float dx_c = ca[0] - c[0], dy_c = ca[1] - c[1], dz_c = ca[2] - c[2];
        float d = std::fmax(std::sqrt(dx_c * dx_c + dy_c * dy_c + dz_c * dz_c), 0.001f);
        float excess = d - prm->shell_radius;
        float f_r = -prm->restraint_k * excess / d;
        fx[r] += f_r * dx_c;
        fy[r] += f_r * dy_c;
        fz[r] += f_r * dz_c;
        float nx = 0.f, ny = 0.f, nz = 0.f;
        if (with_noise) {
            uint32_t d4[4];
            draw(prm->seed, cand, step, STREAM_NOISE, r, d4);
            nx = frange(d4[0], -noise_sigma, noise_sigma);
            ny = frange(d4[1], -noise_sigma, noise_sigma);
            nz = frange(d4[2], -noise_sigma, noise_sigma);
        }
        auto clampf = [&](float v) { return v > prm->max_disp ? prm->max_disp : (v < -prm->max_disp ? -prm->max_disp : v); };
        V3 new_ca = {ca[0] + clampf(prm->step * fx[r]) + nx,
                     ca[1] + clampf(prm->step * fy[r]) + ny,
                     ca[2] + clampf(prm->step * fz[r]) + nz};
        set_ca_pos(P, r, new_ca);
    }
    if (!with_mc) return;
    auto contrib = [&](int r) { return residue_contribution_t<Acc>(A, P, r); };
    auto ds = [&]() { return disulfide_t<Acc>(P); };
    // interface mask (diffusion.rs:343-351)
    std::vector<char> iface(n);
    for (int r = 0; r < n; ++r) {
        V3 p = P.at(r, T_TOPO_CA[P.aa[r]]);
        bool any = false;
        for (int i = 0; i < A->n_res && !any; ++i) {
            float dx = p[0] - A->cx[i], dy = p[1] - A->cy[i], dz = p[2] - A->cz[i];
            any = dx * dx + dy * dy + dz * dz < prm->iface_cutoff_sq;
        }
        iface[r] = any;
    }
    // mutation / rotamer Metropolis (diffusion.rs:354-399)
    for (int r = 0; r < n; ++r) {
        float eff_mut_p = iface[r] ? prm->mutation_p * 3.0f : prm->mutation_p * 0.4f;
        float eff_rot_p = iface[r] ? prm->rotamer_move_p * 2.0f : prm->rotamer_move_p;
        uint32_t d4[4];
        draw(prm->seed, cand, step, STREAM_MC, r, d4);
        if (!(u01(d4[0]) < eff_mut_p)) continue;
        if (u01(d4[1]) < eff_rot_p) {
            int aa = P.aa[r];
            if (T_ROT_N[aa] == 0) continue;
            float old_chi[4];
            for (int k = 0; k < 4; ++k) old_chi[k] = P.chi[r * 4 + k];
            int rot_idx = (int)urange(d4[2], (uint32_t)T_ROT_N[aa]);
            Acc old_e = contrib(r) + ds();
            for (int k = 0; k < 4; ++k) P.chi[r * 4 + k] = T_ROT[aa][rot_idx][k];
            rebuild_side_chain(P, r);
            Acc new_e = contrib(r) + ds();
            bool accept = metropolis(new_e - old_e, temp, u01(d4[3]));
            if (stats) { stats[0]++; stats[1] += accept; }
            if (!accept) {
                for (int k = 0; k < 4; ++k) P.chi[r * 4 + k] = old_chi[k];
                rebuild_side_chain(P, r);
            }
        } else {
            int old_aa = P.aa[r];
            int new_aa = (int)urange(d4[2], 20u);
            float old_chi[4];
            for (int k = 0; k < 4; ++k) old_chi[k] = P.chi[r * 4 + k];
            Acc old_e = contrib(r) + ds();
            float new_chi[4] = {0.f, 0.f, 0.f, 0.f};
            if (T_ROT_N[new_aa] > 0)
                for (int k = 0; k < 4; ++k) new_chi[k] = T_ROT[new_aa][0][k];
            mutate_residue(P, r, new_aa, new_chi);
            Acc new_e = contrib(r) + ds();
            bool accept = metropolis(new_e - old_e, temp, u01(d4[3]));
            if (stats) { stats[0]++; stats[1] += accept; }
            if (!accept) mutate_residue(P, r, old_aa, old_chi);
        }
    }
    // backbone phi/psi Metropolis (diffusion.rs:403-418)
    for (int r = 0; r < n; ++r) {
        uint32_t d4[4];
        draw(prm->seed, cand, step, STREAM_BACKBONE, r, d4);
        if (!(u01(d4[0]) < prm->backbone_move_p)) continue;
        float delta = frange(d4[1], -prm->max_torsion_deg, prm->max_torsion_deg) * RADS_PER_DEG;
        bool do_phi = (d4[2] >> 31) & 1u;
        Acc old_e = 0;
        for (int i = r; i < n; ++i) old_e += contrib(i);
        old_e += ds();
        if (do_phi) perturb_phi(P, r, delta); else perturb_psi(P, r, delta);
        Acc new_e = 0;
        for (int i = r; i < n; ++i) new_e += contrib(i);
        new_e += ds();
        bool accept = metropolis(new_e - old_e, temp, u01(d4[3]));
        if (stats) { stats[2]++; stats[3] += accept; }
        if (!accept) {
            if (do_phi) perturb_phi(P, r, -delta); else perturb_psi(P, r, -delta);
        }
    }
}
// ---- Fv two-chain engine (diffusion.rs:477-827) --------------------------------------
// residue_contribution_allatom (diffusion.rs:425-463) of residue r of P against the
// Calphas of another chain Q (the Fv partner), the same arithmetic as against the antigen.
template <class Acc>
Acc contribution_vs_chain(const Prot& P, int r, const Prot& Q) {
    int baa = P.aa[r];
    int bca = T_TOPO_CA[baa];
    V3 p = P.at(r, bca);
    int bt = T_TOPO_TYPE[baa][bca];
    float brm = T_NB[bt][0], be = T_NB[bt][1], bq = T_TOPO_Q[baa][bca];
    uint8_t bh = T_TOPO_HYD[baa][bca];
    Acc e = 0;
    for (int i = 0; i < Q.n; ++i) {
        int aaa = Q.aa[i];
        int aca = T_TOPO_CA[aaa];
        V3 pa = Q.at(i, aca);
        float dx = p[0] - pa[0], dy = p[1] - pa[1], dz = p[2] - pa[2];
        float r_sq = dx * dx + dy * dy + dz * dz;
        if (r_sq > CUTOFF_SQ || r_sq < 0.25f) continue;
        int at = T_TOPO_TYPE[aaa][aca];
        float arm = T_NB[at][0], ae = T_NB[at][1], aq = T_TOPO_Q[aaa][aca];
        uint8_t ah = T_TOPO_HYD[aaa][aca];
        float r_ij = brm + arm;
        float eps = std::sqrt(be * ae);
        float r2 = (r_ij * r_ij) / r_sq;
        float r6 = r2 * r2 * r2;
        e += (Acc)(eps * (r6 * r6 - 2.0f * r6));
        if (bq != 0.0f && aq != 0.0f) e += (Acc)(332.0f * bq * aq / std::sqrt(r_sq));
        if (bh == 1 && ah == 1 && r_sq < 36.0f) e -= (Acc)0.5f;
        if (hb_pair(bt, at)) e += (Acc)hbond_energy_mc(r_sq);
    }
    return e;
}

// fv_chain_step (diffusion.rs:560-698) of chain `chain` (0 heavy, 1 light) against the
// antigen and the partner chain snapshot Q.  Draws: Philox streams STREAM_* + 4 * chain,
// per residue (d.x the CDR mutation gate, d.y the rotamer-or-mutation choice or the
// relaxation gate, d.z the rotamer / amino-acid index, d.w the acceptance draw).
template <class Acc>
void fv_chain_step(const orc_antigen* A, const orc_params* prm, Prot& P, const uint8_t* cdr, const Prot& Q,
                   int chain, uint32_t cand, uint32_t step, float temp, float target_radius) {
    const int n = P.n;
    std::vector<float> fx(n), fy(n), fz(n);
    for (int r = 0; r < n; ++r) {
        V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
        CgAtom b = cg_atom(ca[0], ca[1], ca[2], P.aa[r]);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        A->grid.query(b.x, b.y, b.z, [&](uint32_t i) { cg_pair(b, A->cg[i], sx, sy, sz); });
        // VH-VL packing force: compute_forces (energy.rs:154-234) over the partner's Calphas
        float px = 0.f, py = 0.f, pz = 0.f;
        for (int i = 0; i < Q.n; ++i) {
            V3 q = Q.at(i, T_TOPO_CA[Q.aa[i]]);
            cg_pair(b, cg_atom(q[0], q[1], q[2], Q.aa[i]), px, py, pz);
        }
        fx[r] = sx + px; fy[r] = sy + py; fz[r] = sz + pz;
    }
    const float sigma = prm->noise_base * std::sqrt(temp);
    const float* c = A->center;
    const uint32_t sh = 4u * (uint32_t)chain;
    for (int r = 0; r < n; ++r) {
        V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
        float dx_c = ca[0] - c[0], dy_c = ca[1] - c[1], dz_c = ca[2] - c[2];
        float d = std::fmax(std::sqrt(dx_c * dx_c + dy_c * dy_c + dz_c * dz_c), 0.001f);
        float excess = d - target_radius;
        float f_r = -prm->restraint_k * excess / d;
        fx[r] += f_r * dx_c;
        fy[r] += f_r * dy_c;
        fz[r] += f_r * dz_c;
        uint32_t d4[4];
        draw(prm->seed, cand, step, STREAM_NOISE + sh, r, d4);
        float nx = frange(d4[0], -sigma, sigma), ny = frange(d4[1], -sigma, sigma), nz = frange(d4[2], -sigma, sigma);
        auto clampf = [&](float v) { return v > prm->max_disp ? prm->max_disp : (v < -prm->max_disp ? -prm->max_disp : v); };
        V3 new_ca = {ca[0] + clampf(prm->step * fx[r]) + nx, ca[1] + clampf(prm->step * fy[r]) + ny,
                     ca[2] + clampf(prm->step * fz[r]) + nz};
        set_ca_pos(P, r, new_ca);
    }
    auto contrib = [&](int r) { return residue_contribution_t<Acc>(A, P, r) + contribution_vs_chain<Acc>(P, r, Q); };
    auto ds = [&]() { return disulfide_t<Acc>(P); };
    auto rot_move = [&](int r, uint32_t dz, uint32_t dw) {
        int aa = P.aa[r];
        if (T_ROT_N[aa] == 0) return;
        float old_chi[4];
        for (int k = 0; k < 4; ++k) old_chi[k] = P.chi[r * 4 + k];
        int rot_idx = (int)urange(dz, (uint32_t)T_ROT_N[aa]);
        Acc old_e = contrib(r) + ds();
        for (int k = 0; k < 4; ++k) P.chi[r * 4 + k] = T_ROT[aa][rot_idx][k];
        rebuild_side_chain(P, r);
        Acc new_e = contrib(r) + ds();
        if (!metropolis(new_e - old_e, temp, u01(dw))) {
            for (int k = 0; k < 4; ++k) P.chi[r * 4 + k] = old_chi[k];
            rebuild_side_chain(P, r);
        }
    };
    const float mut_p = prm->mutation_p * 3.0f, rot_p = prm->rotamer_move_p * 2.0f,
                relax_p = prm->rotamer_move_p * 0.3f;
    for (int r = 0; r < n; ++r) {
        uint32_t d4[4];
        draw(prm->seed, cand, step, STREAM_MC + sh, r, d4);
        if (cdr[r] && u01(d4[0]) < mut_p) {
            if (u01(d4[1]) < rot_p) {
                rot_move(r, d4[2], d4[3]);
            } else {
                int old_aa = P.aa[r];
                int new_aa = (int)urange(d4[2], 20u);
                float old_chi[4];
                for (int k = 0; k < 4; ++k) old_chi[k] = P.chi[r * 4 + k];
                Acc old_e = contrib(r) + ds();
                float new_chi[4] = {0.f, 0.f, 0.f, 0.f};
                if (T_ROT_N[new_aa] > 0)
                    for (int k = 0; k < 4; ++k) new_chi[k] = T_ROT[new_aa][0][k];
                mutate_residue(P, r, new_aa, new_chi);
                Acc new_e = contrib(r) + ds();
                if (!metropolis(new_e - old_e, temp, u01(d4[3]))) mutate_residue(P, r, old_aa, old_chi);
            }
        } else if (u01(d4[1]) < relax_p) {  // framework (or CDR without a draw): rotamer relaxation
            rot_move(r, d4[2], d4[3]);
        }
    }
    for (int r = 0; r < n; ++r) {  // backbone phi / psi moves, the downstream residues re-scored
        uint32_t d4[4];
        draw(prm->seed, cand, step, STREAM_BACKBONE + sh, r, d4);
        if (!(u01(d4[0]) < prm->backbone_move_p)) continue;
        float delta = frange(d4[1], -prm->max_torsion_deg, prm->max_torsion_deg) * RADS_PER_DEG;
        bool do_phi = (d4[2] >> 31) & 1u;
        Acc old_e = 0;
        for (int i = r; i < n; ++i) old_e += contrib(i);
        old_e += ds();
        if (do_phi) perturb_phi(P, r, delta); else perturb_psi(P, r, delta);
        Acc new_e = 0;
        for (int i = r; i < n; ++i) new_e += contrib(i);
        new_e += ds();
        if (!metropolis(new_e - old_e, temp, u01(d4[3]))) {
            if (do_phi) perturb_phi(P, r, -delta); else perturb_psi(P, r, -delta);
        }
    }
}

// interaction_energy_atoms (energy.rs:256-314) of two slot-layout proteins, the five
// terms added as AtomEnergyBreakdown::total does (acc64: their f64 re-evaluation)
double pair_energy(const Prot& G, const Prot& B, int acc64) {
    auto flat = [](const Prot& P, std::vector<float>* v, std::vector<uint8_t>* u) {
        int m = 0;
        for (int r = 0; r < P.n; ++r) m += T_TOPO_N[P.aa[r]];
        for (int k = 0; k < 6; ++k) v[k].resize(m);
        u[0].resize(m); u[1].resize(m);
        orc_flatten(P.n, P.aa, P.pos, v[0].data(), v[1].data(), v[2].data(), v[3].data(), v[4].data(), v[5].data(),
                    u[0].data(), u[1].data(), nullptr);
        return orc_cloud{v[0].data(), v[1].data(), v[2].data(), v[3].data(), v[4].data(), v[5].data(), u[0].data(),
                         u[1].data(), m};
    };
    std::vector<float> gv[6], bv[6];
    std::vector<uint8_t> gu[2], bu[2];
    orc_cloud g = flat(G, gv, gu), b = flat(B, bv, bu);
    if (acc64) {
        double e[5];
        orc_energy_atoms64(&g, &b, e, nullptr);
        return (((e[0] + e[1]) + e[2]) + e[3]) + e[4];
    }
    float e[5];
    orc_energy_atoms32(&g, &b, e);
    return (double)((((e[0] + e[1]) + e[2]) + e[3]) + e[4]);
}

// fv_energy (diffusion.rs:541-547): antigen-VH + antigen-VL + VH-VL + both disulfide terms
double fv_energy(const orc_antigen* A, const Prot& H, const Prot& L, int acc64) {
    std::vector<float> chi((size_t)A->n_res * 4, 0.f);
    Prot G{A->n_res, const_cast<uint8_t*>(A->aa.data()), chi.data(), const_cast<float*>(A->pos.data())};
    if (acc64)
        return pair_energy(G, H, 1) + pair_energy(G, L, 1) + pair_energy(H, L, 1) + (double)disulfide(H) +
               (double)disulfide(L);
    return (double)((((float)pair_energy(G, H, 0) + (float)pair_energy(G, L, 0)) + (float)pair_energy(H, L, 0) +
                     disulfide(H)) + disulfide(L));
}

}  // namespace

extern "C" {

float orc_residue_contribution(const orc_antigen* A, int n_res, const uint8_t* aa, const float* pos, int r) {
    std::vector<uint8_t> a(aa, aa + n_res);
    std::vector<float> chi((size_t)n_res * 4, 0.f);
    Prot P{n_res, a.data(), chi.data(), const_cast<float*>(pos)};
    return residue_contribution(A, P, r);
}

double orc_residue_contribution64(const orc_antigen* A, int n_res, const uint8_t* aa, const float* pos, int r) {
    std::vector<uint8_t> a(aa, aa + n_res);
    std::vector<float> chi((size_t)n_res * 4, 0.f);
    Prot P{n_res, a.data(), chi.data(), const_cast<float*>(pos)};
    return residue_contribution_t<double>(A, P, r);
}

float orc_disulfide(int n_res, const uint8_t* aa, const float* pos) {
    std::vector<uint8_t> a(aa, aa + n_res);
    std::vector<float> chi((size_t)n_res * 4, 0.f);
    Prot P{n_res, a.data(), chi.data(), const_cast<float*>(pos)};
    return disulfide(P);
}

void orc_step(const orc_antigen* A, const orc_params* prm, int n_cand, int n_res, uint8_t* aa, float* chi, float* pos,
              const uint32_t* cand_id, uint32_t step_id, float temp, int with_noise, int with_mc, int64_t* stats,
              int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        Prot P{n_res, aa + (size_t)c * n_res, chi + (size_t)c * n_res * 4, pos + (size_t)c * n_res * SLOTS * 3};
        const uint32_t id = cand_id ? cand_id[c] : (uint32_t)c;
        int64_t* st = stats ? stats + c * 4 : nullptr;
        if (prm->accumulate == 1) step_one<float>(A, prm, P, id, step_id, temp, with_noise != 0, with_mc != 0, st);
        else step_one<double>(A, prm, P, id, step_id, temp, with_noise != 0, with_mc != 0, st);
    });
}

// allatom_energy (diffusion.rs:281-283) when full, else the score_batch terms
void orc_score_slots64(const orc_antigen* A, int n_cand, int n_res, const uint8_t* aa, const float* pos, int full,
                       double* out, double* out_abs, int n_threads) {
    orc_cloud ag{A->x.data(), A->y.data(), A->z.data(), A->q.data(), A->rmh.data(), A->eps.data(), A->hyd.data(),
                 A->type.data(), (int64_t)A->x.size()};
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        const uint8_t* caa = aa + (size_t)c * n_res;
        const float* cpos = pos + (size_t)c * n_res * SLOTS * 3;
        int m = 0;
        for (int r = 0; r < n_res; ++r) m += T_TOPO_N[caa[r]];
        std::vector<float> x(m), y(m), z(m), q(m), rmh(m), eps(m);
        std::vector<uint8_t> hyd(m), type(m);
        orc_flatten(n_res, caa, cpos, x.data(), y.data(), z.data(), q.data(), rmh.data(), eps.data(), hyd.data(),
                    type.data(), nullptr);
        orc_cloud ab{x.data(), y.data(), z.data(), q.data(), rmh.data(), eps.data(), hyd.data(), type.data(), m};
        double e[5], ea[5];
        orc_energy_atoms64(&ag, &ab, e, ea);
        double tot = e[0] + e[1] + e[2];
        double tot_abs = ea[0] + ea[1] + ea[2];
        if (full) {
            std::vector<uint8_t> a2(caa, caa + n_res);
            std::vector<float> chi((size_t)n_res * 4, 0.f);
            Prot P{n_res, a2.data(), chi.data(), const_cast<float*>(cpos)};
            const double ds = (double)disulfide(P);
            tot += e[3] + e[4] + ds;
            tot_abs += ea[3] + ea[4] + std::fabs(ds);
        }
        out[c] = tot;
        if (out_abs) out_abs[c] = tot_abs;
    });
}

// partners_energy (diffusion.rs:835-840) with the antigen as the one partner =
// allatom_energy (diffusion.rs:281-283): interaction_energy_atoms (the five terms of
// energy.rs:261-314 + solvation.rs:52-84, added as AtomEnergyBreakdown::total does)
// plus disulfide_energy.  acc64: the same terms re-evaluated in f64.
static double partner_energy(const orc_antigen* A, const Prot& P, int acc64) {
    int m = 0;
    for (int r = 0; r < P.n; ++r) m += T_TOPO_N[P.aa[r]];
    std::vector<float> x(m), y(m), z(m), q(m), rmh(m), eps(m);
    std::vector<uint8_t> hyd(m), type(m);
    orc_flatten(P.n, P.aa, P.pos, x.data(), y.data(), z.data(), q.data(), rmh.data(), eps.data(), hyd.data(),
                type.data(), nullptr);
    orc_cloud ag{A->x.data(), A->y.data(), A->z.data(), A->q.data(), A->rmh.data(), A->eps.data(), A->hyd.data(),
                 A->type.data(), (int64_t)A->x.size()};
    orc_cloud ab{x.data(), y.data(), z.data(), q.data(), rmh.data(), eps.data(), hyd.data(), type.data(), m};
    if (acc64) {
        double e[5];
        orc_energy_atoms64(&ag, &ab, e, nullptr);
        return (((e[0] + e[1]) + e[2]) + e[3]) + e[4] + (double)disulfide(P);
    }
    float e[5];
    orc_energy_atoms32(&ag, &ab, e);
    return (double)((((e[0] + e[1]) + e[2]) + e[3]) + e[4] + disulfide(P));
}

// minimize (diffusion.rs:854-916) with the antigen as the one partner
// (main.rs:338): steepest descent on the Calpha-level grid force with the step
// decaying linearly (MIN_STEP 0.04, MIN_MAX_DISP 0.5, diffusion.rs:63-64), side
// chains rebuilt after every move, a step kept only when the all-atom energy
// drops.  out_energy = the final best energy.
void orc_minimize(const orc_antigen* A, int n_cand, int n_res, uint8_t* aa, float* chi, float* pos, int steps,
                  int acc64, double* out_energy, double* out_margin, int n_threads) {
    const float MIN_STEP = 0.04f, MIN_MAX_DISP = 0.5f;
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        Prot P{n_res, aa + (size_t)c * n_res, chi + (size_t)c * n_res * 4, pos + (size_t)c * n_res * SLOTS * 3};
        double best = partner_energy(A, P, acc64);
        double margin = INFINITY;  // smallest |e - best| / max(|best|, 1) of any keep / restore decision
        if (n_res > 0 && steps > 0) {
            std::vector<float> fx(n_res), fy(n_res), fz(n_res);
            std::vector<float> keep_pos((size_t)n_res * SLOTS * 3);
            for (int step = 0; step < steps; ++step) {
                const float frac = 1.0f - (float)step / (float)steps;
                const float step_size = MIN_STEP * frac;
                std::copy(P.pos, P.pos + keep_pos.size(), keep_pos.begin());
                for (int r = 0; r < n_res; ++r) {  // compute_forces_with_grid on the pre-step Calphas
                    V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
                    CgAtom b = cg_atom(ca[0], ca[1], ca[2], P.aa[r]);
                    float sx = 0.f, sy = 0.f, sz = 0.f;
                    A->grid.query(b.x, b.y, b.z, [&](uint32_t i) { cg_pair(b, A->cg[i], sx, sy, sz); });
                    // fx_buf (zeroed) += the one partner's force
                    fx[r] = 0.0f + sx; fy[r] = 0.0f + sy; fz[r] = 0.0f + sz;
                }
                auto clampf = [&](float v) { return v < -MIN_MAX_DISP ? -MIN_MAX_DISP : (v > MIN_MAX_DISP ? MIN_MAX_DISP : v); };
                for (int r = 0; r < n_res; ++r) {
                    V3 ca = P.at(r, T_TOPO_CA[P.aa[r]]);
                    V3 disp = {clampf(step_size * fx[r]), clampf(step_size * fy[r]), clampf(step_size * fz[r])};
                    set_ca_pos(P, r, V3{ca[0] + disp[0], ca[1] + disp[1], ca[2] + disp[2]});
                    rebuild_side_chain(P, r);
                }
                const double e = partner_energy(A, P, acc64);
                margin = std::min(margin, std::fabs(e - best) / std::max(std::fabs(best), 1.0));
                if (e < best) best = e;
                else std::copy(keep_pos.begin(), keep_pos.end(), P.pos);
            }
        }
        out_energy[c] = best;
        if (out_margin) out_margin[c] = margin;
    });
}

// is_interface (filters.rs:96-105): some antigen Calpha closer than IFACE_SQ (64)
static bool is_interface(const orc_antigen* A, const Prot& P, int r) {
    V3 p = P.at(r, T_TOPO_CA[P.aa[r]]);
    for (int i = 0; i < A->n_res; ++i) {
        float dx = p[0] - A->cx[i], dy = p[1] - A->cy[i], dz = p[2] - A->cz[i];
        if (dx * dx + dy * dy + dz * dz < 64.0f) return true;
    }
    return false;
}

// affinity_maturation_allatom (diffusion.rs:924-961) over the interface residues
// (main.rs:342-345): for each mutable position in order, the amino acids in
// ALL_AA order (atom.rs:29) other than the current one, each built at its top
// rotamer (chi 0 without rotamers); the first strictly lower allatom_energy is
// kept, otherwise the residue is mutated back to its old amino acid and chi.
// out_energy = the final best score, out_mutated[c] = mutations kept.
void orc_affinity_maturation(const orc_antigen* A, int n_cand, int n_res, uint8_t* aa, float* chi, float* pos,
                             int acc64, double* out_energy, int32_t* out_mutated, double* out_margin,
                             int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        Prot P{n_res, aa + (size_t)c * n_res, chi + (size_t)c * n_res * 4, pos + (size_t)c * n_res * SLOTS * 3};
        std::vector<int> mutable_pos;
        for (int r = 0; r < n_res; ++r)
            if (is_interface(A, P, r)) mutable_pos.push_back(r);
        double best = partner_energy(A, P, acc64);
        double margin = INFINITY;
        int kept = 0;
        for (int r : mutable_pos) {
            const int old_aa = P.aa[r];
            float old_chi[4];
            for (int k = 0; k < 4; ++k) old_chi[k] = P.chi[r * 4 + k];
            for (int cand_aa = 0; cand_aa < 20; ++cand_aa) {
                if (cand_aa == old_aa) continue;
                float new_chi[4] = {0.f, 0.f, 0.f, 0.f};
                if (T_ROT_N[cand_aa] > 0)
                    for (int k = 0; k < 4; ++k) new_chi[k] = T_ROT[cand_aa][0][k];
                mutate_residue(P, r, cand_aa, new_chi);
                const double e = partner_energy(A, P, acc64);
                margin = std::min(margin, std::fabs(e - best) / std::max(std::fabs(best), 1.0));
                if (e < best) {
                    best = e;
                    ++kept;
                    break;
                }
                mutate_residue(P, r, old_aa, old_chi);
            }
        }
        out_energy[c] = best;
        if (out_mutated) out_mutated[c] = kept;
        if (out_margin) out_margin[c] = margin;
    });
}

// ValidationReport::assess (validate.rs:24-32) of one slot-layout protein.
// clash_score (validate.rs:40-63): pairs i < j of the flattened atoms whose residues
// differ by more than one, d^2 < (0.7 (rmh_i + rmh_j))^2.  ramachandran_outliers
// (validate.rs:112-132): phi (validate.rs:89-98) and psi (:101-110) of residues with
// both, dihedral (:72-86) in degrees (f32 to_degrees: x * 57.29578); atan2 is
// evaluated in double and rounded once to f32 (Rust's f32::atan2 is libm's atan2f).
static float dihedral_deg(const V3& p0, const V3& p1, const V3& p2, const V3& p3) {
    V3 b1 = sub3(p1, p0), b2 = sub3(p2, p1), b3 = sub3(p3, p2);
    V3 n1 = norm3(cross3(b1, b2));
    V3 n2 = norm3(cross3(b2, b3));
    V3 m1 = cross3(n1, norm3(b2));
    float x = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    float y = m1[0] * n2[0] + m1[1] * n2[1] + m1[2] * n2[2];
    return (float)std::atan2((double)y, (double)x) * 57.2957795130823208767981548141051703f;
}

static bool in_allowed_basin(float phi, float psi) {  // validate.rs:101-108
    bool alpha_r = (phi >= -100.0f && phi <= -30.0f) && (psi >= -80.0f && psi <= -5.0f);
    bool beta = ((phi >= -170.0f && phi <= -60.0f) && (psi >= 90.0f && psi <= 180.0f)) ||
                ((phi >= -170.0f && phi <= -60.0f) && (psi >= -180.0f && psi <= -150.0f));
    bool alpha_l = (phi >= 30.0f && phi <= 100.0f) && (psi >= -10.0f && psi <= 80.0f);
    return alpha_r || beta || alpha_l;
}

void orc_validate(int n_res, const uint8_t* aa, const float* pos, int32_t* clashes, int32_t* rama) {
    std::vector<float> x, y, z, rmh;
    std::vector<int> ri;
    for (int r = 0; r < n_res; ++r)
        for (int k = 0; k < T_TOPO_N[aa[r]]; ++k) {
            const float* p = pos + ((size_t)r * SLOTS + k) * 3;
            x.push_back(p[0]); y.push_back(p[1]); z.push_back(p[2]);
            rmh.push_back(T_NB[T_TOPO_TYPE[aa[r]][k]][0]);
            ri.push_back(r);
        }
    int32_t c = 0;
    const size_t m = x.size();
    for (size_t i = 0; i < m; ++i)
        for (size_t j = i + 1; j < m; ++j) {
            if (std::abs(ri[i] - ri[j]) <= 1) continue;
            float dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
            float d_sq = dx * dx + dy * dy + dz * dz;
            float thresh = 0.7f * (rmh[i] + rmh[j]);
            if (d_sq < thresh * thresh) ++c;
        }
    *clashes = c;
    Prot P{n_res, const_cast<uint8_t*>(aa), nullptr, const_cast<float*>(pos)};
    int32_t out = 0;
    for (int r = 1; r + 1 < n_res; ++r) {
        float phi = dihedral_deg(P.at(r - 1, 2), P.at(r, 0), P.at(r, 1), P.at(r, 2));
        float psi = dihedral_deg(P.at(r, 0), P.at(r, 1), P.at(r, 2), P.at(r + 1, 0));
        if (!in_allowed_basin(phi, psi)) ++out;
    }
    *rama = out;
}

// The iteration loop of run_fv (diffusion.rs:791-812) for every candidate: per
// iteration the heavy chain steps against the light chain as it was, the light
// chain against the stepped heavy chain, and the pair is kept when fv_energy drops
// below the best, put back to the best pair when it rises (elitist).  Chains in
// place (the best pair at the end); out_energy = best fv_energy; the step draws use
// cand_id[c] (NULL: c); out_margin (may be NULL): the smallest |e - best| / max(|best|, 1)
// of the keep / restore decisions.
void orc_fv_run(const orc_antigen* A, const orc_params* prm, int n_cand, int n_h, int n_l, uint8_t* aa_h,
                float* chi_h, float* pos_h, const uint8_t* cdr_h, uint8_t* aa_l, float* chi_l, float* pos_l,
                const uint8_t* cdr_l, const uint32_t* cand_id, int iterations, float target_radius, int acc64,
                double* out_energy, double* out_margin, int n_threads) {
    parallel_for(n_cand, n_threads, [&](int64_t c) {
        Prot H{n_h, aa_h + (size_t)c * n_h, chi_h + (size_t)c * n_h * 4, pos_h + (size_t)c * n_h * SLOTS * 3};
        Prot L{n_l, aa_l + (size_t)c * n_l, chi_l + (size_t)c * n_l * 4, pos_l + (size_t)c * n_l * SLOTS * 3};
        const uint32_t id = cand_id ? cand_id[c] : (uint32_t)c;
        auto copy_of = [](const Prot& P, std::vector<uint8_t>& a, std::vector<float>& ch, std::vector<float>& p) {
            a.assign(P.aa, P.aa + P.n);
            ch.assign(P.chi, P.chi + (size_t)P.n * 4);
            p.assign(P.pos, P.pos + (size_t)P.n * SLOTS * 3);
            return Prot{P.n, a.data(), ch.data(), p.data()};
        };
        auto put = [](Prot& P, const Prot& S) {
            std::copy(S.aa, S.aa + P.n, P.aa);
            std::copy(S.chi, S.chi + (size_t)P.n * 4, P.chi);
            std::copy(S.pos, S.pos + (size_t)P.n * SLOTS * 3, P.pos);
        };
        std::vector<uint8_t> bha, bla, sa;
        std::vector<float> bhc, bhp, blc, blp, sc, sp;
        Prot BH = copy_of(H, bha, bhc, bhp), BL = copy_of(L, bla, blc, blp);
        double best = fv_energy(A, H, L, acc64), margin = INFINITY;
        for (int it = 0; it < iterations; ++it) {
            const float temp = orc_temperature(it, iterations);
            {
                Prot snap = copy_of(L, sa, sc, sp);
                if (prm->accumulate == 1) fv_chain_step<float>(A, prm, H, cdr_h, snap, 0, id, (uint32_t)it, temp, target_radius);
                else fv_chain_step<double>(A, prm, H, cdr_h, snap, 0, id, (uint32_t)it, temp, target_radius);
            }
            {
                Prot snap = copy_of(H, sa, sc, sp);
                if (prm->accumulate == 1) fv_chain_step<float>(A, prm, L, cdr_l, snap, 1, id, (uint32_t)it, temp, target_radius);
                else fv_chain_step<double>(A, prm, L, cdr_l, snap, 1, id, (uint32_t)it, temp, target_radius);
            }
            const double e = fv_energy(A, H, L, acc64);
            margin = std::min(margin, std::fabs(e - best) / std::max(std::fabs(best), 1.0));
            if (e < best) {
                best = e;
                put(BH, H);
                put(BL, L);
            } else if (e > best) {
                put(H, BH);
                put(L, BL);
            }
        }
        put(H, BH);
        put(L, BL);
        out_energy[c] = best;
        if (out_margin) out_margin[c] = margin;
    });
}

double orc_fv_energy(const orc_antigen* A, int n_h, const uint8_t* aa_h, const float* pos_h, int n_l,
                     const uint8_t* aa_l, const float* pos_l, int acc64) {
    std::vector<float> ch((size_t)n_h * 4), cl((size_t)n_l * 4);
    Prot H{n_h, const_cast<uint8_t*>(aa_h), ch.data(), const_cast<float*>(pos_h)};
    Prot L{n_l, const_cast<uint8_t*>(aa_l), cl.data(), const_cast<float*>(pos_l)};
    return fv_energy(A, H, L, acc64);
}

void orc_topk(const double* e, int64_t n, int64_t k, int32_t* out_idx) {
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::stable_sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) {
        double ea = e[a], eb = e[b];
        bool na = ea != ea, nb = eb != eb;
        if (na || nb) return !na && nb;
        return ea < eb;
    });
    for (int64_t i = 0; i < k && i < n; ++i) out_idx[i] = idx[i];
}

}  // extern "C"
