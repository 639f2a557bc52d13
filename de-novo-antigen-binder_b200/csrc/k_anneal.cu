// k_anneal.cu — allatom_diffusion_step with its Metropolis moves (diffusion.rs:290-463)
// on the GPU: one CTA per candidate, the candidate's residues and its antigen's
// Calphas resident in shared memory for all n_steps of the launch.
//
// Per step, in the reference's order:
//  1. Langevin: coarse-grained force, restraint, noise, 2 A clamp, rigid
//     translation (diffusion.rs:306-339).  A residue's force comes from its Verlet
//     list (8 lanes per residue, 16 in the 16-warp instance), whose in-cutoff
//     entries in list order are the reference's pairs in its order; its lane 0
//     adds their terms in that order, which is the reference's sequential sum.
//     Candidates too long for lists: eight lanes per residue split the 27 probe
//     cells (reference order) into consecutive runs and lane 0 adds the runs'
//     terms lane by lane.
//  2. Interface mask: any antigen Calpha within sqrt(iface_cutoff_sq) (:343-351).
//  3. Mutation / rotamer sweep (:354-399).  A move at residue r changes only
//     residue r's atoms, and the Calpha-level energy of r depends only on r's
//     Calpha and amino acid; residues interact only through the disulfide term.
//     So every residue's proposal, its rejection rebuild and both Calpha energies
//     are computed in parallel (builds on one half of the warps, energies on the
//     other); one thread takes the decisions that involve a Cys in residue order,
//     updating the disulfide energy, and records the disulfide energy current at
//     every other move's turn; those moves, which leave it unchanged, are then
//     decided in parallel — the reference's sequential sweep, exactly.
//  4. Backbone phi/psi sweep (:403-418): sequential over the attempted moves;
//     per move the Calpha energies of residues r..n are evaluated by warps, the
//     downstream atoms rotated by all threads (Rodrigues, allatom.rs:397-479), and
//     the decision broadcast; a rejected move is undone by the opposite rotation,
//     as in the reference.
// Calpha energies are cached per residue and recomputed whenever the Calpha moved.
//
// Accumulation: ACC = float reproduces the reference's f32 sums bit for bit; ACC =
// double sums the same f32 pair terms in double and takes the Metropolis test on
// the double energy difference.
#include "cg_list.cuh"
#include "geom.cuh"
#include "kernels.h"
#include "mlp_tile.cuh"

namespace binder {

cudaError_t anneal_init_tables() { return geom_init_tables(); }

// log1p of the environment counts for the in-kernel features (the same host table
// as the feature kernel's); copied to shared memory by each learned-proposal CTA
__device__ float g_an_log1p[MLP_COUNT_CAP + 1];
cudaError_t anneal_init_mlp_table(const float* t) {
    return cudaMemcpyToSymbol(g_an_log1p, t, sizeof(float) * (MLP_COUNT_CAP + 1));
}

constexpr int AN_WARPS = 8;
constexpr int AN_THREADS = AN_WARPS * 32;
constexpr int CG_LANES = 8;                          // lanes per residue in the Langevin probe
constexpr int CG_RES_PER_PASS = AN_THREADS / CG_LANES;
constexpr int CG_SLOTS = 16;                         // in-cutoff terms a lane holds
static_assert(CG_IN_MAX * (16 + 4) <= CG_LANES * CG_SLOTS * 16, "list scratch must fit a group's term slots");
constexpr int STAGE_CAP = 64;                        // staged in-cutoff terms per warp
constexpr int AG_STAGE_MAX = 1024;                   // antigen Calphas staged in shared memory
constexpr int CELL_STAGE_MAX = 4096;                 // Calpha-grid cells staged in shared memory
enum : int { MV_NONE = 0, MV_ROT = 1, MV_MUT = 2 };
enum : int { SEL_KEEP = 0, SEL_PROP = 1, SEL_REJ = 2 };
enum : int { IS_DVALID = 0, IS_DECISION = 1, IS_NCYS = 2, IS_LASTCYS = 3, IS_NMV = 4, IS_NTASK = 5 };

// Shared-memory carve of one CTA for candidates of up to R residues and antigens
// of up to G staged Calphas.
struct AnSmem {
    float4 *pos, *prop, *rej;  // R * SLOT_STRIDE each: state, proposal, rejection rebuild
    float4* trig;              // 2R: sin/cos of chi1..4
    float4* chi;               // R (degrees)
    float4* ldelta;            // R: Langevin translation
    float4* bb_trig;           // R: cos, sin of the torsion step and of its negation
    float4* terms;             // min(R, 32) * CG_LANES * CG_SLOTS Langevin pair terms; with the learned
                               // proposal also the network tile (the two are never live together)
    float4* stage;             // AN_WARPS * STAGE_CAP: in-cutoff Calpha-energy terms
    float4 *agq, *agp;         // G staged antigen Calphas: x, y, z, q | r_min_half, eps, hyd, type
    float4 *cgq, *cgp;         // G staged Calphas in CG-grid order (AgView::ca_pq, ca_prm)
    float *agx, *agy, *agz;    // anneal_xyz_len(G) each: the staged Calphas' x, y, z (pad +1e30)
    int* cgcell;               // C staged CG-grid cell starts
    AgView* ag;
    double *c_cur, *c_old, *c_new;  // R: Calpha energies (exact f32 values when ACC = float)
    double* dscal;                  // [0] disulfide energy of the current state
    double* lhr;                    // R: log Hastings ratio of the move (network path)
    double* d_turn;                 // R: the disulfide energy current at the move's turn (moves
                                    // without a Cys, decided after the sequential pass)
    float *u_acc, *bb_u;            // R
    int *aa, *kind, *new_aa, *new_rot, *sel, *valid, *bb_att, *bb_phi, *iface;
    int* tcount;                    // L (>= 2R): Langevin term counts of the lanes; after the Langevin step
                                    // the Calpha-energy tasks of the step's moves, 2 r + (0 before, 1 after)
    int *rot, *mvl;                 // R: rotamer index of the state (-1 unknown), residues with a move
    uint32_t* dz;                   // R: the move's choice draw
    int* iscal;
    uint8_t* agaa;                  // learned proposal: G staged antigen amino acids
    float* lg1p;                    // learned proposal: the log1p count table
    float* mbias;                   // learned proposal: the network's biases b1 | b2 | b3
    int* cglist;                    // LR x CG_LIST_MAX: Verlet lists of the Langevin force
    float4* cgcentre;               // LR: list centre, skin
    int* cgnl;                      // LR: list length (-1: none yet)
    // Fv two-chain steps: the partner chain's Calphas, as Calpha atoms (ptq, ptp: the
    // agq / agp layout) and as residue-level bodies of the CG force (pcq, pcp: the
    // AgView::ca_pq / ca_prm layout); R each
    float4 *ptq, *ptp, *pcq, *pcp;
};
// Entries of each staged x / y / z array: room for the pad, a multiple of 4 (the
// arrays after them keep their 16-byte alignment).
__host__ __device__ inline int anneal_xyz_len(int G) { return G > 0 ? (G + 4) & ~3 : 0; }
static_assert(32 * CG_LANES >= 2 * ANNEAL_MAX_RES, "the term counts hold two energy tasks per residue");
// Residues with Verlet lists in shared memory: candidates of up to one Langevin
// pass (CG_RES_PER_PASS residues); longer ones walk the 27 cells every step.
__host__ __device__ inline int anneal_list_res(int R) { return R <= CG_RES_PER_PASS ? R : 0; }
__host__ __device__ inline size_t anneal_terms_bytes(int R, int learned) {
    const int L = (R < CG_RES_PER_PASS ? R : CG_RES_PER_PASS) * CG_LANES;
    const size_t t = (size_t)L * CG_SLOTS * 16;
    return learned && t < (size_t)MT_BYTES ? (size_t)MT_BYTES : t;
}
__host__ __device__ inline size_t anneal_smem_bytes(int R, int G, int C, int learned, int fv = 0,
                                                    int warps = AN_WARPS) {
    const int L = (R < CG_RES_PER_PASS ? R : CG_RES_PER_PASS) * CG_LANES;
    return (size_t)R * SLOT_STRIDE * 16 * 3 + (size_t)R * 16 * 5 + anneal_terms_bytes(R, learned) +
           (size_t)warps * STAGE_CAP * 16 + (size_t)G * 64 + (size_t)anneal_xyz_len(G) * 12 +
           ((size_t)C * 4 + 15) / 16 * 16 +
           ((sizeof(AgView) + 15) / 16) * 16 +
           (size_t)R * 8 * 3 + 16 + (size_t)R * 8 * 2 + (size_t)R * 4 * 2 + (size_t)R * 4 * 9 + (size_t)L * 4 +
           (size_t)R * 4 * 3 + 32 + (learned ? ((size_t)G + 15) / 16 * 16 + (MLP_COUNT_CAP + 1 + MLP_BIASES) * 4 : 0) +
           15 + (size_t)anneal_list_res(R) * (CG_LIST_MAX * 4 + 16 + 4) +  // 15: alignment of cgcentre
           (fv ? 15 + (size_t)R * 64 : 0);
}
__device__ inline AnSmem carve(unsigned char* b, int R, int G, int C, int learned, int fv = 0, int warps = AN_WARPS) {
    AnSmem s;
    const int L = min(R, CG_RES_PER_PASS) * CG_LANES;
    auto take = [&](size_t bytes) { unsigned char* p = b; b += bytes; return p; };
    s.pos = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.prop = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.rej = (float4*)take((size_t)R * SLOT_STRIDE * 16);
    s.trig = (float4*)take((size_t)R * 32);
    s.chi = (float4*)take((size_t)R * 16);
    s.ldelta = (float4*)take((size_t)R * 16);
    s.bb_trig = (float4*)take((size_t)R * 16);
    s.terms = (float4*)take(anneal_terms_bytes(R, learned));
    s.stage = (float4*)take((size_t)warps * STAGE_CAP * 16);
    s.agq = (float4*)take((size_t)G * 16);
    s.agp = (float4*)take((size_t)G * 16);
    s.cgq = (float4*)take((size_t)G * 16);
    s.cgp = (float4*)take((size_t)G * 16);
    s.agx = (float*)take((size_t)anneal_xyz_len(G) * 4);
    s.agy = (float*)take((size_t)anneal_xyz_len(G) * 4);
    s.agz = (float*)take((size_t)anneal_xyz_len(G) * 4);
    s.cgcell = (int*)take(((size_t)C * 4 + 15) / 16 * 16);
    s.ag = (AgView*)take(((sizeof(AgView) + 15) / 16) * 16);
    s.c_cur = (double*)take((size_t)R * 8);
    s.c_old = (double*)take((size_t)R * 8);
    s.c_new = (double*)take((size_t)R * 8);
    s.dscal = (double*)take(16);
    s.lhr = (double*)take((size_t)R * 8);
    s.d_turn = (double*)take((size_t)R * 8);
    s.u_acc = (float*)take((size_t)R * 4);
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
    s.tcount = (int*)take((size_t)L * 4);
    s.rot = (int*)take((size_t)R * 4);
    s.mvl = (int*)take((size_t)R * 4);
    s.dz = (uint32_t*)take((size_t)R * 4);
    s.iscal = (int*)take(32);
    s.agaa = learned ? (uint8_t*)take(((size_t)G + 15) / 16 * 16) : nullptr;
    s.lg1p = learned ? (float*)take((MLP_COUNT_CAP + 1) * 4) : nullptr;
    s.mbias = learned ? (float*)take(MLP_BIASES * 4) : nullptr;
    const int LR = anneal_list_res(R);
    b = (unsigned char*)(((uintptr_t)b + 15) & ~(uintptr_t)15);  // float4 alignment (the arrays before: ints)
    s.cgcentre = (float4*)take((size_t)LR * 16);
    s.cglist = (int*)take((size_t)LR * CG_LIST_MAX * 4);
    s.cgnl = (int*)take((size_t)LR * 4);
    s.ptq = s.ptp = s.pcq = s.pcp = nullptr;
    if (fv) {
        b = (unsigned char*)(((uintptr_t)b + 15) & ~(uintptr_t)15);
        s.ptq = (float4*)take((size_t)R * 16);
        s.ptp = (float4*)take((size_t)R * 16);
        s.pcq = (float4*)take((size_t)R * 16);
        s.pcp = (float4*)take((size_t)R * 16);
    }
    return s;
}

// hbond_energy (energy.rs:32-39) with the Metropolis-path exponential
__device__ __forceinline__ float hbond_mc(float r_sq) {
    if (r_sq > HB_CUTOFF_SQ) return 0.0f;
    const float r = xsqrt(r_sq);
    const float z = xdiv(xsub(r, HB_R0), HB_SIGMA);
    return xmul(-HB_DEPTH, mc_exp(xmul(xmul(-0.5f, z), z)));
}

// Add staged Calpha-energy terms in order (lj; coulomb; hydrophobic; hbond per pair).
template <class ACC>
__device__ __forceinline__ void fold_terms(const float4* stage, int cnt, ACC& e) {
    for (int j = 0; j < cnt; ++j) {
        const float4 v = stage[j];
        const unsigned fl = __float_as_uint(v.w);
        e += (ACC)v.x;
        if (fl & 1u) e += (ACC)v.y;
        if (fl & 2u) e -= (ACC)0.5f;
        if (fl & 4u) e += (ACC)v.z;
    }
}

// The staged terms of one in-cutoff pair (r_sq passed the reference's cutoff test):
// lj; coulomb (flag 1); hydrophobic (flag 2); hbond (flag 4) -- residue_contribution_
// allatom's per-pair arithmetic (diffusion.rs:425-463).  b = the residue's Calpha
// (q, r_min_half, epsilon, hydrophobic), bhb its H-bond role.
__device__ __forceinline__ float4 ca_pair_terms(const float4& b, int bhb, const float4& a, const float4& ap,
                                                float r_sq) {
    float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
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
    return t;
}

// residue_contribution_allatom (diffusion.rs:425-463) of a Calpha at `ca` of amino
// acid `aa`, by one warp: lanes evaluate 32 antigen Calphas at a time (index
// order), in-cutoff terms are compacted into the warp's stage in that order and
// lane 0 adds them in the reference's order.  Result valid in lane 0.
template <class ACC>
__device__ __noinline__ ACC warp_contribution(const float4* __restrict__ agq, const float4* __restrict__ agp, int nag, F3 ca,
                                 int aa, float4* stage) {
    const int lane = threadIdx.x & 31;
    const float4 b = s_ca_atom[aa];  // q, r_min_half, epsilon, hydrophobic
    const int bhb = s_hb_role[s_ca_type[aa]];
    ACC e = 0;
    int cnt = 0;
    for (int base = 0; base < nag; base += 32) {
        const int i = base + lane;
        bool in = false;
        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
        if (i < nag) {
            const float4 a = agq[i];
            const float r_sq = xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z));
            in = !(r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ);
            if (in) t = ca_pair_terms(b, bhb, a, agp[i], r_sq);
        }
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) stage[cnt + __popc(m & ((1u << lane) - 1u))] = t;
        cnt += __popc(m);
        if (cnt > STAGE_CAP - 32) {  // flush before the stage can overflow
            __syncwarp();
            if (lane == 0) fold_terms(stage, cnt, e);
            __syncwarp();
            cnt = 0;
        }
    }
    __syncwarp();
    if (lane == 0) fold_terms(stage, cnt, e);
    __syncwarp();
    return e;
}

// The same for a staged antigen whose Calpha coordinates are also kept as x / y / z
// arrays (ax, ay, az; 8-byte aligned, entry nag a +1e30 pad when nag is odd).  Lane
// l tests Calphas base + 2l and base + 2l + 1 with one packed f32x2 computation (the
// same roundings as xdist2), 64 Calphas per warp step, and stages each in-cutoff
// Calpha's (r^2, index) in index order; the pair terms of everything staged are then
// computed one entry per lane (in place) and lane 0 adds them in order -- so the
// term code runs once per 32 in-cutoff Calphas instead of once per scan step.
template <class ACC>
__device__ __noinline__ ACC warp_contribution_pairs(const float* __restrict__ ax, const float* __restrict__ ay,
                                       const float* __restrict__ az, const float4* __restrict__ agq,
                                       const float4* __restrict__ agp, int nag, F3 ca, int aa, float4* stage) {
    static_assert(STAGE_CAP >= 64, "one step stages up to 64 entries");
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const float4 b = s_ca_atom[aa];
    const int bhb = s_hb_role[s_ca_type[aa]];
    const uint64_t cx = f2_pack(ca.x, ca.x), cy = f2_pack(ca.y, ca.y), cz = f2_pack(ca.z, ca.z);
    ACC e = 0;
    int cnt = 0;
    auto terms_and_fold = [&]() {  // the staged entries' terms, in place, then their sum in order
        __syncwarp();
        for (int k = lane; k < cnt; k += 32) {
            const float4 v = stage[k];
            const int i = __float_as_int(v.y);
            stage[k] = ca_pair_terms(b, bhb, agq[i], agp[i], v.x);
        }
        __syncwarp();
        if (lane == 0) fold_terms(stage, cnt, e);
        __syncwarp();
        cnt = 0;
    };
    for (int base = 0; base < nag; base += 64) {
        const int i = base + 2 * lane;
        bool in0 = false, in1 = false;
        float r0 = 0.0f, r1 = 0.0f;
        if (i < nag) {
            const uint64_t dx = f2_sub(cx, *(const uint64_t*)&ax[i]);
            const uint64_t dy = f2_sub(cy, *(const uint64_t*)&ay[i]);
            const uint64_t dz = f2_sub(cz, *(const uint64_t*)&az[i]);
            f2_dist2(dx, dy, dz, r0, r1);
            in0 = !(r0 > CUTOFF_SQ || r0 < MIN_R_SQ);
            in1 = i + 1 < nag && !(r1 > CUTOFF_SQ || r1 < MIN_R_SQ);
        }
        const unsigned m0 = __ballot_sync(0xffffffffu, in0), m1 = __ballot_sync(0xffffffffu, in1);
        const int n_step = __popc(m0) + __popc(m1);
        if (cnt + n_step > STAGE_CAP) terms_and_fold();
        const int at = cnt + __popc(m0 & lt) + __popc(m1 & lt);  // Calphas before base + 2 * lane
        if (in0) stage[at] = make_float4(r0, __int_as_float(i), 0.f, 0.f);
        if (in1) stage[at + (in0 ? 1 : 0)] = make_float4(r1, __int_as_float(i + 1), 0.f, 0.f);
        cnt += n_step;
    }
    terms_and_fold();
    return e;
}

// Slots of residue j as the sweep currently sees them: its proposal when accepted
// this sweep, its rejection rebuild when rejected, else the state.
__device__ __forceinline__ const float4* cur_slots(const AnSmem& S, int j) {
    const int s = S.sel[j];
    return (s == SEL_PROP ? S.prop : (s == SEL_REJ ? S.rej : S.pos)) + (size_t)j * SLOT_STRIDE;
}

// disulfide_energy (allatom.rs:155-180) over the SG atoms (topology atom 5 of Cys)
// in residue order.  SWEEP: residues take their slots from cur_slots and residue
// `sub` (>= 0) is taken from `sub_slots` with amino acid `sub_aa` instead; else
// every residue is read from the state.
template <class ACC, bool SWEEP>
__device__ ACC disulfide_of(const AnSmem& S, int n, int sub, const float4* sub_slots, int sub_aa) {
    ACC e = 0;
    for (int i = 0; i < n; ++i) {
        const int ai = (SWEEP && i == sub) ? sub_aa : S.aa[i];
        if (ai != CYS) continue;
        const float4 pi = (SWEEP ? (i == sub ? sub_slots : cur_slots(S, i)) : S.pos + (size_t)i * SLOT_STRIDE)[5];
        for (int j = i + 1; j < n; ++j) {
            const int aj = (SWEEP && j == sub) ? sub_aa : S.aa[j];
            if (aj != CYS) continue;
            const float4 pj = (SWEEP ? (j == sub ? sub_slots : cur_slots(S, j)) : S.pos + (size_t)j * SLOT_STRIDE)[5];
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
// Metropolis-Hastings with the log proposal ratio lhr = log q(reverse) - log q(forward):
// accept when u < exp(-dE/T + lhr).  lhr == 0 (uniform proposal) is exactly the
// Metropolis criterion above.
template <class ACC>
__device__ __forceinline__ bool mh_accept(ACC de, float temp, float u, double lhr) {
    if (lhr == 0.0) return metropolis(de, temp, u);
    const double a = -(double)de / (double)temp + lhr;
    return a >= 0.0 || (double)u < exp(a);
}

// ---- learned proposal -------------------------------------------------------------
// Features of the tile rows: row i = residue mvl[base + i]; the one-hot of its amino
// acid for a rotamer query, none for a mutation query (the network's mutation
// outputs then depend on the environment alone, the same before and after the
// move); one warp per row (8 rows, 8 warps).  ag_aa and the log1p table are the
// shared-memory copies when staged.
__device__ void an_tile_features(const AnSmem& S, const MlpTile& T, const int* rows_of, int base, int rows,
                                 const float4* agq, const uint8_t* ag_aa, int nag, const float* lg1p) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < MT_ROWS; i += AN_WARPS) {
        int* cnt = T.cnt + i * MLP_SHELLS * N_AA;
        __nv_bfloat16* x = T.x + i * MT_XS;
        if (i >= rows) {
            for (int j = lane; j < MLP_K1; j += 32) x[j] = __float2bfloat16_rn(0.0f);
            continue;
        }
        const int r = rows_of[base + i];
        for (int j = lane; j < MLP_SHELLS * N_AA; j += 32) cnt[j] = 0;
        __syncwarp();
        const float4 ca = S.pos[r * SLOT_STRIDE + 1];
        mlp_count_env(agq, ag_aa, nag, ca.x, ca.y, ca.z, cnt);
        __syncwarp();
        const int a = S.kind[r] == MV_MUT ? -1 : S.aa[r];
        for (int j = lane; j < MLP_K1; j += 32) {
            float v = 0.0f;
            if (j < N_AA) v = j == a ? 1.0f : 0.0f;
            else if (j < MLP_IN) v = lg1p[min(cnt[j - N_AA], MLP_COUNT_CAP)];
            x[j] = __float2bfloat16_rn(v);
        }
    }
}

// Choice among n options (n <= 32) with probabilities softmax(-y / tp), by one
// warp, lane k holding option k: FP64 weights w_k = exp((min y - y[k]) / tp) (the
// largest is 1) and the inverse CDF on u = dz / 2^32 over their prefix sums (for
// equal outputs exactly urange(dz, n): the prefix sums are then exact integers).
// inv_tp = 1 / tp.  Returns the option (all lanes).  Its log probability is never
// needed: a move's Hastings ratio is a difference of two logits of the same softmax.
__device__ int warp_sample(const float* y, int n, double inv_tp, uint32_t dz) {
    const int lane = threadIdx.x & 31;
    const float yl = lane < n ? y[lane] : INFINITY;
    float ymin = yl;
#pragma unroll
    for (int o = 16; o; o >>= 1) ymin = fminf(ymin, __shfl_xor_sync(0xffffffffu, ymin, o));
    double cum = lane < n ? exp(((double)ymin - (double)yl) * inv_tp) : 0.0;  // inclusive prefix sum in lane order
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double v = __shfl_up_sync(0xffffffffu, cum, o);
        if (lane >= o) cum += v;
    }
    const double total = __shfl_sync(0xffffffffu, cum, 31);
    const double target = (double)dz * (1.0 / 4294967296.0) * total;
    const unsigned hit = __ballot_sync(0xffffffffu, lane < n && target < cum);
    return hit ? __ffs(hit) - 1 : n - 1;
}

// The residue a move leaves: which = SEL_PROP builds the proposal, SEL_REJ the state
// after a rejection (rebuild_side_chain with the old chi, or mutate_residue back to
// the old amino acid around the same Calpha; allatom.rs:244-384).  The two kinds
// differ only in the backbone the side chain is built on (the current one, or the
// ideal one around the Calpha), so lanes of a warp building different kinds share
// the side-chain loop.
__device__ void build_move(const AnSmem& S, int r, int which) {
    const int oa = S.aa[r];
    const int kind = S.kind[r];
    const int na = kind == MV_MUT ? S.new_aa[r] : oa;
    const float4* cur = S.pos + (size_t)r * SLOT_STRIDE;
    float4* out = (which == SEL_PROP ? S.prop : S.rej) + (size_t)r * SLOT_STRIDE;
    const ChiTrig old_t = unpack_trig(S.trig[2 * r], S.trig[2 * r + 1]);
    const bool side_only = kind == MV_ROT || na == oa;  // side chain rebuilt on the current backbone
    F3 atoms[SLOTS];
    int a, n_bb;
    ChiTrig t = old_t;
    if (side_only) {
        a = oa;
        if (which == SEL_PROP) {
            if (kind == MV_ROT) t = rot_trig(oa, S.new_rot[r]);
            else t = s_rot_n[oa] > 0 ? rot_trig(oa, 0) : zero_trig();
        }
        n_bb = 4 + (oa != GLY ? 1 : 0);  // N, CA, C, O[, CB]
        for (int k = 0; k < n_bb; ++k) atoms[k] = f3(cur[k]);
    } else {
        // ideal backbone around the Calpha with the new (or, rejected, the old) residue
        a = which == SEL_PROP ? na : oa;
        if (which == SEL_PROP) t = s_rot_n[na] > 0 ? rot_trig(na, 0) : zero_trig();
        n_bb = ideal_backbone(f3(cur[1]), a, atoms);
    }
    build_side_chain(a, atoms, n_bb, t);
    const int n_at = s_topo_n[a];
    if (side_only) {
        for (int k = 0; k < SLOT_STRIDE; ++k)
            out[k] = (k >= n_bb && k < n_at) ? make_float4(atoms[k].x, atoms[k].y, atoms[k].z, 0.f) : cur[k];
    } else {
        store_residue(out, atoms, n_at);
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
// residues) moves, by the angle whose cosine and sine are ca, sa; allatom.rs:397-455.
__device__ void rotate_downstream(const AnSmem& S, int n, int r, bool phi, float ca, float sa) {
    const float4* rs = S.pos + (size_t)r * SLOT_STRIDE;
    const F3 a0 = f3(rs[phi ? 0 : 1]), a1 = f3(rs[phi ? 1 : 2]);
    const F3 axis = norm3(sub3(a1, a0));
    const F3 origin = a1;
    const int n_at_r = s_topo_n[S.aa[r]];
    for (int idx = threadIdx.x; idx < (n - r) * SLOT_STRIDE; idx += blockDim.x) {
        const int q = r + idx / SLOT_STRIDE, k = idx % SLOT_STRIDE;
        const bool mv = q == r ? (phi ? (k >= 2 && k < n_at_r) : k == 3) : k < s_topo_n[S.aa[q]];
        if (mv) {
            float4* p = S.pos + (size_t)q * SLOT_STRIDE + k;
            *p = rodrigues(*p, origin, axis, ca, sa);
        }
    }
}

// Coarse-grained force on residue r (compute_forces_with_grid, energy.rs:322-398) by
// its group of CG_LANES lanes (gl = lane in group, all lanes of the group call).
// Lane gl evaluates the consecutive probe cells [27 gl / 8, 27 (gl + 1) / 8) of the
// reference's (dx, dy, dz) order into its term slots; lane 0 then adds the terms
// lane by lane.  A lane with more in-cutoff terms than slots sends the residue to
// the one-lane walk (same sum).  Result valid in lane 0 of the group.
__device__ void group_cg_force(const AgView& A, const CgB& body, int gl, unsigned gmask, float4* my_terms,
                               int* my_count, const int* group_counts, const float4* group_terms, float& fx,
                               float& fy, float& fz) {
    const GridView& g = A.ca_grid;
    const int cx = cell_coord(body.x, g.inv), cy = cell_coord(body.y, g.inv), cz = cell_coord(body.z, g.inv);
    const float p[3] = {body.x, body.y, body.z};
    const int c[3] = {cx, cy, cz};
    // squared distance to the lower / own / upper slab per dimension (culling only;
    // the margin covers the f32 rounding of x*inv and of the slab bounds)
    float sl[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int o = 0; o < 3; ++o) {
            const float lo = (float)(c[d] + o - 1) * g.cell, hi = lo + g.cell;
            const float dd = fmaxf(fmaxf(lo - p[d], p[d] - hi), 0.0f);
            sl[d][o] = dd * dd;
        }
    const float reach = 10.001f + 4e-7f * (fabsf(body.x) + fabsf(body.y) + fabsf(body.z));
    const float reach2 = reach * reach;
    const int c_lo = (27 * gl) / CG_LANES, c_hi = (27 * (gl + 1)) / CG_LANES;
    int nt = 0;
    for (int ci = c_lo; ci < c_hi; ++ci) {
        const int dx = ci / 9 - 1, dy = (ci / 3) % 3 - 1, dz = ci % 3 - 1;
        if (sl[0][dx + 1] + sl[1][dy + 1] + sl[2][dz + 1] > reach2) continue;
        int a0, a1;
        if (!probe_cell(g, cx, cy, cz, dx, dy, dz, a0, a1)) continue;
        for (int i = a0; i < a1; ++i) {
            float tx, ty, tz;
            if (!cg_term_parts(body, A.ca_pq[i], A.ca_prm[i], tx, ty, tz)) continue;
            if (nt < CG_SLOTS) my_terms[nt] = make_float4(tx, ty, tz, 0.f);
            ++nt;
        }
    }
    *my_count = nt;
    const bool overflow = (__ballot_sync(gmask, nt > CG_SLOTS) & gmask) != 0u;
    __syncwarp(gmask);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    if (gl == 0) {
        if (!overflow) {
            for (int L = 0; L < CG_LANES; ++L) {
                const int cnt = group_counts[L];
                const float4* t = group_terms + L * CG_SLOTS;
                for (int k = 0; k < cnt; ++k) {
                    sx = xadd(sx, t[k].x);
                    sy = xadd(sy, t[k].y);
                    sz = xadd(sz, t[k].z);
                }
            }
        } else {
            cg_force(A, body, sx, sy, sz);
        }
    }
    fx = sx; fy = sy; fz = sz;
}

// compute_forces_with_grid for the residue of a group of GL lanes from its
// Verlet list (cg_list.cuh), kept in shared memory across the steps of the launch
// and rebuilt, with twice the skin up to CG_SKIN_MAX, when the Calpha leaves the
// skin of the list centre (a backbone move or the steps' drift).  The list entries
// passing the reference's tests, in list order, are the reference's pairs in its
// order: the group compacts them (at most CG_IN_MAX a round), its lanes evaluate the
// terms and lane 0 sums them in that order -- the sum of the 27-cell walk.  A list
// that overflows, or cells near the i32 limits, fall back to the one-lane walk.
// in / terms: the group's per-step scratch.  The force is in lane 0.
template <int GL>
__device__ void group_cg_force_list(const AgView& A, const CgB& body, int gl, unsigned gmask, int* list,
                                    float4* centre, int* nlp, int* in, float4* terms, float& fx, float& fy,
                                    float& fz) {
    static_assert(CG_IN_MAX % GL == 0, "a round compacts whole group steps");
    const GridView& g = A.ca_grid;
    const F3 ca = {body.x, body.y, body.z};
    float4 cc = *centre;
    int nl = *nlp;
    const float mx = ca.x - cc.x, my = ca.y - cc.y, mz = ca.z - cc.z;
    if (nl < 0 || !(mx * mx + my * my + mz * mz <= (cc.w - 0.01f) * (cc.w - 0.01f))) {
        const float skin = nl < 0 ? CG_SKIN : fminf(2.0f * cc.w, CG_SKIN_MAX);
        nl = build_cg_list<GL>(g, A.ca_pq, ca, gl, gmask, list, skin);
        cc = make_float4(ca.x, ca.y, ca.z, skin);
        __syncwarp(gmask);
        if (gl == 0) {
            *centre = cc;
            *nlp = nl;
        }
    }
    const int cx = cell_coord(ca.x, g.inv), cy = cell_coord(ca.y, g.inv), cz = cell_coord(ca.z, g.inv);
    float sx = 0.0f, sy = 0.0f, sz = 0.0f;
    if (nl > CG_LIST_MAX || cell_far(cx, cy, cz)) {
        if (gl == 0) cg_force(A, body, sx, sy, sz);
    } else {
        const bool near_adjacent = g.cell >= 10.0f && fabsf(ca.x) < 1e4f && fabsf(ca.y) < 1e4f &&
                                   fabsf(ca.z) < 1e4f;  // see k_langevin
        const int gshift = (int)(threadIdx.x & 31) & ~(GL - 1);
        const unsigned below = (1u << gl) - 1u;
        int from = 0;
        while (from < nl) {  // group-uniform
            int n_in = 0;
            while (from < nl && n_in + GL <= CG_IN_MAX) {
                const int j = from + gl;
                bool ok = false;
                int i = 0;
                if (j < nl) {
                    i = list[j];
                    const float4 a = A.ca_pq[i];
                    const float r_sq = xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z));
                    ok = !(r_sq > CUTOFF_SQ || r_sq < MIN_R_SQ);
                    if (ok && !(near_adjacent && r_sq <= CG_NEAR_SQ)) {  // the reference's cell test
                        const int4 ce = A.ca_cell[i];
                        ok = abs((long long)ce.x - cx) <= 1 && abs((long long)ce.y - cy) <= 1 &&
                             abs((long long)ce.z - cz) <= 1;
                    }
                }
                const unsigned m = (__ballot_sync(gmask, ok) >> gshift) & (GL == 32 ? ~0u : ((1u << GL) - 1u));
                if (ok) in[n_in + __popc(m & below)] = i;
                n_in += __popc(m);
                from += GL;
            }
            __syncwarp(gmask);
            for (int k = gl; k < n_in; k += GL) {
                const int i = in[k];
                float tx, ty, tz;
                cg_term_parts(body, A.ca_pq[i], A.ca_prm[i], tx, ty, tz);
                terms[k] = make_float4(tx, ty, tz, 0.f);
            }
            __syncwarp(gmask);
            if (gl == 0)
                for (int k = 0; k < n_in; ++k) {
                    const float4 t = terms[k];
                    sx = xadd(sx, t.x);
                    sy = xadd(sy, t.y);
                    sz = xadd(sz, t.z);
                }
            __syncwarp(gmask);  // the scratch is rewritten next round
        }
    }
    fx = sx;
    fy = sy;
    fz = sz;
}

// The network's choice of every mutation and (known-rotamer) rotamer move drawn
// this step and the moves' log Hastings ratios (all threads of the CTA call), one
// network pass per tile of moves.  A move changes neither the residue's environment
// nor its query (mutation: no amino-acid input; rotamer: the unchanged amino acid),
// so the reverse move's proposal is the same softmax: log q(reverse) - log q(move)
// = (y[move] - y[back]) / Tp, the normalisers cancelling.  The shared-memory
// layout is carved again from its base (smem, R, G, C) and the network comes by
// value: a reference to the kernel's copies would put them in local memory.  The
// biases are read from their shared-memory copies (staged by the kernel).
__device__ __noinline__ void an_learned_choices(unsigned char* smem, int R, int G, int C, int n, const float4* agq,
                                                const uint8_t* ag_aa, int nag, MlpDev mlp, float temp) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const AnSmem S = carve(smem, R, G, C, 1);
    mlp.b1 = S.mbias;  // the biases' shared-memory copies
    mlp.b2 = S.mbias + MLP_H;
    mlp.b3 = S.mbias + 2 * MLP_H;
    const MlpTile T = mlp_tile_carve((unsigned char*)S.terms);
    const double inv_tp = 1.0 / (double)fmaxf(temp, mlp.t_prop_min);
    uint4 w[MT_WREGS];
    mlp_tile_prefetch(mlp, w);  // the first weights are on their way during the features
    if (warp == 0) {  // mutations, and rotamer moves from a known library rotamer, in residue order
        int k = 0;
        for (int b = 0; b < n; b += 32) {
            const int r = b + lane;
            const int kind = r < n ? S.kind[r] : MV_NONE;
            const bool m = kind == MV_MUT || (kind == MV_ROT && S.rot[r] >= 0);
            const unsigned bal = __ballot_sync(0xffffffffu, m);
            if (m) S.mvl[k + __popc(bal & ((1u << lane) - 1u))] = r;
            k += __popc(bal);
        }
        if (lane == 0) S.iscal[IS_NMV] = k;
    }
    __syncthreads();
    const int n_mv = S.iscal[IS_NMV];
    for (int base = 0; base < n_mv; base += MT_ROWS) {
        const int rows = min(MT_ROWS, n_mv - base);
        if (base > 0) mlp_tile_prefetch(mlp, w);
        an_tile_features(S, T, S.mvl, base, rows, agq, ag_aa, nag, S.lg1p);
        __syncthreads();
        mlp_tile_forward(mlp, T, w, rows);
        for (int i = warp; i < rows; i += AN_WARPS) {  // one warp per row
            const int r = S.mvl[base + i];
            const bool rot = S.kind[r] == MV_ROT;
            // rotamer query: outputs 20 + j over the residue's rotamers; mutation: outputs 0..19
            const float* y = T.y + i * MT_YS + (rot ? N_AA : 0);
            const int k = warp_sample(y, rot ? s_rot_n[S.aa[r]] : N_AA, inv_tp, S.dz[r]);
            if (lane == 0) {
                const int back = rot ? S.rot[r] : S.aa[r];  // the reverse move's option
                if (rot) S.new_rot[r] = k;
                else S.new_aa[r] = k;
                S.lhr[r] = ((double)y[k] - (double)y[back]) * inv_tp;
            }
        }
        __syncthreads();
    }
}

// EXT: the learned proposal and the proposal log are compiled in (a separate
// instance, so the plain kernel carries none of their registers).
// FV: one chain of each Fv candidate (fv_chain_step, diffusion.rs:560-698): the
// resident state interleaves heavy (2i) and light (2i + 1) chains, this launch steps
// chains 2 * blockIdx.x + fv_chain against the antigen and the other chain of the pair
// as it is in the state; Calpha energies gain the partner chain's contribution, the
// force its compute_forces term, and the mutation / rotamer moves follow the CDR
// flags fv_cdr (per residue) instead of the interface mask.  Draw streams + 4 * chain.
template <class ACC, bool EXT, bool FV, int W>
__global__ void __launch_bounds__(W * 32, W == 8 ? 2 : 1) k_anneal(StateView st, const AgView* __restrict__ ags, StepParams p,
                                                       int n_steps, uint32_t step0, int with_noise,
                                                       const float* __restrict__ temps, int R, int G, int C,
                                                       uint32_t* __restrict__ err, long long* __restrict__ stats,
                                                       MlpDev mlp, int learned, MlpTuple* __restrict__ tlog,
                                                       unsigned long long* __restrict__ log_n, long long log_cap,
                                                       int fv_chain, const uint8_t* __restrict__ fv_cdr) {
    static_assert(W == AN_WARPS || (W == 2 * AN_WARPS && !EXT), "8 warps, or 16 without the network");
    constexpr int NT = W * 32;  // threads of the CTA
    extern __shared__ __align__(16) unsigned char an_smem[];
    const AnSmem S = carve(an_smem, R, G, C, learned, FV ? 1 : 0, W);
    const int c = FV ? 2 * (int)blockIdx.x + fv_chain : (int)blockIdx.x;
    const uint32_t sh = FV ? 4u * (uint32_t)fv_chain : 0u;  // draw stream offset of the chain
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = st.cand_res_off[c];
    const int n = st.cand_res_off[c + 1] - r0;
    if (n <= 0 || n > R) return;
    const uint32_t cid = st.cand_id[c];
    if (tid == 0) *S.ag = ags[st.cand_ag[c]];
    __syncthreads();
    const AgView& A = *S.ag;
    const int nag = A.n_res;
    const bool staged = nag <= G;
    const int ncell = A.ca_grid.nx * A.ca_grid.ny * A.ca_grid.nz + 1;
    const bool cells_staged = staged && ncell <= C;
    for (int i = tid; staged && i < nag; i += NT) {
        const float4 q = A.ca_atom[i];
        S.agq[i] = q;
        S.agp[i] = A.ca_atom_prm[i];
        S.cgq[i] = A.ca_pq[i];
        S.cgp[i] = A.ca_prm[i];
        S.agx[i] = q.x;
        S.agy[i] = q.y;
        S.agz[i] = q.z;
    }
    if (tid == 0 && staged && (nag & 1)) S.agx[nag] = S.agy[nag] = S.agz[nag] = 1e30f;
    for (int i = tid; cells_staged && i < ncell; i += NT) S.cgcell[i] = A.ca_grid.cell_start[i];
    if (EXT && learned) {  // the network's features and epilogues read these every step
        for (int i = tid; staged && i < nag; i += NT) S.agaa[i] = A.res_aa[i];
        for (int i = tid; i <= MLP_COUNT_CAP; i += NT) S.lg1p[i] = g_an_log1p[i];
        for (int i = tid; i < MLP_BIASES; i += NT)
            S.mbias[i] = i < MLP_H ? mlp.b1[i] : i < 2 * MLP_H ? mlp.b2[i - MLP_H] : mlp.b3[i - 2 * MLP_H];
    }
    __syncthreads();
    if (tid == 0 && cells_staged) {  // the CG probe reads the staged copies through the view
        S.ag->ca_pq = S.cgq;
        S.ag->ca_prm = S.cgp;
        S.ag->ca_grid.cell_start = S.cgcell;
    }
    const float4* agq = staged ? S.agq : A.ca_atom;
    const float4* agp = staged ? S.agp : A.ca_atom_prm;
    float4* stage = S.stage + warp * STAGE_CAP;
    // Fv: the partner chain's Calphas (it does not move during this launch)
    int np = 0;
    if (FV) {
        const int pc = c ^ 1, p0 = st.cand_res_off[pc];
        np = min(st.cand_res_off[pc + 1] - p0, R);
        for (int i = tid; i < np; i += NT) {
            const float4 v = st.res_pos[(size_t)(p0 + i) * SLOT_STRIDE + 1];
            const int a = st.res_aa[p0 + i];
            const float4 q = s_ca_atom[a], rl = s_res[a];
            S.ptq[i] = make_float4(v.x, v.y, v.z, q.x);
            S.ptp[i] = make_float4(q.y, q.z, q.w, (float)s_ca_type[a]);
            S.pcq[i] = make_float4(v.x, v.y, v.z, rl.x);
            S.pcp[i] = make_float4(rl.y, rl.z, rl.w, 0.f);
        }
        __syncthreads();
    }
    // residue_contribution_allatom of a Calpha at q with amino acid a, by the warp (the
    // scans are noinline: one copy each instead of one per call site, less code to fetch);
    // Fv: plus the contribution against the partner chain (fv_residue_contribution,
    // diffusion.rs:551-553)
    auto ca_energy = [&](F3 q, int a) -> ACC {
        ACC e = staged ? warp_contribution_pairs<ACC>(S.agx, S.agy, S.agz, agq, agp, nag, q, a, stage)
                       : warp_contribution<ACC>(agq, agp, nag, q, a, stage);
        if (FV) e = e + warp_contribution<ACC>(S.ptq, S.ptp, np, q, a, stage);
        return e;
    };

    for (int i = tid; i < n * SLOT_STRIDE; i += NT) S.pos[i] = st.res_pos[(size_t)r0 * SLOT_STRIDE + i];
    for (int r = tid; r < n; r += NT) {
        const int a = st.res_aa[r0 + r];
        const float4 chi = st.res_chi[r0 + r];
        S.aa[r] = a;
        S.chi[r] = chi;
        S.trig[2 * r] = st.res_trig[2 * (r0 + r)];
        S.trig[2 * r + 1] = st.res_trig[2 * (r0 + r) + 1];
        if (EXT) {
            // rotamer index of the state: the library entry whose chi it holds, else -1
            int k = -1;
            for (int q = 0; q < s_rot_n[a] && k < 0; ++q) {
                const float4 t = s_rot_chi[a][q];
                if (t.x == chi.x && t.y == chi.y && t.z == chi.z && t.w == chi.w) k = q;
            }
            S.rot[r] = k;
            S.lhr[r] = 0.0;
        }
    }
    const bool lists = anneal_list_res(R) > 0;  // Verlet lists of the Langevin force
    for (int r = tid; lists && r < n; r += NT) S.cgnl[r] = -1;
    long long n_mc = 0, n_mc_acc = 0, n_bb = 0, n_bb_acc = 0;
    __syncthreads();

    for (int s = 0; s < n_steps; ++s) {
        const uint32_t step = step0 + (uint32_t)s;
        const float temp = temps ? temps[s] : p.t_hot;
        // ---- 1. Langevin (diffusion.rs:306-339): CG_LANES lanes per residue, LW with
        // Verlet lists (16 in the 16-warp instance: the list scans and terms take half
        // the rounds; the sum in list order by the group's lane 0 is the same) ----
        {
            constexpr int LW = W == 2 * AN_WARPS ? 2 * CG_LANES : CG_LANES;
            const int glanes = lists ? LW : CG_LANES;
            const int gl = tid % glanes;
            const unsigned gmask = ((1u << glanes) - 1u) << (lane & ~(glanes - 1));
            const int g0 = tid - gl;  // first thread of the group
            // the first CG_RES_PER_PASS groups (whole warps; with 16 warps and 8-lane
            // groups the others wait at the barrier below)
            for (int base = 0; tid < CG_RES_PER_PASS * glanes && base < n; base += CG_RES_PER_PASS) {
                const int r = base + tid / glanes;
                if (lists) {
                    // lists the residues' Calphas outran: rebuilt by the whole warp, one
                    // residue after another (a one-pass build with 32 lanes instead of a
                    // two-pass build with the group's 8 lanes)
                    bool need = false;
                    F3 ca = {0.f, 0.f, 0.f};
                    float skin = CG_SKIN;
                    if (gl == 0 && r < n) {
                        ca = f3(S.pos[r * SLOT_STRIDE + 1]);
                        const float4 cc = S.cgcentre[r];
                        const int nl = S.cgnl[r];
                        const float mx = ca.x - cc.x, my = ca.y - cc.y, mz = ca.z - cc.z;
                        need = nl < 0 || !(mx * mx + my * my + mz * mz <= (cc.w - 0.01f) * (cc.w - 0.01f));
                        skin = nl < 0 ? CG_SKIN : fminf(2.0f * cc.w, CG_SKIN_MAX);
                    }
                    for (unsigned m = __ballot_sync(0xffffffffu, need); m; m &= m - 1) {
                        const int q = __ffs(m) - 1;
                        const int rq = __shfl_sync(0xffffffffu, r, q);
                        const F3 cq = {__shfl_sync(0xffffffffu, ca.x, q), __shfl_sync(0xffffffffu, ca.y, q),
                                       __shfl_sync(0xffffffffu, ca.z, q)};
                        const float sq = __shfl_sync(0xffffffffu, skin, q);
                        const int nl = build_cg_list_warp<int>(A.ca_grid, A.ca_pq, cq, lane,
                                                               S.cglist + (size_t)rq * CG_LIST_MAX, sq);
                        if (lane == q) {
                            S.cgcentre[rq] = make_float4(cq.x, cq.y, cq.z, sq);
                            S.cgnl[rq] = nl;
                        }
                    }
                    __syncwarp();
                }
                if (r >= n) continue;  // whole groups leave together
                const F3 ca = f3(S.pos[r * SLOT_STRIDE + 1]);
                if (gl == 0 && err && (!isfinite(ca.x) || !isfinite(ca.y) || !isfinite(ca.z))) atomicOr(err, ERRF_NAN);
                const CgB body = cg_body(ca.x, ca.y, ca.z, S.aa[r]);
                float fx, fy, fz;
                if (lists) {
                    // the group's scratch: the term slots of CG_LANES lanes
                    unsigned char* scratch =
                        (unsigned char*)(S.terms + (size_t)(tid / glanes) * CG_LANES * CG_SLOTS);
                    group_cg_force_list<LW>(A, body, gl, gmask, S.cglist + (size_t)r * CG_LIST_MAX,
                                            S.cgcentre + r, S.cgnl + r, (int*)(scratch + CG_IN_MAX * 16),
                                            (float4*)scratch, fx, fy, fz);
                } else {
                    group_cg_force(A, body, gl, gmask, S.terms + (size_t)tid * CG_SLOTS, S.tcount + tid,
                                   S.tcount + g0, S.terms + (size_t)g0 * CG_SLOTS, fx, fy, fz);
                }
                if (gl == 0) {
                    if (FV) {  // VH-VL packing force: compute_forces over the partner's Calphas
                        float px = 0.0f, py = 0.0f, pz = 0.0f;
                        for (int i = 0; i < np; ++i) cg_term(body, S.pcq[i], S.pcp[i], px, py, pz);
                        fx = xadd(fx, px);
                        fy = xadd(fy, py);
                        fz = xadd(fz, pz);
                    }
                    const float dx_c = xsub(ca.x, A.cx), dy_c = xsub(ca.y, A.cy), dz_c = xsub(ca.z, A.cz);
                    const float d = fmaxf(xsqrt(xdist2(dx_c, dy_c, dz_c)), 0.001f);
                    const float f_r = xdiv(xmul(-p.restraint_k, xsub(d, p.shell_radius)), d);
                    fx = xadd(fx, xmul(f_r, dx_c));
                    fy = xadd(fy, xmul(f_r, dy_c));
                    fz = xadd(fz, xmul(f_r, dz_c));
                    float nx = 0.f, ny = 0.f, nz = 0.f;
                    if (with_noise) {
                        const float sigma = xmul(p.noise_base, xsqrt(temp));
                        const U4 u = rng_draw(p.seed, cid, step, STREAM_NOISE + sh, (uint32_t)r);
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
                __syncwarp(gmask);  // the group's term slots are reused by the next pass
            }
        }
        if (tid == 0) {
            S.iscal[IS_DVALID] = 0;  // disulfide energy stale
            S.iscal[IS_NCYS] = 0;
            S.iscal[IS_LASTCYS] = -1;
            S.iscal[IS_NTASK] = 0;
        }
        __syncthreads();
        for (int i = tid; i < n * SLOT_STRIDE; i += NT) {
            const int r = i / SLOT_STRIDE, k = i % SLOT_STRIDE;
            if (k < s_topo_n[S.aa[r]]) {
                const float4 d = S.ldelta[r];
                float4 v = S.pos[i];
                v.x = xadd(v.x, d.x); v.y = xadd(v.y, d.y); v.z = xadd(v.z, d.z);
                S.pos[i] = v;
            }
        }
        __syncthreads();

        // ---- 2. interface mask (diffusion.rs:343-351; Fv: CDR flags instead) + move draws ----
        for (int r = warp; !FV && r < n; r += W) {
            const F3 ca = f3(S.pos[r * SLOT_STRIDE + 1]);
            bool hit = false;
            for (int base = 0; base < nag && !hit; base += 64) {
                bool h = false;
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int i = base + u * 32 + lane;
                    if (i < nag) {
                        const float4 a = agq[i];
                        h |= xdist2(xsub(ca.x, a.x), xsub(ca.y, a.y), xsub(ca.z, a.z)) < p.iface_cutoff_sq;
                    }
                }
                hit = __any_sync(0xffffffffu, h);
            }
            if (lane == 0) S.iface[r] = hit;
        }
        for (int r = tid; r < n; r += NT) {
            const U4 d = rng_draw(p.seed, cid, step, STREAM_BACKBONE + sh, (uint32_t)r);
            const bool att = u01(d.x) < p.backbone_move_p;
            S.bb_att[r] = att;
            if (att) {
                const float delta = xmul(frange(d.y, -p.max_torsion_deg, p.max_torsion_deg), RADS_PER_DEG);
                S.bb_trig[r] = make_float4(mc_cos(delta), mc_sin(delta), mc_cos(-delta), mc_sin(-delta));
            }
            S.bb_phi[r] = (int)((d.z >> 31) & 1u);
            S.bb_u[r] = u01(d.w);
            S.sel[r] = SEL_KEEP;
        }
        __syncthreads();

        // ---- 3. mutation / rotamer proposals (diffusion.rs:354-399) ----
        for (int r = tid; r < n; r += NT) {
            const U4 d = rng_draw(p.seed, cid, step, STREAM_MC + sh, (uint32_t)r);
            const int aa = S.aa[r];
            int kind = MV_NONE;
            if (FV) {
                // CDR positions: mutation / rotamer moves (MUTATION_P * 3, ROTAMER_MOVE_P * 2);
                // every residue without one: rotamer relaxation (ROTAMER_MOVE_P * 0.3)
                if (fv_cdr[r0 + r] && u01(d.x) < xmul(p.mutation_p, 3.0f)) {
                    if (u01(d.y) < xmul(p.rotamer_move_p, 2.0f)) {
                        if (s_rot_n[aa] > 0) kind = MV_ROT;
                    } else {
                        kind = MV_MUT;
                    }
                } else if (u01(d.y) < xmul(p.rotamer_move_p, 0.3f) && s_rot_n[aa] > 0) {
                    kind = MV_ROT;
                }
                if (kind == MV_ROT) {
                    S.new_rot[r] = (int)urange(d.z, (uint32_t)s_rot_n[aa]);
                    S.new_aa[r] = aa;
                } else if (kind == MV_MUT) {
                    S.new_aa[r] = (int)urange(d.z, (uint32_t)N_AA);
                    S.new_rot[r] = 0;
                }
            }
            const bool itf = !FV && S.iface[r] != 0;
            const float eff_mut_p = itf ? xmul(p.mutation_p, 3.0f) : xmul(p.mutation_p, 0.4f);
            const float eff_rot_p = itf ? xmul(p.rotamer_move_p, 2.0f) : p.rotamer_move_p;
            if (!FV && u01(d.x) < eff_mut_p) {
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
            if (EXT) {
                S.dz[r] = d.z;
                S.lhr[r] = 0.0;
            }
            if (aa == CYS) atomicAdd(&S.iscal[IS_NCYS], 1);
            if (kind != MV_NONE) {  // its two energy tasks (in any order: each writes its own results)
                const int k = atomicAdd(&S.iscal[IS_NTASK], 2);
                S.tcount[k] = 2 * r;  // the Langevin step's term counts are free until the next step
                S.tcount[k + 1] = 2 * r + 1;
            }
        }
        __syncthreads();
        // learned proposal: the choice of each drawn move comes from the network
        // (same draw d.z, inverse CDF) and the move carries its Hastings ratio
        if (EXT && learned && temp <= mlp.t_max)
            an_learned_choices(an_smem, R, G, C, n, agq, staged ? S.agaa : A.res_aa, nag, mlp, temp);
        // proposals and rejection rebuilds on the upper half of the warps (two threads per
        // residue), the Calpha energies before / after each move on the lower half, the
        // listed tasks dealt one per warp in turn
        if (warp >= W / 2) {
            for (int t = tid - NT / 2; t < 2 * n; t += NT / 2) {
                const int r = t >> 1;
                if (S.kind[r] != MV_NONE) build_move(S, r, (t & 1) ? SEL_REJ : SEL_PROP);
            }
        } else {
            const int ntask = S.iscal[IS_NTASK];
            for (int k = warp; k < ntask; k += W / 2) {
                const int t = S.tcount[k];
                const int r = t >> 1, which = t & 1;
                const int kind = S.kind[r];
                const bool same = kind == MV_ROT || S.new_aa[r] == S.aa[r];
                if (which == 1 && same) continue;  // same Calpha, same amino acid: same energy
                const int a = which ? S.new_aa[r] : S.aa[r];
                const ACC e = ca_energy(f3(S.pos[r * SLOT_STRIDE + 1]), a);
                if (lane == 0) {
                    if (which == 0) {
                        S.c_old[r] = (double)e;
                        if (same) S.c_new[r] = (double)e;
                    } else {
                        S.c_new[r] = (double)e;
                    }
                }
            }
        }
        __syncthreads();
        // the sweep's decisions, in residue order; moves without a Cys are deferred to
        // the parallel pass below, except while the proposal log is written (its
        // records keep residue order within a candidate)
        const bool defer = !EXT || !tlog;
        if (tid == 0) {
            int ncys = S.iscal[IS_NCYS];
            bool have_d = false;
            ACC D = 0;
            for (int r = 0; r < n; ++r) {
                const int kind = S.kind[r];
                if (kind == MV_NONE) continue;
                if (!have_d) {
                    D = ncys >= 2 ? disulfide_of<ACC, true>(S, n, -1, nullptr, 0) : (ACC)0;
                    have_d = true;
                }
                const int oa = S.aa[r];
                const int na = kind == MV_MUT ? S.new_aa[r] : oa;
                const bool cys = oa == CYS || na == CYS;
                if (defer && !cys) {  // decided in parallel below, with the disulfide energy of its turn
                    S.d_turn[r] = (double)D;
                    continue;
                }
                const int ncys_new = ncys + (na == CYS) - (oa == CYS);
                ACC Dn = D;
                if (cys)
                    Dn = ncys_new >= 2 ? disulfide_of<ACC, true>(S, n, r, S.prop + (size_t)r * SLOT_STRIDE, na)
                                       : (ACC)0;
                const ACC old_e = (ACC)S.c_old[r] + D;
                const ACC new_e = (ACC)S.c_new[r] + Dn;
                const double lhr = EXT ? S.lhr[r] : 0.0;
                const bool acc = EXT ? mh_accept(new_e - old_e, temp, S.u_acc[r], lhr)
                                     : metropolis(new_e - old_e, temp, S.u_acc[r]);
                ++n_mc;
                n_mc_acc += acc;
                if (EXT && tlog) {
                    const unsigned long long slot = atomicAdd(log_n, 1ull);
                    if ((long long)slot < log_cap) {
                        const float4 ca = S.pos[r * SLOT_STRIDE + 1];
                        MlpTuple t;
                        t.x = ca.x; t.y = ca.y; t.z = ca.z;
                        t.delta_e = (float)(new_e - old_e);
                        t.cand = c;
                        t.log_ratio = (float)lhr;
                        t.residue = (int16_t)r;
                        t.aa = (uint8_t)oa;
                        t.action = (uint8_t)(kind == MV_MUT ? na : N_AA + S.new_rot[r]);
                        t.antigen = (uint8_t)st.cand_ag[c];
                        t.accepted = acc ? 1 : 0;
                        t.pad[0] = t.pad[1] = 0;
                        tlog[slot] = t;
                    }
                }
                if (acc) {
                    if (EXT) S.rot[r] = kind == MV_ROT ? S.new_rot[r] : (s_rot_n[na] > 0 ? 0 : -1);
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
                    ncys = ncys_new;
                } else {
                    S.sel[r] = SEL_REJ;
                    S.c_cur[r] = S.c_old[r];
                    if (oa == CYS && ncys >= 2) D = disulfide_of<ACC, true>(S, n, -1, nullptr, 0);  // SG rebuilt
                }
                S.valid[r] = 1;
            }
            if (have_d) {
                S.dscal[0] = (double)D;
                S.iscal[IS_DVALID] = 1;
            }
        }
        __syncthreads();
        if (defer) {
            // the moves that involve no Cys leave the disulfide energy as it is, so each
            // is decided on its own with the disulfide energy current at its turn (the
            // loop above recorded it): the same decisions as the sequential sweep
            for (int r = tid; r < n; r += NT) {
                const int kind = S.kind[r];
                if (kind == MV_NONE || S.valid[r]) continue;  // valid: decided above (Cys)
                const int oa = S.aa[r];
                const int na = kind == MV_MUT ? S.new_aa[r] : oa;
                const ACC D = (ACC)S.d_turn[r];
                const ACC old_e = (ACC)S.c_old[r] + D;
                const ACC new_e = (ACC)S.c_new[r] + D;
                const bool acc = EXT ? mh_accept(new_e - old_e, temp, S.u_acc[r], S.lhr[r])
                                     : metropolis(new_e - old_e, temp, S.u_acc[r]);
                ++n_mc;
                n_mc_acc += acc;
                if (acc) {
                    if (EXT) S.rot[r] = kind == MV_ROT ? S.new_rot[r] : (s_rot_n[na] > 0 ? 0 : -1);
                    S.sel[r] = SEL_PROP;
                    S.aa[r] = na;
                    const int rot = S.new_rot[r];
                    const bool has = s_rot_n[na] > 0;
                    S.chi[r] = has ? s_rot_chi[na][rot] : make_float4(0.f, 0.f, 0.f, 0.f);
                    const ChiTrig t = has ? rot_trig(na, rot) : zero_trig();
                    S.trig[2 * r] = make_float4(t.t[0].x, t.t[0].y, t.t[1].x, t.t[1].y);
                    S.trig[2 * r + 1] = make_float4(t.t[2].x, t.t[2].y, t.t[3].x, t.t[3].y);
                    S.c_cur[r] = S.c_new[r];
                } else {
                    S.sel[r] = SEL_REJ;
                    S.c_cur[r] = S.c_old[r];
                }
                S.valid[r] = 1;
            }
            __syncthreads();
        }
        for (int i = tid; i < n * SLOT_STRIDE; i += NT) {
            const int r = i / SLOT_STRIDE;
            const int sl = S.sel[r];
            if (sl == SEL_PROP) S.pos[i] = S.prop[i];
            else if (sl == SEL_REJ) S.pos[i] = S.rej[i];
            if ((i % SLOT_STRIDE) == 0 && S.aa[r] == CYS) atomicMax(&S.iscal[IS_LASTCYS], r);
        }
        __syncthreads();

        // ---- 4. backbone phi/psi moves (diffusion.rs:403-418) ----
        const int last_cys = S.iscal[IS_LASTCYS];
        for (int r = 0; r < n; ++r) {
            if (!S.bb_att[r]) continue;
            const bool phi = S.bb_phi[r] != 0;
            const bool cys_down = r <= last_cys;  // a Cys at or after r: the disulfide term can change
            // Calpha energies of residues r..n at the current positions, and the
            // disulfide energy
            if (tid == 0 && !S.iscal[IS_DVALID]) {
                S.dscal[0] = (double)disulfide_of<ACC, false>(S, n, -1, nullptr, 0);
                S.iscal[IS_DVALID] = 1;
            }
            for (int i = r + warp; i < n; i += W) {
                if (S.valid[i]) continue;
                const ACC e = ca_energy(f3(S.pos[i * SLOT_STRIDE + 1]), S.aa[i]);
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
            const float4 bt = S.bb_trig[r];
            rotate_downstream(S, n, r, phi, bt.x, bt.y);
            __syncthreads();
            for (int i = r + 1 + warp; i < n; i += W) {
                const ACC e = ca_energy(f3(S.pos[i * SLOT_STRIDE + 1]), S.aa[i]);
                if (lane == 0) S.c_new[i] = (double)e;
            }
            __syncthreads();
            if (tid == 0) {
                const ACC Dn = cys_down ? disulfide_of<ACC, false>(S, n, -1, nullptr, 0) : (ACC)S.dscal[0];
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
                    if (cys_down) S.iscal[IS_DVALID] = 0;
                }
                S.iscal[IS_DECISION] = acc;
            }
            __syncthreads();
            if (!S.iscal[IS_DECISION]) {
                rotate_downstream(S, n, r, phi, bt.z, bt.w);
                __syncthreads();
            }
        }
    }

    for (int i = tid; i < n * SLOT_STRIDE; i += NT) st.res_pos[(size_t)r0 * SLOT_STRIDE + i] = S.pos[i];
    for (int r = tid; r < n; r += NT) {
        st.res_aa[r0 + r] = (uint8_t)S.aa[r];
        st.res_chi[r0 + r] = S.chi[r];
        st.res_trig[2 * (r0 + r)] = S.trig[2 * r];
        st.res_trig[2 * (r0 + r) + 1] = S.trig[2 * r + 1];
    }
    if (stats && (n_mc || n_bb)) {  // the decisions are spread over the threads
        atomicAdd((unsigned long long*)&stats[4 * c], (unsigned long long)n_mc);
        atomicAdd((unsigned long long*)&stats[4 * c + 1], (unsigned long long)n_mc_acc);
        atomicAdd((unsigned long long*)&stats[4 * c + 2], (unsigned long long)n_bb);
        atomicAdd((unsigned long long*)&stats[4 * c + 3], (unsigned long long)n_bb_acc);
    }
}

// The Metropolis energy of every resident candidate, the energy whose changes
// decide the mutation / rotamer / backbone moves: the sum over its residues of
// residue_contribution_allatom (diffusion.rs:425-463) plus disulfide_energy
// (allatom.rs:155-180), f32 terms summed in double in residue order (the default
// accumulation of k_anneal).  One CTA per candidate, one warp per residue.
__global__ void __launch_bounds__(AN_THREADS) k_mc_energy(StateView st, const AgView* __restrict__ ags,
                                                          double* __restrict__ out) {
    __shared__ float4 s_stage[AN_WARPS * STAGE_CAP];
    __shared__ double s_e[AN_THREADS];
    __shared__ double s_total;
    const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int r0 = st.cand_res_off[c], n = st.cand_res_off[c + 1] - r0;
    const AgView& A = ags[st.cand_ag[c]];
    if (tid == 0) s_total = 0.0;
    for (int base = 0; base < n; base += AN_THREADS) {
        const int m = min(AN_THREADS, n - base);
        for (int i = warp; i < m; i += AN_WARPS) {
            const int r = r0 + base + i;
            const double e = warp_contribution<double>(A.ca_atom, A.ca_atom_prm, A.n_res,
                                                       f3(st.res_pos[(size_t)r * SLOT_STRIDE + 1]), st.res_aa[r],
                                                       s_stage + warp * STAGE_CAP);
            if (lane == 0) s_e[i] = e;
        }
        __syncthreads();
        if (tid == 0)
            for (int i = 0; i < m; ++i) s_total += s_e[i];
        __syncthreads();
    }
    if (tid == 0) {
        double d = 0.0;
        for (int i = 0; i < n; ++i) {
            if (st.res_aa[r0 + i] != CYS) continue;
            const float4 pi = st.res_pos[(size_t)(r0 + i) * SLOT_STRIDE + 5];
            for (int j = i + 1; j < n; ++j) {
                if (st.res_aa[r0 + j] != CYS) continue;
                const float4 pj = st.res_pos[(size_t)(r0 + j) * SLOT_STRIDE + 5];
                const float dd = xsqrt(xdist2(xsub(pi.x, pj.x), xsub(pi.y, pj.y), xsub(pi.z, pj.z)));
                if (dd > 4.0f) continue;
                const float z = xdiv(xsub(dd, 2.05f), 0.4f);
                d -= (double)xmul(4.0f, mc_exp(xmul(xmul(-0.5f, z), z)));
            }
        }
        out[c] = s_total + d;
    }
}

void launch_mc_energy(cudaStream_t s, const StateView& st, const AgView* ags, double* out) {
    if (st.n_cand > 0) k_mc_energy<<<st.n_cand, AN_THREADS, 0, s>>>(st, ags, out);
}

size_t anneal_smem(int max_res, int max_ag_res, int max_cells, int learned) {
    const int G = max_ag_res <= AG_STAGE_MAX ? max_ag_res : 0;
    return anneal_smem_bytes(max_res, G, G && max_cells <= CELL_STAGE_MAX ? max_cells : 0, learned);
}

cudaError_t launch_anneal(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          uint32_t step0, int with_noise, const float* temps, int accumulate, int max_res,
                          int max_ag_res, int max_cells, uint32_t* err, long long* stats, const AnnealExtras& x,
                          int fv_chain, const uint8_t* fv_cdr) {
    if (st.n_cand <= 0 || n_steps <= 0 || max_res <= 0) return cudaSuccess;
    const int G = max_ag_res <= AG_STAGE_MAX ? max_ag_res : 0;
    const int C = G && max_cells <= CELL_STAGE_MAX ? max_cells : 0;
    const bool fv = fv_chain >= 0;
    const int learned = x.learned && !fv ? 1 : 0;
    const size_t smem = anneal_smem_bytes(max_res, G, C, learned, fv ? 1 : 0);
    const bool ext = !fv && (x.learned || x.log);
    const int grid = fv ? st.n_cand / 2 : st.n_cand;
    if (grid <= 0) return cudaSuccess;
    // a grid that leaves SMs idle (the 64 survivors of phase 2) takes 16 warps per
    // candidate: the per-residue passes (Calpha energies, builds, backbone moves) need
    // fewer rounds; the network path keeps 8
    int sms = 148;
    {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const bool wide = !ext && grid <= sms;
    const size_t smem16 = anneal_smem_bytes(max_res, G, C, learned, fv ? 1 : 0, 2 * AN_WARPS);
    auto run = [&](auto kern, int warps) -> cudaError_t {
        const size_t sm = warps == AN_WARPS ? smem : smem16;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        if (e) return e;
        kern<<<grid, warps * 32, sm, s>>>(st, ags, p, n_steps, step0, with_noise, temps, max_res, G, C, err, stats,
                                          x.mlp, learned, x.log, x.log_n, x.log_cap, fv ? fv_chain : 0, fv_cdr);
        return cudaSuccess;
    };
    constexpr int W8 = AN_WARPS, W16 = 2 * AN_WARPS;
    cudaError_t e;
    if (fv) {
        if (accumulate == 1) e = wide ? run(k_anneal<float, false, true, W16>, W16) : run(k_anneal<float, false, true, W8>, W8);
        else e = wide ? run(k_anneal<double, false, true, W16>, W16) : run(k_anneal<double, false, true, W8>, W8);
    } else if (ext) {
        e = accumulate == 1 ? run(k_anneal<float, true, false, W8>, W8) : run(k_anneal<double, true, false, W8>, W8);
    } else if (accumulate == 1) {
        e = wide ? run(k_anneal<float, false, false, W16>, W16) : run(k_anneal<float, false, false, W8>, W8);
    } else {
        e = wide ? run(k_anneal<double, false, false, W16>, W16) : run(k_anneal<double, false, false, W8>, W8);
    }
    if (e) return e;
    return cudaGetLastError();
}

}  // namespace binder
