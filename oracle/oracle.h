/*
 * oracle.h — CPU restatement of the reference's all-atom scoring + search path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA library in
 * de-novo-antigen-binder_b200/: tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg are the only code allowed to load it.  Nothing in the product
 * path links or calls it.
 *
 * Reference (Rust crate DilaDeniz/de-novo-antigen-binder, no Rust toolchain here):
 *   src/amber.rs      force-field tables            (transcribed in oracle_tables.inc)
 *   src/rotamer.rs    rotamer library + NERF        (orc_place_atom, orc_build_residues)
 *   src/allatom.rs    AtomProtein edits             (mutate / rotamer / phi / psi / disulfide)
 *   src/spatial.rs    SpatialHashGrid               (orc_grid_*)
 *   src/energy.rs     pair energies and CG forces   (orc_energy_*, orc_forces_cg_*)
 *   shaders/energy.wgsl + src/gpu.rs score_batch    (orc_score_batch_*)
 *   src/diffusion.rs  allatom_diffusion_step, run_allatom (orc_step, orc_block, orc_run)
 *
 * Two arithmetic variants:
 *   *32  — f32 in the reference's own operation order (no FMA contraction; built
 *          with -ffp-contract=off), i.e. what the Rust code computes.
 *   *64  — the same formulas re-evaluated in f64 from the same f32 inputs; the
 *          accuracy target for the GPU's compensated / FP64-reduced sums.
 *
 * Parity pinning: the reference has no golden energy vectors.  The tables are
 * pinned to the reference source text (tests/golden/reference_tables.json, parsed
 * by tests/golden/gen_reference_tables.py) and the functions to the reference's
 * own unit tests (tests/golden/reference_kats.json); energies beyond those are
 * cross-checked against an independent numpy restatement (tests/golden/).
 *
 * Candidate exchange format ("slot layout"): a protein of n residues is
 *   aa[n] (u8, AminoAcid order of atom.rs:4-25), chi[n*4] (degrees),
 *   pos[n*14*3] (slot k of residue r = topology atom k of amber.rs; unused = 0).
 */
#ifndef BINDER_ORACLE_H
#define BINDER_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SLOTS 14

/* ---- tables -------------------------------------------------------------- */
int orc_topology_size(int aa);                               /* atoms of residue aa */
int orc_topology_atom(int aa, int k, float* charge, int* type, int* hydrophobic);
void orc_amber_nb(int type, float* r_min_half, float* epsilon);
int orc_hbond_flags(int type);                               /* bit0 donor, bit1 acceptor */
void orc_eef1(int type, float* dg_ref, float* vol, float* lambda);
int orc_rotamer_count(int aa);
void orc_rotamer(int aa, int idx, float chi[4], float* prob);
int orc_sidechain_def_count(int aa);
void orc_sidechain_def(int aa, int k, int ref[3], float* bond, float* angle, float* dih_fixed, int* chi_idx);
void orc_residue_level(int aa, float* charge, float* eps, float* sigma, int* hydrophobic);

/* ---- geometry (rotamer.rs / allatom.rs) ---------------------------------- */
void orc_place_atom(const float a[3], const float b[3], const float c[3],
                    float bond, float angle_deg, float dihedral_deg, float out[3]);
/* protein_from_ca_trace (allatom.rs:523-541): chi_or_null = NULL -> top rotamer */
void orc_build_residues(int n, const float* ca_xyz, const uint8_t* aa, const float* chi_or_null,
                        float* out_pos /*n*14*3*/, float* out_chi /*n*4, may be NULL*/);
/* flatten slot layout to the AtomCloud of push_residue (allatom.rs:201-240) */
int orc_flatten(int n, const uint8_t* aa, const float* pos,
                float* x, float* y, float* z, float* q, float* rmh, float* eps,
                uint8_t* hyd, uint8_t* type, uint32_t* resi);
/* ca_center_of_mass (allatom.rs:183-195) */
void orc_ca_center(int n, const float* pos, float out[3]);

/* ---- SpatialHashGrid (spatial.rs) ---------------------------------------- */
void orc_grid_cell(float cell, float x, float y, float z, int32_t out[3]);
/* 27-cell probe for every query point; returns total count or -1 if cap too small */
int64_t orc_grid_neighbors(float cell, const float* ax, const float* ay, const float* az, int64_t n_ag,
                           const float* px, const float* py, const float* pz, int64_t n_q,
                           int64_t* out_offsets, uint32_t* out_idx, int64_t cap);

/* ---- coarse-grained forces (energy.rs:154-234, 322-398) ------------------- */
/* residue clouds: x,y,z + amino acid (ResidueCloud::push, atom.rs:221-231) */
void orc_forces_cg_brute(const float* ax, const float* ay, const float* az, const uint8_t* aaa, int n_ag,
                         const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                         float* fx, float* fy, float* fz);
void orc_forces_cg_grid(float cell,
                        const float* ax, const float* ay, const float* az, const uint8_t* aaa, int n_ag,
                        const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                        float* fx, float* fy, float* fz);
/* same in f64 (for the relative-tolerance gate of the force kernel) */
void orc_forces_cg64(float cell, int use_grid,
                     const float* ax, const float* ay, const float* az, const uint8_t* aaa, int n_ag,
                     const float* bx, const float* by, const float* bz, const uint8_t* baa, int n_ab,
                     double* fx, double* fy, double* fz);

/* ---- all-atom energies (energy.rs:261-314, solvation.rs:34-84) ------------ */
/* clouds are SoA: x,y,z,q,rmh,eps,hyd(u8),type(u8); out[5] = lj,coul,hydro,hbond,solv */
typedef struct orc_cloud {
    const float *x, *y, *z, *q, *rmh, *eps;
    const uint8_t *hyd, *type;
    int64_t n;
} orc_cloud;
void orc_energy_atoms32(const orc_cloud* ag, const orc_cloud* ab, float out[5]);
/* f64: out[5] as above, out_abs[5] = sum of |pair term| per component */
void orc_energy_atoms64(const orc_cloud* ag, const orc_cloud* ab, double out[5], double out_abs[5]);

/* ---- score_batch (gpu.rs:166-267 / energy.wgsl) --------------------------- */
/* GpuAtom = 8 floats {x,y,z,q,r_min_half,epsilon,hydrophobic,_pad}.
   offsets: n_cand+1 atom offsets into cand (ragged); out = LJ+Coulomb+hydrophobic */
void orc_score_batch32(const float* ag, int64_t n_ag, const float* cand, const int64_t* offsets,
                       int64_t n_cand, float* out, int n_threads);
void orc_score_batch64(const float* ag, int64_t n_ag, const float* cand, const int64_t* offsets,
                       int64_t n_cand, double* out, double* out_abs, int n_threads);
/* all-atom force on each candidate atom (f64), -grad of the LJ+Coulomb score */
void orc_forces_allatom64(const float* ag, int64_t n_ag, const float* cand, const int64_t* offsets,
                          int64_t n_cand, double* out_f /*3 per cand atom*/, double* out_e, int n_threads);
/* count pairs with 0.25 <= r2 <= 100 (the pair-evals of one scoring) */
int64_t orc_count_pairs(const float* ag, int64_t n_ag, const float* cand, int64_t n_cand_atoms, int n_threads);

/* ---- Philox4x32-10 (Salmon et al., SC'11) --------------------------------- */
void orc_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* ---- search step (diffusion.rs) ------------------------------------------- */
typedef struct orc_params {
    float step, noise_base, t_hot, t_cold, mutation_p, rotamer_move_p, backbone_move_p,
          max_torsion_deg, iface_cutoff_sq, shell_radius, max_disp, restraint_k, ca_cell;
    /* Metropolis energies: 0 = f32 pair terms summed in double (the CUDA default),
       1 = the reference's f32 sums */
    int32_t accumulate;
    uint64_t seed;
} orc_params;
void orc_default_params(orc_params* p);
float orc_temperature(int iter, int total);     /* diffusion.rs:102-104 */

/* Antigen (slot layout), with its Calpha cloud + grid, held by the oracle */
typedef struct orc_antigen orc_antigen;
orc_antigen* orc_antigen_new(int n_res, const uint8_t* aa, const float* pos, float ca_cell);
void orc_antigen_free(orc_antigen*);
void orc_antigen_center(const orc_antigen*, float out[3]);

/* residue_contribution_allatom (diffusion.rs:425-463), ref f32 order */
float orc_residue_contribution(const orc_antigen*, int n_res, const uint8_t* aa, const float* pos, int r);
/* the same f32 terms summed in double (the GPU's default Metropolis accumulation) */
double orc_residue_contribution64(const orc_antigen*, int n_res, const uint8_t* aa, const float* pos, int r);
/* disulfide_energy (allatom.rs:155-180) */
float orc_disulfide(int n_res, const uint8_t* aa, const float* pos);

/* One allatom_diffusion_step (diffusion.rs:290-419) on a batch of candidates.
   State in slot layout, updated in place: aa[n_cand*n_res], chi[...*4], pos[...*14*3].
   cand_id: Philox counter word 0 per candidate; step_id: counter word 1.
   with_noise / with_mc select the reference's two uses (phase 1 gradient-only,
   phase 2 Langevin + MC).  stats (optional, 4 per cand): mut tried/acc, bb tried/acc. */
void orc_step(const orc_antigen*, const orc_params*, int n_cand, int n_res,
              uint8_t* aa, float* chi, float* pos, const uint32_t* cand_id, uint32_t step_id,
              float temp, int with_noise, int with_mc, int64_t* stats, int n_threads);

/* score every candidate (slot layout) against the antigen with the all-atom
   LJ+Coulomb+hydrophobic (+ hbond + EEF1 + disulfide if full) energy, f64
   accumulation; out_abs (may be NULL) = the sum of |pair term| of the same terms */
void orc_score_slots64(const orc_antigen*, int n_cand, int n_res, const uint8_t* aa, const float* pos,
                       int full, double* out, double* out_abs, int n_threads);

/* minimize (diffusion.rs:854-916) of every candidate against the antigen: steps of
   Calpha-grid steepest descent with side-chain rebuilds, each kept only when
   allatom_energy drops (acc64 = 0: the reference's f32 energy; 1: its f64
   re-evaluation).  In place; out_energy = final energies; out_margin (may be
   NULL) = the smallest |e - best| / max(|best|, 1) met by a keep / restore decision. */
void orc_minimize(const orc_antigen*, int n_cand, int n_res, uint8_t* aa, float* chi, float* pos, int steps,
                  int acc64, double* out_energy, double* out_margin, int n_threads);
/* affinity_maturation_allatom (diffusion.rs:924-961) over each candidate's
   interface residues (filters.rs:96-105).  In place; out_energy = final scores,
   out_mutated (may be NULL) = mutations kept per candidate, out_margin (may be NULL)
   as for orc_minimize. */
void orc_affinity_maturation(const orc_antigen*, int n_cand, int n_res, uint8_t* aa, float* chi, float* pos,
                             int acc64, double* out_energy, int32_t* out_mutated, double* out_margin,
                             int n_threads);

/* ValidationReport::assess (validate.rs:24-132): clash_score and ramachandran_outliers
   of one slot-layout protein */
void orc_validate(int n_res, const uint8_t* aa, const float* pos, int32_t* clashes, int32_t* rama);

/* ---- Fv two-chain engine (diffusion.rs:477-827) ----
   The run_fv iteration loop (diffusion.rs:791-812) of every candidate: heavy chain
   (n_h residues, cdr_h[r] != 0 for CDR positions) and light chain stepped in turn by
   fv_chain_step against the antigen and the other chain, elitist on fv_energy
   (acc64: its f64 re-evaluation); the Metropolis sums follow prm->accumulate.
   Chains in place (the best pair); out_energy = the best fv_energy. */
void orc_fv_run(const orc_antigen*, const orc_params* prm, int n_cand, int n_h, int n_l, uint8_t* aa_h,
                float* chi_h, float* pos_h, const uint8_t* cdr_h, uint8_t* aa_l, float* chi_l, float* pos_l,
                const uint8_t* cdr_l, const uint32_t* cand_id, int iterations, float target_radius, int acc64,
                double* out_energy, double* out_margin, int n_threads);
/* fv_energy (diffusion.rs:541-547) of one heavy / light pair */
double orc_fv_energy(const orc_antigen*, int n_h, const uint8_t* aa_h, const float* pos_h, int n_l,
                     const uint8_t* aa_l, const float* pos_l, int acc64);

/* stable ascending sort of energies, NaN last; first k indices (diffusion.rs:1045-1047) */
void orc_topk(const double* e, int64_t n, int64_t k, int32_t* out_idx);

#ifdef __cplusplus
}
#endif
#endif
