/*
 * binder_gpu.h — C ABI of the B200 (sm_100a) all-atom scoring + search library
 * (libbinder_b200.so).
 *
 * This is the drop-in boundary for the hot path of the reference antibody
 * design engine (Rust crate DilaDeniz/de-novo-antigen-binder).  The reference has
 * no FFI; each entry point below names the Rust item it replaces (file:line in
 * the reference project) so that a Rust caller can bind it with `extern "C"`
 * declarations and keep its call sites unchanged.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Host buffers are caller-owned and only
 *     borrowed for the duration of a call; device memory is owned by the context.
 *   - Every entry point returns a binder_status (0 = BINDER_OK).  Nothing throws
 *     or aborts across the ABI; binder_last_error() describes the last failure.
 *   - One context = one device + one CUDA stream.  Calls on one context are
 *     serialised on that stream and the context is not thread-safe; separate
 *     contexts are independent.
 *   - There is no CPU fallback: a context whose device or kernels are missing
 *     fails binder_create() with BINDER_ERR_NODEVICE / BINDER_ERR_CUDA.
 *   - Candidate proteins use the "slot layout": residue r of a protein owns 14
 *     atom slots; slot k holds topology atom k of the residue's amino acid in the
 *     order of the reference's residue tables (amber.rs:126-351), i.e. the order
 *     AtomProtein::push_residue appends them (allatom.rs:201-240).  Unused slots
 *     are zero.  Positions are float[n_res][14][3]; chi angles float[n_res][4] in
 *     degrees; amino acids uint8 in AminoAcid order (atom.rs:4-25).
 */
#ifndef BINDER_GPU_H
#define BINDER_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BINDER_ABI_VERSION 2
#define BINDER_MAX_SLOTS 14

enum binder_status {
    BINDER_OK = 0,
    BINDER_ERR_ARG = 1,       /* invalid argument (NULL, size, amino acid out of range) */
    BINDER_ERR_CUDA = 2,      /* CUDA runtime error (launch, copy) */
    BINDER_ERR_OOM = 3,       /* device or host allocation failed */
    BINDER_ERR_TIMEOUT = 4,   /* a bounded device wait gave up */
    BINDER_ERR_NAN = 5,       /* non-finite coordinate in an input */
    BINDER_ERR_GRID = 6,      /* spatial grid box too large for the cell size */
    BINDER_ERR_STATE = 7,     /* call out of order (e.g. no antigen / no candidates) */
    BINDER_ERR_NODEVICE = 8,  /* no usable sm_100 device */
    BINDER_ERR_CAPACITY = 9,  /* output buffer too small; required size reported */
    BINDER_ERR_IO = 10        /* a file could not be read */
};

typedef struct binder_ctx binder_ctx;

/* GpuAtom (gpu.rs:17-29): 8 x f32 = 32 bytes, layout identical to the Rust
   #[repr(C)] struct and to the reference shader's storage buffer. */
typedef struct binder_gpu_atom {
    float x, y, z, q, r_min_half, epsilon, hydrophobic, _pad;
} binder_gpu_atom;

/* AtomCloud (allatom.rs:17-31), borrowed structure-of-arrays. */
typedef struct binder_atom_cloud {
    const float* x;
    const float* y;
    const float* z;
    const float* charge;
    const float* r_min_half;
    const float* epsilon;
    const uint8_t* hydrophobic;  /* 1 = hydrophobic */
    const uint8_t* atom_type;    /* AtomType (amber.rs:13-30); may be NULL for scoring */
    const uint32_t* residue_idx; /* may be NULL */
    size_t n;
} binder_atom_cloud;

/* ResidueCloud (atom.rs:185-195): positions + amino acid.  charge, epsilon,
   sigma and hydrophobic are derived from amino_acid as ResidueCloud::push does
   (atom.rs:221-231). */
typedef struct binder_residue_cloud {
    const float* x;
    const float* y;
    const float* z;
    const uint8_t* amino_acid;
    size_t n;
} binder_residue_cloud;

/* Search hyper-parameters.  Defaults = the reference constants
   (diffusion.rs:65-83, energy.rs:13-27, spatial grid cell diffusion.rs:1003). */
typedef struct binder_params {
    float step;             /* STEP 0.08 */
    float noise_base;       /* NOISE_BASE 0.25 */
    float t_hot;            /* T_HOT 3.0 */
    float t_cold;           /* T_COLD 0.02 */
    float mutation_p;       /* MUTATION_P 0.08 */
    float rotamer_move_p;   /* ROTAMER_MOVE_P 0.12 */
    float backbone_move_p;  /* BACKBONE_MOVE_P 0.04 */
    float max_torsion_deg;  /* MAX_TORSION_DEG 15 */
    float iface_cutoff_sq;  /* IFACE_CUTOFF_SQ 64 */
    float shell_radius;     /* restraint radius, INIT_RADIUS 20 */
    float max_disp;         /* MAX_DISP 2.0 */
    float restraint_k;      /* RESTRAINT_K 0.02 */
    float ca_cell;          /* Calpha grid cell for the CG force, 10 A */
    float score_cell;       /* all-atom grid cell for scoring, 8 A */
    int32_t accumulate;     /* BINDER_ACC_KAHAN (default) or BINDER_ACC_F32 */
    int32_t flags;          /* BINDER_FLAG_* (default BINDER_FLAG_GRAPH) */
    uint64_t seed;          /* Philox key for every stochastic move */
} binder_params;

#define BINDER_ACC_KAHAN 0  /* f32 pair terms, compensated per-lane sums, FP64 cross-lane/block reduction */
#define BINDER_ACC_F32 1    /* f32 pair terms, plain f32 per-lane sums, FP64 cross-lane/block reduction */
/* binder_block replays a CUDA graph of its launches (captured on first use,
   re-captured when the state, parameters or launch shapes change) */
#define BINDER_FLAG_GRAPH 1
/* the first binder_block on a new state shape runs binder_autotune */
#define BINDER_FLAG_AUTOTUNE 2

/* ---- force-field tables compiled into the library (amber.rs, rotamer.rs) ----
   Residue aa: its atom count and per-slot partial charge, AMBER type and
   hydrophobic flag (amber.rs:126-378).  Arrays have 14 entries. */
int binder_table_residue(int aa, int* n_atoms, float* charge, uint8_t* atom_type, uint8_t* hydrophobic);
/* AMBER type: r_min_half, epsilon (amber.rs:46-63), H-bond flags bit0 donor /
   bit1 acceptor (amber.rs:72-84), EEF1 dg_ref, vol, lambda (amber.rs:414-431). */
int binder_table_atom_type(int type, float* r_min_half, float* epsilon, int* hbond_flags, float* eef1);
/* rotamers(aa) (rotamer.rs:468): count and chi tuples float[5][4]. */
int binder_table_rotamers(int aa, int* n, float* chi);
/* residue-level charge, epsilon, sigma, hydrophobic (atom.rs:55-104). */
int binder_table_residue_level(int aa, float* out4);

/* ---- context --------------------------------------------------------------- */
int binder_abi_version(void);
const char* binder_status_string(int status);
void binder_default_params(binder_params* out);
/* GpuContext::try_init (gpu.rs:55-155).  params NULL = defaults.  Returns NULL
   and sets *status when no sm_100 device is usable (the reference returns None). */
binder_ctx* binder_create(int device, const binder_params* params, int* status);
void binder_destroy(binder_ctx* ctx);
int binder_set_params(binder_ctx* ctx, const binder_params* params);
const char* binder_last_error(const binder_ctx* ctx);
int binder_synchronize(binder_ctx* ctx);
/* number of kernels this context has launched (instrumentation for benchmarks) */
uint64_t binder_launch_count(const binder_ctx* ctx);

/* ---- score_batch: GpuContext::score_batch (gpu.rs:166-267) --------------------
   energies[c] = AMBER LJ + Coulomb + hydrophobic energy of candidate c against
   the antigen (energy.wgsl:67-94; the LJ/Coulomb/hydrophobic part of
   interaction_energy_atoms_breakdown, energy.rs:261-314).  candidates is the
   flat n_cand*n_ab GpuAtom array; n_cand = n_atoms / n_ab, 0 when n_ab == 0
   (gpu.rs:172-174).  *out_n_cand receives n_cand; out_cap must be >= n_cand.
   The antigen is uploaded and its spatial grid rebuilt only when its contents
   change between calls. */
int binder_score_batch(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                       size_t n_atoms, size_t n_ab, float* out_energies, size_t out_cap, size_t* out_n_cand);
/* same, FP64 energies; out_abs (may be NULL) = sum of |pair term| per candidate */
int binder_score_batch_f64(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                           size_t n_atoms, size_t n_ab, double* out_energies, double* out_abs, size_t out_cap,
                           size_t* out_n_cand);
/* ragged candidates: candidate c is atoms [offsets[c], offsets[c+1]).  Lifts the
   reference's uniform-n_ab restriction (gpu.rs:163). */
int binder_score_batch_ragged(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                              const int64_t* offsets, size_t n_cand, double* out_energies, double* out_abs);
/* make `antigen` the context's resident antigen 0 (upload + grid build) */
int binder_set_antigen_atoms(binder_ctx* ctx, const binder_atom_cloud* antigen);
/* count of (candidate atom, antigen atom) pairs with 0.25 <= r^2 <= 100 among the
   last ragged/uniform batch scored (pair-evals of one scoring) */
int binder_last_pair_count(binder_ctx* ctx, int64_t* out_pairs);

/* ---- SpatialHashGrid (spatial.rs:12-67) --------------------------------------
   Cell of each point: floor(coord * (1/cell)) with the f32 reciprocal
   (spatial.rs:26,61-67).  out_cells = int32[3n]. */
int binder_grid_cells(binder_ctx* ctx, float cell, const float* x, const float* y, const float* z, size_t n,
                      int32_t* out_cells);
/* build(x,y,z) (spatial.rs:31-39) over the n_ag points, then query_neighbors
   (spatial.rs:44-58) for each of the n_q probe points: the candidate indices of
   probe q are out_idx[out_offsets[q] .. out_offsets[q+1]), in the reference's
   callback order (cells dx, dy, dz in -1..1, atoms ascending within a cell).
   Returns BINDER_ERR_CAPACITY with *out_total set when cap is too small. */
int binder_grid_neighbors(binder_ctx* ctx, float cell, const float* ax, const float* ay, const float* az,
                          size_t n_ag, const float* px, const float* py, const float* pz, size_t n_q,
                          int64_t* out_offsets, uint32_t* out_idx, size_t cap, size_t* out_total);

/* No counterpart in the reference.  binder_grid_neighbors for callers that
   cannot allocate device memory: hosts that own all device memory through their
   own pool or arena and cannot let a library call cudaMalloc/cudaFree, or loops
   where an allocation would stall the device.  Inputs (antigen points, probe
   points) and outputs (offsets int64[n_q+1], indices uint32[cap]) are device
   buffers owned by the caller; the kernels' scratch lives in one fixed-size
   device array inside the library (about 4.3 MB, held on every GPU that loads
   the library until the process exits).  No context is needed; work is enqueued
   on `stream` (a cudaStream_t, 0 = legacy default stream) and the call returns
   once the neighbour-list fill is enqueued.  Results equal binder_grid_neighbors.
   Limits: n_ag <= BINDER_NOALLOC_MAX_ATOMS (else BINDER_ERR_ARG) and the box of
   occupied cells <= BINDER_NOALLOC_MAX_CELLS (else BINDER_ERR_GRID);
   BINDER_ERR_CAPACITY with *out_total set when cap is too small.  Every call
   shares the scratch array: calls whose GPU work overlaps (different streams or
   threads) race.  The work runs on the current device, so `stream` must belong
   to it.  The first call on a device looks the array up on that device (make it
   before any stream capture) and keeps the address for the life of the process:
   after cudaDeviceReset on a device, do not call this entry point on it again.
   Each call waits on `stream` twice, to read back the occupied cell box and the
   neighbour count.  A CUDA error left pending by earlier work of the process is
   reported as BINDER_ERR_CUDA before anything is enqueued, and left pending.  */
#define BINDER_NOALLOC_MAX_ATOMS 65536
#define BINDER_NOALLOC_MAX_CELLS 262144
int binder_grid_neighbors_noalloc(float cell, const float* d_ax, const float* d_ay, const float* d_az,
                                  size_t n_ag, const float* d_px, const float* d_py, const float* d_pz,
                                  size_t n_q, int64_t* d_out_offsets, uint32_t* d_out_idx, size_t cap,
                                  size_t* out_total, void* stream);

/* ---- forces ------------------------------------------------------------------
   compute_forces_with_grid (energy.rs:322-398): coarse-grained (Calpha) force on
   every antibody residue from the antigen residues found by the 27-cell probe of
   a grid with the given cell (the reference uses 10 A).  Bit-exact with the
   reference's f32 operation order. */
int binder_compute_forces_with_grid(binder_ctx* ctx, const binder_residue_cloud* antigen, float cell,
                                    const binder_residue_cloud* antibody, float* fx, float* fy, float* fz);
/* All-atom AMBER force (no reference counterpart): -grad of the score's LJ +
   Coulomb terms on every candidate atom, plus each candidate's energy.
   out_force = float[3 * n_atoms]. */
int binder_forces_allatom(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                          const int64_t* offsets, size_t n_cand, float* out_force, double* out_energies);

/* ---- survivor selection (diffusion.rs:1042-1057) ------------------------------
   Indices of the k lowest energies in stable ascending order (ties keep index
   order; NaN sorts after every number). */
int binder_topk(binder_ctx* ctx, const double* energies, size_t n, size_t k, int32_t* out_idx);
/* independent top-k per segment [seg_offsets[s], seg_offsets[s+1]); out_idx is
   int32[n_seg * k] of global indices, -1 where a segment has fewer than k. */
int binder_topk_segmented(binder_ctx* ctx, const double* energies, const int64_t* seg_offsets, size_t n_seg,
                          size_t k, int32_t* out_idx);

/* ---- residue construction (rotamer.rs:198-232, 439-462; allatom.rs:502-541) ---
   protein_from_ca_trace: ideal backbone around each Calpha and side chain placed
   by NERF at the given chi (NULL = the top rotamer of each amino acid).
   out_pos = float[n][14][3], out_chi = float[n][4] (may be NULL). */
int binder_build_residues(binder_ctx* ctx, size_t n, const float* ca_xyz, const uint8_t* aa, const float* chi,
                          float* out_pos, float* out_chi);

/* ---- resident search state ---------------------------------------------------
   The antigen protein (slot layout) for the search.  Uploads its atoms, builds
   the all-atom grid (params.score_cell), its Calpha cloud + grid (params.ca_cell)
   and ca_center_of_mass (allatom.rs:183-195).  Returns the antigen id (>= 0) in
   *out_id; several antigens may be resident (batched workloads). */
int binder_add_antigen(binder_ctx* ctx, size_t n_res, const uint8_t* aa, const float* pos, int32_t* out_id);
int binder_clear_antigens(binder_ctx* ctx);
/* Upload n_cand candidates into device state.  n_res[c] residues each (NULL +
   uniform_n_res for a uniform population), concatenated in candidate order;
   antigen_id[c] (NULL = all 0).  cand_id[c] is the Philox counter word of the
   candidate (NULL = c). */
int binder_state_upload(binder_ctx* ctx, size_t n_cand, const int32_t* n_res, int32_t uniform_n_res,
                        const int32_t* antigen_id, const uint32_t* cand_id, const uint8_t* aa, const float* chi,
                        const float* pos);
/* Copy the device state back (same layout as the upload). */
int binder_state_download(binder_ctx* ctx, uint8_t* aa, float* chi, float* pos);
/* n_steps allatom_diffusion_step's (diffusion.rs:290-419) on every resident
   candidate: CG force + restraint + clamp (+ noise when with_noise) (+ rotamer /
   mutation / backbone Metropolis moves when with_mc).  step0 = Philox counter of
   the first step; temps = per-step temperatures (NULL = t_hot).  With with_mc the
   Metropolis energies follow params.accumulate: BINDER_ACC_F32 = the reference's
   f32 sums, otherwise the same f32 pair terms summed in double and an FP64
   acceptance test.  with_mc holds at most 128 residues per candidate. */
int binder_diffuse(binder_ctx* ctx, int n_steps, uint32_t step0, int with_noise, int with_mc, const float* temps);
/* Metropolis move counts since the upload, int64[n_cand][4]: mutation/rotamer
   tried, accepted, backbone tried, accepted (no reference counterpart).
   reset != 0 zeroes them after the copy. */
int binder_mc_stats(binder_ctx* ctx, int64_t* out, int reset);
/* Keep candidates idx[0..n) of the resident state, in that order (survivor
   selection, diffusion.rs:1044-1057: the kept AtomProteins move into a new Vec). */
int binder_state_select(binder_ctx* ctx, const int32_t* idx, size_t n);
/* Resident candidate count, residue count and, per candidate, its index in the
   last binder_state_upload (orig_idx int32[n_cand], may be NULL). */
int binder_state_info(binder_ctx* ctx, int32_t* n_cand, int32_t* total_res, int32_t* orig_idx);
/* Score every resident candidate against its antigen: LJ + Coulomb + hydrophobic
   (full = 0), allatom_energy (diffusion.rs:281-283: + H-bond + EEF1 +
   disulfide, full = 1), or the Metropolis energy whose changes decide the moves
   (full = 2: the sum over residues of residue_contribution_allatom,
   diffusion.rs:425-463, plus disulfide_energy, f32 terms summed in double).
   out = double[n_cand] (host). */
int binder_score_state(binder_ctx* ctx, int full, double* out_energies);
/* The phase-1 block: n_steps gradient-only steps, one score of every candidate,
   then the k lowest per antigen (diffusion.rs:1018-1057 with scoring every
   n_steps).  out_energies double[n_cand], out_topk int32[n_antigen * k].  When
   both are NULL the block is only enqueued on the context stream (no host
   synchronisation); binder_block_fetch then returns the results of the last
   block and reports any device error. */
int binder_block(binder_ctx* ctx, int n_steps, uint32_t step0, int k, double* out_energies, int32_t* out_topk);
int binder_block_fetch(binder_ctx* ctx, double* out_energies, int32_t* out_topk);
/* One search block on a population that lives in host memory (no reference
   counterpart; the host side of diffusion.rs:1018-1057 when the caller keeps the
   population): binder_state_upload of (n_cand, n_res, uniform_n_res, antigen_id,
   cand_id, aa, chi, pos), binder_block(n_steps, 0, k, out_energies, out_topk),
   then the moved residues written back into aa, chi and pos -- the same results as
   the three calls, with the write-back copied on a second stream while the
   candidates are scored.  Pinned host arrays give the copies full speed. */
int binder_block_io(binder_ctx* ctx, size_t n_cand, const int32_t* n_res, int32_t uniform_n_res,
                    const int32_t* antigen_id, const uint32_t* cand_id, uint8_t* aa, float* chi, float* pos,
                    int n_steps, int k, double* out_energies, int32_t* out_topk);

/* ---- launch shapes and the autotuner (no reference counterpart) ----------------
   Results never depend on these: every residue is computed by the same lanes with
   the same arithmetic whatever the grid. */
typedef struct binder_launch_cfg {
    int32_t score_warps;        /* warps per CTA of the persistent scoring kernel: 4, 8, 16 */
    int32_t score_ctas_per_sm;  /* persistent scoring CTAs per SM: 1..32 */
    int32_t cg_warps;           /* warps per CTA of the gradient-step kernel: 2, 4, 8 */
    int32_t cg_lanes;           /* lanes per residue of the gradient-step kernel: 4 (with 2 or 4
                                   warps per CTA) or 8 */
    int32_t cg_order;           /* residue order of the gradient-step kernel: 0 by Calpha cell,
                                   1 candidate after candidate, 2 strided (work spread out),
                                   3 (flat form) tasks balanced by the work of the previous
                                   launch (Verlet-list lengths, rebuilds): each launch leaves its
                                   residues in work bands for the next, which deals them to its
                                   tasks heaviest first; no extra launch */
    int32_t score_order;        /* work-queue order of the scoring kernel: 0 by Calpha cell (three
                                   sorting launches after every move), 1 residue index */
    int32_t cg_queue;           /* gradient-step kernel: 0 one CTA per residue batch, 1 persistent
                                   CTAs whose warps take residue batches from a work queue */
    int32_t cg_flat;            /* gradient-step kernel: 0 the lane-group form (cg_lanes lanes per
                                   residue); 4, 8, 16 or 32 the flat form with that many residues
                                   per warp (the warp scans their concatenated lists together; 32
                                   with 4 warps per CTA, 4, 8 and 16 with 4 or 8) */
} binder_launch_cfg;
int binder_get_launch_cfg(binder_ctx* ctx, binder_launch_cfg* out);
int binder_set_launch_cfg(binder_ctx* ctx, const binder_launch_cfg* cfg);
/* Time every launch shape on the resident state (median of reps runs each; the
   gradient steps run on a copy of the positions, which are put back), keep the
   fastest and remember it per state shape (candidate / residue counts, antigen
   sizes, SM count).  With the environment variable BINDER_TUNE_CACHE naming a
   file, choices are read from and appended to it.  out may be NULL. */
int binder_autotune(binder_ctx* ctx, int reps, binder_launch_cfg* out);

/* run_allatom (diffusion.rs:983-1107) on the resident state: phase 1 runs
   phase1_steps steps on every candidate in blocks of score_every (score + the
   survivors lowest per antigen after each block), keeps the last block's
   survivors, runs phase2_steps Langevin + Metropolis steps on them, scores them
   with allatom_energy and ranks them (stable, ascending).  out_cand[a * top_n + j]
   = index (in the last upload) of antigen a's j-th best candidate, -1 past the
   end; out_energy likewise (NaN past the end).  Afterwards the resident state
   holds the ranked results, in that order.  Philox step counters: phase 1 uses
   0..phase1_steps-1, phase 2 continues from phase1_steps. */
typedef struct binder_run_cfg {
    int32_t phase1_steps;  /* GPU_STEPS 200 (diffusion.rs:1018) */
    int32_t score_every;   /* steps per scored block, 10; <= 0 = one block */
    int32_t survivors;     /* per antigen, population 64 (diffusion.rs:1047) */
    int32_t phase2_steps;  /* cpu_iterations, 600 */
    int32_t top_n;         /* results per antigen (diffusion.rs:1098) */
    int32_t phase1_mc;     /* 1 = Metropolis moves in phase 1 too, as the reference's
                              loop runs them (diffusion.rs:1023); 0 = gradient only */
} binder_run_cfg;
void binder_default_run_cfg(binder_run_cfg* cfg);
int binder_run_allatom(binder_ctx* ctx, const binder_run_cfg* cfg, int32_t* out_cand, double* out_energy);

/* ---- post-search refinement of the results (main.rs:336-346) ------------------------
   minimize (diffusion.rs:854-916) of every resident candidate against its antigen
   (the one partner, main.rs:338): `steps` steps of steepest descent on the
   Calpha-level grid force (compute_forces_with_grid, energy.rs:322-398) with the
   step size 0.04 * (1 - step / steps), each component clamped to 0.5 A, every
   residue translated and its side chain rebuilt at its chi (allatom.rs:244-293),
   a step kept only when allatom_energy (diffusion.rs:281-283) drops.  In place;
   out_energy double[n_cand] (may be NULL) = each candidate's final energy. */
int binder_minimize(binder_ctx* ctx, int steps, double* out_energy);
/* affinity_maturation_allatom (diffusion.rs:924-961) of every resident candidate
   over its interface residues (Calpha within 8 A of an antigen Calpha,
   filters.rs:96-105, main.rs:342-344): at each such position, in order, the other
   amino acids in AminoAcid order are tried at their top rotamer and the first that
   lowers allatom_energy is kept; otherwise the residue is rebuilt with its old
   amino acid and chi (mutate_residue, allatom.rs:299-384).  In place (at most 128
   residues per candidate); out_energy (may be NULL) = the final score as the
   reference returns it, out_mutated int32[n_cand] (may be NULL) = mutations kept. */
int binder_affinity_maturation(binder_ctx* ctx, double* out_energy, int32_t* out_mutated);

/* ---- Fv two-chain engine (diffusion.rs:477-827) ---------------------------------------
   Upload n_cand Fv candidates: heavy chains of n_heavy residues and light chains of
   n_light (each at most 128), slot layout concatenated per chain, cdr_* = nonzero at
   CDR positions (germline.rs:66-88), all against resident antigen antigen_id;
   cand_id[i] (NULL = i) is the Philox counter word of candidate i.  The resident state
   then holds 2 n_cand chains, heavy i at 2i and light i at 2i + 1 (binder_state_download
   returns them so). */
int binder_fv_upload(binder_ctx* ctx, size_t n_cand, int32_t n_heavy, int32_t n_light, const uint8_t* aa_h,
                     const float* chi_h, const float* pos_h, const uint8_t* cdr_h, const uint8_t* aa_l,
                     const float* chi_l, const float* pos_l, const uint8_t* cdr_l, int32_t antigen_id,
                     const uint32_t* cand_id);
/* The iteration loop of run_fv (diffusion.rs:791-812) on the uploaded Fv population:
   per iteration (temperature(it, iterations)) every heavy chain takes one
   fv_chain_step (diffusion.rs:560-698: Langevin with the grid force of the antigen and
   the compute_forces term of the light chain, restraint to params.shell_radius, CDR
   mutation / rotamer and rotamer-relaxation Metropolis moves, backbone moves, energies
   against the antigen and the partner), then every light chain against the stepped
   heavy chain; the pair is kept when fv_energy (diffusion.rs:541-547) drops below its
   best and put back to the best when it rises.  Draws: Philox with the streams of
   binder_diffuse offset by 4 for the light chain.  Afterwards the state holds the best
   pairs; out_energy double[n_cand] (may be NULL) = their fv_energy. */
int binder_fv_run(binder_ctx* ctx, int iterations, double* out_energy);

/* ---- structure validation (validate.rs:40-132) ---------------------------------------
   ValidationReport::assess of every resident candidate: clash_score (validate.rs:40-63:
   atom pairs of residues more than one apart in sequence closer than 0.7 x the sum of
   their r_min_half) and ramachandran_outliers (validate.rs:112-132: residues with both
   phi and psi whose pair lies outside the alpha-R / beta / alpha-L basins).
   At most 640 residues per candidate.  out_clashes, out_rama int32[n_cand] (either
   may be NULL). */
int binder_validate(binder_ctx* ctx, int32_t* out_clashes, int32_t* out_rama);

/* ---- input and output formats (pdb.rs, report.rs); host code, no context ---------------
   Text results go into out[cap] NUL-terminated; BINDER_ERR_CAPACITY with *out_len =
   the length needed (without the NUL) when cap is too small.
   parse_pdb (pdb.rs:19-57): the CA records of a PDB text (or file) as xyz float[n][3]
   and amino acids (AminoAcid::from_three_letter, atom.rs:127-151); BINDER_ERR_ARG when
   there is none (EmptyInput), BINDER_ERR_CAPACITY with *out_n when cap is too small,
   BINDER_ERR_IO when the file cannot be read. */
int binder_parse_pdb_text(const char* text, size_t len, float* xyz, uint8_t* aa, size_t cap, size_t* out_n);
int binder_parse_pdb_file(const char* path, float* xyz, uint8_t* aa, size_t cap, size_t* out_n);
/* parse_peptide (pdb.rs:64-83): a one-letter sequence on an extended trace along x,
   centred (3.8 A steps); BINDER_ERR_ARG for an empty string or an unknown letter. */
int binder_parse_peptide(const char* seq, float* xyz, uint8_t* aa, size_t cap, size_t* out_n);
/* write_pdb (pdb.rs:90-114): CA-only ATOM records of n residues. */
int binder_write_pdb_ca(size_t n, const float* xyz, const uint8_t* aa, char chain, char* out, size_t cap,
                        size_t* out_len);
/* write_pdb_allatom (pdb.rs:121-152): every heavy atom of a slot-layout protein
   (pos float[n_res][14][3]) with its topology atom name. */
int binder_write_pdb_allatom(size_t n_res, const uint8_t* aa, const float* pos, char chain, char* out, size_t cap,
                             size_t* out_len);
/* write_pdb_multi (pdb.rs:157-191): chains c = 0..n_chains-1 of n_res[c] residues,
   concatenated in aa / pos, chain ids chain_ids[c], one serial numbering, TER after
   each chain. */
int binder_write_pdb_multi(size_t n_chains, const size_t* n_res, const uint8_t* aa, const float* pos,
                           const char* chain_ids, char* out, size_t cap, size_t* out_len);
/* CandidateReport (report.rs:8-20); light_sequence NULL = a single-chain candidate,
   clashes / rama_outliers < 0 = not assessed. */
typedef struct binder_candidate_report {
    int32_t rank;
    const char* sequence;
    const char* light_sequence;
    float energy;
    float entropy_penalty;
    float dg_corrected;
    int32_t net_charge;
    int32_t aggregation_risk;
    int32_t n_interface;
    int32_t clashes;
    int32_t rama_outliers;
} binder_candidate_report;
/* write_fasta / write_json / write_csv (report.rs:41-113). */
int binder_write_fasta(const binder_candidate_report* reports, size_t n, char* out, size_t cap, size_t* out_len);
int binder_write_json(const binder_candidate_report* reports, size_t n, char* out, size_t cap, size_t* out_len);
int binder_write_csv(const binder_candidate_report* reports, size_t n, char* out, size_t cap, size_t* out_len);

/* ---- learned mutation / rotamer proposal (no reference counterpart) ------------------
   A BF16 MLP, 180 -> 256 (SiLU) -> 256 (SiLU) -> 25, FP32 accumulation, trained on
   the GPU on (environment, energy change) tuples of the plain Metropolis moves and
   used as a Metropolis-Hastings proposal for the mutation and rotamer moves of
   binder_diffuse (diffusion.rs:354-399); the exact energy still decides every
   acceptance.
   Features of a residue (180): a one-hot of its amino acid (20), then for shells
   s = 0..7 of 1.25 A around its Calpha and amino acids a = 0..19, log1p of the
   number of antigen Calphas of amino acid a at a distance in [1.25 s, 1.25 (s+1))
   (index 20 + 20 s + a), as BF16.
   Outputs (25): predicted energy change of a mutation to amino acid 0..19, then of
   a move to rotamer 0..4.
   Parameters: one FP32 vector of BINDER_MLP_N_PARAMS values, W1 [256][192] (input
   columns 180..191 zero), b1 [256], W2 [256][256], b2 [256], W3 [32][256] (rows
   25..31 zero), b3 [32] (entries 25..31 zero); W is [out][in]. */
#define BINDER_MLP_IN 180
#define BINDER_MLP_OUT 25
#define BINDER_MLP_N_PARAMS 123424

/* One logged Metropolis proposal (32 bytes). */
typedef struct binder_mc_tuple {
    float x, y, z;     /* Calpha of the residue when the move was proposed */
    float delta_e;     /* Metropolis energy change of the move (kcal/mol) */
    int32_t cand;      /* candidate (resident state index) */
    float log_ratio;   /* log q(reverse move) - log q(move) of the proposal; 0 when uniform */
    int16_t residue;   /* residue within the candidate */
    uint8_t aa;        /* amino acid before the move */
    uint8_t action;    /* 0..19 mutation to that amino acid, 20..24 rotamer 0..4 */
    uint8_t antigen;   /* resident antigen id */
    uint8_t accepted;  /* 1 when the move was accepted */
    uint8_t _pad[2];
} binder_mc_tuple;

/* Set the parameters (resets the optimiser) / read them back. */
int binder_mlp_set_params(binder_ctx* ctx, const float* params);
int binder_mlp_get_params(binder_ctx* ctx, float* params);
/* Amino-acid input of a mutation query: no one-hot.  The network answers a mutation
   query (a residue's environment alone) with outputs 0..19, whose differences
   y[new] - y[old] predict the energy change of mutating old -> new, and a rotamer
   query (environment + the residue's amino acid) with outputs 20..24, the energy
   change of moving to rotamer 0..4. */
#define BINDER_MLP_NO_AA 255
/* Features of n residues (Calpha xyz float[n][3], amino acids or BINDER_MLP_NO_AA)
   against resident antigen antigen_id: out float[n][180] (the BF16 values the
   network sees). */
int binder_mlp_features(binder_ctx* ctx, int32_t antigen_id, size_t n, const float* ca_xyz, const uint8_t* aa,
                        float* out);
/* Network outputs of n feature rows (float[n][180], rounded to BF16): out float[n][25]. */
int binder_mlp_forward(binder_ctx* ctx, size_t n, const float* features, float* out);
/* Mean Huber loss (threshold huber_delta) of the prediction y[action[i]] -
   y[ref[i]] (ref NULL or ref[i] = -1: y[action[i]]) against target[i] over the
   batch -- rows with ref[i] == action[i] contribute zero -- and its gradient with
   respect to every parameter (out_grad float[BINDER_MLP_N_PARAMS], may be NULL).
   Parameters unchanged.  Training on logged tuples uses ref = the amino acid
   before a mutation and -1 for rotamer moves. */
int binder_mlp_loss_grad(binder_ctx* ctx, size_t n, const float* features, const int32_t* action,
                         const int32_t* ref, const float* target, float huber_delta, double* out_loss,
                         float* out_grad);
/* The training set: tuples logged by binder_diffuse (binder_mc_log) or given here. */
int binder_mlp_set_tuples(binder_ctx* ctx, const binder_mc_tuple* tuples, size_t n);
int binder_mlp_tuple_count(binder_ctx* ctx, size_t* out_n);
int binder_mlp_get_tuples(binder_ctx* ctx, binder_mc_tuple* out, size_t cap, size_t* out_n);
/* Log every mutation / rotamer decision of the following binder_diffuse calls with
   Metropolis moves into a device buffer of `capacity` tuples (0 stops logging and
   frees it).  Tuples past the capacity are counted, not stored. */
int binder_mc_log(binder_ctx* ctx, size_t capacity);
int binder_mc_log_count(binder_ctx* ctx, size_t* out_logged, size_t* out_proposed);
int binder_mc_log_fetch(binder_ctx* ctx, binder_mc_tuple* out, size_t cap, size_t* out_n);
/* The logged tuples become the training set (device copy). */
int binder_mlp_take_log(binder_ctx* ctx, size_t* out_n);
/* Proposal of binder_diffuse's mutation and rotamer moves.  UNIFORM: the
   reference's uniform choice.  LEARNED: the choice drawn from softmax(-y / Tp) of
   the network outputs y of the residue's query (mutation: outputs 0..19 of the
   environment; rotamer: outputs 20..24 given the amino acid), Tp = max(T,
   t_prop_min), by inverse CDF on the same random draw (a network with constant
   outputs chooses exactly as UNIFORM does), accepted with probability
   min(1, exp(-dE/T) q(reverse) / q(move)).  The move leaves the query unchanged, so
   q(reverse) / q(move) = exp((y[move] - y[back]) / Tp) exactly, from one network
   evaluation.  Rotamer moves from a chi that is no library rotamer
   stay uniform, and so do all moves of steps whose temperature is above t_max
   (INFINITY: none) -- each step is a Metropolis-Hastings step at its temperature
   either way. */
#define BINDER_PROPOSAL_UNIFORM 0
#define BINDER_PROPOSAL_LEARNED 1
int binder_set_proposal(binder_ctx* ctx, int mode, float t_prop_min, float t_max);
/* n_steps Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on minibatches of `batch`
   tuples drawn uniformly (Philox, key seed) from the training set -- mutations as
   queries without amino acid against y[new] - y[old], rotamer moves as queries
   with it against y[20 + rotamer]; out_losses double[n_steps] (may be NULL) =
   each step's mean Huber loss. */
int binder_mlp_train(binder_ctx* ctx, int n_steps, int batch, float lr, float huber_delta, uint64_t seed,
                     double* out_losses);

/* ---- instrumentation (no reference counterpart) --------------------------------
   The context's CUDA stream (cudaStream_t), for callers that time or order work
   around the library's launches. */
void* binder_stream(binder_ctx* ctx);
/* With timing on, binder_block records CUDA events on the context stream around
   each of its phases (up to 4096 blocks).  binder_timing_summary synchronises,
   returns the summed [gradient steps, scoring, selection] milliseconds and the
   number of blocks recorded since binder_set_timing, and restarts the record.
   Scoring is the residue pair energies; selection is the candidate sums and the
   top-k (one fused launch when k <= 64 and every segment holds at most 4096
   candidates, else the sums are part of scoring). */
int binder_set_timing(binder_ctx* ctx, int on);
int binder_timing_summary(binder_ctx* ctx, double* out_ms_sums, int32_t* out_blocks);
/* In-cutoff pair counts of the resident state: Calpha pairs of n_steps gradient
   steps (state left unchanged) and all-atom pairs of one scoring. */
int binder_state_pair_counts(binder_ctx* ctx, int n_steps, int64_t* out_cg_pairs, int64_t* out_score_pairs);
/* FP32 FMA throughput of the device (TFLOP/s), scalar and packed f32x2. */
int binder_fp32_peak(binder_ctx* ctx, double* out_tflops_scalar, double* out_tflops_packed);

/* ---- failure injection (no reference counterpart; tests) ------------------------
   The bounded device wait every tcgen05 GEMM uses, on a barrier nothing arrives on:
   returns BINDER_ERR_TIMEOUT after max_polls polls and leaves the context usable. */
int binder_selftest_wait(binder_ctx* ctx, uint32_t max_polls);
/* The n-th following device allocation of any context (0 = the next) fails as if
   the device were out of memory (BINDER_ERR_OOM); n < 0 disarms. */
int binder_debug_fail_alloc(int64_t n);

#ifdef __cplusplus
}
#endif
#endif
