// kernels.h — host-side launchers of the sm_100a kernels (one declaration per
// kernel family; definitions live in the k_*.cu translation units).
#pragma once

#include "common.cuh"
#include "mlp.cuh"

namespace binder {

// Launch shapes of the search block, chosen by the autotuner (results do not
// depend on them: every residue is computed by the same lanes with the same
// arithmetic whatever the grid).
struct LaunchCfg {
    int score_warps = 8;         // warps per CTA of the persistent scoring kernel (4, 8, 16)
    int score_ctas_per_sm = 4;   // persistent scoring CTAs per SM
    int cg_warps = 8;            // warps per CTA of the gradient-step kernel (2, 4, 8)
    int cg_lanes = 8;            // lanes per residue of the gradient-step kernel (4, 8)
    int cg_order = 1;            // residue order of the gradient-step kernel: 0 cell, 1 candidate, 2 strided
    int score_order = 0;         // work-queue order of the scoring kernel: 0 cell, 1 residue index
    int cg_queue = 1;            // gradient-step kernel: 0 static grid, 1 persistent CTAs on a work queue
    int cg_flat = 0;             // gradient-step kernel: 0 lane groups (cg_lanes per residue), 8 / 16 / 32 the
                                 // flat form with that many residues per warp
};

// ---- k_grid.cu: SpatialHashGrid ----
void launch_cell_coords(cudaStream_t s, const float* x, const float* y, const float* z, int n, float inv, int4* cells,
                        int* minmax, uint32_t* err);
void launch_cell_hist(cudaStream_t s, int4* cells, int n, int ox, int oy, int oz, int ny, int nz, int* counts);
void launch_exclusive_scan(cudaStream_t s, const int* counts, int n, int* out);
void launch_stable_scatter(cudaStream_t s, const int4* cells, int n, int* cursor, int* sorted_idx);
void launch_gather_atoms(cudaStream_t s, const int* sorted_idx, int n, const float* x, const float* y,
                         const float* z, const float* q, const float* rmh, const float* eps, const uint8_t* hyd,
                         const uint8_t* type, float4* pq, float4* prm);
void launch_gather_ca(cudaStream_t s, const int* sorted_idx, int n, const float* x, const float* y, const float* z,
                      const uint8_t* aa, const float4* res_tab, float inv, float4* pq, float4* prm, int4* cells);
void launch_nb_count(cudaStream_t s, const GridView& g, const float* px, const float* py, const float* pz, int n_q,
                     long long* counts);
void launch_nb_fill(cudaStream_t s, const GridView& g, const int* sorted_idx, const float* px, const float* py,
                    const float* pz, int n_q, const long long* offsets, uint32_t* out);
void launch_cells_out(cudaStream_t s, const float* x, const float* y, const float* z, int n, float inv, int* out);

// ---- k_score.cu: all-atom pair energy / force ----
cudaError_t score_init_tables();
struct ScoreOut {
    double* energy;       // per candidate
    double* abs_sum;      // per candidate sum of |pair term| (may be null)
    float* force;         // per candidate atom, 3 floats (may be null)
    long long* pairs;     // pair counter (may be null)
    uint32_t* err;        // error flags
};
// flat GpuAtom candidates (8 floats per atom), ragged offsets (n_cand + 1)
int launch_score_flat(cudaStream_t s, const float* atoms, const long long* offsets, int n_cand, const AgView* ags,
                      const int* cand_ag, int accumulate, const ScoreOut& out, int grid_ctas, int block);
// resident state (slot layout); full = add H-bond + EEF1 + disulfide.  Persistent
// warps over a residue work queue; per-residue FP64 energies summed per candidate.
struct StateScoreScratch {
    const int* order;  // residue visiting order (may be null)
    int* queue;        // work counter, queue[2] the done count (left zero by queue_retire)
    double* res_e;     // total_res
    double* res_abs;   // total_res (abs sums)
};
// Survivor selection fused into the candidate sums of launch_score_state (k <= 64,
// every segment at most 4096 candidates, listed in ascending candidate index;
// sum_topk_fits): the stable top-k of each segment into out_idx, as
// launch_topk_segments computes it.
struct SumTopk {
    const int* idx_list;
    const long long* seg_off;
    int n_seg;
    int k;
    int* out_idx;
    cudaEvent_t mid;  // recorded between the residue scoring and this launch (may be null)
    bool defer;       // score the residues only; launch_sum_select follows later
};
bool sum_topk_fits(int k, long long max_segment);
// the candidate sums of res_e (residue energies of launch_score_state) and the
// selection, as launch_score_state runs them after the residues
void launch_sum_select(cudaStream_t s, const StateView& st, const double* res_e, int full, double* energy,
                       const SumTopk& tk);
int launch_score_state(cudaStream_t s, const StateView& st, const AgView* ags, int accumulate, int full,
                       const ScoreOut& out, const StateScoreScratch& scr, int grid_ctas, int warps_per_cta,
                       const SumTopk* tk = nullptr);

void launch_uniform_offsets(cudaStream_t s, long long* off, int n_cand, long long n_ab);

// ---- k_topk.cu ----
// idx_list (may be null): segment entries are energies[idx_list[j]] and report idx_list[j]
int launch_topk_segments(cudaStream_t s, const double* energies, const int* idx_list, const long long* seg_off,
                         int n_seg, int k, int* out_idx);

// ---- k_search.cu: residues, CG forces, Langevin, Metropolis ----
cudaError_t search_init_tables();
void launch_build_residues(cudaStream_t s, int n, const float* ca_xyz, const uint8_t* aa, const float4* chi_trig,
                           const float* chi_deg, float4* out_pos, float4* out_chi);
void launch_cg_forces(cudaStream_t s, const AgView* ag, const float* bx, const float* by, const float* bz,
                      const uint8_t* baa, int n, float* fx, float* fy, float* fz);
void launch_diffuse(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                    uint32_t step0, int with_noise, const float* temps, uint32_t* err, const int* order,
                    int warps_per_cta, int lanes_per_res, int order_mode, int max_ag_res, int max_ag_cells,
                    int stage_ag, int* queue, int flat_res);
// residue permutation sorted by (antigen, Calpha cell); key_base[a] = first key of antigen a
void launch_residue_order(cudaStream_t s, const StateView& st, const AgView* ags, const int* key_base, int n_keys,
                          int* keys, int* counts, int* cursor, int* order);
void launch_pack_slots(cudaStream_t s, int n_res, const float* in, float4* out);
// gather residues map[0..total) (slot layout + aa, chi, trig) and the Metropolis
// statistics of candidates cidx[0..n_cand) into fresh buffers
void launch_gather_state(cudaStream_t s, int total, const int* map, const uint8_t* aa, const float4* chi,
                         const float4* trig, const float4* pos, uint8_t* o_aa, float4* o_chi, float4* o_trig,
                         float4* o_pos, int n_cand, const int* cidx, const long long* stats, long long* o_stats);
// pair counting (same trajectory as launch_diffuse with noise off, state not written)
void launch_diffuse_count(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          long long* pairs);
// state scoring pair count
void launch_score_state_count(cudaStream_t s, const StateView& st, const AgView* ags, long long* pairs,
                              uint32_t* err, const StateScoreScratch& scr, int grid_ctas);

// ---- k_anneal.cu: Langevin + Metropolis steps, one CTA per candidate ----
constexpr int ANNEAL_MAX_RES = 128;  // residues per candidate held in shared memory
cudaError_t anneal_init_tables();
cudaError_t anneal_init_mlp_table(const float* log1p_table);
// Metropolis energy (Calpha-level contributions + disulfide) of every candidate
void launch_mc_energy(cudaStream_t s, const StateView& st, const AgView* ags, double* out);
size_t anneal_smem(int max_res, int max_ag_res, int max_cells, int learned);
// The learned proposal (mlp, used when learned) and the proposal log (log may be
// null: every mutation / rotamer decision appends one tuple while *log_n < log_cap;
// *log_n counts all decisions).
struct AnnealExtras {
    MlpDev mlp{};
    bool learned = false;
    MlpTuple* log = nullptr;
    unsigned long long* log_n = nullptr;
    long long log_cap = 0;
};
// accumulate: 1 = the reference's f32 sums, else f32 terms summed in double.
// stats (may be null): 4 per candidate, += mutation/rotamer tried, accepted,
// backbone tried, accepted.
// fv_chain >= 0: the Fv two-chain step of chains 2i + fv_chain (fv_cdr: CDR flag per residue)
cudaError_t launch_anneal(cudaStream_t s, const StateView& st, const AgView* ags, const StepParams& p, int n_steps,
                          uint32_t step0, int with_noise, const float* temps, int accumulate, int max_res,
                          int max_ag_res, int max_cells, uint32_t* err, long long* stats, const AnnealExtras& x,
                          int fv_chain = -1, const uint8_t* fv_cdr = nullptr);

// ---- k_mlp.cu: the learned proposal network (features, tcgen05 GEMM, training) ----
cudaError_t mlp_init_tables(const float* log1p_table);
void launch_features(cudaStream_t s, int n, int n_pad, const float* ca, const uint8_t* aa, const int* ag,
                     const AgView* ags, __nv_bfloat16* X);
void launch_pack_features(cudaStream_t s, int n, int n_pad, const float* f, __nv_bfloat16* X);
void launch_transpose_bf16(cudaStream_t s, int rows, int cols, const __nv_bfloat16* in, __nv_bfloat16* out);
cudaError_t launch_gemm_tc(cudaStream_t s, const GemmArgs& g, uint32_t* err);
cudaError_t launch_wait_selftest(cudaStream_t s, uint32_t max_polls, uint32_t* err);
void launch_mlp_loss(cudaStream_t s, int m, int m_pad, const float* Y, const int* action, const int* ref,
                     const float* target, float delta, __nv_bfloat16* dY, __nv_bfloat16* dYt, double* loss);
void launch_rowsum_bf16(cudaStream_t s, int rows, int m, int ld, const __nv_bfloat16* G, float* out);
void launch_reduce_partials(cudaStream_t s, int n, int n_part, long long stride, const float* part, float* out);
void launch_adam(cudaStream_t s, int n, float* w, const float* g, float* m1, float* m2, float lr, float b1, float b2,
                 float eps, float bc1, float bc2);
void launch_pack_weights(cudaStream_t s, const float* p, const MlpBf16& o);
void launch_gather_tuples(cudaStream_t s, int m, const int* idx, const MlpTuple* tup, float* ca, uint8_t* aa, int* ag,
                          int* action, int* ref, float* target);
void launch_draw_batch(cudaStream_t s, int m, int n_tuples, uint64_t seed, uint32_t step, int* idx);

// ---- k_post.cu: minimize and affinity maturation of the resident candidates ----
cudaError_t post_init_tables();
// every residue: the clamped grid-force step from pos_in, side chain rebuilt, into pos_out
void launch_min_move(cudaStream_t s, const StateView& st, const AgView* ags, const float4* pos_in, float4* pos_out,
                     float step_size);
// per candidate: keep the trial positions when e_trial < best (best updated, kept[c]++)
void launch_min_accept(cudaStream_t s, const StateView& st, const float4* trial, const double* e_trial, double* best,
                       int* kept);
// affinity_maturation_allatom of every candidate over its interface residues; res_e
// (per-residue full energies of the state) kept current
void launch_mature(cudaStream_t s, const StateView& st, const AgView* ags, double* res_e, double* out_best,
                   int* out_kept, uint32_t* err);

// Fv pairs (chains 2i, 2i + 1 of the state): the all-atom energy between the chains (at
// most 160 residues per chain, else NaN), and the elitist keep / restore of each pair
void launch_fv_pair(cudaStream_t s, const StateView& st, double* out);
void launch_fv_keep(cudaStream_t s, const StateView& st, const double* e_chain, const double* e_pair, double* best,
                    float4* b_pos, uint8_t* b_aa, float4* b_chi, float4* b_trig, int restore);
// ValidationReport::assess of every candidate: clash_score and ramachandran_outliers
// (at most 640 residues per candidate, else cudaErrorInvalidValue and no launch)
cudaError_t launch_validate(cudaStream_t s, const StateView& st, int* clashes, int* rama);

// ---- k_micro.cu: FP32 peak microbenchmark; returns the flops of the launch ----
double launch_ffma(cudaStream_t s, float* scratch, int ctas, int iters, bool packed);
void launch_unpack_slots(cudaStream_t s, int n_res, const float4* in, float* out);

}  // namespace binder
