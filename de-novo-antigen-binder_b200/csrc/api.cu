// api.cu — the extern "C" boundary (include/binder_gpu.h): context, device
// buffers, antigen residency, resident search state and every entry point.
//
// Host code here only validates, lays data out, moves it and launches kernels;
// every computation of the hot path runs in the k_*.cu kernels.  Nothing throws
// across the ABI: each entry point returns a binder_status and records a message
// for binder_last_error().
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "binder_gpu.h"
#include "kernels.h"

using namespace binder;

namespace {

// Host-side fault injection for the tests: the device allocation that brings the
// countdown to zero fails as if the device were out of memory (no GPU fault).
long long g_alloc_countdown = -1;
bool injected_alloc_failure() {
    if (g_alloc_countdown < 0) return false;
    if (g_alloc_countdown == 0) {
        g_alloc_countdown = -1;
        return true;
    }
    --g_alloc_countdown;
    return false;
}

template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { release(); }
    void swap(DBuf& o) {
        std::swap(p, o.p);
        std::swap(n, o.n);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t m) {
        if (m <= n && p) return cudaSuccess;
        release();
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T));
        if (e == cudaSuccess) n = std::max<size_t>(m, 1);
        else p = nullptr;
        return e;
    }
};

template <class T>
struct HBuf {  // pinned host staging
    T* p = nullptr;
    size_t n = 0;
    HBuf() = default;
    HBuf(const HBuf&) = delete;
    ~HBuf() { if (p) cudaFreeHost(p); }
    cudaError_t ensure(size_t m) {
        if (m <= n && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMallocHost(&p, std::max<size_t>(m, 1) * sizeof(T));
        if (e == cudaSuccess) n = std::max<size_t>(m, 1);
        return e;
    }
};

struct GridBuf {
    DBuf<int4> cells;
    DBuf<int> counts, cell_start, cursor, sorted_idx;
    DBuf<int> minmax;
    GridView view{};
};

// One resident antigen: all-atom records + score grid, Calpha cloud + CG grid.
struct Antigen {
    int n_atoms = 0, n_res = 0;
    DBuf<float> x, y, z, q, rmh, eps;
    DBuf<uint8_t> hyd, type;
    GridBuf grid;
    DBuf<float4> pq, prm;
    DBuf<float> cax, cay, caz;
    DBuf<uint8_t> caa;
    GridBuf ca_grid;
    DBuf<float4> ca_pq, ca_prm, ca_atom, ca_atom_prm;
    DBuf<int4> ca_cell;
    AgView view{};
};

struct State {
    int n_cand = 0, total_res = 0, n_ag_groups = 0;
    DBuf<int> cand_res_off, cand_ag, res_cand, ag_cand_idx;
    DBuf<long long> ag_cand_off;
    DBuf<uint32_t> cand_id;
    DBuf<uint8_t> res_aa;
    DBuf<float4> res_chi, res_pos, res_trig;
    DBuf<float> stage;  // packed slot staging for upload/download
    std::vector<int> h_res_off, h_cand_ag;
    std::vector<uint32_t> h_cand_id;
    std::vector<int> h_orig;  // index of each candidate in the last full upload
    int meta_epoch = -1;      // the antigen-set epoch the device metadata was built for
    int max_res = 0;
    // chi sin/cos for the Metropolis kernel, derived from the uploaded chi on first use
    bool trig_valid = false;
    // Metropolis statistics, 4 per candidate (tried / accepted: mutation+rotamer, backbone)
    DBuf<long long> mc_stats;
    int n_segments = 0;
    long long max_segment = 0;  // candidates of the largest segment
    // residue order by Calpha cell (an autotuned order of the gradient-step and
    // scoring kernels)
    DBuf<int> key_base, keys, key_counts, key_cursor, order;
    int n_keys = 0;
    bool order_valid = false;
    // the gradient-step kernel's Verlet lists (csrc/k_search.cu), valid per residue
    DBuf<int> cg_list;
    DBuf<float4> cg_centre;
    DBuf<int4> cg_meta;
    DBuf<int> cg_bal;  // the flat gradient-step kernel's work-balanced order (cg_bal_* in common.cuh)
    const int* ag_epoch = nullptr;  // the context's device epoch word
    // scoring work queue and per-residue energies
    DBuf<int> queue;
    DBuf<double> res_e, res_abs;
    // survivor selection gathers into these and swaps them in (the replaced buffers
    // become the next selection's), so that selections allocate nothing once grown
    DBuf<uint8_t> alt_aa;
    DBuf<float4> alt_chi, alt_trig, alt_pos;
    DBuf<long long> alt_stats;
    DBuf<int> sel_map, sel_cidx;
    StateView view() {
        StateView v;
        v.n_cand = n_cand;
        v.total_res = total_res;
        v.cand_res_off = cand_res_off.p;
        v.cand_ag = cand_ag.p;
        v.cand_id = cand_id.p;
        v.res_aa = res_aa.p;
        v.res_chi = res_chi.p;
        v.res_pos = res_pos.p;
        v.res_trig = res_trig.p;
        v.res_cand = res_cand.p;
        v.cg_list = cg_list.p;
        v.cg_centre = cg_centre.p;
        v.cg_meta = cg_meta.p;
        v.cg_bal = cg_bal.p;
        v.ag_epoch = ag_epoch;
        return v;
    }
};

const float RADS_PER_DEG = 3.14159265358979323846f / 180.0f;
const size_t MAX_GRID_CELLS = (size_t)1 << 24;

}  // namespace

// Learned proposal network: parameters, Adam moments, BF16 copies, the logged
// Metropolis tuples and the activations of up to `cap` rows.
struct MlpState {
    bool ready = false;
    int adam_t = 0;
    DBuf<float> w, g, m1, m2;
    DBuf<__nv_bfloat16> w1, w2, w2t, w3, w3t;
    DBuf<uint4> f1, f2, f3;
    int cap = 0;
    DBuf<__nv_bfloat16> X, Xt, H1, H1t, H2, H2t, dY, dYt, dZ2, dZ2t, dZ1t, S1, S2;
    DBuf<float> Y, part, feat, ca, target;
    DBuf<uint8_t> aa;
    DBuf<int> ag, action, ref, idx;
    DBuf<double> loss;
    DBuf<MlpTuple> tuples;
    size_t n_tuples = 0;
    // proposal of binder_diffuse's mutation / rotamer moves, and the proposal log
    bool learned = false;
    float t_prop_min = 0.5f, t_max = INFINITY;
    DBuf<MlpTuple> log;
    DBuf<unsigned long long> log_n;
    size_t log_cap = 0;
    MlpBf16 bf16() { return MlpBf16{w1.p, w2.p, w2t.p, w3.p, w3t.p, f1.p, f2.p, f3.p}; }
    MlpDev dev() const {
        return MlpDev{f1.p, f2.p, f3.p, w.p + MLP_OFF_B1, w.p + MLP_OFF_B2, w.p + MLP_OFF_B3, t_prop_min, t_max};
    }
};

struct binder_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    binder_params params{};
    std::string err;
    uint64_t launches = 0;
    int num_sms = 148;
    // drop-in antigen (score_batch path) and its host copy for change detection
    Antigen dropin;
    DBuf<AgView> d_dropin_view;
    bool dropin_valid = false;
    std::vector<float> dropin_key;
    // resident search antigens
    std::vector<std::unique_ptr<Antigen>> ags;
    DBuf<AgView> d_views;
    DBuf<float4> d_res_tab;
    // scratch
    DBuf<float> cand;
    DBuf<long long> off;
    DBuf<double> energy, energy_abs;
    DBuf<float> force;
    DBuf<long long> pairs;
    DBuf<uint32_t> errf;
    DBuf<int> topk;
    DBuf<float> temps;
    DBuf<float> tmp_f;
    DBuf<uint8_t> tmp_u8;
    DBuf<float4> tmp_f4a, tmp_f4b;
    DBuf<long long> tmp_ll;
    DBuf<uint32_t> tmp_u32;
    HBuf<double> h_energy;
    HBuf<uint32_t> h_err;
    size_t last_n_cand = 0;
    bool last_batch_valid = false;
    State st;
    // per-phase event timing of binder_block: a ring of 4 events per block
    bool timing = false;
    std::vector<cudaEvent_t> ev;
    int ev_blocks = 0;
    int last_k = 0;
    bool async_pending = false;
    // launch shapes (autotuned) and the CUDA graph of the search block
    LaunchCfg cfg;
    cudaGraphExec_t block_graph = nullptr;
    std::vector<uint64_t> block_graph_sig;  // what the captured launches baked in
    int block_graph_launches = 0;
    bool block_graph_order = false;  // the residue order is valid after a replay
    // enqueued (binder_block without outputs) blocks run as a pipeline: each block's
    // graph sums and selects the previous block's residue energies on the side stream
    // beside its own gradient steps; sel_pending: the last block's selection (top-sel_k)
    // is still to run (flushed by the next call that is not such a block)
    cudaGraphExec_t pipe_graph = nullptr;
    std::vector<uint64_t> pipe_graph_sig;
    int pipe_graph_launches = 0;
    bool pipe_graph_order = false;
    bool sel_pending = false;
    int sel_k = 0;
    // binder_block_io as one graph (copies in, block, copies out) for pinned host arrays
    cudaGraphExec_t io_graph = nullptr;
    std::vector<uint64_t> io_graph_sig;
    int io_graph_launches = 0;
    bool io_graph_order = false;
    std::vector<std::pair<std::string, LaunchCfg>> tune_cache;
    MlpState mlp;
    // antigen-set epoch (device word read by the gradient-step kernel)
    DBuf<int> d_ag_epoch;
    int ag_epoch = 0;
    // Fv two-chain population (binder_fv_upload): the state interleaves the heavy (2i)
    // and light (2i + 1) chains of fv_pairs candidates; CDR flag per residue; the best
    // pairs of binder_fv_run
    int fv_pairs = 0;
    DBuf<uint8_t> fv_cdr, fv_baa;
    DBuf<double> fv_best, fv_pair_e;
    DBuf<float4> fv_bpos, fv_bchi, fv_btrig;
    // binder_block_io: the state download runs on a second stream beside the score
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void drop_block_graph() {
        if (block_graph) cudaGraphExecDestroy(block_graph);
        block_graph = nullptr;
    }
    void drop_pipe_graph() {
        if (pipe_graph) cudaGraphExecDestroy(pipe_graph);
        pipe_graph = nullptr;
    }
    void drop_io_graph() {
        if (io_graph) cudaGraphExecDestroy(io_graph);
        io_graph = nullptr;
    }
    void drop_graph() {
        drop_block_graph();
        drop_pipe_graph();
        drop_io_graph();
    }
    ~binder_ctx() {
        drop_graph();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (side) cudaStreamDestroy(side);
    }
};
static const int TIMING_RING = 4096;

namespace {

int fail(binder_ctx* ctx, int status, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return status;
}

int cuda_fail(binder_ctx* ctx, cudaError_t e, const char* what) {
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return fail(ctx, BINDER_ERR_OOM, "%s: out of device memory", what);
    }
    return fail(ctx, BINDER_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                                      \
    do {                                                    \
        cudaError_t e__ = (call);                           \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, what); \
    } while (0)

#define LAUNCHED(what)                                      \
    do {                                                    \
        ctx->launches++;                                    \
        cudaError_t e__ = cudaGetLastError();               \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, what); \
    } while (0)

// log1p(n) of the environment counts, n = 0..255, rounded once to f32
cudaError_t init_mlp_tables() {
    float t[MLP_COUNT_CAP + 1];
    for (int n = 0; n <= MLP_COUNT_CAP; ++n) t[n] = (float)std::log1p((double)n);
    cudaError_t e = mlp_init_tables(t);
    return e ? e : anneal_init_mlp_table(t);
}

int flush_select(binder_ctx* ctx);

// Every entry point starts here; the pending selection of an enqueued block runs
// first, so that nothing sees or replaces the residue energies before it.
int enter_keep(binder_ctx* ctx) {
    if (!ctx) return BINDER_ERR_ARG;
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaSetDevice");
    ctx->err.clear();
    return BINDER_OK;
}
int enter(binder_ctx* ctx) {
    int s = enter_keep(ctx);
    if (s) return s;
    return ctx->sel_pending ? flush_select(ctx) : BINDER_OK;
}

// Reset the device error word before a group of launches.
int clear_err(binder_ctx* ctx) {
    CK(ctx->errf.ensure(1), "alloc err");
    CK(cudaMemsetAsync(ctx->errf.p, 0, sizeof(uint32_t), ctx->stream), "memset err");
    // the persistent kernels' work queues, left zero by every launch that completes
    if (ctx->st.queue.p) CK(cudaMemsetAsync(ctx->st.queue.p, 0, 4 * sizeof(int), ctx->stream), "memset queues");
    return BINDER_OK;
}

// Copy the device error word back (synchronises the stream) and map it to a status.
int check_err(binder_ctx* ctx) {
    CK(ctx->h_err.ensure(1), "alloc host err");
    CK(cudaMemcpyAsync(ctx->h_err.p, ctx->errf.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream), "err D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    uint32_t f = ctx->h_err.p[0];
    if (f & ERRF_NAN) return fail(ctx, BINDER_ERR_NAN, "non-finite coordinate in input");
    if (f & ERRF_TIMEOUT) return fail(ctx, BINDER_ERR_TIMEOUT, "device wait timed out");
    if (f & ERRF_RANGE) return fail(ctx, BINDER_ERR_ARG, "device index out of range");
    return BINDER_OK;
}

template <class T>
int upload(binder_ctx* ctx, DBuf<T>& d, const T* h, size_t n, const char* what) {
    CK(d.ensure(n), what);
    if (n) CK(cudaMemcpyAsync(d.p, h, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream), what);
    return BINDER_OK;
}

// New antigen set: every stored Verlet list of the gradient-step kernel is stale.
int bump_antigen_epoch(binder_ctx* ctx) {
    CK(ctx->d_ag_epoch.ensure(1), "alloc");
    ++ctx->ag_epoch;
    CK(cudaMemcpyAsync(ctx->d_ag_epoch.p, &ctx->ag_epoch, sizeof(int), cudaMemcpyHostToDevice, ctx->stream),
       "epoch H2D");
    ctx->st.ag_epoch = ctx->d_ag_epoch.p;
    return BINDER_OK;
}

// Counting-sort grid over n points (device x/y/z).  spatial.rs:23-39 semantics.
int build_grid(binder_ctx* ctx, const float* x, const float* y, const float* z, int n, float cell, GridBuf& G) {
    if (!(cell > 0.0f) || !std::isfinite(cell)) return fail(ctx, BINDER_ERR_ARG, "grid cell must be positive");
    const float inv = 1.0f / cell;
    G.view.inv = inv;
    G.view.cell = cell;
    int h_mm[6] = {INT32_MAX, INT32_MAX, INT32_MAX, INT32_MIN, INT32_MIN, INT32_MIN};
    CK(G.minmax.ensure(6), "grid alloc");
    CK(G.cells.ensure(n), "grid alloc");
    CK(cudaMemcpyAsync(G.minmax.p, h_mm, sizeof(h_mm), cudaMemcpyHostToDevice, ctx->stream), "grid H2D");
    int st = clear_err(ctx);
    if (st) return st;
    launch_cell_coords(ctx->stream, x, y, z, n, inv, G.cells.p, G.minmax.p, ctx->errf.p);
    if (n > 0) LAUNCHED("cell_coords");
    CK(cudaMemcpyAsync(h_mm, G.minmax.p, sizeof(h_mm), cudaMemcpyDeviceToHost, ctx->stream), "grid D2H");
    st = check_err(ctx);
    if (st) return st;
    if (n == 0) {
        for (int k = 0; k < 3; ++k) h_mm[k] = 0, h_mm[k + 3] = 0;
    }
    const long long nx = (long long)h_mm[3] - h_mm[0] + 1, ny = (long long)h_mm[4] - h_mm[1] + 1,
                    nz = (long long)h_mm[5] - h_mm[2] + 1;
    if (nx <= 0 || ny <= 0 || nz <= 0 || (double)nx * ny * nz > (double)MAX_GRID_CELLS)
        return fail(ctx, BINDER_ERR_GRID, "grid box %lldx%lldx%lld exceeds %zu cells (cell %.3g)", nx, ny, nz,
                    MAX_GRID_CELLS, (double)cell);
    const int ncell = (int)(nx * ny * nz);
    G.view.ox = h_mm[0]; G.view.oy = h_mm[1]; G.view.oz = h_mm[2];
    G.view.nx = (int)nx; G.view.ny = (int)ny; G.view.nz = (int)nz;
    CK(G.counts.ensure(ncell), "grid alloc");
    CK(G.cell_start.ensure(ncell + 1), "grid alloc");
    CK(G.cursor.ensure(ncell + 1), "grid alloc");
    CK(G.sorted_idx.ensure(n), "grid alloc");
    CK(cudaMemsetAsync(G.counts.p, 0, ncell * sizeof(int), ctx->stream), "grid memset");
    launch_cell_hist(ctx->stream, G.cells.p, n, G.view.ox, G.view.oy, G.view.oz, G.view.ny, G.view.nz, G.counts.p);
    if (n > 0) LAUNCHED("cell_hist");
    launch_exclusive_scan(ctx->stream, G.counts.p, ncell, G.cell_start.p);
    LAUNCHED("exclusive_scan");
    CK(cudaMemcpyAsync(G.cursor.p, G.cell_start.p, (ncell + 1) * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream),
       "grid D2D");
    launch_stable_scatter(ctx->stream, G.cells.p, n, G.cursor.p, G.sorted_idx.p);
    LAUNCHED("stable_scatter");
    G.view.cell_start = G.cell_start.p;
    return BINDER_OK;
}

// All-atom records + score grid of an antigen given as a host AtomCloud.
int build_antigen_atoms(binder_ctx* ctx, Antigen& A, const float* x, const float* y, const float* z, const float* q,
                        const float* rmh, const float* eps, const uint8_t* hyd, const uint8_t* type, size_t n) {
    if (n > (size_t)INT32_MAX / 2) return fail(ctx, BINDER_ERR_ARG, "antigen too large");
    int s;
    if ((s = upload(ctx, A.x, x, n, "antigen x")) || (s = upload(ctx, A.y, y, n, "antigen y")) ||
        (s = upload(ctx, A.z, z, n, "antigen z")) || (s = upload(ctx, A.q, q, n, "antigen q")) ||
        (s = upload(ctx, A.rmh, rmh, n, "antigen rmh")) || (s = upload(ctx, A.eps, eps, n, "antigen eps")) ||
        (s = upload(ctx, A.hyd, hyd, n, "antigen hyd")))
        return s;
    if (type) {
        if ((s = upload(ctx, A.type, type, n, "antigen type"))) return s;
    }
    A.n_atoms = (int)n;
    if ((s = build_grid(ctx, A.x.p, A.y.p, A.z.p, (int)n, ctx->params.score_cell, A.grid))) return s;
    CK(A.pq.ensure(n), "antigen alloc");
    CK(A.prm.ensure(n), "antigen alloc");
    launch_gather_atoms(ctx->stream, A.grid.sorted_idx.p, (int)n, A.x.p, A.y.p, A.z.p, A.q.p, A.rmh.p, A.eps.p,
                        A.hyd.p, type ? A.type.p : nullptr, A.pq.p, A.prm.p);
    if (n > 0) LAUNCHED("gather_atoms");
    A.view.pq = A.pq.p;
    A.view.prm = A.prm.p;
    A.view.grid = A.grid.view;
    A.view.n_atoms = (int)n;
    return BINDER_OK;
}

// Residue-level Calpha cloud + CG grid (run_allatom ag_ca, diffusion.rs:994-1004).
int build_antigen_ca(binder_ctx* ctx, Antigen& A, const float* x, const float* y, const float* z, const uint8_t* aa,
                     size_t n, float cell) {
    int s;
    if ((s = upload(ctx, A.cax, x, n, "ca x")) || (s = upload(ctx, A.cay, y, n, "ca y")) ||
        (s = upload(ctx, A.caz, z, n, "ca z")) || (s = upload(ctx, A.caa, aa, n, "ca aa")))
        return s;
    A.n_res = (int)n;
    if ((s = build_grid(ctx, A.cax.p, A.cay.p, A.caz.p, (int)n, cell, A.ca_grid))) return s;
    CK(A.ca_pq.ensure(n), "ca alloc");
    CK(A.ca_prm.ensure(n), "ca alloc");
    CK(A.ca_cell.ensure(n), "ca alloc");
    launch_gather_ca(ctx->stream, A.ca_grid.sorted_idx.p, (int)n, A.cax.p, A.cay.p, A.caz.p, A.caa.p,
                     ctx->d_res_tab.p, A.ca_grid.view.inv, A.ca_pq.p, A.ca_prm.p, A.ca_cell.p);
    if (n > 0) LAUNCHED("gather_ca");
    A.view.ca_pq = A.ca_pq.p;
    A.view.ca_prm = A.ca_prm.p;
    A.view.ca_cell = A.ca_cell.p;
    A.view.res_aa = A.caa.p;
    A.view.ca_grid = A.ca_grid.view;
    A.view.n_res = (int)n;
    return BINDER_OK;
}

int validate_cloud(binder_ctx* ctx, const binder_atom_cloud* c, const char* what) {
    if (!c) return fail(ctx, BINDER_ERR_ARG, "%s: NULL cloud", what);
    if (c->n && (!c->x || !c->y || !c->z || !c->charge || !c->r_min_half || !c->epsilon || !c->hydrophobic))
        return fail(ctx, BINDER_ERR_ARG, "%s: NULL array", what);
    return BINDER_OK;
}

// Upload the drop-in antigen when its contents differ from the resident copy.
int ensure_dropin(binder_ctx* ctx, const binder_atom_cloud* ag) {
    int s = validate_cloud(ctx, ag, "antigen");
    if (s) return s;
    const size_t n = ag->n;
    std::vector<float> key;
    key.reserve(n * 7 + 2);
    key.push_back((float)n);
    key.push_back(ag->atom_type ? 1.0f : 0.0f);
    for (size_t i = 0; i < n; ++i) {
        key.push_back(ag->x[i]); key.push_back(ag->y[i]); key.push_back(ag->z[i]);
        key.push_back(ag->charge[i]); key.push_back(ag->r_min_half[i]); key.push_back(ag->epsilon[i]);
        key.push_back((float)ag->hydrophobic[i] + (ag->atom_type ? 256.0f * ag->atom_type[i] : 0.0f));
    }
    if (ctx->dropin_valid && key.size() == ctx->dropin_key.size() &&
        std::memcmp(key.data(), ctx->dropin_key.data(), key.size() * sizeof(float)) == 0)
        return BINDER_OK;
    ctx->dropin_valid = false;
    if ((s = build_antigen_atoms(ctx, ctx->dropin, ag->x, ag->y, ag->z, ag->charge, ag->r_min_half, ag->epsilon,
                                 ag->hydrophobic, ag->atom_type, n)))
        return s;
    CK(ctx->d_dropin_view.ensure(1), "view alloc");
    CK(cudaMemcpyAsync(ctx->d_dropin_view.p, &ctx->dropin.view, sizeof(AgView), cudaMemcpyHostToDevice, ctx->stream),
       "view H2D");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    ctx->dropin_key.swap(key);
    ctx->dropin_valid = true;
    return BINDER_OK;
}

int grid_ctas(binder_ctx* ctx, int n_cand) { return std::min(n_cand, ctx->num_sms * 8); }

// Score n_cand ragged candidates already in ctx->cand / ctx->off against the drop-in antigen.
int score_resident_batch(binder_ctx* ctx, int n_cand, bool want_abs) {
    int s;
    CK(ctx->energy.ensure(n_cand), "alloc energy");
    if (want_abs) CK(ctx->energy_abs.ensure(n_cand), "alloc energy");
    if ((s = clear_err(ctx))) return s;
    ScoreOut o{ctx->energy.p, want_abs ? ctx->energy_abs.p : nullptr, nullptr, nullptr, ctx->errf.p};
    launch_score_flat(ctx->stream, ctx->cand.p, ctx->off.p, n_cand, ctx->d_dropin_view.p, nullptr,
                      ctx->params.accumulate, o, grid_ctas(ctx, n_cand), 256);
    LAUNCHED("score_flat");
    ctx->last_n_cand = (size_t)n_cand;
    ctx->last_batch_valid = true;
    return BINDER_OK;
}

int fetch_energies(binder_ctx* ctx, int n, double* out, double* out_abs, float* out32) {
    CK(ctx->h_energy.ensure(2 * (size_t)n), "alloc host");
    CK(cudaMemcpyAsync(ctx->h_energy.p, ctx->energy.p, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
       "energy D2H");
    if (out_abs)
        CK(cudaMemcpyAsync(ctx->h_energy.p + n, ctx->energy_abs.p, n * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "energy D2H");
    int s = check_err(ctx);
    if (s) return s;
    if (out) std::memcpy(out, ctx->h_energy.p, n * sizeof(double));
    if (out_abs) std::memcpy(out_abs, ctx->h_energy.p + n, n * sizeof(double));
    if (out32)
        for (int i = 0; i < n; ++i) out32[i] = (float)ctx->h_energy.p[i];
    return BINDER_OK;
}

int score_batch_common(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                       size_t n_atoms, size_t n_ab, double* out64, double* out_abs, float* out32, size_t out_cap,
                       size_t* out_n_cand) {
    int s = enter(ctx);
    if (s) return s;
    const size_t n_cand = n_ab == 0 ? 0 : n_atoms / n_ab;
    if (out_n_cand) *out_n_cand = n_cand;
    if (n_cand == 0) return BINDER_OK;
    if (!candidates) return fail(ctx, BINDER_ERR_ARG, "candidates is NULL");
    if (out_cap < n_cand) return fail(ctx, BINDER_ERR_CAPACITY, "out_cap %zu < n_cand %zu", out_cap, n_cand);
    if (n_cand > (size_t)INT32_MAX) return fail(ctx, BINDER_ERR_ARG, "too many candidates");
    if ((s = ensure_dropin(ctx, antigen))) return s;
    const size_t used = n_cand * n_ab;
    CK(ctx->cand.ensure(used * 8), "alloc candidates");
    CK(cudaMemcpyAsync(ctx->cand.p, candidates, used * sizeof(binder_gpu_atom), cudaMemcpyHostToDevice, ctx->stream),
       "candidates H2D");
    CK(ctx->off.ensure(n_cand + 1), "alloc offsets");
    launch_uniform_offsets(ctx->stream, ctx->off.p, (int)n_cand, (long long)n_ab);
    LAUNCHED("uniform_offsets");
    if ((s = score_resident_batch(ctx, (int)n_cand, out_abs != nullptr))) return s;
    return fetch_energies(ctx, (int)n_cand, out64, out_abs, out32);
}

void refresh_views(binder_ctx* ctx, std::vector<AgView>& v) {
    v.clear();
    for (auto& a : ctx->ags) v.push_back(a->view);
}

}  // namespace

// =============================================================================
extern "C" {

int binder_abi_version(void) { return BINDER_ABI_VERSION; }

int binder_table_residue(int aa, int* n_atoms, float* charge, uint8_t* atom_type, uint8_t* hydrophobic) {
    if (aa < 0 || aa >= N_AA) return BINDER_ERR_ARG;
    if (n_atoms) *n_atoms = BT_TOPO_N[aa];
    for (int k = 0; k < SLOTS; ++k) {
        if (charge) charge[k] = BT_SLOT_Q[aa][k];
        if (atom_type) atom_type[k] = BT_SLOT_TYPE[aa][k];
        if (hydrophobic) hydrophobic[k] = BT_SLOT_HYD[aa][k];
    }
    return BINDER_OK;
}

int binder_table_atom_type(int t, float* rmh, float* eps, int* hb, float* eef1) {
    if (t < 0 || t >= 16) return BINDER_ERR_ARG;
    if (rmh) *rmh = BT_NB[t][0];
    if (eps) *eps = BT_NB[t][1];
    if (hb) *hb = BT_HB[t];
    if (eef1)
        for (int k = 0; k < 3; ++k) eef1[k] = BT_EEF1[t][k];
    return BINDER_OK;
}

int binder_table_rotamers(int aa, int* n, float* chi) {
    if (aa < 0 || aa >= N_AA) return BINDER_ERR_ARG;
    if (n) *n = BT_ROT_N[aa];
    if (chi)
        for (int r = 0; r < 5; ++r)
            for (int c = 0; c < 4; ++c) chi[r * 4 + c] = BT_ROT_CHI[aa][r][c];
    return BINDER_OK;
}

int binder_table_residue_level(int aa, float* out4) {
    if (aa < 0 || aa >= N_AA || !out4) return BINDER_ERR_ARG;
    for (int k = 0; k < 4; ++k) out4[k] = BT_RES[aa][k];
    return BINDER_OK;
}

const char* binder_status_string(int s) {
    switch (s) {
        case BINDER_OK: return "ok";
        case BINDER_ERR_ARG: return "invalid argument";
        case BINDER_ERR_CUDA: return "CUDA error";
        case BINDER_ERR_OOM: return "out of memory";
        case BINDER_ERR_TIMEOUT: return "device wait timed out";
        case BINDER_ERR_NAN: return "non-finite input";
        case BINDER_ERR_GRID: return "grid too large";
        case BINDER_ERR_STATE: return "call out of order";
        case BINDER_ERR_NODEVICE: return "no usable sm_100 device";
        case BINDER_ERR_CAPACITY: return "output buffer too small";
        case BINDER_ERR_IO: return "file could not be read";
        default: return "unknown status";
    }
}

void binder_default_params(binder_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->step = 0.08f;
    p->noise_base = 0.25f;
    p->t_hot = 3.0f;
    p->t_cold = 0.02f;
    p->mutation_p = 0.08f;
    p->rotamer_move_p = 0.12f;
    p->backbone_move_p = 0.04f;
    p->max_torsion_deg = 15.0f;
    p->iface_cutoff_sq = 64.0f;
    p->shell_radius = 20.0f;
    p->max_disp = 2.0f;
    p->restraint_k = 0.02f;
    p->ca_cell = 10.0f;
    p->score_cell = 8.0f;
    p->accumulate = BINDER_ACC_KAHAN;
    p->flags = BINDER_FLAG_GRAPH;
    p->seed = 0;
}

binder_ctx* binder_create(int device, const binder_params* params, int* status) {
    int dummy;
    if (!status) status = &dummy;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        *status = BINDER_ERR_NODEVICE;
        return nullptr;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) {
        cudaGetLastError();
        *status = BINDER_ERR_NODEVICE;
        return nullptr;
    }
    binder_ctx* ctx = new (std::nothrow) binder_ctx();
    if (!ctx) {
        *status = BINDER_ERR_OOM;
        return nullptr;
    }
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    if (params) ctx->params = *params;
    else binder_default_params(&ctx->params);
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        score_init_tables() != cudaSuccess || search_init_tables() != cudaSuccess ||
        anneal_init_tables() != cudaSuccess || init_mlp_tables() != cudaSuccess || post_init_tables() != cudaSuccess) {
        cudaGetLastError();
        delete ctx;
        *status = BINDER_ERR_CUDA;
        return nullptr;
    }
    float4 tab[N_AA];
    for (int a = 0; a < N_AA; ++a) tab[a] = make_float4(BT_RES[a][0], BT_RES[a][1], BT_RES[a][2], BT_RES[a][3]);
    if (ctx->d_res_tab.ensure(N_AA) != cudaSuccess ||
        cudaMemcpy(ctx->d_res_tab.p, tab, sizeof(tab), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaGetLastError();
        cudaStreamDestroy(ctx->stream);
        delete ctx;
        *status = BINDER_ERR_CUDA;
        return nullptr;
    }
    *status = BINDER_OK;
    return ctx;
}

void binder_destroy(binder_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaStream_t s = ctx->stream;
    delete ctx;
    if (s) cudaStreamDestroy(s);
}

int binder_set_params(binder_ctx* ctx, const binder_params* p) {
    if (!ctx || !p) return BINDER_ERR_ARG;
    if (!(p->score_cell > 0.f) || !(p->ca_cell > 0.f)) return fail(ctx, BINDER_ERR_ARG, "cell sizes must be positive");
    if (p->score_cell != ctx->params.score_cell) ctx->dropin_valid = false;
    ctx->params = *p;
    return BINDER_OK;
}

const char* binder_last_error(const binder_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int binder_synchronize(binder_ctx* ctx) {
    int s = enter(ctx);
    if (s) return s;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

uint64_t binder_launch_count(const binder_ctx* ctx) { return ctx ? ctx->launches : 0; }

int binder_score_batch(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                       size_t n_atoms, size_t n_ab, float* out, size_t out_cap, size_t* out_n_cand) {
    if (!out && n_ab && n_atoms / n_ab) return fail(ctx, BINDER_ERR_ARG, "out_energies is NULL");
    return score_batch_common(ctx, antigen, candidates, n_atoms, n_ab, nullptr, nullptr, out, out_cap, out_n_cand);
}

int binder_score_batch_f64(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                           size_t n_atoms, size_t n_ab, double* out, double* out_abs, size_t out_cap,
                           size_t* out_n_cand) {
    if (!out && n_ab && n_atoms / n_ab) return fail(ctx, BINDER_ERR_ARG, "out_energies is NULL");
    return score_batch_common(ctx, antigen, candidates, n_atoms, n_ab, out, out_abs, nullptr, out_cap, out_n_cand);
}

int binder_score_batch_ragged(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                              const int64_t* offsets, size_t n_cand, double* out, double* out_abs) {
    int s = enter(ctx);
    if (s) return s;
    if (n_cand == 0) return BINDER_OK;
    if (!offsets || !out) return fail(ctx, BINDER_ERR_ARG, "NULL offsets/out");
    if (n_cand > (size_t)INT32_MAX) return fail(ctx, BINDER_ERR_ARG, "too many candidates");
    if (offsets[0] != 0) return fail(ctx, BINDER_ERR_ARG, "offsets[0] must be 0");
    for (size_t c = 0; c < n_cand; ++c)
        if (offsets[c + 1] < offsets[c]) return fail(ctx, BINDER_ERR_ARG, "offsets must be non-decreasing");
    const size_t n_atoms = (size_t)offsets[n_cand];
    if (n_atoms && !candidates) return fail(ctx, BINDER_ERR_ARG, "candidates is NULL");
    if ((s = ensure_dropin(ctx, antigen))) return s;
    CK(ctx->cand.ensure(n_atoms * 8), "alloc candidates");
    if (n_atoms)
        CK(cudaMemcpyAsync(ctx->cand.p, candidates, n_atoms * sizeof(binder_gpu_atom), cudaMemcpyHostToDevice,
                           ctx->stream),
           "candidates H2D");
    if ((s = upload(ctx, ctx->off, (const long long*)offsets, n_cand + 1, "offsets H2D"))) return s;
    if ((s = score_resident_batch(ctx, (int)n_cand, out_abs != nullptr))) return s;
    return fetch_energies(ctx, (int)n_cand, out, out_abs, nullptr);
}

int binder_set_antigen_atoms(binder_ctx* ctx, const binder_atom_cloud* antigen) {
    int s = enter(ctx);
    if (s) return s;
    return ensure_dropin(ctx, antigen);
}

int binder_last_pair_count(binder_ctx* ctx, int64_t* out_pairs) {
    int s = enter(ctx);
    if (s) return s;
    if (!out_pairs) return fail(ctx, BINDER_ERR_ARG, "NULL out");
    if (!ctx->last_batch_valid || !ctx->dropin_valid) return fail(ctx, BINDER_ERR_STATE, "no scored batch");
    const int n_cand = (int)ctx->last_n_cand;
    CK(ctx->pairs.ensure(1), "alloc");
    CK(cudaMemsetAsync(ctx->pairs.p, 0, sizeof(long long), ctx->stream), "memset");
    if ((s = clear_err(ctx))) return s;
    ScoreOut o{ctx->energy.p, nullptr, nullptr, ctx->pairs.p, ctx->errf.p};
    launch_score_flat(ctx->stream, ctx->cand.p, ctx->off.p, n_cand, ctx->d_dropin_view.p, nullptr, 0, o,
                      grid_ctas(ctx, n_cand), 256);
    LAUNCHED("score_flat_count");
    long long h = 0;
    CK(cudaMemcpyAsync(&h, ctx->pairs.p, sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if ((s = check_err(ctx))) return s;
    *out_pairs = h;
    return BINDER_OK;
}

int binder_grid_cells(binder_ctx* ctx, float cell, const float* x, const float* y, const float* z, size_t n,
                      int32_t* out) {
    int s = enter(ctx);
    if (s) return s;
    if (n == 0) return BINDER_OK;
    if (!x || !y || !z || !out) return fail(ctx, BINDER_ERR_ARG, "NULL array");
    if (!(cell > 0.0f)) return fail(ctx, BINDER_ERR_ARG, "cell must be positive");
    CK(ctx->tmp_f.ensure(3 * n), "alloc");
    CK(cudaMemcpyAsync(ctx->tmp_f.p, x, n * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    CK(cudaMemcpyAsync(ctx->tmp_f.p + n, y, n * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    CK(cudaMemcpyAsync(ctx->tmp_f.p + 2 * n, z, n * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    DBuf<int> d_out;
    CK(d_out.ensure(3 * n), "alloc");
    launch_cells_out(ctx->stream, ctx->tmp_f.p, ctx->tmp_f.p + n, ctx->tmp_f.p + 2 * n, (int)n, 1.0f / cell, d_out.p);
    LAUNCHED("cells_out");
    CK(cudaMemcpyAsync(out, d_out.p, 3 * n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_grid_neighbors(binder_ctx* ctx, float cell, const float* ax, const float* ay, const float* az, size_t n_ag,
                          const float* px, const float* py, const float* pz, size_t n_q, int64_t* out_offsets,
                          uint32_t* out_idx, size_t cap, size_t* out_total) {
    int s = enter(ctx);
    if (s) return s;
    if (!out_offsets || (n_q && (!px || !py || !pz)) || (n_ag && (!ax || !ay || !az)))
        return fail(ctx, BINDER_ERR_ARG, "NULL array");
    if (n_ag > (size_t)INT32_MAX / 2 || n_q > (size_t)INT32_MAX / 2) return fail(ctx, BINDER_ERR_ARG, "too many points");
    DBuf<float> pts;
    CK(pts.ensure(3 * (n_ag + n_q) + 1), "alloc");
    float* dax = pts.p;
    float* day = dax + n_ag;
    float* daz = day + n_ag;
    float* dpx = daz + n_ag;
    float* dpy = dpx + n_q;
    float* dpz = dpy + n_q;
    if (n_ag) {
        CK(cudaMemcpyAsync(dax, ax, n_ag * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(day, ay, n_ag * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(daz, az, n_ag * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    }
    if (n_q) {
        CK(cudaMemcpyAsync(dpx, px, n_q * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(dpy, py, n_q * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(dpz, pz, n_q * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    }
    GridBuf G;
    if ((s = build_grid(ctx, dax, day, daz, (int)n_ag, cell, G))) return s;
    DBuf<long long> counts;
    CK(counts.ensure(n_q + 1), "alloc");
    launch_nb_count(ctx->stream, G.view, dpx, dpy, dpz, (int)n_q, counts.p);
    if (n_q) LAUNCHED("nb_count");
    std::vector<long long> h(n_q + 1, 0);
    if (n_q) CK(cudaMemcpyAsync(h.data(), counts.p, n_q * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    long long total = 0;
    for (size_t q = 0; q < n_q; ++q) {
        long long c = h[q];
        out_offsets[q] = total;
        h[q] = total;
        total += c;
    }
    out_offsets[n_q] = total;
    h[n_q] = total;
    if (out_total) *out_total = (size_t)total;
    if ((size_t)total > cap) return fail(ctx, BINDER_ERR_CAPACITY, "neighbour list needs %lld entries", total);
    if (total == 0) return BINDER_OK;
    if (!out_idx) return fail(ctx, BINDER_ERR_ARG, "NULL out_idx");
    CK(cudaMemcpyAsync(counts.p, h.data(), (n_q + 1) * sizeof(long long), cudaMemcpyHostToDevice, ctx->stream), "H2D");
    DBuf<uint32_t> idx;
    CK(idx.ensure(total), "alloc");
    launch_nb_fill(ctx->stream, G.view, G.sorted_idx.p, dpx, dpy, dpz, (int)n_q, counts.p, idx.p);
    LAUNCHED("nb_fill");
    CK(cudaMemcpyAsync(out_idx, idx.p, total * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_compute_forces_with_grid(binder_ctx* ctx, const binder_residue_cloud* antigen, float cell,
                                    const binder_residue_cloud* antibody, float* fx, float* fy, float* fz) {
    int s = enter(ctx);
    if (s) return s;
    if (!antigen || !antibody) return fail(ctx, BINDER_ERR_ARG, "NULL cloud");
    const size_t na = antigen->n, nb = antibody->n;
    if (nb == 0) return BINDER_OK;
    if (!fx || !fy || !fz || !antibody->x || !antibody->y || !antibody->z || !antibody->amino_acid ||
        (na && (!antigen->x || !antigen->y || !antigen->z || !antigen->amino_acid)))
        return fail(ctx, BINDER_ERR_ARG, "NULL array");
    for (size_t i = 0; i < na; ++i)
        if (antigen->amino_acid[i] >= N_AA) return fail(ctx, BINDER_ERR_ARG, "antigen amino acid out of range");
    for (size_t i = 0; i < nb; ++i)
        if (antibody->amino_acid[i] >= N_AA) return fail(ctx, BINDER_ERR_ARG, "antibody amino acid out of range");
    Antigen A;
    if ((s = build_antigen_ca(ctx, A, antigen->x, antigen->y, antigen->z, antigen->amino_acid, na, cell))) return s;
    DBuf<AgView> dv;
    CK(dv.ensure(1), "alloc");
    CK(cudaMemcpyAsync(dv.p, &A.view, sizeof(AgView), cudaMemcpyHostToDevice, ctx->stream), "H2D");
    DBuf<float> b;
    DBuf<uint8_t> baa;
    CK(b.ensure(6 * nb), "alloc");
    CK(cudaMemcpyAsync(b.p, antibody->x, nb * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    CK(cudaMemcpyAsync(b.p + nb, antibody->y, nb * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    CK(cudaMemcpyAsync(b.p + 2 * nb, antibody->z, nb * 4, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    if ((s = upload(ctx, baa, antibody->amino_acid, nb, "aa H2D"))) return s;
    launch_cg_forces(ctx->stream, dv.p, b.p, b.p + nb, b.p + 2 * nb, baa.p, (int)nb, b.p + 3 * nb, b.p + 4 * nb,
                     b.p + 5 * nb);
    LAUNCHED("cg_forces");
    CK(cudaMemcpyAsync(fx, b.p + 3 * nb, nb * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaMemcpyAsync(fy, b.p + 4 * nb, nb * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaMemcpyAsync(fz, b.p + 5 * nb, nb * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_forces_allatom(binder_ctx* ctx, const binder_atom_cloud* antigen, const binder_gpu_atom* candidates,
                          const int64_t* offsets, size_t n_cand, float* out_force, double* out_e) {
    int s = enter(ctx);
    if (s) return s;
    if (n_cand == 0) return BINDER_OK;
    if (!offsets || !out_force) return fail(ctx, BINDER_ERR_ARG, "NULL offsets/out");
    if (offsets[0] != 0) return fail(ctx, BINDER_ERR_ARG, "offsets[0] must be 0");
    for (size_t c = 0; c < n_cand; ++c)
        if (offsets[c + 1] < offsets[c]) return fail(ctx, BINDER_ERR_ARG, "offsets must be non-decreasing");
    const size_t n_atoms = (size_t)offsets[n_cand];
    if ((s = ensure_dropin(ctx, antigen))) return s;
    CK(ctx->cand.ensure(n_atoms * 8), "alloc");
    if (n_atoms)
        CK(cudaMemcpyAsync(ctx->cand.p, candidates, n_atoms * 32, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    if ((s = upload(ctx, ctx->off, (const long long*)offsets, n_cand + 1, "offsets H2D"))) return s;
    CK(ctx->energy.ensure(n_cand), "alloc");
    CK(ctx->force.ensure(3 * n_atoms), "alloc");
    if ((s = clear_err(ctx))) return s;
    ScoreOut o{ctx->energy.p, nullptr, ctx->force.p, nullptr, ctx->errf.p};
    launch_score_flat(ctx->stream, ctx->cand.p, ctx->off.p, (int)n_cand, ctx->d_dropin_view.p, nullptr,
                      ctx->params.accumulate, o, grid_ctas(ctx, (int)n_cand), 256);
    LAUNCHED("score_flat_force");
    ctx->last_batch_valid = false;
    if (n_atoms)
        CK(cudaMemcpyAsync(out_force, ctx->force.p, 3 * n_atoms * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    return fetch_energies(ctx, (int)n_cand, out_e, nullptr, nullptr);
}

int binder_topk_segmented(binder_ctx* ctx, const double* e, const int64_t* seg_off, size_t n_seg, size_t k,
                          int32_t* out) {
    int s = enter(ctx);
    if (s) return s;
    if (n_seg == 0 || k == 0) return BINDER_OK;
    if (!seg_off || !out) return fail(ctx, BINDER_ERR_ARG, "NULL array");
    if (k > 1024) return fail(ctx, BINDER_ERR_ARG, "k must be <= 1024");
    if (seg_off[0] < 0) return fail(ctx, BINDER_ERR_ARG, "negative offset");
    for (size_t i = 0; i < n_seg; ++i)
        if (seg_off[i + 1] < seg_off[i]) return fail(ctx, BINDER_ERR_ARG, "offsets must be non-decreasing");
    const size_t n = (size_t)seg_off[n_seg];
    if (n > (size_t)INT32_MAX) return fail(ctx, BINDER_ERR_ARG, "too many energies");
    if (n && !e) return fail(ctx, BINDER_ERR_ARG, "NULL energies");
    if ((s = upload(ctx, ctx->energy, e, n, "energies H2D"))) return s;
    if ((s = upload(ctx, ctx->tmp_ll, (const long long*)seg_off, n_seg + 1, "offsets H2D"))) return s;
    CK(ctx->topk.ensure(n_seg * k), "alloc");
    launch_topk_segments(ctx->stream, ctx->energy.p, nullptr, ctx->tmp_ll.p, (int)n_seg, (int)k, ctx->topk.p);
    LAUNCHED("topk");
    CK(cudaMemcpyAsync(out, ctx->topk.p, n_seg * k * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_topk(binder_ctx* ctx, const double* e, size_t n, size_t k, int32_t* out) {
    if (!ctx) return BINDER_ERR_ARG;
    if (k > n) return fail(ctx, BINDER_ERR_ARG, "k > n");
    const int64_t off[2] = {0, (int64_t)n};
    return binder_topk_segmented(ctx, e, off, 1, k, out);
}

int binder_build_residues(binder_ctx* ctx, size_t n, const float* ca_xyz, const uint8_t* aa, const float* chi,
                          float* out_pos, float* out_chi) {
    int s = enter(ctx);
    if (s) return s;
    if (n == 0) return BINDER_OK;
    if (!ca_xyz || !aa || !out_pos) return fail(ctx, BINDER_ERR_ARG, "NULL array");
    for (size_t i = 0; i < n; ++i)
        if (aa[i] >= N_AA) return fail(ctx, BINDER_ERR_ARG, "amino acid %d out of range", (int)aa[i]);
    if ((s = upload(ctx, ctx->tmp_f, ca_xyz, 3 * n, "ca H2D"))) return s;
    if ((s = upload(ctx, ctx->tmp_u8, aa, n, "aa H2D"))) return s;
    DBuf<float4> trig;
    DBuf<float> chi_d;
    if (chi) {
        // sin/cos of chi*PI/180 with the host C library, as for the rotamer table
        std::vector<float4> h(2 * n);
        for (size_t r = 0; r < n; ++r) {
            float t[8];
            for (int c = 0; c < 4; ++c) {
                const float x = chi[4 * r + c] * RADS_PER_DEG;
                t[2 * c] = std::sin(x);
                t[2 * c + 1] = std::cos(x);
            }
            h[2 * r] = make_float4(t[0], t[1], t[2], t[3]);
            h[2 * r + 1] = make_float4(t[4], t[5], t[6], t[7]);
        }
        if ((s = upload(ctx, trig, h.data(), 2 * n, "trig H2D"))) return s;
        if ((s = upload(ctx, chi_d, chi, 4 * n, "chi H2D"))) return s;
        CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    }
    CK(ctx->tmp_f4a.ensure(n * SLOT_STRIDE), "alloc");
    CK(ctx->tmp_f4b.ensure(n), "alloc");
    launch_build_residues(ctx->stream, (int)n, ctx->tmp_f.p, ctx->tmp_u8.p, chi ? trig.p : nullptr,
                          chi ? chi_d.p : nullptr, ctx->tmp_f4a.p, ctx->tmp_f4b.p);
    LAUNCHED("build_residues");
    DBuf<float> outd;
    CK(outd.ensure(n * SLOTS * 3), "alloc");
    launch_unpack_slots(ctx->stream, (int)n, ctx->tmp_f4a.p, outd.p);
    LAUNCHED("unpack_slots");
    CK(cudaMemcpyAsync(out_pos, outd.p, n * SLOTS * 3 * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (out_chi) CK(cudaMemcpyAsync(out_chi, ctx->tmp_f4b.p, n * 16, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_add_antigen(binder_ctx* ctx, size_t n_res, const uint8_t* aa, const float* pos, int32_t* out_id) {
    int s = enter(ctx);
    if (s) return s;
    if (n_res == 0 || !aa || !pos) return fail(ctx, BINDER_ERR_ARG, "empty antigen");
    for (size_t r = 0; r < n_res; ++r)
        if (aa[r] >= N_AA) return fail(ctx, BINDER_ERR_ARG, "amino acid out of range");
    // flatten the slot layout into the AtomCloud of push_residue (allatom.rs:201-240)
    std::vector<float> x, y, z, q, rmh, eps;
    std::vector<uint8_t> hyd, type;
    std::vector<float> cx(n_res), cy(n_res), cz(n_res);
    std::vector<float4> ca_atom(n_res), ca_prm(n_res);
    for (size_t r = 0; r < n_res; ++r) {
        const int a = aa[r];
        for (int k = 0; k < BT_TOPO_N[a]; ++k) {
            const float* p = pos + (r * SLOTS + k) * 3;
            const int t = BT_SLOT_TYPE[a][k];
            x.push_back(p[0]); y.push_back(p[1]); z.push_back(p[2]);
            q.push_back(BT_SLOT_Q[a][k]);
            rmh.push_back(BT_NB[t][0]);
            eps.push_back(BT_NB[t][1]);
            hyd.push_back(BT_SLOT_HYD[a][k]);
            type.push_back((uint8_t)t);
        }
        const float* ca = pos + (r * SLOTS + 1) * 3;
        cx[r] = ca[0]; cy[r] = ca[1]; cz[r] = ca[2];
        const int t = BT_SLOT_TYPE[a][1];
        ca_atom[r] = make_float4(ca[0], ca[1], ca[2], BT_SLOT_Q[a][1]);
        ca_prm[r] = make_float4(BT_NB[t][0], BT_NB[t][1], (float)BT_SLOT_HYD[a][1], (float)t);
    }
    std::unique_ptr<Antigen> A(new (std::nothrow) Antigen());
    if (!A) return fail(ctx, BINDER_ERR_OOM, "host allocation");
    if ((s = build_antigen_atoms(ctx, *A, x.data(), y.data(), z.data(), q.data(), rmh.data(), eps.data(), hyd.data(),
                                 type.data(), x.size())))
        return s;
    if ((s = build_antigen_ca(ctx, *A, cx.data(), cy.data(), cz.data(), aa, n_res, ctx->params.ca_cell))) return s;
    if ((s = upload(ctx, A->ca_atom, ca_atom.data(), n_res, "ca atoms"))) return s;
    if ((s = upload(ctx, A->ca_atom_prm, ca_prm.data(), n_res, "ca atoms"))) return s;
    A->view.ca_atom = A->ca_atom.p;
    A->view.ca_atom_prm = A->ca_atom_prm.p;
    // ca_center_of_mass (allatom.rs:183-195): sequential f32 sums
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for (size_t r = 0; r < n_res; ++r) { sx += cx[r]; sy += cy[r]; sz += cz[r]; }
    const float nf = (float)n_res;
    A->view.cx = sx / nf;
    A->view.cy = sy / nf;
    A->view.cz = sz / nf;
    ctx->ags.push_back(std::move(A));
    if ((s = bump_antigen_epoch(ctx))) return s;
    std::vector<AgView> views;
    refresh_views(ctx, views);
    CK(ctx->d_views.ensure(views.size()), "alloc");
    CK(cudaMemcpyAsync(ctx->d_views.p, views.data(), views.size() * sizeof(AgView), cudaMemcpyHostToDevice, ctx->stream),
       "views H2D");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    if (out_id) *out_id = (int32_t)(ctx->ags.size() - 1);
    return BINDER_OK;
}

int binder_clear_antigens(binder_ctx* ctx) {
    int s = enter(ctx);
    if (s) return s;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    ctx->ags.clear();
    ctx->st.n_cand = 0;
    ctx->st.total_res = 0;
    return bump_antigen_epoch(ctx);
}

}  // extern "C"

namespace {
// sin/cos of every chi (the NERF dihedrals of a rejected move's rebuild), computed
// from the uploaded chi with the C library's sinf/cosf of chi * PI/180 as
// place_atom does; the Metropolis kernel keeps them current afterwards.
int ensure_trig(binder_ctx* ctx) {
    State& S = ctx->st;
    if (S.trig_valid) return BINDER_OK;
    const int total = S.total_res;
    // the device chi are still the uploaded ones: only Metropolis steps change chi,
    // and they run after this
    std::vector<float> chi((size_t)4 * std::max(total, 1));
    if (total) {
        CK(cudaMemcpyAsync(chi.data(), S.res_chi.p, (size_t)total * 16, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    }
    std::vector<float4> trig((size_t)2 * std::max(total, 1));
    for (int r = 0; r < total; ++r) {
        float sc[8];
        for (int k = 0; k < 4; ++k) {
            const float x = chi[4 * r + k] * RADS_PER_DEG;
            sc[2 * k] = std::sin(x);
            sc[2 * k + 1] = std::cos(x);
        }
        trig[2 * r] = make_float4(sc[0], sc[1], sc[2], sc[3]);
        trig[2 * r + 1] = make_float4(sc[4], sc[5], sc[6], sc[7]);
    }
    int s = upload(ctx, S.res_trig, trig.data(), trig.size(), "trig");
    if (s) return s;
    S.trig_valid = true;
    return BINDER_OK;
}

// Candidate metadata of the resident state: residue offsets, antigen, Philox id,
// per-antigen candidate groups, sort keys and scratch sizes.
int set_state_meta(binder_ctx* ctx, const std::vector<int>& off, const std::vector<int>& ag,
                   const std::vector<uint32_t>& ids, const std::vector<int>& orig) {
    State& S = ctx->st;
    const size_t n_cand = ag.size();
    const int total = off[n_cand];
    std::vector<int> res_cand(total);
    int max_res = 0;
    for (size_t c = 0; c < n_cand; ++c) {
        max_res = std::max(max_res, off[c + 1] - off[c]);
        for (int r = off[c]; r < off[c + 1]; ++r) res_cand[r] = (int)c;
    }
    // candidates grouped by antigen (stable) for per-antigen survivor selection
    const int n_ag = (int)ctx->ags.size();
    std::vector<long long> g_off(n_ag + 1, 0);
    for (size_t c = 0; c < n_cand; ++c) g_off[ag[c] + 1]++;
    for (int a = 0; a < n_ag; ++a) g_off[a + 1] += g_off[a];
    std::vector<int> g_idx(n_cand);
    std::vector<long long> cur(g_off.begin(), g_off.end() - 1);
    for (size_t c = 0; c < n_cand; ++c) g_idx[cur[ag[c]]++] = (int)c;
    S.n_cand = (int)n_cand;
    S.total_res = total;
    S.max_res = max_res;
    S.h_res_off = off;
    S.h_cand_ag = ag;
    S.h_cand_id = ids;
    S.h_orig = orig;
    S.n_segments = n_ag;
    S.max_segment = 0;
    for (int a = 0; a < n_ag; ++a) S.max_segment = std::max(S.max_segment, g_off[a + 1] - g_off[a]);
    int s;
    if ((s = upload(ctx, S.cand_res_off, off.data(), off.size(), "state")) ||
        (s = upload(ctx, S.cand_ag, ag.data(), ag.size(), "state")) ||
        (s = upload(ctx, S.cand_id, ids.data(), ids.size(), "state")) ||
        (s = upload(ctx, S.res_cand, res_cand.data(), res_cand.size(), "state")) ||
        (s = upload(ctx, S.ag_cand_idx, g_idx.data(), g_idx.size(), "state")) ||
        (s = upload(ctx, S.ag_cand_off, g_off.data(), g_off.size(), "state")))
        return s;
    // sort keys: one range of Calpha-grid cells per antigen
    std::vector<int> kb(n_ag);
    int nk = 0;
    for (int a = 0; a < n_ag; ++a) {
        kb[a] = nk;
        const GridView& g = ctx->ags[a]->view.ca_grid;
        nk += (g.nx + 2 * RES_KEY_MARGIN) * (g.ny + 2 * RES_KEY_MARGIN) * (g.nz + 2 * RES_KEY_MARGIN);
    }
    S.n_keys = nk;
    if ((s = upload(ctx, S.key_base, kb.data(), kb.size(), "state"))) return s;
    CK(S.keys.ensure(std::max(total, 1)), "alloc");
    CK(S.order.ensure(std::max(total, 1)), "alloc");
    // the flat gradient-step kernel's balanced order: epoch, counts and buckets start empty
    CK(S.cg_bal.ensure(cg_bal_ints(std::max(total, 1))), "alloc");
    CK(cudaMemsetAsync(S.cg_bal.p, 0, CG_BAL_HEADER * sizeof(int), ctx->stream), "memset");
    CK(S.key_counts.ensure(nk + 1), "alloc");
    CK(S.key_cursor.ensure(nk + 1), "alloc");
    // scoring and gradient-step work queues ([0], [1]) and their done counts ([2], [3])
    CK(S.queue.ensure(4), "alloc");
    CK(cudaMemsetAsync(S.queue.p, 0, 4 * sizeof(int), ctx->stream), "memset");
    CK(S.res_e.ensure(std::max(total, 1)), "alloc");
    CK(S.res_abs.ensure(std::max(total, 1)), "alloc");
    S.order_valid = false;
    S.meta_epoch = ctx->ag_epoch;
    return BINDER_OK;
}
}  // namespace

extern "C" {

// The upload; sync = wait for the copies (the caller may reuse its arrays at once).
// copy_data false: validate, set the metadata and size the buffers, but leave the
// residue arrays and their packing to the caller (binder_block_io's graph)
static int state_upload_impl(binder_ctx* ctx, size_t n_cand, const int32_t* n_res, int32_t uniform_n_res,
                             const int32_t* antigen_id, const uint32_t* cand_id, const uint8_t* aa,
                             const float* chi, const float* pos, bool sync, bool copy_data = true) {
    int s = enter(ctx);
    if (s) return s;
    if (ctx->ags.empty()) return fail(ctx, BINDER_ERR_STATE, "no antigen added");
    if (n_cand == 0 || n_cand > (size_t)INT32_MAX / 64) return fail(ctx, BINDER_ERR_ARG, "bad candidate count");
    State& S = ctx->st;
    std::vector<int> off(n_cand + 1, 0), ag(n_cand, 0), orig(n_cand);
    std::vector<uint32_t> ids(n_cand);
    for (size_t c = 0; c < n_cand; ++c) {
        const int nr = n_res ? n_res[c] : uniform_n_res;
        if (nr < 0 || nr > 4096) return fail(ctx, BINDER_ERR_ARG, "bad residue count %d", nr);
        off[c + 1] = off[c] + nr;
        ag[c] = antigen_id ? antigen_id[c] : 0;
        if (ag[c] < 0 || ag[c] >= (int)ctx->ags.size()) return fail(ctx, BINDER_ERR_ARG, "bad antigen id");
        ids[c] = cand_id ? cand_id[c] : (uint32_t)c;
        orig[c] = (int)c;
    }
    const int total = off[n_cand];
    if (total > 0 && (!aa || !chi || !pos)) return fail(ctx, BINDER_ERR_ARG, "NULL state array");
    uint8_t aa_max = 0;  // a branch-free scan (vectorised): this runs on every upload
    for (int r = 0; r < total; ++r) aa_max = aa[r] > aa_max ? aa[r] : aa_max;
    if (aa_max >= N_AA) return fail(ctx, BINDER_ERR_ARG, "amino acid out of range");
    // a population of the same shape (candidates, residue counts, antigens, ids)
    // against the same antigen set keeps the device metadata; only the residues move
    ctx->fv_pairs = 0;  // a new population (binder_fv_upload sets it again for an Fv one)
    const bool same_meta = S.n_cand == (int)n_cand && S.meta_epoch == ctx->ag_epoch && S.h_res_off == off &&
                           S.h_cand_ag == ag && S.h_cand_id == ids && S.h_orig == orig;
    if (same_meta) S.order_valid = false;
    else if ((s = set_state_meta(ctx, off, ag, ids, orig))) return s;
    S.trig_valid = false;
    CK(S.res_aa.ensure(total), "alloc");
    CK(S.res_chi.ensure(total), "alloc");
    CK(S.stage.ensure((size_t)total * SLOTS * 3), "alloc");
    CK(S.res_pos.ensure((size_t)total * SLOT_STRIDE), "alloc");
    if (copy_data && total) {
        CK(cudaMemcpyAsync(S.res_aa.p, aa, (size_t)total, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(S.res_chi.p, chi, (size_t)total * 16, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        CK(cudaMemcpyAsync(S.stage.p, pos, (size_t)total * SLOTS * 3 * 4, cudaMemcpyHostToDevice, ctx->stream),
           "H2D");
    }
    if (S.cg_meta.n < (size_t)total || !S.cg_meta.p) {  // fresh list storage: every list invalid
        CK(S.cg_list.ensure((size_t)total * CG_LIST_CAP), "alloc");
        CK(S.cg_centre.ensure(total), "alloc");
        CK(S.cg_meta.ensure(total), "alloc");
        CK(cudaMemsetAsync(S.cg_meta.p, 0xFF, S.cg_meta.n * sizeof(int4), ctx->stream), "memset");
    }
    if (copy_data) {
        launch_pack_slots(ctx->stream, total, S.stage.p, S.res_pos.p);
        if (total) LAUNCHED("pack_slots");
    }
    CK(S.mc_stats.ensure(4 * n_cand), "alloc");
    CK(cudaMemsetAsync(S.mc_stats.p, 0, 4 * n_cand * sizeof(long long), ctx->stream), "memset");
    if (sync) CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_state_upload(binder_ctx* ctx, size_t n_cand, const int32_t* n_res, int32_t uniform_n_res,
                        const int32_t* antigen_id, const uint32_t* cand_id, const uint8_t* aa, const float* chi,
                        const float* pos) {
    return state_upload_impl(ctx, n_cand, n_res, uniform_n_res, antigen_id, cand_id, aa, chi, pos, true);
}

int binder_state_select(binder_ctx* ctx, const int32_t* idx, size_t n) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no state");
    if (n == 0 || !idx) return fail(ctx, BINDER_ERR_ARG, "empty selection");
    std::vector<int> off(n + 1, 0), ag(n), orig(n), map;
    std::vector<uint32_t> ids(n);
    for (size_t j = 0; j < n; ++j) {
        const int c = idx[j];
        if (c < 0 || c >= S.n_cand) return fail(ctx, BINDER_ERR_ARG, "candidate index %d out of range", c);
        off[j + 1] = off[j] + (S.h_res_off[c + 1] - S.h_res_off[c]);
        ag[j] = S.h_cand_ag[c];
        ids[j] = S.h_cand_id[c];
        orig[j] = S.h_orig[c];
        for (int r = S.h_res_off[c]; r < S.h_res_off[c + 1]; ++r) map.push_back(r);
    }
    const int total = off[n];
    ctx->fv_pairs = 0;
    // gather residues (and statistics) into the alternate buffers, then swap them in;
    // chi sin/cos are gathered when current, else derived later for the selection only
    const bool trig = S.trig_valid && S.res_trig.p;
    if ((s = upload(ctx, S.sel_map, map.data(), map.size(), "select")) ||
        (s = upload(ctx, S.sel_cidx, idx, n, "select")))
        return s;
    CK(S.alt_aa.ensure(std::max(total, 1)), "alloc");
    CK(S.alt_chi.ensure(std::max(total, 1)), "alloc");
    CK(S.alt_trig.ensure(2 * std::max(total, 1)), "alloc");
    CK(S.alt_pos.ensure((size_t)std::max(total, 1) * SLOT_STRIDE), "alloc");
    CK(S.alt_stats.ensure(4 * n), "alloc");
    launch_gather_state(ctx->stream, total, S.sel_map.p, S.res_aa.p, S.res_chi.p, trig ? S.res_trig.p : nullptr,
                        S.res_pos.p, S.alt_aa.p, S.alt_chi.p, S.alt_trig.p, S.alt_pos.p, (int)n, S.sel_cidx.p,
                        S.mc_stats.p, S.alt_stats.p);
    LAUNCHED("gather_state");
    S.res_aa.swap(S.alt_aa);
    S.res_chi.swap(S.alt_chi);
    S.res_trig.swap(S.alt_trig);
    S.res_pos.swap(S.alt_pos);
    S.mc_stats.swap(S.alt_stats);
    S.trig_valid = trig;
    if ((s = set_state_meta(ctx, off, ag, ids, orig))) return s;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_state_info(binder_ctx* ctx, int32_t* n_cand, int32_t* total_res, int32_t* orig_idx) {
    int s = enter(ctx);
    if (s) return s;
    const State& S = ctx->st;
    if (n_cand) *n_cand = S.n_cand;
    if (total_res) *total_res = S.total_res;
    if (orig_idx)
        for (int c = 0; c < S.n_cand; ++c) orig_idx[c] = S.h_orig[c];
    return BINDER_OK;
}

int binder_mc_stats(binder_ctx* ctx, int64_t* out, int reset) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no state");
    if (out)
        CK(cudaMemcpyAsync(out, S.mc_stats.p, (size_t)S.n_cand * 4 * sizeof(long long), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "D2H");
    if (reset) CK(cudaMemsetAsync(S.mc_stats.p, 0, (size_t)S.n_cand * 4 * sizeof(long long), ctx->stream), "memset");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_state_download(binder_ctx* ctx, uint8_t* aa, float* chi, float* pos) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no state");
    const int total = S.total_res;
    if (total == 0) return BINDER_OK;
    if (aa) CK(cudaMemcpyAsync(aa, S.res_aa.p, total, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (chi) CK(cudaMemcpyAsync(chi, S.res_chi.p, (size_t)total * 16, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (pos) {
        CK(S.stage.ensure((size_t)total * SLOTS * 3), "alloc");
        launch_unpack_slots(ctx->stream, total, S.res_pos.p, S.stage.p);
        LAUNCHED("unpack_slots");
        CK(cudaMemcpyAsync(pos, S.stage.p, (size_t)total * SLOTS * 3 * 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    }
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

}  // extern "C"

namespace {
StepParams step_params(const binder_params& p) {
    StepParams s;
    s.step = p.step;
    s.noise_base = p.noise_base;
    s.t_hot = p.t_hot;
    s.t_cold = p.t_cold;
    s.mutation_p = p.mutation_p;
    s.rotamer_move_p = p.rotamer_move_p;
    s.backbone_move_p = p.backbone_move_p;
    s.max_torsion_deg = p.max_torsion_deg;
    s.iface_cutoff_sq = p.iface_cutoff_sq;
    s.shell_radius = p.shell_radius;
    s.max_disp = p.max_disp;
    s.restraint_k = p.restraint_k;
    s.seed = p.seed;
    return s;
}

// residues sorted by (antigen, Calpha cell): thread order of the Langevin kernel and
// visiting order of the scoring work queue
int enqueue_order(binder_ctx* ctx) {
    State& S = ctx->st;
    launch_residue_order(ctx->stream, S.view(), ctx->d_views.p, S.key_base.p, S.n_keys, S.keys.p, S.key_counts.p,
                         S.key_cursor.p, S.order.p);
    ctx->launches += 3;
    LAUNCHED("residue_order");
    S.order_valid = true;
    return BINDER_OK;
}

int enqueue_diffuse(binder_ctx* ctx, int n_steps, uint32_t step0, int with_noise, int with_mc, const float* temps) {
    State& S = ctx->st;
    if (temps) {
        int s = upload(ctx, ctx->temps, temps, (size_t)n_steps, "temps H2D");
        if (s) return s;
    }
    if (with_mc) {
        if (S.max_res > ANNEAL_MAX_RES)
            return fail(ctx, BINDER_ERR_ARG, "Metropolis steps hold at most %d residues per candidate", ANNEAL_MAX_RES);
        int s = ensure_trig(ctx);
        if (s) return s;
        int max_ag = 0, max_cells = 0;
        for (const auto& a : ctx->ags) {
            const GridView& g = a->view.ca_grid;
            max_ag = std::max(max_ag, a->n_res);
            max_cells = std::max(max_cells, g.nx * g.ny * g.nz + 1);
        }
        AnnealExtras x;
        if (ctx->mlp.learned) {
            if (!ctx->mlp.ready) return fail(ctx, BINDER_ERR_STATE, "learned proposal without network parameters");
            x.learned = true;
            x.mlp = ctx->mlp.dev();
        }
        if (ctx->mlp.log_cap) {
            x.log = ctx->mlp.log.p;
            x.log_n = ctx->mlp.log_n.p;
            x.log_cap = (long long)ctx->mlp.log_cap;
        }
        CK(launch_anneal(ctx->stream, S.view(), ctx->d_views.p, step_params(ctx->params), n_steps, step0, with_noise,
                         temps ? ctx->temps.p : nullptr, ctx->params.accumulate, S.max_res, max_ag, max_cells,
                         ctx->errf.p, S.mc_stats.p, x),
           "anneal");
        LAUNCHED("anneal");
        S.order_valid = false;  // residues moved: the cell order is stale
        return BINDER_OK;
    }
    int s;
    const int* order = S.order.p;
    if (ctx->cfg.cg_order == 0) {
        if ((s = enqueue_order(ctx))) return s;  // sorted before the steps, kept for the score
    } else {
        S.order_valid = false;  // residues move: the cell order is stale
    }
    // order 3 (work-balanced tasks) is built by the flat kernel for its next launch
    int order_mode = ctx->cfg.cg_order;
    if (order_mode == 3 && (!ctx->cfg.cg_flat || !S.cg_bal.p)) order_mode = 1;
    int max_ag = 0, max_cells = 0;
    for (const auto& a : ctx->ags) {
        const GridView& gv = a->view.ca_grid;
        max_ag = std::max(max_ag, a->n_res);
        max_cells = std::max(max_cells, gv.nx * gv.ny * gv.nz);
    }
    // the antigen every candidate probes, if they share one (staged in shared memory)
    int stage_ag = S.h_cand_ag.empty() ? -1 : S.h_cand_ag[0];
    for (int a : S.h_cand_ag)
        if (a != stage_ag) {
            stage_ag = -1;
            break;
        }
    launch_diffuse(ctx->stream, S.view(), ctx->d_views.p, step_params(ctx->params), n_steps, step0, with_noise,
                   temps ? ctx->temps.p : nullptr, ctx->errf.p, order, ctx->cfg.cg_warps, ctx->cfg.cg_lanes,
                   order_mode, max_ag, max_cells, stage_ag, ctx->cfg.cg_queue ? S.queue.p + 1 : nullptr,
                   ctx->cfg.cg_flat);
    LAUNCHED("diffuse");
    return BINDER_OK;
}

StateScoreScratch score_scratch(binder_ctx* ctx) {
    State& S = ctx->st;
    const bool cell = S.order_valid && ctx->cfg.score_order == 0;
    return StateScoreScratch{cell ? S.order.p : nullptr, S.queue.p, S.res_e.p, S.res_abs.p};
}

int persistent_ctas(binder_ctx* ctx) { return ctx->num_sms * ctx->cfg.score_ctas_per_sm; }

int enqueue_score_state(binder_ctx* ctx, int full) {
    State& S = ctx->st;
    CK(ctx->energy.ensure(S.n_cand), "alloc");
    if (full == 2) {
        launch_mc_energy(ctx->stream, S.view(), ctx->d_views.p, ctx->energy.p);
        LAUNCHED("mc_energy");
        return BINDER_OK;
    }
    if (!S.order_valid && ctx->cfg.score_order == 0) {
        int s = enqueue_order(ctx);
        if (s) return s;
    }
    ScoreOut o{ctx->energy.p, nullptr, nullptr, nullptr, ctx->errf.p};
    ctx->launches += launch_score_state(ctx->stream, S.view(), ctx->d_views.p, ctx->params.accumulate, full, o,
                                        score_scratch(ctx), persistent_ctas(ctx), ctx->cfg.score_warps) - 1;
    LAUNCHED("score_state");
    return BINDER_OK;
}

// Score the resident state and select each segment's stable top-k into ctx->topk:
// one fused launch for the candidate sums and the selection when it fits (k <= 64,
// segments of at most 4096 candidates), else the sums and launch_topk_segments.
int enqueue_score_topk(binder_ctx* ctx, int full, int k, cudaEvent_t mid = nullptr, bool defer = false) {
    State& S = ctx->st;
    if (k <= 0 && !mid) return enqueue_score_state(ctx, full);
    if (k > 0 && full != 2 && S.n_segments > 0 && sum_topk_fits(k, S.max_segment)) {
        CK(ctx->energy.ensure(S.n_cand), "alloc");
        if (!S.order_valid && ctx->cfg.score_order == 0) {
            int s = enqueue_order(ctx);
            if (s) return s;
        }
        ScoreOut o{ctx->energy.p, nullptr, nullptr, nullptr, ctx->errf.p};
        const SumTopk tk{S.ag_cand_idx.p, S.ag_cand_off.p, S.n_segments, k, ctx->topk.p, mid, defer};
        ctx->launches += launch_score_state(ctx->stream, S.view(), ctx->d_views.p, ctx->params.accumulate, full, o,
                                            score_scratch(ctx), persistent_ctas(ctx), ctx->cfg.score_warps, &tk) - 1;
        LAUNCHED("score_state_topk");
        return BINDER_OK;
    }
    int s = enqueue_score_state(ctx, full);
    if (s) return s;
    if (mid) CK(cudaEventRecord(mid, ctx->stream), "event");
    if (k > 0) {
        launch_topk_segments(ctx->stream, ctx->energy.p, S.ag_cand_idx.p, S.ag_cand_off.p, S.n_segments, k,
                             ctx->topk.p);
        LAUNCHED("topk");
    }
    return BINDER_OK;
}

// The candidate sums and top-k of the residue energies the last enqueued block left
// (binder_block without outputs, pipelined graph), on the context stream.
int flush_select(binder_ctx* ctx) {
    State& S = ctx->st;
    ctx->sel_pending = false;
    if (S.n_cand == 0 || ctx->sel_k <= 0) return BINDER_OK;
    const SumTopk tk{S.ag_cand_idx.p, S.ag_cand_off.p, S.n_segments, ctx->sel_k, ctx->topk.p, nullptr, false};
    launch_sum_select(ctx->stream, S.view(), S.res_e.p, 0, ctx->energy.p, tk);
    LAUNCHED("sum_select");
    return BINDER_OK;
}
}  // namespace

extern "C" {

int binder_diffuse(binder_ctx* ctx, int n_steps, uint32_t step0, int with_noise, int with_mc, const float* temps) {
    int s = enter(ctx);
    if (s) return s;
    if (ctx->st.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (n_steps < 0) return fail(ctx, BINDER_ERR_ARG, "negative step count");
    if (n_steps == 0) return BINDER_OK;
    if ((s = clear_err(ctx))) return s;
    if ((s = enqueue_diffuse(ctx, n_steps, step0, with_noise, with_mc, temps))) return s;
    return check_err(ctx);
}

int binder_score_state(binder_ctx* ctx, int full, double* out) {
    int s = enter(ctx);
    if (s) return s;
    if (ctx->st.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (!out) return fail(ctx, BINDER_ERR_ARG, "NULL out");
    if (full < 0 || full > 2) return fail(ctx, BINDER_ERR_ARG, "unknown score mode %d", full);
    if ((s = clear_err(ctx))) return s;
    if ((s = enqueue_score_state(ctx, full))) return s;
    return fetch_energies(ctx, ctx->st.n_cand, out, nullptr, nullptr);
}

}  // extern "C"

namespace {
// One search block on the context stream: n_steps gradient steps (no noise, so
// the steps' Philox counters are not read), one score of every candidate, the k
// lowest per antigen.  ev (4 events) brackets the phases when timing.
int enqueue_block(binder_ctx* ctx, int n_steps, int k, cudaEvent_t* ev) {
    State& S = ctx->st;
    int s;
    if (ev) CK(cudaEventRecord(ev[0], ctx->stream), "event");
    if (n_steps > 0 && (s = enqueue_diffuse(ctx, n_steps, 0, 0, 0, nullptr))) return s;
    if (ev) CK(cudaEventRecord(ev[1], ctx->stream), "event");
    // timed: ev[2] between the residue scoring and the candidate sums + selection
    if ((s = enqueue_score_topk(ctx, 0, k, ev ? ev[2] : nullptr))) return s;
    if (ev) CK(cudaEventRecord(ev[3], ctx->stream), "event");
    return BINDER_OK;
}

// Everything a captured block bakes into its launches: sizes, buffer addresses,
// parameters and launch shapes.  Buffer contents are read at replay time.
std::vector<uint64_t> block_sig(binder_ctx* ctx, int n_steps, int k) {
    const State& S = ctx->st;
    std::vector<uint64_t> v = {
        (uint64_t)n_steps, (uint64_t)k, (uint64_t)S.n_cand, (uint64_t)S.total_res, (uint64_t)S.n_segments,
        (uint64_t)S.n_keys, (uint64_t)ctx->cfg.score_warps, (uint64_t)ctx->cfg.score_ctas_per_sm,
        (uint64_t)ctx->cfg.cg_warps, (uint64_t)ctx->cfg.cg_lanes, (uint64_t)ctx->cfg.cg_order,
        (uint64_t)ctx->cfg.score_order, (uint64_t)ctx->cfg.cg_queue, (uint64_t)ctx->cfg.cg_flat,
        (uint64_t)ctx->ags.size()};
    const void* ptrs[] = {S.cand_res_off.p, S.cand_ag.p, S.cand_id.p, S.res_aa.p, S.res_chi.p, S.res_pos.p,
                          S.res_trig.p, S.res_cand.p, S.ag_cand_idx.p, S.ag_cand_off.p, S.key_base.p, S.keys.p,
                          S.key_counts.p, S.key_cursor.p, S.order.p, S.cg_bal.p, S.queue.p, S.res_e.p,
                          S.res_abs.p,
                          ctx->energy.p, ctx->topk.p, ctx->errf.p, ctx->d_views.p};
    for (const void* q : ptrs) v.push_back((uint64_t)(uintptr_t)q);
    unsigned char pb[sizeof(binder_params)];
    std::memcpy(pb, &ctx->params, sizeof(pb));
    for (size_t i = 0; i < sizeof(pb); i += 8) {
        uint64_t w = 0;
        std::memcpy(&w, pb + i, std::min<size_t>(8, sizeof(pb) - i));
        v.push_back(w);
    }
    return v;
}

// The second stream and its fork / join events (created on first use).
int ensure_side(binder_ctx* ctx) {
    if (!ctx->side) {
        CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking), "stream");
        CK(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming), "event");
        CK(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming), "event");
    }
    return BINDER_OK;
}

// A block of the pipeline: the previous block's candidate sums and top-k on the side
// stream beside this block's gradient steps, then this block's residue energies
// (their sums and top-k follow in the next block, or in flush_select).  The sums
// read only the residue energies, which nothing rewrites before the join.
int enqueue_block_pipe(binder_ctx* ctx, int n_steps, int k) {
    State& S = ctx->st;
    int s;
    CK(cudaEventRecord(ctx->ev_fork, ctx->stream), "event");
    CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0), "event");
    const SumTopk tk{S.ag_cand_idx.p, S.ag_cand_off.p, S.n_segments, k, ctx->topk.p, nullptr, false};
    launch_sum_select(ctx->side, S.view(), S.res_e.p, 0, ctx->energy.p, tk);
    LAUNCHED("sum_select");
    CK(cudaEventRecord(ctx->ev_join, ctx->side), "event");
    if (n_steps > 0 && (s = enqueue_diffuse(ctx, n_steps, 0, 0, 0, nullptr))) return s;
    CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0), "event");
    return enqueue_score_topk(ctx, 0, k, nullptr, true);
}

int capture_pipe(binder_ctx* ctx, int n_steps, int k) {
    ctx->drop_pipe_graph();
    int s = ensure_side(ctx);
    if (s) return s;
    const uint64_t l0 = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    s = enqueue_block_pipe(ctx, n_steps, k);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (s || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        ctx->launches = l0;
        return s ? s : cuda_fail(ctx, e, "end capture");
    }
    e = cudaGraphInstantiate(&ctx->pipe_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        ctx->pipe_graph = nullptr;
        ctx->launches = l0;
        return cuda_fail(ctx, e, "graph instantiate");
    }
    ctx->pipe_graph_launches = (int)(ctx->launches - l0);
    ctx->pipe_graph_order = ctx->st.order_valid;
    ctx->launches = l0;
    ctx->pipe_graph_sig = block_sig(ctx, n_steps, k);
    return BINDER_OK;
}

// Capture enqueue_block into ctx->block_graph (buffers are sized beforehand, so
// the capture allocates nothing).
int capture_block(binder_ctx* ctx, int n_steps, int k) {
    ctx->drop_block_graph();
    const uint64_t l0 = ctx->launches;
    CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    int s = enqueue_block(ctx, n_steps, k, nullptr);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
    if (s || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        ctx->launches = l0;
        return s ? s : cuda_fail(ctx, e, "end capture");
    }
    e = cudaGraphInstantiate(&ctx->block_graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        ctx->block_graph = nullptr;
        ctx->launches = l0;
        return cuda_fail(ctx, e, "graph instantiate");
    }
    ctx->block_graph_launches = (int)(ctx->launches - l0);
    ctx->block_graph_order = ctx->st.order_valid;
    ctx->launches = l0;
    ctx->block_graph_sig = block_sig(ctx, n_steps, k);
    return BINDER_OK;
}

std::string tune_key(binder_ctx* ctx) {
    const State& S = ctx->st;
    std::string k = "sm" + std::to_string(ctx->num_sms) + ":c" + std::to_string(S.n_cand) + ":r" +
                    std::to_string(S.total_res) + ":m" + std::to_string(S.max_res);
    for (const auto& a : ctx->ags) k += ":a" + std::to_string(a->n_atoms) + "/" + std::to_string(a->n_res);
    return k;
}

void tune_cache_load(binder_ctx* ctx) {
    const char* path = std::getenv("BINDER_TUNE_CACHE");
    if (!path || !ctx->tune_cache.empty()) return;
    FILE* f = std::fopen(path, "r");
    if (!f) return;
    char key[1024];
    LaunchCfg c;
    while (std::fscanf(f, "%1023s %d %d %d %d %d %d %d %d", key, &c.score_warps, &c.score_ctas_per_sm, &c.cg_warps,
                       &c.cg_lanes, &c.cg_order, &c.score_order, &c.cg_queue, &c.cg_flat) == 9)
        ctx->tune_cache.emplace_back(key, c);
    std::fclose(f);
}

void tune_cache_store(binder_ctx* ctx, const std::string& key, const LaunchCfg& c) {
    ctx->tune_cache.emplace_back(key, c);
    const char* path = std::getenv("BINDER_TUNE_CACHE");
    if (!path) return;
    FILE* f = std::fopen(path, "a");
    if (!f) return;
    std::fprintf(f, "%s %d %d %d %d %d %d %d %d\n", key.c_str(), c.score_warps, c.score_ctas_per_sm, c.cg_warps,
                 c.cg_lanes, c.cg_order, c.score_order, c.cg_queue, c.cg_flat);
    std::fclose(f);
}

// Median device time (ms) of `reps` runs of fn on the context stream.
template <class F>
int time_ms(binder_ctx* ctx, int reps, F&& fn, float* out) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a), "event");
    CK(cudaEventCreate(&b), "event");
    std::vector<float> t;
    int s = BINDER_OK;
    for (int i = 0; i <= reps && !s; ++i) {
        cudaEventRecord(a, ctx->stream);
        s = fn();
        cudaEventRecord(b, ctx->stream);
        cudaError_t e = cudaEventSynchronize(b);
        if (!s && e != cudaSuccess) s = cuda_fail(ctx, e, "autotune");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (i) t.push_back(ms);  // the first run warms up
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (s) return s;
    std::sort(t.begin(), t.end());
    *out = t[t.size() / 2];
    return BINDER_OK;
}
}  // namespace

extern "C" {

int binder_get_launch_cfg(binder_ctx* ctx, binder_launch_cfg* out) {
    if (!ctx || !out) return BINDER_ERR_ARG;
    out->score_warps = ctx->cfg.score_warps;
    out->score_ctas_per_sm = ctx->cfg.score_ctas_per_sm;
    out->cg_warps = ctx->cfg.cg_warps;
    out->cg_lanes = ctx->cfg.cg_lanes;
    out->cg_order = ctx->cfg.cg_order;
    out->score_order = ctx->cfg.score_order;
    out->cg_queue = ctx->cfg.cg_queue;
    out->cg_flat = ctx->cfg.cg_flat;
    return BINDER_OK;
}

int binder_set_launch_cfg(binder_ctx* ctx, const binder_launch_cfg* c) {
    if (!ctx || !c) return BINDER_ERR_ARG;
    if ((c->score_warps != 4 && c->score_warps != 8 && c->score_warps != 16) || c->score_ctas_per_sm < 1 ||
        c->score_ctas_per_sm > 32 || (c->cg_warps != 2 && c->cg_warps != 4 && c->cg_warps != 8) ||
        (c->cg_lanes != 4 && c->cg_lanes != 8) || (c->cg_lanes == 4 && c->cg_warps == 8) || c->cg_order < 0 ||
        c->cg_order > 3 || c->score_order < 0 || c->score_order > 1 ||
        c->cg_queue < 0 || c->cg_queue > 1 ||
        (c->cg_flat != 0 && c->cg_flat != 4 && c->cg_flat != 8 && c->cg_flat != 16 && c->cg_flat != 32) ||
        (c->cg_flat == 32 && c->cg_warps != 4) || (c->cg_flat && c->cg_warps != 4 && c->cg_warps != 8))
        return fail(ctx, BINDER_ERR_ARG, "unsupported launch shape");
    ctx->cfg.score_warps = c->score_warps;
    ctx->cfg.score_ctas_per_sm = c->score_ctas_per_sm;
    ctx->cfg.cg_warps = c->cg_warps;
    ctx->cfg.cg_lanes = c->cg_lanes;
    ctx->cfg.cg_order = c->cg_order;
    ctx->cfg.score_order = c->score_order;
    ctx->cfg.cg_queue = c->cg_queue;
    ctx->cfg.cg_flat = c->cg_flat;
    return BINDER_OK;
}

int binder_autotune(binder_ctx* ctx, int reps, binder_launch_cfg* out) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (reps < 1) reps = 5;
    tune_cache_load(ctx);
    const std::string key = tune_key(ctx);
    for (const auto& e : ctx->tune_cache)
        if (e.first == key) {
            ctx->cfg = e.second;
            return out ? binder_get_launch_cfg(ctx, out) : BINDER_OK;
        }
    if ((s = clear_err(ctx))) return s;
    CK(ctx->energy.ensure(S.n_cand), "alloc");
    // gradient steps move the candidates: time them on a copy and put the state back
    DBuf<float4> saved;
    const size_t n_slots = (size_t)S.total_res * SLOT_STRIDE;
    CK(saved.ensure(n_slots), "alloc");
    CK(cudaMemcpyAsync(saved.p, S.res_pos.p, n_slots * sizeof(float4), cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    LaunchCfg best = ctx->cfg;
    float best_ms = 1e30f;
    // lane-group shapes (flat 0: lanes x warps) and flat shapes (residues per warp x warps)
    const int shapes[][3] = {{0, 4, 2}, {0, 4, 4}, {0, 8, 2}, {0, 8, 4}, {0, 8, 8},
                             {32, 8, 4}, {16, 8, 4}, {16, 8, 8}, {8, 8, 4}, {8, 8, 8}, {4, 8, 4}, {4, 8, 8}};
    for (int queue : {0, 1})
    for (int order : {0, 1, 2, 3})
        for (const auto& sh : shapes) {
            if (s) break;
            ctx->cfg.cg_flat = sh[0];
            ctx->cfg.cg_lanes = sh[1];
            ctx->cfg.cg_warps = sh[2];
            ctx->cfg.cg_order = order;
            ctx->cfg.cg_queue = queue;
            float ms = 0.f;
            if ((s = time_ms(ctx, reps, [&] { return enqueue_diffuse(ctx, 10, 0, 0, 0, nullptr); }, &ms))) break;
            if (ms < best_ms) {
                best_ms = ms;
                best.cg_flat = sh[0];
                best.cg_warps = sh[2];
                best.cg_lanes = sh[1];
                best.cg_order = order;
                best.cg_queue = queue;
            }
            CK(cudaMemcpyAsync(S.res_pos.p, saved.p, n_slots * sizeof(float4), cudaMemcpyDeviceToDevice,
                               ctx->stream),
               "copy");
        }
    best_ms = 1e30f;
    // the cell order is timed with its sorting launches, as a block after moves runs it
    for (int order : {0, 1})
    for (int nw : {4, 8, 16})
        for (int per_sm : {1, 2, 4, 8}) {
            if (s) break;
            ctx->cfg.score_warps = nw;
            ctx->cfg.score_ctas_per_sm = per_sm;
            ctx->cfg.score_order = order;
            float ms = 0.f;
            auto one = [&] {
                S.order_valid = false;
                return enqueue_score_state(ctx, 0);
            };
            if ((s = time_ms(ctx, reps, one, &ms))) break;
            if (ms < best_ms) {
                best_ms = ms;
                best.score_warps = nw;
                best.score_ctas_per_sm = per_sm;
                best.score_order = order;
            }
        }
    CK(cudaMemcpyAsync(S.res_pos.p, saved.p, n_slots * sizeof(float4), cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    ctx->cfg = best;
    if (s) return s;
    if ((s = check_err(ctx))) return s;
    tune_cache_store(ctx, key, best);
    return out ? binder_get_launch_cfg(ctx, out) : BINDER_OK;
}

int binder_block(binder_ctx* ctx, int n_steps, uint32_t step0, int k, double* out_e, int32_t* out_topk) {
    (void)step0;
    const bool async = out_e == nullptr && out_topk == nullptr;
    int s = async ? enter_keep(ctx) : enter(ctx);  // an enqueued block may take over the pending selection
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (n_steps < 0 || k < 0 || k > 1024) return fail(ctx, BINDER_ERR_ARG, "bad n_steps or k");
    if ((ctx->params.flags & BINDER_FLAG_AUTOTUNE) && !ctx->async_pending) {
        const std::string key = tune_key(ctx);
        bool known = false;
        for (const auto& e : ctx->tune_cache) known |= e.first == key;
        if (!known && (s = binder_autotune(ctx, 5, nullptr))) return s;
    }
    // the device error word accumulates over a run of enqueued blocks until fetched
    if (!ctx->async_pending && (s = clear_err(ctx))) return s;
    ctx->async_pending = async;
    CK(ctx->energy.ensure(S.n_cand), "alloc");
    if (k > 0) CK(ctx->topk.ensure((size_t)S.n_segments * k), "alloc");
    const bool tm = ctx->timing && ctx->ev_blocks < TIMING_RING;
    const bool pipe = async && !tm && (ctx->params.flags & BINDER_FLAG_GRAPH) && k > 0 && S.n_segments > 0 &&
                      sum_topk_fits(k, S.max_segment);
    if (ctx->sel_pending && (!pipe || ctx->sel_k != k) && (s = flush_select(ctx))) return s;
    if (tm) {
        // per-phase events: the launches are issued one by one
        if ((s = enqueue_block(ctx, n_steps, k, &ctx->ev[4 * ctx->ev_blocks]))) return s;
        ctx->ev_blocks++;
    } else if (pipe) {
        if (!ctx->pipe_graph || ctx->pipe_graph_sig != block_sig(ctx, n_steps, k)) {
            if ((s = capture_pipe(ctx, n_steps, k))) return s;
        }
        CK(cudaGraphLaunch(ctx->pipe_graph, ctx->stream), "graph launch");
        ctx->launches += ctx->pipe_graph_launches;
        S.order_valid = ctx->pipe_graph_order;
        ctx->sel_pending = true;
        ctx->sel_k = k;
    } else if (ctx->params.flags & BINDER_FLAG_GRAPH) {
        if (!ctx->block_graph || ctx->block_graph_sig != block_sig(ctx, n_steps, k)) {
            if ((s = capture_block(ctx, n_steps, k))) return s;
        }
        CK(cudaGraphLaunch(ctx->block_graph, ctx->stream), "graph launch");
        ctx->launches += ctx->block_graph_launches;
        S.order_valid = ctx->block_graph_order;
    } else if ((s = enqueue_block(ctx, n_steps, k, nullptr))) {
        return s;
    }
    ctx->last_k = k;
    if (async) return BINDER_OK;
    return binder_block_fetch(ctx, out_e, out_topk);
}

int binder_block_fetch(binder_ctx* ctx, double* out_e, int32_t* out_topk) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    ctx->async_pending = false;
    if (ctx->last_k > 0 && out_topk)
        CK(cudaMemcpyAsync(out_topk, ctx->topk.p, (size_t)S.n_segments * ctx->last_k * sizeof(int),
                           cudaMemcpyDeviceToHost, ctx->stream),
           "D2H");
    return fetch_energies(ctx, S.n_cand, out_e, nullptr, nullptr);
}

int binder_block_io(binder_ctx* ctx, size_t n_cand, const int32_t* n_res, int32_t uniform_n_res,
                    const int32_t* antigen_id, const uint32_t* cand_id, uint8_t* aa, float* chi, float* pos,
                    int n_steps, int k, double* out_e, int32_t* out_topk) {
    if (n_steps < 0 || k < 0 || k > 1024) return fail(ctx, BINDER_ERR_ARG, "bad n_steps or k");
    // the metadata and buffers first; the residue arrays travel with the block
    int s = state_upload_impl(ctx, n_cand, n_res, uniform_n_res, antigen_id, cand_id, aa, chi, pos, false, false);
    if (s) return s;
    State& S = ctx->st;
    if ((s = ensure_side(ctx))) return s;
    bool tuned = true;
    if (ctx->params.flags & BINDER_FLAG_AUTOTUNE) {
        const std::string key = tune_key(ctx);
        bool known = false;
        for (const auto& e : ctx->tune_cache) known |= e.first == key;
        tuned = known;
    }
    ctx->async_pending = false;  // any enqueued blocks ran on the replaced state
    if ((s = clear_err(ctx))) return s;
    CK(ctx->energy.ensure(S.n_cand), "alloc");
    if (k > 0) CK(ctx->topk.ensure((size_t)S.n_segments * k), "alloc");
    CK(ctx->h_energy.ensure(2 * (size_t)S.n_cand), "alloc host");
    ctx->last_k = k;
    const int total = S.total_res;
    if (!tuned) {  // the autotuner times launch shapes on the uploaded state
        if (total) {
            CK(cudaMemcpyAsync(S.res_aa.p, aa, (size_t)total, cudaMemcpyHostToDevice, ctx->stream), "H2D");
            CK(cudaMemcpyAsync(S.res_chi.p, chi, (size_t)total * 16, cudaMemcpyHostToDevice, ctx->stream), "H2D");
            CK(cudaMemcpyAsync(S.stage.p, pos, (size_t)total * SLOTS * 3 * 4, cudaMemcpyHostToDevice, ctx->stream),
               "H2D");
            launch_pack_slots(ctx->stream, total, S.stage.p, S.res_pos.p);
            LAUNCHED("pack_slots");
        }
        if ((s = binder_autotune(ctx, 5, nullptr))) return s;
        if ((s = clear_err(ctx))) return s;
    }
    // the copies in, the block, the moved residues out on the second stream while
    // the first one scores them (both only read the positions), the energies and
    // survivors out: one graph when every host array is pinned (it bakes their
    // addresses in), else the same launches one by one
    auto enqueue = [&]() -> int {
        int e = 0;
        if (total) {
            CK(cudaMemcpyAsync(S.res_aa.p, aa, (size_t)total, cudaMemcpyHostToDevice, ctx->stream), "H2D");
            CK(cudaMemcpyAsync(S.res_chi.p, chi, (size_t)total * 16, cudaMemcpyHostToDevice, ctx->stream), "H2D");
            CK(cudaMemcpyAsync(S.stage.p, pos, (size_t)total * SLOTS * 3 * 4, cudaMemcpyHostToDevice, ctx->stream),
               "H2D");
            launch_pack_slots(ctx->stream, total, S.stage.p, S.res_pos.p);
            LAUNCHED("pack_slots");
        }
        if (n_steps > 0 && (e = enqueue_diffuse(ctx, n_steps, 0, 0, 0, nullptr))) return e;
        CK(cudaEventRecord(ctx->ev_fork, ctx->stream), "event");
        CK(cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0), "event");
        if (total) {
            launch_unpack_slots(ctx->side, total, S.res_pos.p, S.stage.p);
            LAUNCHED("unpack_slots");
            CK(cudaMemcpyAsync(pos, S.stage.p, (size_t)total * SLOTS * 3 * 4, cudaMemcpyDeviceToHost, ctx->side),
               "D2H");
            CK(cudaMemcpyAsync(chi, S.res_chi.p, (size_t)total * 16, cudaMemcpyDeviceToHost, ctx->side), "D2H");
            CK(cudaMemcpyAsync(aa, S.res_aa.p, total, cudaMemcpyDeviceToHost, ctx->side), "D2H");
        }
        CK(cudaEventRecord(ctx->ev_join, ctx->side), "event");
        if ((e = enqueue_score_topk(ctx, 0, k))) return e;
        if (k > 0 && out_topk)
            CK(cudaMemcpyAsync(out_topk, ctx->topk.p, (size_t)S.n_segments * k * sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream),
               "D2H");
        CK(cudaStreamWaitEvent(ctx->stream, ctx->ev_join, 0), "event");
        CK(cudaMemcpyAsync(ctx->h_energy.p, ctx->energy.p, S.n_cand * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "energy D2H");
        return BINDER_OK;
    };
    auto pinned = [](const void* p) {
        if (!p) return true;
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    };
    const bool graph = (ctx->params.flags & BINDER_FLAG_GRAPH) && !ctx->timing && total > 0 && pinned(aa) &&
                       pinned(chi) && pinned(pos) && (k == 0 || !out_topk || pinned(out_topk));
    if (graph) {
        std::vector<uint64_t> sig = block_sig(ctx, n_steps, k);
        for (const void* q : {(const void*)aa, (const void*)chi, (const void*)pos, (const void*)out_topk,
                              (const void*)ctx->h_energy.p, (const void*)S.stage.p, (const void*)ctx->side})
            sig.push_back((uint64_t)(uintptr_t)q);
        if (!ctx->io_graph || ctx->io_graph_sig != sig) {
            ctx->drop_io_graph();
            const uint64_t l0 = ctx->launches;
            CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            s = enqueue();
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
            if (s || e != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                cudaGetLastError();
                ctx->launches = l0;
                return s ? s : cuda_fail(ctx, e, "end capture");
            }
            e = cudaGraphInstantiate(&ctx->io_graph, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                ctx->io_graph = nullptr;
                ctx->launches = l0;
                return cuda_fail(ctx, e, "graph instantiate");
            }
            ctx->io_graph_launches = (int)(ctx->launches - l0);
            ctx->io_graph_order = S.order_valid;
            ctx->launches = l0;
            ctx->io_graph_sig = sig;
        }
        CK(cudaGraphLaunch(ctx->io_graph, ctx->stream), "graph launch");
        ctx->launches += ctx->io_graph_launches;
        S.order_valid = ctx->io_graph_order;
    } else if ((s = enqueue())) {
        return s;
    }
    if ((s = check_err(ctx))) return s;  // synchronises; the side stream joined before the energies
    if (out_e) std::memcpy(out_e, ctx->h_energy.p, S.n_cand * sizeof(double));
    return BINDER_OK;
}

void binder_default_run_cfg(binder_run_cfg* c) {
    if (!c) return;
    c->phase1_steps = 200;
    c->score_every = 10;
    c->survivors = 64;
    c->phase2_steps = 600;
    c->top_n = 64;
    c->phase1_mc = 0;
}

int binder_run_allatom(binder_ctx* ctx, const binder_run_cfg* cfg_in, int32_t* out_cand, double* out_energy) {
    int s = enter(ctx);
    if (s) return s;
    binder_run_cfg cfg;
    if (cfg_in) cfg = *cfg_in;
    else binder_default_run_cfg(&cfg);
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (cfg.phase1_steps < 0 || cfg.phase2_steps < 0 || cfg.survivors < 1 || cfg.survivors > 1024 || cfg.top_n < 1 ||
        cfg.top_n > 1024)
        return fail(ctx, BINDER_ERR_ARG, "bad run configuration");
    const binder_params& P = ctx->params;
    // temperature (diffusion.rs:102-104): phase 1 on the schedule of both phases
    // (diffusion.rs:1019), phase 2 on its own (:1089)
    auto temp = [&](int iter, int total) {
        return P.t_hot * std::pow(P.t_cold / P.t_hot, (float)iter / (float)total);
    };
    const int n1 = cfg.phase1_steps, n2 = cfg.phase2_steps;
    std::vector<float> t1(std::max(n1, 1)), t2(std::max(n2, 1));
    for (int i = 0; i < n1; ++i) t1[i] = temp(i, n1 + n2);
    for (int i = 0; i < n2; ++i) t2[i] = temp(i, n2);
    const int k1 = cfg.survivors;
    CK(ctx->topk.ensure((size_t)S.n_segments * std::max(k1, cfg.top_n)), "alloc");
    CK(ctx->energy.ensure(S.n_cand), "alloc");  // before the block graph's capture
    if ((s = clear_err(ctx))) return s;
    // ---- phase 1: blocks of score_every steps, each scored with its survivors ----
    const int per = cfg.score_every > 0 ? cfg.score_every : std::max(n1, 1);
    // gradient-only blocks are the search block: replayed from its CUDA graph
    const bool graph = (P.flags & BINDER_FLAG_GRAPH) && !cfg.phase1_mc && !ctx->timing;
    int s0 = 0;
    do {
        const int ns = std::min(per, n1 - s0);
        if (graph) {
            if (!ctx->block_graph || ctx->block_graph_sig != block_sig(ctx, ns, k1)) {
                if ((s = capture_block(ctx, ns, k1))) return s;
            }
            CK(cudaGraphLaunch(ctx->block_graph, ctx->stream), "graph launch");
            ctx->launches += ctx->block_graph_launches;
            S.order_valid = ctx->block_graph_order;
        } else {
            if (ns > 0 && (s = enqueue_diffuse(ctx, ns, (uint32_t)s0, 0, cfg.phase1_mc, &t1[s0]))) return s;
            if ((s = enqueue_score_topk(ctx, 0, k1))) return s;
        }
        s0 += std::max(ns, 1);
    } while (s0 < n1);
    if ((s = check_err(ctx))) return s;
    std::vector<int32_t> top((size_t)S.n_segments * k1);
    CK(cudaMemcpyAsync(top.data(), ctx->topk.p, top.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream),
       "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    std::vector<int32_t> surv;
    for (int32_t i : top)
        if (i >= 0) surv.push_back(i);
    if ((s = binder_state_select(ctx, surv.data(), surv.size()))) return s;
    // ---- phase 2: Langevin + Metropolis on the survivors (diffusion.rs:1083-1095) ----
    if ((s = clear_err(ctx))) return s;
    if (n2 > 0 && (s = enqueue_diffuse(ctx, n2, (uint32_t)n1, 1, 1, t2.data()))) return s;
    // final allatom_energy and ranking (diffusion.rs:1092-1098)
    const int k2 = cfg.top_n;
    if ((s = enqueue_score_topk(ctx, 1, k2))) return s;
    std::vector<double> e(S.n_cand);
    std::vector<int32_t> rank((size_t)S.n_segments * k2);
    if ((s = fetch_energies(ctx, S.n_cand, e.data(), nullptr, nullptr))) return s;
    CK(cudaMemcpyAsync(rank.data(), ctx->topk.p, rank.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream),
       "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    std::vector<int32_t> keep;
    for (size_t j = 0; j < rank.size(); ++j) {
        const int32_t i = rank[j];
        if (out_cand) out_cand[j] = i >= 0 ? S.h_orig[i] : -1;
        if (out_energy) out_energy[j] = i >= 0 ? e[i] : std::nan("");
        if (i >= 0) keep.push_back(i);
    }
    // the resident state becomes the results in rank order
    return binder_state_select(ctx, keep.data(), keep.size());
}

int binder_minimize(binder_ctx* ctx, int steps, double* out_energy) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (steps < 0) return fail(ctx, BINDER_ERR_ARG, "negative step count");
    if ((s = ensure_trig(ctx))) return s;
    if ((s = clear_err(ctx))) return s;
    DBuf<float4> trial;
    DBuf<double> best, e_trial;
    CK(trial.ensure((size_t)S.total_res * SLOT_STRIDE), "alloc");
    CK(best.ensure(S.n_cand), "alloc");
    CK(e_trial.ensure(S.n_cand), "alloc");
    // the energy minimize starts from (partners_energy, diffusion.rs:859)
    if ((s = enqueue_score_state(ctx, 1))) return s;
    CK(cudaMemcpyAsync(best.p, ctx->energy.p, S.n_cand * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream),
       "copy");
    StateView tv = S.view();
    tv.res_pos = trial.p;
    const StateScoreScratch scr{nullptr, S.queue.p, S.res_e.p, S.res_abs.p};
    const ScoreOut o{e_trial.p, nullptr, nullptr, nullptr, ctx->errf.p};
    for (int step = 0; step < steps; ++step) {
        // step size decaying linearly to zero (diffusion.rs:880-881), f32 as the reference
        const float frac = 1.0f - (float)step / (float)steps;
        const float step_size = 0.04f * frac;
        launch_min_move(ctx->stream, S.view(), ctx->d_views.p, S.res_pos.p, trial.p, step_size);
        LAUNCHED("min_move");
        ctx->launches += launch_score_state(ctx->stream, tv, ctx->d_views.p, ctx->params.accumulate, 1, o, scr,
                                            persistent_ctas(ctx), ctx->cfg.score_warps) - 1;
        LAUNCHED("score_state");
        launch_min_accept(ctx->stream, S.view(), trial.p, e_trial.p, best.p, nullptr);
        LAUNCHED("min_accept");
    }
    S.order_valid = false;  // residues moved
    if ((s = check_err(ctx))) return s;
    if (out_energy)
        CK(cudaMemcpyAsync(out_energy, best.p, S.n_cand * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_affinity_maturation(binder_ctx* ctx, double* out_energy, int32_t* out_mutated) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if (S.max_res > ANNEAL_MAX_RES)
        return fail(ctx, BINDER_ERR_ARG, "affinity maturation holds at most %d residues per candidate", ANNEAL_MAX_RES);
    if ((s = ensure_trig(ctx))) return s;
    if ((s = clear_err(ctx))) return s;
    DBuf<double> best;
    DBuf<int> kept;
    CK(best.ensure(S.n_cand), "alloc");
    CK(kept.ensure(S.n_cand), "alloc");
    // per-residue full energies of the state (the scan changes one residue at a time)
    if ((s = enqueue_score_state(ctx, 1))) return s;
    launch_mature(ctx->stream, S.view(), ctx->d_views.p, S.res_e.p, best.p, kept.p, ctx->errf.p);
    LAUNCHED("mature");
    S.order_valid = false;
    if ((s = check_err(ctx))) return s;
    if (out_energy)
        CK(cudaMemcpyAsync(out_energy, best.p, S.n_cand * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if (out_mutated)
        CK(cudaMemcpyAsync(out_mutated, kept.p, S.n_cand * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_validate(binder_ctx* ctx, int32_t* out_clashes, int32_t* out_rama) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    if ((s = clear_err(ctx))) return s;
    DBuf<int> counts;
    CK(counts.ensure(2 * (size_t)S.n_cand), "alloc");
    if (S.max_res > 640) return fail(ctx, BINDER_ERR_ARG, "validation holds at most 640 residues per candidate");
    CK(launch_validate(ctx->stream, S.view(), counts.p, counts.p + S.n_cand), "validate");
    LAUNCHED("validate");
    std::vector<int> h(2 * (size_t)S.n_cand);
    CK(cudaMemcpyAsync(h.data(), counts.p, h.size() * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if ((s = check_err(ctx))) return s;  // synchronises
    for (int c = 0; c < S.n_cand; ++c) {
        if (out_clashes) out_clashes[c] = h[c];
        if (out_rama) out_rama[c] = h[S.n_cand + c];
    }
    return BINDER_OK;
}

int binder_fv_upload(binder_ctx* ctx, size_t n_cand, int32_t n_heavy, int32_t n_light, const uint8_t* aa_h,
                     const float* chi_h, const float* pos_h, const uint8_t* cdr_h, const uint8_t* aa_l,
                     const float* chi_l, const float* pos_l, const uint8_t* cdr_l, int32_t antigen_id,
                     const uint32_t* cand_id) {
    int s = enter(ctx);
    if (s) return s;
    if (n_cand == 0 || n_heavy <= 0 || n_light <= 0 || n_heavy > ANNEAL_MAX_RES || n_light > ANNEAL_MAX_RES)
        return fail(ctx, BINDER_ERR_ARG, "Fv chains hold 1..%d residues", ANNEAL_MAX_RES);
    if (!aa_h || !chi_h || !pos_h || !cdr_h || !aa_l || !chi_l || !pos_l || !cdr_l)
        return fail(ctx, BINDER_ERR_ARG, "NULL chain array");
    // interleave: chain 2i = heavy i, 2i + 1 = light i; both chains draw with candidate id i
    const size_t per = (size_t)n_heavy + n_light, total = n_cand * per;
    std::vector<int32_t> nres(2 * n_cand), agid(2 * n_cand, antigen_id);
    std::vector<uint32_t> ids(2 * n_cand);
    std::vector<uint8_t> aa(total), cdr(total);
    std::vector<float> chi(total * 4), pos(total * SLOTS * 3);
    for (size_t i = 0; i < n_cand; ++i) {
        nres[2 * i] = n_heavy;
        nres[2 * i + 1] = n_light;
        ids[2 * i] = ids[2 * i + 1] = cand_id ? cand_id[i] : (uint32_t)i;
        const size_t o = i * per;
        std::memcpy(&aa[o], aa_h + i * n_heavy, n_heavy);
        std::memcpy(&aa[o + n_heavy], aa_l + i * n_light, n_light);
        std::memcpy(&cdr[o], cdr_h + i * n_heavy, n_heavy);
        std::memcpy(&cdr[o + n_heavy], cdr_l + i * n_light, n_light);
        std::memcpy(&chi[o * 4], chi_h + i * n_heavy * 4, n_heavy * 16);
        std::memcpy(&chi[(o + n_heavy) * 4], chi_l + i * n_light * 4, n_light * 16);
        std::memcpy(&pos[o * SLOTS * 3], pos_h + i * n_heavy * SLOTS * 3, (size_t)n_heavy * SLOTS * 12);
        std::memcpy(&pos[(o + n_heavy) * SLOTS * 3], pos_l + i * n_light * SLOTS * 3, (size_t)n_light * SLOTS * 12);
    }
    if ((s = state_upload_impl(ctx, 2 * n_cand, nres.data(), 0, agid.data(), ids.data(), aa.data(), chi.data(),
                                pos.data(), true)))
        return s;
    if ((s = upload(ctx, ctx->fv_cdr, cdr.data(), total, "cdr"))) return s;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    ctx->fv_pairs = (int)n_cand;
    return BINDER_OK;
}

int binder_fv_run(binder_ctx* ctx, int iterations, double* out_energy) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (ctx->fv_pairs <= 0 || S.n_cand != 2 * ctx->fv_pairs)
        return fail(ctx, BINDER_ERR_STATE, "no Fv population uploaded");
    if (iterations < 0) return fail(ctx, BINDER_ERR_ARG, "negative iteration count");
    const int np = ctx->fv_pairs;
    if ((s = ensure_trig(ctx))) return s;
    if ((s = clear_err(ctx))) return s;
    // temperature (diffusion.rs:102-104) of every iteration (diffusion.rs:792)
    const binder_params& P = ctx->params;
    std::vector<float> t(std::max(iterations, 1));
    for (int it = 0; it < iterations; ++it)
        t[it] = P.t_hot * std::pow(P.t_cold / P.t_hot, (float)it / (float)iterations);
    if ((s = upload(ctx, ctx->temps, t.data(), t.size(), "temps"))) return s;
    CK(ctx->energy.ensure(S.n_cand), "alloc");
    CK(ctx->fv_best.ensure(np), "alloc");
    CK(ctx->fv_pair_e.ensure(np), "alloc");
    CK(ctx->fv_bpos.ensure((size_t)S.total_res * SLOT_STRIDE), "alloc");
    CK(ctx->fv_baa.ensure(S.total_res), "alloc");
    CK(ctx->fv_bchi.ensure(S.total_res), "alloc");
    CK(ctx->fv_btrig.ensure(2 * (size_t)S.total_res), "alloc");
    int max_ag = 0, max_cells = 0;
    for (const auto& a : ctx->ags) {
        const GridView& g = a->view.ca_grid;
        max_ag = std::max(max_ag, a->n_res);
        max_cells = std::max(max_cells, g.nx * g.ny * g.nz + 1);
    }
    const StepParams sp = step_params(P);
    AnnealExtras none;
    // fv_energy of the pairs as they are (the first best)
    auto energies_and_keep = [&](int restore) -> int {
        int st_ = enqueue_score_state(ctx, 1);  // each chain vs the antigen + its disulfide term
        if (st_) return st_;
        launch_fv_pair(ctx->stream, S.view(), ctx->fv_pair_e.p);
        LAUNCHED("fv_pair");
        launch_fv_keep(ctx->stream, S.view(), ctx->energy.p, ctx->fv_pair_e.p, ctx->fv_best.p, ctx->fv_bpos.p,
                       ctx->fv_baa.p, ctx->fv_bchi.p, ctx->fv_btrig.p, restore);
        LAUNCHED("fv_keep");
        return BINDER_OK;
    };
    if ((s = energies_and_keep(2))) return s;
    for (int it = 0; it < iterations; ++it) {
        // heavy chains against the light chains as they are, then light against heavy
        for (int chain = 0; chain < 2; ++chain) {
            CK(launch_anneal(ctx->stream, S.view(), ctx->d_views.p, sp, 1, (uint32_t)it, 1, ctx->temps.p + it,
                             P.accumulate, S.max_res, max_ag, max_cells, ctx->errf.p, S.mc_stats.p, none, chain,
                             ctx->fv_cdr.p),
               "fv step");
            LAUNCHED("fv_step");
        }
        if ((s = energies_and_keep(0))) return s;
    }
    // the result is the best pair of every candidate
    launch_fv_keep(ctx->stream, S.view(), ctx->energy.p, ctx->fv_pair_e.p, ctx->fv_best.p, ctx->fv_bpos.p,
                   ctx->fv_baa.p, ctx->fv_bchi.p, ctx->fv_btrig.p, 1);
    LAUNCHED("fv_keep");
    S.order_valid = false;
    if ((s = check_err(ctx))) return s;
    if (out_energy)
        CK(cudaMemcpyAsync(out_energy, ctx->fv_best.p, np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
           "D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

void* binder_stream(binder_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int binder_set_timing(binder_ctx* ctx, int on) {
    int s = enter(ctx);
    if (s) return s;
    if (ctx->ev.empty()) {
        ctx->ev.assign(4 * TIMING_RING, nullptr);
        for (auto& e : ctx->ev) CK(cudaEventCreate(&e), "event");
    }
    ctx->timing = on != 0;
    ctx->ev_blocks = 0;
    return BINDER_OK;
}

int binder_timing_summary(binder_ctx* ctx, double* sums, int32_t* n_blocks) {
    int s = enter(ctx);
    if (s) return s;
    if (!sums) return fail(ctx, BINDER_ERR_ARG, "NULL out");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    sums[0] = sums[1] = sums[2] = 0.0;
    for (int b = 0; b < ctx->ev_blocks; ++b)
        for (int i = 0; i < 3; ++i) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, ctx->ev[4 * b + i], ctx->ev[4 * b + i + 1]), "event");
            sums[i] += ms;
        }
    if (n_blocks) *n_blocks = ctx->ev_blocks;
    ctx->ev_blocks = 0;
    return BINDER_OK;
}

int binder_state_pair_counts(binder_ctx* ctx, int n_steps, int64_t* out_cg, int64_t* out_score) {
    int s = enter(ctx);
    if (s) return s;
    State& S = ctx->st;
    if (S.n_cand == 0) return fail(ctx, BINDER_ERR_STATE, "no candidates uploaded");
    CK(ctx->pairs.ensure(2), "alloc");
    CK(cudaMemsetAsync(ctx->pairs.p, 0, 2 * sizeof(long long), ctx->stream), "memset");
    if ((s = clear_err(ctx))) return s;
    launch_diffuse_count(ctx->stream, S.view(), ctx->d_views.p, step_params(ctx->params), n_steps, ctx->pairs.p);
    if (n_steps > 0) LAUNCHED("diffuse_count");
    launch_score_state_count(ctx->stream, S.view(), ctx->d_views.p, ctx->pairs.p + 1, ctx->errf.p,
                             score_scratch(ctx), persistent_ctas(ctx));
    LAUNCHED("score_state_count");
    long long h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, ctx->pairs.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
    if ((s = check_err(ctx))) return s;
    if (out_cg) *out_cg = h[0];
    if (out_score) *out_score = h[1];
    return BINDER_OK;
}

int binder_fp32_peak(binder_ctx* ctx, double* scalar, double* packed) {
    int s = enter(ctx);
    if (s) return s;
    DBuf<float> scratch;
    const int ctas = ctx->num_sms * 8;
    CK(scratch.ensure(ctas), "alloc");
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a), "event");
    CK(cudaEventCreate(&b), "event");
    for (int v = 0; v < 2; ++v) {
        double best = 0.0;
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(a, ctx->stream);
            const double flops = launch_ffma(ctx->stream, scratch.p, ctas, 2048, v == 1);
            ctx->launches++;
            cudaEventRecord(b, ctx->stream);
            cudaError_t e = cudaEventSynchronize(b);
            if (e != cudaSuccess) {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
                return cuda_fail(ctx, e, "ffma");
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0) best = std::max(best, flops / (ms * 1e-3) / 1e12);
        }
        if (v == 0 && scalar) *scalar = best;
        if (v == 1 && packed) *packed = best;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return BINDER_OK;
}

}  // extern "C"

// ---- learned proposal network: host side of k_mlp.cu ----------------------------------
namespace {

int round_up(int x, int m) { return (x + m - 1) / m * m; }

// activations for up to `rows` rows (rounded up to the 128-row GEMM tile)
int mlp_reserve(binder_ctx* ctx, int rows) {
    MlpState& M = ctx->mlp;
    const int cap = round_up(std::max(rows, 1), 128);
    if (cap <= M.cap) return BINDER_OK;
    const size_t c = (size_t)cap;
    CK(M.X.ensure(c * MLP_K1), "mlp alloc");
    CK(M.Xt.ensure(c * MLP_K1), "mlp alloc");
    CK(M.H1.ensure(c * MLP_H), "mlp alloc");
    CK(M.H1t.ensure(c * MLP_H), "mlp alloc");
    CK(M.H2.ensure(c * MLP_H), "mlp alloc");
    CK(M.H2t.ensure(c * MLP_H), "mlp alloc");
    CK(M.dY.ensure(c * MLP_OUT_PAD), "mlp alloc");
    CK(M.dYt.ensure(c * MLP_OUT_PAD), "mlp alloc");
    CK(M.dZ2.ensure(c * MLP_H), "mlp alloc");
    CK(M.dZ2t.ensure(c * MLP_H), "mlp alloc");
    CK(M.dZ1t.ensure(c * MLP_H), "mlp alloc");
    CK(M.S1.ensure(c * MLP_H), "mlp alloc");
    CK(M.S2.ensure(c * MLP_H), "mlp alloc");
    CK(M.Y.ensure(c * MLP_OUT_PAD), "mlp alloc");
    CK(M.feat.ensure(c * MLP_IN), "mlp alloc");
    CK(M.ca.ensure(c * 3), "mlp alloc");
    CK(M.target.ensure(c), "mlp alloc");
    CK(M.aa.ensure(c), "mlp alloc");
    CK(M.ag.ensure(c), "mlp alloc");
    CK(M.action.ensure(c), "mlp alloc");
    CK(M.ref.ensure(c), "mlp alloc");
    CK(M.idx.ensure(c), "mlp alloc");
    M.cap = cap;
    return BINDER_OK;
}

constexpr int MLP_KSPLIT = 512;  // batch rows per split-K slice of the weight-gradient GEMMs

int gemm(binder_ctx* ctx, const GemmArgs& g, const char* what) {
    CK(launch_gemm_tc(ctx->stream, g, ctx->errf.p), what);
    ctx->launches++;
    return BINDER_OK;
}

// Forward pass of rows 0..m-1 of M.X (BF16, rows up to m_pad zero).  train keeps
// what the backward pass needs (pre-activations and transposed activations).
int mlp_forward_dev(binder_ctx* ctx, int m, bool train) {
    MlpState& M = ctx->mlp;
    const int mp = round_up(m, 128);
    int s;
    GemmArgs g;
    // layer 1: Z1 = X W1^T + b1, H1 = silu(Z1)
    g.a = M.X.p; g.lda = MLP_K1; g.m = mp;
    g.b = M.w1.p; g.ldb = MLP_K1; g.n = MLP_H; g.k = MLP_K1; g.k_split = MLP_K1;
    g.e = GemmEpi{};
    g.e.mode = EPI_SILU; g.e.bias = M.w.p + MLP_OFF_B1;
    g.e.sp = train ? M.S1.p : nullptr; g.e.ldsp = MLP_H;
    g.e.h = M.H1.p; g.e.ldh = MLP_H; g.e.h_rows = mp;
    g.e.ht = train ? M.H1t.p : nullptr; g.e.ldht = mp; g.e.ht_rows = mp;
    g.e.n_valid = MLP_H; g.e.m_valid = m;
    if ((s = gemm(ctx, g, "mlp layer 1"))) return s;
    // layer 2
    g.a = M.H1.p; g.lda = MLP_H; g.b = M.w2.p; g.ldb = MLP_H; g.k = MLP_H; g.k_split = MLP_H;
    g.e.bias = M.w.p + MLP_OFF_B2; g.e.sp = train ? M.S2.p : nullptr;
    g.e.h = M.H2.p; g.e.ht = train ? M.H2t.p : nullptr;
    if ((s = gemm(ctx, g, "mlp layer 2"))) return s;
    // layer 3: Y = H2 W3^T + b3 (FP32)
    g.a = M.H2.p; g.lda = MLP_H; g.b = M.w3.p; g.ldb = MLP_H; g.n = MLP_OUT_PAD; g.k = MLP_H; g.k_split = MLP_H;
    g.e = GemmEpi{};
    g.e.mode = EPI_F32; g.e.bias = M.w.p + MLP_OFF_B3; g.e.c = M.Y.p; g.e.ldc = MLP_OUT_PAD;
    g.e.n_valid = MLP_OUT_PAD; g.e.m_valid = mp;
    return gemm(ctx, g, "mlp layer 3");
}

// dW = G^T * A over the batch: G^T [rows][mp] and A^T [n][mp] (BF16), split-K
// partials reduced in a fixed order into grad (FP32 [rows][n]).
int mlp_weight_grad(binder_ctx* ctx, const __nv_bfloat16* Gt, int rows, const __nv_bfloat16* At, int n, int mp,
                    float* grad) {
    MlpState& M = ctx->mlp;
    const int slices = (mp + MLP_KSPLIT - 1) / MLP_KSPLIT;
    const long long stride = (long long)rows * n;
    CK(M.part.ensure((size_t)slices * stride), "mlp alloc");
    GemmArgs g;
    g.a = Gt; g.lda = mp; g.m = rows;
    g.b = At; g.ldb = mp; g.n = n; g.k = mp; g.k_split = MLP_KSPLIT;
    g.e.mode = EPI_PARTIAL; g.e.c = M.part.p; g.e.ldc = n; g.e.part_stride = stride;
    g.e.n_valid = n; g.e.m_valid = rows;
    int s = gemm(ctx, g, "mlp weight grad");
    if (s) return s;
    launch_reduce_partials(ctx->stream, (int)stride, slices, stride, M.part.p, grad);
    LAUNCHED("mlp reduce");
    return BINDER_OK;
}

// Loss and gradient of the batch in M.X / M.action / M.target (m rows; reference
// outputs in M.ref when with_ref) into M.g.
int mlp_backward_dev(binder_ctx* ctx, int m, float delta, bool with_ref) {
    MlpState& M = ctx->mlp;
    const int mp = round_up(m, 128);
    int s;
    launch_mlp_loss(ctx->stream, m, mp, M.Y.p, M.action.p, with_ref ? M.ref.p : nullptr, M.target.p, delta, M.dY.p,
                    M.dYt.p, M.loss.p);
    LAUNCHED("mlp loss");
    // layer 3: dW3 = dY^T H2, db3 = colsum dY, dZ2 = (dY W3) * silu'(Z2)
    if ((s = mlp_weight_grad(ctx, M.dYt.p, MLP_OUT_PAD, M.H2t.p, MLP_H, mp, M.g.p + MLP_OFF_W3))) return s;
    launch_rowsum_bf16(ctx->stream, MLP_OUT_PAD, mp, mp, M.dYt.p, M.g.p + MLP_OFF_B3);
    LAUNCHED("mlp bias grad");
    GemmArgs g;
    g.a = M.dY.p; g.lda = MLP_OUT_PAD; g.m = mp;
    g.b = M.w3t.p; g.ldb = MLP_OUT_PAD; g.n = MLP_H; g.k = MLP_OUT_PAD; g.k_split = 64;
    g.e.mode = EPI_DSILU; g.e.sp = M.S2.p; g.e.ldsp = MLP_H;
    g.e.h = M.dZ2.p; g.e.ldh = MLP_H; g.e.h_rows = mp;
    g.e.ht = M.dZ2t.p; g.e.ldht = mp; g.e.ht_rows = mp;
    g.e.n_valid = MLP_H; g.e.m_valid = m;
    if ((s = gemm(ctx, g, "mlp dZ2"))) return s;
    // layer 2: dW2 = dZ2^T H1, db2, dZ1 = (dZ2 W2) * silu'(Z1)
    if ((s = mlp_weight_grad(ctx, M.dZ2t.p, MLP_H, M.H1t.p, MLP_H, mp, M.g.p + MLP_OFF_W2))) return s;
    launch_rowsum_bf16(ctx->stream, MLP_H, mp, mp, M.dZ2t.p, M.g.p + MLP_OFF_B2);
    LAUNCHED("mlp bias grad");
    g.a = M.dZ2.p; g.lda = MLP_H; g.b = M.w2t.p; g.ldb = MLP_H; g.k = MLP_H; g.k_split = MLP_H;
    g.e.sp = M.S1.p; g.e.h = nullptr; g.e.ht = M.dZ1t.p;
    if ((s = gemm(ctx, g, "mlp dZ1"))) return s;
    // layer 1: dW1 = dZ1^T X, db1
    if ((s = mlp_weight_grad(ctx, M.dZ1t.p, MLP_H, M.Xt.p, MLP_K1, mp, M.g.p + MLP_OFF_W1))) return s;
    launch_rowsum_bf16(ctx->stream, MLP_H, mp, mp, M.dZ1t.p, M.g.p + MLP_OFF_B1);
    LAUNCHED("mlp bias grad");
    return BINDER_OK;
}

int mlp_check_ready(binder_ctx* ctx) {
    if (!ctx->mlp.ready) return fail(ctx, BINDER_ERR_STATE, "proposal network has no parameters (binder_mlp_set_params)");
    return BINDER_OK;
}

int mlp_pack(binder_ctx* ctx) {
    launch_pack_weights(ctx->stream, ctx->mlp.w.p, ctx->mlp.bf16());
    LAUNCHED("mlp pack weights");
    return BINDER_OK;
}

}  // namespace

extern "C" {

int binder_mlp_set_params(binder_ctx* ctx, const float* params) {
    int s = enter(ctx);
    if (s) return s;
    if (!params) return fail(ctx, BINDER_ERR_ARG, "NULL parameters");
    MlpState& M = ctx->mlp;
    for (int i = 0; i < MLP_N_PARAMS; ++i)
        if (!std::isfinite(params[i])) return fail(ctx, BINDER_ERR_NAN, "non-finite parameter %d", i);
    // padding entries (W1 columns >= 180, W3 rows and b3 entries >= 25) must be zero
    for (int n = 0; n < MLP_H; ++n)
        for (int k = MLP_IN; k < MLP_K1; ++k)
            if (params[MLP_OFF_W1 + n * MLP_K1 + k] != 0.0f) return fail(ctx, BINDER_ERR_ARG, "W1 padding not zero");
    for (int i = MLP_OUT * MLP_H; i < MLP_OUT_PAD * MLP_H; ++i)
        if (params[MLP_OFF_W3 + i] != 0.0f) return fail(ctx, BINDER_ERR_ARG, "W3 padding not zero");
    for (int i = MLP_OUT; i < MLP_OUT_PAD; ++i)
        if (params[MLP_OFF_B3 + i] != 0.0f) return fail(ctx, BINDER_ERR_ARG, "b3 padding not zero");
    CK(M.w.ensure(MLP_N_PARAMS), "mlp alloc");
    CK(M.g.ensure(MLP_N_PARAMS), "mlp alloc");
    CK(M.m1.ensure(MLP_N_PARAMS), "mlp alloc");
    CK(M.m2.ensure(MLP_N_PARAMS), "mlp alloc");
    CK(M.w1.ensure(MLP_H * MLP_K1), "mlp alloc");
    CK(M.w2.ensure(MLP_H * MLP_H), "mlp alloc");
    CK(M.w2t.ensure(MLP_H * MLP_H), "mlp alloc");
    CK(M.w3.ensure(MLP_OUT_PAD * MLP_H), "mlp alloc");
    CK(M.w3t.ensure(MLP_OUT_PAD * MLP_H), "mlp alloc");
    CK(M.f1.ensure((MLP_H / 16) * (MLP_K1 / 16) * 32), "mlp alloc");
    CK(M.f2.ensure((MLP_H / 16) * (MLP_H / 16) * 32), "mlp alloc");
    CK(M.f3.ensure((MLP_OUT_PAD / 16) * (MLP_H / 16) * 32), "mlp alloc");
    CK(M.loss.ensure(1), "mlp alloc");
    CK(cudaMemcpyAsync(M.w.p, params, MLP_N_PARAMS * sizeof(float), cudaMemcpyHostToDevice, ctx->stream), "mlp H2D");
    CK(cudaMemsetAsync(M.g.p, 0, MLP_N_PARAMS * sizeof(float), ctx->stream), "mlp memset");
    CK(cudaMemsetAsync(M.m1.p, 0, MLP_N_PARAMS * sizeof(float), ctx->stream), "mlp memset");
    CK(cudaMemsetAsync(M.m2.p, 0, MLP_N_PARAMS * sizeof(float), ctx->stream), "mlp memset");
    M.adam_t = 0;
    if ((s = mlp_pack(ctx))) return s;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    M.ready = true;
    return BINDER_OK;
}

int binder_mlp_get_params(binder_ctx* ctx, float* params) {
    int s = enter(ctx);
    if (s) return s;
    if (!params) return fail(ctx, BINDER_ERR_ARG, "NULL output");
    if ((s = mlp_check_ready(ctx))) return s;
    CK(cudaMemcpyAsync(params, ctx->mlp.w.p, MLP_N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
       "mlp D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_mlp_features(binder_ctx* ctx, int32_t antigen_id, size_t n, const float* ca_xyz, const uint8_t* aa,
                        float* out) {
    int s = enter(ctx);
    if (s) return s;
    if (n && (!ca_xyz || !aa || !out)) return fail(ctx, BINDER_ERR_ARG, "NULL array");
    if (antigen_id < 0 || antigen_id >= (int)ctx->ags.size()) return fail(ctx, BINDER_ERR_ARG, "no antigen %d", antigen_id);
    if (n > (1u << 24)) return fail(ctx, BINDER_ERR_ARG, "too many rows");
    for (size_t i = 0; i < n; ++i)
        if (aa[i] >= N_AA && aa[i] != MLP_NO_AA)
            return fail(ctx, BINDER_ERR_ARG, "amino acid %d out of range", (int)aa[i]);
    if (n == 0) return BINDER_OK;
    MlpState& M = ctx->mlp;
    if ((s = mlp_reserve(ctx, (int)n))) return s;
    std::vector<int> agv(n, antigen_id);
    if ((s = upload(ctx, M.ca, ca_xyz, 3 * n, "features H2D")) || (s = upload(ctx, M.aa, aa, n, "features H2D")) ||
        (s = upload(ctx, M.ag, agv.data(), n, "features H2D")))
        return s;
    launch_features(ctx->stream, (int)n, (int)n, M.ca.p, M.aa.p, M.ag.p, ctx->d_views.p, M.X.p);
    LAUNCHED("features");
    std::vector<__nv_bfloat16> h(n * MLP_K1);
    CK(cudaMemcpyAsync(h.data(), M.X.p, h.size() * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost, ctx->stream),
       "features D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    for (size_t r = 0; r < n; ++r)
        for (int j = 0; j < MLP_IN; ++j) out[r * MLP_IN + j] = __bfloat162float(h[r * MLP_K1 + j]);
    return BINDER_OK;
}

int binder_mlp_forward(binder_ctx* ctx, size_t n, const float* features, float* out) {
    int s = enter(ctx);
    if (s) return s;
    if (n && (!features || !out)) return fail(ctx, BINDER_ERR_ARG, "NULL array");
    if (n > (1u << 24)) return fail(ctx, BINDER_ERR_ARG, "too many rows");
    if ((s = mlp_check_ready(ctx))) return s;
    if (n == 0) return BINDER_OK;
    MlpState& M = ctx->mlp;
    if ((s = mlp_reserve(ctx, (int)n)) || (s = clear_err(ctx))) return s;
    if ((s = upload(ctx, M.feat, features, n * MLP_IN, "mlp H2D"))) return s;
    const int mp = round_up((int)n, 128);
    launch_pack_features(ctx->stream, (int)n, mp, M.feat.p, M.X.p);
    LAUNCHED("mlp pack features");
    if ((s = mlp_forward_dev(ctx, (int)n, false))) return s;
    CK(cudaMemcpy2DAsync(out, MLP_OUT * sizeof(float), M.Y.p, MLP_OUT_PAD * sizeof(float), MLP_OUT * sizeof(float), n,
                         cudaMemcpyDeviceToHost, ctx->stream),
       "mlp D2H");
    return check_err(ctx);
}

int binder_mlp_loss_grad(binder_ctx* ctx, size_t n, const float* features, const int32_t* action,
                         const int32_t* ref, const float* target, float huber_delta, double* out_loss,
                         float* out_grad) {
    int s = enter(ctx);
    if (s) return s;
    if (!n || !features || !action || !target) return fail(ctx, BINDER_ERR_ARG, "empty or NULL batch");
    if (n > (1u << 24)) return fail(ctx, BINDER_ERR_ARG, "too many rows");
    if (!(huber_delta > 0.0f)) return fail(ctx, BINDER_ERR_ARG, "huber_delta must be positive");
    for (size_t i = 0; i < n; ++i) {
        if (action[i] < 0 || action[i] >= MLP_OUT) return fail(ctx, BINDER_ERR_ARG, "action %d out of range", action[i]);
        if (ref && (ref[i] < -1 || ref[i] >= MLP_OUT))
            return fail(ctx, BINDER_ERR_ARG, "reference output %d out of range", ref[i]);
    }
    if ((s = mlp_check_ready(ctx))) return s;
    MlpState& M = ctx->mlp;
    if ((s = mlp_reserve(ctx, (int)n)) || (s = clear_err(ctx))) return s;
    if ((s = upload(ctx, M.feat, features, n * MLP_IN, "mlp H2D")) ||
        (s = upload(ctx, M.action, (const int*)action, n, "mlp H2D")) ||
        (s = upload(ctx, M.target, target, n, "mlp H2D")) ||
        (ref && (s = upload(ctx, M.ref, (const int*)ref, n, "mlp H2D"))))
        return s;
    const int mp = round_up((int)n, 128);
    launch_pack_features(ctx->stream, (int)n, mp, M.feat.p, M.X.p);
    LAUNCHED("mlp pack features");
    launch_transpose_bf16(ctx->stream, mp, MLP_K1, M.X.p, M.Xt.p);
    LAUNCHED("mlp transpose");
    CK(cudaMemsetAsync(M.loss.p, 0, sizeof(double), ctx->stream), "mlp memset");
    if ((s = mlp_forward_dev(ctx, (int)n, true)) || (s = mlp_backward_dev(ctx, (int)n, huber_delta, ref != nullptr)))
        return s;
    double loss = 0.0;
    CK(cudaMemcpyAsync(&loss, M.loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream), "mlp D2H");
    if (out_grad)
        CK(cudaMemcpyAsync(out_grad, M.g.p, MLP_N_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream),
           "mlp D2H");
    if ((s = check_err(ctx))) return s;
    if (out_loss) *out_loss = loss;
    return BINDER_OK;
}

int binder_mlp_set_tuples(binder_ctx* ctx, const binder_mc_tuple* t, size_t n) {
    int s = enter(ctx);
    if (s) return s;
    if (n && !t) return fail(ctx, BINDER_ERR_ARG, "NULL tuples");
    for (size_t i = 0; i < n; ++i)
        if (t[i].action >= MLP_OUT || t[i].aa >= N_AA || t[i].antigen >= ctx->ags.size() || !std::isfinite(t[i].x) ||
            !std::isfinite(t[i].y) || !std::isfinite(t[i].z) || !std::isfinite(t[i].delta_e))
            return fail(ctx, BINDER_ERR_ARG, "invalid tuple %zu", i);
    if ((s = upload(ctx, ctx->mlp.tuples, (const MlpTuple*)t, n, "tuples H2D"))) return s;
    ctx->mlp.n_tuples = n;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_mlp_tuple_count(binder_ctx* ctx, size_t* out_n) {
    if (!ctx || !out_n) return BINDER_ERR_ARG;
    *out_n = ctx->mlp.n_tuples;
    return BINDER_OK;
}

int binder_mlp_get_tuples(binder_ctx* ctx, binder_mc_tuple* out, size_t cap, size_t* out_n) {
    int s = enter(ctx);
    if (s) return s;
    if (!out_n) return fail(ctx, BINDER_ERR_ARG, "NULL count");
    *out_n = ctx->mlp.n_tuples;
    if (cap < ctx->mlp.n_tuples) return fail(ctx, BINDER_ERR_CAPACITY, "need %zu tuples", ctx->mlp.n_tuples);
    if (ctx->mlp.n_tuples)
        CK(cudaMemcpyAsync(out, ctx->mlp.tuples.p, ctx->mlp.n_tuples * sizeof(MlpTuple), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "tuples D2H");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_mlp_train(binder_ctx* ctx, int n_steps, int batch, float lr, float huber_delta, uint64_t seed,
                     double* out_losses) {
    int s = enter(ctx);
    if (s) return s;
    if (n_steps < 0 || batch <= 0 || batch > (1 << 20) || !(lr > 0.0f) || !(huber_delta > 0.0f))
        return fail(ctx, BINDER_ERR_ARG, "invalid training arguments");
    if ((s = mlp_check_ready(ctx))) return s;
    MlpState& M = ctx->mlp;
    if (M.n_tuples == 0) return fail(ctx, BINDER_ERR_STATE, "no tuples to train on");
    if ((s = mlp_reserve(ctx, batch)) || (s = clear_err(ctx))) return s;
    CK(M.loss.ensure((size_t)std::max(1, n_steps)), "mlp alloc");
    CK(cudaMemsetAsync(M.loss.p, 0, (size_t)std::max(1, n_steps) * sizeof(double), ctx->stream), "mlp memset");
    const int mp = round_up(batch, 128);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    double* loss_base = M.loss.p;
    for (int step = 0; step < n_steps; ++step) {
        launch_draw_batch(ctx->stream, batch, (int)std::min<size_t>(M.n_tuples, INT32_MAX), seed, (uint32_t)M.adam_t,
                          M.idx.p);
        LAUNCHED("mlp draw batch");
        launch_gather_tuples(ctx->stream, batch, M.idx.p, M.tuples.p, M.ca.p, M.aa.p, M.ag.p, M.action.p, M.ref.p,
                             M.target.p);
        LAUNCHED("mlp gather");
        launch_features(ctx->stream, batch, mp, M.ca.p, M.aa.p, M.ag.p, ctx->d_views.p, M.X.p);
        LAUNCHED("features");
        launch_transpose_bf16(ctx->stream, mp, MLP_K1, M.X.p, M.Xt.p);
        LAUNCHED("mlp transpose");
        M.loss.p = loss_base + step;  // per-step loss slot
        s = mlp_forward_dev(ctx, batch, true);
        if (!s) s = mlp_backward_dev(ctx, batch, huber_delta, true);
        M.loss.p = loss_base;
        if (s) return s;
        M.adam_t += 1;
        const float bc1 = 1.0f - std::pow(b1, (float)M.adam_t), bc2 = 1.0f - std::pow(b2, (float)M.adam_t);
        launch_adam(ctx->stream, MLP_N_PARAMS, M.w.p, M.g.p, M.m1.p, M.m2.p, lr, b1, b2, eps, bc1, bc2);
        LAUNCHED("mlp adam");
        if ((s = mlp_pack(ctx))) return s;
    }
    if (out_losses && n_steps > 0)
        CK(cudaMemcpyAsync(out_losses, loss_base, (size_t)n_steps * sizeof(double), cudaMemcpyDeviceToHost,
                           ctx->stream),
           "mlp D2H");
    return check_err(ctx);
}

}  // extern "C"

extern "C" {

int binder_set_proposal(binder_ctx* ctx, int mode, float t_prop_min, float t_max) {
    int s = enter(ctx);
    if (s) return s;
    if (mode != BINDER_PROPOSAL_UNIFORM && mode != BINDER_PROPOSAL_LEARNED)
        return fail(ctx, BINDER_ERR_ARG, "unknown proposal mode %d", mode);
    if (!(t_prop_min > 0.0f) || !std::isfinite(t_prop_min)) return fail(ctx, BINDER_ERR_ARG, "t_prop_min must be > 0");
    if (!(t_max > 0.0f)) return fail(ctx, BINDER_ERR_ARG, "t_max must be > 0");
    if (mode == BINDER_PROPOSAL_LEARNED && (s = mlp_check_ready(ctx))) return s;
    ctx->mlp.learned = mode == BINDER_PROPOSAL_LEARNED;
    ctx->mlp.t_prop_min = t_prop_min;
    ctx->mlp.t_max = t_max;
    return BINDER_OK;
}

int binder_mc_log(binder_ctx* ctx, size_t capacity) {
    int s = enter(ctx);
    if (s) return s;
    MlpState& M = ctx->mlp;
    if (capacity == 0) {
        M.log.release();
        M.log_n.release();
        M.log_cap = 0;
        return BINDER_OK;
    }
    CK(M.log.ensure(capacity), "log alloc");
    CK(M.log_n.ensure(1), "log alloc");
    CK(cudaMemsetAsync(M.log_n.p, 0, sizeof(unsigned long long), ctx->stream), "log memset");
    M.log_cap = capacity;
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    return BINDER_OK;
}

int binder_mc_log_count(binder_ctx* ctx, size_t* out_logged, size_t* out_proposed) {
    int s = enter(ctx);
    if (s) return s;
    unsigned long long n = 0;
    if (ctx->mlp.log_cap) {
        CK(cudaMemcpyAsync(&n, ctx->mlp.log_n.p, sizeof(n), cudaMemcpyDeviceToHost, ctx->stream), "log D2H");
        CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    }
    if (out_proposed) *out_proposed = (size_t)n;
    if (out_logged) *out_logged = std::min<size_t>((size_t)n, ctx->mlp.log_cap);
    return BINDER_OK;
}

int binder_mc_log_fetch(binder_ctx* ctx, binder_mc_tuple* out, size_t cap, size_t* out_n) {
    size_t n = 0;
    int s = binder_mc_log_count(ctx, &n, nullptr);
    if (s) return s;
    if (!out_n) return fail(ctx, BINDER_ERR_ARG, "NULL count");
    *out_n = n;
    if (cap < n) return fail(ctx, BINDER_ERR_CAPACITY, "need %zu tuples", n);
    if (n) {
        if (!out) return fail(ctx, BINDER_ERR_ARG, "NULL output");
        CK(cudaMemcpyAsync(out, ctx->mlp.log.p, n * sizeof(MlpTuple), cudaMemcpyDeviceToHost, ctx->stream), "log D2H");
        CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    }
    return BINDER_OK;
}

int binder_mlp_take_log(binder_ctx* ctx, size_t* out_n) {
    size_t n = 0;
    int s = binder_mc_log_count(ctx, &n, nullptr);
    if (s) return s;
    MlpState& M = ctx->mlp;
    CK(M.tuples.ensure(std::max<size_t>(n, 1)), "tuples alloc");
    if (n)
        CK(cudaMemcpyAsync(M.tuples.p, M.log.p, n * sizeof(MlpTuple), cudaMemcpyDeviceToDevice, ctx->stream),
           "tuples copy");
    CK(cudaStreamSynchronize(ctx->stream), "synchronize");
    M.n_tuples = n;
    if (out_n) *out_n = n;
    return BINDER_OK;
}

}  // extern "C"

extern "C" {

int binder_debug_fail_alloc(int64_t n) {
    g_alloc_countdown = n < 0 ? -1 : n;
    return BINDER_OK;
}

int binder_selftest_wait(binder_ctx* ctx, uint32_t max_polls) {
    int s = enter(ctx);
    if (s) return s;
    if ((s = clear_err(ctx))) return s;
    CK(launch_wait_selftest(ctx->stream, max_polls, ctx->errf.p), "wait self-test");
    ctx->launches++;
    return check_err(ctx);
}

}  // extern "C"
