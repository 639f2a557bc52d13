// common.cuh — shared definitions of the sm_100a kernels: constants, packed
// force-field tables, exact-rounding helpers, the Philox generator, the device
// views of antigens and of the resident candidate state.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace binder {

#include "binder_tables.inc"  // host copies of the reference tables (BT_*)

constexpr int SLOTS = 14;        // max heavy atoms per residue (TRP, amber.rs:311-326)
constexpr int SLOT_STRIDE = 16;  // float4 slots per residue in device state (256 B, two 128 B lines)
constexpr int N_AA = 20;
constexpr int GLY = 7;
constexpr int CYS = 4;

// energy.rs:13-27
constexpr float COULOMB_K = 332.0f;
constexpr float CUTOFF_SQ = 100.0f;
constexpr float MIN_R_SQ = 0.25f;
constexpr float HYDRO_CUTOFF_SQ = 36.0f;
constexpr float HYDRO_BONUS = -0.5f;
constexpr float HB_R0 = 2.9f;
constexpr float HB_SIGMA = 0.35f;
constexpr float HB_DEPTH = 1.5f;
constexpr float HB_CUTOFF_SQ = 25.0f;
// solvation.rs:23-27
constexpr float PI32 = 5.568328f;
constexpr float SOLV_CUTOFF_SQ = 81.0f;
// allatom.rs:494-497
constexpr float N_CA_BOND = 1.46f;
constexpr float CA_C_BOND = 1.52f;
constexpr float C_O_BOND = 1.23f;
constexpr float CA_CB_BOND = 1.52f;

// entries of a residue's Verlet list in the gradient-step kernel (k_search.cu)
constexpr int CG_LIST_CAP = 128;

// residue sort keys cover the antigen's Calpha-grid box widened by this many cells
constexpr int RES_KEY_MARGIN = 3;

// error flags a kernel may raise (read back by the host after the launch)
enum : uint32_t { ERRF_NAN = 1u, ERRF_TIMEOUT = 2u, ERRF_RANGE = 4u };

// ---- exact-rounding helpers: one IEEE rounding per operation, never fused --------
// The reference is Rust, which never contracts a*b+c; where bit-exact parity with
// its f32 results is required these helpers stop nvcc from forming FMAs.
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float xsqrt(float a) { return __fsqrt_rn(a); }
// squared distance with the reference's rounding: (dx*dx + dy*dy) + dz*dz
__device__ __forceinline__ float xdist2(float dx, float dy, float dz) {
    return xadd(xadd(xmul(dx, dx), xmul(dy, dy)), xmul(dz, dz));
}

// Packed pairs of f32 (element 0 in the low word) and the sm_100 two-wide FP32
// instructions; each element is rounded exactly as the scalar instruction rounds it.
// A packed multiply feeding a packed add may still be fused by the code generator
// (measured on sm_100a: a pair at r^2 = 100.000008 in the reference's rounding came
// out as 100.0), so wherever a result must keep the reference's two roundings the
// products and sums go through the scalar x* helpers above (f2_dist2 below).
__device__ __forceinline__ uint64_t f2_pack(float lo, float hi) {
    return (uint64_t)__float_as_uint(lo) | ((uint64_t)__float_as_uint(hi) << 32);
}
__device__ __forceinline__ uint64_t f2_sub(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_mul(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ uint64_t f2_add(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ float f2_lo(uint64_t v) { return __uint_as_float((uint32_t)v); }
__device__ __forceinline__ float f2_hi(uint64_t v) { return __uint_as_float((uint32_t)(v >> 32)); }
// the reference's r^2 of both elements of packed differences (scalar, never fused)
__device__ __forceinline__ void f2_dist2(uint64_t dx, uint64_t dy, uint64_t dz, float& lo, float& hi) {
    lo = xdist2(f2_lo(dx), f2_lo(dy), f2_lo(dz));
    hi = xdist2(f2_hi(dx), f2_hi(dy), f2_hi(dz));
}

// Transcendentals of the Metropolis path (acceptance exp, H-bond and disulfide
// Gaussians, rotation by a random torsion): evaluated in double and rounded once
// to f32, on the device and in the CPU restatement alike.  Both double functions
// are within 1 ulp of the exact value, so the two f32 results agree unless the
// exact value lies within about 2^-29 (relative) of an f32 rounding boundary.
__host__ __device__ __forceinline__ float mc_exp(float x) { return (float)exp((double)x); }
__host__ __device__ __forceinline__ float mc_sin(float x) { return (float)sin((double)x); }
__host__ __device__ __forceinline__ float mc_cos(float x) { return (float)cos((double)x); }

// Rust `f32 as i32`: saturating, NaN -> 0
__host__ __device__ __forceinline__ int32_t sat_i32(float v) {
    if (v != v) return 0;
    if (v >= 2147483648.0f) return INT32_MAX;
    if (v < -2147483648.0f) return INT32_MIN;
    return (int32_t)v;
}

// ---- Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) --------------------------
struct U4 { uint32_t x, y, z, w; };
__host__ __device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                               uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return U4{c0, c1, c2, c3};
}
// Draw conventions (identical in the oracle): counter = (candidate, step,
// stream << 16 | residue, 0), key = seed.  Uniform float from the top 24 bits,
// integer range by multiply-shift, float range lo + u*(hi-lo) rounded per op.
enum : uint32_t { STREAM_NOISE = 0, STREAM_MC = 1, STREAM_BACKBONE = 2 };
__host__ __device__ __forceinline__ U4 rng_draw(uint64_t seed, uint32_t cand, uint32_t step, uint32_t stream,
                                                 uint32_t r) {
    return philox(cand, step, (stream << 16) | (r & 0xFFFFu), 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
}
__device__ __forceinline__ float u01(uint32_t x) { return xmul((float)(x >> 8), 1.0f / 16777216.0f); }
__device__ __forceinline__ uint32_t urange(uint32_t x, uint32_t n) { return (uint32_t)(((uint64_t)x * n) >> 32); }
__device__ __forceinline__ float frange(uint32_t x, float lo, float hi) { return xadd(lo, xmul(u01(x), xsub(hi, lo))); }

// ---- device views ----------------------------------------------------------------
// A uniform cell box over the cells that contain atoms (the reference's HashMap
// holds exactly those cells; a probe outside the box finds nothing, as a missing
// HashMap key does).
struct GridView {
    const int* cell_start;  // ncell + 1
    int ox, oy, oz;         // cell index of box corner
    int nx, ny, nz;
    float inv;              // f32 reciprocal of the cell edge (spatial.rs:26)
    float cell;
};

// One resident antigen.
struct AgView {
    // all atoms, sorted by score-grid cell (ascending original index within a cell)
    const float4* pq;   // x, y, z, q*sqrt(332)
    const float4* prm;  // r_min_half, sqrt(epsilon), hydrophobic (0/1), atom type
    GridView grid;
    int n_atoms;
    // Calpha cloud (run_allatom ag_ca, diffusion.rs:994-1002) sorted by CA-grid cell
    const float4* ca_pq;   // x, y, z, residue-level charge (atom.rs:55-63)
    const float4* ca_prm;  // residue-level epsilon, sigma, hydrophobic, 0
    const int4* ca_cell;   // CA-grid cell of each sorted Calpha
    GridView ca_grid;
    // Calpha atoms in residue order with their AMBER parameters (diffusion.rs:440-446)
    const float4* ca_atom;      // x, y, z, partial charge
    const float4* ca_atom_prm;  // r_min_half, epsilon, hydrophobic, atom type
    const uint8_t* res_aa;      // amino acid of each antigen residue (residue order)
    int n_res;
    float cx, cy, cz;  // ca_center_of_mass (allatom.rs:183-195)
};

// Resident candidate state (slot layout).
struct StateView {
    int n_cand;
    int total_res;
    const int* cand_res_off;  // n_cand + 1
    const int* cand_ag;       // n_cand
    const uint32_t* cand_id;  // n_cand
    uint8_t* res_aa;          // total_res
    float4* res_chi;          // total_res (degrees)
    float4* res_trig;         // 2 * total_res: sin/cos of chi1, chi2 | chi3, chi4
    float4* res_pos;          // total_res * SLOT_STRIDE
    const int* res_cand;      // total_res
    // Verlet lists of the gradient-step kernel kept between launches
    int* cg_list;             // total_res * CG list capacity: sorted antigen Calpha positions
    float4* cg_centre;        // total_res: list centre
    int4* cg_meta;            // total_res: {length, antigen, antigen-set epoch, 0}
    int* cg_bal;              // work-balanced residue order of the flat gradient-step kernel (cg_bal_*)
    const int* ag_epoch;      // device word: the antigen-set epoch (bumped when antigens change)
};

// Work-balanced residue order of the flat gradient-step kernel, built by the kernel
// itself for its next launch: every residue, at the end of its task, appends its
// index to the bucket of its work band (Verlet-list length plus a charge per rebuild,
// CG_BAL_BINS bands, heaviest first) of the buffer of parity epoch ^ 1; the next
// launch reads the buckets of its own parity as the ranks 0..n-1 (band by band) and
// deals them to its tasks in snake order.  Layout of cg_bal: [0] epoch, [1] CTAs
// done, [2 + 16 * parity + band] bucket counts, then the buckets, total_res entries
// each.  The last CTA of a launch zeroes the counts it read and advances the epoch.
constexpr int CG_BAL_BINS = 16;
constexpr int CG_BAL_HEADER = 2 + 2 * CG_BAL_BINS;
__host__ __device__ inline size_t cg_bal_ints(int total_res) {
    return (size_t)CG_BAL_HEADER + (size_t)2 * CG_BAL_BINS * (size_t)total_res;
}
__device__ __forceinline__ int* cg_bal_count(int* bal, int parity) { return bal + 2 + CG_BAL_BINS * parity; }
__device__ __forceinline__ int* cg_bal_bucket(int* bal, int total_res, int parity, int band) {
    return bal + CG_BAL_HEADER + ((size_t)(parity * CG_BAL_BINS + band)) * (size_t)total_res;
}

// Work queues of persistent kernels: queue[0] hands out tasks, queue[2] counts the
// CTAs that are done.  Every CTA calls queue_retire once at its end; the last one
// leaves both counters zero for the next launch, so that no reset is launched
// between kernels.  (The host zeroes them when it allocates them and before each
// call's first launch.)
__device__ __forceinline__ void queue_retire(int* queue) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 2, 1) == (int)gridDim.x - 1) {
            atomicExch(queue, 0);
            atomicExch(queue + 2, 0);
        }
    }
}

// spatial.rs:61-67: (x * inv).floor() as i32 — one f32 multiply, floor, saturating cast
__device__ __forceinline__ int cell_coord(float v, float inv) { return sat_i32(floorf(xmul(v, inv))); }

// Range of atoms of cell (cx+dx, cy+dy, cz+dz); false when the cell holds none.
// i32 addition wraps, as in the reference's release build (spatial.rs:52).
__device__ __forceinline__ bool probe_cell(const GridView& g, int cx, int cy, int cz, int dx, int dy, int dz, int& a0,
                                           int& a1) {
    int nx_ = (int)((unsigned)cx + (unsigned)dx), ny_ = (int)((unsigned)cy + (unsigned)dy),
        nz_ = (int)((unsigned)cz + (unsigned)dz);
    long long ix = (long long)nx_ - g.ox, iy = (long long)ny_ - g.oy, iz = (long long)nz_ - g.oz;
    if (ix < 0 || iy < 0 || iz < 0 || ix >= g.nx || iy >= g.ny || iz >= g.nz) return false;
    int lin = ((int)ix * g.ny + (int)iy) * g.nz + (int)iz;
    a0 = g.cell_start[lin];
    a1 = g.cell_start[lin + 1];
    return a1 > a0;
}

// Search parameters as the kernels see them.
struct StepParams {
    float step, noise_base, t_hot, t_cold, mutation_p, rotamer_move_p, backbone_move_p, max_torsion_deg,
        iface_cutoff_sq, shell_radius, max_disp, restraint_k;
    uint64_t seed;
};

}  // namespace binder
