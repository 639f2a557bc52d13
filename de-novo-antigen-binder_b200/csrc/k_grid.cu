// k_grid.cu — SpatialHashGrid (spatial.rs:12-67) on the GPU.
//
// The reference hashes cell keys (floor(x*inv) as i32, ...) into a HashMap of
// index vectors built in insertion order.  Here the occupied cells span a dense
// box; the build is a counting sort (histogram, exclusive scan, stable scatter)
// so that every cell holds its atoms in ascending original index, which is the
// reference's insertion order.  A probe walks the 27 cells in the reference's
// (dx, dy, dz) order, giving the same callback sequence bit for bit.
#include "kernels.h"

namespace binder {

__global__ void k_cell_coords(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                              int n, float inv, int4* __restrict__ cells, int* __restrict__ minmax,
                              uint32_t* __restrict__ err) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float px = x[i], py = y[i], pz = z[i];
    if (!isfinite(px) || !isfinite(py) || !isfinite(pz)) atomicOr(err, ERRF_NAN);
    int cx = cell_coord(px, inv), cy = cell_coord(py, inv), cz = cell_coord(pz, inv);
    cells[i] = make_int4(cx, cy, cz, 0);
    atomicMin(&minmax[0], cx); atomicMin(&minmax[1], cy); atomicMin(&minmax[2], cz);
    atomicMax(&minmax[3], cx); atomicMax(&minmax[4], cy); atomicMax(&minmax[5], cz);
}

__global__ void k_cell_hist(int4* __restrict__ cells, int n, int ox, int oy, int oz, int ny, int nz,
                            int* __restrict__ counts) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int4 c = cells[i];
    int lin = ((c.x - ox) * ny + (c.y - oy)) * nz + (c.z - oz);
    cells[i].w = lin;
    atomicAdd(&counts[lin], 1);
}

// Exclusive scan of counts[0..n) into out[0..n], out[n] = total.  One CTA of
// 1024 threads walks the array in chunks; the cell box is small (hundreds to a
// few million cells) and this runs once per antigen.
__global__ void k_exclusive_scan(const int* __restrict__ counts, int n, int* __restrict__ out) {
    __shared__ int warp_sums[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        int i = base + threadIdx.x;
        int v = i < n ? counts[i] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int ws = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int t = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += t;
            }
            warp_sums[lane] = ws;  // inclusive prefix over warps
        }
        __syncthreads();
        int warp_prefix = warp > 0 ? warp_sums[warp - 1] : 0;
        if (i < n) out[i] = carry + warp_prefix + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += warp_prefix + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) out[n] = carry;
}

// Stable scatter: one warp walks the atoms in index order 32 at a time; lanes
// that share a cell take consecutive slots in lane (= index) order.
__global__ void k_stable_scatter(const int4* __restrict__ cells, int n, int* __restrict__ cursor,
                                 int* __restrict__ sorted_idx) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    for (int base = 0; base < n; base += 32) {
        int i = base + lane;
        bool valid = i < n;
        int lin = valid ? cells[i].w : -1 - lane;  // invalid lanes never match a valid cell
        unsigned peers = __match_any_sync(0xffffffffu, lin);
        int start = valid ? cursor[lin] : 0;
        __syncwarp();
        if (valid) {
            sorted_idx[start + __popc(peers & lt)] = i;
            if ((peers & lt) == 0) cursor[lin] = start + __popc(peers);
        }
        __syncwarp();
    }
}

// Atom records of the antigen in grid order.  q' = q*sqrt(332) folds the Coulomb
// constant into the charges; sqrt(epsilon) turns the geometric mix into a product.
__global__ void k_gather_atoms(const int* __restrict__ sorted_idx, int n, const float* __restrict__ x,
                               const float* __restrict__ y, const float* __restrict__ z, const float* __restrict__ q,
                               const float* __restrict__ rmh, const float* __restrict__ eps,
                               const uint8_t* __restrict__ hyd, const uint8_t* __restrict__ type,
                               float4* __restrict__ pq, float4* __restrict__ prm) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int i = sorted_idx[j];
    const float sqrt_k = 18.220867f;  // sqrt(332) rounded to f32
    pq[j] = make_float4(x[i], y[i], z[i], q[i] * sqrt_k);
    prm[j] = make_float4(rmh[i], sqrtf(eps[i]), hyd[i] == 1 ? 1.0f : 0.0f, type ? (float)type[i] : 0.0f);
}

// Residue-level Calpha records (ResidueCloud::push, atom.rs:221-231) in grid order.
__global__ void k_gather_ca(const int* __restrict__ sorted_idx, int n, const float* __restrict__ x,
                            const float* __restrict__ y, const float* __restrict__ z, const uint8_t* __restrict__ aa,
                            const float4* __restrict__ res_tab, float inv, float4* __restrict__ pq,
                            float4* __restrict__ prm, int4* __restrict__ cells) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int i = sorted_idx[j];
    float4 t = res_tab[aa[i]];  // charge, epsilon, sigma, hydrophobic
    pq[j] = make_float4(x[i], y[i], z[i], t.x);
    prm[j] = make_float4(t.y, t.z, t.w, __int_as_float(i));
    cells[j] = make_int4(cell_coord(x[i], inv), cell_coord(y[i], inv), cell_coord(z[i], inv), 0);
}

// ---- 27-cell probe in the reference's callback order (probe_cell, common.cuh) ----
__global__ void k_nb_count(GridView g, const float* __restrict__ px, const float* __restrict__ py,
                           const float* __restrict__ pz, int n_q, long long* __restrict__ counts) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_q) return;
    int cx = cell_coord(px[q], g.inv), cy = cell_coord(py[q], g.inv), cz = cell_coord(pz[q], g.inv);
    long long c = 0;
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                int a0, a1;
                if (probe_cell(g, cx, cy, cz, dx, dy, dz, a0, a1)) c += a1 - a0;
            }
    counts[q] = c;
}

__global__ void k_nb_fill(GridView g, const int* __restrict__ sorted_idx, const float* __restrict__ px,
                          const float* __restrict__ py, const float* __restrict__ pz, int n_q,
                          const long long* __restrict__ offsets, uint32_t* __restrict__ out) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_q) return;
    int cx = cell_coord(px[q], g.inv), cy = cell_coord(py[q], g.inv), cz = cell_coord(pz[q], g.inv);
    long long m = offsets[q];
    for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dz = -1; dz <= 1; ++dz) {
                int a0, a1;
                if (!probe_cell(g, cx, cy, cz, dx, dy, dz, a0, a1)) continue;
                for (int j = a0; j < a1; ++j) out[m++] = (uint32_t)sorted_idx[j];
            }
}

__global__ void k_cells_out(const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
                            int n, float inv, int* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[3 * i] = cell_coord(x[i], inv);
    out[3 * i + 1] = cell_coord(y[i], inv);
    out[3 * i + 2] = cell_coord(z[i], inv);
}

// ---- host launchers ---------------------------------------------------------------
static inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

void launch_cell_coords(cudaStream_t s, const float* x, const float* y, const float* z, int n, float inv, int4* cells,
                        int* minmax, uint32_t* err) {
    if (n > 0) k_cell_coords<<<nblk(n, 256), 256, 0, s>>>(x, y, z, n, inv, cells, minmax, err);
}
void launch_cell_hist(cudaStream_t s, int4* cells, int n, int ox, int oy, int oz, int ny, int nz, int* counts) {
    if (n > 0) k_cell_hist<<<nblk(n, 256), 256, 0, s>>>(cells, n, ox, oy, oz, ny, nz, counts);
}
void launch_exclusive_scan(cudaStream_t s, const int* counts, int n, int* out) {
    k_exclusive_scan<<<1, 1024, 0, s>>>(counts, n, out);
}
void launch_stable_scatter(cudaStream_t s, const int4* cells, int n, int* cursor, int* sorted_idx) {
    k_stable_scatter<<<1, 32, 0, s>>>(cells, n, cursor, sorted_idx);
}
void launch_gather_atoms(cudaStream_t s, const int* sorted_idx, int n, const float* x, const float* y,
                         const float* z, const float* q, const float* rmh, const float* eps, const uint8_t* hyd,
                         const uint8_t* type, float4* pq, float4* prm) {
    if (n > 0) k_gather_atoms<<<nblk(n, 256), 256, 0, s>>>(sorted_idx, n, x, y, z, q, rmh, eps, hyd, type, pq, prm);
}
void launch_gather_ca(cudaStream_t s, const int* sorted_idx, int n, const float* x, const float* y, const float* z,
                      const uint8_t* aa, const float4* res_tab, float inv, float4* pq, float4* prm, int4* cells) {
    if (n > 0) k_gather_ca<<<nblk(n, 256), 256, 0, s>>>(sorted_idx, n, x, y, z, aa, res_tab, inv, pq, prm, cells);
}
void launch_nb_count(cudaStream_t s, const GridView& g, const float* px, const float* py, const float* pz, int n_q,
                     long long* counts) {
    if (n_q > 0) k_nb_count<<<nblk(n_q, 128), 128, 0, s>>>(g, px, py, pz, n_q, counts);
}
void launch_nb_fill(cudaStream_t s, const GridView& g, const int* sorted_idx, const float* px, const float* py,
                    const float* pz, int n_q, const long long* offsets, uint32_t* out) {
    if (n_q > 0) k_nb_fill<<<nblk(n_q, 128), 128, 0, s>>>(g, sorted_idx, px, py, pz, n_q, offsets, out);
}
void launch_cells_out(cudaStream_t s, const float* x, const float* y, const float* z, int n, float inv, int* out) {
    if (n > 0) k_cells_out<<<nblk(n, 256), 256, 0, s>>>(x, y, z, n, inv, out);
}

}  // namespace binder
