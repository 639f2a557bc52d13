// noalloc.cu — binder_grid_neighbors_noalloc: the spatial-grid build and 27-cell
// probe of binder_grid_neighbors for callers that cannot allocate device memory.
//
// Some hosts own every byte of device memory themselves — an arena or pool that
// the host program (or another framework sharing the GPU) carves up ahead of time —
// and cannot let a library call cudaMalloc/cudaFree behind their back; others run
// latency-critical loops where an allocation or free would stall the device.  This
// entry point takes only caller-owned device buffers for its inputs and outputs and
// keeps the kernels' scratch (cell keys, histogram, cell offsets, sorted indices)
// in one fixed-size file-scope device array instead of allocating it.
//
// The array is part of the loaded library: every GPU that loads it holds its
// NOALLOC_SCRATCH_BYTES until the process exits.  All calls share it and it keeps
// the previous call's contents, so every call clears what must start at zero, and
// two calls whose work overlaps on the GPU (different streams, or different host
// threads) race on it.  The device address of the array is looked up once per
// device, on that device's first call (cudaGetSymbolAddress with the device
// current); make that first call before any stream capture.  The work goes to the
// current device: the caller's stream must belong to it.  The looked-up address
// is kept for the life of the process, so after cudaDeviceReset on a device (which
// unloads the library's module there) this entry point must not be called on that
// device again.  Each call waits on the caller's stream twice (to read the
// occupied cell box and the neighbour count back to the host).
#include <cstring>
#include <mutex>

#include "binder_gpu.h"
#include "kernels.h"

namespace binder {

namespace {
constexpr size_t NA_MAX_ATOMS = BINDER_NOALLOC_MAX_ATOMS;
constexpr size_t NA_MAX_CELLS = BINDER_NOALLOC_MAX_CELLS;
constexpr size_t NA_ALIGN = 256;
constexpr size_t na_round(size_t b) { return (b + NA_ALIGN - 1) / NA_ALIGN * NA_ALIGN; }
// sub-buffers of the scratch array, in order
constexpr size_t NA_CELLS_OFF = 0;                                                  // int4[NA_MAX_ATOMS]
constexpr size_t NA_COUNTS_OFF = NA_CELLS_OFF + na_round(NA_MAX_ATOMS * 16);        // int[NA_MAX_CELLS]
constexpr size_t NA_START_OFF = NA_COUNTS_OFF + na_round(NA_MAX_CELLS * 4);         // int[NA_MAX_CELLS + 1]
constexpr size_t NA_CURSOR_OFF = NA_START_OFF + na_round((NA_MAX_CELLS + 1) * 4);   // int[NA_MAX_CELLS + 1]
constexpr size_t NA_SORTED_OFF = NA_CURSOR_OFF + na_round((NA_MAX_CELLS + 1) * 4);  // int[NA_MAX_ATOMS]
constexpr size_t NA_MINMAX_OFF = NA_SORTED_OFF + na_round(NA_MAX_ATOMS * 4);        // int[6]
constexpr size_t NA_ERR_OFF = NA_MINMAX_OFF + NA_ALIGN;                             // uint32
constexpr size_t NOALLOC_SCRATCH_BYTES = NA_ERR_OFF + NA_ALIGN;
constexpr int NA_MAX_DEVICES = 64;
}  // namespace

// The scratch of binder_grid_neighbors_noalloc (about 4.3 MB per device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {
std::mutex g_na_mutex;
unsigned char* g_na_base[NA_MAX_DEVICES] = {};

// In-place inclusive scan of v[0..n) (64-bit), one CTA.
__global__ void k_inclusive_scan_ll(long long* __restrict__ v, int n) {
    __shared__ long long warp_sums[32];
    __shared__ long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        long long x = i < n ? v[i] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            long long w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const long long t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            warp_sums[lane] = w;
        }
        __syncthreads();
        const long long incl = carry + (warp > 0 ? warp_sums[warp - 1] : 0) + x;
        if (i < n) v[i] = incl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
}

// Device address of the scratch array on the current device (looked up once).
int scratch_base(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return BINDER_ERR_NODEVICE;
    }
    if (dev < 0 || dev >= NA_MAX_DEVICES) return BINDER_ERR_NODEVICE;
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_base[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return BINDER_ERR_CUDA;
        }
        g_na_base[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_na_base[dev];
    return BINDER_OK;
}
}  // namespace

}  // namespace binder

using namespace binder;

#define NA_CK(call)                          \
    do {                                     \
        if ((call) != cudaSuccess) {         \
            cudaGetLastError();              \
            return BINDER_ERR_CUDA;          \
        }                                    \
    } while (0)

extern "C" int binder_grid_neighbors_noalloc(float cell, const float* ax, const float* ay, const float* az,
                                             size_t n_ag, const float* px, const float* py, const float* pz,
                                             size_t n_q, int64_t* d_offsets, uint32_t* d_idx, size_t cap,
                                             size_t* out_total, void* stream_handle) {
    if (!(cell > 0.0f) || !(cell < 3.0e38f)) return BINDER_ERR_ARG;
    if (n_ag > NA_MAX_ATOMS) return BINDER_ERR_ARG;  // beyond the scratch array
    if (n_q > (size_t)INT32_MAX / 2) return BINDER_ERR_ARG;
    if (!d_offsets || !out_total || (n_ag && (!ax || !ay || !az)) || (n_q && (!px || !py || !pz)))
        return BINDER_ERR_ARG;
    // an error left pending by earlier work of the process is not this call's: report
    // it without consuming it, so that the launch checks below see only this call's
    if (cudaPeekAtLastError() != cudaSuccess) return BINDER_ERR_CUDA;
    unsigned char* base = nullptr;
    int s = scratch_base(&base);
    if (s) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream_handle);
    int4* cells = reinterpret_cast<int4*>(base + NA_CELLS_OFF);
    int* counts = reinterpret_cast<int*>(base + NA_COUNTS_OFF);
    int* cell_start = reinterpret_cast<int*>(base + NA_START_OFF);
    int* cursor = reinterpret_cast<int*>(base + NA_CURSOR_OFF);
    int* sorted = reinterpret_cast<int*>(base + NA_SORTED_OFF);
    int* minmax = reinterpret_cast<int*>(base + NA_MINMAX_OFF);
    uint32_t* err = reinterpret_cast<uint32_t*>(base + NA_ERR_OFF);

    // cell of every antigen point + occupied box (the scratch keeps the previous
    // call's values: min/max and the error word are re-initialised here)
    const float inv = 1.0f / cell;
    int h_mm[6] = {INT32_MAX, INT32_MAX, INT32_MAX, INT32_MIN, INT32_MIN, INT32_MIN};
    NA_CK(cudaMemcpyAsync(minmax, h_mm, sizeof(h_mm), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
    launch_cell_coords(st, ax, ay, az, (int)n_ag, inv, cells, minmax, err);
    NA_CK(cudaGetLastError());
    uint32_t h_err = 0;
    NA_CK(cudaMemcpyAsync(h_mm, minmax, sizeof(h_mm), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    if (h_err & ERRF_NAN) return BINDER_ERR_NAN;
    if (n_ag == 0)
        for (int k = 0; k < 3; ++k) h_mm[k] = 0, h_mm[k + 3] = 0;
    const long long nx = (long long)h_mm[3] - h_mm[0] + 1, ny = (long long)h_mm[4] - h_mm[1] + 1,
                    nz = (long long)h_mm[5] - h_mm[2] + 1;
    if ((double)nx * (double)ny * (double)nz > (double)NA_MAX_CELLS) return BINDER_ERR_GRID;
    const int ncell = (int)(nx * ny * nz);

    // counting sort into the scratch (histogram cleared first)
    NA_CK(cudaMemsetAsync(counts, 0, (size_t)ncell * sizeof(int), st));
    launch_cell_hist(st, cells, (int)n_ag, h_mm[0], h_mm[1], h_mm[2], (int)ny, (int)nz, counts);
    launch_exclusive_scan(st, counts, ncell, cell_start);
    NA_CK(cudaMemcpyAsync(cursor, cell_start, (size_t)(ncell + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st));
    launch_stable_scatter(st, cells, (int)n_ag, cursor, sorted);
    NA_CK(cudaGetLastError());

    GridView g;
    g.cell_start = cell_start;
    g.ox = h_mm[0]; g.oy = h_mm[1]; g.oz = h_mm[2];
    g.nx = (int)nx; g.ny = (int)ny; g.nz = (int)nz;
    g.inv = inv;
    g.cell = cell;

    // per-probe counts into the caller's offsets[1..n_q], then an in-place scan
    NA_CK(cudaMemsetAsync(d_offsets, 0, sizeof(int64_t), st));
    launch_nb_count(st, g, px, py, pz, (int)n_q, reinterpret_cast<long long*>(d_offsets) + 1);
    if (n_q > 0) k_inclusive_scan_ll<<<1, 1024, 0, st>>>(reinterpret_cast<long long*>(d_offsets) + 1, (int)n_q);
    NA_CK(cudaGetLastError());
    long long total = 0;
    NA_CK(cudaMemcpyAsync(&total, d_offsets + n_q, sizeof(long long), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaStreamSynchronize(st));
    *out_total = (size_t)total;
    if ((size_t)total > cap) return BINDER_ERR_CAPACITY;
    if (total == 0) return BINDER_OK;
    if (!d_idx) return BINDER_ERR_ARG;
    launch_nb_fill(st, g, sorted, px, py, pz, (int)n_q, reinterpret_cast<const long long*>(d_offsets), d_idx);
    NA_CK(cudaGetLastError());
    return BINDER_OK;
}
