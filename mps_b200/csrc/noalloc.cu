// noalloc.cu -- the cell counting sort without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// neighbour structure: code running under an allocator that forbids
// cudaMalloc/cudaFree (a frozen memory pool, a graph-replay harness that
// pins every address, an embedding host that hands out only the buffers it
// owns), or code that must not incur allocation latency inside a time step.
// mps_cell_sort_noalloc serves them: the caller passes its own device
// input and output arrays, and the only scratch the sort needs lives in one
// file-scope static device array, reserved when the library is loaded.
//
// Limits and sharing (also stated in include/mps_b200.h):
//   - at most NOALLOC_MAX_PARTICLES particles and NOALLOC_MAX_CELLS cells per
//     call; larger requests are rejected with MPS_ERR_INVALID;
//   - every GPU that loads the library holds the array (about 4 MB) until the
//     process exits;
//   - all calls on a device share the one array, which keeps the previous
//     call's contents: the counters that must start at zero are cleared at
//     the start of every call, and two calls whose work overlaps on the GPU
//     (different streams, no ordering between them) race on it.
//
// The device address of the array is obtained once per device, with that
// device current, by cudaGetSymbolAddress on the first call made on it (the
// array's name in host code is only a host-side handle, never a device
// address).  That first call therefore should come before any stream
// capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/mps_b200.h"
#include "device.cuh"
#include "scan.cuh"

namespace {

constexpr int NOALLOC_MAX_PARTICLES = MPS_NOALLOC_MAX_PARTICLES;
constexpr int NOALLOC_MAX_CELLS = MPS_NOALLOC_MAX_CELLS;
constexpr int NOALLOC_MAX_DEVICES = 64;

// Partition of the scratch array (ints).
constexpr size_t OFF_COUNT = 0;                                            // histogram, then cursors
constexpr size_t OFF_SLOT = OFF_COUNT + (size_t)NOALLOC_MAX_CELLS + 64;    // unordered cell slots
constexpr size_t OFF_FLAG = OFF_SLOT + (size_t)NOALLOC_MAX_PARTICLES + 64; // "not binned" flags
constexpr size_t OFF_EXOFF = OFF_FLAG + (size_t)NOALLOC_MAX_PARTICLES + 64;// their exclusive scan
constexpr size_t OFF_WS = OFF_EXOFF + (size_t)NOALLOC_MAX_PARTICLES + 64;  // scan workspace
constexpr size_t WS_INTS = 4096;
constexpr size_t SCRATCH_INTS = OFF_WS + WS_INTS;

static __device__ __align__(256) int g_sort_scratch[SCRATCH_INTS];

std::mutex g_setup_mutex;
int *g_scratch_dev[NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array for the current device.
int scratch_for_current_device(int **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return MPS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_dev[dev]) {
        int *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "mps_cell_sort_noalloc: cudaGetSymbolAddress failed: %s\n",
                         cudaGetErrorString(e));
            return MPS_ERR_CUDA;
        }
        g_scratch_dev[dev] = p;
    }
    *out = g_scratch_dev[dev];
    return MPS_OK;
}

struct NaGrid {
    double origin[3];
    double cs_inv;
    int dims[3];
    int dim;
};

// Cell of particle i as the reference computes it, -1 when not binned.
__global__ void k_na_bin(NaGrid g, const double *__restrict__ pos, const int *__restrict__ type, int n,
                         int *__restrict__ cell, int *__restrict__ count, int *__restrict__ flag)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = -1;
    if (type[i] != mps::GHOST) {
        c = 0;
        for (int d = g.dim - 1; d >= 0; d--) {
            double t = (pos[(size_t)i * g.dim + d] - g.origin[d]) * g.cs_inv;
            if (!(t > -1.0 && t < 2147483647.0)) { c = -1; break; }
            int k = __double2int_rz(t);
            if (k < 0 || k >= g.dims[d]) { c = -1; break; }
            c = c * g.dims[d] + k;
        }
    }
    cell[i] = c;
    flag[i] = (c < 0);
    if (c >= 0) atomicAdd(&count[c], 1);
}

__global__ void k_na_scatter(int n, int total, const int *__restrict__ cell, const int *__restrict__ start,
                             int *__restrict__ cursor, const int *__restrict__ exoff, int *__restrict__ slot,
                             int *__restrict__ order)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cell[i];
    if (c >= 0) slot[start[c] + atomicAdd(&cursor[c], 1)] = i;
    else order[start[total] + exoff[i]] = i;   // not binned: trailing, ascending index
}

// Within a cell: descending particle index, the reference's chain order.
__global__ void k_na_rank(const int *__restrict__ nbinned, const int *__restrict__ slot,
                          const int *__restrict__ cell, const int *__restrict__ start, int *__restrict__ order)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nbinned) return;
    int i = slot[t];
    int c = cell[i];
    int b = start[c], e = start[c + 1];
    int r = 0;
    for (int u = b; u < e; u++) r += (slot[u] > i);
    order[b + r] = i;
}

}  // namespace

extern "C" int mps_cell_sort_noalloc(const mps_grid_t *grid, const double *pos, const int *type, int num,
                                     int *cell, int *order, int *cell_start, void *stream)
{
    if (!grid || num < 0 || (num > 0 && (!pos || !type || !cell || !order)) || !cell_start) return MPS_ERR_INVALID;
    if (grid->dim != 2 && grid->dim != 3) return MPS_ERR_INVALID;
    long long total = 1;
    for (int d = 0; d < grid->dim; d++) {
        if (grid->dims[d] <= 0) return MPS_ERR_INVALID;
        total *= grid->dims[d];
    }
    if (num > NOALLOC_MAX_PARTICLES || total > NOALLOC_MAX_CELLS) {
        std::fprintf(stderr,
                     "mps_cell_sort_noalloc: %d particles / %lld cells exceed the static scratch limit of "
                     "%d particles / %d cells\n",
                     num, total, NOALLOC_MAX_PARTICLES, NOALLOC_MAX_CELLS);
        return MPS_ERR_INVALID;
    }
    if (!(grid->cell_size > 0.0)) return MPS_ERR_INVALID;
    // an error already pending in the caller's context is theirs: report it
    // without clearing it, and queue no work
    if (cudaPeekAtLastError() != cudaSuccess) return MPS_ERR_CUDA;
    int *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != MPS_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    NaGrid g{};
    g.dim = grid->dim;
    g.cs_inv = 1.0 / grid->cell_size;
    for (int d = 0; d < grid->dim; d++) {
        g.origin[d] = grid->origin[d];
        g.dims[d] = grid->dims[d];
    }
    int tot = (int)total;
    int *count = scratch + OFF_COUNT, *slot = scratch + OFF_SLOT, *flag = scratch + OFF_FLAG;
    int *exoff = scratch + OFF_EXOFF, *ws = scratch + OFF_WS;
    if (mps::scan_workspace(NOALLOC_MAX_PARTICLES + 1) > WS_INTS) return MPS_ERR_INVALID;
    // the previous call's counters: clear
    if (cudaMemsetAsync(count, 0, sizeof(int) * (tot + 1), st) != cudaSuccess) return MPS_ERR_CUDA;
    const int B = 256;
    int nb = (num + B - 1) / B;
    if (num) mps::launch(k_na_bin, nb, B, 0, st, g, pos, type, num, cell, count, flag);
    mps::scan_exclusive<int>(count, cell_start, tot, ws, st);
    mps::scan_exclusive<int>(flag, exoff, num, ws, st);
    if (cudaMemsetAsync(count, 0, sizeof(int) * (tot + 1), st) != cudaSuccess) return MPS_ERR_CUDA;
    if (num) {
        mps::launch(k_na_scatter, nb, B, 0, st, num, tot, (const int *)cell, (const int *)cell_start, count,
                    (const int *)exoff, slot, order);
        mps::launch(k_na_rank, nb, B, 0, st, (const int *)cell_start + tot, (const int *)slot, (const int *)cell,
                    (const int *)cell_start, order);
    }
    // a failed launch of this call stays pending for the caller to see
    return cudaPeekAtLastError() == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}
