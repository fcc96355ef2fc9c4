// scan.cuh -- exclusive prefix sum over device arrays (any length).
//
// Template-only, so several translation units can include it.
#pragma once

#include "device.cuh"

namespace mps {

// ---- exclusive scan (any length, recursive over block sums) -------------

constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <class T>
__global__ void k_scan_tile(const T *__restrict__ in, T *__restrict__ out, T *__restrict__ sums, int n)
{
    __shared__ T warp_tot[SCAN_THREADS / 32];
    int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    T v[SCAN_ITEMS];
    T run = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        T x = (base + k < n) ? in[base + k] : T(0);
        v[k] = run;
        run += x;
    }
    // inclusive warp scan of the per-thread totals
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
        T t = (lane < SCAN_THREADS / 32) ? warp_tot[lane] : T(0);
        T ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        if (lane < SCAN_THREADS / 32) warp_tot[lane] = ti - t;   // exclusive
        if (lane == SCAN_THREADS / 32 - 1 && sums) sums[blockIdx.x] = ti;
    }
    __syncthreads();
    T off = warp_tot[w] + (inc - run);
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++)
        if (base + k < n) out[base + k] = v[k] + off;
}

template <class T>
__global__ void k_scan_add(T *__restrict__ out, const T *__restrict__ offs, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += offs[i / SCAN_TILE];
}

// out[0..n) = exclusive scan of in[0..n); out[n] = total.  `ws` needs
// scan_workspace(n) elements.
inline size_t scan_workspace(int n)
{
    size_t s = 0;
    int m = n;
    while (m > SCAN_TILE) {
        m = (m + SCAN_TILE - 1) / SCAN_TILE;
        s += 2 * (size_t)m + 1;
    }
    return s + 2;
}

template <class T>
__global__ void k_scan_total(const T *in, const T *out, T *tot, int n)
{
    if (n == 0) { *tot = 0; return; }
    *tot = out[n - 1] + in[n - 1];
}

template <class T>
void scan_exclusive(const T *in, T *out, int n, T *ws, cudaStream_t st)
{
    if (n <= 0) {
        launch(k_scan_total<T>, 1, 1, 0, st, in, out, out, 0);
        return;
    }
    int nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        launch(k_scan_tile<T>, 1, SCAN_THREADS, 0, st, in, out, nullptr, n);
    } else {
        T *sums = ws;
        T *sums_scan = ws + nb;   // nb + 1 entries via the recursion
        launch(k_scan_tile<T>, nb, SCAN_THREADS, 0, st, in, out, sums, n);
        scan_exclusive<T>(sums, sums_scan, nb, ws + 2 * nb + 1, st);
        launch(k_scan_add<T>, (n + 255) / 256, 256, 0, st, out, sums_scan, n);
    }
    launch(k_scan_total<T>, 1, 1, 0, st, in, out, out + n, n);
}

}  // namespace mps
