// k_sort.cuh -- cell binning, counting sort and reorder (the neighbour search).
//
// Replaces the reference's cell linked list (neighbor_search.c:146-240).  The
// reference prepends particles to per-cell chains, so its neighbour lists
// visit a cell's particles in descending index order.  Here the particles
// are physically reordered every step by (cell, descending reference index):
// a histogram of cell counts, an exclusive scan, an atomic scatter into the
// cell's slot range, and a per-cell rank by index that makes the order within
// a cell deterministic.  Particles that are not binned (ghosts, outside the
// grid) go to a trailing bucket in their previous relative order.
#pragma once

#include "device.cuh"
#include "scan.cuh"

namespace mps {

// ---- binning --------------------------------------------------------------

template <int D>
__global__ void k_bin(State<D> s, Grid<D> g, int n, int *__restrict__ kcell,
                      int *__restrict__ count, int *__restrict__ excl)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = -1;
    if (s.type[i] != GHOST) {
        double p[D];
        load_vec<D>(p, s.pos, i);
        c = cell_of_pos<D>(g, p);
    }
    kcell[i] = c;
    excl[i] = (c < 0);
    if (c >= 0) atomicAdd(&count[c], 1);
}

__global__ void k_scatter(int n, int total, const int *__restrict__ kcell, const int *__restrict__ start,
                          int *__restrict__ cursor, const int *__restrict__ exoff,
                          int *__restrict__ tmp, int *__restrict__ perm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = kcell[i];
    if (c >= 0) {
        int slot = start[c] + atomicAdd(&cursor[c], 1);
        tmp[slot] = i;
    } else {
        perm[start[total] + exoff[i]] = i;
    }
}

// Position within the cell = number of cell members with a larger
// reference index (descending order, as the reference's chains).
__global__ void k_rank(const int *__restrict__ nbinned, const int *__restrict__ tmp, const int *__restrict__ kcell,
                       const int *__restrict__ start, const int *__restrict__ id, int *__restrict__ perm)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= *nbinned) return;
    int i = tmp[t];
    int c = kcell[i];
    int me = id[i];
    int b = start[c], e = start[c + 1];
    int r = 0;
    for (int u = b; u < e; u++) r += (id[tmp[u]] > me);
    perm[b + r] = i;
}

template <int D>
__global__ void k_gather(State<D> dst, State<D> src, const int *__restrict__ perm,
                         const int *__restrict__ kcell, int n, int *__restrict__ where)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int i = perm[q];
#pragma unroll
    for (int d = 0; d < D; d++) {
        double x = src.pos[d][i];
        dst.pos[d][q] = x;
        dst.key[d][q] = x;
        dst.vel[d][q] = src.vel[d][i];
        dst.acc[d][q] = src.acc[d][i];
    }
    dst.p[q] = src.p[i];
    dst.n[q] = src.n[i];
    dst.type[q] = src.type[i];
    dst.surf[q] = src.surf[i];
    dst.ncount[q] = src.ncount[i];
    int id = src.id[i];
    dst.id[q] = id;
    dst.cell[q] = kcell[i];
    where[id] = q;
}

// Reorder to reference order (engine index == reference index).
template <int D>
__global__ void k_unsort(State<D> dst, State<D> src, const int *__restrict__ where, int n)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    int q = where[r];
#pragma unroll
    for (int d = 0; d < D; d++) {
        dst.pos[d][r] = src.pos[d][q];
        dst.key[d][r] = src.key[d][q];
        dst.vel[d][r] = src.vel[d][q];
        dst.acc[d][r] = src.acc[d][q];
    }
    dst.p[r] = src.p[q];
    dst.n[r] = src.n[q];
    dst.type[r] = src.type[q];
    dst.surf[r] = src.surf[q];
    dst.ncount[r] = src.ncount[q];
    dst.id[r] = r;
    dst.cell[r] = -1;
}

// Neighbour list in the reference's layout (rows by reference index,
// entries as reference indices, reference order).  Row r starts at
// out_nb[r * pitch]; rows longer than max_nb raise the overflow flag.
template <int D>
__global__ void k_build_list(CellSource<D> src, const int *__restrict__ id, int n, int max_nb, int pitch,
                             int *__restrict__ out_nb, int *__restrict__ out_cnt, unsigned *err)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int row = id[q];
    int cnt = 0;
    size_t base = (size_t)row * (size_t)pitch;
    src.for_each(q, [&](int t) {
        if (cnt < pitch && out_nb) out_nb[base + cnt] = id[t];
        cnt++;
    });
    if (cnt > max_nb) {
        atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
        cnt = max_nb;
    }
    out_cnt[row] = cnt;
}

// Rows of a pitched host list (already on the device) into CSR.
__global__ void k_compact_list(const int *__restrict__ rows, int pitch, const int *__restrict__ cnt,
                               const int *__restrict__ ptr, int n, int *__restrict__ idx, unsigned *err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cnt[i], o = ptr[i];
    const int *r = rows + (size_t)i * pitch;
    for (int k = 0; k < c; k++) {
        int j = r[k];
        if (j < 0 || j >= n) { atomicOr(err, ERR_LIST_MISMATCH); j = 0; }
        idx[o + k] = j;
    }
}

// The same compaction read straight from a caller's list in page-locked host
// memory (device-addressable under unified addressing): one warp per row, the
// lanes striding over the row's count, so only the used entries cross the
// host link, in 128-byte runs.
__global__ void k_gather_host_list(const int *__restrict__ rows, int pitch, const int *__restrict__ cnt,
                                   const int *__restrict__ ptr, int n, int *__restrict__ idx, unsigned *err)
{
    long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (w >= n) return;
    int c = min(cnt[w], pitch), o = ptr[w];
    const int *r = rows + (size_t)w * pitch;
    for (int k = lane; k < c; k += 32) {
        int j = r[k];
        if (j < 0 || j >= n) { atomicOr(err, ERR_LIST_MISMATCH); j = 0; }
        idx[o + k] = j;
    }
}

template <int D>
__global__ void k_cell_ref_order(const int *__restrict__ cell, const int *__restrict__ id, int n, int *out)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) out[id[q]] = cell[q];
}

// Compare a caller's list (CSR by reference index, reference indices) with
// the cell structure's list, entry by entry.
template <int D>
__global__ void k_compare_list(CellSource<D> src, const int *__restrict__ id, int n,
                               const int *__restrict__ lptr, const int *__restrict__ lidx, unsigned *err)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int row = id[q];
    int k = lptr[row], e = lptr[row + 1];
    bool bad = false;
    src.for_each(q, [&](int t) {
        if (k >= e || lidx[k] != id[t]) bad = true;
        k++;
    });
    if (k != e) bad = true;
    if (bad) atomicOr(err, ERR_LIST_MISMATCH);
}

}  // namespace mps
