// k_ppe.cuh -- pressure Poisson equation: numbering, CSR assembly, IC(0)
// factorisation and the preconditioned CG iteration (FP64).
//
// Reference: mps_fluid3D_parallel/src/pressure_solver.c:368-570.
//
// Unknowns are the interior fluid and wall particles (:411-422).  The
// reference numbers them in particle order, which makes its IC(0) triangular
// solves a chain of ~1/l0 dependent levels.  Here they are numbered in block
// colour order: cells are the blocks, a cell's colour is the parity of its
// coordinates (2^dim colours), and rows go colour by colour, cell by cell,
// particle by particle.  Cells of one colour never share a matrix entry (a
// pair is coupled only when it sits in adjacent cells), so every cell of a
// colour is solved in parallel and only the rows inside a cell form a chain.
// The factor is IC(0) of this permuted matrix: the same preconditioner
// family, a different elimination order.
//
// The matrix values, diagonal sums and right-hand side are computed in the
// reference's order and are bit-identical to its assembly (tests compare the
// CSR after renumbering); rows are emitted with sorted columns directly.
#pragma once

#include "device.cuh"

namespace mps {

struct CGScalars {
    double rz, rr, pAp, alpha, beta, rz_new;
    double tol;
    double rr_outer;        // ||b - A x||^2 of the FP64 refinement (mixed form)
    int iter, done, maxit, breakdown;
};

// Visit order of the 3^D neighbour cells for PPE rows: by (colour, linear
// index), so that the columns they contribute come out ascending.  One table
// per parity of the centre cell; entries are offsets in {-1,0,1}^D.
__constant__ signed char c_order3[8][27][3];
__constant__ signed char c_order2[4][9][2];

template <int D>
__device__ __forceinline__ const signed char *order_entry(int par, int k)
{
    if (D == 3) return c_order3[par][k];
    return c_order2[par][k];
}

__device__ __forceinline__ bool is_unknown(int type, int surf)
{
    return (type == FLUID && !surf) || type == WALL;
}

// ---- numbering -------------------------------------------------------------

template <int D>
__global__ void k_cell_unknowns(State<D> s, const int *__restrict__ start, int total, int *__restrict__ ucount)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= total) return;
    int u = 0;
    for (int t = start[c]; t < start[c + 1]; t++) u += is_unknown(s.type[t], s.surf[t]);
    ucount[c] = u;
}

__global__ void k_color_gather(const int *__restrict__ ccells, const int *__restrict__ ucount, int total,
                               int *__restrict__ ucol)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < total) ucol[k] = ucount[ccells[k]];
}

// Cells holding unknowns, in colour order: flag, scan, scatter.
__global__ void k_active_flag(const int *__restrict__ ucol, int total, int *__restrict__ flag)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < total) flag[k] = ucol[k] > 0;
}

__global__ void k_active_scatter(const int *__restrict__ ccells, const int *__restrict__ ucol,
                                 const int *__restrict__ apos, int total, int *__restrict__ acells)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < total && ucol[k] > 0) acells[apos[k]] = ccells[k];
}

// Row counts and colour offsets read back in one copy.
__global__ void k_ppe_sizes(const int *__restrict__ rs, const int *__restrict__ apos, const int *__restrict__ start,
                            int total, const int *__restrict__ color_off, int ncol, int *__restrict__ out)
{
    out[0] = rs[total];        // n_eq
    out[1] = start[total];     // binned particles
    for (int c = 0; c <= ncol; c++) out[2 + c] = apos[color_off[c]];             // active cells per colour
    for (int c = 0; c <= ncol; c++) out[3 + ncol + c] = rs[color_off[c]];        // rows per colour
}

template <int D>
__global__ void k_assign_rows(State<D> s, const int *__restrict__ start, const int *__restrict__ ccells,
                              const int *__restrict__ rs, int total, int *__restrict__ cell_row0,
                              int *__restrict__ row_of, int *__restrict__ part_of_row)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= total) return;
    int c = ccells[k];
    int r = rs[k];
    cell_row0[c] = r;
    for (int t = start[c]; t < start[c + 1]; t++) {
        if (is_unknown(s.type[t], s.surf[t])) {
            row_of[t] = r;
            part_of_row[r] = t;
            r++;
        } else {
            row_of[t] = -1;
        }
    }
}

// Particles outside every cell get no row; an unknown among them would be
// a row the block order cannot place (a wall particle beyond the grid).
template <int D>
__global__ void k_offgrid_rows(State<D> s, int first, int n, int *__restrict__ row_of, unsigned *err)
{
    int t = first + blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    row_of[t] = -1;
    if (is_unknown(s.type[t], s.surf[t])) atomicOr(err, ERR_UNKNOWN_OFF_GRID);
}

// ---- assembly --------------------------------------------------------------

template <int D, class Src>
__global__ void k_row_count(Src src, State<D> s, const int *__restrict__ part_of_row,
                            const int *__restrict__ row_of, int n_eq, int *__restrict__ rcount)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int i = part_of_row[r];
    int cnt = 1;
    src.for_each(i, [&](int j) { cnt += (s.type[j] != DUMMY && row_of[j] >= 0); });
    rcount[r] = cnt;
}

// Right-hand side of one unknown row (pressure_solver.c:328-362, 524-529).
template <int D, class Src>
__device__ double ppe_rhs(const Src &src, const State<D> &s, const Consts &k, int i, const double *pi)
{
    int t = s.type[i];
    if (t == WALL) return 0.0;
    if (k.hs_mode == 1) {
        double vi[D];
        load_vec<D>(vi, s.vel, i);
        double acc = 0.0;
        src.for_each(i, [&](int j) {
            if (s.type[j] == DUMMY) return;
            double pj[D], dr[D];
            load_vec<D>(pj, s.pos, j);
            double r2 = dist2v<D>(pi, pj, dr);
            if (r2 < 1.0e-24) return;
            double r = sqrt(r2);
            double dv = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) dv += dr[d] * (s.vel[d][j] - vi[d]);
            acc += k.re_lap / (r * r * r) * dv;
        });
        return k.rhs_hs * acc;
    }
    double n0 = k.n0;
    if (k.ppe_type == 1) {
        double div = 0.0;
        if (t == FLUID) {
            double vi[D];
            load_vec<D>(vi, s.vel, i);
            double acc = 0.0;
            src.for_each(i, [&](int j) {
                if (s.type[j] == DUMMY) return;
                double pj[D], dr[D];
                load_vec<D>(pj, s.pos, j);
                double r2 = dist2v<D>(pi, pj, dr);
                if (r2 < 1.0e-24) return;
                double dv = 0.0;
#pragma unroll
                for (int d = 0; d < D; d++) dv += (s.vel[d][j] - vi[d]) * dr[d];
                acc += dv / r2 * kweight(sqrt(r2), k.re_lap, k.rmin);
            });
            div = k.grad_coeff * acc;
        }
        return k.rhs_na * div + k.rhs_nb * (s.n[i] - n0) / n0;
    }
    return k.rhs_k * (s.n[i] - n0) / n0;
}

// One row of A and b.  Pass 1 walks the list in the reference's order for
// the diagonal sum and the source term; pass 2 walks the neighbour cells in
// (colour, index) order so the off-diagonals come out with ascending
// columns, the diagonal in its place.
template <int D>
__global__ void k_fill(CellSource<D> src, State<D> s, Consts k, const int *__restrict__ part_of_row,
                       const int *__restrict__ row_of, int n_eq, const int *__restrict__ row_ptr,
                       int *__restrict__ col, double *__restrict__ val, int *__restrict__ diagpos,
                       double *__restrict__ b, unsigned *err)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int i = part_of_row[r];
    double pi[D];
    load_vec<D>(pi, s.pos, i);

    double sum_w = 0.0;
    src.for_each(i, [&](int j) {
        if (s.type[j] == DUMMY) return;
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        sum_w += kweight(sqrt(dist2<D>(pi, pj)), k.re_lap, k.rmin);
    });
    double diag = k.diag_scale * sum_w;
    b[r] = ppe_rhs<D>(src, s, k, i, pi);

    int c = s.cell[i];
    int cc[D];
    int rem = c;
#pragma unroll
    for (int d = 0; d < D; d++) { cc[d] = rem % src.g.dims[d]; rem /= src.g.dims[d]; }
    int par = 0;
#pragma unroll
    for (int d = 0; d < D; d++) par |= (cc[d] & 1) << d;
    double ki[D];
    load_vec<D>(ki, s.key, i);
    int pos = row_ptr[r];
    int end = row_ptr[r + 1];
    const int NC = (D == 3) ? 27 : 9;
    for (int q = 0; q < NC; q++) {
        const signed char *off = order_entry<D>(par, q);
        int lin = 0;
        bool inside = true;
#pragma unroll
        for (int d = D - 1; d >= 0; d--) {
            int x = cc[d] + off[d];
            if (x < 0 || x >= src.g.dims[d]) inside = false;
            lin = lin * src.g.dims[d] + x;
        }
        if (!inside) continue;
        for (int t = src.g.start[lin]; t < src.g.start[lin + 1]; t++) {
            if (t == i) {
                diagpos[r] = pos;
                col[pos] = r;
                val[pos] = diag;
                pos++;
                continue;
            }
            int rj = row_of[t];
            if (rj < 0 || s.type[t] == DUMMY) continue;
            double kt[D];
            load_vec<D>(kt, s.key, t);
            if (!(dist2<D>(ki, kt) < src.re2)) continue;
            double pt[D];
            load_vec<D>(pt, s.pos, t);
            double w = kweight(sqrt(dist2<D>(pi, pt)), k.re_lap, k.rmin);
            if (pos < end) {
                col[pos] = rj;
                val[pos] = k.neg_coeff * w;
            }
            pos++;
        }
    }
    if (pos != end) atomicOr(err, ERR_COLORING);
}

// ---- IC(0) factorisation ---------------------------------------------------
// F holds the factor in A's pattern: F[p] = L_ik below the diagonal, the
// diagonal slot holds 1/L_ii, and above the diagonal F[p] = L_ki (the
// transposed copy the backward sweep reads row-wise).

constexpr int IC_MAXM = 128;
constexpr int SWEEP_WARPS_IC = 4;

__device__ __forceinline__ int find_col(const int *__restrict__ col, int lo, int hi, int key)
{
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        int v = col[mid];
        if (v == key) return mid;
        if (v < key) lo = mid + 1; else hi = mid;
    }
    return -1;
}

__device__ __forceinline__ double warp_allsum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Entry L_rk = (A_rk - sum_{j<k} L_rj L_kj) / L_kk of row r at position p
// (column k), with the sum in ascending j as pressure_solver.c:203-219; the
// transposed copy goes to row k's upper run.
__device__ __forceinline__ void ic0_entry(int r, int p, const int *__restrict__ row_ptr,
                                          const int *__restrict__ diagpos, const int *__restrict__ col,
                                          const double *__restrict__ A, double *F)
{
    int kc = col[p];
    int a = row_ptr[r], b = row_ptr[kc], kd = diagpos[kc];
    double s = A[p];
    while (a < p && b < kd) {
        int ja = col[a], jb = col[b];
        if (ja < jb) a++;
        else if (ja > jb) b++;
        else { s -= F[a] * F[b]; a++; b++; }
    }
    double lik = s * F[kd];
    F[p] = lik;
    int up = find_col(col, kd + 1, row_ptr[kc + 1], r);
    if (up >= 0) F[up] = lik;
}

__device__ __forceinline__ void ic0_diag(int r, const int *__restrict__ row_ptr, const int *__restrict__ diagpos,
                                         const double *__restrict__ A, double *F)
{
    int pd = diagpos[r];
    double a = A[pd];
    double d = a;
    for (int q = row_ptr[r]; q < pd; q++) d -= F[q] * F[q];
    if (d <= 0.0) d = (a > 0.0) ? a : 1.0e-30;   // pressure_solver.c:200
    F[pd] = 1.0 / sqrt(d);
}

// Phase A of a colour: the cross-cell entries of its rows [rbeg, rend),
// which depend only on finished colours and on earlier entries of the same
// row.  Thread per row.
__global__ void k_ic0_cross(int rbeg, int rend, const int *__restrict__ row_ptr, const int *__restrict__ diagpos,
                            const int *__restrict__ inpos, const int *__restrict__ col,
                            const double *__restrict__ A, double *F)
{
    int r = rbeg + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rend) return;
    int pin = inpos[r];
    for (int p = row_ptr[r]; p < pin; p++) ic0_entry(r, p, row_ptr, diagpos, col, A, F);
}

// Phase B of a colour: in-cell entries and diagonals.  Warp per cell; lane l
// owns rows l, l+32, ...  At step k the owner of row k (complete by then)
// forms its diagonal, then every row with an entry in column k computes it.
__global__ void __launch_bounds__(32 * SWEEP_WARPS_IC)
k_ic0_incell(int kbeg, int kend, const int *__restrict__ acells, const int *__restrict__ cell_row0,
             const int *__restrict__ ucount, const int *__restrict__ row_ptr, const int *__restrict__ diagpos,
             const int *__restrict__ inpos, const int *__restrict__ col, const double *__restrict__ A, double *F)
{
    int lane = threadIdx.x & 31;
    int kk = kbeg + blockIdx.x * SWEEP_WARPS_IC + (threadIdx.x >> 5);
    if (kk >= kend) return;
    int c = acells[kk];
    int r0 = cell_row0[c], m = ucount[c];
    if (m > IC_MAXM) {
        if (lane == 0) {
            for (int r = r0; r < r0 + m; r++) {
                for (int p = inpos[r]; p < diagpos[r]; p++) ic0_entry(r, p, row_ptr, diagpos, col, A, F);
                ic0_diag(r, row_ptr, diagpos, A, F);
            }
        }
        __syncwarp();
        return;
    }
    constexpr int R = IC_MAXM / 32;
    int cur[R], stop[R], ccol[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        int t = lane + 32 * j;
        cur[j] = stop[j] = 0;
        ccol[j] = -1;
        if (t < m) {
            cur[j] = inpos[r0 + t];
            stop[j] = diagpos[r0 + t];
            if (cur[j] < stop[j]) ccol[j] = col[cur[j]];
        }
    }
    for (int k = 0; k < m; k++) {
        if (lane == (k & 31)) ic0_diag(r0 + k, row_ptr, diagpos, A, F);
        __syncwarp();
        int ck = r0 + k;
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (ccol[j] == ck) {
                ic0_entry(r0 + lane + 32 * j, cur[j], row_ptr, diagpos, col, A, F);
                cur[j]++;
                ccol[j] = (cur[j] < stop[j]) ? col[cur[j]] : -1;
            }
        }
        __syncwarp();
    }
}

// ---- preconditioner sweeps ------------------------------------------------
//
// Rows of a cell are contiguous, [r0, r0 + m), and the sorted columns of a
// row split into four runs: lower cross-cell (earlier colours, col < r0),
// lower in-cell (r0 <= col < row), the diagonal, upper in-cell, upper
// cross-cell (col >= r0 + m).  `inpos[r]` is the first in-cell position and
// `outpos[r]` the first upper cross-cell position of row r.
//
// A sweep over one colour runs a warp per cell in two phases:
//   1. the cross-cell products of every row of the cell, which depend only on
//      finished colours: 8 lanes per row, 4 rows at a time, into shared memory;
//   2. the in-cell triangular solve: lane l owns rows l, l+32, ...; at step k
//      the owner of row k finishes it and broadcasts the value with a
//      shuffle, and every lane whose row has an entry in column k applies it
//      (each lane walks its row's in-cell run with a cursor).
// Cells with more than SWEEP_MAXM unknowns (4x the rest density; only in a
// blow-up) take a row-by-row path with the same result.

constexpr int SWEEP_MAXM = 128;
constexpr int SWEEP_WARPS = 4;   // warps per block

// Row positions of the in-cell runs; one thread per row.
__global__ void k_row_splits(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ diagpos,
                             const int *__restrict__ col, const int *__restrict__ part_of_row,
                             const int *__restrict__ cell, const int *__restrict__ cell_row0,
                             const int *__restrict__ ucount, int *__restrict__ inpos, int *__restrict__ outpos)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int c = cell[part_of_row[r]];
    int r0 = cell_row0[c], r1 = r0 + ucount[c];
    int pd = diagpos[r];
    int q = pd;
    while (q > row_ptr[r] && col[q - 1] >= r0) q--;
    inpos[r] = q;
    q = pd + 1;
    int e = row_ptr[r + 1];
    while (q < e && col[q] < r1) q++;
    outpos[r] = q;
}

// ---- split sweeps: cross-cell products, then the in-cell solve -------------
//
// k_sweep_cross: every row of a colour (rows [rbeg, rend) are contiguous)
// sums its cross-cell run against the finished colours, LPR lanes per row,
// into part[r] = rhs[r] - sum.  k_sweep_cell: a warp per cell stages the
// cell's in-cell runs (local column index and value) and the diagonal
// inverses in shared memory, then runs the lane-per-row solve from there.

template <bool FWD, int LPR, class T>
__global__ void k_sweep_cross(int rbeg, int rend, const int *__restrict__ row_ptr, const int *__restrict__ inpos,
                              const int *__restrict__ outpos, const int *__restrict__ col,
                              const T *__restrict__ F, const T *__restrict__ rhs, const T *x,
                              T *__restrict__ part, const CGScalars *sc)
{
    if (sc->done) return;
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    int r = rbeg + t / LPR;
    int lane = t % LPR;
    T s = T(0);
    if (r < rend) {
        int a = FWD ? __ldg(&row_ptr[r]) : __ldg(&outpos[r]);
        int b = FWD ? __ldg(&inpos[r]) : __ldg(&row_ptr[r + 1]);
#pragma unroll 4
        for (int q = a + lane; q < b; q += LPR) s += __ldg(&F[q]) * x[__ldg(&col[q])];
    }
#pragma unroll
    for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
    if (lane == 0 && r < rend) part[r] = rhs[r] - s;
}

constexpr int CELL_MAXE = 1536;  // staged in-cell entries per warp (larger cells read the packed runs directly)
constexpr int CELL_WARPS = 2;    // warps per block of k_sweep_cell

// Packed in-cell factor, built once per step after the factorisation.  For
// every row r, lo: its in-cell lower entries in ascending column order
// (forward walk order), up: its in-cell upper entries in descending column
// order (backward walk order); entries hold the column's index within the
// cell and the factor value.  Rows are numbered cell by cell, so a cell's
// entries form one contiguous block.  dinv[r] = 1 / L_rr.
__global__ void k_pack_lengths(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ diagpos,
                               const int *__restrict__ inpos, const int *__restrict__ outpos,
                               int *__restrict__ len_lo, int *__restrict__ len_up)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int pd = diagpos[r];
    len_lo[r] = pd - inpos[r];
    len_up[r] = outpos[r] - pd - 1;
}

__global__ void k_pack_fill(int n_eq, const int *__restrict__ diagpos, const int *__restrict__ inpos,
                            const int *__restrict__ outpos, const int *__restrict__ col, const double *__restrict__ F,
                            const int *__restrict__ part_of_row, const int *__restrict__ cell,
                            const int *__restrict__ cell_row0, const int *__restrict__ off_lo,
                            const int *__restrict__ off_up, double *__restrict__ lo_val,
                            unsigned char *__restrict__ lo_k, double *__restrict__ up_val,
                            unsigned char *__restrict__ up_k, double *__restrict__ dinv, unsigned *err)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int r0 = cell_row0[cell[part_of_row[r]]];
    if (r - r0 > 255) atomicOr(err, ERR_CELL_OVERFULL);
    int pd = diagpos[r];
    dinv[r] = F[pd];
    int o = off_lo[r];
    for (int q = inpos[r]; q < pd; q++, o++) {
        lo_val[o] = F[q];
        lo_k[o] = (unsigned char)(col[q] - r0);
    }
    o = off_up[r];
    for (int q = outpos[r] - 1; q > pd; q--, o++) {
        up_val[o] = F[q];
        up_k[o] = (unsigned char)(col[q] - r0);
    }
}

// (first row, unknowns) of every active cell
__global__ void k_cell_desc(int nact, const int *__restrict__ acells, const int *__restrict__ cell_row0,
                            const int *__restrict__ ucount, int2 *__restrict__ desc)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nact) return;
    int c = acells[k];
    desc[k] = make_int2(cell_row0[c], ucount[c]);
}

// Lane-per-row solve of one cell from a staged entry block (lo/up runs in
// walk order, local column index in `ks`).  R = row slots per lane.
template <bool FWD, int R, class T>
__device__ __forceinline__ void cell_solve(int r0, int m, const int *off, const int *len, T *acc,
                                           const T *dv, const T *vals, const unsigned char *ks,
                                           T *__restrict__ x)
{
    int lane = threadIdx.x & 31;
    int cur[R], ck[R];
    T cv[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        cur[j] = off[j];
        int end = off[j] + len[j];
        ck[j] = (cur[j] < end) ? (int)ks[cur[j]] : -1;
        cv[j] = (cur[j] < end) ? vals[cur[j]] : T(0);
    }
    for (int sidx = 0; sidx < m; sidx++) {
        int k = FWD ? sidx : m - 1 - sidx;
        int owner = k & 31;
        T v = T(0);
        if (R == 1) {
            if (lane == owner) {
                v = acc[0] * dv[0];
                x[r0 + k] = v;
            }
        } else {
            int slot = k >> 5;
#pragma unroll
            for (int j = 0; j < R; j++)
                if (j == slot && lane == owner) {
                    v = acc[j] * dv[j];
                    x[r0 + k] = v;
                }
        }
        v = __shfl_sync(0xffffffffu, v, owner);
#pragma unroll
        for (int j = 0; j < R; j++) {
            if (ck[j] == k) {
                acc[j] -= cv[j] * v;
                ++cur[j];
                bool more = cur[j] < off[j] + len[j];
                ck[j] = more ? (int)ks[cur[j]] : -1;
                cv[j] = more ? vals[cur[j]] : T(0);
            }
        }
    }
}

// In-cell solve of one colour, a warp per cell (see the section comment).
// part[r] = rhs[r] - cross-cell sum; writes x for the cell's rows.
template <bool FWD, class T>
__global__ void __launch_bounds__(32 * CELL_WARPS)
k_sweep_cell(int kbeg, int kend, const int2 *__restrict__ desc, const int *__restrict__ pk_off,
             const int *__restrict__ pk_len, const T *__restrict__ pk_val,
             const unsigned char *__restrict__ pk_k, const T *__restrict__ dinv,
             const T *__restrict__ part, T *__restrict__ x, const CGScalars *sc)
{
    __shared__ T s_val[CELL_WARPS][CELL_MAXE];
    __shared__ unsigned char s_k[CELL_WARPS][CELL_MAXE];
    if (sc->done) return;
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int kk = kbeg + blockIdx.x * CELL_WARPS + w;
    if (kk >= kend) return;
    int2 dd = desc[kk];
    int r0 = dd.x, m = dd.y;
    if (m > SWEEP_MAXM) {
        // larger than the lane slots: row by row from the packed runs
        for (int t = 0; t < m; t++) {
            int r = FWD ? r0 + t : r0 + m - 1 - t;
            int o = pk_off[r], l = pk_len[r];
            T ps = T(0);
            for (int e = lane; e < l; e += 32) ps += pk_val[o + e] * x[r0 + pk_k[o + e]];
#pragma unroll
            for (int q = 16; q > 0; q >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, q);
            if (lane == 0) x[r] = (part[r] - ps) * dinv[r];
            __syncwarp();
        }
        return;
    }
    constexpr int R = SWEEP_MAXM / 32;
    int off[R], len[R];
    T acc[R], dv[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        int t = lane + 32 * j;
        off[j] = len[j] = 0;
        acc[j] = dv[j] = T(0);
        if (t < m) {
            int r = r0 + t;
            off[j] = pk_off[r];
            len[j] = pk_len[r];
            acc[j] = part[r];
            dv[j] = dinv[r];
        }
    }
    int base = __shfl_sync(0xffffffffu, off[0], 0);
    int endo = 0;
#pragma unroll
    for (int j = 0; j < R; j++) endo = max(endo, len[j] > 0 ? off[j] + len[j] : 0);
#pragma unroll
    for (int q = 16; q > 0; q >>= 1) endo = max(endo, __shfl_xor_sync(0xffffffffu, endo, q));
    int total = endo > base ? endo - base : 0;
    const T *vals;
    const unsigned char *ks;
    if (total <= CELL_MAXE) {
#pragma unroll 4
        for (int e = lane; e < total; e += 32) {
            s_val[w][e] = pk_val[base + e];
            s_k[w][e] = pk_k[base + e];
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < R; j++) off[j] -= base;
        vals = s_val[w];
        ks = s_k[w];
    } else {
        vals = pk_val;
        ks = pk_k;
    }
    if (m <= 32) cell_solve<FWD, 1, T>(r0, m, off, len, acc, dv, vals, ks, x);
    else if (m <= 64) cell_solve<FWD, 2, T>(r0, m, off, len, acc, dv, vals, ks, x);
    else cell_solve<FWD, 4, T>(r0, m, off, len, acc, dv, vals, ks, x);
}

// ---- CG vector kernels ------------------------------------------------------

constexpr int CG_BLOCK = 256;

// Sum of partials[0..n) (stride `stride`, offset `o`) by the whole last
// block: thread t adds slots t, t+CG_BLOCK, ... in order, then a fixed
// tree; the result (valid in thread 0) is the same on every run.
__device__ __forceinline__ double final_sum(const double *partials, unsigned n, int stride, int o, double *sh)
{
    double a = 0.0;
    for (unsigned b = threadIdx.x; b < n; b += CG_BLOCK) a += __ldcg(&partials[(size_t)b * stride + o]);
    return block_sum<CG_BLOCK>(a, sh);
}

// Ap = A p and the p.Ap partial; the last block forms alpha.  The kernel
// also performs the loop-head test of the reference (sqrt(r.r) < tol, and
// the iteration cap) before any work.
template <int LPR, class T>
__global__ void k_cg_spmv(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                          const T *__restrict__ A, const T *__restrict__ p, T *__restrict__ Ap,
                          double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    if (sc->done) return;
    if (sqrt(sc->rr) < sc->tol || sc->iter >= sc->maxit) {
        if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 1;
        return;
    }
    int lane = threadIdx.x % LPR;
    int rows_per_block = CG_BLOCK / LPR;
    double acc = 0.0;
    for (int rb = blockIdx.x * rows_per_block; rb < n_eq; rb += gridDim.x * rows_per_block) {
        int r = rb + threadIdx.x / LPR;
        T s = T(0);
        if (r < n_eq) {
            int q1 = __ldg(&row_ptr[r + 1]);
#pragma unroll 4
            for (int q = __ldg(&row_ptr[r]) + lane; q < q1; q += LPR) s += __ldg(&A[q]) * p[__ldg(&col[q])];
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && r < n_eq) {
            Ap[r] = s;
            acc += (double)p[r] * (double)s;
        }
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) {
            sc->pAp = tot;
            if (fabs(tot) < 1.0e-30) { sc->done = 1; sc->breakdown = 1; }
            else sc->alpha = sc->rz / tot;
        }
    }
}

// x += alpha p, r -= alpha Ap, and r.r.
template <class T>
__global__ void k_cg_axpy(int n_eq, T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
                          const T *__restrict__ Ap, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    if (sc->done) return;
    T alpha = (T)sc->alpha;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        T ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        acc += (double)ri * (double)ri;
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) sc->rr = tot;
    }
}

// rz_new = r.z, the breakdown test on the previous rz, beta.
template <class T>
__global__ void k_cg_rz(int n_eq, const T *__restrict__ r, const T *__restrict__ z,
                        double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    if (sc->done) return;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x)
        acc += (double)r[i] * (double)z[i];
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) {
            sc->rz_new = tot;
            if (fabs(sc->rz) < 1.0e-60) { sc->done = 1; sc->breakdown = 1; }
            else { sc->beta = tot / sc->rz; sc->rz = tot; }
        }
    }
}

template <class T>
__global__ void k_cg_update_p(int n_eq, T *__restrict__ p, const T *__restrict__ z, CGScalars *sc)
{
    if (sc->done) return;
    T beta = (T)sc->beta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->iter += 1;
}

// x = 0, r = b.
template <class T>
__global__ void k_cg_init(int n_eq, T *__restrict__ x, T *__restrict__ r, const T *__restrict__ b)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        x[i] = T(0);
        r[i] = b[i];
    }
}

// p = z, rz = r.z, rr = r.r.
template <class T>
__global__ void k_cg_init2(int n_eq, const T *__restrict__ r, const T *__restrict__ z,
                           T *__restrict__ p, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double a = 0.0, b2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        T ri = r[i], zi = z[i];
        p[i] = zi;
        a += (double)ri * (double)zi;
        b2 += (double)ri * (double)ri;
    }
    double ta = block_sum<CG_BLOCK>(a, sh);
    double tb = block_sum<CG_BLOCK>(b2, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = ta;
        partials[2 * blockIdx.x + 1] = tb;
    }
    if (last_block(ticket, gridDim.x)) {
        double sa = final_sum(partials, gridDim.x, 2, 0, sh);
        double sb = final_sum(partials, gridDim.x, 2, 1, sh);
        if (threadIdx.x == 0) {
            sc->rz = sa;
            sc->rr = sb;
            sc->iter = 0;
            sc->done = 0;
            sc->breakdown = 0;
        }
    }
}

// ---- mixed precision: conversions and the FP64 refinement --------------------

template <class S, class T>
__global__ void k_convert(size_t n, const S *__restrict__ in, T *__restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = (T)in[i];
}

// x64 = 0, r64 = b, r32 = (float) b, ||b||^2 into sc->rr_outer.
__global__ void k_refine_init(int n_eq, double *__restrict__ x, double *__restrict__ r, float *__restrict__ r32,
                              const double *__restrict__ b, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        double bi = b[i];
        x[i] = 0.0;
        r[i] = bi;
        r32[i] = (float)bi;
        acc += bi * bi;
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) sc->rr_outer = tot;
    }
}

// x64 += (double) d32; then the FP64 residual r = b - A x with the FP64
// matrix, its FP32 copy and ||r||^2 (8 lanes per row).
__global__ void k_refine_update(int n_eq, double *__restrict__ x, const float *__restrict__ d)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x)
        x[i] += (double)d[i];
}

__global__ void k_refine_residual(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                                  const double *__restrict__ A, const double *__restrict__ x,
                                  const double *__restrict__ b, double *__restrict__ r, float *__restrict__ r32,
                                  double *partials, unsigned *ticket, CGScalars *sc)
{
    constexpr int LPR = 8;
    __shared__ double sh[CG_BLOCK / 32];
    int lane = threadIdx.x % LPR;
    int rows_per_block = CG_BLOCK / LPR;
    double acc = 0.0;
    for (int rb = blockIdx.x * rows_per_block; rb < n_eq; rb += gridDim.x * rows_per_block) {
        int i = rb + threadIdx.x / LPR;
        double s = 0.0;
        if (i < n_eq) {
            int q1 = __ldg(&row_ptr[i + 1]);
            for (int q = __ldg(&row_ptr[i]) + lane; q < q1; q += LPR) s += __ldg(&A[q]) * x[__ldg(&col[q])];
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && i < n_eq) {
            double ri = b[i] - s;
            r[i] = ri;
            r32[i] = (float)ri;
            acc += ri * ri;
        }
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) sc->rr_outer = tot;
    }
}

template <int D>
__global__ void k_writeback(State<D> s, const int *__restrict__ row_of, const double *__restrict__ x, int n,
                            int clamp)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = row_of[i];
    double P = (r >= 0) ? x[r] : 0.0;
    if (clamp && s.type[i] == FLUID && P < 0.0) P = 0.0;
    s.p[i] = P;
}

// PPE in the reference's numbering, for parity checks: entries of row r go
// to row eq(i) with columns eq(j).
__global__ void k_ref_eq(const int *__restrict__ row_of, const int *__restrict__ id, int n,
                         int *__restrict__ unknown_by_id)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) unknown_by_id[id[q]] = row_of[q];
}

// ---- initial parameters (particle.c:69-221) -------------------------------

// Per fluid particle: n0_i over re_n and the lambda numerator/denominator
// over re_lap, summed in ascending reference index j as the reference's
// all-pairs loop does; candidates come from a grid of cell size
// rmax*(1+1e-9) over the particles' bounding box.  Also the count of
// r2 < re_n^2 for N0.
template <int D>
__global__ void k_initial_params(State<D> s, int n, Grid<D> g, const int *__restrict__ gcell,
                                 const int *__restrict__ order, double rmax, double re_n, double re_lap,
                                 double rmin, double *__restrict__ n0i, double *__restrict__ numi,
                                 double *__restrict__ deni, int *__restrict__ cnti, unsigned *err)
{
    constexpr int CAP = 640;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    n0i[i] = -1.0;
    if (s.type[i] != FLUID) return;
    int cj[CAP];
    double cr[CAP];
    int m = 0;
    double pi[D];
    load_vec<D>(pi, s.pos, i);
    double rmax2 = rmax * rmax, re_n2 = re_n * re_n;
    int c = gcell[i];
    int cc[D];
    int rem = c;
#pragma unroll
    for (int d = 0; d < D; d++) { cc[d] = rem % g.dims[d]; rem /= g.dims[d]; }
    int lo[D], hi[D], k[D];
#pragma unroll
    for (int d = 0; d < D; d++) {
        lo[d] = cc[d] > 0 ? cc[d] - 1 : 0;
        hi[d] = cc[d] < g.dims[d] - 1 ? cc[d] + 1 : g.dims[d] - 1;
        k[d] = lo[d];
    }
    bool overflow = false;
    for (;;) {
        int lin = 0;
#pragma unroll
        for (int d = D - 1; d >= 0; d--) lin = lin * g.dims[d] + k[d];
        for (int t = g.start[lin]; t < g.start[lin + 1]; t++) {
            int j = order[t];
            if (j == i) continue;
            double pj[D];
            load_vec<D>(pj, s.pos, j);
            double r2 = dist2<D>(pi, pj);
            if (!(r2 < rmax2) && !(sqrt(r2) < rmax)) continue;
            if (m < CAP) {
                // insertion by reference index keeps the candidates sorted
                int idj = s.id[j];
                int q = m;
                while (q > 0 && cj[q - 1] > idj) { cj[q] = cj[q - 1]; cr[q] = cr[q - 1]; q--; }
                cj[q] = idj;
                cr[q] = r2;
                m++;
            } else {
                overflow = true;
            }
        }
        int d = 0;
        while (d < D && ++k[d] > hi[d]) { k[d] = lo[d]; d++; }
        if (d == D) break;
    }
    if (overflow) atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
    double a = 0.0, num = 0.0, den = 0.0;
    int cnt = 0;
    for (int q = 0; q < m; q++) {
        double r2 = cr[q];
        double r = sqrt(r2);
        double wn = kweight(r, re_n, rmin);
        if (wn > 0.0) a += wn;
        double wl = kweight(r, re_lap, rmin);
        if (wl > 0.0) { num += r2 * wl; den += wl; }
        cnt += (r2 < re_n2);
    }
    n0i[i] = a;
    numi[i] = num;
    deni[i] = den;
    cnti[i] = cnt;
}

template <int D>
__global__ void k_bbox_cell(State<D> s, int n, Grid<D> g, double cs, const double *lo, int *__restrict__ gcell,
                            int *__restrict__ count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int lin = 0;
#pragma unroll
    for (int d = D - 1; d >= 0; d--) {
        int x = (int)((s.pos[d][i] - lo[d]) / cs);
        if (x >= g.dims[d]) x = g.dims[d] - 1;
        if (x < 0) x = 0;
        lin = lin * g.dims[d] + x;
    }
    gcell[i] = lin;
    atomicAdd(&count[lin], 1);
}

__global__ void k_bbox_scatter(int n, const int *__restrict__ gcell, const int *__restrict__ start,
                               int *__restrict__ cursor, int *__restrict__ order)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = gcell[i];
    order[start[c] + atomicAdd(&cursor[c], 1)] = i;
}

// Arg-max of n0_i: the largest value, the smallest reference index among
// equal values (the serial reference's first strict maximum).  Single block.
template <int D>
__global__ void k_initial_argmax(State<D> s, int n, const double *__restrict__ n0i, const int *__restrict__ cnti,
                                 double *out_val, int *out_q, int *out_cnt)
{
    __shared__ double sv[1024];
    __shared__ int si[1024];
    __shared__ int sq[1024];
    __shared__ int sc[1024];
    double bv = -1.0;
    int bi = 0x7fffffff, bq = -1, bc = 0;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        double v = n0i[q];
        int id = s.id[q];
        if (v > bv || (v == bv && id < bi)) { bv = v; bi = id; bq = q; }
        if (v >= 0.0 && cnti[q] > bc) bc = cnti[q];
    }
    sv[threadIdx.x] = bv;
    si[threadIdx.x] = bi;
    sq[threadIdx.x] = bq;
    sc[threadIdx.x] = bc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            double v = sv[threadIdx.x + o];
            int id = si[threadIdx.x + o];
            if (v > sv[threadIdx.x] || (v == sv[threadIdx.x] && id < si[threadIdx.x])) {
                sv[threadIdx.x] = v;
                si[threadIdx.x] = id;
                sq[threadIdx.x] = sq[threadIdx.x + o];
            }
            if (sc[threadIdx.x + o] > sc[threadIdx.x]) sc[threadIdx.x] = sc[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *out_val = sv[0];
        *out_q = sq[0];
        *out_cnt = sc[0];
    }
}

}  // namespace mps
