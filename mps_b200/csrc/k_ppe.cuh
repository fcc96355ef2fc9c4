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
    double bb;              // ||b||^2 (k_true_residual)
    double ff;              // || |b| + |A| |x| ||^2 (k_true_residual, k_refine_residual)
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

// Phase A, warp per row: the entries of the row stay sequential (each needs
// the row's earlier entries), but each entry's sparse dot product
// sum_{j<k} L_rj L_kj is spread over the lanes: they take row k's lower
// entries j and look each up in the row's finished prefix by binary search,
// then a warp sum.  This is phase A of a colour: the cross-cell entries of
// its rows [rbeg, rend), which depend only on finished colours and on
// earlier entries of the same row.
__global__ void k_ic0_cross_warp(int rbeg, int rend, const int *__restrict__ row_ptr,
                                 const int *__restrict__ diagpos, const int *__restrict__ inpos,
                                 const int *__restrict__ col, const double *__restrict__ A, double *F)
{
    int r = rbeg + (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (r >= rend) return;   // warp-uniform
    int a0 = row_ptr[r], pin = inpos[r];
    for (int p = a0; p < pin; p++) {
        int kc = col[p];
        int b = row_ptr[kc], kd = diagpos[kc];
        double s = 0.0;
        for (int q = b + lane; q < kd; q += 32) {
            int f = find_col(col, a0, p, col[q]);
            if (f >= 0) s += F[f] * F[q];
        }
        s = warp_allsum(s);
        if (lane == 0) {
            double lik = (A[p] - s) * F[kd];
            F[p] = lik;
            int up = find_col(col, kd + 1, row_ptr[kc + 1], r);
            if (up >= 0) F[up] = lik;
        }
        __syncwarp();
    }
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
// A colour's part of a sweep is its cross-cell products (which depend only
// on finished colours) followed by its in-cell triangular solve.  The solve
// is the product with the inverse of the cell's diagonal block of the factor
// (formed once per step after the factorisation, k_cell_inverse): the same
// preconditioner as substitution, rounded differently, with no serial chain
// through the cell's rows.  Cells with more than SWEEP_MAXM unknowns (over
// twice the most a cell of side re holds at rest spacing; only in a blow-up)
// are solved row by row by substitution from the packed in-cell runs.  One
// launch per colour (k_sweep_colour) does the colour's in-cell part and the
// next colour's cross products from colours already finished.

constexpr int SWEEP_MAXM = 64;

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

// ---- packed cross-cell runs ----------------------------------------------------

// Cross-cell runs of the factor, packed once per step into their own CSR
// (lo: the lower cross run [row_ptr, inpos) of every row, for the forward
// sweep; up: the upper cross run [outpos, row_ptr+1), for the backward one)
// so that a colour's cross entries are one contiguous stream.
__global__ void k_cross_lengths(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ inpos,
                                const int *__restrict__ outpos, int *__restrict__ len_lo, int *__restrict__ len_up)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    len_lo[r] = inpos[r] - row_ptr[r];
    len_up[r] = row_ptr[r + 1] - outpos[r];
}

// Colour bookkeeping of the sweeps: the first row of each colour, and per
// colour the column thresholds that split a row's packed cross runs by the
// colour of their entries (rows are numbered colour by colour, so columns
// are ordered by colour too):
//   lo run (forward): entries with col >= thr_lo[k] come from the colour
//     swept just before colour k (its "tail"), the others from earlier ones;
//   up run (backward): entries with col < thr_up[k] come from the colour
//     swept just before colour k in the backward order (the tail).
struct SweepColours {
    int row_off[9];
    int thr_lo[8], thr_up[8];
    int ncol;
};

__global__ void k_cross_fill(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ inpos,
                             const int *__restrict__ outpos, const int *__restrict__ col,
                             const double *__restrict__ F, const int *__restrict__ xp_lo,
                             const int *__restrict__ xp_up, int *__restrict__ xc_lo, double *__restrict__ xf_lo,
                             int *__restrict__ xc_up, double *__restrict__ xf_up, SweepColours sc,
                             int *__restrict__ xs_lo, int *__restrict__ xs_up)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int k = 0;
    while (k + 1 < sc.ncol && r >= sc.row_off[k + 1]) k++;
    int o = xp_lo[r], split = o;
    for (int q = row_ptr[r]; q < inpos[r]; q++, o++) {
        xc_lo[o] = col[q];
        xf_lo[o] = F[q];
        split += col[q] < sc.thr_lo[k];
    }
    xs_lo[r] = split;
    o = xp_up[r];
    split = o;
    for (int q = outpos[r]; q < row_ptr[r + 1]; q++, o++) {
        xc_up[o] = col[q];
        xf_up[o] = F[q];
        split += col[q] < sc.thr_up[k];
    }
    xs_up[r] = split;
}

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

// ---- in-cell block inverses ---------------------------------------------------
//
// The in-cell diagonal block L_cc of the factor is inverted once per step, so
// that the in-cell part of a sweep is a dense triangular product, a warp per
// cell with no serial chain.  Each cell of at most SWEEP_MAXM unknowns owns
// m(m+1)/2 entries (padded to a multiple of 4) at inv_off[k] in two layouts:
//   column-major (forward sweep):  (L^-1)_{ij}, i >= j, at colofs(j) + i - j,
//   row-major    (backward sweep): (L^-1)_{ji}, i <= j, at j(j+1)/2 + i,
// so that at step j the warp's lanes read consecutive addresses.

__host__ __device__ __forceinline__ int tri_colofs(int j, int m) { return j * m - (j * (j - 1)) / 2; }

// Entries of every active cell's inverse, padded to a multiple of 4 so that
// every block starts 16-byte aligned in both the FP64 and FP32 copies (0 for
// cells above SWEEP_MAXM).
__global__ void k_inv_sizes(int nact, const int2 *__restrict__ desc, int *__restrict__ len)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nact) return;
    int m = desc[k].y;
    len[k] = m <= SWEEP_MAXM ? ((m * (m + 1) / 2) + 3) & ~3 : 0;
}

// Column c of L_cc^-1 by forward substitution over the packed lower runs,
// lane per column (columns lane and lane + 32), rows in order:
//   X_ic = (delta_ic - sum_{c <= k < i} L_ik X_kc) / L_ii.
// The rows' runs are read by all lanes at once; X is kept in the
// column-major output and mirrored into the row-major one.
__global__ void __launch_bounds__(128)
k_cell_inverse(int nact, const int2 *__restrict__ desc, const int *__restrict__ inv_off,
               const int *__restrict__ pk_off, const int *__restrict__ pk_len, const double *__restrict__ pk_val,
               const unsigned char *__restrict__ pk_k, const double *__restrict__ dinv, double *inv_cm,
               double *__restrict__ inv_rm)
{
    int lane = threadIdx.x & 31;
    int kk = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (kk >= nact) return;
    int2 dd = desc[kk];
    int r0 = dd.x, m = dd.y;
    if (m > SWEEP_MAXM) return;
    double *cm = inv_cm + inv_off[kk];
    double *rm = inv_rm + inv_off[kk];
    for (int i = 0; i < m; i++) {
        int r = r0 + i;
        int ro = pk_off[r], rl = pk_len[r];
        double di = dinv[r];
#pragma unroll
        for (int j = 0; j < SWEEP_MAXM / 32; j++) {
            int c = lane + 32 * j;
            if (c > i) continue;
            const double *xc = cm + tri_colofs(c, m) - c;   // X_kc at xc[k]
            double s = (c == i) ? 1.0 : 0.0;
            for (int e = 0; e < rl; e++) {
                int k = pk_k[ro + e];
                if (k >= c) s -= pk_val[ro + e] * xc[k];
            }
            double v = s * di;
            cm[tri_colofs(c, m) + i - c] = v;
            rm[i * (i + 1) / 2 + c] = v;
        }
    }
}

// ---- bulk copies into shared memory (cp.async.bulk + mbarrier) ----------------

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// One bulk copy global -> shared of `bytes` (a multiple of 16; both
// addresses 16-byte aligned), completing on the mbarrier at `bar`.
__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(bar)
                 : "memory");
}

// Bounded wait for phase `parity` of the mbarrier: false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, int limit)
{
    for (int i = 0; i < limit; i++) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

constexpr int MBAR_POLLS = 1 << 20;
constexpr int MBAR_DRAIN_POLLS = 1 << 26;

// Bounded wait for a warp's bulk copy: false (and ERR_COPY_TIMEOUT set)
// after `polls` polls, in which case the copy is first waited for with the
// long bound, so that the warp never leaves it in flight.
__device__ __forceinline__ bool stage_wait(unsigned bar, int polls, unsigned *err)
{
    if (mbar_wait(bar, 0, polls)) return true;
    atomicOr(err, ERR_COPY_TIMEOUT);
    for (int i = 0; i < MBAR_DRAIN_POLLS; i++) {
        if (mbar_wait(bar, 0, 1)) break;
        __nanosleep(64);
    }
    return false;
}


// ---- staged in-cell sweep -----------------------------------------------------
//
// The cells of one colour are consecutive in the block-inverse arrays, so a
// colour splits into windows of CELL_WIN entries: window w holds the cells
// whose blocks start in [w CELL_WIN, (w+1) CELL_WIN) of the colour's range,
// one contiguous run of at most win + CELL_MAXBLK entries (the stage).  A CTA per window copies
// its run into shared memory with one bulk copy, issued before pdl_wait() so
// that it overlaps the preceding cross-cell kernel, then its warps take the
// window's cells in turn.

constexpr int CELL_WIN = 1024;        // default FP64 window (entries; 8 KB); MPS_CELL_WIN selects 256..4096
constexpr int CELL_WIN_MAX = 4096;
constexpr int CELL_MAXBLK = ((SWEEP_MAXM * (SWEEP_MAXM + 1) / 2) + 3) & ~3;
constexpr int CELL_STAGE_MAX = CELL_WIN_MAX + CELL_MAXBLK;
constexpr int CELL_THREADS = 256;

// First cell of every window of one colour (cells [kbeg, kend)); entry nwin
// is kend.  Lower bound of the window start among the cells' offsets.
__global__ void k_inv_windows(int kbeg, int kend, const int *__restrict__ inv_off, int win, int nwin,
                              int *__restrict__ wfirst)
{
    int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w > nwin) return;
    if (w == nwin) {
        wfirst[w] = kend;
        return;
    }
    int target = inv_off[kbeg] + w * win;
    int lo = kbeg, hi = kend;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (inv_off[mid] < target) lo = mid + 1;
        else hi = mid;
    }
    wfirst[w] = lo;
}

struct ColourIdx {
    int k[9];
};

// inv_off at the colour boundaries (the colours' ranges and the total).
__global__ void k_gather_colour_offsets(ColourIdx at, int n, const int *__restrict__ inv_off, int *__restrict__ out)
{
    int t = threadIdx.x;
    if (t < n) out[t] = inv_off[at.k[t]];
}

// ---- packed FP32 entries -------------------------------------------------------
//
// The mixed form's FP32 matrix and cross runs can be stored as one 8-byte
// word per entry (the value's bits, the column): one load per entry instead
// of a 4-byte value load and a 4-byte column load, so a warp's load request
// moves as many bytes as an FP64 value load does.

// out[i] = (bits of (float)val[i], col[i]): the FP32 value rounds to
// nearest, as k_convert<double, float> does.
__global__ void k_pack_fc(size_t n, const double *__restrict__ val, const int *__restrict__ col,
                          uint2 *__restrict__ out)
{
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        out[i] = make_uint2(__float_as_uint((float)val[i]), (unsigned)col[i]);
}

// Entry q of a run (value v, column k): from the packed words when PK, else
// from the value and column arrays; (0, -1) when !ok.
template <class TM, bool PK>
__device__ __forceinline__ void load_entry(const TM *__restrict__ f, const int *__restrict__ c,
                                           const uint2 *__restrict__ fc, int q, bool ok, TM &v, int &k)
{
    if (PK) {
        uint2 e = ok ? __ldg(&fc[q]) : make_uint2(0u, 0xffffffffu);
        v = TM(__uint_as_float(e.x));
        k = (int)e.y;
    } else {
        v = ok ? __ldg(&f[q]) : TM(0);
        k = ok ? __ldg(&c[q]) : -1;
    }
}

// ---- one launch per colour ---------------------------------------------------
//
// k_sweep_colour finishes colour c and starts the next colour of the sweep
// in one launch, with two kinds of CTA:
//   window CTAs (blockIdx < nwin): for the rows of one window of colour c,
//     part[r] = base[r] - F x over the row's tail (the entries from the
//     colour swept just before c, finished by the previous launch), where
//     base is rhs for the sweep's first colour and otherwise the head sums
//     left in part by the previous launch; then, after a block barrier, the
//     in-cell product of every cell of the window from its block inverse,
//     staged in shared memory by one bulk copy issued before pdl_wait();
//   cross CTAs: for the rows of the next colour, part[r] = rhs[r] - F x over
//     the row's head (entries from colours swept before c, all finished).
// Forward: the lo runs, head [xp, xs), tail [xs, xp+1); backward: the up
// runs, tail [xp, xs), head [xs, xp+1).  Launched as a programmatic
// dependent: what it loads before pdl_wait() (row bounds, factor values and
// columns, block inverses, cell descriptors) is written once per step,
// before the CG loop; x, part and the CG scalars are read only after it.
// PK (FP32 only): the cross entries come from the packed words xfc instead of
// xf and xc, with the same sums in the same order.
template <bool FWD, class TM, int HB = 4, int MINB = 6, int HR = 1, bool PK = false>
__global__ void __launch_bounds__(CELL_THREADS, MINB)
k_sweep_colour(const int *__restrict__ wfirst, int nwin, const int2 *__restrict__ desc,
               const int *__restrict__ inv_off, const TM *__restrict__ inv, const int *__restrict__ pk_off,
               const int *__restrict__ pk_len, const TM *__restrict__ pk_val, const unsigned char *__restrict__ pk_k,
               const TM *__restrict__ dinv, const int *__restrict__ xp, const int *__restrict__ xs,
               const int *__restrict__ xc, const TM *__restrict__ xf, int first, int nrb, int nre, const double *rhs,
               double *part, double *x, const CGScalars *sc, int stage_elems, int first_polls, unsigned *err,
               const uint2 *__restrict__ xfc = nullptr)
{
    using T = double;   // vectors and sums; TM is the storage type of the factor
    constexpr int LPR = 8;
    extern __shared__ __align__(128) unsigned char cell_stage[];
    __shared__ __align__(8) unsigned long long bar;
    pdl_trigger();
    if ((int)blockIdx.x >= nwin) {
        // cross CTA: head sums of the next colour's rows, HR rows per group
        // of LPR lanes (the CTA's groups take GPB consecutive rows per h),
        // all their first entries loaded before the wait
        constexpr int GPB = CELL_THREADS / LPR;
        int blk = blockIdx.x - nwin;
        int lane = threadIdx.x % LPR;
        int r[HR], a[HR], b[HR];
#pragma unroll
        for (int h = 0; h < HR; h++) {
            r[h] = nrb + (blk * HR + h) * GPB + threadIdx.x / LPR;
            a[h] = 0;
            b[h] = 0;
            if (r[h] < nre) {
                a[h] = FWD ? __ldg(&xp[r[h]]) : __ldg(&xs[r[h]]);
                b[h] = FWD ? __ldg(&xs[r[h]]) : __ldg(&xp[r[h] + 1]);
            }
        }
        // the first HB entries of each lane in one batch, before the wait
        TM f[HR][HB];
        int cc[HR][HB];
#pragma unroll
        for (int h = 0; h < HR; h++)
#pragma unroll
            for (int u = 0; u < HB; u++) {
                int q = a[h] + lane + u * LPR;
                load_entry<TM, PK>(xf, xc, xfc, q, q < b[h], f[h][u], cc[h][u]);
            }
        pdl_wait();
        if (sc->done) return;
        T s[HR];
#pragma unroll
        for (int h = 0; h < HR; h++) {
            s[h] = T(0);
#pragma unroll
            for (int u = 0; u < HB; u++)
                if (cc[h][u] >= 0) s[h] += T(f[h][u]) * x[cc[h][u]];
        }
#pragma unroll
        for (int h = 0; h < HR; h++)
            for (int q = a[h] + lane + HB * LPR; q < b[h]; q += LPR) {
                TM fv;
                int k;
                load_entry<TM, PK>(xf, xc, xfc, q, true, fv, k);
                s[h] += T(fv) * x[k];
            }
#pragma unroll
        for (int h = 0; h < HR; h++) {
#pragma unroll
            for (int o = LPR / 2; o > 0; o >>= 1) s[h] += __shfl_down_sync(0xffffffffu, s[h], o, LPR);
            if (lane == 0 && r[h] < nre) part[r[h]] = rhs[r[h]] - s[h];
        }
        return;
    }
    // window CTA
    TM *stage = reinterpret_cast<TM *>(cell_stage);
    int ka = __ldg(&wfirst[blockIdx.x]), kb = __ldg(&wfirst[blockIdx.x + 1]);
    int o0 = 0, nel = 0, R0 = 0, R1 = 0;
    if (ka < kb) {
        o0 = __ldg(&inv_off[ka]);
        nel = __ldg(&inv_off[kb]) - o0;
        int2 d0 = __ldg(&desc[ka]), d1 = __ldg(&desc[kb - 1]);
        R0 = d0.x;
        R1 = d1.x + d1.y;
    }
    bool staged = nel > 0 && nel <= stage_elems;
    unsigned b = smem_u32(&bar);
    if (threadIdx.x == 0 && staged) mbar_init(b, 1);
    __syncthreads();
    if (threadIdx.x == 0 && staged) {
        unsigned bytes = (unsigned)nel * (unsigned)sizeof(TM);
        mbar_arrive_expect_tx(b, bytes);
        bulk_g2s(smem_u32(stage), inv + o0, bytes, b);
    }
    pdl_wait();
    bool done = sc->done;
    if (!done) {
        // tails of the window's rows: a few entries each (one neighbouring
        // colour), so TL lanes per row and CELL_THREADS / TL rows per pass
        constexpr int TL = 2;
        int lane = threadIdx.x % TL;
        for (int base = R0; base < R1; base += CELL_THREADS / TL) {   // block-uniform trip count
            int r = base + threadIdx.x / TL;
            T s = T(0);
            if (r < R1) {
                int a = FWD ? __ldg(&xs[r]) : __ldg(&xp[r]);
                int e = FWD ? __ldg(&xp[r + 1]) : __ldg(&xs[r]);
                // the first TB entries of each lane in one batch of loads
                constexpr int TB = 4;
                TM tf[TB];
                int tc[TB];
#pragma unroll
                for (int u = 0; u < TB; u++) {
                    int q = a + lane + u * TL;
                    load_entry<TM, PK>(xf, xc, xfc, q, q < e, tf[u], tc[u]);
                }
#pragma unroll
                for (int u = 0; u < TB; u++)
                    if (tc[u] >= 0) s += T(tf[u]) * x[tc[u]];
                for (int q = a + lane + TB * TL; q < e; q += TL) {
                    TM fv;
                    int k;
                    load_entry<TM, PK>(xf, xc, xfc, q, true, fv, k);
                    s += T(fv) * x[k];
                }
            }
            s += __shfl_down_sync(0xffffffffu, s, 1, TL);
            if (lane == 0 && r < R1) part[r] = (first ? rhs[r] : part[r]) - s;
        }
    }
    __syncthreads();
    // on a timeout the copy is still waited for (long bound) before the CTA returns
    if (staged && !stage_wait(b, first_polls, err)) return;
    // a window larger than the stage reads its block inverses from global memory
    if (done) return;
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const TM *src = staged ? stage : inv + o0;
    for (int k = ka + w; k < kb; k += CELL_THREADS / 32) {
        int2 dd = __ldg(&desc[k]);
        int r0 = dd.x, m = dd.y;
        const TM *blk = src + (__ldg(&inv_off[k]) - o0);
        if (m > SWEEP_MAXM) {
            for (int t = 0; t < m; t++) {
                int r = FWD ? r0 + t : r0 + m - 1 - t;
                int po = pk_off[r], l = pk_len[r];
                T ps = T(0);
                for (int e = lane; e < l; e += 32) ps += T(pk_val[po + e]) * x[r0 + pk_k[po + e]];
#pragma unroll
                for (int q = 16; q > 0; q >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, q);
                if (lane == 0) x[r] = (part[r] - ps) * T(dinv[r]);
                __syncwarp();
            }
            continue;
        }
        int i0 = lane, i1 = lane + 32;
        T p0 = i0 < m ? part[r0 + i0] : T(0);
        T p1 = i1 < m ? part[r0 + i1] : T(0);
        T a0 = T(0), a1 = T(0), b0 = T(0), b1 = T(0);
        if (m <= 32) {
#pragma unroll 2
            for (int j = 0; j < m; j += 2) {
                int kk = j + 1;
                T pj = __shfl_sync(0xffffffffu, p0, j);
                T pk = __shfl_sync(0xffffffffu, p0, kk & 31);
                if (FWD) {
                    if (i0 >= j && i0 < m) a0 += T(blk[tri_colofs(j, m) + i0 - j]) * pj;
                    if (kk < m && i0 >= kk && i0 < m) b0 += T(blk[tri_colofs(kk, m) + i0 - kk]) * pk;
                } else {
                    if (i0 <= j) a0 += T(blk[j * (j + 1) / 2 + i0]) * pj;
                    if (kk < m && i0 <= kk) b0 += T(blk[kk * (kk + 1) / 2 + i0]) * pk;
                }
            }
        } else {
            for (int j = 0; j < m; j += 2) {
                int kk = j + 1;
                T pj = __shfl_sync(0xffffffffu, j < 32 ? p0 : p1, j & 31);
                T pk = __shfl_sync(0xffffffffu, kk < 32 ? p0 : p1, kk & 31);
                if (FWD) {
                    const TM *cj = blk + tri_colofs(j, m) - j;
                    if (i0 >= j) a0 += T(cj[i0]) * pj;
                    if (i1 >= j && i1 < m) a1 += T(cj[i1]) * pj;
                    if (kk < m) {
                        const TM *ck = blk + tri_colofs(kk, m) - kk;
                        if (i0 >= kk) b0 += T(ck[i0]) * pk;
                        if (i1 >= kk && i1 < m) b1 += T(ck[i1]) * pk;
                    }
                } else {
                    const TM *rj = blk + j * (j + 1) / 2;
                    if (i0 <= j) a0 += T(rj[i0]) * pj;
                    if (i1 <= j) a1 += T(rj[i1]) * pj;
                    if (kk < m) {
                        const TM *rk = blk + kk * (kk + 1) / 2;
                        if (i0 <= kk) b0 += T(rk[i0]) * pk;
                        if (i1 <= kk) b1 += T(rk[i1]) * pk;
                    }
                }
            }
        }
        a0 += b0;
        a1 += b1;
        if (i0 < m) x[r0 + i0] = a0;
        if (i1 < m) x[r0 + i1] = a1;
    }
}

// ---- warp-per-cell sweep over jagged-diagonal cross runs ----------------------
//
// k_sweep_cell does colour c's whole part of a sweep in one launch, a warp
// per cell: the cross-cell products of the cell's rows from colours swept
// before c, then the in-cell product with the cell's block inverse.
//
// The cross entries of a cell's rows are stored cell by cell in
// jagged-diagonal order (built once per step by k_jds_fill): the rows are
// ranked by their number of cross entries, longest first, and entry k of the
// row of rank q sits at jdp[k] + q, jdp[k] = first slot of the cell's k-th
// diagonal.  A warp reads a diagonal with consecutive lanes on consecutive
// addresses, every row's sum runs in its own entry order in one lane, and no
// padding is stored (diagonal k holds only the rows that have a k-th entry).
// The cell's block inverse is staged in shared memory by one bulk copy per
// warp, issued with the other loads before pdl_wait().

constexpr int JW = 4;                 // warps per cell (a CTA per cell)
constexpr int JSTAGE_M = 40;          // cells of up to this many unknowns stage their block inverse
constexpr int JSTAGE = ((JSTAGE_M * (JSTAGE_M + 1) / 2) + 3) & ~3;
constexpr int JU = 4;                 // diagonals per warp loaded in one batch
constexpr int JMAXL = 512;            // cross entries of one row, at most (the list's max_neighbors bound)

// Diagonals of every active cell's jagged-diagonal block: 1 + the longest
// cross run among its rows (xp: the runs' offsets in row order).
__global__ void k_jds_sizes(int nact, const int2 *__restrict__ desc, const int *__restrict__ xp,
                            int *__restrict__ jlen, unsigned *err)
{
    int kk = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    int lane = threadIdx.x & 31;
    if (kk >= nact) return;   // warp-uniform
    int2 dd = desc[kk];
    int lmax = 0;
    for (int i = lane; i < dd.y; i += 32) lmax = max(lmax, xp[dd.x + i + 1] - xp[dd.x + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
    if (lane == 0) {
        if (lmax > JMAXL || dd.y > 255) atomicOr(err, ERR_CELL_OVERFULL);
        jlen[kk] = min(lmax, JMAXL) + 1;
    }
}

// Jagged-diagonal block of every active cell (a warp per cell, 4 per CTA):
// ranks (longest run first, ties by row), jperm[r0 + rank] = row within the
// cell, jdp[jdc[kk] + k] = slot of diagonal k (k = 0 .. longest; the last is
// the block's end), and the entries: lo (forward) the lower cross run
// [row_ptr, inpos) of each row, up (backward) the upper one [outpos,
// row_ptr + 1).  The block occupies the same slots [xp[r0], xp[r0 + m]) as
// the runs in row order.
template <bool LO>
__global__ void __launch_bounds__(128)
k_jds_fill(int nact, const int2 *__restrict__ desc, const int *__restrict__ xp, const int *__restrict__ jdc,
           const int *__restrict__ row_ptr, const int *__restrict__ inpos, const int *__restrict__ outpos,
           const int *__restrict__ col, const double *__restrict__ F, int *__restrict__ jdp,
           unsigned char *__restrict__ jperm, int *__restrict__ xc, double *__restrict__ xf)
{
    __shared__ int slen[4][256];
    __shared__ int sjd[4][JMAXL + 1];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int kk = blockIdx.x * 4 + w;
    if (kk >= nact) return;   // warp-uniform; no block barrier below
    int2 dd = desc[kk];
    int r0 = dd.x, m = min(dd.y, 255);
    int j0 = jdc[kk], nk = jdc[kk + 1] - j0 - 1;
    int base = xp[r0];
    for (int i = lane; i < m; i += 32) slen[w][i] = min(xp[r0 + i + 1] - xp[r0 + i], JMAXL);
    __syncwarp();
    // diagonal k holds the rows longer than k; its slot is the sum of the
    // earlier diagonals' sizes
    int carry = 0;
    for (int k0 = 0; k0 <= nk; k0 += 32) {
        int k = k0 + lane;
        int cnt = 0;
        if (k < nk)
            for (int i = 0; i < m; i++) cnt += slen[w][i] > k;
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (k <= nk) sjd[w][k] = base + carry + incl - cnt;
        carry += __shfl_sync(0xffffffffu, incl, 31);
    }
    __syncwarp();
    for (int k = lane; k <= nk; k += 32) jdp[j0 + k] = sjd[w][k];
    for (int i = lane; i < m; i += 32) {
        int li = slen[w][i];
        int rank = 0;
        for (int j = 0; j < m; j++) {
            int lj = slen[w][j];
            rank += (lj > li) || (lj == li && j < i);
        }
        jperm[r0 + rank] = (unsigned char)i;
        int r = r0 + i;
        int src = LO ? row_ptr[r] : outpos[r];
        for (int k = 0; k < li; k++) {
            int dst = sjd[w][k] + rank;
            xc[dst] = col[src + k];
            xf[dst] = F[src + k];
        }
    }
}

template <bool FWD, class TM>
__global__ void __launch_bounds__(32 * JW)
k_sweep_cell(int kbeg, int kend, const int2 *__restrict__ desc, const int *__restrict__ inv_off,
             const TM *__restrict__ inv, const int *__restrict__ pk_off, const int *__restrict__ pk_len,
             const TM *__restrict__ pk_val, const unsigned char *__restrict__ pk_k, const TM *__restrict__ dinv,
             const int *__restrict__ jdc, const int *__restrict__ jdp, const unsigned char *__restrict__ jperm,
             const int *__restrict__ xc, const TM *__restrict__ xf, const double *rhs, double *x,
             const CGScalars *sc, int first_polls, int trigger_from, unsigned *err)
{
    using T = double;   // vectors and sums; TM is the storage type of the factor
    __shared__ __align__(128) TM stage[JSTAGE];
    __shared__ T sacc[JW][SWEEP_MAXM];
    __shared__ T spart[SWEEP_MAXM];
    __shared__ int sjd[JMAXL + 1];
    __shared__ __align__(8) unsigned long long bar;
    // CTAs of the grid's last wave let the next launch start at once; the
    // others count as triggered when they exit
    if ((int)blockIdx.x >= trigger_from) pdl_trigger();
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int kk = kbeg + blockIdx.x;   // grid = cells of the colour
    int2 dd = __ldg(&desc[kk]);
    int r0 = dd.x, m = dd.y;
    int io = __ldg(&inv_off[kk]);
    int nb = __ldg(&inv_off[kk + 1]) - io;
    bool staged = m <= JSTAGE_M && nb > 0;
    unsigned b = smem_u32(&bar);
    if (staged && threadIdx.x == 0) {
        mbar_init(b, 1);
        mbar_arrive_expect_tx(b, (unsigned)nb * (unsigned)sizeof(TM));
        bulk_g2s(smem_u32(stage), inv + io, (unsigned)nb * (unsigned)sizeof(TM), b);
    }
    int jb = __ldg(&jdc[kk]);
    int nk = __ldg(&jdc[kk + 1]) - jb - 1;   // diagonals
    for (int k = threadIdx.x; k <= nk; k += 32 * JW) sjd[k] = __ldg(&jdp[jb + k]);
    __syncthreads();
    // warp w takes diagonals w, w + JW, ...; lane q the row of rank q (and
    // q + 32); the first batch is loaded before the dependency wait (factor
    // values and columns are written once per step, before the CG loop)
    TM f[JU][2];
    int c[JU][2];
    auto load = [&](int k0) {
#pragma unroll
        for (int u = 0; u < JU; u++) {
            int k = k0 + u * JW;
            int a = k < nk ? sjd[k] : 0, cnt = k < nk ? sjd[k + 1] - a : 0;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                int q = lane + 32 * h;
                bool ok = q < cnt;
                f[u][h] = ok ? __ldg(&xf[a + q]) : TM(0);
                c[u][h] = ok ? __ldg(&xc[a + q]) : -1;
            }
        }
    };
    load(w);
    pdl_wait();
    if (sc->done) {
        if (staged && threadIdx.x == 0) stage_wait(b, MBAR_DRAIN_POLLS, err);
        return;
    }
    T s0 = T(0), s1 = T(0);
    for (int k0 = w; k0 < nk; k0 += JU * JW) {
        if (k0 != w) load(k0);
#pragma unroll
        for (int u = 0; u < JU; u++) {
            if (c[u][0] >= 0) s0 += T(f[u][0]) * x[c[u][0]];
            if (c[u][1] >= 0) s1 += T(f[u][1]) * x[c[u][1]];
        }
    }
    if (m > SWEEP_MAXM) {
        // only in a blow-up: rank by rank cross sums (thread per rank, in
        // diagonal order) into x, then substitution in place
        for (int q = threadIdx.x; q < m; q += 32 * JW) {
            T v = T(0);
            for (int k = 0; k < nk && q < sjd[k + 1] - sjd[k]; k++) {
                int e = sjd[k] + q;
                v += T(__ldg(&xf[e])) * x[__ldg(&xc[e])];
            }
            int i = __ldg(&jperm[r0 + q]);
            x[r0 + i] = rhs[r0 + i] - v;
        }
        __threadfence_block();
        __syncthreads();
        if (w == 0) {
            for (int t = 0; t < m; t++) {
                int r = FWD ? r0 + t : r0 + m - 1 - t;
                int po = pk_off[r], l = pk_len[r];
                T ps = T(0);
                for (int e = lane; e < l; e += 32) ps += T(pk_val[po + e]) * x[r0 + pk_k[po + e]];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) ps += __shfl_xor_sync(0xffffffffu, ps, o);
                if (lane == 0) x[r] = (x[r] - ps) * T(dinv[r]);
                __threadfence_block();
                __syncwarp();
            }
        }
        return;
    }
    sacc[w][lane] = s0;
    sacc[w][lane + 32] = s1;
    __syncthreads();
    if (threadIdx.x < m) {
        int q = threadIdx.x;
        T t = T(0);
#pragma unroll
        for (int ww = 0; ww < JW; ww++) t += sacc[ww][q];
        int i = __ldg(&jperm[r0 + q]);
        spart[i] = rhs[r0 + i] - t;
    }
    __syncthreads();
    const TM *blk = inv + io;
    if (staged) {
        if (!stage_wait(b, first_polls, err)) return;
        blk = stage;
    }
    // in-cell product, a thread per row
    for (int i = threadIdx.x; i < m; i += 32 * JW) {
        T y = T(0);
        if (FWD) {
            for (int j = 0; j <= i; j++) y += T(blk[tri_colofs(j, m) + i - j]) * spart[j];
        } else {
            for (int j = i; j < m; j++) y += T(blk[j * (j + 1) / 2 + i]) * spart[j];
        }
        x[r0 + i] = y;
    }
}

// ---- CG vector kernels ------------------------------------------------------
//
// The kernels of one CG iteration (SpMV, axpy, the sweeps, r.z, p update) are
// launched as programmatic dependents of one another: each waits for its
// predecessor before it touches a vector or the scalars, so only the launch
// latency overlaps.

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

constexpr int SPMV_U = 8;   // entries per lane loaded in one batch by the FP32 k_cg_spmv

// Ap = A p and the p.Ap partial; the last block forms alpha.  The kernel
// also performs the loop-head test of the reference (sqrt(r.r) < tol, and
// the iteration cap) before any work.
//
// DIFF (the mixed form's FP32 matrix): the product in difference form,
// (A p)_i = dsum_i p_i + sum_j A_ij (p_j - p_i), dsum_i the FP64 row sum of A
// (the diagonal entry contributes nothing to the second sum).  Rounding A_ij
// to FP32 then perturbs the product in proportion to the differences of p
// across a pair, not to |A_ij| |p_j|, whose cancellation in a Laplacian row
// would amplify the rounding by orders of magnitude.
// PK (FP32 only): the entries come from the packed words ac instead of A and
// col, with the same sums in the same order.
template <int LPR, class TM, bool DIFF = false, bool PK = false>
__global__ void __launch_bounds__(CG_BLOCK, 8) k_cg_spmv(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                          const TM *__restrict__ A, const double *p, double *Ap,
                          double *partials, unsigned *ticket, CGScalars *sc,
                          const double *__restrict__ dsum = nullptr, const uint2 *__restrict__ ac = nullptr)
{
    using T = double;   // vectors and sums; TM is the storage type of the matrix
    __shared__ double sh[CG_BLOCK / 32];
    pdl_trigger();
    pdl_wait();
    if (sc->done) return;
    if (sqrt(sc->rr) < sc->tol || sc->iter >= sc->maxit) {
        if (blockIdx.x == 0 && threadIdx.x == 0) sc->done = 1;
        return;
    }
    // a NaN residual (a blown-up state) stays NaN: the reference would run on
    // to cg_max_iter and end with the same NaN solution; stop now instead
    if (isnan(sc->rr)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc->done = 1;
            sc->breakdown = 1;
        }
        return;
    }
    int lane = threadIdx.x % LPR;
    int rows_per_block = CG_BLOCK / LPR;
    double acc = 0.0;
    for (int rb = blockIdx.x * rows_per_block; rb < n_eq; rb += gridDim.x * rows_per_block) {
        int r = rb + threadIdx.x / LPR;
        T s = T(0);
        if (r < n_eq && sizeof(TM) == 8) {
            int q1 = __ldg(&row_ptr[r + 1]);
#pragma unroll 4
            for (int q = __ldg(&row_ptr[r]) + lane; q < q1; q += LPR) s += T(__ldg(&A[q])) * p[__ldg(&col[q])];
        } else if (r < n_eq) {
            // FP32 matrix: a lane's first SPMV_U entries are loaded in one
            // batch (predicated), so a row of up to SPMV_U * LPR nonzeros costs
            // one round trip for A and col and one for the gathers (an FP32
            // entry moves two thirds of an FP64 one per trip); the sum runs in
            // entry order, in FP64
            int q0 = __ldg(&row_ptr[r]) + lane, q1 = __ldg(&row_ptr[r + 1]);
            TM a[SPMV_U];
            int c[SPMV_U];
#pragma unroll
            for (int u = 0; u < SPMV_U; u++) {
                int q = q0 + u * LPR;
                a[u] = TM(0);
                c[u] = -1;
                if (q < q1) load_entry<TM, PK>(A, col, ac, q, true, a[u], c[u]);
            }
            T pi = DIFF ? p[r] : T(0);
#pragma unroll
            for (int u = 0; u < SPMV_U; u++)
                if (c[u] >= 0) s += T(a[u]) * (DIFF ? p[c[u]] - pi : p[c[u]]);
            for (int q = q0 + SPMV_U * LPR; q < q1; q += LPR) {
                TM av;
                int k;
                load_entry<TM, PK>(A, col, ac, q, true, av, k);
                s += T(av) * (DIFF ? p[k] - pi : p[k]);
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && r < n_eq) {
            double pr = p[r];
            if (DIFF) s += __ldg(&dsum[r]) * pr;
            Ap[r] = s;
            acc += pr * s;
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
__global__ void k_cg_axpy(int n_eq, T *x, T *r, const T *p, const T *Ap, double *partials, unsigned *ticket,
                          CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    pdl_trigger();
    pdl_wait();
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
__global__ void k_cg_rz(int n_eq, const T *r, const T *z, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    pdl_trigger();
    pdl_wait();
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
__global__ void k_cg_update_p(int n_eq, T *p, const T *z, CGScalars *sc)
{
    pdl_trigger();
    pdl_wait();
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

// dsum_i = sum_j A_ij in FP64, in entry order (the difference-form SpMV).
__global__ void k_row_sum(int n_eq, const int *__restrict__ row_ptr, const double *__restrict__ A,
                          double *__restrict__ dsum)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    double s = 0.0;
    for (int q = row_ptr[r]; q < row_ptr[r + 1]; q++) s += A[q];
    dsum[r] = s;
}

// x = 0, r = b, ||b||^2 into sc->rr_outer.
__global__ void k_refine_init(int n_eq, double *__restrict__ x, double *__restrict__ r,
                              const double *__restrict__ b, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        double bi = b[i];
        x[i] = 0.0;
        r[i] = bi;
        acc += bi * bi;
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) sc->rr_outer = tot;
    }
}

// Reliable update of the CG on the FP32 matrix (mixed form): r now holds
// the true residual b - A x with the FP64 matrix and z its preconditioned
// value; the search direction keeps its history, p = z + beta p_prev with
// the new z, i.e. p += z - zprev.  New r.z and r.r; the loop resumes with
// `tol`.
template <class T>
__global__ void k_reliable_fix(int n_eq, const T *__restrict__ r, const T *__restrict__ z,
                               const T *__restrict__ zprev, T *__restrict__ p, double tol, double *partials,
                               unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double a = 0.0, b2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        T ri = r[i], zi = z[i];
        p[i] = p[i] + (zi - zprev[i]);
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
            sc->tol = tol;
            sc->done = 0;
            sc->breakdown = 0;
        }
    }
}

// The true residual r = b - A x with the FP64 matrix, ||r||^2 into
// sc->rr_outer and || |b| + |A| |x| ||^2 into sc->ff (8 lanes per row).
__global__ void k_refine_residual(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                                  const double *__restrict__ A, const double *__restrict__ x,
                                  const double *__restrict__ b, double *__restrict__ r,
                                  double *partials, unsigned *ticket, CGScalars *sc)
{
    constexpr int LPR = 8;
    __shared__ double sh[CG_BLOCK / 32];
    int lane = threadIdx.x % LPR;
    int rows_per_block = CG_BLOCK / LPR;
    double acc = 0.0, accf = 0.0;
    for (int rb = blockIdx.x * rows_per_block; rb < n_eq; rb += gridDim.x * rows_per_block) {
        int i = rb + threadIdx.x / LPR;
        double s = 0.0, sa = 0.0;
        if (i < n_eq) {
            int q1 = __ldg(&row_ptr[i + 1]);
            for (int q = __ldg(&row_ptr[i]) + lane; q < q1; q += LPR) {
                double t = __ldg(&A[q]) * x[__ldg(&col[q])];
                s += t;
                sa += fabs(t);
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o, LPR);
            sa += __shfl_down_sync(0xffffffffu, sa, o, LPR);
        }
        if (lane == 0 && i < n_eq) {
            double bi = b[i];
            double ri = bi - s;
            double fi = fabs(bi) + sa;
            r[i] = ri;
            acc += ri * ri;
            accf += fi * fi;
        }
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    double tf = block_sum<CG_BLOCK>(accf, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = t;
        partials[2 * blockIdx.x + 1] = tf;
    }
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 2, 0, sh);
        double totf = final_sum(partials, gridDim.x, 2, 1, sh);
        if (threadIdx.x == 0) {
            sc->rr_outer = tot;
            sc->ff = totf;
        }
    }
}

// ||b - A x||^2, ||b||^2 and || |b| + |A| |x| ||^2 with the FP64 matrix (8
// lanes per row), into sc->rr_outer, sc->bb and sc->ff: the true residual of
// a finished solve, which the recursive residual of the CG loop only tracks
// until rounding takes over, and the scale of the rounding error of b - A x
// in FP64 (unit roundoff times the last norm).
__global__ void k_true_residual(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                                const double *__restrict__ A, const double *__restrict__ x,
                                const double *__restrict__ b, double *partials, unsigned *ticket, CGScalars *sc)
{
    constexpr int LPR = 8;
    __shared__ double sh[CG_BLOCK / 32];
    int lane = threadIdx.x % LPR;
    int rows_per_block = CG_BLOCK / LPR;
    double acc = 0.0, accb = 0.0, accf = 0.0;
    for (int rb = blockIdx.x * rows_per_block; rb < n_eq; rb += gridDim.x * rows_per_block) {
        int i = rb + threadIdx.x / LPR;
        double s = 0.0, sa = 0.0;
        if (i < n_eq) {
            int q1 = __ldg(&row_ptr[i + 1]);
            for (int q = __ldg(&row_ptr[i]) + lane; q < q1; q += LPR) {
                double t = __ldg(&A[q]) * x[__ldg(&col[q])];
                s += t;
                sa += fabs(t);
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) {
            s += __shfl_down_sync(0xffffffffu, s, o, LPR);
            sa += __shfl_down_sync(0xffffffffu, sa, o, LPR);
        }
        if (lane == 0 && i < n_eq) {
            double bi = b[i];
            double ri = bi - s;
            double fi = fabs(bi) + sa;
            acc += ri * ri;
            accb += bi * bi;
            accf += fi * fi;
        }
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    double tb = block_sum<CG_BLOCK>(accb, sh);
    double tf = block_sum<CG_BLOCK>(accf, sh);
    if (threadIdx.x == 0) {
        partials[3 * blockIdx.x] = t;
        partials[3 * blockIdx.x + 1] = tb;
        partials[3 * blockIdx.x + 2] = tf;
    }
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 3, 0, sh);
        double totb = final_sum(partials, gridDim.x, 3, 1, sh);
        double totf = final_sum(partials, gridDim.x, 3, 2, sh);
        if (threadIdx.x == 0) {
            sc->rr_outer = tot;
            sc->bb = totb;
            sc->ff = totf;
        }
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
