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

// One warp per cell of the colour; the cell's rows in order.
__global__ void k_ic0_color(int kbeg, int kend, const int *__restrict__ ccells, const int *__restrict__ cell_row0,
                            const int *__restrict__ ucount, const int *__restrict__ row_ptr,
                            const int *__restrict__ diagpos, const int *__restrict__ col,
                            const double *__restrict__ A, double *F)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int kk = kbeg + warp;
    if (kk >= kend) return;
    int c = ccells[kk];
    int r0 = cell_row0[c], m = ucount[c];
    for (int r = r0; r < r0 + m; r++) {
        int p0 = row_ptr[r], pd = diagpos[r];
        for (int p = p0; p < pd; p++) {
            int kc = col[p];
            int k0 = row_ptr[kc], kd = diagpos[kc];
            double part = 0.0;
            for (int q = p0 + lane; q < p; q += 32) {
                int pos = find_col(col, k0, kd, col[q]);
                if (pos >= 0) part += F[q] * F[pos];
            }
            double s = A[p] - warp_allsum(part);
            double lik = s * F[kd];
            if (lane == 0) {
                F[p] = lik;
                int up = find_col(col, kd + 1, row_ptr[kc + 1], r);
                if (up >= 0) F[up] = lik;
            }
            __syncwarp();
        }
        double part = 0.0;
        for (int q = p0 + lane; q < pd; q += 32) part += F[q] * F[q];
        double a = A[pd];
        double d = a - warp_allsum(part);
        if (d <= 0.0) d = (a > 0.0) ? a : 1.0e-30;
        if (lane == 0) F[pd] = 1.0 / sqrt(d);
        __syncwarp();
    }
}

// ---- preconditioner sweeps ------------------------------------------------

// Forward L y = r on the cells of one colour.
__global__ void k_fwd_color(int kbeg, int kend, const int *__restrict__ ccells, const int *__restrict__ cell_row0,
                            const int *__restrict__ ucount, const int *__restrict__ row_ptr,
                            const int *__restrict__ diagpos, const int *__restrict__ col,
                            const double *__restrict__ F, const double *__restrict__ rhs, double *y,
                            const CGScalars *sc)
{
    if (sc->done) return;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int kk = kbeg + warp;
    if (kk >= kend) return;
    int c = ccells[kk];
    int r0 = cell_row0[c], m = ucount[c];
    for (int r = r0; r < r0 + m; r++) {
        int p0 = row_ptr[r], pd = diagpos[r];
        double part = 0.0;
        for (int q = p0 + lane; q < pd; q += 32) part += F[q] * y[col[q]];
        double s = warp_allsum(part);
        if (lane == 0) y[r] = (rhs[r] - s) * F[pd];
        __syncwarp();
    }
}

// Backward L^T z = y on the cells of one colour (colours in reverse).
__global__ void k_bwd_color(int kbeg, int kend, const int *__restrict__ ccells, const int *__restrict__ cell_row0,
                            const int *__restrict__ ucount, const int *__restrict__ row_ptr,
                            const int *__restrict__ diagpos, const int *__restrict__ col,
                            const double *__restrict__ F, const double *__restrict__ y, double *z,
                            const CGScalars *sc)
{
    if (sc->done) return;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int kk = kbeg + warp;
    if (kk >= kend) return;
    int c = ccells[kk];
    int r0 = cell_row0[c], m = ucount[c];
    for (int r = r0 + m - 1; r >= r0; r--) {
        int pd = diagpos[r], p1 = row_ptr[r + 1];
        double part = 0.0;
        for (int q = pd + 1 + lane; q < p1; q += 32) part += F[q] * z[col[q]];
        double s = warp_allsum(part);
        if (lane == 0) z[r] = (y[r] - s) * F[pd];
        __syncwarp();
    }
}

// ---- CG vector kernels ------------------------------------------------------

constexpr int CG_BLOCK = 256;

// Ap = A p and the p.Ap partial; the last block forms alpha.  The kernel
// also performs the loop-head test of the reference (sqrt(r.r) < tol, and
// the iteration cap) before any work.
template <int LPR>
__global__ void k_cg_spmv(int n_eq, const int *__restrict__ row_ptr, const int *__restrict__ col,
                          const double *__restrict__ A, const double *__restrict__ p, double *__restrict__ Ap,
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
        double s = 0.0;
        if (r < n_eq) {
            for (int q = row_ptr[r] + lane; q < row_ptr[r + 1]; q += LPR) s += A[q] * p[col[q]];
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && r < n_eq) {
            Ap[r] = s;
            acc += p[r] * s;
        }
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block_done(ticket, gridDim.x)) {
        double tot = 0.0;
        for (unsigned b = 0; b < gridDim.x; b++) tot += __ldcg(&partials[b]);
        sc->pAp = tot;
        if (fabs(tot) < 1.0e-30) { sc->done = 1; sc->breakdown = 1; }
        else sc->alpha = sc->rz / tot;
    }
}

// x += alpha p, r -= alpha Ap, and r.r.
__global__ void k_cg_axpy(int n_eq, double *__restrict__ x, double *__restrict__ r, const double *__restrict__ p,
                          const double *__restrict__ Ap, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    if (sc->done) return;
    double alpha = sc->alpha;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        x[i] += alpha * p[i];
        double ri = r[i] - alpha * Ap[i];
        r[i] = ri;
        acc += ri * ri;
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block_done(ticket, gridDim.x)) {
        double tot = 0.0;
        for (unsigned b = 0; b < gridDim.x; b++) tot += __ldcg(&partials[b]);
        sc->rr = tot;
    }
}

// rz_new = r.z, the breakdown test on the previous rz, beta.
__global__ void k_cg_rz(int n_eq, const double *__restrict__ r, const double *__restrict__ z,
                        double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    if (sc->done) return;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x)
        acc += r[i] * z[i];
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block_done(ticket, gridDim.x)) {
        double tot = 0.0;
        for (unsigned b = 0; b < gridDim.x; b++) tot += __ldcg(&partials[b]);
        sc->rz_new = tot;
        if (fabs(sc->rz) < 1.0e-60) { sc->done = 1; sc->breakdown = 1; }
        else { sc->beta = tot / sc->rz; sc->rz = tot; }
    }
}

__global__ void k_cg_update_p(int n_eq, double *__restrict__ p, const double *__restrict__ z, CGScalars *sc)
{
    if (sc->done) return;
    double beta = sc->beta;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->iter += 1;
}

// x = 0, r = b.
__global__ void k_cg_init(int n_eq, double *__restrict__ x, double *__restrict__ r, const double *__restrict__ b)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        x[i] = 0.0;
        r[i] = b[i];
    }
}

// p = z, rz = r.z, rr = r.r.
__global__ void k_cg_init2(int n_eq, const double *__restrict__ r, const double *__restrict__ z,
                           double *__restrict__ p, double *partials, unsigned *ticket, CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double a = 0.0, b2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_eq; i += gridDim.x * blockDim.x) {
        double ri = r[i], zi = z[i];
        p[i] = zi;
        a += ri * zi;
        b2 += ri * ri;
    }
    double ta = block_sum<CG_BLOCK>(a, sh);
    double tb = block_sum<CG_BLOCK>(b2, sh);
    if (threadIdx.x == 0) {
        partials[2 * blockIdx.x] = ta;
        partials[2 * blockIdx.x + 1] = tb;
    }
    if (last_block_done(ticket, gridDim.x)) {
        double sa = 0.0, sb = 0.0;
        for (unsigned k = 0; k < gridDim.x; k++) {
            sa += __ldcg(&partials[2 * k]);
            sb += __ldcg(&partials[2 * k + 1]);
        }
        sc->rz = sa;
        sc->rr = sb;
        sc->iter = 0;
        sc->done = 0;
        sc->breakdown = 0;
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
