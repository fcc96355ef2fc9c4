// k_pcg.cuh -- the ICCG loop of the PPE solve as one persistent kernel.
//
// The PCG of pressure_solver.c:261-322 on the block-colour system, a batch
// of iterations per cooperative launch.  Every CTA stays resident for the
// whole batch and the phases of an iteration are separated by grid
// barriers instead of kernel boundaries:
//
//   SpMV      Ap = A p, p.Ap; p = z + beta p of the previous iteration is
//             applied on the fly (p double-buffered)           | barrier, alpha
//   F_c       for each colour but the last, in sweep order: its rows'
//             x += alpha p, r -= alpha Ap, r.r; the cross-cell products
//             from earlier colours and the in-cell product with the
//             block inverse (y = forward sweep)                 | barrier
//   F_L + B_L the last colour: as F_c, then at once its backward in-cell
//             product (no later colour feeds it)                | barrier, r.r
//   B_c       for each colour but the last, in reverse: the cross-cell
//             products from later colours and the in-cell product with
//             the transposed block inverse (z), r.z             | barrier, beta
//
// so an iteration is 2^D + 1 phases, not the 2^(D+1) + 4 kernels of the
// launch-per-colour form.  A warp takes one cell at a time (the cells of a
// colour are spread over all warps of the grid); its cross entries are
// stored cell by cell in jagged-diagonal order (k_jds_fill), so the warp
// reads a diagonal with consecutive lanes on consecutive addresses and
// each row's sum runs in its own entry order in one lane.  The test of the
// reference's loop head (sqrt(r.r) < tol, or the iteration cap) runs at
// the top of each iteration with the previous iteration's r.r, as the
// launch-per-colour form runs it.
//
// Every grid sum adds warp, CTA and grid partials in a fixed order, so
// every CTA holds the same scalars and a rerun gives the same bits.  The
// barrier waits are bounded: on expiry a CTA sets ERR_GRID_TIMEOUT and
// returns, and so in turn does every other CTA at its next barrier.
#pragma once

#include "k_ppe.cuh"

namespace mps {

constexpr int PCG_THREADS = 512;
constexpr int PCG_WARPS = PCG_THREADS / 32;
constexpr int PCG_BAR_POLLS = 1 << 22;   // polls of one grid-barrier wait, at most (about a second)
constexpr int PCG_SLOTS = 4;             // rotating slots of the grid partial sums
constexpr int PCG_MAXM = 256;            // row buffer of a warp: a cell's unknowns (ERR_CELL_OVERFULL above 255)
constexpr int PCG_DIAG_BATCH = 8;        // jagged diagonals loaded per batch

template <class TM>
struct PcgArgs {
    int n_eq;
    int ncol;                  // non-empty colours, in forward sweep order
    int kb[8], ke[8];          // their active-cell ranges
    const int *row_ptr, *colidx;
    const TM *A;
    const double *dsum;        // the SpMV in difference form when non-null (FP32 matrix)
    const int2 *desc;          // (first row, unknowns) of each active cell
    const int *inv_off;
    const TM *inv_cm, *inv_rm; // in-cell block inverses, column- and row-major
    const int *jdc_lo, *jdp_lo, *jdc_up, *jdp_up;
    const unsigned char *jperm_lo, *jperm_up;
    const int *xc_lo, *xc_up;
    const TM *xf_lo, *xf_up;
    const int *pk_off_lo, *pk_len_lo, *pk_off_up, *pk_len_up;   // packed in-cell runs (cells > SWEEP_MAXM)
    const TM *pkv_lo, *pkv_up;
    const unsigned char *pkk_lo, *pkk_up;
    const TM *dinv;
    double *x, *r, *y, *z, *Ap;
    double *p, *p2;            // search direction and its second buffer
    CGScalars *sc;
    double *partials;          // PCG_SLOTS x gridDim.x
    unsigned *bar;             // barrier counter, zero at launch
    unsigned *err;
    int batch;                 // iterations in this launch, at most
    int apply;                 // 1: only z = M^-1 r (both sweeps), no CG update
    int bar_polls;             // polls of one grid-barrier wait, at most
    // profiling: CTA 0 writes the global timer at its start (trace[0]) and as
    // it leaves barrier k (trace[k], k <= PCG_TRACE), and the number of
    // barriers passed at trace[PCG_TRACE + 1]; null when off
    unsigned long long *trace;
};

constexpr int PCG_TRACE = 4096;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Barrier of all CTAs of the cooperative launch: the counter reaches
// `target` once every CTA has arrived.  Writes made before it by any CTA
// are visible after it in every CTA.  Bounded: false (and ERR_GRID_TIMEOUT)
// after `polls` polls.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, int polls, unsigned *err, int *s_ok)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        int ok = 1;
        for (int i = 0; ld_acquire_gpu(bar) < target; i++) {
            if (i >= polls) {
                ok = 0;
                atomicOr(err, ERR_GRID_TIMEOUT);
                break;
            }
            __nanosleep(32);
        }
        __threadfence();
        *s_ok = ok;
    }
    __syncthreads();
    return *s_ok != 0;
}

// Grid sum of one value per thread with a barrier: warp tree, the block's
// warps in order, the CTAs' partials in order (slot `slot` of partials), so
// that every thread of every CTA gets the same bits.
__device__ __forceinline__ bool grid_sum(double v, double *partials, int slot, unsigned *bar, unsigned target,
                                         int polls, unsigned *err, double *sh, int *s_ok, double *out)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int k = 0; k < PCG_WARPS; k++) t += sh[k];
        __stcg(&partials[(size_t)slot * gridDim.x + blockIdx.x], t);
    }
    if (!grid_barrier(bar, target, polls, err, s_ok)) return false;
    if (w == 0) {
        double a = 0.0;
        for (unsigned b = lane; b < gridDim.x; b += 32) a += __ldcg(&partials[(size_t)slot * gridDim.x + b]);
        a = warp_sum(a);
        if (lane == 0) sh[PCG_WARPS] = a;
    }
    __syncthreads();
    *out = sh[PCG_WARPS];
    return true;
}

// ---- SpMV phase --------------------------------------------------------------

// Ap = A p over a grid-stride of row groups, LPR lanes per row; returns the
// thread's part of p.Ap.  With `pend`, p = z + beta pold is formed on the
// fly (the same expression for the row's own entry and every gathered one)
// and written to pnew by the row's owner.
template <int LPR, class TM, bool DIFF>
__device__ __forceinline__ double pcg_spmv(const PcgArgs<TM> &a, bool pend, double beta, const double *pold,
                                           double *pnew)
{
    constexpr int RPB = PCG_THREADS / LPR;
    int lane = threadIdx.x % LPR;
    const double *z = a.z;
    double acc = 0.0;
    for (int rb = blockIdx.x * RPB; rb < a.n_eq; rb += gridDim.x * RPB) {
        int r = rb + threadIdx.x / LPR;
        double s = 0.0, pr = 0.0;
        if (r < a.n_eq) {
            pr = pend ? z[r] + beta * pold[r] : pold[r];
            int q0 = __ldg(&a.row_ptr[r]), q1 = __ldg(&a.row_ptr[r + 1]);
            if (sizeof(TM) == 8) {
#pragma unroll 4
                for (int q = q0 + lane; q < q1; q += LPR) {
                    int c = __ldg(&a.colidx[q]);
                    double pc = pend ? z[c] + beta * pold[c] : pold[c];
                    s += double(__ldg(&a.A[q])) * (DIFF ? pc - pr : pc);
                }
            } else {
                TM av[SPMV_U];
                int cv[SPMV_U];
#pragma unroll
                for (int u = 0; u < SPMV_U; u++) {
                    int q = q0 + lane + u * LPR;
                    bool ok = q < q1;
                    av[u] = ok ? __ldg(&a.A[q]) : TM(0);
                    cv[u] = ok ? __ldg(&a.colidx[q]) : -1;
                }
#pragma unroll
                for (int u = 0; u < SPMV_U; u++)
                    if (cv[u] >= 0) {
                        double pc = pend ? z[cv[u]] + beta * pold[cv[u]] : pold[cv[u]];
                        s += double(av[u]) * (DIFF ? pc - pr : pc);
                    }
                for (int q = q0 + lane + SPMV_U * LPR; q < q1; q += LPR) {
                    int c = __ldg(&a.colidx[q]);
                    double pc = pend ? z[c] + beta * pold[c] : pold[c];
                    s += double(__ldg(&a.A[q])) * (DIFF ? pc - pr : pc);
                }
            }
        }
#pragma unroll
        for (int o = LPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, LPR);
        if (lane == 0 && r < a.n_eq) {
            if (DIFF) s += __ldg(&a.dsum[r]) * pr;
            a.Ap[r] = s;
            acc += pr * s;
            if (pend) pnew[r] = pr;
        }
    }
    return acc;
}

// ---- one cell of a sweep ---------------------------------------------------------

enum : int {
    CELL_CG = 1,      // forward: x += alpha p, r -= alpha Ap on the cell's rows first, r.r
    CELL_FUSED = 2,   // forward of the last colour: continue with its backward in-cell product
    CELL_RZ = 4,      // accumulate r.z over the z rows written
};

// Dense in-cell product of a warp: v_i = sum_j B_ij s_j for the cell's rows
// i = lane, lane + 32, with B = L_cc^-1 (FWD, column-major block: entries
// i >= j of column j at colofs(j) + i - j) or L_cc^-T (row-major block of
// L_cc^-1: entries i <= j of row j at j(j+1)/2 + i); s in shared memory.
template <bool FWD, class TM>
__device__ __forceinline__ void incell_product(const TM *__restrict__ blk, const double *sp, int m, int lane,
                                               double &v0, double &v1)
{
    int i0 = lane, i1 = lane + 32;
    v0 = 0.0;
    v1 = 0.0;
    constexpr int U = 4;
    for (int j0 = 0; j0 < m; j0 += U) {
        TM e0[U], e1[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            int j = j0 + u;
            bool ok0, ok1;
            int o0, o1;
            if (FWD) {
                ok0 = j < m && i0 >= j && i0 < m;
                ok1 = j < m && i1 >= j && i1 < m;
                o0 = tri_colofs(j, m) + i0 - j;
                o1 = tri_colofs(j, m) + i1 - j;
            } else {
                ok0 = j < m && i0 <= j;
                ok1 = j < m && i1 <= j;
                o0 = j * (j + 1) / 2 + i0;
                o1 = j * (j + 1) / 2 + i1;
            }
            e0[u] = ok0 ? __ldg(&blk[o0]) : TM(0);
            e1[u] = ok1 ? __ldg(&blk[o1]) : TM(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            int j = j0 + u;
            if (j < m) {
                double sj = sp[j];
                v0 += double(e0[u]) * sj;
                v1 += double(e1[u]) * sj;
            }
        }
    }
}

// In-place substitution on sp (cells above SWEEP_MAXM unknowns, only in a
// blow-up): forward over the packed lower in-cell runs, or backward over
// the upper ones, a warp reduction per row.
template <bool FWD, class TM>
__device__ void incell_substitute(const PcgArgs<TM> &a, int r0, int m, double *sp)
{
    int lane = threadIdx.x & 31;
    const int *po = FWD ? a.pk_off_lo : a.pk_off_up, *pl = FWD ? a.pk_len_lo : a.pk_len_up;
    const TM *pv = FWD ? a.pkv_lo : a.pkv_up;
    const unsigned char *pk = FWD ? a.pkk_lo : a.pkk_up;
    for (int t = 0; t < m; t++) {
        int i = FWD ? t : m - 1 - t;
        int r = r0 + i;
        int o = __ldg(&po[r]), l = __ldg(&pl[r]);
        double ps = 0.0;
        for (int e = lane; e < l; e += 32) ps += double(__ldg(&pv[o + e])) * sp[__ldg(&pk[o + e])];
        ps = warp_sum(ps);
        if (lane == 0) sp[i] = (sp[i] - ps) * double(__ldg(&a.dinv[r]));
        __syncwarp();
    }
}

// The cell's part of a sweep, one warp: right-hand sides (r, updated first
// with CELL_CG, or y), minus the cross-cell products by rank, then the
// in-cell product; writes y (FWD) or z.  sp: the warp's shared row buffer.
template <bool FWD, class TM>
__device__ void pcg_cell(const PcgArgs<TM> &a, const double *p, int kk, int mode, double alpha, double *sp,
                         double &arr, double &arz)
{
    int lane = threadIdx.x & 31;
    int2 dd = __ldg(&a.desc[kk]);
    int r0 = dd.x, m = min(dd.y, 255);   // larger cells have set ERR_CELL_OVERFULL (k_jds_sizes)
    for (int i = lane; i < m; i += 32) {
        int row = r0 + i;
        double v;
        if (FWD) {
            v = a.r[row];
            if (mode & CELL_CG) {
                a.x[row] += alpha * p[row];
                v = v - alpha * a.Ap[row];
                a.r[row] = v;
                arr += v * v;
            }
        } else {
            v = a.y[row];
        }
        sp[i] = v;
    }
    // cross-cell products, rank q = lane + 32 h; diagonal k of the cell's
    // block holds the ranks below its length at jdp[k] + rank
    const int *jdc = FWD ? a.jdc_lo : a.jdc_up, *jdp = FWD ? a.jdp_lo : a.jdp_up;
    const unsigned char *jperm = FWD ? a.jperm_lo : a.jperm_up;
    const int *xc = FWD ? a.xc_lo : a.xc_up;
    const TM *xf = FWD ? a.xf_lo : a.xf_up;
    const double *xv = FWD ? a.y : a.z;
    int jb = __ldg(&jdc[kk]);
    int nk = __ldg(&jdc[kk + 1]) - jb - 1;
    __syncwarp();
    for (int h = 0; h * 32 < m; h++) {
        int q = lane + 32 * h;
        double s = 0.0;
        for (int k0 = 0; k0 < nk; k0 += 32) {
            int kn = min(32, nk - k0);
            int st = lane < kn ? __ldg(&jdp[jb + k0 + lane]) : 0;
            int en = lane < kn ? __ldg(&jdp[jb + k0 + lane + 1]) : 0;
            for (int u0 = 0; u0 < kn; u0 += PCG_DIAG_BATCH) {
                TM f[PCG_DIAG_BATCH];
                int c[PCG_DIAG_BATCH];
#pragma unroll
                for (int u = 0; u < PCG_DIAG_BATCH; u++) {
                    int k = u0 + u;
                    int s0 = __shfl_sync(0xffffffffu, st, k & 31);
                    int e0 = __shfl_sync(0xffffffffu, en, k & 31);
                    bool ok = k < kn && s0 + q < e0;
                    f[u] = ok ? __ldg(&xf[s0 + q]) : TM(0);
                    c[u] = ok ? __ldg(&xc[s0 + q]) : -1;
                }
#pragma unroll
                for (int u = 0; u < PCG_DIAG_BATCH; u++)
                    if (c[u] >= 0) s += double(f[u]) * xv[c[u]];
            }
        }
        if (q < m) {
            int i = __ldg(&jperm[r0 + q]);
            sp[i] -= s;
        }
    }
    __syncwarp();
    // in-cell product
    if (m > SWEEP_MAXM) {
        incell_substitute<FWD>(a, r0, m, sp);
        for (int i = lane; i < m; i += 32) {
            if (FWD) a.y[r0 + i] = sp[i];
            else {
                a.z[r0 + i] = sp[i];
                if (mode & CELL_RZ) arz += a.r[r0 + i] * sp[i];
            }
        }
        if (FWD && (mode & CELL_FUSED)) {
            __syncwarp();
            incell_substitute<false>(a, r0, m, sp);
            for (int i = lane; i < m; i += 32) {
                a.z[r0 + i] = sp[i];
                if (mode & CELL_RZ) arz += a.r[r0 + i] * sp[i];
            }
        }
        __syncwarp();
        return;
    }
    int io = __ldg(&a.inv_off[kk]);
    double v0, v1;
    incell_product<FWD>((FWD ? a.inv_cm : a.inv_rm) + io, sp, m, lane, v0, v1);
    int i0 = lane, i1 = lane + 32;
    if (FWD) {
        if (i0 < m) a.y[r0 + i0] = v0;
        if (i1 < m) a.y[r0 + i1] = v1;
        if (mode & CELL_FUSED) {
            // backward in-cell product of the last colour: t = y (no later colour)
            __syncwarp();
            if (i0 < m) sp[i0] = v0;
            if (i1 < m) sp[i1] = v1;
            __syncwarp();
            incell_product<false>(a.inv_rm + io, sp, m, lane, v0, v1);
        }
    }
    if (!FWD || (mode & CELL_FUSED)) {
        if (i0 < m) {
            a.z[r0 + i0] = v0;
            if (mode & CELL_RZ) arz += a.r[r0 + i0] * v0;
        }
        if (i1 < m) {
            a.z[r0 + i1] = v1;
            if (mode & CELL_RZ) arz += a.r[r0 + i1] * v1;
        }
    }
    __syncwarp();
}

// ---- the kernel ---------------------------------------------------------------------

template <class TM, bool DIFF>
__global__ void __launch_bounds__(PCG_THREADS, 2) k_pcg(PcgArgs<TM> a)
{
    __shared__ double s_sp[PCG_WARPS][PCG_MAXM];
    __shared__ double s_red[PCG_WARPS + 1];
    __shared__ int s_ok;
    const int w = threadIdx.x >> 5;
    const int gw = blockIdx.x * PCG_WARPS + w, nw = gridDim.x * PCG_WARPS;
    double *sp = s_sp[w];
    const unsigned G = gridDim.x;
    unsigned nbar = 0;
    int nsum = 0;
    const bool tr = a.trace && blockIdx.x == 0 && threadIdx.x == 0;
    if (tr) a.trace[0] = global_ns();
    auto mark = [&]() {
        if (tr && nbar <= PCG_TRACE) a.trace[nbar] = global_ns();
    };
    auto barrier = [&]() {
        bool ok = grid_barrier(a.bar, ++nbar * G, a.bar_polls, a.err, &s_ok);
        mark();
        return ok;
    };
    auto gsum = [&](double v, double *out) {
        bool ok = grid_sum(v, a.partials, (nsum++) % PCG_SLOTS, a.bar, ++nbar * G, a.bar_polls, a.err, s_red,
                           &s_ok, out);
        mark();
        return ok;
    };
    const int nc = a.ncol;
    double arr = 0.0, arz = 0.0;

    if (a.apply) {
        for (int ci = 0; ci < nc; ci++) {
            int mode = ci == nc - 1 ? CELL_FUSED : 0;
            for (int kk = a.kb[ci] + gw; kk < a.ke[ci]; kk += nw) pcg_cell<true>(a, a.p, kk, mode, 0.0, sp, arr, arz);
            if (!barrier()) return;
        }
        for (int ci = nc - 2; ci >= 0; ci--) {
            for (int kk = a.kb[ci] + gw; kk < a.ke[ci]; kk += nw) pcg_cell<false>(a, a.p, kk, 0, 0.0, sp, arr, arz);
            if (ci > 0 && !barrier()) return;
        }
        return;
    }

    CGScalars *sc = a.sc;
    double rz = __ldcg(&sc->rz), rr = __ldcg(&sc->rr), tol = __ldcg(&sc->tol);
    double alpha = __ldcg(&sc->alpha), beta = __ldcg(&sc->beta), pAp = __ldcg(&sc->pAp);
    double rz_new = __ldcg(&sc->rz_new);
    int iter = __ldcg(&sc->iter), maxit = __ldcg(&sc->maxit), done = __ldcg(&sc->done);
    int brk = __ldcg(&sc->breakdown);
    bool pend = false;   // p = z + beta p not yet applied
    int pb = 0;          // p lives in a.p (0) or a.p2 (1)
    for (int it = 0; it < a.batch && !done; it++) {
        if (sqrt(rr) < tol || iter >= maxit || isnan(rr)) {   // NaN: see k_cg_spmv
            done = 1;
            if (isnan(rr)) brk = 1;
            break;
        }
        double *pold = pb ? a.p2 : a.p, *pnew = pb ? a.p : a.p2;
        double part;
        if (sizeof(TM) == 8) part = pcg_spmv<8, TM, DIFF>(a, pend, beta, pold, pnew);
        else part = pcg_spmv<16, TM, DIFF>(a, pend, beta, pold, pnew);
        if (pend) pb ^= 1;
        pend = false;
        double tot;
        if (!gsum(part, &tot)) return;
        pAp = tot;
        if (fabs(tot) < 1.0e-30) {
            done = 1;
            brk = 1;
            break;
        }
        alpha = rz / tot;
        const double *pc = pb ? a.p2 : a.p;
        arr = 0.0;
        arz = 0.0;
        for (int ci = 0; ci < nc; ci++) {
            int mode = CELL_CG | (ci == nc - 1 ? CELL_FUSED | CELL_RZ : 0);
            for (int kk = a.kb[ci] + gw; kk < a.ke[ci]; kk += nw) pcg_cell<true>(a, pc, kk, mode, alpha, sp, arr, arz);
            if (ci < nc - 1 && !barrier()) return;
        }
        if (!gsum(arr, &rr)) return;
        for (int ci = nc - 2; ci >= 0; ci--) {
            for (int kk = a.kb[ci] + gw; kk < a.ke[ci]; kk += nw) pcg_cell<false>(a, pc, kk, CELL_RZ, 0.0, sp, arr, arz);
            if (ci > 0 && !barrier()) return;
        }
        double rzn;
        if (!gsum(arz, &rzn)) return;
        rz_new = rzn;
        if (fabs(rz) < 1.0e-60) {
            done = 1;
            brk = 1;
            break;
        }
        beta = rzn / rz;
        rz = rzn;
        pend = true;
        iter += 1;
    }
    // leave p = z + beta p in a.p for the host and the next launch
    if (pend || pb) {
        const double *pold = pb ? a.p2 : a.p;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_eq; i += gridDim.x * blockDim.x)
            a.p[i] = pend ? a.z[i] + beta * pold[i] : pold[i];
    }
    if (tr) a.trace[PCG_TRACE + 1] = nbar;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->rz = rz;
        sc->rr = rr;
        sc->pAp = pAp;
        sc->alpha = alpha;
        sc->beta = beta;
        sc->rz_new = rz_new;
        sc->iter = iter;
        sc->done = done;
        sc->breakdown = brk;
    }
}

}  // namespace mps
