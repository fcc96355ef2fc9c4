// k_adj.cuh -- adjoint (vector-Jacobian product) of one MPS time step, FP64.
//
// The forward step (simulation.c:19-118) is recomputed from its input state
// with a few intermediates recorded, then these kernels run its stages in
// reverse.  Every discrete decision of the forward step is held fixed: list
// membership, collision partners, their order and the vn > 0 branch, the
// free-surface flags, the PPE unknown set, the P_min argument and ghosting.
// Derivatives of the kernel weight w(r) = re/max(r, rmin) - 1 (kernel.c:12-20)
// are -re/r^2 for rmin <= r < re and 0 elsewhere.
//
// Indexing.  The engine reorders particles at every cell sort, so every
// adjoint array is indexed by the particle's reference index (State::id)
// and the kernels read the engine state in whatever order it currently has.
// Neighbour sums that feed another particle's adjoint are evaluated in
// gather form -- each particle loops over its own (symmetric) neighbour set
// and adds the terms in which it appears as the partner -- so that no kernel
// scatters with atomics and every result is deterministic.
//
// Supported switches: hs_mode 0, ppe_type 0, cmps_gradient 0, no pressure
// clamp, no surface tension (the dam-break configurations).
#pragma once

#include "device.cuh"
#include "k_ppe.cuh"

namespace mps {

constexpr int ADJ_MAXEV = 8;   // collision impulses recorded per particle and step

enum : unsigned { ERR_ADJ_EVENTS = 128u };   // more than ADJ_MAXEV impulses on one particle

template <int D>
struct Adj {
    double *lx[D], *lu[D];     // in: adjoint of the step's output; out: of its input
    double *xs[D], *us[D];     // x*, u* after the explicit update (recorded)
    double *lxc[D], *luc[D];   // adjoint of the post-collision state x^c, u^c
    double *lxs[D], *lus[D];   // adjoint of x*, u*
    double *lap[D];            // adjoint of the pressure-gradient acceleration
    double *la[D];             // adjoint of the explicit acceleration
    double *gv[D];             // per-particle gravity gradient terms
    double *pmv;               // P_min value
    double *psc;               // adjoint flowing into P at the P_min argument
    double *lp;                // adjoint of P
    double *mu;                // PPE adjoint solution
    double *nv;                // per-particle viscosity gradient terms
    double *dA, *df;           // per-particle wall-drive gradient terms (amplitude, frequency)
    int *pmi;                  // P_min argument (reference index)
    int *evn, *evj;            // collision impulses per particle, partner of each
    double *evd;               // per impulse: partner velocity adjoint (D), separation adjoint (D)
};

// w and dw/dr of kernel.c:12-20.
__device__ __forceinline__ void kweight_d(double r, double re, double rmin, double &w, double &dw)
{
    if (r >= re) {
        w = 0.0;
        dw = 0.0;
    } else if (r < rmin) {
        w = re / rmin - 1.0;
        dw = 0.0;
    } else {
        w = re / r - 1.0;
        dw = -re / (r * r);
    }
}

template <int D>
__device__ __forceinline__ void load_id(double *out, double *const *a, int q)
{
#pragma unroll
    for (int d = 0; d < D; d++) out[d] = a[d][q];
}

// x*, u* (or any state pair) by reference index.
template <int D>
__global__ void k_adj_record(State<D> s, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.xs[d][q] = s.pos[d][i];
        a.us[d][q] = s.vel[d][i];
    }
}

// Correction (simulation.c:100-108) and ghosting (boundary.c:31-61), in
// reverse: state = after the gradient, before the correction.  A particle
// that stays fluid passes its output adjoint to x^c, u^c and to its
// pressure-gradient acceleration (u = u^c + dt a, x = x^c + dt (dt a));
// walls, dummies and particles ghosted by this step have constant outputs.
template <int D>
__global__ void k_adj_seed(State<D> s, Consts k, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    bool keep = s.type[i] == FLUID;
    if (keep) {
#pragma unroll
        for (int d = 0; d < D; d++) {
            double du = k.dt * s.acc[d][i];
            double x = s.pos[d][i] + k.dt * du;
            if (x < k.oob_lo[d] || x > k.oob_hi[d] || isnan(x)) keep = false;
        }
    }
#pragma unroll
    for (int d = 0; d < D; d++) {
        double lx = keep ? a.lx[d][q] : 0.0, lu = keep ? a.lu[d][q] : 0.0;
        a.lap[d][q] = k.dt * lu + k.dt * k.dt * lx;
        a.lxc[d][q] = lx;
        a.luc[d][q] = lu;
    }
}

// A loss's own derivative with respect to this step's pressures (reference
// order), added to the adjoint of P that the gradient stage left.
__global__ void k_adj_add(int n, const double *__restrict__ src, double *dst)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) dst[q] += src[q];
}

// P_min argument (first strictly smaller value in list order, as k_pmin)
// and, for fluid i, the adjoint that reaches P at that argument:
//   psc_i = -Kc sum_j phi_ij (e_ij . lap_i),  phi = w / r^2, e_ij = x_j - x_i.
template <int D>
__global__ void k_adj_pmin(CellSource<D> src, State<D> s, Consts k, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    double m = s.p[i];
    int am = i;
    src.for_each(i, [&](int j) {
        double pj = s.p[j];
        if (pj < m) {
            m = pj;
            am = j;
        }
    });
    a.pmv[q] = m;
    a.pmi[q] = s.id[am];
    double acc = 0.0;
    if (s.type[i] == FLUID) {
        double pi[D], l[D];
        load_vec<D>(pi, s.pos, i);
        load_id<D>(l, a.lap, q);
        src.for_each(i, [&](int j) {
            double pj[D], e[D];
            load_vec<D>(pj, s.pos, j);
            double r2 = dist2v<D>(pi, pj, e);
            if (r2 < k.grad_r2min) return;
            double w = kweight(sqrt(r2), k.re_lap, k.rmin);
            double el = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) el += e[d] * l[d];
            acc += w / r2 * el;
        });
    }
    a.psc[q] = -(k.neg_grad / k.density) * acc;
}

// Pressure gradient (operators.c:102-181, cmps 0) in reverse, gather form
// for particle p: the adjoint of P_p and of x^c_p from every term T_ij =
// (P_j - Pmin_i) phi(r) e_ij of a fluid particle's acceleration
// a_i = Kc sum_j T_ij in which p appears (i = p, j = p, or p = argmin_i).
//   dT_ij/dx_j = (P_j - Pmin_i) M(e),  M(e) = phi I + (phi'/r) e e^T,
//   dT_ij/dx_i = -dT_ij/dx_j,  dT_ij/dP_j = phi e.
template <int D>
__global__ void k_adj_gradient(CellSource<D> src, State<D> s, Consts k, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    const double Kc = k.neg_grad / k.density;
    bool fi = s.type[i] == FLUID;
    double pi[D], li[D], lx[D];
    load_vec<D>(pi, s.pos, i);
    load_id<D>(li, a.lap, q);
#pragma unroll
    for (int d = 0; d < D; d++) lx[d] = 0.0;
    double Pi = s.p[i], Pmi = a.pmv[q];
    double lp = (fi && a.pmi[q] == q) ? a.psc[q] : 0.0;
    src.for_each(i, [&](int j) {
        int qj = s.id[j];
        bool fj = s.type[j] == FLUID;
        if (fj && a.pmi[qj] == q) lp += a.psc[qj];
        double pj[D], e[D];
        load_vec<D>(pj, s.pos, j);
        double r2 = dist2v<D>(pi, pj, e);
        if (r2 < k.grad_r2min) return;
        double r = sqrt(r2), w, dw;
        kweight_d(r, k.re_lap, k.rmin, w, dw);
        double phi = w / r2;
        double dphi_r = (dw / r2 - 2.0 * w / (r2 * r)) / r;   // phi'(r) / r
        if (fi) {
            double el = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) el += e[d] * li[d];
            double c = -Kc * (s.p[j] - Pmi);
#pragma unroll
            for (int d = 0; d < D; d++) lx[d] += c * (phi * li[d] + dphi_r * el * e[d]);
        }
        if (fj) {
            double lj[D];
            load_id<D>(lj, a.lap, qj);
            double el = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) el += e[d] * lj[d];
            double c = Kc * (Pi - a.pmv[qj]);
#pragma unroll
            for (int d = 0; d < D; d++) lx[d] += c * (phi * lj[d] + dphi_r * el * e[d]);
            lp += -Kc * phi * el;
        }
    });
    a.lp[q] = lp;
#pragma unroll
    for (int d = 0; d < D; d++) a.lxc[d][q] += lx[d];
}

// PPE adjoint right-hand side: b_e = lambda_P of row e's particle, and
// ||b||^2 into sc->rr_outer.
__global__ void k_adj_rhs(int n_eq, const int *__restrict__ part_of_row, const int *__restrict__ id,
                          const double *__restrict__ lp, double *__restrict__ b, double *partials, unsigned *ticket,
                          CGScalars *sc)
{
    __shared__ double sh[CG_BLOCK / 32];
    double acc = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eq; e += gridDim.x * blockDim.x) {
        double v = lp[id[part_of_row[e]]];
        b[e] = v;
        acc += v * v;
    }
    double t = block_sum<CG_BLOCK>(acc, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
    if (last_block(ticket, gridDim.x)) {
        double tot = final_sum(partials, gridDim.x, 1, 0, sh);
        if (threadIdx.x == 0) sc->rr_outer = tot;
    }
}

// b /= ||b||: the adjoint solve runs on a unit right-hand side, so that the
// CG's absolute breakdown guards (|p.Ap| < 1e-30, |r.z| < 1e-60, kept from
// pressure_solver.c:294-309 for the forward solve's parity) cannot stop it
// early when the loss is small.
__global__ void k_adj_scale(int n_eq, double *__restrict__ b, double s)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eq; e += gridDim.x * blockDim.x) b[e] *= s;
}

__global__ void k_adj_mu(int n_eq, const int *__restrict__ part_of_row, const int *__restrict__ id,
                         const double *__restrict__ x, double scale, double *__restrict__ mu)
{
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n_eq; e += gridDim.x * blockDim.x)
        mu[id[part_of_row[e]]] = x[e] * scale;
}

// PPE matrix and right-hand side (pressure_solver.c:411-551, rhs :328-340)
// and number density (operators.c:17-38) in reverse, gather form.  With mu
// the solution of A mu = lambda_P, row i contributes through each weight:
//   dL/dw_L(r_ij) = c mu_i (P_j - P_i)        (i unknown, j not dummy; P_j = 0
//                                              off the unknown set)
//   dL/dn_i       = mu_i rhs_k / n0           (i a fluid unknown)
// and the weights move x^c through r_ij.
template <int D>
__global__ void k_adj_ppe_pairs(CellSource<D> src, State<D> s, Consts k, int n, Adj<D> a,
                                const int *__restrict__ row_of)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    bool ui = row_of[i] >= 0, ndi = s.type[i] != DUMMY;
    double mui = ui ? a.mu[q] : 0.0, Pi = s.p[i];
    double lni = (ui && s.type[i] == FLUID) ? mui * k.rhs_k / k.n0 : 0.0;
    double pi[D], lx[D];
    load_vec<D>(pi, s.pos, i);
#pragma unroll
    for (int d = 0; d < D; d++) lx[d] = 0.0;
    src.for_each(i, [&](int j) {
        double pj[D], e[D];
        load_vec<D>(pj, s.pos, j);
        double r2 = dist2v<D>(pi, pj, e);
        if (!(r2 > 0.0)) return;
        double r = sqrt(r2), wl, dwl, wn, dwn;
        kweight_d(r, k.re_lap, k.rmin, wl, dwl);
        kweight_d(r, k.re_n, k.rmin, wn, dwn);
        bool uj = row_of[j] >= 0, ndj = s.type[j] != DUMMY;
        double Pj = s.p[j];
        double h = lni * dwn;
        if (ui && ndj) h += k.coeff * mui * (Pj - Pi) * dwl;
        if (uj) {
            double muj = a.mu[s.id[j]];
            if (ndi) h += k.coeff * muj * (Pi - Pj) * dwl;
            if (s.type[j] == FLUID) h += muj * k.rhs_k / k.n0 * dwn;
        }
#pragma unroll
        for (int d = 0; d < D; d++) lx[d] -= h * e[d] / r;
    });
#pragma unroll
    for (int d = 0; d < D; d++) a.lxc[d][q] += lx[d];
}

// One recorded impulse of the collision (operators.c:407-427) in reverse:
// v_out = v_in - h ((v_in - u_j) . n) n,  n = (x_j - x_i) / r.
template <int D>
__device__ __forceinline__ void collide_reverse(const double *vin, const double *xi, const double *xj,
                                                const double *uj, double half1pe, double *lv, double *luj,
                                                double *ldr)
{
    double dr[D];
    double r2 = dist2v<D>(xi, xj, dr);
    double r = sqrt(r2);
    double nv[D], av[D];
    double vn = 0.0, s1 = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        nv[d] = dr[d] / r;
        av[d] = vin[d] - uj[d];
        vn += av[d] * nv[d];
        s1 += nv[d] * lv[d];
    }
    double ln[D], nln = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        luj[d] = half1pe * s1 * nv[d];
        ln[d] = -half1pe * (av[d] * s1 + vn * lv[d]);
        nln += nv[d] * ln[d];
    }
#pragma unroll
    for (int d = 0; d < D; d++) {
        ldr[d] = (ln[d] - nv[d] * nln) / r;
        lv[d] -= half1pe * s1 * nv[d];
    }
}

// Collision in reverse for fluid i: the impulses are replayed from x*, u*
// (partners and order as k_collision_list, 3-D, or k_collision_allpairs,
// 2-D), then walked backwards from the adjoint of x^c = x* + dt (v - u*_i)
// and u^c = v.  The partner terms go to the impulse records, gathered by
// the partners in k_adj_collision_gather.
template <int D, bool LIST>
__global__ void k_adj_collision(CellSource<D> src, State<D> s, Consts k, int n, Adj<D> a, unsigned *err)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    if (s.type[i] != FLUID) {
        // walls and dummies pass through the collision unchanged (x^c = x*, u^c = u*)
        bool g = s.type[i] == GHOST;
#pragma unroll
        for (int d = 0; d < D; d++) {
            a.lxs[d][q] = g ? 0.0 : a.lxc[d][q];
            a.lus[d][q] = g ? 0.0 : a.luc[d][q];
        }
        a.evn[q] = 0;
        return;
    }
    double xi[D], v[D];
    load_id<D>(xi, a.xs, q);
    load_id<D>(v, a.us, q);
    int ev_j[ADJ_MAXEV];
    double ev_v[ADJ_MAXEV][D];
    int nev = 0;
    auto visit = [&](int j) {
        int qj = s.id[j];
        double xj[D], uj[D], dr[D];
        load_id<D>(xj, a.xs, qj);
        load_id<D>(uj, a.us, qj);
        double r2 = dist2v<D>(xi, xj, dr);
        if (r2 >= k.col2) return;
        double r = sqrt(r2);
        if (r < k.col_rmin) return;
        double vn = 0.0;
#pragma unroll
        for (int d = 0; d < D; d++) vn += (v[d] - uj[d]) * (dr[d] / r);
        if (vn <= 0.0) return;
        if (nev < ADJ_MAXEV) {
            ev_j[nev] = qj;
#pragma unroll
            for (int d = 0; d < D; d++) ev_v[nev][d] = v[d];
        }
        nev++;
        double imp = k.half1pe * vn;
#pragma unroll
        for (int d = 0; d < D; d++) v[d] -= imp * (dr[d] / r);
    };
    if (LIST) {
        src.for_each(i, [&](int j) {
            if (s.type[j] != GHOST) visit(j);
        });
    } else {
        int last = -1;
        for (;;) {
            int best = 0x7fffffff, bt = -1;
            src.for_each(i, [&](int t) {
                if (s.type[t] == GHOST) return;
                int idt = s.id[t];
                if (idt <= last || idt >= best) return;
                double xt[D];
                load_id<D>(xt, a.xs, idt);
                if (dist2<D>(xi, xt) >= k.col2) return;
                best = idt;
                bt = t;
            });
            if (bt < 0) break;
            visit(bt);
            last = best;
        }
    }
    if (nev > ADJ_MAXEV) {
        atomicOr(err, ERR_ADJ_EVENTS);
        nev = ADJ_MAXEV;
    }
    double lv[D], lxs[D], lus[D];
#pragma unroll
    for (int d = 0; d < D; d++) {
        double lxc = a.lxc[d][q];
        lv[d] = a.luc[d][q] + k.dt * lxc;
        lxs[d] = lxc;
        lus[d] = -k.dt * lxc;
    }
    for (int e = nev - 1; e >= 0; e--) {
        int qj = ev_j[e];
        double xj[D], uj[D], luj[D], ldr[D];
        load_id<D>(xj, a.xs, qj);
        load_id<D>(uj, a.us, qj);
        collide_reverse<D>(ev_v[e], xi, xj, uj, k.half1pe, lv, luj, ldr);
        size_t o = (size_t)q * ADJ_MAXEV + e;
        a.evj[o] = qj;
#pragma unroll
        for (int d = 0; d < D; d++) {
            a.evd[o * 2 * D + d] = luj[d];
            a.evd[o * 2 * D + D + d] = ldr[d];
            lxs[d] -= ldr[d];
        }
    }
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.lxs[d][q] = lxs[d];
        a.lus[d][q] = lus[d] + lv[d];
    }
    a.evn[q] = nev;
}

// Partner terms of the impulses: particle p (fluid, or a wall or dummy, whose
// adjoint feeds the wall drive's gradient) adds what every fluid i that hit
// it recorded (i is in p's candidate set, which is symmetric).
template <int D>
__global__ void k_adj_collision_gather(CellSource<D> src, State<D> s, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    if (s.type[i] == GHOST) return;
    double lu[D], lx[D];
#pragma unroll
    for (int d = 0; d < D; d++) lu[d] = lx[d] = 0.0;
    src.for_each(i, [&](int j) {
        if (s.type[j] != FLUID) return;
        int qj = s.id[j];
        int ne = a.evn[qj];
        for (int e = 0; e < ne; e++) {
            size_t o = (size_t)qj * ADJ_MAXEV + e;
            if (a.evj[o] != q) continue;
#pragma unroll
            for (int d = 0; d < D; d++) {
                lu[d] += a.evd[o * 2 * D + d];
                lx[d] += a.evd[o * 2 * D + D + d];
            }
        }
    });
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.lus[d][q] += lu[d];
        a.lxs[d][q] += lx[d];
    }
}

// Without collision x^c = x*, u^c = u*.
template <int D>
__global__ void k_adj_no_collision(State<D> s, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    bool f = s.type[i] != GHOST;
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.lxs[d][q] = f ? a.lxc[d][q] : 0.0;
        a.lus[d][q] = f ? a.luc[d][q] : 0.0;
    }
}

// Explicit update (simulation.c:52-67) in reverse: x* = x + dt u*,
// u* = u + dt a, so the acceleration's adjoint is dt (lus + dt lxs).
template <int D>
__global__ void k_adj_accel(State<D> s, Consts k, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    bool f = s.type[i] == FLUID;
#pragma unroll
    for (int d = 0; d < D; d++) a.la[d][q] = f ? k.dt * (a.lus[d][q] + k.dt * a.lxs[d][q]) : 0.0;
}

// Viscosity (operators.c:50-85) and the explicit update in reverse, gather
// form, on the previous step's list (state = the step's input):
//   a_i = g + nu c sum_j (u_j - u_i) w_L(r_ij)   (fluid i)
// Writes the adjoint of the step's input x, u over a.lx, a.lu (walls and
// dummies: of their prescribed positions and velocities at the step's
// start, for the wall drive's gradient), and the per-particle gravity and
// viscosity gradient terms.
template <int D>
__global__ void k_adj_viscosity(CellSource<D> src, State<D> s, Consts k, int n, Adj<D> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    bool fi = s.type[i] == FLUID;
    double pi[D], ui[D], lai[D], lu[D], lx[D];
    load_vec<D>(pi, s.pos, i);
    load_vec<D>(ui, s.vel, i);
    load_id<D>(lai, a.la, q);
#pragma unroll
    for (int d = 0; d < D; d++) {
        lu[d] = fi ? a.lus[d][q] + k.dt * a.lxs[d][q] : 0.0;
        lx[d] = fi ? a.lxs[d][q] : 0.0;
    }
    const double vc = k.visc_coeff;
    double vterm = 0.0;
    src.for_each(i, [&](int j) {
        int qj = s.id[j];
        double pj[D], uj[D], e[D];
        load_vec<D>(pj, s.pos, j);
        load_vec<D>(uj, s.vel, j);
        double r2 = dist2v<D>(pi, pj, e);
        double r = sqrt(r2), w, dw;
        kweight_d(r, k.re_lap, k.rmin, w, dw);
        double h = 0.0;
        if (fi) {
            double du_l = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) {
                lu[d] -= vc * w * lai[d];
                du_l += (uj[d] - ui[d]) * lai[d];
            }
            vterm += du_l * w;
            h += vc * du_l * dw;
        }
        if (s.type[j] == FLUID) {
            double laj[D];
            load_id<D>(laj, a.la, qj);
            double du_l = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) {
                lu[d] += vc * w * laj[d];
                du_l += (ui[d] - uj[d]) * laj[d];
            }
            h += vc * du_l * dw;
        }
        if (r > 0.0) {
#pragma unroll
            for (int d = 0; d < D; d++) lx[d] -= h * e[d] / r;
        }
    });
    bool live = s.type[i] != GHOST;
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.lx[d][q] = live ? lx[d] : 0.0;
        a.lu[d][q] = live ? lu[d] : 0.0;
        a.gv[d][q] = fi ? lai[d] : 0.0;
    }
    a.nv[q] = fi ? k.coeff * vterm : 0.0;
}

// Wall drive x = rest + A sin(w t), u = A w cos(w t), w = 2 pi f, along the
// drive axis: a wall or dummy particle's adjoints of its prescribed
// position and velocity at the step's end (t1: lxs, lus) and start (t0:
// lx, lu) give its terms of dL/dA and dL/df; its step-start adjoints are
// then cleared (a prescribed state has no earlier dependence).  `first`:
// the step starts from the uploaded state, whose wall velocity is not the
// drive's.
struct DriveT {
    double A, w, t0, t1, s0, c0, s1, c1;
    int axis, first;
};

template <int D>
__global__ void k_adj_drive(State<D> s, int n, Adj<D> a, DriveT dv)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int q = s.id[i];
    int t = s.type[i];
    double gA = 0.0, gf = 0.0;
    if (t == WALL || t == DUMMY) {
        const double tp = 2.0 * 3.14159265358979323846;
        double lx1 = a.lxs[dv.axis][q], lu1 = a.lus[dv.axis][q];
        double lx0 = a.lx[dv.axis][q], lu0 = dv.first ? 0.0 : a.lu[dv.axis][q];
        gA = lx1 * dv.s1 + lu1 * dv.w * dv.c1 + lx0 * dv.s0 + lu0 * dv.w * dv.c0;
        gf = tp * (lx1 * dv.A * dv.c1 * dv.t1 + lu1 * (dv.A * dv.c1 - dv.A * dv.w * dv.s1 * dv.t1) +
                   lx0 * dv.A * dv.c0 * dv.t0 + lu0 * (dv.A * dv.c0 - dv.A * dv.w * dv.s0 * dv.t0));
    }
    a.dA[q] = gA;
    a.df[q] = gf;
    if (t != FLUID) {
#pragma unroll
        for (int d = 0; d < D; d++) {
            a.lx[d][q] = 0.0;
            a.lu[d][q] = 0.0;
        }
    }
}

// Deterministic sums of the per-particle gravity (D), viscosity and wall
// drive (amplitude, frequency) terms over [0, n), added to out[0..D+2].
template <int D>
__global__ void k_adj_param_sum(int n, Adj<D> a, double *partials, unsigned *ticket, double *out)
{
    constexpr int NC = D + 3;
    __shared__ double sh[CG_BLOCK / 32];
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = 0.0;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
#pragma unroll
        for (int d = 0; d < D; d++) acc[d] += a.gv[d][q];
        acc[D] += a.nv[q];
        acc[D + 1] += a.dA[q];
        acc[D + 2] += a.df[q];
    }
#pragma unroll
    for (int c = 0; c < NC; c++) {
        double t = block_sum<CG_BLOCK>(acc[c], sh);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * NC + c] = t;
    }
    if (last_block(ticket, gridDim.x)) {
#pragma unroll
        for (int c = 0; c < NC; c++) {
            double tot = final_sum(partials, gridDim.x, NC, c, sh);
            if (threadIdx.x == 0) out[c] += tot;
        }
    }
}

// Seeds in reference order: lam[q * D + d] (AoS) into the SoA arrays.
template <int D>
__global__ void k_adj_set(int n, const double *__restrict__ lam_x, const double *__restrict__ lam_u, Adj<D> a)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        a.lx[d][q] = lam_x ? lam_x[(size_t)q * D + d] : 0.0;
        a.lu[d][q] = lam_u ? lam_u[(size_t)q * D + d] : 0.0;
    }
}

template <int D>
__global__ void k_adj_get(int n, double *__restrict__ lam_x, double *__restrict__ lam_u, Adj<D> a)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        lam_x[(size_t)q * D + d] = a.lx[d][q];
        lam_u[(size_t)q * D + d] = a.lu[d][q];
    }
}

}  // namespace mps
