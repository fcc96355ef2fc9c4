// k_ops.cuh -- particle operators of the time step, FP64, thread per particle.
//
// Each kernel is templated on its neighbour source: CellSource (the sorted
// cell structure, membership decided on the positions of the last sort) or
// ListSource (a caller-supplied NeighborList).  The loop bodies restate the
// reference operators in their exact floating-point order:
//   viscosity            operators.c:50-85 + simulation.c:31-40
//   explicit update      simulation.c:52-67
//   collision            operators.c:371-446 (3-D), 2D operators.c:324-392
//   number density       operators.c:17-38
//   neighbour count      operators.c:226-246
//   surface flags        operators.c:206-219, 253-267
//   P_min + gradient     operators.c:102-181
//   correction, wall, out-of-bounds   simulation.c:100-117, boundary.c:12-61
//   driven walls                      no counterpart (fixed walls when A = 0)
#pragma once

#include "device.cuh"

namespace mps {

// Step mode: acc = g + nu*coeff*lap for fluid, 0 otherwise (simulation.c:31-43).
// Accumulate mode: acc += nu*coeff*lap for fluid only (calc_viscosity_term).
template <int D, class Src>
__global__ void k_viscosity(Src src, State<D> s, Consts k, int n, int accumulate)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (s.type[i] != FLUID) {
        if (!accumulate) {
#pragma unroll
            for (int d = 0; d < D; d++) s.acc[d][i] = 0.0;
        }
        return;
    }
    double pi[D], vi[D], lap[D];
    load_vec<D>(pi, s.pos, i);
    load_vec<D>(vi, s.vel, i);
#pragma unroll
    for (int d = 0; d < D; d++) lap[d] = 0.0;
    src.for_each(i, [&](int j) {
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        double w = kweight(sqrt(dist2<D>(pi, pj)), k.re_lap, k.rmin);
#pragma unroll
        for (int d = 0; d < D; d++) lap[d] += (s.vel[d][j] - vi[d]) * w;
    });
#pragma unroll
    for (int d = 0; d < D; d++) {
        double a = accumulate ? s.acc[d][i] : k.gravity[d];
        a += k.visc_coeff * lap[d];
        s.acc[d][i] = a;
    }
}

// Surface tension of the potential model (operators.c:281-354, 2-D
// operators.c:231-309), added to the acceleration of every fluid particle:
// first the fluid neighbours (liquid-liquid, coefficient ll = C_LL / (rho
// l0^D)), then, when `sl_on`, the wall neighbours (solid-liquid, sl), each in
// list order, for pairs with 1e-9 l0 <= r < re_st:
//   acc += (coeff * f) * (dr / r),  f = -(r - l0) (r - re_st).
// which: 1 the fluid pass, 2 the wall pass, 3 both (the step).
template <int D, class Src>
__global__ void k_surface_tension(Src src, State<D> s, Consts k, int n, int which)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
    double pi[D], a[D];
    load_vec<D>(pi, s.pos, i);
    load_vec<D>(a, s.acc, i);
    for (int pass = 0; pass < 2; pass++) {
        if (!(which & (1 << pass))) continue;
        if (pass == 1 && !k.st_sl_on) continue;
        int want = pass == 0 ? FLUID : WALL;
        double coeff = pass == 0 ? k.st_ll : k.st_sl;
        src.for_each(i, [&](int j) {
            if (s.type[j] != want) return;
            double pj[D], dr[D];
            load_vec<D>(pj, s.pos, j);
            double r = sqrt(dist2v<D>(pi, pj, dr));
            if (r < k.st_rmin || r >= k.re_st) return;
            double f = -(r - k.l0) * (r - k.re_st);
            double cf = coeff * f;
#pragma unroll
            for (int d = 0; d < D; d++) a[d] += cf * (dr[d] / r);
        });
    }
#pragma unroll
    for (int d = 0; d < D; d++) s.acc[d][i] = a[d];
}

// Hybrid contact-line friction of the 3-D serial variant (mps_fluid3D
// operators.c:337-492), between the velocity and the position updates.  A
// fluid particle with a wall neighbour within re_st (the nearest, first in
// list order, is j*) and a fluid-only number density below the surface
// threshold is on the contact line.  Its wall normal comes from the walls in
// j*'s list, its free-surface normal from its fluid neighbours (weights
// w(r, re_st)), cos theta = -n_w . n_lv, and the slide direction is n_lv
// projected on the wall's tangent plane.  Slow particles (|v| <= v_c) stop
// when theta is within dtheta of the wetting angle; fast ones lose a share of
// their slide velocity, clipped so it never reverses.  Each thread changes
// only its own velocity, from positions that no thread changes here.
template <int D, class Src>
__global__ void k_friction(Src src, State<D> s, Consts k, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
    double pi[D];
    load_vec<D>(pi, s.pos, i);
    double re_st2 = k.re_st * k.re_st, re_n2 = k.re_n * k.re_n;
    double n_fluid = 0.0, r2_star = 1.0e30;
    int j_star = -1;
    src.for_each(i, [&](int j) {
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        double r2 = dist2<D>(pi, pj);
        if (s.type[j] == FLUID) {
            if (r2 < re_n2) n_fluid += kweight(sqrt(r2), k.re_n, k.rmin);
        } else if (s.type[j] == WALL) {
            if (r2 < re_st2 && r2 < r2_star) {
                r2_star = r2;
                j_star = j;
            }
        }
    });
    if (j_star < 0 || n_fluid >= k.surf_thr) return;
    double ps[D], nw[D], nlv[D];
    load_vec<D>(ps, s.pos, j_star);
#pragma unroll
    for (int d = 0; d < D; d++) nw[d] = nlv[d] = 0.0;
    src.for_each(j_star, [&](int m) {
        if (s.type[m] != WALL) return;
        double pm[D], dr[D], r2 = 0.0;
        load_vec<D>(pm, s.pos, m);
#pragma unroll
        for (int d = 0; d < D; d++) {
            dr[d] = ps[d] - pm[d];
            r2 += dr[d] * dr[d];
        }
        double r = sqrt(r2);
        if (r < k.st_rmin) return;
        double w = kweight(r, k.re_st, k.rmin);
#pragma unroll
        for (int d = 0; d < D; d++) nw[d] += w * dr[d] / r;
    });
    double mag = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) mag += nw[d] * nw[d];
    mag = sqrt(mag);
    if (mag < 1.0e-9) return;
#pragma unroll
    for (int d = 0; d < D; d++) nw[d] /= mag;
    int fluid_count = 0;
    src.for_each(i, [&](int j) {
        if (s.type[j] != FLUID) return;
        double pj[D], dr[D];
        load_vec<D>(pj, s.pos, j);
        double r = sqrt(dist2v<D>(pi, pj, dr));
        if (r < k.st_rmin) return;
        double w = kweight(r, k.re_st, k.rmin);
#pragma unroll
        for (int d = 0; d < D; d++) nlv[d] -= w * dr[d] / r;
        fluid_count++;
    });
    if (fluid_count == 0) return;
    mag = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) mag += nlv[d] * nlv[d];
    mag = sqrt(mag);
    if (mag < 1.0e-9) return;
#pragma unroll
    for (int d = 0; d < D; d++) nlv[d] /= mag;
    double cos_th = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) cos_th -= nw[d] * nlv[d];
    cos_th = fmax(-1.0, fmin(1.0, cos_th));
    double theta = acos(cos_th);
    double dot = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) dot += nlv[d] * nw[d];
    double e[D], emag = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        e[d] = nlv[d] - dot * nw[d];
        emag += e[d] * e[d];
    }
    emag = sqrt(emag);
    if (emag < 1.0e-9) return;
#pragma unroll
    for (int d = 0; d < D; d++) e[d] /= emag;
    double v[D], v2 = 0.0;
    load_vec<D>(v, s.vel, i);
#pragma unroll
    for (int d = 0; d < D; d++) v2 += v[d] * v[d];
    if (sqrt(v2) <= k.fr_vc) {
        if (fabs(theta - k.fr_theta_s) <= k.fr_dtheta) {
#pragma unroll
            for (int d = 0; d < D; d++) s.vel[d][i] = 0.0;
        }
        return;
    }
    double sum_w = 0.0;
    src.for_each(i, [&](int j) {
        if (s.type[j] != WALL) return;
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        double r = sqrt(dist2<D>(pi, pj));
        if (r < k.st_rmin) return;
        sum_w += kweight(r, k.re_st, k.rmin);
    });
    double vn = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) vn += v[d] * e[d];
    double dvn = -k.fr_dyn * k.dt * sum_w * vn;
    if (dvn > vn) dvn = vn;
    if (dvn < -vn) dvn = -vn;
#pragma unroll
    for (int d = 0; d < D; d++) s.vel[d][i] = v[d] + dvn * e[d];
}

// The explicit update in two passes, friction between them (3S
// simulation.c:43-60): mode 1, u* = u + dt a; mode 2, r* = r + dt u*.
template <int D>
__global__ void k_explicit_part(State<D> s, Consts k, int n, int mode)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        if (mode == 1) s.vel[d][i] = s.vel[d][i] + k.dt * s.acc[d][i];
        else s.pos[d][i] = s.pos[d][i] + k.dt * s.vel[d][i];
    }
}

template <int D>
__global__ void k_explicit_update(State<D> s, Consts k, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        double v = s.vel[d][i] + k.dt * s.acc[d][i];
        s.vel[d][i] = v;
        s.pos[d][i] = s.pos[d][i] + k.dt * v;
    }
}

// Driven walls (no counterpart in the reference): every WALL and DUMMY
// particle at rest + dx along `axis` with velocity vel there, the values of
// the drive at the end of the step.
template <int D>
__global__ void k_drive_walls(State<D> s, int n, const double *__restrict__ rest, int axis, double dx, double vel)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = s.type[i];
    if (t != WALL && t != DUMMY) return;
    s.pos[axis][i] = rest[s.id[i]] + dx;
#pragma unroll
    for (int d = 0; d < D; d++) s.vel[d][i] = 0.0;
    s.vel[axis][i] = vel;
}

// Rest position of every particle, rest[d * stride + reference index].
template <int D>
__global__ void k_set_rest(State<D> s, int n, int stride, double *__restrict__ rest)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
#pragma unroll
    for (int d = 0; d < D; d++) rest[(size_t)d * stride + s.id[i]] = s.pos[d][i];
}

// Impulse of partner j on v_i; the same tests and order as the reference.
template <int D>
__device__ __forceinline__ void collide(double *vi, const double *pi, const double *pj,
                                        const double *vj, const Consts &k)
{
    double dr[D];
    double r2 = dist2v<D>(pi, pj, dr);
    if (r2 >= k.col2) return;
    double r = sqrt(r2);
    if (r < k.col_rmin) return;
    double vn = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) vn += (vi[d] - vj[d]) * (dr[d] / r);
    if (vn <= 0.0) return;
    double imp = k.half1pe * vn;
#pragma unroll
    for (int d = 0; d < D; d++) vi[d] -= imp * (dr[d] / r);
}

// 3-D collision: partners from the previous step's list, in list order.
template <int D, class Src>
__global__ void k_collision_list(Src src, State<D> s, Consts k, int n, double *__restrict__ vafter)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double vi[D];
    load_vec<D>(vi, s.vel, i);
    if (s.type[i] == FLUID) {
        double pi[D];
        load_vec<D>(pi, s.pos, i);
        src.for_each(i, [&](int j) {
            if (s.type[j] == GHOST) return;
            double pj[D], vj[D];
            load_vec<D>(pj, s.pos, j);
            load_vec<D>(vj, s.vel, j);
            collide<D>(vi, pi, pj, vj, k);
        });
    }
#pragma unroll
    for (int d = 0; d < D; d++) vafter[(size_t)d * n + i] = vi[d];
}

// 2-D collision (2D operators.c:341-379): every non-ghost particle is a
// candidate, applied in ascending reference index.  Partners lie within
// collision_distance < cell size of i, so they sit in the 3x3 cells of a
// structure sorted at the current positions; the ascending order is
// produced by repeatedly taking the smallest index above the last one.
template <int D>
__global__ void k_collision_allpairs(CellSource<D> src, State<D> s, Consts k, int n,
                                     double *__restrict__ vafter)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double vi[D];
    load_vec<D>(vi, s.vel, i);
    if (s.type[i] == FLUID) {
        double pi[D];
        load_vec<D>(pi, s.pos, i);
        int last = -1;
        for (;;) {
            int best = 0x7fffffff, bt = -1;
            src.for_each(i, [&](int t) {
                if (s.type[t] == GHOST) return;
                int idt = s.id[t];
                if (idt <= last || idt >= best) return;
                double pt[D];
                load_vec<D>(pt, s.pos, t);
                if (dist2<D>(pi, pt) >= k.col2) return;
                best = idt;
                bt = t;
            });
            if (bt < 0) break;
            double pj[D], vj[D];
            load_vec<D>(pj, s.pos, bt);
            load_vec<D>(vj, s.vel, bt);
            collide<D>(vi, pi, pj, vj, k);
            last = best;
        }
    }
#pragma unroll
    for (int d = 0; d < D; d++) vafter[(size_t)d * n + i] = vi[d];
}

template <int D>
__global__ void k_collision_apply(State<D> s, Consts k, int n, const double *__restrict__ vafter)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        double va = vafter[(size_t)d * n + i];
        double dv = va - s.vel[d][i];
        s.pos[d][i] = s.pos[d][i] + k.dt * dv;
        s.vel[d][i] = va;
    }
}

// Number density, optional neighbour count and the surface flag.  `count`
// receives the list length for the overflow check of the cell structure.
template <int D, class Src>
__global__ void k_density(Src src, State<D> s, Consts k, int n, unsigned *err, int check_overflow,
                          int set_flags)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double pi[D];
    load_vec<D>(pi, s.pos, i);
    double sum = 0.0;
    int len = 0, cnt = 0;
    src.for_each(i, [&](int j) {
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        double r2 = dist2<D>(pi, pj);
        sum += kweight(sqrt(r2), k.re_n, k.rmin);
        cnt += (r2 < k.re_n2);
        len++;
    });
    if (check_overflow && len > k.max_nb) atomicOr(err, ERR_NEIGHBOR_OVERFLOW);
    s.n[i] = sum;
    if (!set_flags) return;
    int fluid = s.type[i] == FLUID;
    if (k.surf_method == 1) {
        s.ncount[i] = cnt;
        s.surf[i] = (fluid && (double)cnt < k.count_thr) ? 1 : 0;
    } else {
        s.surf[i] = (fluid && sum < k.surf_thr) ? 1 : 0;
    }
}

template <int D, class Src>
__global__ void k_neighbor_count(Src src, State<D> s, Consts k, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double pi[D];
    load_vec<D>(pi, s.pos, i);
    int cnt = 0;
    src.for_each(i, [&](int j) {
        double pj[D];
        load_vec<D>(pj, s.pos, j);
        cnt += (dist2<D>(pi, pj) < k.re_n2);
    });
    s.ncount[i] = cnt;
}

template <int D>
__global__ void k_surface(State<D> s, Consts k, int n, int by_count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int fluid = s.type[i] == FLUID;
    if (by_count)
        s.surf[i] = (fluid && (double)s.ncount[i] < k.count_thr) ? 1 : 0;
    else
        s.surf[i] = (fluid && s.n[i] < k.surf_thr) ? 1 : 0;
}

template <int D, class Src>
__global__ void k_pmin(Src src, State<D> s, int n, double *__restrict__ pmin)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double m = s.p[i];
    src.for_each(i, [&](int j) {
        double pj = s.p[j];
        if (pj < m) m = pj;
    });
    pmin[i] = m;
}

template <int D, class Src>
__global__ void k_gradient(Src src, State<D> s, Consts k, int n, const double *__restrict__ pmin)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || s.type[i] != FLUID) return;
    double pi[D], g[D];
    load_vec<D>(pi, s.pos, i);
    double Pi = s.p[i];
    double pim = pmin ? pmin[i] : 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) g[d] = 0.0;
    src.for_each(i, [&](int j) {
        double pj[D], dr[D];
        load_vec<D>(pj, s.pos, j);
        double r2 = dist2v<D>(pi, pj, dr);
        if (r2 < k.grad_r2min) return;
        double w = kweight(sqrt(r2), k.re_lap, k.rmin);
        double dp;
        if (k.cmps == 1)      dp = Pi + s.p[j] - pim - pmin[j];
        else if (k.cmps == 2) dp = Pi + s.p[j];
        else                  dp = s.p[j] - pim;
#pragma unroll
        for (int d = 0; d < D; d++) g[d] += dp / r2 * dr[d] * w;
    });
#pragma unroll
    for (int d = 0; d < D; d++) s.acc[d][i] = k.neg_grad * g[d] / k.density;
}

// u += dt*acc, r += dt*(dt*acc) for fluid; walls and ghosts get zero
// velocity/acceleration; fluid outside domain +- l0*(wall_layers+1) or NaN
// becomes a ghost with P = n = v = a = 0.
template <int D>
__global__ void k_correct(State<D> s, Consts k, int n, int do_correct, int do_wall, int do_oob)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int t = s.type[i];
    if (do_correct && t == FLUID) {
#pragma unroll
        for (int d = 0; d < D; d++) {
            double du = k.dt * s.acc[d][i];
            s.vel[d][i] = s.vel[d][i] + du;
            s.pos[d][i] = s.pos[d][i] + k.dt * du;
        }
    }
    if (do_wall && (t == GHOST || (t == WALL && !k.drive_on))) {
#pragma unroll
        for (int d = 0; d < D; d++) { s.vel[d][i] = 0.0; s.acc[d][i] = 0.0; }
    }
    if (do_wall && t == WALL && k.drive_on) {   // driven walls keep their prescribed velocity
#pragma unroll
        for (int d = 0; d < D; d++) s.acc[d][i] = 0.0;
    }
    if (do_oob && t == FLUID) {
        bool out = false;
#pragma unroll
        for (int d = 0; d < D; d++) {
            double x = s.pos[d][i];
            if (x < k.oob_lo[d] || x > k.oob_hi[d] || isnan(x)) out = true;
        }
        if (out) {
            s.type[i] = GHOST;
            s.p[i] = 0.0;
            s.n[i] = 0.0;
#pragma unroll
            for (int d = 0; d < D; d++) { s.vel[d][i] = 0.0; s.acc[d][i] = 0.0; }
        }
    }
}

template <int D>
__global__ void k_clamp(State<D> s, int n)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && s.type[i] == FLUID && s.p[i] < 0.0) s.p[i] = 0.0;
}

}  // namespace mps
