/*
 * mps_oracle.c -- CPU restatement of the reference MPS time step (checker).
 *
 * TEST INFRASTRUCTURE ONLY: see mps_oracle.h.  Built twice by oracle/Makefile
 * (MPS_DIM=3 -> liboracle3d.so, MPS_DIM=2 -> liboracle2d.so) with
 * -O2 -ffp-contract=off.  Citations name the reference function each block
 * restates; 3P = mps_fluid3D_parallel, 2D = mps_fluid2D.
 *
 * Floating-point order is part of the contract: every sum runs in the same
 * order and association as the reference, so that outputs are bit-identical
 * to the reference built from its own sources.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mps_oracle.h"

#define D MPS_DIM

static int    g_last_iters = 0;
static double g_last_resid = 0.0;

int    oracle_last_iterations(void) { return g_last_iters; }
double oracle_last_residual(void)   { return g_last_resid; }

/* Squared distance accumulated as ((0 + dx^2) + dy^2) + dz^2 with dx = pj - pi,
 * the order of every distance loop in the reference (e.g. 3P operators.c:28-32). */
static inline double dist2(const double *pi, const double *pj)
{
    double acc = 0.0;
    for (int d = 0; d < D; d++) {
        double t = pj[d] - pi[d];
        acc += t * t;
    }
    return acc;
}

static inline double dist2_vec(const double *pi, const double *pj, double *dr)
{
    double acc = 0.0;
    for (int d = 0; d < D; d++) {
        dr[d] = pj[d] - pi[d];
        acc += dr[d] * dr[d];
    }
    return acc;
}

/* 3P kernel.c:12-20: w = re/r - 1 with r clamped below at 0.01*l0, 0 beyond re. */
double oracle_kernel_weight(double r, double re, const SimConfig *cfg)
{
    if (r >= re) return 0.0;
    double rmin = 0.01 * cfg->particle_distance;
    double rr = (r < rmin) ? rmin : r;
    return re / rr - 1.0;
}
#define KW(r, re) oracle_kernel_weight((r), (re), cfg)

/* ------------------------------------------------------------------ */
/* Initial parameters n0, lambda, N0  (3P particle.c:69-221)           */
/* ------------------------------------------------------------------ */

/* Serial semantics of the reference: first strictly larger n0_i in particle
 * index order wins and carries its lambda numerator/denominator.  (The OpenMP
 * build merges per-thread maxima with the same strict '>' and equals this
 * unless two n0_i are bitwise equal.) */
static void finish_initial_params(ParticleSystem *ps, const SimConfig *cfg, int found,
                                  double best_n0, double best_num, double best_den)
{
    double re_lap = cfg->influence_radius_lap;
    if (!found) {
        ps->n0 = 1.0;
        ps->lambda = 1.0;
        return;
    }
    ps->n0 = best_n0;
    if (cfg->use_analytical_lambda)
        ps->lambda = re_lap * re_lap * (double)D * (double)(D - 1)
                   / ((double)(D + 1) * (double)(D + 2));
    else
        ps->lambda = (best_den > 1.0e-10) ? best_num / best_den : 1.0;
}

/* Surface-tension coefficients, 3P particle.c:185-211 (2D particle.c:154-180):
 * the potential's interaction energy summed over rest-lattice pairs across a
 * flat interface; C_LL = sigma l0^(D-1) / sum, C_SL = (1 + cos theta) / 2 C_LL. */
static void surface_tension_coeffs(ParticleSystem *ps, const SimConfig *cfg)
{
    if (!cfg->surface_tension_enabled) return;
    double l0 = cfg->particle_distance, re_st = cfg->influence_radius_st;
    int nmax = (int)ceil(re_st / l0);
    double sum = 0.0;
    for (int dxa = 1; dxa <= nmax; dxa++)
        for (int dxb = -(nmax - 1); dxb <= 0; dxb++)
            for (int dyb = -nmax; dyb <= nmax; dyb++) {
#if D == 3
                for (int dzb = -nmax; dzb <= nmax; dzb++) {
                    double rx = (double)(dxa - dxb) * l0;
                    double ry = (double)dyb * l0;
                    double rz = (double)dzb * l0;
                    double rab = sqrt(rx * rx + ry * ry + rz * rz);
                    if (rab > 0.0 && rab < re_st)
                        sum += (1.0 / 3.0) * (rab - 1.5 * l0 + 0.5 * re_st) * (rab - re_st) * (rab - re_st);
                }
#else
                double rx = (double)(dxa - dxb) * l0;
                double ry = (double)dyb * l0;
                double rab = sqrt(rx * rx + ry * ry);
                if (rab > 0.0 && rab < re_st)
                    sum += (1.0 / 3.0) * (rab - 1.5 * l0 + 0.5 * re_st) * (rab - re_st) * (rab - re_st);
#endif
            }
    if (sum > 0.0) {
#if D == 3
        ps->C_LL = cfg->surface_tension_coeff * l0 * l0 / sum;
#else
        ps->C_LL = cfg->surface_tension_coeff * l0 / sum;
#endif
        double theta = cfg->wetting_angle_SL * M_PI / 180.0;
        ps->C_SL = 0.5 * (1.0 + cos(theta)) * ps->C_LL;
    }
}

static int initial_count_for(const ParticleSystem *ps, int i, double re_n2)
{
    int c = 0;
    for (int j = 0; j < ps->num; j++) {
        if (j == i) continue;
        if (dist2(ps->particles[i].pos, ps->particles[j].pos) < re_n2) c++;
    }
    return c;
}

void oracle_calc_initial_params(ParticleSystem *ps, const SimConfig *cfg)
{
    double re_n = cfg->influence_radius_n, re_lap = cfg->influence_radius_lap;
    double best_n0 = 0.0, best_num = 0.0, best_den = 0.0;
    int found = 0;

    for (int i = 0; i < ps->num; i++) {
        const Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        double n0_i = 0.0, num_i = 0.0, den_i = 0.0;
        for (int j = 0; j < ps->num; j++) {
            if (j == i) continue;
            double r2 = dist2(pi->pos, ps->particles[j].pos);
            double r = sqrt(r2);
            double wn = KW(r, re_n);
            if (wn > 0.0) n0_i += wn;
            double wl = KW(r, re_lap);
            if (wl > 0.0) { num_i += r2 * wl; den_i += wl; }
        }
        if (n0_i > best_n0) { best_n0 = n0_i; best_num = num_i; best_den = den_i; found = 1; }
    }
    finish_initial_params(ps, cfg, found, best_n0, best_num, best_den);
    if (!found) return;   /* the reference returns before N0 (3P particle.c:159-164) */

    if (cfg->surface_detection_method == 1) {
        int best = 0;
        double re_n2 = re_n * re_n;
        for (int i = 0; i < ps->num; i++) {
            if (ps->particles[i].type != MPS_FLUID) continue;
            int c = initial_count_for(ps, i, re_n2);
            if (c > best) best = c;
        }
        ps->n0_count = best;
    }
    surface_tension_coeffs(ps, cfg);
}

/* Same result bit for bit, O(N*K) instead of O(N^2): candidates come from a
 * uniform grid over the particles' own bounding box (so no particle is left
 * out), and each particle's contributions are summed in ascending j, the
 * reference's loop order.  Terms with w <= 0 are skipped by the reference too,
 * and they are the only pairs a radius test drops. */
typedef struct { int j; double r2; } Cand;

static int cand_cmp(const void *a, const void *b)
{
    int x = ((const Cand *)a)->j, y = ((const Cand *)b)->j;
    return (x > y) - (x < y);
}

void oracle_calc_initial_params_cells(ParticleSystem *ps, const SimConfig *cfg)
{
    int n = ps->num;
    double re_n = cfg->influence_radius_n, re_lap = cfg->influence_radius_lap;
    double rmax = re_n > re_lap ? re_n : re_lap;
    double cs = rmax * (1.0 + 1.0e-9);
    double lo[D], hi[D];
    int dims[D];
    long long ncell = 1;
    for (int d = 0; d < D; d++) { lo[d] = INFINITY; hi[d] = -INFINITY; }
    for (int i = 0; i < n; i++)
        for (int d = 0; d < D; d++) {
            double v = ps->particles[i].pos[d];
            if (v < lo[d]) lo[d] = v;
            if (v > hi[d]) hi[d] = v;
        }
    /* Non-finite coordinates would break the grid; fall back to all pairs. */
    for (int d = 0; d < D; d++) {
        if (!isfinite(lo[d]) || !isfinite(hi[d])) { oracle_calc_initial_params(ps, cfg); return; }
        dims[d] = (int)((hi[d] - lo[d]) / cs) + 1;
        ncell *= dims[d];
    }
    if (ncell > 200000000LL) { oracle_calc_initial_params(ps, cfg); return; }

    int *cell_of = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    int *start = (int *)calloc((size_t)ncell + 1, sizeof(int));
    int *order = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    Cand *cand = NULL;
    int cand_cap = 0;
    if (!cell_of || !start || !order) {
        free(cell_of); free(start); free(order);
        oracle_calc_initial_params(ps, cfg);
        return;
    }
    for (int i = 0; i < n; i++) {
        long long c = 0;
        for (int d = D - 1; d >= 0; d--) {
            int k = (int)((ps->particles[i].pos[d] - lo[d]) / cs);
            if (k >= dims[d]) k = dims[d] - 1;
            c = c * dims[d] + k;
        }
        cell_of[i] = (int)c;
        start[c + 1]++;
    }
    for (long long c = 0; c < ncell; c++) start[c + 1] += start[c];
    {
        int *fill = (int *)malloc(sizeof(int) * (size_t)ncell);
        memcpy(fill, start, sizeof(int) * (size_t)ncell);
        for (int i = 0; i < n; i++) order[fill[cell_of[i]]++] = i;
        free(fill);
    }

    double best_n0 = 0.0, best_num = 0.0, best_den = 0.0;
    int found = 0, best_cnt = 0;
    double re_n2 = re_n * re_n, rmax2 = rmax * rmax;
    for (int i = 0; i < n; i++) {
        const Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        int ci[D];
        long long c = cell_of[i];
        for (int d = 0; d < D; d++) { ci[d] = (int)(c % dims[d]); c /= dims[d]; }
        int nc = 0;
        int lo_k[D], hi_k[D], k[D];
        for (int d = 0; d < D; d++) {
            lo_k[d] = ci[d] > 0 ? ci[d] - 1 : 0;
            hi_k[d] = ci[d] < dims[d] - 1 ? ci[d] + 1 : dims[d] - 1;
            k[d] = lo_k[d];
        }
        for (;;) {
            long long cc = 0;
            for (int d = D - 1; d >= 0; d--) cc = cc * dims[d] + k[d];
            for (int s = start[cc]; s < start[cc + 1]; s++) {
                int j = order[s];
                if (j == i) continue;
                double r2 = dist2(pi->pos, ps->particles[j].pos);
                /* keep every pair that can carry a positive weight or count */
                if (!(r2 < rmax2) && !(sqrt(r2) < rmax)) continue;
                if (nc == cand_cap) {
                    cand_cap = cand_cap ? 2 * cand_cap : 1024;
                    cand = (Cand *)realloc(cand, sizeof(Cand) * (size_t)cand_cap);
                }
                cand[nc].j = j;
                cand[nc].r2 = r2;
                nc++;
            }
            int d = 0;
            while (d < D && ++k[d] > hi_k[d]) { k[d] = lo_k[d]; d++; }
            if (d == D) break;
        }
        qsort(cand, (size_t)nc, sizeof(Cand), cand_cmp);
        double n0_i = 0.0, num_i = 0.0, den_i = 0.0;
        int cnt = 0;
        for (int q = 0; q < nc; q++) {
            double r2 = cand[q].r2;
            double r = sqrt(r2);
            double wn = KW(r, re_n);
            if (wn > 0.0) n0_i += wn;
            double wl = KW(r, re_lap);
            if (wl > 0.0) { num_i += r2 * wl; den_i += wl; }
            if (r2 < re_n2) cnt++;
        }
        if (n0_i > best_n0) { best_n0 = n0_i; best_num = num_i; best_den = den_i; found = 1; }
        if (cnt > best_cnt) best_cnt = cnt;
    }
    finish_initial_params(ps, cfg, found, best_n0, best_num, best_den);
    if (found && cfg->surface_detection_method == 1) ps->n0_count = best_cnt;
    if (found) surface_tension_coeffs(ps, cfg);
    free(cand); free(cell_of); free(start); free(order);
}

/* ------------------------------------------------------------------ */
/* Cell linked list and neighbour search (3P neighbor_search.c:92-240) */
/* ------------------------------------------------------------------ */

int oracle_cell_list_init(CellList *cl, int num_particles, double re,
                          const double *domain_min, const double *domain_max)
{
    double margin = 4.0 * re;
    cl->cell_size = re;
    for (int d = 0; d < D; d++) cl->origin[d] = domain_min[d] - margin;
    cl->nx = (int)(((domain_max[0] + margin) - cl->origin[0]) / re) + 2;
    cl->ny = (int)(((domain_max[1] + margin) - cl->origin[1]) / re) + 2;
#if D == 3
    cl->nz = (int)(((domain_max[2] + margin) - cl->origin[2]) / re) + 2;
    cl->total_cells = cl->nx * cl->ny * cl->nz;
#else
    cl->total_cells = cl->nx * cl->ny;
#endif
    cl->head = (int *)malloc(sizeof(int) * (size_t)cl->total_cells);
    cl->next = (int *)malloc(sizeof(int) * (size_t)(num_particles > 0 ? num_particles : 1));
    return (cl->head && cl->next) ? 0 : -1;
}

/* Cell coordinate of a position, (int) truncation of (p - origin) * (1/cs)
 * exactly as 3P neighbor_search.c:155,171-173.  Returns 0 when outside. */
static int cell_coords(const CellList *cl, double cs_inv, const double *p, int *c)
{
    int lim[D];
    lim[0] = cl->nx; lim[1] = cl->ny;
#if D == 3
    lim[2] = cl->nz;
#endif
    for (int d = 0; d < D; d++) {
        double t = (p[d] - cl->origin[d]) * cs_inv;
        /* (int) of NaN or of an out-of-range value is undefined in C; x86
         * yields INT_MIN, which the reference's range test rejects.  Make
         * that rejection explicit. */
        if (!(t > -1.0 && t < 2147483647.0)) return 0;
        c[d] = (int)t;
        if (c[d] < 0 || c[d] >= lim[d]) return 0;
    }
    return 1;
}

static int cell_linear(const CellList *cl, const int *c)
{
#if D == 3
    return (c[2] * cl->ny + c[1]) * cl->nx + c[0];
#else
    return c[1] * cl->nx + c[0];
#endif
}

int oracle_neighbor_search(NeighborList *nl, const ParticleSystem *ps, CellList *cl, double re)
{
    int n = ps->num, maxnb = nl->max_neighbors;
    double re2 = re * re, cs_inv = 1.0 / cl->cell_size;
    memset(nl->count, 0, sizeof(int) * (size_t)n);
    for (int c = 0; c < cl->total_cells; c++) cl->head[c] = -1;

    /* Phase 1: prepend each particle to its cell; within a cell the chain
     * therefore runs in descending particle index. */
    for (int i = 0; i < n; i++) {
        int c[D];
        cl->next[i] = -1;
        if (ps->particles[i].type == MPS_GHOST) continue;
        if (!cell_coords(cl, cs_inv, ps->particles[i].pos, c)) continue;
        int ci = cell_linear(cl, c);
        cl->next[i] = cl->head[ci];
        cl->head[ci] = i;
    }

    /* Phase 2: scan the 3^D block of cells (z, then y, then x outermost to
     * innermost) and keep pairs with r2 < re^2. */
    int lim[D];
    lim[0] = cl->nx; lim[1] = cl->ny;
#if D == 3
    lim[2] = cl->nz;
#endif
    for (int i = 0; i < n; i++) {
        int c[D];
        if (ps->particles[i].type == MPS_GHOST) continue;
        if (!cell_coords(cl, cs_inv, ps->particles[i].pos, c)) continue;
        int lo[D], hi[D];
        for (int d = 0; d < D; d++) {
            lo[d] = c[d] > 0 ? c[d] - 1 : 0;
            hi[d] = c[d] < lim[d] - 1 ? c[d] + 1 : lim[d] - 1;
        }
        int cnt = 0;
        int *row = nl->neighbors + (size_t)i * (size_t)maxnb;
#if D == 3
        for (int z = lo[2]; z <= hi[2]; z++)
#endif
        for (int y = lo[1]; y <= hi[1]; y++)
        for (int x = lo[0]; x <= hi[0]; x++) {
#if D == 3
            int cc[3] = {x, y, z};
#else
            int cc[2] = {x, y};
#endif
            for (int j = cl->head[cell_linear(cl, cc)]; j >= 0; j = cl->next[j]) {
                if (j == i || ps->particles[j].type == MPS_GHOST) continue;
                if (dist2(ps->particles[i].pos, ps->particles[j].pos) < re2) {
                    if (cnt >= maxnb) return -(i + 1);   /* reference: exit(1) */
                    row[cnt++] = j;
                }
            }
        }
        nl->count[i] = cnt;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* Particle operators (3P operators.c)                                 */
/* ------------------------------------------------------------------ */

#define NB(nl, i, k) ((nl)->neighbors[(size_t)(i) * (size_t)(nl)->max_neighbors + (k)])

/* 3P operators.c:17-38 */
void oracle_number_density(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    double re = cfg->influence_radius_n;
    for (int i = 0; i < ps->num; i++) {
        Particle *pi = &ps->particles[i];
        double s = 0.0;
        for (int k = 0; k < nl->count[i]; k++) {
            const Particle *pj = &ps->particles[NB(nl, i, k)];
            s += KW(sqrt(dist2(pi->pos, pj->pos)), re);
        }
        pi->n = s;
    }
}

/* 3P operators.c:50-85: acc += (nu * 2d/(n0 lambda)) * sum (u_j - u_i) w */
/* Surface tension, 3P operators.c:281-354 (2D operators.c:231-309): the
 * potential force f(r) = -(r - l0)(r - re_st) of the fluid neighbours (C_LL)
 * and, unless C_SL is 0, of the wall neighbours (C_SL), on fluid particles,
 * coeff = C / (rho l0^D), acc += coeff * f * (dr / r) in list order. */
static void surface_tension_pass(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg, double C,
                                 int partner)
{
    double re_st = cfg->influence_radius_st;
    double l0 = cfg->particle_distance;
#if D == 3
    double coeff = C / (cfg->density * l0 * l0 * l0);
#else
    double coeff = C / (cfg->density * l0 * l0);
#endif
    for (int i = 0; i < ps->num; i++) {
        Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            if (ps->particles[j].type != partner) continue;
            double dr[D];
            double r = sqrt(dist2_vec(pi->pos, ps->particles[j].pos, dr));
            if (r < 1.0e-9 * l0 || r >= re_st) continue;
            double force_mag = -(r - l0) * (r - re_st);
            for (int d = 0; d < D; d++) pi->acc[d] += coeff * force_mag * (dr[d] / r);
        }
    }
}

void oracle_surface_tension(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    surface_tension_pass(ps, nl, cfg, ps->C_LL, MPS_FLUID);
}

void oracle_surface_tension_SL(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    if (ps->C_SL == 0.0) return;
    surface_tension_pass(ps, nl, cfg, ps->C_SL, MPS_WALL);
}

/* Hybrid static / dynamic friction at the contact line, 3S (mps_fluid3D)
 * operators.c:337-492.  The friction parameters live in the 3-D serial
 * variant's SimConfig only, so they are set apart (oracle_set_friction).
 * For every fluid particle i, with its list: the fluid-only number density
 * n_f (re_n) and the nearest wall particle j* within re_st; a contact-line
 * particle has j* and n_f < surface_threshold * n0.  The wall normal n_w is
 * the normalised sum of w(r, re_st) (j* - k)/r over the walls k in j*'s
 * list, the free-surface normal n_lv the normalised -sum of w(r, re_st)
 * (j - i)/r over i's fluid neighbours, cos theta_i = -n_w . n_lv, and the
 * slide direction e the normalised projection of n_lv on the wall's tangent
 * plane.  Static (|v_i| <= v_c): v_i = 0 when |theta_i - theta_s| <= dtheta.
 * Dynamic: v_n = v_i . e damped by dv_n = -alpha nu (2D / (n0 lambda)) dt
 * (sum of w(r, re_st) over wall neighbours) v_n, clipped to |v_n|.  Each
 * particle changes only its own velocity from positions and its own
 * velocity, so the loop order does not matter. */
#if D == 3
static OracleFriction g_friction = {0, 30.0, 600.0, 0.01};

void oracle_set_friction(const OracleFriction *f) { g_friction = *f; }

void oracle_apply_friction(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    if (!g_friction.enabled) return;
    double re_st = cfg->influence_radius_st;
    double l0 = cfg->particle_distance;
    double theta_s = cfg->wetting_angle_SL * M_PI / 180.0;
    double delta_th = g_friction.delta_theta * M_PI / 180.0;
    double v_c = g_friction.velocity_threshold;
    double alpha = g_friction.alpha;
    double nu = cfg->viscosity;
    double dyn_coeff = alpha * nu * 2.0 * D / (ps->n0 * ps->lambda);
    double re_n = cfg->influence_radius_n;
    double surf_thr = cfg->surface_threshold;
    for (int i = 0; i < ps->num; i++) {
        Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        double n_fluid = 0.0, r2_star = 1.0e30;
        int j_star = -1;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            double r2 = dist2(pi->pos, ps->particles[j].pos);
            if (ps->particles[j].type == MPS_FLUID) {
                if (r2 < re_n * re_n) n_fluid += KW(sqrt(r2), re_n);
            } else if (ps->particles[j].type == MPS_WALL) {
                if (r2 < re_st * re_st && r2 < r2_star) { r2_star = r2; j_star = j; }
            }
        }
        if (j_star < 0) continue;
        if (n_fluid >= surf_thr * ps->n0) continue;
        const Particle *ps_ = &ps->particles[j_star];
        double n_w[D] = {0.0, 0.0, 0.0};
        for (int k = 0; k < nl->count[j_star]; k++) {
            int m = NB(nl, j_star, k);
            if (ps->particles[m].type != MPS_WALL) continue;
            double dr[D], r2 = 0.0;
            for (int d = 0; d < D; d++) {
                dr[d] = ps_->pos[d] - ps->particles[m].pos[d];
                r2 += dr[d] * dr[d];
            }
            double r = sqrt(r2);
            if (r < 1.0e-9 * l0) continue;
            double w = KW(r, re_st);
            for (int d = 0; d < D; d++) n_w[d] += w * dr[d] / r;
        }
        double n_w_mag = 0.0;
        for (int d = 0; d < D; d++) n_w_mag += n_w[d] * n_w[d];
        n_w_mag = sqrt(n_w_mag);
        if (n_w_mag < 1.0e-9) continue;
        for (int d = 0; d < D; d++) n_w[d] /= n_w_mag;
        double n_lv[D] = {0.0, 0.0, 0.0};
        int fluid_count = 0;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            if (ps->particles[j].type != MPS_FLUID) continue;
            double dr[D];
            double r = sqrt(dist2_vec(pi->pos, ps->particles[j].pos, dr));
            if (r < 1.0e-9 * l0) continue;
            double w = KW(r, re_st);
            for (int d = 0; d < D; d++) n_lv[d] -= w * dr[d] / r;
            fluid_count++;
        }
        if (fluid_count == 0) continue;
        double n_lv_mag = 0.0;
        for (int d = 0; d < D; d++) n_lv_mag += n_lv[d] * n_lv[d];
        n_lv_mag = sqrt(n_lv_mag);
        if (n_lv_mag < 1.0e-9) continue;
        for (int d = 0; d < D; d++) n_lv[d] /= n_lv_mag;
        double cos_th = 0.0;
        for (int d = 0; d < D; d++) cos_th -= n_w[d] * n_lv[d];
        cos_th = fmax(-1.0, fmin(1.0, cos_th));
        double theta_i = acos(cos_th);
        double dot_lv_w = 0.0;
        for (int d = 0; d < D; d++) dot_lv_w += n_lv[d] * n_w[d];
        double e_slide[D], e_slide_mag = 0.0;
        for (int d = 0; d < D; d++) {
            e_slide[d] = n_lv[d] - dot_lv_w * n_w[d];
            e_slide_mag += e_slide[d] * e_slide[d];
        }
        e_slide_mag = sqrt(e_slide_mag);
        if (e_slide_mag < 1.0e-9) continue;
        for (int d = 0; d < D; d++) e_slide[d] /= e_slide_mag;
        double v2 = 0.0;
        for (int d = 0; d < D; d++) v2 += pi->vel[d] * pi->vel[d];
        if (sqrt(v2) <= v_c) {
            if (fabs(theta_i - theta_s) <= delta_th)
                for (int d = 0; d < D; d++) pi->vel[d] = 0.0;
        } else {
            double sum_w_wall = 0.0;
            for (int k = 0; k < nl->count[i]; k++) {
                int j = NB(nl, i, k);
                if (ps->particles[j].type != MPS_WALL) continue;
                double r = sqrt(dist2(pi->pos, ps->particles[j].pos));
                if (r < 1.0e-9 * l0) continue;
                sum_w_wall += KW(r, re_st);
            }
            double v_n = 0.0;
            for (int d = 0; d < D; d++) v_n += pi->vel[d] * e_slide[d];
            double dv_n = -dyn_coeff * cfg->dt * sum_w_wall * v_n;
            if (dv_n > v_n) dv_n = v_n;
            if (dv_n < -v_n) dv_n = -v_n;
            for (int d = 0; d < D; d++) pi->vel[d] += dv_n * e_slide[d];
        }
    }
}
#endif

void oracle_viscosity(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    double re = cfg->influence_radius_lap;
    double coeff = 2.0 * D / (ps->n0 * ps->lambda);
    double nu = cfg->viscosity;
    for (int i = 0; i < ps->num; i++) {
        Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        double lap[D];
        for (int d = 0; d < D; d++) lap[d] = 0.0;
        for (int k = 0; k < nl->count[i]; k++) {
            const Particle *pj = &ps->particles[NB(nl, i, k)];
            double w = KW(sqrt(dist2(pi->pos, pj->pos)), re);
            for (int d = 0; d < D; d++) lap[d] += (pj->vel[d] - pi->vel[d]) * w;
        }
        for (int d = 0; d < D; d++) pi->acc[d] += nu * coeff * lap[d];
    }
}

/* 3P operators.c:102-181: two passes, P_min then the gradient. */
int oracle_pressure_gradient(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    int n = ps->num, mode = cfg->cmps_gradient;
    double re = cfg->influence_radius_lap;
    double gcoef = (double)D / ps->n0;
    double l0 = cfg->particle_distance, rho = cfg->density;
    double *pmin = NULL;
    if (mode != 2) {
        pmin = (double *)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        if (!pmin) return -1;
        for (int i = 0; i < n; i++) {
            double m = ps->particles[i].pressure;
            for (int k = 0; k < nl->count[i]; k++) {
                double pj = ps->particles[NB(nl, i, k)].pressure;
                if (pj < m) m = pj;
            }
            pmin[i] = m;
        }
    }
    for (int i = 0; i < n; i++) {
        Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        double pim = pmin ? pmin[i] : 0.0;
        double g[D];
        for (int d = 0; d < D; d++) g[d] = 0.0;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            const Particle *pj = &ps->particles[j];
            double dr[D];
            double r2 = dist2_vec(pi->pos, pj->pos, dr);
            if (r2 < l0 * l0 * 1.0e-12) continue;
            double w = KW(sqrt(r2), re);
            double dp;
            if (mode == 1)      dp = pi->pressure + pj->pressure - pim - pmin[j];
            else if (mode == 2) dp = pi->pressure + pj->pressure;
            else                dp = pj->pressure - pim;
            for (int d = 0; d < D; d++) g[d] += dp / r2 * dr[d] * w;
        }
        for (int d = 0; d < D; d++) pi->acc[d] = -gcoef * g[d] / rho;
    }
    free(pmin);
    return 0;
}

/* 3P operators.c:188-199 */
void oracle_clamp_pressure(ParticleSystem *ps)
{
    for (int i = 0; i < ps->num; i++)
        if (ps->particles[i].type == MPS_FLUID && ps->particles[i].pressure < 0.0)
            ps->particles[i].pressure = 0.0;
}

/* 3P operators.c:206-219 */
void oracle_judge_free_surface(ParticleSystem *ps, double threshold)
{
    double lim = threshold * ps->n0;
    for (int i = 0; i < ps->num; i++) {
        Particle *p = &ps->particles[i];
        p->on_surface = (p->type == MPS_FLUID && p->n < lim) ? 1 : 0;
    }
}

/* 3P operators.c:226-246 */
void oracle_neighbor_count(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    double re2 = cfg->influence_radius_n * cfg->influence_radius_n;
    for (int i = 0; i < ps->num; i++) {
        int c = 0;
        for (int k = 0; k < nl->count[i]; k++)
            if (dist2(ps->particles[i].pos, ps->particles[NB(nl, i, k)].pos) < re2) c++;
        ps->particles[i].neighbor_count = c;
    }
}

/* 3P operators.c:253-267 */
void oracle_judge_free_surface_by_count(ParticleSystem *ps, double beta)
{
    double lim = beta * ps->n0_count;
    for (int i = 0; i < ps->num; i++) {
        Particle *p = &ps->particles[i];
        p->on_surface = (p->type == MPS_FLUID && p->neighbor_count < lim) ? 1 : 0;
    }
}

/* Impulse of one candidate partner on v_i (3P operators.c:407-427). */
static inline void collide_with(double *vi, const Particle *pi, const Particle *pj,
                                double col2, double l0, double half1pe)
{
    double dr[D];
    double r2 = dist2_vec(pi->pos, pj->pos, dr);
    if (r2 >= col2) return;
    double r = sqrt(r2);
    if (r < 1.0e-12 * l0) return;
    double vn = 0.0;
    for (int d = 0; d < D; d++) vn += (vi[d] - pj->vel[d]) * (dr[d] / r);
    if (vn <= 0.0) return;
    double imp = half1pe * vn;
    for (int d = 0; d < D; d++) vi[d] -= imp * (dr[d] / r);
}

/* 3-D: partners from the (previous step's) neighbour list, 3P operators.c:371-446.
 * 2-D: partners from all particles in index order, 2D operators.c:324-392. */
int oracle_collision(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    int n = ps->num;
    double l0 = cfg->particle_distance;
    double cd = cfg->collision_distance_ratio * l0;
    double col2 = cd * cd, dt = cfg->dt;
    double half1pe = (1.0 + cfg->restitution_coeff) * 0.5;
    double *after = (double *)malloc(sizeof(double) * D * (size_t)(n > 0 ? n : 1));
    if (!after) return -1;
    for (int i = 0; i < n; i++)
        for (int d = 0; d < D; d++) after[(size_t)i * D + d] = ps->particles[i].vel[d];
    for (int i = 0; i < n; i++) {
        const Particle *pi = &ps->particles[i];
        if (pi->type != MPS_FLUID) continue;
        double vi[D];
        for (int d = 0; d < D; d++) vi[d] = pi->vel[d];
#if D == 3
        (void)0;
        for (int k = 0; k < nl->count[i]; k++) {
            const Particle *pj = &ps->particles[NB(nl, i, k)];
            if (pj->type == MPS_GHOST) continue;
            collide_with(vi, pi, pj, col2, l0, half1pe);
        }
#else
        (void)nl;
        for (int j = 0; j < n; j++) {
            if (j == i || ps->particles[j].type == MPS_GHOST) continue;
            collide_with(vi, pi, &ps->particles[j], col2, l0, half1pe);
        }
#endif
        for (int d = 0; d < D; d++) after[(size_t)i * D + d] = vi[d];
    }
    for (int i = 0; i < n; i++) {
        Particle *p = &ps->particles[i];
        if (p->type != MPS_FLUID) continue;
        for (int d = 0; d < D; d++) {
            double va = after[(size_t)i * D + d];
            double dv = va - p->vel[d];
            p->pos[d] += dt * dv;
            p->vel[d] = va;
        }
    }
    free(after);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Pressure Poisson equation (3P pressure_solver.c; 2D dense variant)  */
/* ------------------------------------------------------------------ */

static inline int is_unknown(const Particle *p)
{
    return (p->type == MPS_FLUID && !p->on_surface) || p->type == MPS_WALL;
}

/* 3P pressure_solver.c:342-362 (high-order source term) */
static double source_hs(const ParticleSystem *ps, const NeighborList *nl, int i,
                        double re, const SimConfig *cfg)
{
    const Particle *pi = &ps->particles[i];
    double s = 0.0;
    for (int k = 0; k < nl->count[i]; k++) {
        const Particle *pj = &ps->particles[NB(nl, i, k)];
        if (pj->type == MPS_DUMMY) continue;
        double dr[D];
        double r2 = dist2_vec(pi->pos, pj->pos, dr);
        if (r2 < 1.0e-24) continue;
        double r = sqrt(r2);
        double dv = 0.0;
        for (int d = 0; d < D; d++) dv += dr[d] * (pj->vel[d] - pi->vel[d]);
        s += re / (r * r * r) * dv;
    }
    return -(cfg->density / ps->n0 / cfg->dt) * s;
}

/* 3P pressure_solver.c:381-409 (velocity divergence for ppe_type 1) */
static double vel_divergence(const ParticleSystem *ps, const NeighborList *nl, int i,
                             double re, const SimConfig *cfg)
{
    const Particle *pi = &ps->particles[i];
    double s = 0.0;
    for (int k = 0; k < nl->count[i]; k++) {
        const Particle *pj = &ps->particles[NB(nl, i, k)];
        if (pj->type == MPS_DUMMY) continue;
        double dr[D];
        double r2 = dist2_vec(pi->pos, pj->pos, dr);
        if (r2 < 1.0e-24) continue;
        double dv = 0.0;
        for (int d = 0; d < D; d++) dv += (pj->vel[d] - pi->vel[d]) * dr[d];
        s += dv / r2 * KW(sqrt(r2), re);
    }
    return (double)D / ps->n0 * s;
}

/* Right-hand side of one unknown row, 3P pressure_solver.c:328-340,524-529. */
static double ppe_rhs(const ParticleSystem *ps, const NeighborList *nl, int i,
                      double re, const SimConfig *cfg)
{
    const Particle *p = &ps->particles[i];
    double n0 = ps->n0, dt = cfg->dt, dt2 = dt * dt;
    if (p->type == MPS_WALL) return 0.0;
    if (cfg->hs_mode == 1) return source_hs(ps, nl, i, re, cfg);
    if (cfg->ppe_type == 1) {
        double div = (p->type == MPS_FLUID) ? vel_divergence(ps, nl, i, re, cfg) : 0.0;
        return -cfg->density / dt * div
               + cfg->gamma_ppe * (cfg->density / dt2) * (p->n - n0) / n0;
    }
    return cfg->relaxation_coeff * (cfg->density / dt2) * (p->n - n0) / n0;
}

int oracle_assemble_ppe(const ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg,
                        int *eq_idx, int *row_ptr, int *col_idx, double *val, double *b,
                        long long *nnz_out)
{
    int n = ps->num;
    double re = cfg->influence_radius_lap;
    double coeff = 2.0 * D / (ps->n0 * ps->lambda);
    int n_eq = 0;
    /* 3P pressure_solver.c:411-422: unknowns numbered in particle order. */
    for (int i = 0; i < n; i++) eq_idx[i] = is_unknown(&ps->particles[i]) ? n_eq++ : -1;

    long long nnz = 0;
    for (int i = 0; i < n; i++) {
        if (eq_idx[i] < 0) continue;
        nnz += 1;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            if (ps->particles[j].type == MPS_DUMMY) continue;
            if (eq_idx[j] >= 0) nnz++;
        }
    }
    if (nnz_out) *nnz_out = nnz;
    if (!row_ptr) return n_eq;

    /* 3P pressure_solver.c:437-530: off-diagonals in list order, diagonal
     * last, then the per-row insertion sort of :536-551. */
    long long pos = 0;
    row_ptr[0] = 0;
    for (int i = 0; i < n; i++) {
        int e = eq_idx[i];
        if (e < 0) continue;
        const Particle *pi = &ps->particles[i];
        long long lo = pos;
        double sum_w = 0.0;
        for (int k = 0; k < nl->count[i]; k++) {
            int j = NB(nl, i, k);
            const Particle *pj = &ps->particles[j];
            if (pj->type == MPS_DUMMY) continue;
            double w = KW(sqrt(dist2(pi->pos, pj->pos)), re);
            sum_w += w;
            if (eq_idx[j] >= 0) { col_idx[pos] = eq_idx[j]; val[pos] = -coeff * w; pos++; }
        }
        double dv = (cfg->ppe_type == 1) ? cfg->c_ppe * coeff * sum_w : coeff * sum_w;
        col_idx[pos] = e; val[pos] = dv; pos++;
        for (long long p = lo + 1; p < pos; p++) {
            int c = col_idx[p];
            double v = val[p];
            long long q = p - 1;
            while (q >= lo && col_idx[q] > c) { col_idx[q + 1] = col_idx[q]; val[q + 1] = val[q]; q--; }
            col_idx[q + 1] = c; val[q + 1] = v;
        }
        row_ptr[e + 1] = (int)pos;
        b[e] = ppe_rhs(ps, nl, i, re, cfg);
    }
    return n_eq;
}

/* Sequential dot product, 3P pressure_solver.c:79-84. */
static double vdot(const double *a, const double *b, int n)
{
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

typedef struct { int n; const int *rp; const int *ci; const double *v; } Csr;

static void csr_apply(const Csr *A, const double *x, double *y)
{
    for (int i = 0; i < A->n; i++) {
        double s = 0.0;
        for (int p = A->rp[i]; p < A->rp[i + 1]; p++) s += A->v[p] * x[A->ci[p]];
        y[i] = s;
    }
}

/* 3P pressure_solver.c:90-131 */
static int cg_sparse(const Csr *A, double *x, const double *b, int maxit, double tol)
{
    int n = A->n;
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n),
           *Ap = malloc(sizeof(double) * n);
    if (!r || !p || !Ap) { free(r); free(p); free(Ap); return 0; }
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    memcpy(p, r, sizeof(double) * n);
    double rr = vdot(r, r, n);
    int it;
    for (it = 0; it < maxit; it++) {
        if (sqrt(rr) < tol) break;
        csr_apply(A, p, Ap);
        double pAp = vdot(p, Ap, n);
        if (fabs(pAp) < 1.0e-30) break;
        double alpha = rr / pAp;
        for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        double rr_new = vdot(r, r, n);
        if (rr < 1.0e-60) break;
        double beta = rr_new / rr;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
        rr = rr_new;
    }
    g_last_resid = sqrt(rr);
    free(r); free(p); free(Ap);
    return it;
}

/* IC(0) on the strictly-lower pattern of A, 3P pressure_solver.c:156-232. */
typedef struct { int n; int *rp; int *ci; double *v; double *dinv; } Lfac;

static void lfac_free(Lfac *L)
{
    free(L->rp); free(L->ci); free(L->v); free(L->dinv);
}

static int ic0_factor(const Csr *A, const double *diag, Lfac *L)
{
    int n = A->n;
    long long m = 0;
    for (int i = 0; i < n; i++)
        for (int p = A->rp[i]; p < A->rp[i + 1]; p++) if (A->ci[p] < i) m++;
    L->n = n;
    L->rp = malloc(sizeof(int) * (size_t)(n + 1));
    L->ci = malloc(sizeof(int) * (size_t)(m + 1));
    L->v = calloc((size_t)(m + 1), sizeof(double));
    L->dinv = malloc(sizeof(double) * (size_t)n);
    if (!L->rp || !L->ci || !L->v || !L->dinv) { lfac_free(L); return -1; }
    L->rp[0] = 0;
    for (int i = 0; i < n; i++) {
        int q = L->rp[i];
        for (int p = A->rp[i]; p < A->rp[i + 1]; p++)
            if (A->ci[p] < i) { L->ci[q] = A->ci[p]; L->v[q] = A->v[p]; q++; }
        L->rp[i + 1] = q;
    }
    for (int k = 0; k < n; k++) {
        double d = diag[k];
        for (int p = L->rp[k]; p < L->rp[k + 1]; p++) d -= L->v[p] * L->v[p];
        if (d <= 0.0) d = (diag[k] > 0.0) ? diag[k] : 1.0e-30;
        L->dinv[k] = 1.0 / sqrt(d);
        for (int pk = A->rp[k]; pk < A->rp[k + 1]; pk++) {
            int i = A->ci[pk];
            if (i <= k) continue;
            double s = A->v[pk];
            int a = L->rp[i], ae = L->rp[i + 1], c = L->rp[k], ce = L->rp[k + 1];
            while (a < ae && c < ce) {
                int ja = L->ci[a], jc = L->ci[c];
                if (ja < jc) a++;
                else if (ja > jc) c++;
                else { s -= L->v[a] * L->v[c]; a++; c++; }
            }
            for (int p = L->rp[i]; p < L->rp[i + 1] && L->ci[p] <= k; p++)
                if (L->ci[p] == k) { L->v[p] = s * L->dinv[k]; break; }
        }
    }
    return 0;
}

/* IC(0) of a CSR matrix (sorted columns, diagonal included) in its own row
 * order, the algorithm of pressure_solver.c:156-232 (ic0_factor above) on
 * whatever unknown numbering the caller gives: here the GPU solver's block
 * colour order.  F receives the factor in A's pattern as that solver stores
 * it: L_ij below the diagonal, 1/L_ii on it, L_ji above it.  0, -1 on OOM. */
int oracle_ic0_csr(int n, const int *rp, const int *ci, const double *v, double *F)
{
    Csr A = {n, rp, ci, v};
    double *diag = calloc((size_t)(n + 1), sizeof(double));
    if (!diag) return -1;
    for (int i = 0; i < n; i++) {
        for (int p = rp[i]; p < rp[i + 1]; p++) if (ci[p] == i) diag[i] = v[p];
    }
    Lfac L;
    if (ic0_factor(&A, diag, &L) != 0) { free(diag); return -1; }
    for (int i = 0; i < n; i++) {
        int q = L.rp[i];
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            int j = ci[p];
            if (j < i) F[p] = L.v[q++];
            else if (j == i) F[p] = L.dinv[i];
            else {
                /* L_ji: row j's lower entry in column i */
                int lo = L.rp[j], hi = L.rp[j + 1];
                double f = 0.0;
                while (lo < hi) {
                    int mid = (lo + hi) / 2;
                    if (L.ci[mid] == i) { f = L.v[mid]; break; }
                    if (L.ci[mid] < i) lo = mid + 1; else hi = mid;
                }
                F[p] = f;
            }
        }
    }
    lfac_free(&L);
    free(diag);
    return 0;
}

/* The inverse of each cell's diagonal block of L, the factor F in the
 * solver's convention: cells[2k] = first row r0, cells[2k+1] = unknowns m;
 * column-major lower triangle at inv + inv_off[k]: X_ij (i >= j) at
 * j*m - j*(j-1)/2 + (i - j), by forward substitution column by column,
 * X_ic = (delta_ic - sum_{c <= k < i} L_ik X_kc) / L_ii.  Cells above
 * max_m unknowns are skipped. */
void oracle_cell_inverses(int ncells, const int *cells, const int *inv_off, const int *rp, const int *ci,
                          const double *F, int max_m, double *inv)
{
    for (int k = 0; k < ncells; k++) {
        int r0 = cells[2 * k], m = cells[2 * k + 1];
        if (m > max_m) continue;
        double *X = inv + inv_off[k];
        double *Ld = malloc(sizeof(double) * (size_t)m * (size_t)m);
        if (!Ld) return;
        for (int i = 0; i < m * m; i++) Ld[i] = 0.0;
        for (int i = 0; i < m; i++)
            for (int p = rp[r0 + i]; p < rp[r0 + i + 1]; p++) {
                int j = ci[p] - r0;
                if (j >= 0 && j < i) Ld[i * m + j] = F[p];
                if (j == i) Ld[i * m + i] = F[p];   /* 1 / L_ii */
            }
        for (int c = 0; c < m; c++) {
            int off = c * m - (c * (c - 1)) / 2;
            for (int i = c; i < m; i++) {
                double s = (i == c) ? 1.0 : 0.0;
                for (int kk = c; kk < i; kk++) s -= Ld[i * m + kk] * X[off + kk - c];
                X[off + i - c] = s * Ld[i * m + i];
            }
        }
        free(Ld);
    }
}

/* z = (L L^T)^-1 r with the factor F in the solver's convention: forward
 * L y = r over the lower entries, backward L^T z = y over the upper copy
 * (the sweeps of pressure_solver.c:235-255). */
void oracle_ic0_apply_csr(int n, const int *rp, const int *ci, const double *F, const double *r, double *z)
{
    double *y = malloc(sizeof(double) * (size_t)(n + 1));
    if (!y) return;
    for (int i = 0; i < n; i++) {
        double s = r[i], d = 0.0;
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            if (ci[p] < i) s -= F[p] * y[ci[p]];
            else if (ci[p] == i) d = F[p];
        }
        y[i] = s * d;
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = y[i], d = 0.0;
        for (int p = rp[i]; p < rp[i + 1]; p++) {
            if (ci[p] > i) s -= F[p] * z[ci[p]];
            else if (ci[p] == i) d = F[p];
        }
        z[i] = s * d;
    }
    free(y);
}

/* Forward L y = r and backward L^T z = y (scatter form), 3P :235-255. */
static void ic0_apply(const Lfac *L, const double *r, double *tmp, double *z)
{
    int n = L->n;
    for (int i = 0; i < n; i++) {
        double s = r[i];
        for (int p = L->rp[i]; p < L->rp[i + 1]; p++) s -= L->v[p] * tmp[L->ci[p]];
        tmp[i] = s * L->dinv[i];
    }
    for (int i = 0; i < n; i++) z[i] = tmp[i];
    for (int i = n - 1; i >= 0; i--) {
        z[i] *= L->dinv[i];
        for (int p = L->rp[i]; p < L->rp[i + 1]; p++) z[L->ci[p]] -= L->v[p] * z[i];
    }
}

/* 3P pressure_solver.c:261-322; note the breakdown guard tests the OLD rz. */
static int iccg_sparse(const Csr *A, const double *diag, double *x, const double *b,
                       int maxit, double tol)
{
    int n = A->n;
    Lfac L;
    if (ic0_factor(A, diag, &L) != 0) return cg_sparse(A, x, b, maxit, tol);
    double *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n),
           *p = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n),
           *t = malloc(sizeof(double) * n);
    if (!r || !z || !p || !Ap || !t) {
        free(r); free(z); free(p); free(Ap); free(t); lfac_free(&L);
        return cg_sparse(A, x, b, maxit, tol);
    }
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    ic0_apply(&L, r, t, z);
    memcpy(p, z, sizeof(double) * n);
    double rz = vdot(r, z, n);
    double rn = 0.0;
    int it;
    for (it = 0; it < maxit; it++) {
        rn = sqrt(vdot(r, r, n));
        if (rn < tol) break;
        csr_apply(A, p, Ap);
        double pAp = vdot(p, Ap, n);
        if (fabs(pAp) < 1.0e-30) break;
        double alpha = rz / pAp;
        for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        ic0_apply(&L, r, t, z);
        double rz_new = vdot(r, z, n);
        if (fabs(rz) < 1.0e-60) break;
        double beta = rz_new / rz;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    g_last_resid = rn;
    free(r); free(z); free(p); free(Ap); free(t); lfac_free(&L);
    return it;
}

#if D == 2
/* Dense PPE solver of the 2-D variant, 2D pressure_solver.c:35-219.  The
 * factor keeps IC(0)'s pattern through the |A| > 0 tests and uses
 * division by L_kk rather than a stored inverse. */
static void dense_matvec(const double *A, const double *x, double *y, int n)
{
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        const double *a = A + (size_t)i * n;
        for (int j = 0; j < n; j++) s += a[j] * x[j];
        y[i] = s;
    }
}

static int dense_cg(const double *A, double *x, const double *b, int n, int maxit, double tol)
{
    double *r = malloc(sizeof(double) * n), *p = malloc(sizeof(double) * n),
           *Ap = malloc(sizeof(double) * n);
    if (!r || !p || !Ap) { free(r); free(p); free(Ap); return 0; }
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    memcpy(p, r, sizeof(double) * n);
    double rr = vdot(r, r, n);
    int it;
    for (it = 0; it < maxit; it++) {
        if (sqrt(rr) < tol) break;
        dense_matvec(A, p, Ap, n);
        double pAp = vdot(p, Ap, n);
        if (fabs(pAp) < 1.0e-30) break;
        double alpha = rr / pAp;
        for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        double rr_new = vdot(r, r, n);
        if (rr < 1.0e-60) break;
        double beta = rr_new / rr;
        for (int i = 0; i < n; i++) p[i] = r[i] + beta * p[i];
        rr = rr_new;
    }
    g_last_resid = sqrt(rr);
    free(r); free(p); free(Ap);
    return it;
}

static void dense_ic(const double *A, double *L, int n)
{
    memset(L, 0, sizeof(double) * (size_t)n * n);
    for (int k = 0; k < n; k++) {
        const double *ak = A + (size_t)k * n;
        double *lk = L + (size_t)k * n;
        double s = 0.0;
        for (int j = 0; j < k; j++) if (fabs(ak[j]) > 0.0) s += lk[j] * lk[j];
        double dg = ak[k] - s;
        if (dg <= 0.0) dg = ak[k] > 0.0 ? ak[k] : 1.0e-30;
        lk[k] = sqrt(dg);
        double inv = 1.0 / lk[k];
        for (int i = k + 1; i < n; i++) {
            const double *ai = A + (size_t)i * n;
            if (fabs(ai[k]) < 1.0e-30) continue;
            double *li = L + (size_t)i * n;
            double t = 0.0;
            for (int j = 0; j < k; j++)
                if (fabs(ai[j]) > 0.0 && fabs(ak[j]) > 0.0) t += li[j] * lk[j];
            li[k] = (ai[k] - t) * inv;
        }
    }
}

static void dense_precond(const double *L, const double *r, double *z, double *w, int n)
{
    for (int i = 0; i < n; i++) {
        const double *li = L + (size_t)i * n;
        double s = 0.0;
        for (int j = 0; j < i; j++) s += li[j] * w[j];
        w[i] = (r[i] - s) / li[i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = 0.0;
        for (int j = i + 1; j < n; j++) s += L[(size_t)j * n + i] * z[j];
        z[i] = (w[i] - s) / L[(size_t)i * n + i];
    }
}

static int dense_iccg(const double *A, double *x, const double *b, int n, int maxit, double tol)
{
    double *L = calloc((size_t)n * n, sizeof(double));
    double *r = malloc(sizeof(double) * n), *z = malloc(sizeof(double) * n),
           *p = malloc(sizeof(double) * n), *Ap = malloc(sizeof(double) * n),
           *w = malloc(sizeof(double) * n);
    if (!L || !r || !z || !p || !Ap || !w) {
        free(L); free(r); free(z); free(p); free(Ap); free(w);
        memset(x, 0, sizeof(double) * n);
        return 0;
    }
    dense_ic(A, L, n);
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    dense_precond(L, r, z, w, n);
    memcpy(p, z, sizeof(double) * n);
    double rz = vdot(r, z, n), rn = 0.0;
    int it;
    for (it = 0; it < maxit; it++) {
        rn = sqrt(vdot(r, r, n));
        if (rn < tol) break;
        dense_matvec(A, p, Ap, n);
        double pAp = vdot(p, Ap, n);
        if (fabs(pAp) < 1.0e-30) break;
        double alpha = rz / pAp;
        for (int i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        dense_precond(L, r, z, w, n);
        double rz_new = vdot(r, z, n);
        if (fabs(rz) < 1.0e-60) break;
        double beta = rz_new / rz;
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
    g_last_resid = rn;
    free(L); free(r); free(z); free(p); free(Ap); free(w);
    return it;
}
#endif

int oracle_solve_pressure(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg)
{
    int n = ps->num;
    int *eq = malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    if (!eq) return -1;
    long long nnz = 0;
    int n_eq = oracle_assemble_ppe(ps, nl, cfg, eq, NULL, NULL, NULL, NULL, &nnz);
    g_last_iters = 0;
    g_last_resid = 0.0;
    if (n_eq == 0) {
        for (int i = 0; i < n; i++) ps->particles[i].pressure = 0.0;
        free(eq);
        return 0;
    }
    int *rp = malloc(sizeof(int) * (size_t)(n_eq + 1));
    int *ci = malloc(sizeof(int) * (size_t)nnz);
    double *v = malloc(sizeof(double) * (size_t)nnz);
    double *b = calloc((size_t)n_eq, sizeof(double));
    double *x = calloc((size_t)n_eq, sizeof(double));
    double *dg = calloc((size_t)n_eq, sizeof(double));
    if (!rp || !ci || !v || !b || !x || !dg) {
        free(eq); free(rp); free(ci); free(v); free(b); free(x); free(dg);
        return -1;
    }
    oracle_assemble_ppe(ps, nl, cfg, eq, rp, ci, v, b, NULL);
    for (int e = 0; e < n_eq; e++)
        for (int p = rp[e]; p < rp[e + 1]; p++) if (ci[p] == e) dg[e] = v[p];

    int it;
#if D == 3
    Csr A = {n_eq, rp, ci, v};
    it = (cfg->solver_type == 1) ? iccg_sparse(&A, dg, x, b, cfg->cg_max_iter, cfg->cg_tolerance)
                                 : cg_sparse(&A, x, b, cfg->cg_max_iter, cfg->cg_tolerance);
#else
    /* The 2-D reference builds a dense n_eq x n_eq matrix (2D :346). */
    double *M = calloc((size_t)n_eq * n_eq, sizeof(double));
    if (!M) {
        free(eq); free(rp); free(ci); free(v); free(b); free(x); free(dg);
        return -1;
    }
    for (int e = 0; e < n_eq; e++)
        for (int p = rp[e]; p < rp[e + 1]; p++) M[(size_t)e * n_eq + ci[p]] = v[p];
    it = (cfg->solver_type == 1) ? dense_iccg(M, x, b, n_eq, cfg->cg_max_iter, cfg->cg_tolerance)
                                 : dense_cg(M, x, b, n_eq, cfg->cg_max_iter, cfg->cg_tolerance);
    free(M);
#endif
    g_last_iters = it;
    for (int i = 0; i < n; i++) ps->particles[i].pressure = (eq[i] >= 0) ? x[eq[i]] : 0.0;
    free(eq); free(rp); free(ci); free(v); free(b); free(x); free(dg);
    return it;
}

/* ------------------------------------------------------------------ */
/* Boundary bookkeeping (3P boundary.c:12-61)                          */
/* ------------------------------------------------------------------ */

void oracle_apply_wall_boundary(ParticleSystem *ps)
{
    for (int i = 0; i < ps->num; i++) {
        Particle *p = &ps->particles[i];
        if (p->type == MPS_WALL || p->type == MPS_GHOST)
            for (int d = 0; d < D; d++) { p->vel[d] = 0.0; p->acc[d] = 0.0; }
    }
}

void oracle_remove_out_of_bounds(ParticleSystem *ps, const SimConfig *cfg)
{
    double m = cfg->particle_distance * (cfg->wall_layers + 1);
    for (int i = 0; i < ps->num; i++) {
        Particle *p = &ps->particles[i];
        if (p->type != MPS_FLUID) continue;
        int out = 0;
        for (int d = 0; d < D; d++) {
            double x = p->pos[d];
            if (x < cfg->domain_min[d] - m || x > cfg->domain_max[d] + m || isnan(x)) out = 1;
        }
        if (out) {
            p->type = MPS_GHOST;
            p->pressure = 0.0;
            p->n = 0.0;
            for (int d = 0; d < D; d++) { p->vel[d] = 0.0; p->acc[d] = 0.0; }
        }
    }
}

/* ------------------------------------------------------------------ */
/* One time step (3P simulation.c:19-118; 2D simulation.c:25-118)      */
/* ------------------------------------------------------------------ */

/* Driven walls (no counterpart in the reference): the phase terms of a wall
 * drive at time t, evaluated with the expressions the GPU engine uses on its
 * host, so both produce the same bits. */
void oracle_wall_drive_terms(double amp, double freq, double t, double *dx, double *vel)
{
    double w = 2.0 * 3.14159265358979323846 * freq;
    double ph = w * t;
    *dx = amp * sin(ph);
    *vel = amp * w * cos(ph);
}

int oracle_step(ParticleSystem *ps, NeighborList *nl, CellList *cl, const SimConfig *cfg)
{
    return oracle_step_driven(ps, nl, cl, cfg, NULL, 0.0, 0.0, 0, 0);
}

/* oracle_step with driven walls: after the explicit update every WALL and
 * DUMMY particle is put at rest[i] + A sin(2 pi f t1) along `axis` with the
 * matching velocity (t1 = (step + 1) dt, the time at the end of the step),
 * and the wall boundary keeps that velocity instead of zeroing it.  amp = 0
 * is oracle_step. */
int oracle_step_driven(ParticleSystem *ps, NeighborList *nl, CellList *cl, const SimConfig *cfg,
                       const double *rest, double amp, double freq, int axis, int step)
{
    double re = fmax(cfg->influence_radius_lap, cfg->influence_radius_n);
    if (cfg->surface_tension_enabled) re = fmax(re, cfg->influence_radius_st);
    double dt = cfg->dt;
    int n = ps->num;

    for (int i = 0; i < n; i++) {
        Particle *p = &ps->particles[i];
        for (int d = 0; d < D; d++) p->acc[d] = (p->type == MPS_FLUID) ? cfg->gravity[d] : 0.0;
    }
    oracle_viscosity(ps, nl, cfg);
    if (cfg->surface_tension_enabled) {
        oracle_surface_tension(ps, nl, cfg);
        oracle_surface_tension_SL(ps, nl, cfg);
    }
    for (int i = 0; i < n; i++) {
        Particle *p = &ps->particles[i];
        if (p->type != MPS_FLUID) continue;
        for (int d = 0; d < D; d++) p->vel[d] += dt * p->acc[d];
    }
#if D == 3
    oracle_apply_friction(ps, nl, cfg);   /* 3S simulation.c:52-53 */
#endif
    for (int i = 0; i < n; i++) {
        Particle *p = &ps->particles[i];
        if (p->type != MPS_FLUID) continue;
        for (int d = 0; d < D; d++) p->pos[d] += dt * p->vel[d];
    }
    int driven = amp != 0.0 && rest != NULL;
    if (driven) {
        double dx, vel;
        oracle_wall_drive_terms(amp, freq, (double)(step + 1) * dt, &dx, &vel);
        for (int i = 0; i < n; i++) {
            Particle *p = &ps->particles[i];
            if (p->type != MPS_WALL && p->type != MPS_DUMMY) continue;
            p->pos[axis] = rest[i] + dx;
            for (int d = 0; d < D; d++) p->vel[d] = 0.0;
            p->vel[axis] = vel;
        }
    }
#if D == 3
    if (cfg->collision_distance_ratio > 0.0)
#endif
        if (oracle_collision(ps, nl, cfg) != 0) return -1;

    int rc = oracle_neighbor_search(nl, ps, cl, re);
    if (rc != 0) return rc;
    oracle_number_density(ps, nl, cfg);
    if (cfg->surface_detection_method == 1) {
        oracle_neighbor_count(ps, nl, cfg);
        oracle_judge_free_surface_by_count(ps, cfg->surface_count_threshold);
    } else {
        oracle_judge_free_surface(ps, cfg->surface_threshold);
    }
    if (oracle_solve_pressure(ps, nl, cfg) < 0) return -1;
    if (cfg->clamp_negative_pressure) oracle_clamp_pressure(ps);
    if (oracle_pressure_gradient(ps, nl, cfg) != 0) return -1;
    for (int i = 0; i < n; i++) {
        Particle *p = &ps->particles[i];
        if (p->type != MPS_FLUID) continue;
        for (int d = 0; d < D; d++) {
            double du = dt * p->acc[d];
            p->vel[d] += du;
            p->pos[d] += dt * du;
        }
    }
    if (driven) {
        for (int i = 0; i < n; i++) {
            Particle *p = &ps->particles[i];
            if (p->type == MPS_GHOST)
                for (int d = 0; d < D; d++) { p->vel[d] = 0.0; p->acc[d] = 0.0; }
            else if (p->type == MPS_WALL)
                for (int d = 0; d < D; d++) p->acc[d] = 0.0;
        }
    } else {
        oracle_apply_wall_boundary(ps);
    }
    oracle_remove_out_of_bounds(ps, cfg);
    return 0;
}
