/*
 * mps_b200.h -- C ABI of the B200 (sm_100a) MPS time-step library.
 *
 * Two layers, both plain C (pointers, sizes, status codes; no torch types):
 *
 *  1. The session API below (mps_*).  A session owns one device-resident
 *     particle system on the current CUDA device and runs the whole time
 *     step there.  It takes a dimension-independent parameter struct.
 *
 *  2. The drop-in API (include/mps_dropin.h): the reference solver's own
 *     function names and structs, implemented over the session API and built
 *     per dimension into libmps3d.so / libmps2d.so.
 *
 * Every entry point returns MPS_OK (0) or a negative MPS_ERR_* code; the
 * reference's exit(1) / silent-return failure modes become codes here.
 */
#ifndef MPS_B200_H
#define MPS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPS_OK                      0
#define MPS_ERR_INVALID           (-1)  /* bad argument or state */
#define MPS_ERR_CUDA              (-2)  /* a CUDA call failed */
#define MPS_ERR_OOM               (-3)  /* device allocation failed */
#define MPS_ERR_NEIGHBOR_OVERFLOW (-4)  /* a particle has more than max_neighbors
                                           (reference: neighbor_search.c:221-228 exit) */
#define MPS_ERR_UNSUPPORTED       (-5)  /* switch outside the implemented path */
#define MPS_ERR_NOT_CONVERGED     (-6)  /* reported, never raised by default */
#define MPS_ERR_NAN               (-7)

/* Precision forms of the step. */
#define MPS_PREC_FP64  0   /* the reference's arithmetic, FP64 everywhere */
#define MPS_PREC_MIXED 1   /* PPE matrix and IC(0) factor stored in FP32 (SpMV in difference
                              form), FP64 vectors, dot products, refinement residuals and
                              everything outside the PPE solve; the adjoint PPE solve too */

/* PPE unknown orderings for the IC(0) preconditioner. */
#define MPS_ORDER_BLOCK_COLOR 0  /* cells as blocks, 2^dim colours (default) */

/* Simulation parameters, the hot-path subset of the reference SimConfig
 * (mps_fluid3D_parallel/include/sim_config.h:10-78) with radii already
 * derived (re = ratio * l0) and fixed 3-element vectors for both dims. */
typedef struct {
    int    dim;                       /* 2 or 3 */
    double particle_distance;         /* l0 */
    double influence_radius_lap;
    double influence_radius_n;
    int    max_neighbors;
    int    wall_layers;
    double density;
    double viscosity;
    double gravity[3];
    double dt;
    int    solver_type;               /* 0: CG, 1: ICCG */
    int    cg_max_iter;
    double cg_tolerance;
    double relaxation_coeff;
    int    clamp_negative_pressure;
    int    ppe_type;
    double c_ppe;
    double gamma_ppe;
    double surface_threshold;
    int    surface_detection_method;
    double surface_count_threshold;
    double restitution_coeff;
    double collision_distance_ratio;
    int    surface_tension_enabled;   /* potential-force surface tension (operators.c:281-354); its
                                         radius, coefficient and contact angle are at the end */
    double domain_min[3];
    double domain_max[3];
    int    cmps_gradient;
    int    use_analytical_lambda;
    int    hs_mode;
    int    precision;                 /* MPS_PREC_* */
    double refine_tolerance;          /* mixed form: stop at ||b - A x|| <= max(cg_tolerance,
                                         refine_tolerance * ||b||, 4 u || |b| + |A| |x| ||),
                                         u = 2^-53: the last term is where FP64 residuals
                                         bottom out (0: that term alone decides) */
    /* Driven walls (no counterpart in the reference, whose walls never move):
     * every WALL and DUMMY particle follows x_axis = rest + A sin(2 pi f t),
     * u_axis = 2 pi f A cos(2 pi f t), rest = its position at upload, t the
     * session time (steps taken x dt).  A = 0 is the reference's fixed walls,
     * bit for bit. */
    double wall_drive_amp;            /* A (m) */
    double wall_drive_freq;           /* f (Hz) */
    int    wall_drive_axis;           /* 0 = x, 1 = y, 2 = z */
    /* Surface tension (sim_config.h: influence_radius_st = re_ratio * l0,
     * surface_tension_coeff sigma, wetting_angle_SL theta in degrees); read
     * only when surface_tension_enabled.  The list radius then includes
     * influence_radius_st, as simulation.c:22-24 does. */
    double influence_radius_st;
    double surface_tension_coeff;
    double wetting_angle_SL;
    /* Hybrid contact-line friction of the 3-D serial variant
     * (mps_fluid3D/src/operators.c:337-492; 3-D only): static below the
     * velocity threshold (m/s) within delta_theta (degrees) of the contact
     * angle wetting_angle_SL, dynamic damping with alpha above it. */
    int    friction_enabled;
    double friction_delta_theta;
    double dynamic_friction_alpha;
    double friction_velocity_threshold;
} mps_params_t;

/* Per-step metrics (the reference computes and discards its iteration count,
 * pressure_solver.c:553-561). */
typedef struct {
    int    ppe_iterations;            /* CG iterations of the last step (inner, summed) */
    int    ppe_outer;                 /* reliable updates (mixed form), else 1 */
    double ppe_residual;              /* final recursive residual norm */
    int    n_eq;
    long long nnz;
    int    n_fluid;
    int    n_ghost;
    int    converged;
    long long total_iterations;       /* over the session */
    long long total_steps;
    double ms_ops;                    /* device time of the last step outside the PPE */
    double ms_assembly;
    double ms_factor;
    double ms_solve;
    /* Per-kernel device time summed over the session while profiling is on
     * (mps_set_profiling): the SpMV of the CG loop, the forward and backward
     * colour sweeps of the IC(0) preconditioner, and the CG vector kernels;
     * only iterations that did work are counted. */
    double prof_spmv_ms;
    long long prof_spmv_launches;
    double prof_fwd_ms;
    long long prof_fwd_sweeps;
    double prof_bwd_ms;
    long long prof_bwd_sweeps;
    double prof_vec_ms;
    long long prof_iterations;
    long long prof_nnz_sum;           /* sum over profiled iterations of nnz */
    long long prof_rows_sum;          /* sum over profiled iterations of n_eq */
    /* The last step's PPE solution x against its FP64 matrix and right-hand
     * side, in both precision forms: ||b - A x||_2 (the true residual, which
     * the CG loop's recursive residual stops tracking once rounding
     * dominates), ||b||_2, and the FP64 rounding floor of that residual,
     * u || |b| + |A| |x| ||_2 with u = 2^-53. */
    double ppe_true_residual;
    double ppe_bnorm;
    double ppe_rounding_floor;
    /* Sizes of the last step's IC(0) sweep data: cross-cell entries of the
     * factor read by the forward and the backward sweep, and the entries of
     * the in-cell block inverses (read once per sweep). */
    long long sweep_cross_lo;
    long long sweep_cross_up;
    long long sweep_inverse_entries;
    /* Device time of the persistent ICCG kernel (one cooperative launch per
     * batch of CG iterations) summed over the session while profiling is
     * on, its launches and the iterations they ran. */
    double prof_pcg_ms;
    long long prof_pcg_launches;
    long long prof_pcg_iterations;
} mps_metrics_t;

typedef struct mps_session mps_session;

int  mps_version(void);
const char *mps_error_string(int code);

/* Lifetime.  Creates device buffers for up to `capacity` particles on the
 * current CUDA device (cudaSetDevice beforehand picks the GPU). */
int  mps_session_create(mps_session **out, const mps_params_t *params, int capacity);
int  mps_session_destroy(mps_session *s);
/* Replace the parameters (a changed domain or radius rebuilds the grid and
 * requires a new neighbour search). */
int  mps_update_params(mps_session *s, const mps_params_t *params);
/* Select the precision form, MPS_PREC_FP64 or MPS_PREC_MIXED, from the next
 * step on, every other parameter kept; MPS_ERR_INVALID for any other value.
 * No counterpart in the reference, whose solver is FP64 only. */
int  mps_set_precision(mps_session *s, int precision);
/* Human-readable detail of the session's last failure. */
const char *mps_last_error(mps_session *s);

/* State transfer in the reference's particle order.  `particles` points at
 * `num` AoS Particle records of the session's dimension (104 bytes each in
 * 3-D, 80 in 2-D; include/mps_types.h).  Upload replaces the state; download
 * writes pos, vel, acc, pressure, n, neighbor_count, type and on_surface. */
int  mps_upload_particles(mps_session *s, const void *particles, int num);
int  mps_download_particles(mps_session *s, void *particles, int num);
/* SoA transfer of positions/velocities/types only (host arrays of num*dim
 * doubles, particle-major). */
int  mps_upload_soa(mps_session *s, const double *pos, const double *vel, const int *type, int num);
int  mps_download_pressure(mps_session *s, double *pressure, int num);

/* Reference quantities n0, lambda, N0.  compute: on the device, with the
 * reference's rule (particle.c:69-221: first strictly largest n0_i in index
 * order, sums in ascending j).  set: take them from the caller. */
int  mps_compute_initial_params(mps_session *s, double *n0, double *lambda, int *n0_count);
int  mps_set_initial_params(mps_session *s, double n0, double lambda, int n0_count);

/* Neighbour search at the current positions (the step's cell sort).  Must run
 * once after an upload and before the first step, as simulation_run does. */
int  mps_neighbor_search(mps_session *s);

/* `nsteps` full time steps, device-resident (simulation.c:19-118). */
int  mps_step(mps_session *s, int nsteps);

/* One full step whose explicit stage (viscosity, 3-D collision) uses the
 * caller's neighbour list from the previous step, as the reference's
 * simulation_step(ps, nl, cl, step) does; the state comes from the last
 * upload.  Afterwards the session holds the fresh structure. */
int  mps_step_with_list(mps_session *s, const int *neighbors, const int *count, int max_nb);

/* Neighbour sets of the current structure in the reference's layout: for
 * each particle i (reference order) count[i] entries neighbors[i*max_nb+k]
 * in the reference's list order.  Either pointer may be NULL. */
int  mps_get_neighbor_list(mps_session *s, int *neighbors, int *count, int max_nb);
/* Cell index of each particle (reference order) as the reference computes
 * it, -1 for ghosts and particles outside the grid. */
int  mps_get_cell_index(mps_session *s, int *cell);
/* The reference's CellList chains of the current structure: head[total_cells]
 * (first = largest index of each cell, -1 if empty) and next[num]. */
int  mps_get_cell_links(mps_session *s, int *head, int *next, int total_cells);

/* PPE of the current state in the reference's unknown numbering (particle
 * order): eq_idx[num], row_ptr[n_eq+1], col_idx/val[nnz] (sorted columns,
 * diagonal included), b[n_eq].  Call with row_ptr == NULL to get sizes. */
int  mps_get_ppe(mps_session *s, int *eq_idx, int *row_ptr, int *col_idx, double *val,
                 double *b, int *n_eq, long long *nnz);

/* The last step's PPE and IC(0) preconditioner in the solver's own unknown
 * numbering (block colour order: colour by colour, cell by cell), for
 * checking the factorisation (pressure_solver.c:156-232 restated on this
 * ordering) and the sweeps.  ICCG sessions only.
 *
 * mps_get_ic0: row_ptr[n_eq+1], col[nnz] (sorted), A[nnz] and b[n_eq] (FP64)
 * and F[nnz], the factor in A's pattern: L_ij below the diagonal, 1/L_ii on
 * it, L_ji above it.  row_ptr == NULL returns the sizes only; other NULL
 * pointers are skipped.
 * mps_get_cell_blocks: per active cell k in colour order cells[2k] = first
 * row, cells[2k+1] = unknowns m; inv_off[ncells+1]; inv[ninv] the inverse of
 * each cell's diagonal block of L (FP64) at inv_off[k], column-major over
 * the lower triangle: (L_cc^-1)_ij (i >= j) at j*m - j*(j-1)/2 + (i - j)
 * (0 entries for cells above 64 unknowns, which the sweeps solve by
 * substitution); colour_rows[2^dim + 1] the first row of each colour.
 * mps_apply_preconditioner: z = (L L^T)^-1 r by the device sweeps of the
 * last solve's form (the FP32 factor copies after a mixed-form solve); r, z
 * are host arrays of n_eq doubles in the solver's numbering. */
int  mps_get_ic0(mps_session *s, int *row_ptr, int *col, double *A, double *F, double *b, int *n_eq,
                 long long *nnz);
int  mps_get_cell_blocks(mps_session *s, int *cells, int *inv_off, double *inv, int *colour_rows, int *ncells,
                         long long *ninv);
int  mps_apply_preconditioner(mps_session *s, const double *r, double *z);

int  mps_get_metrics(mps_session *s, mps_metrics_t *m);

/* Kernels launched by this library in this process so far. */
unsigned long long mps_launch_count(void);

/* The surface-tension coefficients the reference calibrates in
 * particle_system_calc_initial_params (particle.c:185-211, 2-D
 * particle.c:154-180): C_LL from the potential's interaction energy across a
 * flat interface of the rest lattice, C_SL = (1 + cos theta) / 2 C_LL.  Both
 * 0 when surface tension is off.  Host arithmetic, no device needed. */
int  mps_surface_tension_coeffs(const mps_params_t *params, double *c_ll, double *c_sl);

/* Per-kernel timing of the CG loop with CUDA events (adds no host sync). */
int  mps_set_profiling(mps_session *s, int on);
/* Zero the accumulated metrics. */
int  mps_reset_metrics(mps_session *s);

/* The stream all session work is issued on (a cudaStream_t). */
void *mps_get_stream(mps_session *s);

/* Stage entry points over a caller-supplied neighbour list (the reference's
 * NeighborList layout; host pointers).  The state is taken from the last
 * upload in reference order; results are read back with download.  These
 * back the drop-in's fine-grained functions. */
#define MPS_STAGE_DENSITY        1   /* calc_particle_number_density  (operators.c:17) */
#define MPS_STAGE_VISCOSITY      2   /* calc_viscosity_term           (operators.c:50) */
#define MPS_STAGE_GRADIENT       3   /* calc_pressure_gradient        (operators.c:102) */
#define MPS_STAGE_NEIGHBOR_COUNT 4   /* calc_neighbor_count           (operators.c:226) */
#define MPS_STAGE_COLLISION      5   /* collision                     (operators.c:371) */
#define MPS_STAGE_SOLVE_PRESSURE 6   /* solve_pressure                (pressure_solver.c:368) */
#define MPS_STAGE_SURFACE        7   /* judge_free_surface            (operators.c:206); arg = threshold */
#define MPS_STAGE_CLAMP          8   /* clamp_pressure                (operators.c:188) */
#define MPS_STAGE_WALL           9   /* apply_wall_boundary           (boundary.c:12) */
#define MPS_STAGE_OUT_OF_BOUNDS 10   /* remove_out_of_bounds          (boundary.c:33) */
#define MPS_STAGE_SURFACE_BY_COUNT 11 /* judge_free_surface_by_count (operators.c:253); arg = beta */
#define MPS_STAGE_SURFACE_TENSION 12  /* calc_surface_tension      (operators.c:281) */
#define MPS_STAGE_SURFACE_TENSION_SL 13 /* calc_surface_tension_SL (operators.c:322) */
int  mps_run_stage(mps_session *s, int stage, const int *neighbors, const int *count,
                   int max_nb, double arg);

/* ---- differentiation form (adjoint of the time step) --------------------
 *
 * No counterpart in the reference, which has no adjoint and no restart
 * format (its CSV output loses n0 / lambda and the sort state).
 *
 * Checkpoints.  mps_state_bytes gives the size of one checkpoint of the
 * session's current state (positions, velocities, sort keys, pressures,
 * flags, reference indices and the cell structure: all the next step
 * reads).  mps_state_save / mps_state_load copy it to / from a caller
 * buffer in host or device memory; loading and stepping reproduces the
 * saved run bit for bit.  A checkpoint only loads into the session that
 * wrote it (same capacity and grid).
 *
 * Adjoint.  mps_adjoint_seed sets the adjoint of a step's output state:
 * lam_pos, lam_vel are host arrays of num*dim doubles in reference particle
 * order (particle-major; NULL = zero); it also clears the accumulated
 * parameter gradients.  With the session holding that step's INPUT state
 * (mps_state_load), mps_step_adjoint recomputes the step and replaces the
 * seeds by the adjoint of the step's input, adding the step's terms to the
 * gradients with respect to gravity (dim components) and kinematic
 * viscosity; the session again holds the step's input state afterwards.
 * Every discrete decision of the step is held fixed (neighbour sets,
 * collision partners, order and branches, free-surface flags, the PPE
 * unknown set, the P_min argument, ghosting); the PPE adjoint is a second
 * ICCG solve with the step's matrix and IC(0) factor to relative residual
 * 1e-12 (in the session's precision form: with MPS_PREC_MIXED, the mixed
 * solve with reliable updates, to 1e-12 or the FP64 rounding floor if
 * that is higher).  Walls, dummies and ghosts get zero adjoints.  Supported: hs_mode
 * 0, ppe_type 0, cmps_gradient 0, no pressure clamp; other switches return
 * MPS_ERR_UNSUPPORTED, as do more than 8 collision impulses on one
 * particle in one step.  mps_adjoint_get reads the current seeds (NULL
 * skips) and the accumulated gradients; grad_drive receives the gradients
 * with respect to the wall drive's amplitude and frequency (2 doubles). */
int  mps_state_bytes(mps_session *s, size_t *bytes);
int  mps_state_save(mps_session *s, void *buf);
int  mps_state_load(mps_session *s, const void *buf);
int  mps_adjoint_seed(mps_session *s, const double *lam_pos, const double *lam_vel);
/* A loss on the pressures a step computes: dLdP (num doubles, reference
 * particle order; NULL clears) is added to the adjoint of the pressure of
 * the step that the next mps_step_adjoint reverses, before its adjoint PPE
 * solve, and is consumed by it.  Pressures that are not PPE unknowns
 * (surface and dummy particles) carry no gradient.  No counterpart in the
 * reference. */
int  mps_adjoint_pressure_seed(mps_session *s, const double *dLdP, int num);
int  mps_step_adjoint(mps_session *s);
int  mps_adjoint_get(mps_session *s, double *lam_pos, double *lam_vel, double *grad_gravity,
                     double *grad_viscosity, double *grad_drive);

/* ---- cell sort without device allocation ------------------------------
 *
 * No counterpart in the reference (its cell list is host memory allocated
 * by cell_list_create).  For callers that cannot allocate device memory
 * where they need the neighbour structure -- a frozen memory pool, a
 * replayed graph whose addresses must not change, a host program that owns
 * every buffer -- this sorts particles into the reference's cell grid using
 * only the caller's arrays plus one static device array of the library
 * (about 4 MB on every GPU that loads it, held until exit).
 *
 * pos: num*dim doubles, particle-major; type: num ints (ghosts are not
 * binned); all pointers are device memory.  Outputs: cell[num] (the
 * reference's cell index, -1 if not binned), cell_start[total_cells + 1]
 * (first slot of each cell; cell_start[total_cells] = binned particles) and
 * order[num] (particle indices, cell by cell, descending index within a
 * cell as the reference's chains, then the unbinned ones ascending).
 * Work is queued on `stream` (a cudaStream_t, 0 = default).
 *
 * Limits: num <= MPS_NOALLOC_MAX_PARTICLES, total cells <=
 * MPS_NOALLOC_MAX_CELLS; larger requests return MPS_ERR_INVALID.  The first
 * call on a device looks up the static array's device address and should
 * come before any stream capture.  The address is kept for the life of the
 * process; a cudaDeviceReset (or any reset of the device's primary context)
 * unloads the library's module and makes it stale, so no call may follow
 * one.  All calls share that array: calls whose work overlaps on the GPU
 * race on it and must be ordered by the caller.  A CUDA error already
 * pending in the calling thread is returned as MPS_ERR_CUDA without being
 * cleared, and no work is queued. */
#define MPS_NOALLOC_MAX_PARTICLES 262144
#define MPS_NOALLOC_MAX_CELLS     262144

typedef struct {
    int    dim;          /* 2 or 3 */
    double origin[3];    /* cell grid origin (cell_list_create: domain_min - 4 re) */
    double cell_size;    /* re */
    int    dims[3];      /* cells per axis */
} mps_grid_t;

int  mps_cell_sort_noalloc(const mps_grid_t *grid, const double *pos, const int *type, int num,
                           int *cell, int *order, int *cell_start, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MPS_B200_H */
