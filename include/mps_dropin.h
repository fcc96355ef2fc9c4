/*
 * mps_dropin.h -- the reference solver's C entry points, served by the B200
 * library (libmps3d.so for 3-D, libmps2d.so for 2-D; build with the matching
 * MPS_DIM).  A program written against the reference's headers links one of
 * these instead of the reference's src/*.c and keeps its calls, structs
 * (include/mps_types.h) and the global `SimConfig *g_config`.
 *
 * Each declaration names the reference interface it replaces
 * (mps_fluid3D_parallel/include/...; the 2-D variant mps_fluid2D/include/...
 * differs only where noted).  Semantics:
 *
 *   - Time step, neighbour search, operators, PPE and boundary functions run
 *     on the GPU through the session API (include/mps_b200.h); particle data
 *     is copied host->device before and device->host after each call, so the
 *     caller's AoS arrays, NeighborList and CellList hold the reference's
 *     results.  simulation_run keeps the state on the device between outputs.
 *   - Failures the reference turns into exit(EXIT_FAILURE) (neighbour
 *     overflow) still exit with a message; CUDA and device errors do too,
 *     with the error text.  There is no CPU fallback.
 *   - The parameter-file, particle and output helpers are host code with the
 *     reference's conventions.
 */
#ifndef MPS_DROPIN_H
#define MPS_DROPIN_H

#include "mps_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sim_config.h:84-93 */
extern SimConfig *g_config;
void config_set_defaults(SimConfig *config);                       /* sim_config.c:20 */
int  config_load_cal(const char *cal_path, SimConfig *config);     /* sim_config.c:120 */
int  config_load_params(const char *param_path, SimConfig *config);/* sim_config.c:166 */
void config_print(const SimConfig *config);                        /* sim_config.c:279 */

/* particle.h:32-38 */
ParticleSystem *particle_system_create(int capacity);
void            particle_system_free(ParticleSystem *ps);
int             particle_system_add(ParticleSystem *ps, double pos[], double vel[], int type);
void            particle_system_calc_initial_params(ParticleSystem *ps);   /* GPU */

/* kernel.h:5-8 */
double kernel_weight(double r, double re);
double kernel_weight_derivative(double r, double re);

/* neighbor_search.h:33-50 */
NeighborList *neighbor_list_create(int num_particles, int max_neighbors);
void          neighbor_list_free(NeighborList *nl);
CellList     *cell_list_create(int num_particles, double re,
                               const double domain_min[MPS_DIM], const double domain_max[MPS_DIM]);
void          cell_list_free(CellList *cl);
void          neighbor_search_brute_force(NeighborList *nl, ParticleSystem *ps, double re);       /* GPU */
void          neighbor_search_cell_linked_list(NeighborList *nl, ParticleSystem *ps,
                                               CellList *cl, double re);                         /* GPU */
int           neighbor_get(NeighborList *nl, int i, int j);

/* operators.h:8-36 (GPU) */
void calc_particle_number_density(ParticleSystem *ps, NeighborList *nl);
void calc_viscosity_term(ParticleSystem *ps, NeighborList *nl);
void calc_pressure_gradient(ParticleSystem *ps, NeighborList *nl);
void judge_free_surface(ParticleSystem *ps, double threshold);
void calc_neighbor_count(ParticleSystem *ps, NeighborList *nl);
void judge_free_surface_by_count(ParticleSystem *ps, double beta);
void clamp_pressure(ParticleSystem *ps);
#if MPS_DIM == 3
void collision(ParticleSystem *ps, NeighborList *nl);
#else
void collision(ParticleSystem *ps);                                 /* 2D operators.h: all pairs */
#endif
/* Not on this path: print an error and exit when called. */
void calc_surface_tension(ParticleSystem *ps, NeighborList *nl);
void calc_surface_tension_SL(ParticleSystem *ps, NeighborList *nl);

/* pressure_solver.h:8 (GPU) */
void solve_pressure(ParticleSystem *ps, NeighborList *nl);

/* boundary.h:8-14 (GPU) */
void apply_wall_boundary(ParticleSystem *ps);
#if MPS_DIM == 3
void remove_out_of_bounds(ParticleSystem *ps, double xmin, double xmax, double ymin, double ymax,
                          double zmin, double zmax);
#else
void remove_out_of_bounds(ParticleSystem *ps, double xmin, double xmax, double ymin, double ymax);
#endif

/* simulation.h:8,17 (GPU) */
void simulation_run(ParticleSystem *ps);
void simulation_step(ParticleSystem *ps, NeighborList *nl, CellList *cl, int step);

/* io.h:8-11 */
void output_csv(const ParticleSystem *ps, int step, const char *output_dir);
void output_vtk(const ParticleSystem *ps, int step, const char *output_dir);

/* Not in the reference: the status of the last drop-in call (MPS_OK or an
 * MPS_ERR_* code of include/mps_b200.h), for callers that install
 * mps_dropin_set_exit_on_error(0) and check instead of exiting. */
int  mps_dropin_last_status(void);
void mps_dropin_set_exit_on_error(int on);
/* Not in the reference (FP64 only): the precision form of the drop-in's
 * steps from the next call on, MPS_PREC_FP64 (default) or MPS_PREC_MIXED;
 * returns MPS_OK, or MPS_ERR_INVALID for any other value. */
int  mps_dropin_set_precision(int precision);
/* Not in the reference: release the device session bound to `ps`. */
void mps_dropin_release(ParticleSystem *ps);

#ifdef __cplusplus
}
#endif

#endif /* MPS_DROPIN_H */
