/*
 * mps_oracle.h -- CPU restatement of the reference MPS time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA path is compared
 * against; it is never linked into the product library and never timed as
 * the product.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * Every function restates one reference function with the same floating-point
 * operation order (no FMA contraction: build with -ffp-contract=off), so that
 * its outputs are bit-identical to the reference compiled from source.  The
 * config is passed explicitly instead of through a global.
 *
 * Parity is pinned two ways (tests/test_oracle_pin.py):
 *   - against the reference's own sources compiled into oracle/_ref/ by
 *     oracle/Makefile (bit-exact, every stage);
 *   - against the reference's shipped 3-D dam-break trajectory
 *     (mps_fluid3D_parallel/output/output_000100.csv), committed as the
 *     fixture tests/golden/dambreak3d_fluid_*.npz.
 */
#ifndef MPS_ORACLE_H
#define MPS_ORACLE_H

#include "../include/mps_types.h"

#ifdef __cplusplus
extern "C" {
#endif

double oracle_kernel_weight(double r, double re, const SimConfig *cfg);

void oracle_calc_initial_params(ParticleSystem *ps, const SimConfig *cfg);
void oracle_calc_initial_params_cells(ParticleSystem *ps, const SimConfig *cfg);

int  oracle_cell_list_init(CellList *cl, int num_particles, double re,
                           const double *domain_min, const double *domain_max);
int  oracle_neighbor_search(NeighborList *nl, const ParticleSystem *ps,
                            CellList *cl, double re);

void oracle_number_density(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
void oracle_viscosity(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
void oracle_surface_tension(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
void oracle_surface_tension_SL(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
/* Friction of the 3-D serial variant (3-D builds only): its four SimConfig
 * fields, kept apart because the OpenMP layout has none; off by default. */
typedef struct {
    int    enabled;
    double delta_theta;          /* degrees */
    double alpha;
    double velocity_threshold;   /* m/s */
} OracleFriction;
void oracle_set_friction(const OracleFriction *f);
void oracle_apply_friction(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
int  oracle_pressure_gradient(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
void oracle_judge_free_surface(ParticleSystem *ps, double threshold);
void oracle_neighbor_count(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);
void oracle_judge_free_surface_by_count(ParticleSystem *ps, double beta);
void oracle_clamp_pressure(ParticleSystem *ps);
int  oracle_collision(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);

/* PPE: assembly into reference-ordered CSR (unknowns numbered by particle
 * index), then CG / ICCG.  Returns the iteration count, -1 on OOM. */
int  oracle_solve_pressure(ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg);

/* Assembly only: fills eq_idx[num], and if row_ptr != NULL the CSR (sorted
 * columns, diagonal included) and b.  Returns n_eq; *nnz_out receives nnz.
 * Call first with row_ptr == NULL to size the buffers. */
int  oracle_assemble_ppe(const ParticleSystem *ps, const NeighborList *nl, const SimConfig *cfg,
                         int *eq_idx, int *row_ptr, int *col_idx, double *val, double *b,
                         long long *nnz_out);

void oracle_apply_wall_boundary(ParticleSystem *ps);
void oracle_remove_out_of_bounds(ParticleSystem *ps, const SimConfig *cfg);

/* Stage hooks of one time step, in the reference's order. */
int  oracle_step(ParticleSystem *ps, NeighborList *nl, CellList *cl, const SimConfig *cfg);
int  oracle_step_driven(ParticleSystem *ps, NeighborList *nl, CellList *cl, const SimConfig *cfg,
                        const double *rest, double amp, double freq, int axis, int step);
void oracle_wall_drive_terms(double amp, double freq, double t, double *dx, double *vel);

/* IC(0) on any unknown numbering (pressure_solver.c:156-232 applied to the
 * caller's CSR, e.g. the GPU solver's block colour order), the in-cell block
 * inverses and the preconditioner apply, in the GPU solver's factor
 * convention (F: L below the diagonal, 1/L_ii on it, L^T above). */
int  oracle_ic0_csr(int n, const int *rp, const int *ci, const double *v, double *F);
void oracle_cell_inverses(int ncells, const int *cells, const int *inv_off, const int *rp, const int *ci,
                          const double *F, int max_m, double *inv);
void oracle_ic0_apply_csr(int n, const int *rp, const int *ci, const double *F, const double *r, double *z);

/* Iteration count and final recursive residual of the last PPE solve. */
int    oracle_last_iterations(void);
double oracle_last_residual(void);

#ifdef __cplusplus
}
#endif

#endif /* MPS_ORACLE_H */
