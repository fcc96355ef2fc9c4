/*
 * mps_types.h -- the particle data model shared by the drop-in library, the
 * CLI and the CPU oracle.
 *
 * These structs are the ABI of the reference solver's hot path: callers that
 * link the reference's sources hand AoS `Particle` arrays, a `NeighborList`, a
 * `CellList` and a global `SimConfig *g_config` to every stage function.  To be
 * a drop-in, the layouts below keep the same fields, types and order as the
 * reference headers:
 *
 *   Particle / ParticleSystem  <- mps_fluid3D_parallel/include/particle.h:7-30
 *                                 (2-D: mps_fluid2D/include/particle.h)
 *   NeighborList / CellList    <- mps_fluid3D_parallel/include/neighbor_search.h:8-30
 *   SimConfig                  <- mps_fluid3D_parallel/include/sim_config.h:10-78
 *                                 (2-D differs only through DIM)
 *   particle type codes        <- mps_fluid3D_parallel/include/config.h:8-11
 *
 * The dimension is a compile-time constant exactly as in the reference
 * (`DIM` there, `MPS_DIM` here; default 3).  3-D Particle is 104 bytes,
 * 2-D Particle is 80 bytes.
 */
#ifndef MPS_TYPES_H
#define MPS_TYPES_H

#ifndef MPS_DIM
#define MPS_DIM 3
#endif

#if MPS_DIM != 2 && MPS_DIM != 3
#error "MPS_DIM must be 2 or 3"
#endif

#define MPS_FLUID 0
#define MPS_WALL  1
#define MPS_GHOST 2
#define MPS_DUMMY 3

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double pos[MPS_DIM];
    double vel[MPS_DIM];
    double acc[MPS_DIM];
    double pressure;
    double n;               /* particle number density */
    int    neighbor_count;  /* N_i for count-based surface detection */
    int    type;            /* MPS_FLUID / MPS_WALL / MPS_GHOST / MPS_DUMMY */
    int    on_surface;
} Particle;

typedef struct {
    Particle *particles;
    int       num;
    int       capacity;
    double    n0;
    double    lambda;
    double    C_LL;
    double    C_SL;
    int       n0_count;
} ParticleSystem;

typedef struct {
    int *neighbors;      /* [num_particles * max_neighbors] */
    int *count;          /* [num_particles] */
    int  max_neighbors;
} NeighborList;

typedef struct {
    int   *head;         /* [total_cells] first particle of each cell, -1 = empty */
    int   *next;         /* [num_particles] next particle in the same cell, -1 = end */
    int    nx;
    int    ny;
#if MPS_DIM == 3
    int    nz;
#endif
    int    total_cells;
    double cell_size;
    double origin[MPS_DIM];
} CellList;

typedef struct {
    double particle_distance;
    double influence_ratio_lap;
    double influence_radius_lap;
    double influence_ratio_n;
    double influence_radius_n;
    int    max_neighbors;
    int    wall_layers;
    int    dummy_layers;

    double density;
    double viscosity;
    double gravity[MPS_DIM];

    double dt;
    double t_end;
    int    output_interval;

    int    solver_type;              /* 0: CG, 1: ICCG */
    int    cg_max_iter;
    double cg_tolerance;
    double relaxation_coeff;
    int    clamp_negative_pressure;
    int    ppe_type;                 /* 0: density source, 1: weakly compressible (Natsui) */
    double c_ppe;
    double gamma_ppe;

    double surface_threshold;
    int    surface_detection_method; /* 0: number density, 1: neighbour count */
    double surface_count_threshold;

    double restitution_coeff;
    double collision_distance_ratio;

    int    surface_tension_enabled;
    double surface_tension_coeff;
    double surface_tension_re_ratio;
    double influence_radius_st;

    double wetting_angle_SL;

    double domain_min[MPS_DIM];
    double domain_max[MPS_DIM];

    int    cmps_gradient;            /* 0: P_j - P_min, 1: CMPS, 2: Oochi */
    int    use_analytical_lambda;
    int    hs_mode;

    char   output_dir[256];
    char   particle_file[256];
    char   param_file[256];
} SimConfig;

#ifdef __cplusplus
}
#endif

#endif /* MPS_TYPES_H */
