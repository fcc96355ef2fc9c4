/* mps_sim.c -- command-line driver: `mps_sim <cal.txt>`, the reference's CLI
 * (mps_fluid3D_parallel/src/main.c:87-138) on the B200 drop-in library.
 *
 * Reads cal.txt, then params.txt, then particles.txt ("count" line after
 * comments, then "x y [z] vx vy [vz] type" lines; malformed lines are skipped
 * with a warning), computes n0/lambda and runs simulation_run.  Unlike the
 * reference, the particle capacity is the file's count instead of a fixed
 * 100000 (main.c:115), so large decks are not silently truncated. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "../../include/mps_b200.h"
#include "../../include/mps_dropin.h"

static int skip_line(const char *p)
{
    while (*p == ' ' || *p == '\t') p++;
    return *p == '#' || *p == '\n' || *p == '\r' || *p == '\0';
}

static ParticleSystem *load_particles(const char *path)
{
    FILE *fp = fopen(path, "r");
    if (!fp) {
        fprintf(stderr, "Error: cannot open particle file '%s'\n", path);
        return NULL;
    }
    char line[512];
    int count = 0;
    while (fgets(line, sizeof(line), fp)) {
        if (skip_line(line)) continue;
        if (sscanf(line, "%d", &count) == 1) break;
    }
    if (count <= 0) {
        fprintf(stderr, "Error: invalid particle count in '%s'\n", path);
        fclose(fp);
        return NULL;
    }
    ParticleSystem *ps = particle_system_create(count);
    if (!ps) {
        fprintf(stderr, "Error: failed to create particle system\n");
        fclose(fp);
        return NULL;
    }
    int loaded = 0, n_fluid = 0, n_wall = 0;
    while (loaded < count && fgets(line, sizeof(line), fp)) {
        if (skip_line(line)) continue;
        double pos[MPS_DIM], vel[MPS_DIM];
        int type;
#if MPS_DIM == 3
        int got = sscanf(line, "%lf %lf %lf %lf %lf %lf %d", &pos[0], &pos[1], &pos[2], &vel[0], &vel[1], &vel[2],
                         &type);
        if (got != 7) {
#else
        int got = sscanf(line, "%lf %lf %lf %lf %d", &pos[0], &pos[1], &vel[0], &vel[1], &type);
        if (got != 5) {
#endif
            fprintf(stderr, "Warning: skipping malformed line: %s", line);
            continue;
        }
        particle_system_add(ps, pos, vel, type);
        loaded++;
        if (type == MPS_FLUID) n_fluid++;
        else if (type == MPS_WALL) n_wall++;
    }
    fclose(fp);
    if (loaded != count) fprintf(stderr, "Warning: expected %d particles but loaded %d\n", count, loaded);
    printf("Loaded particles: %d fluid, %d wall, %d total\n", n_fluid, n_wall, ps->num);
    return ps;
}

int main(int argc, char **argv)
{
    if (argc < 2 || argc > 3) {
        fprintf(stderr, "Usage: %s <cal_file> [fp64|mixed]\n", argv[0]);
        return 1;
    }
    /* optional precision form (not in the reference, which is FP64 only) */
    if (argc == 3) {
        int prec = strcmp(argv[2], "mixed") == 0 ? MPS_PREC_MIXED : strcmp(argv[2], "fp64") == 0 ? MPS_PREC_FP64 : -1;
        if (mps_dropin_set_precision(prec) != 0) {
            fprintf(stderr, "Unknown precision '%s' (fp64 or mixed)\n", argv[2]);
            return 1;
        }
    }
    SimConfig config;
    config_set_defaults(&config);
    if (config_load_cal(argv[1], &config) != 0) return 1;
    if (config_load_params(config.param_file, &config) != 0) return 1;
    g_config = &config;
    printf("=== MPS %dD Fluid Simulation (B200) ===\n\n", MPS_DIM);
    config_print(&config);
    mkdir(config.output_dir, 0755);
    ParticleSystem *ps = load_particles(config.particle_file);
    if (!ps) return 1;
    particle_system_calc_initial_params(ps);
    simulation_run(ps);
    int status = mps_dropin_last_status();
    particle_system_free(ps);
    return status == 0 ? 0 : 1;
}
