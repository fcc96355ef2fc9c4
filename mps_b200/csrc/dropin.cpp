// dropin.cpp -- the reference solver's C entry points over the B200 session API.
//
// Built twice: -DMPS_DIM=3 -> libmps3d.so, -DMPS_DIM=2 -> libmps2d.so (each
// links libmps_b200.so).  Declarations and semantics: include/mps_dropin.h.
// Each GPU-backed call binds a session to the ParticleSystem pointer,
// refreshes its parameters from g_config, uploads the AoS particles, runs
// the stage on the device and downloads the results.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sys/stat.h>
#include <vector>

#include "../../include/mps_b200.h"
#include "../../include/mps_dropin.h"

#define D MPS_DIM

extern "C" {
SimConfig *g_config = NULL;
}

namespace {

struct Ctx {
    mps_session *s = nullptr;
    mps_params_t p{};
    int capacity = 0;
};

std::map<const ParticleSystem *, Ctx> g_ctx;
int g_status = MPS_OK;
int g_exit_on_error = 1;
int g_precision = MPS_PREC_FP64;   // mps_dropin_set_precision

void fail(const char *where, int rc, mps_session *s)
{
    g_status = rc;
    const char *detail = s ? mps_last_error(s) : "";
    if (rc == MPS_ERR_NEIGHBOR_OVERFLOW) {
        // the reference's message and exit (neighbor_search.c:221-228)
        std::fprintf(stderr,
                     "Error: neighbor count exceeded max_neighbors (%d). Increase max_neighbors in params.txt.\n",
                     g_config ? g_config->max_neighbors : -1);
    } else {
        std::fprintf(stderr, "Error: %s: %s%s%s\n", where, mps_error_string(rc), detail && *detail ? ": " : "",
                     detail ? detail : "");
    }
    if (g_exit_on_error) std::exit(EXIT_FAILURE);
}

bool ok(const char *where, int rc, mps_session *s)
{
    if (rc == MPS_OK) return true;
    fail(where, rc, s);
    return false;
}

mps_params_t params_from(const SimConfig *c)
{
    mps_params_t p;
    std::memset(&p, 0, sizeof(p));
    p.dim = D;
    p.particle_distance = c->particle_distance;
    p.influence_radius_lap = c->influence_radius_lap;
    p.influence_radius_n = c->influence_radius_n;
    p.max_neighbors = c->max_neighbors;
    p.wall_layers = c->wall_layers;
    p.density = c->density;
    p.viscosity = c->viscosity;
    for (int d = 0; d < D; d++) {
        p.gravity[d] = c->gravity[d];
        p.domain_min[d] = c->domain_min[d];
        p.domain_max[d] = c->domain_max[d];
    }
    p.dt = c->dt;
    p.solver_type = c->solver_type;
    p.cg_max_iter = c->cg_max_iter;
    p.cg_tolerance = c->cg_tolerance;
    p.relaxation_coeff = c->relaxation_coeff;
    p.clamp_negative_pressure = c->clamp_negative_pressure;
    p.ppe_type = c->ppe_type;
    p.c_ppe = c->c_ppe;
    p.gamma_ppe = c->gamma_ppe;
    p.surface_threshold = c->surface_threshold;
    p.surface_detection_method = c->surface_detection_method;
    p.surface_count_threshold = c->surface_count_threshold;
    p.restitution_coeff = c->restitution_coeff;
    p.collision_distance_ratio = c->collision_distance_ratio;
    p.surface_tension_enabled = c->surface_tension_enabled;
    p.influence_radius_st = c->influence_radius_st;
    p.surface_tension_coeff = c->surface_tension_coeff;
    p.wetting_angle_SL = c->wetting_angle_SL;
    p.cmps_gradient = c->cmps_gradient;
    p.use_analytical_lambda = c->use_analytical_lambda;
    p.hs_mode = c->hs_mode;
    p.precision = g_precision;
    p.refine_tolerance = 0.0;
    return p;
}

// The session bound to `ps`, with parameters refreshed from g_config.
Ctx *ctx_for(const ParticleSystem *ps, const mps_params_t *override = nullptr)
{
    if (!g_config) {
        std::fprintf(stderr, "Error: g_config is not set\n");
        g_status = MPS_ERR_INVALID;
        if (g_exit_on_error) std::exit(EXIT_FAILURE);
        return nullptr;
    }
    mps_params_t p = override ? *override : params_from(g_config);
    Ctx &c = g_ctx[ps];
    int cap = ps->capacity > ps->num ? ps->capacity : ps->num;
    if (cap < 1) cap = 1;
    if (!c.s || c.capacity < cap) {
        if (c.s) mps_session_destroy(c.s);
        c.s = nullptr;
        int rc = mps_session_create(&c.s, &p, cap);
        if (rc != MPS_OK) {
            fail("mps_session_create", rc, nullptr);
            return nullptr;
        }
        c.capacity = cap;
        c.p = p;
    } else if (std::memcmp(&p, &c.p, sizeof(p)) != 0) {
        if (!ok("mps_update_params", mps_update_params(c.s, &p), c.s)) return nullptr;
        c.p = p;
    }
    g_status = MPS_OK;
    return &c;
}

bool upload(Ctx *c, const ParticleSystem *ps, bool ref_params)
{
    if (!ok("mps_upload_particles", mps_upload_particles(c->s, ps->particles, ps->num), c->s)) return false;
    if (ref_params && !ok("mps_set_initial_params", mps_set_initial_params(c->s, ps->n0, ps->lambda, ps->n0_count), c->s))
        return false;
    return true;
}

bool download(Ctx *c, ParticleSystem *ps)
{
    return ok("mps_download_particles", mps_download_particles(c->s, ps->particles, ps->num), c->s);
}

void stage(ParticleSystem *ps, NeighborList *nl, int st, double arg, bool ref_params, const char *name)
{
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, ref_params)) return;
    int rc = mps_run_stage(c->s, st, nl ? nl->neighbors : nullptr, nl ? nl->count : nullptr,
                           nl ? nl->max_neighbors : 0, arg);
    if (!ok(name, rc, c->s)) return;
    download(c, ps);
}

double list_radius()
{
    double re = std::fmax(g_config->influence_radius_lap, g_config->influence_radius_n);
    if (g_config->surface_tension_enabled) re = std::fmax(re, g_config->influence_radius_st);
    return re;
}

// ---- parameter files (sim_config.c conventions) ---------------------------

char *trim(char *s)
{
    while (std::isspace((unsigned char)*s)) s++;
    if (*s == '\0') return s;
    char *e = s + std::strlen(s) - 1;
    while (e > s && std::isspace((unsigned char)*e)) *e-- = '\0';
    return s;
}

void resolve_path(const char *cal_path, const char *value, char *out, size_t n)
{
    if (value[0] == '/') {
        std::snprintf(out, n, "%s", value);
        return;
    }
    char dir[256];
    std::snprintf(dir, sizeof(dir), "%s", cal_path);
    char *slash = std::strrchr(dir, '/');
    if (slash) {
        slash[1] = '\0';
        std::snprintf(out, n, "%s%s", dir, value);
    } else {
        std::snprintf(out, n, "%s", value);
    }
}

}  // namespace

extern "C" {

int mps_dropin_last_status(void) { return g_status; }
void mps_dropin_set_exit_on_error(int on) { g_exit_on_error = on; }

int mps_dropin_set_precision(int precision)
{
    if (precision != MPS_PREC_FP64 && precision != MPS_PREC_MIXED) return MPS_ERR_INVALID;
    g_precision = precision;
    return MPS_OK;
}

void mps_dropin_release(ParticleSystem *ps)
{
    auto it = g_ctx.find(ps);
    if (it == g_ctx.end()) return;
    if (it->second.s) mps_session_destroy(it->second.s);
    g_ctx.erase(it);
}

// ---- configuration ----------------------------------------------------------

void config_set_defaults(SimConfig *c)
{
    std::memset(c, 0, sizeof(SimConfig));
    c->particle_distance = 0.025;
    c->influence_ratio_lap = 2.1;
    c->influence_radius_lap = 2.1 * 0.025;
    c->influence_ratio_n = 2.1;
    c->influence_radius_n = 2.1 * 0.025;
    c->max_neighbors = (D == 3) ? 512 : 256;
    c->wall_layers = 2;
    c->dummy_layers = 2;
    c->density = 1000.0;
    c->viscosity = 1.0e-6;
    c->gravity[1] = -9.81;
    c->dt = 5.0e-4;
    c->t_end = 2.0;
    c->output_interval = 100;
    c->solver_type = 0;
    c->cg_max_iter = 10000;
    c->cg_tolerance = 1.0e-8;
    c->relaxation_coeff = 0.2;
    c->ppe_type = 0;
    c->c_ppe = 1.01;
    c->gamma_ppe = 0.01;
    c->surface_threshold = 0.97;
    c->surface_count_threshold = 0.85;
    c->restitution_coeff = 0.2;
    c->collision_distance_ratio = 0.5;
    c->surface_tension_coeff = 0.0728;
    c->surface_tension_re_ratio = 3.2;
    c->influence_radius_st = 3.2 * 0.025;
    c->wetting_angle_SL = 90.0;
#if D == 3
    c->domain_max[0] = 0.4;
    c->domain_max[1] = 0.3;
    c->domain_max[2] = 0.2;
#else
    c->domain_max[0] = 1.0;
    c->domain_max[1] = 0.6;
#endif
    std::snprintf(c->output_dir, sizeof(c->output_dir), "output");
}

int config_load_cal(const char *cal_path, SimConfig *c)
{
    FILE *fp = std::fopen(cal_path, "r");
    if (!fp) {
        std::fprintf(stderr, "Error: cannot open cal file '%s'\n", cal_path);
        return -1;
    }
    char line[512];
    while (std::fgets(line, sizeof(line), fp)) {
        char *p = trim(line);
        if (*p == '\0' || *p == '#') continue;
        char key[128], val[256];
        if (std::sscanf(p, "%127s %255s", key, val) != 2) continue;
        if (!std::strcmp(key, "particle_file")) resolve_path(cal_path, val, c->particle_file, sizeof(c->particle_file));
        else if (!std::strcmp(key, "param_file")) resolve_path(cal_path, val, c->param_file, sizeof(c->param_file));
        else std::fprintf(stderr, "Warning: unknown key in cal file: '%s'\n", key);
    }
    std::fclose(fp);
    if (!c->particle_file[0]) {
        std::fprintf(stderr, "Error: particle_file not specified in '%s'\n", cal_path);
        return -1;
    }
    if (!c->param_file[0]) {
        std::fprintf(stderr, "Error: param_file not specified in '%s'\n", cal_path);
        return -1;
    }
    return 0;
}

int config_load_params(const char *param_path, SimConfig *c)
{
    FILE *fp = std::fopen(param_path, "r");
    if (!fp) {
        std::fprintf(stderr, "Error: cannot open param file '%s'\n", param_path);
        return -1;
    }
    struct F { const char *k; double *d; int *i; };
    const F table[] = {
        {"particle_distance", &c->particle_distance, nullptr},
        {"influence_ratio_lap", &c->influence_ratio_lap, nullptr},
        {"influence_ratio_n", &c->influence_ratio_n, nullptr},
        {"max_neighbors", nullptr, &c->max_neighbors},
        {"wall_layers", nullptr, &c->wall_layers},
        {"dummy_layers", nullptr, &c->dummy_layers},
        {"density", &c->density, nullptr},
        {"viscosity", &c->viscosity, nullptr},
        {"gravity_x", &c->gravity[0], nullptr},
        {"gravity_y", &c->gravity[1], nullptr},
#if D == 3
        {"gravity_z", &c->gravity[2], nullptr},
#endif
        {"dt", &c->dt, nullptr},
        {"t_end", &c->t_end, nullptr},
        {"output_interval", nullptr, &c->output_interval},
        {"solver_type", nullptr, &c->solver_type},
        {"cg_max_iter", nullptr, &c->cg_max_iter},
        {"cg_tolerance", &c->cg_tolerance, nullptr},
        {"relaxation_coeff", &c->relaxation_coeff, nullptr},
        {"clamp_negative_pressure", nullptr, &c->clamp_negative_pressure},
        {"ppe_type", nullptr, &c->ppe_type},
        {"c_ppe", &c->c_ppe, nullptr},
        {"gamma_ppe", &c->gamma_ppe, nullptr},
        {"surface_threshold", &c->surface_threshold, nullptr},
        {"surface_detection_method", nullptr, &c->surface_detection_method},
        {"surface_count_threshold", &c->surface_count_threshold, nullptr},
        {"restitution_coeff", &c->restitution_coeff, nullptr},
        {"collision_distance_ratio", &c->collision_distance_ratio, nullptr},
        {"surface_tension_enabled", nullptr, &c->surface_tension_enabled},
        {"surface_tension_coeff", &c->surface_tension_coeff, nullptr},
        {"surface_tension_re_ratio", &c->surface_tension_re_ratio, nullptr},
        {"wetting_angle_SL", &c->wetting_angle_SL, nullptr},
        {"domain_x_min", &c->domain_min[0], nullptr},
        {"domain_x_max", &c->domain_max[0], nullptr},
        {"domain_y_min", &c->domain_min[1], nullptr},
        {"domain_y_max", &c->domain_max[1], nullptr},
#if D == 3
        {"domain_z_min", &c->domain_min[2], nullptr},
        {"domain_z_max", &c->domain_max[2], nullptr},
#endif
        {"cmps_gradient", nullptr, &c->cmps_gradient},
        {"use_analytical_lambda", nullptr, &c->use_analytical_lambda},
        {"hs_mode", nullptr, &c->hs_mode},
    };
    char line[512];
    while (std::fgets(line, sizeof(line), fp)) {
        char *p = trim(line);
        if (*p == '\0' || *p == '#') continue;
        char key[128], val[256];
        if (std::sscanf(p, "%127s %255s", key, val) != 2) continue;
        if (!std::strcmp(key, "output_dir")) {
            std::strncpy(c->output_dir, val, sizeof(c->output_dir) - 1);
            continue;
        }
        bool found = false;
        for (const F &f : table) {
            if (std::strcmp(key, f.k)) continue;
            if (f.d) *f.d = std::atof(val);
            else *f.i = std::atoi(val);
            found = true;
            break;
        }
        if (!found) std::fprintf(stderr, "Warning: unknown parameter '%s'\n", key);
    }
    std::fclose(fp);
    c->influence_radius_lap = c->influence_ratio_lap * c->particle_distance;
    c->influence_radius_n = c->influence_ratio_n * c->particle_distance;
    c->influence_radius_st = c->surface_tension_re_ratio * c->particle_distance;
    return 0;
}

// The configuration report printed at start-up.  Its text is a user-visible
// format, kept line for line as the reference prints it (3-D OpenMP
// sim_config.c:279-334, 2-D sim_config.c:261-322; the two variants differ in
// labels and in where the surface-tension lines go).
void config_print(const SimConfig *c)
{
    const bool nat_ppe = c->ppe_type == 1, by_count = c->surface_detection_method == 1;
    const bool st = c->surface_tension_enabled != 0;
    const char *on_off[2] = {"OFF", "ON"};
    const char *lambda_src = c->use_analytical_lambda ? "analytical" : "from initial particles";
    const char *hs = c->hs_mode ? "ON (High order Source term)" : "OFF (standard)";
    const double col_dist = c->collision_distance_ratio * c->particle_distance;

    std::printf("=== Simulation Configuration ===\n");
    std::printf("particle_distance:    %.6f m\n", c->particle_distance);
    std::printf("influence_radius_lap: %.6f m  (ratio = %.2f)  [Laplacian]\n", c->influence_radius_lap,
                c->influence_ratio_lap);
    std::printf("influence_radius_n:   %.6f m  (ratio = %.2f)  [number density]\n", c->influence_radius_n,
                c->influence_ratio_n);
    std::printf("max_neighbors:        %d\n", c->max_neighbors);
    std::printf("wall_layers:          %d\n", c->wall_layers);
    std::printf(D == 3 ? "dummy_layers:          %d\n" : "dummy_layers:         %d\n", c->dummy_layers);
    std::printf("density:              %.1f kg/m^3\n", c->density);
    std::printf("viscosity:            %.2e m^2/s\n", c->viscosity);
#if D == 3
    std::printf("gravity:              (%.4f, %.4f, %.4f) m/s^2\n", c->gravity[0], c->gravity[1], c->gravity[2]);
#else
    std::printf("gravity:              (%.4f, %.4f) m/s^2\n", c->gravity[0], c->gravity[1]);
#endif
    std::printf("dt:                   %.2e s\n", c->dt);
    std::printf("t_end:                %.4f s\n", c->t_end);
    std::printf("output_interval:      %d steps\n", c->output_interval);
    std::printf("solver_type:          %s\n", c->solver_type == 1 ? "ICCG" : "CG");
    std::printf("cg_max_iter:          %d\n", c->cg_max_iter);
    std::printf("cg_tolerance:         %.2e\n", c->cg_tolerance);
    std::printf("relaxation_coeff:     %.4f\n", c->relaxation_coeff);
    std::printf("clamp_negative_pressure: %s\n", on_off[c->clamp_negative_pressure ? 1 : 0]);
#if D == 3
    std::printf("ppe_type:             %d  (%s)\n", c->ppe_type,
                nat_ppe ? "Natsui weak-compressible" : "standard density");
    if (nat_ppe) std::printf("  c_ppe=%.3f  gamma_ppe=%.4f\n", c->c_ppe, c->gamma_ppe);
    std::printf("surface_threshold:    %.4f\n", c->surface_threshold);
    std::printf("surface_detection:    %s\n", by_count ? "neighbor count (Natsui)" : "number density");
    if (by_count) std::printf("  surface_count_threshold=%.3f\n", c->surface_count_threshold);
    if (st)
        std::printf("surface_tension:      ON  sigma=%.4e  re_ratio=%.2f  theta_SL=%.1f deg\n",
                    c->surface_tension_coeff, c->surface_tension_re_ratio, c->wetting_angle_SL);
    std::printf("restitution_coeff:         %.4f\n", c->restitution_coeff);
    std::printf("collision_distance_ratio:  %.4f  (col_dist = %.6f m)\n", c->collision_distance_ratio, col_dist);
    std::printf("domain:               [%.3f, %.3f] x [%.3f, %.3f] x [%.3f, %.3f]\n", c->domain_min[0],
                c->domain_max[0], c->domain_min[1], c->domain_max[1], c->domain_min[2], c->domain_max[2]);
    std::printf("cmps_gradient:        %s\n", c->cmps_gradient ? "CMPS (symmetric)" : "standard");
#else
    std::printf("ppe_type:             %d  (%s)\n", c->ppe_type, nat_ppe ? "Natsui weakly-compressible" : "density-based");
    if (nat_ppe) std::printf("  c_ppe = %.4f  gamma_ppe = %.4f\n", c->c_ppe, c->gamma_ppe);
    std::printf("surface_threshold:    %.4f\n", c->surface_threshold);
    std::printf("surface_detection_method: %d  (%s)\n", c->surface_detection_method,
                by_count ? "neighbor_count (Natsui)" : "number_density");
    if (by_count) std::printf("surface_count_threshold:  %.4f\n", c->surface_count_threshold);
    std::printf("restitution_coeff:         %.4f\n", c->restitution_coeff);
    std::printf("collision_distance_ratio:  %.4f  (col_dist = %.6f m)\n", c->collision_distance_ratio, col_dist);
    std::printf("surface_tension:      %s\n", on_off[st ? 1 : 0]);
    if (st) {
        std::printf("  surface_tension_coeff:    %.4f N/m\n", c->surface_tension_coeff);
        std::printf("  surface_tension_re_ratio: %.2f  (re_st = %.6f m)\n", c->surface_tension_re_ratio,
                    c->influence_radius_st);
        std::printf("  wetting_angle_SL:         %.2f deg\n", c->wetting_angle_SL);
    }
    std::printf("domain:               [%.3f, %.3f] x [%.3f, %.3f]\n", c->domain_min[0], c->domain_max[0],
                c->domain_min[1], c->domain_max[1]);
    std::printf("cmps_gradient:        %d  (%s)\n", c->cmps_gradient,
                c->cmps_gradient ? "CMPS symmetric (P_i+P_j-P_imin-P_jmin)" : "standard (P_j-P_min)");
#endif
    std::printf("use_analytical_lambda: %d  (%s)\n", c->use_analytical_lambda, lambda_src);
    std::printf("hs_mode:              %d  (%s)\n", c->hs_mode, hs);
    std::printf("output_dir:           %s\n", c->output_dir);
    std::printf("particle_file:        %s\n", c->particle_file);
    std::printf("param_file:           %s\n", c->param_file);
    std::printf("================================\n\n");
}

// ---- particle system ----------------------------------------------------------

ParticleSystem *particle_system_create(int capacity)
{
    ParticleSystem *ps = (ParticleSystem *)std::malloc(sizeof(ParticleSystem));
    if (!ps) return NULL;
    ps->particles = (Particle *)std::calloc((size_t)(capacity > 0 ? capacity : 1), sizeof(Particle));
    if (!ps->particles) {
        std::free(ps);
        return NULL;
    }
    ps->num = 0;
    ps->capacity = capacity;
    ps->n0 = ps->lambda = ps->C_LL = ps->C_SL = 0.0;
    ps->n0_count = 0;
    return ps;
}

void particle_system_free(ParticleSystem *ps)
{
    if (!ps) return;
    mps_dropin_release(ps);
    std::free(ps->particles);
    std::free(ps);
}

int particle_system_add(ParticleSystem *ps, double pos[], double vel[], int type)
{
    if (ps->num >= ps->capacity) {
        std::fprintf(stderr, "Error: particle capacity exceeded (%d)\n", ps->capacity);
        return -1;
    }
    Particle *p = &ps->particles[ps->num];
    for (int d = 0; d < D; d++) {
        p->pos[d] = pos[d];
        p->vel[d] = vel[d];
        p->acc[d] = 0.0;
    }
    p->pressure = 0.0;
    p->n = 0.0;
    p->type = type;
    p->on_surface = 0;
    return ps->num++;
}

void particle_system_calc_initial_params(ParticleSystem *ps)
{
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, false)) return;
    double n0 = 0, lam = 0;
    int n0c = 0;
    if (!ok("mps_compute_initial_params", mps_compute_initial_params(c->s, &n0, &lam, &n0c), c->s)) return;
    ps->n0 = n0;
    ps->lambda = lam;
    if (g_config->surface_detection_method == 1) ps->n0_count = n0c;
    if (g_config->surface_tension_enabled) {
        mps_params_t p = params_from(g_config);
        mps_surface_tension_coeffs(&p, &ps->C_LL, &ps->C_SL);
    }
    std::printf("Initial params: n0 = %.6f (re_n=%.4f)  N0 = %d  lambda = %.6f (re_lap=%.4f)%s\n", ps->n0,
                g_config->influence_radius_n, ps->n0_count, ps->lambda, g_config->influence_radius_lap,
                g_config->use_analytical_lambda ? "  [analytical]" : "");
    if (g_config->surface_tension_enabled)
        std::printf("  C_LL = %.6e  C_SL = %.6e (theta=%.1f deg, re_st=%.4f)\n", ps->C_LL, ps->C_SL,
                    g_config->wetting_angle_SL, g_config->influence_radius_st);
}

// ---- kernel function (kernel.c:12-30) -------------------------------------------

double kernel_weight(double r, double re)
{
    if (r >= re) return 0.0;
    double rmin = 0.01 * g_config->particle_distance;
    if (r < rmin) r = rmin;
    return re / r - 1.0;
}

double kernel_weight_derivative(double r, double re)
{
    if (r >= re) return 0.0;
    double rmin = 0.01 * g_config->particle_distance;
    if (r < rmin) r = rmin;
    return -re / (r * r);
}

// ---- neighbour lists ------------------------------------------------------------

NeighborList *neighbor_list_create(int num_particles, int max_neighbors)
{
    NeighborList *nl = (NeighborList *)std::malloc(sizeof(NeighborList));
    if (!nl) return NULL;
    nl->neighbors = (int *)std::malloc(sizeof(int) * (size_t)num_particles * (size_t)max_neighbors);
    nl->count = (int *)std::calloc((size_t)num_particles, sizeof(int));
    nl->max_neighbors = max_neighbors;
    if (!nl->neighbors || !nl->count) {
        std::free(nl->neighbors);
        std::free(nl->count);
        std::free(nl);
        return NULL;
    }
    return nl;
}

void neighbor_list_free(NeighborList *nl)
{
    if (!nl) return;
    std::free(nl->neighbors);
    std::free(nl->count);
    std::free(nl);
}

int neighbor_get(NeighborList *nl, int i, int j) { return nl->neighbors[(size_t)i * nl->max_neighbors + j]; }

CellList *cell_list_create(int num_particles, double re, const double domain_min[D], const double domain_max[D])
{
    CellList *cl = (CellList *)std::malloc(sizeof(CellList));
    if (!cl) return NULL;
    cl->cell_size = re;
    double margin = 4.0 * re;
    for (int d = 0; d < D; d++) cl->origin[d] = domain_min[d] - margin;
    cl->nx = (int)(((domain_max[0] + margin) - cl->origin[0]) / re) + 2;
    cl->ny = (int)(((domain_max[1] + margin) - cl->origin[1]) / re) + 2;
#if D == 3
    cl->nz = (int)(((domain_max[2] + margin) - cl->origin[2]) / re) + 2;
    cl->total_cells = cl->nx * cl->ny * cl->nz;
#else
    cl->total_cells = cl->nx * cl->ny;
#endif
    cl->head = (int *)std::malloc(sizeof(int) * (size_t)cl->total_cells);
    cl->next = (int *)std::malloc(sizeof(int) * (size_t)(num_particles > 0 ? num_particles : 1));
    if (!cl->head || !cl->next) {
        cell_list_free(cl);
        return NULL;
    }
    return cl;
}

void cell_list_free(CellList *cl)
{
    if (!cl) return;
    std::free(cl->head);
    std::free(cl->next);
    std::free(cl);
}

// The device search uses the session grid (cell size = list radius from
// g_config, domain from g_config), which is the grid cell_list_create builds
// for simulation_run's call; `cl` receives the same chains.
void neighbor_search_cell_linked_list(NeighborList *nl, ParticleSystem *ps, CellList *cl, double re)
{
    (void)re;
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, false)) return;
    if (!ok("mps_neighbor_search", mps_neighbor_search(c->s), c->s)) return;
    if (!ok("mps_get_neighbor_list", mps_get_neighbor_list(c->s, nl->neighbors, nl->count, nl->max_neighbors), c->s))
        return;
    if (cl) ok("mps_get_cell_links", mps_get_cell_links(c->s, cl->head, cl->next, cl->total_cells), c->s);
}

// All pairs closer than re, in ascending index (neighbor_search.c:44-81).
// Served by the device cell search, whose cells are at least re wide, with
// each row put in ascending order; re must not exceed the list radius.
void neighbor_search_brute_force(NeighborList *nl, ParticleSystem *ps, double re)
{
    if (re > list_radius()) {
        fail("neighbor_search_brute_force (re above the list radius)", MPS_ERR_UNSUPPORTED, nullptr);
        return;
    }
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, false)) return;
    if (!ok("mps_neighbor_search", mps_neighbor_search(c->s), c->s)) return;
    int m = nl->max_neighbors;
    if (!ok("mps_get_neighbor_list", mps_get_neighbor_list(c->s, nl->neighbors, nl->count, m), c->s)) return;
    double re2 = re * re;
    for (int i = 0; i < ps->num; i++) {
        int *row = nl->neighbors + (size_t)i * m;
        int k = 0;
        for (int q = 0; q < nl->count[i]; q++) {
            int j = row[q];
            double r2 = 0.0;
            for (int d = 0; d < D; d++) {
                double t = ps->particles[j].pos[d] - ps->particles[i].pos[d];
                r2 += t * t;
            }
            if (r2 < re2) row[k++] = j;
        }
        std::vector<int> tmp(row, row + k);
        std::sort(tmp.begin(), tmp.end());
        std::copy(tmp.begin(), tmp.end(), row);
        nl->count[i] = k;
    }
}

// ---- operators, PPE, boundary (GPU) -------------------------------------------------

void calc_particle_number_density(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_DENSITY, 0.0, false, "calc_particle_number_density");
}

void calc_viscosity_term(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_VISCOSITY, 0.0, true, "calc_viscosity_term");
}

void calc_pressure_gradient(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_GRADIENT, 0.0, true, "calc_pressure_gradient");
}

void judge_free_surface(ParticleSystem *ps, double threshold)
{
    stage(ps, nullptr, MPS_STAGE_SURFACE, threshold, true, "judge_free_surface");
}

void calc_neighbor_count(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_NEIGHBOR_COUNT, 0.0, false, "calc_neighbor_count");
}

void judge_free_surface_by_count(ParticleSystem *ps, double beta)
{
    stage(ps, nullptr, MPS_STAGE_SURFACE_BY_COUNT, beta, true, "judge_free_surface_by_count");
}

void clamp_pressure(ParticleSystem *ps) { stage(ps, nullptr, MPS_STAGE_CLAMP, 0.0, false, "clamp_pressure"); }

#if D == 3
void collision(ParticleSystem *ps, NeighborList *nl) { stage(ps, nl, MPS_STAGE_COLLISION, 0.0, false, "collision"); }
#else
void collision(ParticleSystem *ps) { stage(ps, nullptr, MPS_STAGE_COLLISION, 0.0, false, "collision"); }
#endif

// The coefficients come from the caller's particle system (ps->C_LL,
// ps->C_SL), as the reference's functions read them.
void calc_surface_tension(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_SURFACE_TENSION, ps->C_LL, false, "calc_surface_tension");
}

void calc_surface_tension_SL(ParticleSystem *ps, NeighborList *nl)
{
    if (ps->C_SL == 0.0) return;
    stage(ps, nl, MPS_STAGE_SURFACE_TENSION_SL, ps->C_SL, false, "calc_surface_tension_SL");
}

void solve_pressure(ParticleSystem *ps, NeighborList *nl)
{
    stage(ps, nl, MPS_STAGE_SOLVE_PRESSURE, 0.0, true, "solve_pressure");
}

void apply_wall_boundary(ParticleSystem *ps) { stage(ps, nullptr, MPS_STAGE_WALL, 0.0, false, "apply_wall_boundary"); }

#if D == 3
void remove_out_of_bounds(ParticleSystem *ps, double xmin, double xmax, double ymin, double ymax, double zmin,
                          double zmax)
#else
void remove_out_of_bounds(ParticleSystem *ps, double xmin, double xmax, double ymin, double ymax)
#endif
{
    if (!g_config) {
        fail("remove_out_of_bounds (g_config is not set)", MPS_ERR_INVALID, nullptr);
        return;
    }
    mps_params_t p = params_from(g_config);
    p.domain_min[0] = xmin;
    p.domain_max[0] = xmax;
    p.domain_min[1] = ymin;
    p.domain_max[1] = ymax;
#if D == 3
    p.domain_min[2] = zmin;
    p.domain_max[2] = zmax;
#endif
    Ctx *c = ctx_for(ps, &p);
    if (!c || !upload(c, ps, false)) return;
    if (!ok("remove_out_of_bounds", mps_run_stage(c->s, MPS_STAGE_OUT_OF_BOUNDS, nullptr, nullptr, 0, 0.0), c->s))
        return;
    download(c, ps);
}

// ---- time stepping -----------------------------------------------------------------

// One step; the caller's `nl` is the previous step's list (used by the
// viscosity and 3-D collision stages) and receives the new one, `cl` the new
// chains (simulation.c:19-118).
void simulation_step(ParticleSystem *ps, NeighborList *nl, CellList *cl, int step)
{
    (void)step;
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, true)) return;
    if (!ok("simulation_step", mps_step_with_list(c->s, nl->neighbors, nl->count, nl->max_neighbors), c->s)) return;
    if (!download(c, ps)) return;
    if (!ok("mps_get_neighbor_list", mps_get_neighbor_list(c->s, nl->neighbors, nl->count, nl->max_neighbors), c->s))
        return;
    if (cl) ok("mps_get_cell_links", mps_get_cell_links(c->s, cl->head, cl->next, cl->total_cells), c->s);
}

// The whole run with the state resident on the device; particles come back
// to the host only at output steps (simulation.c:123-181).
void simulation_run(ParticleSystem *ps)
{
    if (!g_config) {
        fail("simulation_run (g_config is not set)", MPS_ERR_INVALID, nullptr);
        return;
    }
    double dt = g_config->dt;
    int total_steps = (int)(g_config->t_end / dt);
    int out_interval = g_config->output_interval;
    const char *out_dir = g_config->output_dir;
    Ctx *c = ctx_for(ps);
    if (!c || !upload(c, ps, true)) return;
    std::printf("B200: device-resident time stepping\n");
    if (!ok("mps_neighbor_search", mps_neighbor_search(c->s), c->s)) return;
    output_csv(ps, 0, out_dir);
    output_vtk(ps, 0, out_dir);
    std::printf("Starting simulation (%dD, B200): %d steps, dt = %.2e\n", D, total_steps, dt);
    for (int step = 1; step <= total_steps; step++) {
        if (!ok("mps_step", mps_step(c->s, 1), c->s)) return;
        if (out_interval > 0 && step % out_interval == 0) {
            if (!download(c, ps)) return;
            int fluid = 0;
            for (int i = 0; i < ps->num; i++) fluid += ps->particles[i].type == MPS_FLUID;
            std::printf("Step %6d / %d  (t = %.4f s)  fluid particles: %d\n", step, total_steps, step * dt, fluid);
            output_csv(ps, step, out_dir);
            output_vtk(ps, step, out_dir);
        }
    }
    download(c, ps);
    std::printf("Simulation complete.\n");
}

// ---- output files (io.c:10-107 formats) ----------------------------------------------

void output_csv(const ParticleSystem *ps, int step, const char *output_dir)
{
    char fn[256];
    std::snprintf(fn, sizeof(fn), "%s/output_%06d.csv", output_dir, step);
    FILE *fp = std::fopen(fn, "w");
    if (!fp) {
        std::fprintf(stderr, "Error: cannot open %s\n", fn);
        return;
    }
#if D == 3
    std::fprintf(fp, "x,y,z,vx,vy,vz,pressure,type\n");
#else
    std::fprintf(fp, "x,y,vx,vy,pressure,type\n");
#endif
    for (int i = 0; i < ps->num; i++) {
        const Particle *p = &ps->particles[i];
        if (p->type == MPS_GHOST) continue;
#if D == 3
        std::fprintf(fp, "%.8e,%.8e,%.8e,%.8e,%.8e,%.8e,%.8e,%d\n", p->pos[0], p->pos[1], p->pos[2], p->vel[0],
                     p->vel[1], p->vel[2], p->pressure, p->type);
#else
        std::fprintf(fp, "%.8e,%.8e,%.8e,%.8e,%.8e,%d\n", p->pos[0], p->pos[1], p->vel[0], p->vel[1], p->pressure,
                     p->type);
#endif
    }
    std::fclose(fp);
}

void output_vtk(const ParticleSystem *ps, int step, const char *output_dir)
{
    char fn[256];
    std::snprintf(fn, sizeof(fn), "%s/output_%06d.vtk", output_dir, step);
    int count = 0;
    for (int i = 0; i < ps->num; i++) count += ps->particles[i].type != MPS_GHOST;
    FILE *fp = std::fopen(fn, "w");
    if (!fp) {
        std::fprintf(stderr, "Error: cannot open %s\n", fn);
        return;
    }
    std::fprintf(fp, "# vtk DataFile Version 3.0\n");
#if D == 3
    std::fprintf(fp, "MPS 3D Simulation Step %d\n", step);
#else
    std::fprintf(fp, "MPS Simulation Step %d\n", step);
#endif
    std::fprintf(fp, "ASCII\n");
    std::fprintf(fp, "DATASET UNSTRUCTURED_GRID\n");
    std::fprintf(fp, "POINTS %d double\n", count);
    for (int i = 0; i < ps->num; i++) {
        const Particle *p = &ps->particles[i];
        if (p->type == MPS_GHOST) continue;
#if D == 3
        std::fprintf(fp, "%.8e %.8e %.8e\n", p->pos[0], p->pos[1], p->pos[2]);
#else
        std::fprintf(fp, "%.8e %.8e 0.0\n", p->pos[0], p->pos[1]);
#endif
    }
    std::fprintf(fp, "CELLS %d %d\n", count, count * 2);
    int idx = 0;
    for (int i = 0; i < ps->num; i++) {
        if (ps->particles[i].type == MPS_GHOST) continue;
        std::fprintf(fp, "1 %d\n", idx++);
    }
    std::fprintf(fp, "CELL_TYPES %d\n", count);
    for (int i = 0; i < count; i++) std::fprintf(fp, "1\n");
    std::fprintf(fp, "POINT_DATA %d\n", count);
    std::fprintf(fp, "SCALARS pressure double 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < ps->num; i++) {
        if (ps->particles[i].type == MPS_GHOST) continue;
        std::fprintf(fp, "%.8e\n", ps->particles[i].pressure);
    }
    std::fprintf(fp, "SCALARS type int 1\n");
    std::fprintf(fp, "LOOKUP_TABLE default\n");
    for (int i = 0; i < ps->num; i++) {
        if (ps->particles[i].type == MPS_GHOST) continue;
        std::fprintf(fp, "%d\n", ps->particles[i].type);
    }
    std::fprintf(fp, "VECTORS velocity double\n");
    for (int i = 0; i < ps->num; i++) {
        const Particle *p = &ps->particles[i];
        if (p->type == MPS_GHOST) continue;
#if D == 3
        std::fprintf(fp, "%.8e %.8e %.8e\n", p->vel[0], p->vel[1], p->vel[2]);
#else
        std::fprintf(fp, "%.8e %.8e 0.0\n", p->vel[0], p->vel[1]);
#endif
    }
    std::fclose(fp);
}

}  // extern "C"
