// device.cuh -- shared device-side definitions of the MPS engine.
//
// All FP64 particle arithmetic here reproduces the reference's operation
// order (mps_fluid3D_parallel/src/operators.c, kernel.c) and the library is
// compiled with --fmad=false, so products and sums are never contracted into
// FMAs: neighbour sets, cell indices, number densities, surface flags and the
// PPE matrix come out bit-identical to the reference for identical inputs.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <cstdlib>

namespace mps {

// Every kernel of the library is launched through launch(), which counts
// launches process-wide (mps_launch_count in the C ABI).
inline unsigned long long &launch_counter()
{
    static unsigned long long c = 0;
    return c;
}

template <class... KArgs, class... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
{
    kernel<<<grid, block, smem, st>>>(args...);
    ++launch_counter();
}

// Programmatic dependent launch (sm_90+): the kernel may be scheduled while
// its predecessor in the stream is still running.  Kernels launched this way
// call pdl_trigger() first, load only data that no earlier kernel of the
// chain writes, then call pdl_wait() on every path -- after it the
// predecessor grid has completed and its writes are visible -- before they
// read anything a predecessor produced or return.  MPS_PDL=0 in the
// environment launches them as ordinary kernels (same results, bit for bit).
inline bool pdl_enabled()
{
    static const bool on = [] {
        const char *e = std::getenv("MPS_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args)
{
    if (!pdl_enabled()) {
        launch(kernel, grid, block, smem, st, args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
    ++launch_counter();
}

// griddepcontrol (PTX ISA 7.8): both are no-ops in a kernel launched
// without the programmatic attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

enum : int { FLUID = 0, WALL = 1, GHOST = 2, DUMMY = 3 };

// Device error bits (Engine::err_), turned into MPS_ERR_* codes on the host.
enum : unsigned {
    ERR_NEIGHBOR_OVERFLOW = 1u,   // > max_neighbors in some list (neighbor_search.c:221)
    ERR_UNKNOWN_OFF_GRID  = 2u,   // a PPE unknown outside the cell grid
    ERR_LIST_MISMATCH     = 4u,   // caller list differs from the cell structure
    ERR_COLORING          = 8u,   // matrix couples two same-coloured cells
    ERR_CELL_OVERFULL     = 16u,  // more than 255 unknowns in one cell
    ERR_COPY_TIMEOUT      = 32u,  // a bulk copy into shared memory did not complete in time
    ERR_GRID_TIMEOUT      = 128u, // a grid barrier of the persistent PCG kernel did not complete in time
};

// Constants of one session, evaluated on the host with the reference's
// expressions (so each equals the reference's value bit for bit).
struct Consts {
    double l0;
    double rmin;          // 0.01 * l0                         kernel.c:15
    double re_lap, re_n;
    double re_list2;      // re*re of the list radius         neighbor_search.c:150
    double re_n2;         // re_n*re_n                        operators.c:228
    double coeff;         // 2*DIM/(n0*lambda)                operators.c:55, pressure_solver.c:374
    double visc_coeff;    // viscosity*coeff                  operators.c:82
    double grad_coeff;    // DIM/n0                           operators.c:106
    double neg_grad;      // -grad_coeff                      operators.c:176
    double density;
    double gravity[3];
    double dt;
    double col2;          // (ratio*l0)^2                     operators.c:375
    double col_rmin;      // 1e-12*l0                         operators.c:417
    double half1pe;       // (1+e)*0.5                        operators.c:425
    double grad_r2min;    // l0*l0*1e-12                      operators.c:153
    double surf_thr;      // threshold*n0                     operators.c:214
    double count_thr;     // beta*n0_count                    operators.c:262
    double diag_scale;    // c_ppe*coeff (ppe_type 1) or coeff
    double neg_coeff;     // -coeff                           pressure_solver.c:510
    double rhs_k;         // relaxation*(density/dt^2)        pressure_solver.c:337
    double rhs_hs;        // -(density/n0/dt)                 pressure_solver.c:361
    double rhs_na;        // -density/dt                      pressure_solver.c:333
    double rhs_nb;        // gamma*(density/dt^2)             pressure_solver.c:334
    double n0;
    double oob_lo[3], oob_hi[3];   // domain -/+ l0*(wall_layers+1)  boundary.c:25
    int    max_nb;
    int    ppe_type, hs_mode, cmps, surf_method, clamp;
    int    collision_on;
    int    drive_on, drive_axis;   // driven walls (A != 0) and their axis
    int    st_on, st_sl_on;        // surface tension; its wall term (C_SL != 0)
    double st_ll, st_sl;           // C_LL / (rho l0^D), C_SL / (rho l0^D)   operators.c:284, :326
    double re_st, st_rmin;         // influence_radius_st, 1e-9 * l0          operators.c:303
    int    fr_on;                  // contact-line friction (3-D serial variant operators.c:337)
    double fr_theta_s, fr_dtheta;  // wetting angle, critical deviation (radians)   :341-342
    double fr_vc, fr_dyn;          // velocity threshold; alpha nu 2D / (n0 lambda)  :343-346
};

// Structure-of-arrays particle state.  `key` holds the positions at the
// last cell sort and `cell` the cell each particle was binned into then (-1:
// not binned); list membership is always decided on them, which reproduces
// the reference's use of the previous step's list in the explicit stage.
template <int D>
struct State {
    double *pos[D];
    double *vel[D];
    double *acc[D];
    double *key[D];
    double *p;
    double *n;
    int    *type;
    int    *surf;
    int    *ncount;
    int    *id;       // reference particle index
    int    *cell;
};

template <int D>
struct Grid {
    double origin[D];
    double cs_inv;    // 1.0 / cell_size                  neighbor_search.c:155
    int    dims[D];
    int    total;
    const int *start; // [total + 2] first engine index of each cell
};

// Squared distance ((0 + dx^2) + dy^2) + dz^2 with dx = pj - pi.
template <int D>
__device__ __forceinline__ double dist2(const double *pi, const double *pj)
{
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        double t = pj[d] - pi[d];
        s += t * t;
    }
    return s;
}

template <int D>
__device__ __forceinline__ double dist2v(const double *pi, const double *pj, double *dr)
{
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < D; d++) {
        dr[d] = pj[d] - pi[d];
        s += dr[d] * dr[d];
    }
    return s;
}

// kernel.c:12-20.  IEEE division and square root (default -prec-div and
// -prec-sqrt) match the CPU's correctly rounded results.
__device__ __forceinline__ double kweight(double r, double re, double rmin)
{
    if (r >= re) return 0.0;
    if (r < rmin) r = rmin;
    return re / r - 1.0;
}

template <int D>
__device__ __forceinline__ void load_vec(double *out, double *const *a, int i)
{
#pragma unroll
    for (int d = 0; d < D; d++) out[d] = a[d][i];
}

// Cell of a position, the reference's (int)((p - origin) * cs_inv) with its
// range test; -1 outside the grid (NaN and out-of-range values included,
// which C leaves undefined and x86 maps to INT_MIN, i.e. rejected).
template <int D>
__device__ __forceinline__ int cell_of_pos(const Grid<D> &g, const double *p)
{
    int lin = 0;
#pragma unroll
    for (int d = D - 1; d >= 0; d--) {
        double t = (p[d] - g.origin[d]) * g.cs_inv;
        if (!(t > -1.0 && t < 2147483647.0)) return -1;
        int c = __double2int_rz(t);
        if (c < 0 || c >= g.dims[d]) return -1;
        lin = lin * g.dims[d] + c;
    }
    return lin;
}

// Neighbour candidates from the cell structure: the 3^D block of cells in
// the reference's scan order (z, y, x from outer to inner, clamped at the
// grid edge); within a cell, engine order is descending reference index, the
// order of the reference's prepend-built chains.  The x-neighbours of a cell
// are contiguous, so each (z, y) pair is one run.  Members pass
// r2(key_i, key_j) < re^2.
template <int D>
struct CellSource {
    Grid<D> g;
    const double *key[D];
    const int *cell;
    double re2;

    template <class F>
    __device__ __forceinline__ void for_each(int i, F &&f) const
    {
        int c = cell[i];
        if (c < 0) return;
        double ki[D];
#pragma unroll
        for (int d = 0; d < D; d++) ki[d] = key[d][i];
        int cc[D];
        int rem = c;
#pragma unroll
        for (int d = 0; d < D; d++) { cc[d] = rem % g.dims[d]; rem /= g.dims[d]; }
        int x0 = cc[0] > 0 ? cc[0] - 1 : 0;
        int x1 = cc[0] < g.dims[0] - 1 ? cc[0] + 1 : g.dims[0] - 1;
        int y0 = cc[1] > 0 ? cc[1] - 1 : 0;
        int y1 = cc[1] < g.dims[1] - 1 ? cc[1] + 1 : g.dims[1] - 1;
        int z0 = 0, z1 = 0;
        if (D == 3) {
            z0 = cc[D - 1] > 0 ? cc[D - 1] - 1 : 0;
            z1 = cc[D - 1] < g.dims[D - 1] - 1 ? cc[D - 1] + 1 : g.dims[D - 1] - 1;
        }
        for (int z = z0; z <= z1; z++) {
            for (int y = y0; y <= y1; y++) {
                int base = (D == 3) ? (z * g.dims[1] + y) * g.dims[0] : y * g.dims[0];
                int t0 = g.start[base + x0], t1 = g.start[base + x1 + 1];
                for (int t = t0; t < t1; t++) {
                    if (t == i) continue;
                    double kt[D];
#pragma unroll
                    for (int d = 0; d < D; d++) kt[d] = key[d][t];
                    if (dist2<D>(ki, kt) < re2) f(t);
                }
            }
        }
    }
};

// Neighbours from a caller-supplied list (CSR of the reference's
// NeighborList, entries in engine indices).
struct ListSource {
    const int *ptr;
    const int *idx;

    template <class F>
    __device__ __forceinline__ void for_each(int i, F &&f) const
    {
        int e = ptr[i + 1];
        for (int k = ptr[i]; k < e; k++) f(idx[k]);
    }
};

// ---- deterministic reductions -------------------------------------------
// Block partials land in fixed slots and the last block to finish adds them
// in slot order, so every rerun produces the same bits.

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double *sh)
{
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (lane < BLOCK / 32) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;   // valid in thread 0
}

// True in every thread of the last block to arrive (which then owns
// partials[0..nblocks)); the ticket is reset for the next launch.
__device__ __forceinline__ bool last_block(unsigned *ticket, unsigned nblocks)
{
    __shared__ bool last;
    __threadfence();
    if (threadIdx.x == 0) {
        unsigned t = atomicAdd(ticket, 1u);
        last = (t == nblocks - 1);
        if (last) *ticket = 0u;
    }
    __syncthreads();
    return last;
}

}  // namespace mps
