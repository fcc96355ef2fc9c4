// engine.cu -- the device-resident MPS time step on sm_100a and its C ABI.
//
// One Engine<D> owns a particle system in HBM as structure-of-arrays, kept
// sorted by (cell, descending reference index) and re-sorted at every
// neighbour search.  A step is (mps_fluid3D_parallel/src/simulation.c:19-118):
//
//   viscosity + gravity        k_viscosity       previous step's structure
//   explicit u*, r*            k_explicit_update
//   collision                  k_collision_*     previous structure (3-D) or
//                                                a fresh sort (2-D all-pairs)
//   neighbour search           sort()            counting sort by cell
//   number density + surface   k_density
//   PPE                        ppe()             assembly, IC(0), PCG
//   clamp (optional)           k_writeback
//   pressure gradient          k_pmin, k_gradient
//   correction, wall, ghosts   k_correct
//
// All work is issued on one stream; the host synchronises twice per step
// to size the PPE (n_eq, nnz) and once per CG batch to test convergence.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>

#include "engine.cuh"
#include "k_ops.cuh"
#include "k_ppe.cuh"
#include "k_pcg.cuh"
#include "k_sort.cuh"
#include "k_adj.cuh"

namespace mps {

static inline int nblk(long long n, int b) { return (int)((n + b - 1) / b); }

// The neighbour-list radius (simulation.c:22-24): the largest active radius.
static double list_radius(const mps_params_t &p)
{
    double re = std::fmax(p.influence_radius_lap, p.influence_radius_n);
    if (p.surface_tension_enabled) re = std::fmax(re, p.influence_radius_st);
    return re;
}

// Surface-tension coefficients of particle.c:185-211 (2-D particle.c:154-180):
// the potential's interaction energy summed over lattice pairs across a flat
// interface, C_LL = sigma l0^(D-1) / sum, C_SL = (1 + cos theta) / 2 C_LL;
// the same expressions in the same order, so the values are the reference's.
static void surface_tension_coeffs(const mps_params_t &p, double *cll, double *csl)
{
    *cll = 0.0;
    *csl = 0.0;
    if (!p.surface_tension_enabled) return;
    double l0 = p.particle_distance, re_st = p.influence_radius_st;
    int nmax = (int)std::ceil(re_st / l0);
    double sum = 0.0;
    for (int dxa = 1; dxa <= nmax; dxa++)
        for (int dxb = -(nmax - 1); dxb <= 0; dxb++)
            for (int dyb = -nmax; dyb <= nmax; dyb++)
                for (int dzb = (p.dim == 3 ? -nmax : 0); dzb <= (p.dim == 3 ? nmax : 0); dzb++) {
                    double rx = (double)(dxa - dxb) * l0;
                    double ry = (double)dyb * l0;
                    double rab;
                    if (p.dim == 3) {
                        double rz = (double)dzb * l0;
                        rab = std::sqrt(rx * rx + ry * ry + rz * rz);
                    } else {
                        rab = std::sqrt(rx * rx + ry * ry);
                    }
                    if (rab > 0.0 && rab < re_st)
                        sum += (1.0 / 3.0) * (rab - 1.5 * l0 + 0.5 * re_st) * (rab - re_st) * (rab - re_st);
                }
    if (sum > 0.0) {
        *cll = (p.dim == 3) ? p.surface_tension_coeff * l0 * l0 / sum : p.surface_tension_coeff * l0 / sum;
        double theta = p.wetting_angle_SL * M_PI / 180.0;
        *csl = 0.5 * (1.0 + std::cos(theta)) * *cll;
    }
}

constexpr int TPB = 256;             // threads per block, particle kernels
constexpr int RED_BLOCKS = 148 * 8;  // fixed grid of the reduction kernels: full occupancy at 256 threads
constexpr int CG_BATCH = 8;          // CG iterations between convergence reads

template <int D>
struct AosLayout {
    static constexpr int size = (24 * D + 28 + 7) / 8 * 8;   // 104 (3-D), 80 (2-D)
    static constexpr int pos = 0, vel = 8 * D, acc = 16 * D, pressure = 24 * D, n = 24 * D + 8,
                         ncount = 24 * D + 16, type = 24 * D + 20, surf = 24 * D + 24;
};

template <int D>
__global__ void k_unpack(const unsigned char *__restrict__ aos, State<D> s, int num)
{
    using L = AosLayout<D>;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num) return;
    const unsigned char *r = aos + (size_t)i * L::size;
#pragma unroll
    for (int d = 0; d < D; d++) {
        double x = *(const double *)(r + L::pos + 8 * d);
        s.pos[d][i] = x;
        s.key[d][i] = x;
        s.vel[d][i] = *(const double *)(r + L::vel + 8 * d);
        s.acc[d][i] = *(const double *)(r + L::acc + 8 * d);
    }
    s.p[i] = *(const double *)(r + L::pressure);
    s.n[i] = *(const double *)(r + L::n);
    s.ncount[i] = *(const int *)(r + L::ncount);
    s.type[i] = *(const int *)(r + L::type);
    s.surf[i] = *(const int *)(r + L::surf);
    s.id[i] = i;
    s.cell[i] = -1;
}

template <int D>
__global__ void k_pack(unsigned char *__restrict__ aos, State<D> s, int num)
{
    using L = AosLayout<D>;
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= num) return;
    unsigned char *r = aos + (size_t)s.id[q] * L::size;
#pragma unroll
    for (int d = 0; d < D; d++) {
        *(double *)(r + L::pos + 8 * d) = s.pos[d][q];
        *(double *)(r + L::vel + 8 * d) = s.vel[d][q];
        *(double *)(r + L::acc + 8 * d) = s.acc[d][q];
    }
    *(double *)(r + L::pressure) = s.p[q];
    *(double *)(r + L::n) = s.n[q];
    *(int *)(r + L::ncount) = s.ncount[q];
    *(int *)(r + L::type) = s.type[q];
    *(int *)(r + L::surf) = s.surf[q];
    *(int *)(r + L::surf + 4) = 0;
}

template <int D>
__global__ void k_unpack_soa(const double *__restrict__ pos, const double *__restrict__ vel,
                             const int *__restrict__ type, State<D> s, int num)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= num) return;
#pragma unroll
    for (int d = 0; d < D; d++) {
        double x = pos[(size_t)i * D + d];
        s.pos[d][i] = x;
        s.key[d][i] = x;
        s.vel[d][i] = vel[(size_t)i * D + d];
        s.acc[d][i] = 0.0;
    }
    s.p[i] = 0.0;
    s.n[i] = 0.0;
    s.ncount[i] = 0;
    s.type[i] = type[i];
    s.surf[i] = 0;
    s.id[i] = i;
    s.cell[i] = -1;
}

template <int D>
__global__ void k_pressure_ref(State<D> s, int num, double *__restrict__ out)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < num) out[s.id[q]] = s.p[q];
}

__global__ void k_cell_links(const int *__restrict__ start, const int *__restrict__ id, const int *__restrict__ cell,
                             int total, int n, int *__restrict__ head, int *__restrict__ next)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < total) {
        int b = start[q], e = start[q + 1];
        head[q] = (b < e) ? id[b] : -1;
    }
    if (q < n) {
        int c = cell[q];
        int nx = -1;
        if (c >= 0 && q + 1 < start[c + 1]) nx = id[q + 1];
        next[id[q]] = nx;
    }
}

// CSR rows in the reference's numbering (for parity checks): row of
// reference particle i = eq[i]; columns renumbered, then sorted by the host.
__global__ void k_ppe_to_ref(int n_eq, const int *__restrict__ part_of_row, const int *__restrict__ id,
                             const int *__restrict__ eq_by_id, const int *__restrict__ row_ptr,
                             const int *__restrict__ col, const double *__restrict__ val,
                             const double *__restrict__ b, const int *__restrict__ part_of_col_row,
                             const int *__restrict__ ref_row_ptr, int *__restrict__ out_col,
                             double *__restrict__ out_val, double *__restrict__ out_b)
{
    int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_eq) return;
    int i = id[part_of_row[r]];
    int er = eq_by_id[i];
    int o = ref_row_ptr[er];
    for (int q = row_ptr[r]; q < row_ptr[r + 1]; q++) {
        out_col[o] = eq_by_id[id[part_of_col_row[col[q]]]];
        out_val[o] = val[q];
        o++;
    }
    out_b[er] = b[r];
}

template <int D>
class Engine final : public EngineBase {
public:
    Engine(const mps_params_t &p, int capacity);
    ~Engine() override;
    int dim() const override { return D; }
    void update_params(const mps_params_t &p) override;
    void upload_aos(const void *aos, int num) override;
    void download_aos(void *aos, int num) override;
    void upload_soa(const double *pos, const double *vel, const int *type, int num) override;
    void download_pressure(double *p, int num) override;
    void compute_initial_params(double *n0, double *lambda, int *n0_count) override;
    void set_initial_params(double n0, double lambda, int n0_count) override;
    void neighbor_search() override;
    void step(int nsteps) override;
    void step_with_list(const int *nb, const int *cnt, int max_nb) override;
    void get_neighbor_list(int *nb, int *cnt, int max_nb) override;
    void get_cell_index(int *cell) override;
    void get_cell_links(int *head, int *next, int total) override;
    // the window tables keep the window they were built with (win_), so a
    // change between the factorisation and the solve stays consistent
    void set_precision(int precision) override { prm_.precision = precision; }
    void get_ppe(int *eq_idx, int *row_ptr, int *col, double *val, double *b, int *n_eq,
                 long long *nnz) override;
    void run_stage(int stage, const int *nb, const int *cnt, int max_nb, double arg) override;
    void get_ic0(int *row_ptr, int *col, double *A, double *F, double *b, int *n_eq, long long *nnz) override;
    void get_cell_blocks(int *cells, int *inv_off, double *inv, int *colour_rows, int *ncells,
                         long long *ninv) override;
    void apply_preconditioner(const double *r, double *z) override;
    cudaStream_t stream() const override { return st_; }
    size_t state_bytes() const override;
    void state_save(void *dst) override;
    void state_load(const void *src) override;
    void adjoint_seed(const double *lam_pos, const double *lam_vel) override;
    void adjoint_pressure_seed(const double *dLdP, int num) override;
    void step_adjoint() override;
    void adjoint_get(double *lam_pos, double *lam_vel, double *grad_gravity, double *grad_viscosity,
                     double *grad_drive) override;

private:
    // ---- configuration
    mps_params_t prm_{};
    Consts k_{};
    Grid<D> g_{};
    double re_list_ = 0.0;
    double n0_ = 0.0, lambda_ = 0.0;
    int n0_count_ = 0;
    bool have_ref_ = false;
    int cap_ = 0, n_ = 0;
    cudaStream_t st_ = nullptr;

    // ---- particle state, double-buffered across sorts
    DevArray<double> dbuf_[2];
    DevArray<int> ibuf_[2];
    State<D> S_[2];
    int cur_ = 0;
    bool structure_ = false;   // cell structure valid for S_[cur_]

    // ---- sort
    DevArray<int> kcell_, count_, start_, cursor_, excl_, exoff_, tmp_, perm_, where_, scanws_;
    DevArray<long long> scanws64_;

    // ---- block colouring
    DevArray<int> ccells_, color_off_dev_, aflag_, apos_, acells_, sizes_;
    std::vector<int> color_off_;   // cells of each colour in ccells_
    std::vector<int> act_off_;     // cells with unknowns of each colour in acells_
    std::vector<int> row_off_;     // first row of each colour
    DevArray<int> inpos_, outpos_, pk_len_lo_, pk_len_up_, pk_off_lo_, pk_off_up_;
    DevArray<double> pk_val_lo_, pk_val_up_, dinv_;
    DevArray<unsigned char> pk_k_lo_, pk_k_up_;
    DevArray<int2> adesc_;
    DevArray<int> xlen_lo_, xlen_up_, xp_lo_, xp_up_, xc_lo_, xc_up_;   // packed cross-cell runs (CSR)
    DevArray<int> xs_lo_, xs_up_;                                        // head/tail split of each run
    DevArray<double> xf_lo_, xf_up_;
    DevArray<int> inv_len_, inv_off_;        // in-cell block inverses: entries, offsets per active cell
    DevArray<double> inv_cm_, inv_rm_;       // column-major (forward) and row-major (backward) copies
    DevArray<int> colinv_, wfirst_;          // inverse offsets at colour boundaries; first cell per window
    // jagged-diagonal cross blocks of the warp-per-cell sweep: diagonals per
    // cell (jlen_, its scan jdc_*), diagonal slots (jdp_*), row of each rank
    DevArray<int> jlen_, jdc_lo_, jdc_up_, jdp_lo_, jdp_up_;
    DevArray<unsigned char> jperm_lo_, jperm_up_;
    // ICCG loop (MPS_SWEEP): 2 the persistent k_pcg (one cooperative launch
    // per batch of iterations), 0 the launch-per-colour k_sweep_colour with
    // separate SpMV and vector kernels, 1 the same with the CTA-per-cell
    // k_sweep_cell over jagged-diagonal cross blocks
    int sweep_mode_ = 0;
    DevArray<unsigned> pcg_bar_;   // grid-barrier counter of k_pcg
    DevArray<unsigned long long> pcg_trace_;    // k_pcg phase timestamps while profiling
    std::vector<unsigned long long> trace_host_;
    int pcg_batch_ = 16;           // k_pcg iterations per launch (MPS_PCG_BATCH)
    int pcg_grid_[3] = {0, 0, 0};  // k_pcg grid per variant (FP64; FP32 difference form; FP32)
    // polls of a k_pcg grid-barrier wait (MPS_TEST_BAR_POLLS lowers it, down
    // to 0, to exercise the timeout path)
    int bar_polls_ = PCG_BAR_POLLS;
    // entries per lane loaded in one batch by k_sweep_colour's head sums
    // (MPS_SWEEP_HB: 4 or 8)
    int head_batch_ = 4;
    // CTAs per SM the colour sweep is compiled for (MPS_SWEEP_OCC: 6 or 8;
    // 0 = by storage type)
    int sweep_occ_ = 0;
    // head rows per lane group of the colour sweep (MPS_SWEEP_HR: 1 or 2); 2
    // measured at c2: FP64 sweeps 3 % faster, FP32 forward 4 % faster and
    // backward level, results bit-identical
    int head_rows_ = 2;
    // polls of the first wait for a staged block inverse (MPS_TEST_MBAR_POLLS
    // lowers it, down to 0, to exercise the timeout path)
    int first_polls_ = MBAR_POLLS;
    // k_sweep_cell lets its dependent launch start at its beginning (1) or
    // only as its CTAs exit (0); MPS_CELL_EARLY overrides
    int cell_early_ = 0;
    int num_sms_ = 148;
    std::vector<int> nwin_, win_off_;        // windows per colour, their table offsets


    // ---- PPE
    DevArray<int> ucount_, ucol_, rs_, cell_row0_, row_of_, part_of_row_, rcount_, row_ptr_, diagpos_, col_;
    DevArray<double> A_, F_, b_, x_, r_, z_, p_, Ap_, y_, part_, partials_, p2_;
    DevArray<float> A32_, xf32_lo_, xf32_up_, pkv32_lo_, pkv32_up_, inv32_cm_, inv32_rm_, dinv32_;
    DevArray<double> zprev_, dsum_;
    DevArray<uint2> ac32_, xfc32_lo_, xfc32_up_;   // packed FP32 matrix and cross runs (mixed form)
    // mixed form: the FP32 matrix and cross runs as packed 8-byte words (1,
    // default) or as separate value and column arrays (0; MPS_PACK)
    int pack_ = 1;
    bool packed_ = false;   // the last mixed solve used the packed words
    DevArray<CGScalars> sc_;
    DevArray<unsigned> ticket_, err_;
    int n_eq_ = 0;
    long long nnz_ = 0;
    int nx_lo_ = 0, nx_up_ = 0;   // entries of the packed cross-cell runs
    int ninv_ = 0;            // entries of the in-cell block inverses
    // lanes per row of the CG SpMV: MPS_SPMV_LPR (8, 16 or 32) if set, else 8
    // in FP64 and 16 in the mixed form's FP32 solve
    int spmv_lpr_ = 0;
    // mixed form: residual reduction between reliable updates (MPS_RELIABLE_DELTA
    // overrides) and the SpMV of its inner loop (MPS_MIXED_SPMV): 0 the FP32
    // copy of A, 1 the FP64 matrix, 2 the FP32 copy in difference form
    double rel_delta_ = kDelta;
    int mixed_spmv_ = 2;
    // CG-loop kernels launched as programmatic dependents (MPS_PDL_MASK): 2 the
    // colour sweep kernel, 4 SpMV and vector kernels
    int pdl_mask_ = 6;
    // entries per window of the staged in-cell sweep: MPS_CELL_WIN (256..4096)
    // if set, else 8 KB of inverse entries (1,024 FP64, 2,048 in the mixed
    // form's FP32 sweeps); win_ is the window of the current tables
    int cell_win_ = 0;
    int win_ = CELL_WIN;
    bool win_valid_ = false;               // the window tables match the current factor and win_
    std::vector<int> inv_col_off_;         // block-inverse offsets at the colour boundaries
    bool ppe_valid_ = false;
    bool ic0_valid_ = false;     // the IC(0) factor and its sweep tables belong to the last PPE
    bool last_fp32_ = false;     // the last solve ran the mixed form (FP32 factor copies exist)

    // ---- driven walls
    long long tstep_ = 0;                    // steps taken since the last upload (time = tstep_ dt)
    DevArray<double> rest_;                  // rest positions at upload, [axis][reference index]
    void drive_terms(double t, double *dx, double *vel) const;

    // ---- differentiation form (arrays indexed by reference particle index)
    DevArray<double> adjd_, adjsum_;
    DevArray<int> adji_;
    DevArray<double> pseed_;     // dL/dP of the step the next step_adjoint reverses (reference order)
    bool pseed_on_ = false;
    DevArray<unsigned char> snap_;           // the step's input state, for the recompute
    Adj<D> adj_{};
    size_t adj_cap_ = 0;
    bool adj_rec_ = false;                   // explicit_stage records x*, u*
    void ensure_adj();

    // ---- misc
    DevArray<double> vafter_, pmin_;
    DevArray<int> lptr_, lidx_, lout_, lcnt_;
    DevArray<int> link_head_, link_next_;   // get_cell_links output, kept across calls
    DevArray<unsigned char> aos_;
    DevArray<double> soa_in_;
    DevArray<int> int_in_;
    CGScalars *sc_host_ = nullptr;
    int *int_host_ = nullptr;
    cudaEvent_t ev_[6];
    static constexpr int PEV = 5;                 // events per profiled iteration
    cudaEvent_t pev_[CG_BATCH * PEV];

    State<D> &S() { return S_[cur_]; }
    CellSource<D> cells() const
    {
        CellSource<D> c;
        c.g = g_;
        for (int d = 0; d < D; d++) c.key[d] = S_[cur_].key[d];
        c.cell = S_[cur_].cell;
        c.re2 = k_.re_list2;
        return c;
    }

    void alloc_state();
    void build_grid();
    void compute_consts();
    void sort();
    void unsort();
    void ppe(bool clamp);
    // CG buffers: the matrix and the factor stored as TM (double in the FP64
    // form, float in the mixed form), the vectors always FP64
    template <class TM>
    struct PcgBufs {
        const TM *A, *xf_lo, *xf_up, *pkv_lo, *pkv_up, *dinv, *inv_cm, *inv_rm;
        double *x, *r, *z, *p, *Ap, *y, *part;
        const double *b;
        const double *A64 = nullptr;   // if set, the SpMV reads this FP64 matrix instead of A
        const double *dsum = nullptr;  // if set, the SpMV is in difference form with these row sums
        // FP32 only: packed (value bits, column) words of the matrix and of
        // the cross runs; if set, the SpMV and the colour sweeps read these
        const uint2 *ac = nullptr, *xfc_lo = nullptr, *xfc_up = nullptr;
    };
    template <class TM>
    void pcg_solve(const PcgBufs<TM> &v, double tol, int maxit, bool icc, int n_eq, long long nnz,
                   const double *zprev = nullptr);
    template <class TM>
    void run_sweep(const PcgBufs<TM> &v, bool fwdir);
    // one cooperative launch of k_pcg: `batch` CG iterations, or (apply) the
    // two sweeps z = M^-1 r only
    template <class TM>
    void launch_pcg(const PcgBufs<TM> &v, bool apply, int batch);
    int pcg_grid(const void *kernel);
    void trace_phases(int iterations);
    // adjoint: stop at kAdjRtol ||b|| (or the rounding floor) and leave the
    // step's metrics as they are
    void mixed_solve(int n_eq, long long nnz, bool icc, bool adjoint = false);
    void build_windows(bool fp32);
    static constexpr int kMaxUpdates = 200;      // reliable updates of the mixed form, at most
    static constexpr double kDelta = 0.01;       // residual reduction between reliable updates (mixed form)
    static constexpr double kStall = 0.5;        // a reliable update that does not halve the best true
    static constexpr int kMaxStalls = 2;         // residual is a stall; this many in a row end the solve
    static constexpr double kUnitRoundoff = 1.1102230246251565e-16;   // 2^-53
    static constexpr double kFloor = 4.0;        // mixed form: stop at kFloor * (FP64 rounding floor)
    static constexpr double kAdjRtol = 1.0e-12;  // relative residual of the adjoint PPE solve
    int read_int(const int *dev);
    void check_err();
    void upload_list(const int *nb, const int *cnt, int max_nb);
    ListSource list() const { return ListSource{lptr_.p, lidx_.p}; }
    void explicit_stage(bool from_list);
    void implicit_stage();
    void require_ref() const
    {
        if (!have_ref_) throw CudaError("n0/lambda not set: call compute or set initial params", MPS_ERR_INVALID);
    }
};

// ---------------------------------------------------------------------------

template <int D>
Engine<D>::Engine(const mps_params_t &p, int capacity)
{
    if (p.dim != D) throw CudaError("dimension mismatch", MPS_ERR_INVALID);
    if (capacity <= 0) throw CudaError("capacity must be positive", MPS_ERR_INVALID);
    if (p.wall_drive_axis < 0 || p.wall_drive_axis >= D) throw CudaError("wall_drive_axis out of range", MPS_ERR_INVALID);
    if (D == 2 && p.friction_enabled) throw CudaError("friction is a 3-D model", MPS_ERR_UNSUPPORTED);
    cap_ = capacity;
    prm_ = p;
    if (const char *e = std::getenv("MPS_SPMV_LPR")) {
        int v = std::atoi(e);
        if (v == 8 || v == 16 || v == 32) spmv_lpr_ = v;
    }
    if (const char *e = std::getenv("MPS_PDL_MASK")) pdl_mask_ = std::atoi(e) & 7;
    if (const char *e = std::getenv("MPS_RELIABLE_DELTA")) {
        double v = std::atof(e);
        if (v > 0.0 && v < 1.0) rel_delta_ = v;
    }
    if (const char *e = std::getenv("MPS_MIXED_SPMV")) mixed_spmv_ = std::atoi(e);
    if (const char *e = std::getenv("MPS_PACK")) pack_ = std::atoi(e) ? 1 : 0;
    if (const char *e = std::getenv("MPS_SWEEP")) {
        int v = std::atoi(e);
        sweep_mode_ = (v == 0 || v == 1) ? v : 2;
    }
    if (const char *e = std::getenv("MPS_SWEEP_HB")) head_batch_ = std::atoi(e) == 8 ? 8 : 4;
    if (const char *e = std::getenv("MPS_SWEEP_OCC")) sweep_occ_ = std::atoi(e) == 8 ? 8 : 6;
    if (const char *e = std::getenv("MPS_SWEEP_HR")) head_rows_ = std::atoi(e) == 2 ? 2 : 1;
    if (const char *e = std::getenv("MPS_PCG_BATCH")) {
        int v = std::atoi(e);
        if (v >= 1 && v <= 1024) pcg_batch_ = v;
    }
    if (const char *e = std::getenv("MPS_TEST_BAR_POLLS")) {
        int v = std::atoi(e);
        if (v >= 0 && v < PCG_BAR_POLLS) bar_polls_ = v;
    }
    if (const char *e = std::getenv("MPS_CELL_EARLY")) cell_early_ = std::atoi(e) != 0;
    {
        int dev = 0;
        MPS_CUDA(cudaGetDevice(&dev));
        MPS_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    }
    if (const char *e = std::getenv("MPS_TEST_MBAR_POLLS")) {
        int v = std::atoi(e);
        if (v >= 0 && v < MBAR_POLLS) first_polls_ = v;
    }
    if (const char *e = std::getenv("MPS_CELL_WIN")) {
        int v = std::atoi(e);
        if (v >= 256 && v <= CELL_WIN_MAX && v % 4 == 0) cell_win_ = v;
    }

    MPS_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    for (auto &e : ev_) MPS_CUDA(cudaEventCreate(&e));
    for (auto &e : pev_) MPS_CUDA(cudaEventCreate(&e));
    MPS_CUDA(cudaMallocHost((void **)&sc_host_, sizeof(CGScalars)));
    MPS_CUDA(cudaMallocHost((void **)&int_host_, 64 * sizeof(int)));
    // the staged in-cell sweeps take more than the default 48 KB of dynamic shared memory
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<false, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<true, double, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<false, double, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<true, double, 4, 6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    MPS_CUDA(cudaFuncSetAttribute(k_sweep_colour<false, double, 4, 6, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(double) * CELL_STAGE_MAX)));
    alloc_state();
    build_grid();
    compute_consts();
    sc_.reserve(1);
    ticket_.reserve(4);
    err_.reserve(1);
    pcg_bar_.reserve(1);
    partials_.reserve(6 * RED_BLOCKS + 8);
    MPS_CUDA(cudaMemsetAsync(ticket_.p, 0, 4 * sizeof(unsigned), st_));
    MPS_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(unsigned), st_));

    // Neighbour-cell visit orders for PPE rows: sorted by (colour, z, y, x).
    signed char t3[8][27][3], t2[4][9][2];
    for (int par = 0; par < (1 << D); par++) {
        std::vector<std::array<int, 3>> offs;
        for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); dz++)
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) offs.push_back({dx, dy, dz});
        auto color = [&](const std::array<int, 3> &o) {
            int c = 0;
            for (int d = 0; d < D; d++) c |= (((par >> d) & 1) ^ (o[d] & 1)) << d;
            return c;
        };
        std::stable_sort(offs.begin(), offs.end(),
                         [&](const std::array<int, 3> &a, const std::array<int, 3> &b) {
                             return color(a) < color(b);
                         });
        for (size_t q = 0; q < offs.size(); q++)
            for (int d = 0; d < D; d++) {
                if (D == 3) t3[par][q][d] = (signed char)offs[q][d];
                else t2[par][q][d] = (signed char)offs[q][d];
            }
    }
    if (D == 3) MPS_CUDA(cudaMemcpyToSymbol(c_order3, t3, sizeof(t3)));
    else MPS_CUDA(cudaMemcpyToSymbol(c_order2, t2, sizeof(t2)));

}

template <int D>
Engine<D>::~Engine()
{
    if (st_) cudaStreamSynchronize(st_);
    for (auto &e : ev_) cudaEventDestroy(e);
    for (auto &e : pev_) cudaEventDestroy(e);
    if (sc_host_) cudaFreeHost(sc_host_);
    if (int_host_) cudaFreeHost(int_host_);
    if (st_) cudaStreamDestroy(st_);
}

template <int D>
void Engine<D>::alloc_state()
{
    size_t nd = (size_t)(4 * D + 2), ni = 5;
    for (int b = 0; b < 2; b++) {
        dbuf_[b].reserve(nd * cap_);
        ibuf_[b].reserve(ni * cap_);
        double *dp = dbuf_[b].p;
        int *ip = ibuf_[b].p;
        State<D> &s = S_[b];
        for (int d = 0; d < D; d++) {
            s.pos[d] = dp + (size_t)(0 * D + d) * cap_;
            s.vel[d] = dp + (size_t)(1 * D + d) * cap_;
            s.acc[d] = dp + (size_t)(2 * D + d) * cap_;
            s.key[d] = dp + (size_t)(3 * D + d) * cap_;
        }
        s.p = dp + (size_t)(4 * D) * cap_;
        s.n = dp + (size_t)(4 * D + 1) * cap_;
        s.type = ip;
        s.surf = ip + (size_t)cap_;
        s.ncount = ip + 2 * (size_t)cap_;
        s.id = ip + 3 * (size_t)cap_;
        s.cell = ip + 4 * (size_t)cap_;
    }
    kcell_.reserve(cap_);
    excl_.reserve(cap_);
    exoff_.reserve(cap_ + 1);
    tmp_.reserve(cap_);
    perm_.reserve(cap_);
    where_.reserve(cap_);
    vafter_.reserve((size_t)D * cap_);
    pmin_.reserve(cap_);
    rest_.reserve((size_t)D * cap_);
    row_of_.reserve(cap_);
    part_of_row_.reserve(cap_);
    rcount_.reserve(cap_ + 1);
    row_ptr_.reserve(cap_ + 1);
    diagpos_.reserve(cap_);
    inpos_.reserve(cap_);
    outpos_.reserve(cap_);
    for (auto *v : {&pk_len_lo_, &pk_len_up_, &pk_off_lo_, &pk_off_up_}) v->reserve((size_t)cap_ + 1);
    dinv_.reserve(cap_);
    for (auto *v : {&b_, &x_, &r_, &z_, &p_, &Ap_, &y_, &part_, &p2_}) v->reserve(cap_);
}

// cell_list_create (neighbor_search.c:92-122) with cell size = list radius.
template <int D>
void Engine<D>::build_grid()
{
    double re = list_radius(prm_);
    re_list_ = re;
    double margin = 4.0 * re;
    long long total = 1;
    for (int d = 0; d < D; d++) {
        g_.origin[d] = prm_.domain_min[d] - margin;
        double span = (prm_.domain_max[d] + margin) - g_.origin[d];
        g_.dims[d] = (int)(span / re) + 2;
        total *= g_.dims[d];
    }
    if (total <= 0 || total > (1LL << 30)) throw CudaError("cell grid too large", MPS_ERR_INVALID);
    g_.total = (int)total;
    g_.cs_inv = 1.0 / re;
    count_.reserve(total + 1);
    cursor_.reserve(total + 1);
    start_.reserve(total + 2);
    ucount_.reserve(total);
    ucol_.reserve(total);
    rs_.reserve(total + 1);
    cell_row0_.reserve(total);
    size_t ws = std::max(scan_workspace((int)std::max<long long>(total + 1, cap_ + 1)), (size_t)64);
    scanws_.reserve(ws);
    g_.start = start_.p;

    // cells sorted by (colour, linear index)
    std::vector<int> cc((size_t)total);
    int ncol = 1 << D;
    std::vector<int> cnt(ncol + 1, 0);
    auto color_of = [&](long long lin) {
        int c = 0;
        for (int d = 0; d < D; d++) {
            c |= (int)((lin % g_.dims[d]) & 1) << d;
            lin /= g_.dims[d];
        }
        return c;
    };
    for (long long l = 0; l < total; l++) cnt[color_of(l) + 1]++;
    for (int c = 0; c < ncol; c++) cnt[c + 1] += cnt[c];
    color_off_ = cnt;
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (long long l = 0; l < total; l++) cc[(size_t)fill[color_of(l)]++] = (int)l;
    ccells_.reserve(total);
    MPS_CUDA(cudaMemcpy(ccells_.p, cc.data(), sizeof(int) * (size_t)total, cudaMemcpyHostToDevice));
    color_off_dev_.reserve(ncol + 1);
    MPS_CUDA(cudaMemcpy(color_off_dev_.p, color_off_.data(), sizeof(int) * (ncol + 1), cudaMemcpyHostToDevice));
    aflag_.reserve(total + 1);
    apos_.reserve(total + 1);
    acells_.reserve(total + 1);
    sizes_.reserve(16);

}

// Constants evaluated with the reference's expressions.
template <int D>
void Engine<D>::compute_consts()
{
    const mps_params_t &p = prm_;
    Consts &k = k_;
    k.l0 = p.particle_distance;
    k.rmin = 0.01 * p.particle_distance;
    k.re_lap = p.influence_radius_lap;
    k.re_n = p.influence_radius_n;
    k.re_list2 = re_list_ * re_list_;
    k.re_n2 = p.influence_radius_n * p.influence_radius_n;
    double n0 = have_ref_ ? n0_ : 1.0, lambda = have_ref_ ? lambda_ : 1.0;
    k.n0 = n0;
    k.coeff = 2.0 * D / (n0 * lambda);
    k.visc_coeff = p.viscosity * k.coeff;
    k.grad_coeff = (double)D / n0;
    k.neg_grad = -k.grad_coeff;
    k.density = p.density;
    for (int d = 0; d < 3; d++) k.gravity[d] = d < D ? p.gravity[d] : 0.0;
    k.dt = p.dt;
    double cd = p.collision_distance_ratio * p.particle_distance;
    k.col2 = cd * cd;
    k.col_rmin = 1.0e-12 * p.particle_distance;
    k.half1pe = (1.0 + p.restitution_coeff) * 0.5;
    k.grad_r2min = p.particle_distance * p.particle_distance * 1.0e-12;
    k.surf_thr = p.surface_threshold * n0;
    k.count_thr = p.surface_count_threshold * n0_count_;
    k.diag_scale = (p.ppe_type == 1) ? p.c_ppe * k.coeff : k.coeff;
    k.neg_coeff = -k.coeff;
    double dt2 = p.dt * p.dt;
    k.rhs_k = p.relaxation_coeff * (p.density / dt2);
    k.rhs_hs = -(p.density / n0 / p.dt);
    k.rhs_na = -p.density / p.dt;
    k.rhs_nb = p.gamma_ppe * (p.density / dt2);
    double margin = p.particle_distance * (p.wall_layers + 1);
    for (int d = 0; d < 3; d++) {
        k.oob_lo[d] = p.domain_min[d] - margin;
        k.oob_hi[d] = p.domain_max[d] + margin;
    }
    k.max_nb = p.max_neighbors;
    k.ppe_type = p.ppe_type;
    k.hs_mode = p.hs_mode;
    k.cmps = p.cmps_gradient;
    k.surf_method = p.surface_detection_method;
    k.clamp = p.clamp_negative_pressure;
    k.collision_on = (D == 2) ? 1 : (p.collision_distance_ratio > 0.0);
    k.drive_on = p.wall_drive_amp != 0.0;
    k.drive_axis = p.wall_drive_axis;
    // surface tension (operators.c:283-285, 2-D :233-235): coeff = C / (rho l0^D)
    k.st_on = p.surface_tension_enabled != 0;
    double cll = 0.0, csl = 0.0;
    surface_tension_coeffs(p, &cll, &csl);
    double l0 = p.particle_distance;
    k.st_ll = (D == 3) ? cll / (p.density * l0 * l0 * l0) : cll / (p.density * l0 * l0);
    k.st_sl = (D == 3) ? csl / (p.density * l0 * l0 * l0) : csl / (p.density * l0 * l0);
    k.st_sl_on = csl != 0.0;
    k.re_st = p.influence_radius_st;
    k.st_rmin = 1.0e-9 * l0;
    // friction (3S operators.c:341-346), with the reference's expressions
    k.fr_on = D == 3 && p.friction_enabled != 0;
    k.fr_theta_s = p.wetting_angle_SL * M_PI / 180.0;
    k.fr_dtheta = p.friction_delta_theta * M_PI / 180.0;
    k.fr_vc = p.friction_velocity_threshold;
    k.fr_dyn = p.dynamic_friction_alpha * p.viscosity * 2.0 * D / (n0 * lambda);
}

template <int D>
void Engine<D>::update_params(const mps_params_t &p)
{
    if (p.dim != D) throw CudaError("dimension mismatch", MPS_ERR_INVALID);
    if (p.wall_drive_axis < 0 || p.wall_drive_axis >= D) throw CudaError("wall_drive_axis out of range", MPS_ERR_INVALID);
    if (D == 2 && p.friction_enabled) throw CudaError("friction is a 3-D model", MPS_ERR_UNSUPPORTED);
    bool regrid = false;
    for (int d = 0; d < D; d++)
        regrid |= p.domain_min[d] != prm_.domain_min[d] || p.domain_max[d] != prm_.domain_max[d];
    regrid |= list_radius(p) != re_list_;
    prm_ = p;
    if (regrid) {
        build_grid();
        structure_ = false;
    }
    compute_consts();
}

template <int D>
int Engine<D>::read_int(const int *dev)
{
    MPS_CUDA(cudaMemcpyAsync(int_host_, dev, sizeof(int), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    return int_host_[0];
}

template <int D>
void Engine<D>::check_err()
{
    unsigned e = 0;
    MPS_CUDA(cudaMemcpyAsync(int_host_, err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    MPS_CUDA(cudaGetLastError());
    std::memcpy(&e, int_host_, sizeof(unsigned));
    if (e) {
        MPS_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(unsigned), st_));
        if (e & ERR_NEIGHBOR_OVERFLOW) throw CudaError("neighbour count exceeded max_neighbors", MPS_ERR_NEIGHBOR_OVERFLOW);
        if (e & ERR_UNKNOWN_OFF_GRID) throw CudaError("a PPE unknown lies outside the cell grid", MPS_ERR_UNSUPPORTED);
        if (e & ERR_LIST_MISMATCH) throw CudaError("neighbour list does not match the cell structure", MPS_ERR_UNSUPPORTED);
        if (e & ERR_COLORING) throw CudaError("PPE row count mismatch", MPS_ERR_INVALID);
        if (e & ERR_CELL_OVERFULL) throw CudaError("more than 255 PPE unknowns in one cell", MPS_ERR_UNSUPPORTED);
        if (e & ERR_COPY_TIMEOUT) throw CudaError("a bulk copy into shared memory timed out", MPS_ERR_CUDA);
        if (e & ERR_GRID_TIMEOUT) throw CudaError("a grid barrier of the persistent PCG kernel timed out", MPS_ERR_CUDA);
        throw CudaError("device error", MPS_ERR_INVALID);
    }
}

// ---- state transfer ---------------------------------------------------------

template <int D>
void Engine<D>::upload_aos(const void *aos, int num)
{
    if (num < 0 || num > cap_) throw CudaError("particle count exceeds capacity", MPS_ERR_INVALID);
    n_ = num;
    size_t bytes = (size_t)num * AosLayout<D>::size;
    aos_.reserve(bytes + 8);
    MPS_CUDA(cudaMemcpyAsync(aos_.p, aos, bytes, cudaMemcpyHostToDevice, st_));
    if (num) launch(k_unpack<D>, nblk(num, TPB), TPB, 0, st_, aos_.p, S(), num);
    if (num) launch(k_set_rest<D>, nblk(num, TPB), TPB, 0, st_, S(), num, cap_, rest_.p);
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(cudaStreamSynchronize(st_));
    tstep_ = 0;
    structure_ = false;
    ppe_valid_ = false;
}

template <int D>
void Engine<D>::download_aos(void *aos, int num)
{
    if (num != n_) throw CudaError("download count differs from the uploaded count", MPS_ERR_INVALID);
    size_t bytes = (size_t)num * AosLayout<D>::size;
    aos_.reserve(bytes + 8);
    if (num) launch(k_pack<D>, nblk(num, TPB), TPB, 0, st_, aos_.p, S(), num);
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(cudaMemcpyAsync(aos, aos_.p, bytes, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::upload_soa(const double *pos, const double *vel, const int *type, int num)
{
    if (num < 0 || num > cap_) throw CudaError("particle count exceeds capacity", MPS_ERR_INVALID);
    n_ = num;
    soa_in_.reserve((size_t)2 * D * num + 2);
    int_in_.reserve((size_t)num + 1);
    MPS_CUDA(cudaMemcpyAsync(soa_in_.p, pos, sizeof(double) * D * num, cudaMemcpyHostToDevice, st_));
    MPS_CUDA(cudaMemcpyAsync(soa_in_.p + (size_t)D * num, vel, sizeof(double) * D * num,
                             cudaMemcpyHostToDevice, st_));
    MPS_CUDA(cudaMemcpyAsync(int_in_.p, type, sizeof(int) * num, cudaMemcpyHostToDevice, st_));
    if (num)
        launch(k_unpack_soa<D>, nblk(num, TPB), TPB, 0, st_, soa_in_.p, soa_in_.p + (size_t)D * num, int_in_.p, S(),
                                                         num);
    if (num) launch(k_set_rest<D>, nblk(num, TPB), TPB, 0, st_, S(), num, cap_, rest_.p);
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(cudaStreamSynchronize(st_));
    tstep_ = 0;
    structure_ = false;
    ppe_valid_ = false;
}

template <int D>
void Engine<D>::download_pressure(double *p, int num)
{
    if (num != n_) throw CudaError("download count differs from the uploaded count", MPS_ERR_INVALID);
    soa_in_.reserve((size_t)num + 2);
    if (num) launch(k_pressure_ref<D>, nblk(num, TPB), TPB, 0, st_, S(), num, soa_in_.p);
    MPS_CUDA(cudaMemcpyAsync(p, soa_in_.p, sizeof(double) * num, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

// ---- neighbour search -------------------------------------------------------

template <int D>
void Engine<D>::sort()
{
    int n = n_, total = g_.total;
    State<D> &src = S_[cur_];
    State<D> &dst = S_[cur_ ^ 1];
    MPS_CUDA(cudaMemsetAsync(count_.p, 0, sizeof(int) * (total + 1), st_));
    MPS_CUDA(cudaMemsetAsync(cursor_.p, 0, sizeof(int) * (total + 1), st_));
    if (n) launch(k_bin<D>, nblk(n, TPB), TPB, 0, st_, src, g_, n, kcell_.p, count_.p, excl_.p);
    scan_exclusive<int>(count_.p, start_.p, total, scanws_.p, st_);
    scan_exclusive<int>(excl_.p, exoff_.p, n, scanws_.p, st_);
    if (n) {
        launch(k_scatter, nblk(n, TPB), TPB, 0, st_, n, total, kcell_.p, start_.p, cursor_.p, exoff_.p, tmp_.p,
                                                 perm_.p);
        // ranks for the binned prefix [0, start[total])
        launch(k_rank, nblk(n, TPB), TPB, 0, st_, start_.p + total, tmp_.p, kcell_.p, start_.p, src.id, perm_.p);
        launch(k_gather<D>, nblk(n, TPB), TPB, 0, st_, dst, src, perm_.p, kcell_.p, n, where_.p);
    }
    MPS_CUDA(cudaGetLastError());
    cur_ ^= 1;
    g_.start = start_.p;
    structure_ = true;
    ppe_valid_ = false;
}

template <int D>
void Engine<D>::unsort()
{
    int n = n_;
    if (n) launch(k_unsort<D>, nblk(n, TPB), TPB, 0, st_, S_[cur_ ^ 1], S_[cur_], where_.p, n);
    MPS_CUDA(cudaGetLastError());
    cur_ ^= 1;
    structure_ = false;
    ppe_valid_ = false;
}

template <int D>
void Engine<D>::neighbor_search()
{
    sort();
    if (n_) {
        // list lengths only: the reference aborts on overflow during the search
        lcnt_.reserve((size_t)n_ + 1);
        launch(k_build_list<D>, nblk(n_, TPB), TPB, 0, st_, cells(), (const int *)S().id, n_, k_.max_nb, 0,
               (int *)nullptr, lcnt_.p, err_.p);
    }
    check_err();
}

// ---- initial parameters (f1) -----------------------------------------------

template <int D>
void Engine<D>::compute_initial_params(double *n0, double *lambda, int *n0_count)
{
    int n = n_;
    if (n == 0) throw CudaError("no particles", MPS_ERR_INVALID);
    // bounding box on the host side of a copy of the positions
    std::vector<double> h((size_t)n * D);
    for (int d = 0; d < D; d++)
        MPS_CUDA(cudaMemcpyAsync(h.data() + (size_t)d * n, S().pos[d], sizeof(double) * n, cudaMemcpyDeviceToHost,
                                 st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    double lo[D], hi[D];
    for (int d = 0; d < D; d++) {
        lo[d] = INFINITY;
        hi[d] = -INFINITY;
        for (int i = 0; i < n; i++) {
            double v = h[(size_t)d * n + i];
            lo[d] = std::min(lo[d], v);
            hi[d] = std::max(hi[d], v);
        }
        if (!std::isfinite(lo[d]) || !std::isfinite(hi[d]))
            throw CudaError("non-finite particle position", MPS_ERR_NAN);
    }
    double re_n = prm_.influence_radius_n, re_lap = prm_.influence_radius_lap;
    double rmax = std::max(re_n, re_lap);
    double cs = rmax * (1.0 + 1.0e-9);
    Grid<D> bg{};
    long long total = 1;
    for (int d = 0; d < D; d++) {
        bg.origin[d] = lo[d];
        bg.dims[d] = (int)((hi[d] - lo[d]) / cs) + 1;
        total *= bg.dims[d];
    }
    if (total > (1LL << 30)) throw CudaError("bounding-box grid too large", MPS_ERR_INVALID);
    bg.total = (int)total;
    DevArray<int> gcell, cnt, st, cur, order, cnti, qbest;
    DevArray<double> dlo, n0i, numi, deni, best;
    gcell.reserve(n);
    cnt.reserve(total + 1);
    st.reserve(total + 2);
    cur.reserve(total + 1);
    order.reserve(n);
    cnti.reserve(n);
    qbest.reserve(4);
    dlo.reserve(D);
    n0i.reserve(n);
    numi.reserve(n);
    deni.reserve(n);
    best.reserve(2);
    DevArray<int> ws;
    ws.reserve(scan_workspace((int)total + 1) + 8);
    MPS_CUDA(cudaMemcpyAsync(dlo.p, lo, sizeof(double) * D, cudaMemcpyHostToDevice, st_));
    MPS_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int) * (total + 1), st_));
    MPS_CUDA(cudaMemsetAsync(cur.p, 0, sizeof(int) * (total + 1), st_));
    launch(k_bbox_cell<D>, nblk(n, TPB), TPB, 0, st_, S(), n, bg, cs, dlo.p, gcell.p, cnt.p);
    scan_exclusive<int>(cnt.p, st.p, (int)total, ws.p, st_);
    launch(k_bbox_scatter, nblk(n, TPB), TPB, 0, st_, n, gcell.p, st.p, cur.p, order.p);
    bg.start = st.p;
    launch(k_initial_params<D>, nblk(n, 128), 128, 0, st_, S(), n, bg, gcell.p, order.p, rmax, re_n, re_lap,
                                                       0.01 * prm_.particle_distance, n0i.p, numi.p, deni.p,
                                                       cnti.p, err_.p);
    launch(k_initial_argmax<D>, 1, 1024, 0, st_, S(), n, n0i.p, cnti.p, best.p, qbest.p, qbest.p + 1);
    MPS_CUDA(cudaGetLastError());
    check_err();
    double bv;
    int q[2];
    MPS_CUDA(cudaMemcpy(&bv, best.p, sizeof(double), cudaMemcpyDeviceToHost));
    MPS_CUDA(cudaMemcpy(q, qbest.p, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    double num = 0.0, den = 0.0;
    if (bv > 0.0 && q[0] >= 0) {
        MPS_CUDA(cudaMemcpy(&num, numi.p + q[0], sizeof(double), cudaMemcpyDeviceToHost));
        MPS_CUDA(cudaMemcpy(&den, deni.p + q[0], sizeof(double), cudaMemcpyDeviceToHost));
        n0_ = bv;
        if (prm_.use_analytical_lambda)
            lambda_ = re_lap * re_lap * (double)D * (double)(D - 1) / ((double)(D + 1) * (double)(D + 2));
        else
            lambda_ = (den > 1.0e-10) ? num / den : 1.0;
        if (prm_.surface_detection_method == 1) n0_count_ = q[1];
    } else {
        // particle.c:159-164: no fluid particle with a positive n0
        n0_ = 1.0;
        lambda_ = 1.0;
    }
    have_ref_ = true;
    compute_consts();
    if (n0) *n0 = n0_;
    if (lambda) *lambda = lambda_;
    if (n0_count) *n0_count = n0_count_;
}

template <int D>
void Engine<D>::set_initial_params(double n0, double lambda, int n0_count)
{
    n0_ = n0;
    lambda_ = lambda;
    n0_count_ = n0_count;
    have_ref_ = true;
    compute_consts();
}

// ---- the step -------------------------------------------------------------------

// The caller's list (reference layout: row i at nb[i * max_nb], count[i]
// entries) to CSR on the device: one pitched copy of the used columns, a
// scan of the counts and a compaction kernel.
template <int D>
void Engine<D>::upload_list(const int *nb, const int *cnt, int max_nb)
{
    int n = n_;
    if (max_nb <= 0) throw CudaError("max_neighbors must be positive", MPS_ERR_INVALID);
    int mc = 0;
    for (int i = 0; i < n; i++) {
        if (cnt[i] < 0 || cnt[i] > max_nb) throw CudaError("bad neighbour count", MPS_ERR_INVALID);
        mc = std::max(mc, cnt[i]);
    }
    lcnt_.reserve((size_t)n + 1);
    lptr_.reserve((size_t)n + 1);
    MPS_CUDA(cudaMemcpyAsync(lcnt_.p, cnt, sizeof(int) * n, cudaMemcpyHostToDevice, st_));
    scan_exclusive<int>(lcnt_.p, lptr_.p, n, scanws_.p, st_);
    // a list in page-locked host memory is read in place by the gather
    // kernel (only the used entries cross the link); a pageable one goes
    // through a pitched copy of its used columns
    cudaPointerAttributes pa{};
    bool mapped = false;
    if (cudaPointerGetAttributes(&pa, nb) == cudaSuccess)
        mapped = pa.type == cudaMemoryTypeHost && pa.devicePointer != nullptr;
    else
        (void)cudaGetLastError();
    if (mc > 0 && n > 0 && mapped) {
        lidx_.reserve((size_t)n * mc);
        launch(k_gather_host_list, nblk((long long)n * 32, TPB), TPB, 0, st_, (const int *)pa.devicePointer,
               max_nb, (const int *)lcnt_.p, (const int *)lptr_.p, n, lidx_.p, err_.p);
    } else if (mc > 0 && n > 0) {
        lout_.reserve((size_t)n * mc);
        lidx_.reserve((size_t)n * mc);
        MPS_CUDA(cudaMemcpy2DAsync(lout_.p, sizeof(int) * mc, nb, sizeof(int) * (size_t)max_nb, sizeof(int) * mc,
                                   n, cudaMemcpyHostToDevice, st_));
        launch(k_compact_list, nblk(n, TPB), TPB, 0, st_, (const int *)lout_.p, mc, (const int *)lcnt_.p,
               (const int *)lptr_.p, n, lidx_.p, err_.p);
    } else {
        lidx_.reserve(1);
    }
    check_err();
}

template <int D>
void Engine<D>::explicit_stage(bool from_list)
{
    int n = n_;
    if (!n) return;
    int nb = nblk(n, TPB);
    if (from_list) launch(k_viscosity<D, ListSource>, nb, TPB, 0, st_, list(), S(), k_, n, 0);
    else launch(k_viscosity<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, 0);
    if (k_.st_on) {
        if (from_list) launch(k_surface_tension<D, ListSource>, nb, TPB, 0, st_, list(), S(), k_, n, 3);
        else launch(k_surface_tension<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, 3);
    }
    if (k_.fr_on) {
        launch(k_explicit_part<D>, nb, TPB, 0, st_, S(), k_, n, 1);
        if (from_list) launch(k_friction<D, ListSource>, nb, TPB, 0, st_, list(), S(), k_, n);
        else launch(k_friction<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n);
        launch(k_explicit_part<D>, nb, TPB, 0, st_, S(), k_, n, 2);
    } else {
        launch(k_explicit_update<D>, nb, TPB, 0, st_, S(), k_, n);
    }
    if (k_.drive_on) {
        double dx, vel;
        drive_terms((double)(tstep_ + 1) * prm_.dt, &dx, &vel);
        launch(k_drive_walls<D>, nb, TPB, 0, st_, S(), n, (const double *)rest_.p + (size_t)k_.drive_axis * cap_,
               k_.drive_axis, dx, vel);
    }
    if (adj_rec_) launch(k_adj_record<D>, nb, TPB, 0, st_, S(), n, adj_);
    if (k_.collision_on) {
        if (D == 3) {
            if (from_list) launch(k_collision_list<D, ListSource>, nb, TPB, 0, st_, list(), S(), k_, n, vafter_.p);
            else launch(k_collision_list<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, vafter_.p);
        } else {
            sort();
            launch(k_collision_allpairs<D>, nb, TPB, 0, st_, cells(), S(), k_, n, vafter_.p);
        }
        launch(k_collision_apply<D>, nb, TPB, 0, st_, S(), k_, n, vafter_.p);
    }
    MPS_CUDA(cudaGetLastError());
}

template <int D>
void Engine<D>::implicit_stage()
{
    int n = n_;
    sort();
    if (!n) return;
    int nb = nblk(n, TPB);
    launch(k_density<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, err_.p, 1, 1);
    MPS_CUDA(cudaEventRecord(ev_[1], st_));
    ppe(k_.clamp != 0);
    MPS_CUDA(cudaEventRecord(ev_[4], st_));
    if (k_.cmps != 2) launch(k_pmin<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), n, pmin_.p);
    launch(k_gradient<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, k_.cmps != 2 ? pmin_.p : nullptr);
    launch(k_correct<D>, nb, TPB, 0, st_, S(), k_, n, 1, 1, 1);
    MPS_CUDA(cudaGetLastError());
}

template <int D>
void Engine<D>::step(int nsteps)
{
    require_ref();
    if (!structure_) throw CudaError("no neighbour structure: run the neighbour search first", MPS_ERR_INVALID);
    for (int s = 0; s < nsteps; s++) {
        MPS_CUDA(cudaEventRecord(ev_[0], st_));
        explicit_stage(false);
        implicit_stage();
        MPS_CUDA(cudaEventRecord(ev_[5], st_));
        check_err();
        float t01 = 0, t12 = 0, t23 = 0, t34 = 0, t45 = 0;
        cudaEventElapsedTime(&t01, ev_[0], ev_[1]);
        cudaEventElapsedTime(&t12, ev_[1], ev_[2]);
        cudaEventElapsedTime(&t23, ev_[2], ev_[3]);
        cudaEventElapsedTime(&t34, ev_[3], ev_[4]);
        cudaEventElapsedTime(&t45, ev_[4], ev_[5]);
        met.ms_ops = t01 + t45;
        met.ms_assembly = t12;
        met.ms_factor = t23;
        met.ms_solve = t34;
        met.total_steps++;
        tstep_++;
    }
}

template <int D>
void Engine<D>::step_with_list(const int *nb, const int *cnt, int max_nb)
{
    require_ref();
    if (structure_) unsort();
    upload_list(nb, cnt, max_nb);
    MPS_CUDA(cudaEventRecord(ev_[0], st_));
    explicit_stage(true);
    implicit_stage();
    MPS_CUDA(cudaEventRecord(ev_[5], st_));
    check_err();
    met.total_steps++;
    tstep_++;
}

// ---- PPE ------------------------------------------------------------------------

template <int D>
void Engine<D>::ppe(bool clamp)
{
    int n = n_, total = g_.total;
    int ncol = 1 << D;
    State<D> &s = S();
    launch(k_cell_unknowns<D>, nblk(total, TPB), TPB, 0, st_, s, start_.p, total, ucount_.p);
    launch(k_color_gather, nblk(total, TPB), TPB, 0, st_, ccells_.p, ucount_.p, total, ucol_.p);
    scan_exclusive<int>(ucol_.p, rs_.p, total, scanws_.p, st_);
    launch(k_assign_rows<D>, nblk(total, TPB), TPB, 0, st_, s, (const int *)start_.p, (const int *)ccells_.p,
           (const int *)rs_.p, total, cell_row0_.p, row_of_.p, part_of_row_.p);
    launch(k_active_flag, nblk(total, TPB), TPB, 0, st_, (const int *)ucol_.p, total, aflag_.p);
    scan_exclusive<int>(aflag_.p, apos_.p, total, scanws_.p, st_);
    launch(k_active_scatter, nblk(total, TPB), TPB, 0, st_, (const int *)ccells_.p, (const int *)ucol_.p,
           (const int *)apos_.p, total, acells_.p);
    launch(k_ppe_sizes, 1, 1, 0, st_, (const int *)rs_.p, (const int *)apos_.p, (const int *)start_.p, total,
           (const int *)color_off_dev_.p, ncol, sizes_.p);
    MPS_CUDA(cudaMemcpyAsync(int_host_, sizes_.p, sizeof(int) * (2 * ncol + 4), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    int n_eq = int_host_[0];
    int nbinned = int_host_[1];
    act_off_.assign(int_host_ + 2, int_host_ + 3 + ncol);
    row_off_.assign(int_host_ + 3 + ncol, int_host_ + 4 + 2 * ncol);
    if (n > nbinned)
        launch(k_offgrid_rows<D>, nblk(n - nbinned, TPB), TPB, 0, st_, s, nbinned, n, row_of_.p, err_.p);
    n_eq_ = n_eq;
    met.n_eq = n_eq;
    int nb = nblk(n, TPB);
    if (n_eq == 0) {
        met.ppe_iterations = 0;
        met.ppe_residual = 0.0;
        met.ppe_true_residual = 0.0;
        met.ppe_bnorm = 0.0;
        met.ppe_rounding_floor = 0.0;
        met.converged = 1;
        met.nnz = 0;
        MPS_CUDA(cudaEventRecord(ev_[2], st_));
        MPS_CUDA(cudaEventRecord(ev_[3], st_));
        launch(k_writeback<D>, nb, TPB, 0, st_, s, row_of_.p, x_.p, n, clamp);
        ppe_valid_ = true;
        return;
    }
    CellSource<D> src = cells();
    launch(k_row_count<D, CellSource<D>>, nblk(n_eq, TPB), TPB, 0, st_, src, s, part_of_row_.p, row_of_.p, n_eq,
                                                                     rcount_.p);
    scan_exclusive<int>(rcount_.p, row_ptr_.p, n_eq, scanws_.p, st_);
    int nnz = read_int(row_ptr_.p + n_eq);
    if (nnz < 0) throw CudaError("PPE too large for 32-bit row pointers", MPS_ERR_UNSUPPORTED);
    nnz_ = nnz;
    met.nnz = nnz;
    col_.reserve(nnz);
    A_.reserve(nnz);
    F_.reserve(nnz);
    launch(k_fill<D>, nblk(n_eq, 128), 128, 0, st_, src, s, k_, part_of_row_.p, row_of_.p, n_eq, row_ptr_.p, col_.p,
                                                A_.p, diagpos_.p, b_.p, err_.p);
    MPS_CUDA(cudaEventRecord(ev_[2], st_));
    bool icc = prm_.solver_type == 1;
    if (icc) {
        launch(k_row_splits, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)row_ptr_.p, (const int *)diagpos_.p,
               (const int *)col_.p, (const int *)part_of_row_.p, (const int *)s.cell, (const int *)cell_row0_.p,
               (const int *)ucount_.p, inpos_.p, outpos_.p);
        MPS_CUDA(cudaMemcpyAsync(F_.p, A_.p, sizeof(double) * nnz, cudaMemcpyDeviceToDevice, st_));
        for (int c = 0; c < ncol; c++) {
            int rb = row_off_[c], re = row_off_[c + 1];
            if (re > rb)
                launch(k_ic0_cross_warp, nblk((long long)(re - rb) * 32, 256), 256, 0, st_, rb, re,
                       (const int *)row_ptr_.p, (const int *)diagpos_.p, (const int *)inpos_.p, (const int *)col_.p,
                       (const double *)A_.p, F_.p);
            int kb = act_off_[c], ke = act_off_[c + 1];
            if (ke > kb)
                launch(k_ic0_incell, nblk(ke - kb, SWEEP_WARPS_IC), 32 * SWEEP_WARPS_IC, 0, st_, kb, ke,
                       (const int *)acells_.p, (const int *)cell_row0_.p, (const int *)ucount_.p,
                       (const int *)row_ptr_.p, (const int *)diagpos_.p, (const int *)inpos_.p,
                       (const int *)col_.p, (const double *)A_.p, F_.p);
        }
        // packed in-cell factor and cell descriptors for the sweeps
        launch(k_pack_lengths, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)row_ptr_.p,
               (const int *)diagpos_.p, (const int *)inpos_.p, (const int *)outpos_.p, pk_len_lo_.p, pk_len_up_.p);
        scan_exclusive<int>(pk_len_lo_.p, pk_off_lo_.p, n_eq, scanws_.p, st_);
        scan_exclusive<int>(pk_len_up_.p, pk_off_up_.p, n_eq, scanws_.p, st_);
        size_t in_cap = (size_t)nnz;   // in-cell entries are a subset of the nonzeros
        pk_val_lo_.reserve(in_cap);
        pk_val_up_.reserve(in_cap);
        pk_k_lo_.reserve(in_cap);
        pk_k_up_.reserve(in_cap);
        launch(k_pack_fill, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)diagpos_.p, (const int *)inpos_.p,
               (const int *)outpos_.p, (const int *)col_.p, (const double *)F_.p, (const int *)part_of_row_.p,
               (const int *)s.cell, (const int *)cell_row0_.p, (const int *)pk_off_lo_.p,
               (const int *)pk_off_up_.p, pk_val_lo_.p, pk_k_lo_.p, pk_val_up_.p, pk_k_up_.p, dinv_.p, err_.p);
        // packed cross-cell runs of the factor for the sweeps
        for (auto *v : {&xlen_lo_, &xlen_up_, &xp_lo_, &xp_up_, &xs_lo_, &xs_up_}) v->reserve((size_t)n_eq + 1);
        launch(k_cross_lengths, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)row_ptr_.p, (const int *)inpos_.p,
               (const int *)outpos_.p, xlen_lo_.p, xlen_up_.p);
        scan_exclusive<int>(xlen_lo_.p, xp_lo_.p, n_eq, scanws_.p, st_);
        scan_exclusive<int>(xlen_up_.p, xp_up_.p, n_eq, scanws_.p, st_);
        nx_lo_ = read_int(xp_lo_.p + n_eq);
        nx_up_ = read_int(xp_up_.p + n_eq);
        xc_lo_.reserve((size_t)nx_lo_ + 1);
        xf_lo_.reserve((size_t)nx_lo_ + 1);
        xc_up_.reserve((size_t)nx_up_ + 1);
        xf_up_.reserve((size_t)nx_up_ + 1);
        SweepColours swc{};
        swc.ncol = ncol;
        for (int c = 0; c <= ncol; c++) swc.row_off[c] = row_off_[c];
        for (int k = 0; k < ncol; k++) {
            // the colour swept just before k, forward (largest non-empty below) and backward
            int pf = -1, pb = -1;
            for (int j = k - 1; j >= 0 && pf < 0; j--)
                if (row_off_[j + 1] > row_off_[j]) pf = j;
            for (int j = k + 1; j < ncol && pb < 0; j++)
                if (row_off_[j + 1] > row_off_[j]) pb = j;
            swc.thr_lo[k] = pf >= 0 ? row_off_[pf] : 0;
            swc.thr_up[k] = pb >= 0 ? row_off_[pb + 1] : 0x7fffffff;
        }
        int nact = act_off_[ncol];
        adesc_.reserve((size_t)nact + 1);
        if (nact)
            launch(k_cell_desc, nblk(nact, TPB), TPB, 0, st_, nact, (const int *)acells_.p,
                   (const int *)cell_row0_.p, (const int *)ucount_.p, adesc_.p);
        if (sweep_mode_ != 0) {
            // the cross runs of each cell in jagged-diagonal order (k_sweep_cell, k_pcg)
            for (auto *v : {&jlen_, &jdc_lo_, &jdc_up_}) v->reserve((size_t)nact + 1);
            for (auto *v : {&jperm_lo_, &jperm_up_}) v->reserve((size_t)n_eq + 1);
            for (int lo = 1; lo >= 0; lo--) {
                DevArray<int> &jdc = lo ? jdc_lo_ : jdc_up_, &jdp = lo ? jdp_lo_ : jdp_up_;
                const int *xp = lo ? xp_lo_.p : xp_up_.p;
                if (nact)
                    launch(k_jds_sizes, nblk((long long)nact * 32, 256), 256, 0, st_, nact, (const int2 *)adesc_.p,
                           xp, jlen_.p, err_.p);
                scan_exclusive<int>(jlen_.p, jdc.p, nact, scanws_.p, st_);
                jdp.reserve((size_t)read_int(jdc.p + nact) + 1);
                if (!nact) continue;
                if (lo)
                    launch(k_jds_fill<true>, nblk(nact, 4), 128, 0, st_, nact, (const int2 *)adesc_.p, xp,
                           (const int *)jdc.p, (const int *)row_ptr_.p, (const int *)inpos_.p,
                           (const int *)outpos_.p, (const int *)col_.p, (const double *)F_.p, jdp.p, jperm_lo_.p,
                           xc_lo_.p, xf_lo_.p);
                else
                    launch(k_jds_fill<false>, nblk(nact, 4), 128, 0, st_, nact, (const int2 *)adesc_.p, xp,
                           (const int *)jdc.p, (const int *)row_ptr_.p, (const int *)inpos_.p,
                           (const int *)outpos_.p, (const int *)col_.p, (const double *)F_.p, jdp.p, jperm_up_.p,
                           xc_up_.p, xf_up_.p);
            }
        } else {
            launch(k_cross_fill, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)row_ptr_.p,
                   (const int *)inpos_.p, (const int *)outpos_.p, (const int *)col_.p, (const double *)F_.p,
                   (const int *)xp_lo_.p, (const int *)xp_up_.p, xc_lo_.p, xf_lo_.p, xc_up_.p, xf_up_.p, swc,
                   xs_lo_.p, xs_up_.p);
        }
        // inverses of the in-cell diagonal blocks of the factor, and the
        // windows of each colour's range for the staged in-cell sweeps
        inv_len_.reserve((size_t)nact + 1);
        inv_off_.reserve((size_t)nact + 1);
        if (nact) launch(k_inv_sizes, nblk(nact, TPB), TPB, 0, st_, nact, (const int2 *)adesc_.p, inv_len_.p);
        scan_exclusive<int>(inv_len_.p, inv_off_.p, nact, scanws_.p, st_);
        ColourIdx at{};
        for (int c = 0; c <= ncol; c++) at.k[c] = act_off_[c];
        colinv_.reserve(16);
        launch(k_gather_colour_offsets, 1, 32, 0, st_, at, ncol + 1, (const int *)inv_off_.p, colinv_.p);
        MPS_CUDA(cudaMemcpyAsync(int_host_, colinv_.p, sizeof(int) * (ncol + 1), cudaMemcpyDeviceToHost, st_));
        MPS_CUDA(cudaStreamSynchronize(st_));
        int ninv = int_host_[ncol];
        if (ninv < 0) throw CudaError("in-cell inverses too large for 32-bit offsets", MPS_ERR_UNSUPPORTED);
        inv_col_off_.assign(int_host_, int_host_ + ncol + 1);
        inv_cm_.reserve((size_t)ninv + 1);
        inv_rm_.reserve((size_t)ninv + 1);
        ninv_ = ninv;
        if (nact)
            launch(k_cell_inverse, nblk(nact, 4), 128, 0, st_, nact, (const int2 *)adesc_.p,
                   (const int *)inv_off_.p, (const int *)pk_off_lo_.p, (const int *)pk_len_lo_.p,
                   (const double *)pk_val_lo_.p, (const unsigned char *)pk_k_lo_.p, (const double *)dinv_.p,
                   inv_cm_.p, inv_rm_.p);
        win_valid_ = false;
        if (sweep_mode_ == 0) build_windows(prm_.precision == MPS_PREC_MIXED);
        met.sweep_cross_lo = nx_lo_;
        met.sweep_cross_up = nx_up_;
        met.sweep_inverse_entries = ninv_;
    }
    MPS_CUDA(cudaEventRecord(ev_[3], st_));

    ic0_valid_ = icc;
    last_fp32_ = prm_.precision == MPS_PREC_MIXED;
    if (prm_.precision == MPS_PREC_MIXED) {
        mixed_solve(n_eq, nnz, icc);
    } else {
        PcgBufs<double> v{A_.p,         xf_lo_.p,  xf_up_.p,  pk_val_lo_.p, pk_val_up_.p, dinv_.p, inv_cm_.p,
                          inv_rm_.p,    x_.p,      r_.p,      z_.p,         p_.p,         Ap_.p,   y_.p,
                          part_.p,      b_.p};
        pcg_solve<double>(v, prm_.cg_tolerance, prm_.cg_max_iter, icc, n_eq, nnz);
        met.ppe_iterations = sc_host_->iter;
        met.ppe_outer = 1;
        met.ppe_residual = std::sqrt(sc_host_->rr);
        met.converged = std::sqrt(sc_host_->rr) < prm_.cg_tolerance;
        met.total_iterations += sc_host_->iter;
        launch(k_true_residual, RED_BLOCKS, CG_BLOCK, 0, st_, n_eq, (const int *)row_ptr_.p, (const int *)col_.p,
               (const double *)A_.p, (const double *)x_.p, (const double *)b_.p, partials_.p, ticket_.p, sc_.p);
        MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
        MPS_CUDA(cudaStreamSynchronize(st_));
        met.ppe_true_residual = std::sqrt(sc_host_->rr_outer);
        met.ppe_bnorm = std::sqrt(sc_host_->bb);
        met.ppe_rounding_floor = kUnitRoundoff * std::sqrt(sc_host_->ff);
    }
    launch(k_writeback<D>, nb, TPB, 0, st_, s, row_of_.p, x_.p, n, clamp);
    MPS_CUDA(cudaGetLastError());
    ppe_valid_ = true;
}

// One IC(0) sweep of the current factor, forward (rhs v.r, result v.y) or
// backward (rhs v.y, result v.z), colour by colour: the cross-cell products
// of each colour's rows from the colours swept before it, then the in-cell
// products with the block inverses.
template <int D>
template <class TM>
void Engine<D>::run_sweep(const PcgBufs<TM> &v, bool fwdir)
{
    using T = double;
    int ncol = 1 << D;
    auto lk = [&](int bit, auto kern, dim3 g, dim3 b, size_t sm, auto... args) {
        if (pdl_mask_ & bit) launch_pdl(kern, g, b, sm, st_, args...);
        else launch(kern, g, b, sm, st_, args...);
    };
    {
        const T *rhs = fwdir ? v.r : v.y;
        T *out = fwdir ? v.y : v.z;
        const int *pko = fwdir ? pk_off_lo_.p : pk_off_up_.p, *pkl = fwdir ? pk_len_lo_.p : pk_len_up_.p;
        const TM *pkv = fwdir ? v.pkv_lo : v.pkv_up;
        const unsigned char *pkk = fwdir ? pk_k_lo_.p : pk_k_up_.p;
        int order[8], nc = 0;
        for (int i = 0; i < ncol; i++) {
            int c = fwdir ? i : ncol - 1 - i;
            if (act_off_[c + 1] > act_off_[c]) order[nc++] = c;
        }
        if (sweep_mode_ == 1) {
            auto cellk = fwdir ? k_sweep_cell<true, TM> : k_sweep_cell<false, TM>;
            int resident = 0;
            MPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, cellk, 32 * JW, 0));
            resident *= num_sms_;
            for (int i = 0; i < nc; i++) {
                int c = order[i];
                int kb = act_off_[c], ke = act_off_[c + 1];
                // the last wave's CTAs trigger the next launch (cell_early_: all of them)
                int from = cell_early_ ? 0 : std::max(0, ke - kb - resident);
                lk(2, cellk, ke - kb, 32 * JW, 0, kb, ke, (const int2 *)adesc_.p, (const int *)inv_off_.p,
                   fwdir ? v.inv_cm : v.inv_rm, pko, pkl, pkv, pkk, v.dinv,
                   (const int *)(fwdir ? jdc_lo_.p : jdc_up_.p), (const int *)(fwdir ? jdp_lo_.p : jdp_up_.p),
                   (const unsigned char *)(fwdir ? jperm_lo_.p : jperm_up_.p),
                   (const int *)(fwdir ? xc_lo_.p : xc_up_.p), fwdir ? v.xf_lo : v.xf_up, (const T *)rhs, out,
                   (const CGScalars *)sc_.p, first_polls_, from, err_.p);
            }
            return;
        }
        auto colk = fwdir ? k_sweep_colour<true, TM> : k_sweep_colour<false, TM>;
        if (head_batch_ == 8) colk = fwdir ? k_sweep_colour<true, TM, 8> : k_sweep_colour<false, TM, 8>;
        // 8 CTAs per SM: 32 registers per thread and, in FP64, a stage that
        // holds the window plus one cell of up to 40 unknowns.  The default
        // is 8 for the mixed form's FP32 factor and 6 in FP64 (measured at c2:
        // FP32 sweeps 4.5 % faster at 8, FP64 sweeps 23 % slower)
        int stage = win_ + CELL_MAXBLK;
        int occ = sweep_occ_ ? sweep_occ_ : (sizeof(TM) == 4 ? 8 : 6);
        if (occ == 8) {
            colk = fwdir ? k_sweep_colour<true, TM, 4, 8> : k_sweep_colour<false, TM, 4, 8>;
            if (sizeof(TM) == 8) stage = win_ + 824;
        }
        // two head rows per lane group: half the cross CTAs, each with two
        // rows' loads in flight
        if (head_rows_ == 2) {
            if (occ == 8) colk = fwdir ? k_sweep_colour<true, TM, 4, 8, 2> : k_sweep_colour<false, TM, 4, 8, 2>;
            else colk = fwdir ? k_sweep_colour<true, TM, 4, 6, 2> : k_sweep_colour<false, TM, 4, 6, 2>;
        }
        // the FP32 cross runs as packed words
        if constexpr (sizeof(TM) == 4) {
            if (v.xfc_lo) {
                if (occ == 8 && head_rows_ == 2)
                    colk = fwdir ? k_sweep_colour<true, TM, 4, 8, 2, true> : k_sweep_colour<false, TM, 4, 8, 2, true>;
                else if (occ == 8)
                    colk = fwdir ? k_sweep_colour<true, TM, 4, 8, 1, true> : k_sweep_colour<false, TM, 4, 8, 1, true>;
                else if (head_rows_ == 2)
                    colk = fwdir ? k_sweep_colour<true, TM, 4, 6, 2, true> : k_sweep_colour<false, TM, 4, 6, 2, true>;
                else
                    colk = fwdir ? k_sweep_colour<true, TM, 4, 6, 1, true> : k_sweep_colour<false, TM, 4, 6, 1, true>;
            }
        }
        for (int i = 0; i < nc; i++) {
            int c = order[i], cn = i + 1 < nc ? order[i + 1] : -1;
            int nrb = cn >= 0 ? row_off_[cn] : 0, nre = cn >= 0 ? row_off_[cn + 1] : 0;
            int ncb = cn >= 0 ? nblk((long long)(nre - nrb) * 8, CELL_THREADS * head_rows_) : 0;
            lk(2, colk, nwin_[c] + ncb, CELL_THREADS, sizeof(TM) * stage,
               (const int *)wfirst_.p + win_off_[c], nwin_[c], (const int2 *)adesc_.p, (const int *)inv_off_.p,
               fwdir ? v.inv_cm : v.inv_rm, pko, pkl, pkv, pkk, v.dinv, (const int *)(fwdir ? xp_lo_.p : xp_up_.p),
               (const int *)(fwdir ? xs_lo_.p : xs_up_.p), (const int *)(fwdir ? xc_lo_.p : xc_up_.p),
               fwdir ? v.xf_lo : v.xf_up, (int)(i == 0), nrb, nre, rhs, v.part, out, (const CGScalars *)sc_.p,
               stage, first_polls_, err_.p, fwdir ? v.xfc_lo : v.xfc_up);
        }
    }
}

// PCG of pressure_solver.c:261-322 (CG of :90-131 when icc is false) on the
// block-colour system, values and vectors of type T, dot products in FP64.
// r is initialised from v.b (which may alias r); stops at sqrt(r.r) < tol,
// the reference's test, or after maxit iterations.  Leaves the final
// scalars in *sc_host_.
template <int D>
template <class TM>
void Engine<D>::pcg_solve(const PcgBufs<TM> &v, double tol, int maxit, bool icc, int n_eq, long long nnz,
                          const double *zprev)
{
    using T = double;
    int ncol = 1 << D;
    const int RB = RED_BLOCKS;
    int iter_before = 0;
    if (!zprev) {
        CGScalars init{};
        init.tol = tol;
        init.maxit = maxit;
        MPS_CUDA(cudaMemcpyAsync(sc_.p, &init, sizeof(CGScalars), cudaMemcpyHostToDevice, st_));
        launch(k_cg_init<T>, RB, CG_BLOCK, 0, st_, n_eq, v.x, v.r, v.b);
    } else {
        // resumed after a reliable update: the scalars of the stopped loop stay
        iter_before = sc_host_->iter;
        MPS_CUDA(cudaMemsetAsync(&sc_.p->done, 0, sizeof(int), st_));
    }
    T *z = icc ? v.z : v.r;
    // CG-loop launch: as a programmatic dependent when its group's bit is in pdl_mask_
    auto lk = [&](int bit, auto kern, dim3 g, dim3 b, size_t sm, auto... args) {
        if (pdl_mask_ & bit) launch_pdl(kern, g, b, sm, st_, args...);
        else launch(kern, g, b, sm, st_, args...);
    };
    auto sweep = [&](bool fwdir) { run_sweep<TM>(v, fwdir); };
    const int lpr = spmv_lpr_ ? spmv_lpr_ : (sizeof(TM) == 8 ? 8 : 16);
    auto spmv = [&]() {
        const int *rp = row_ptr_.p, *ci = col_.p;
        if (v.A64)
            lk(4, k_cg_spmv<8, double>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A64, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, (const double *)nullptr, (const uint2 *)nullptr);
        else if (v.dsum && v.ac) {
            if constexpr (sizeof(TM) == 4) {
                if (lpr == 16)
                    lk(4, k_cg_spmv<16, TM, true, true>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap,
                       partials_.p, ticket_.p, sc_.p, v.dsum, v.ac);
                else
                    lk(4, k_cg_spmv<8, TM, true, true>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap,
                       partials_.p, ticket_.p, sc_.p, v.dsum, v.ac);
            }
        }
        else if (v.dsum && lpr == 16)
            lk(4, k_cg_spmv<16, TM, true>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, v.dsum, (const uint2 *)nullptr);
        else if (v.dsum)
            lk(4, k_cg_spmv<8, TM, true>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, v.dsum, (const uint2 *)nullptr);
        else if (lpr == 16)
            lk(4, k_cg_spmv<16, TM>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, (const double *)nullptr, (const uint2 *)nullptr);
        else if (lpr == 32)
            lk(4, k_cg_spmv<32, TM>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, (const double *)nullptr, (const uint2 *)nullptr);
        else
            lk(4, k_cg_spmv<8, TM>, RB, CG_BLOCK, 0, n_eq, rp, ci, v.A, (const T *)v.p, v.Ap, partials_.p,
               ticket_.p, sc_.p, (const double *)nullptr, (const uint2 *)nullptr);
    };
    const bool persist = icc && sweep_mode_ == 2;
    if (icc) {
        if (persist) launch_pcg<TM>(v, true, 0);
        else {
            sweep(true);
            sweep(false);
        }
    }
    if (!zprev)
        launch(k_cg_init2<T>, RB, CG_BLOCK, 0, st_, n_eq, (const T *)v.r, (const T *)z, v.p, partials_.p, ticket_.p,
               sc_.p);
    else
        launch(k_reliable_fix<T>, RB, CG_BLOCK, 0, st_, n_eq, (const T *)v.r, (const T *)z, zprev, v.p, tol,
               partials_.p, ticket_.p, sc_.p);
    if (persist) {
        // one cooperative launch per batch; the kernel stops by itself at
        // convergence, so the host only reads the scalars between batches
        for (;;) {
            bool prof = profiling;
            if (prof) MPS_CUDA(cudaEventRecord(pev_[0], st_));
            launch_pcg<TM>(v, false, pcg_batch_);
            if (prof) MPS_CUDA(cudaEventRecord(pev_[1], st_));
            MPS_CUDA(cudaGetLastError());
            MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
            MPS_CUDA(cudaMemcpyAsync(int_host_ + 60, err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st_));
            MPS_CUDA(cudaStreamSynchronize(st_));
            if (int_host_[60]) check_err();
            int worked = sc_host_->iter - iter_before;
            if (prof) {
                float ms = 0;
                cudaEventElapsedTime(&ms, pev_[0], pev_[1]);
                met.prof_pcg_ms += ms;
                met.prof_pcg_launches += 1;
                met.prof_pcg_iterations += worked;
                met.prof_iterations += worked;
                met.prof_nnz_sum += (long long)worked * nnz;
                met.prof_rows_sum += (long long)worked * n_eq;
            }
            if (prof) trace_phases(worked);
            iter_before = sc_host_->iter;
            if (sc_host_->done) break;
        }
        return;
    }
    for (;;) {
        bool prof = profiling;
        for (int it = 0; it < CG_BATCH; it++) {
            cudaEvent_t *e = pev_ + it * PEV;
            if (prof) MPS_CUDA(cudaEventRecord(e[0], st_));
            spmv();
            if (prof) MPS_CUDA(cudaEventRecord(e[1], st_));
            lk(4, k_cg_axpy<T>, RB, CG_BLOCK, 0, n_eq, v.x, v.r, (const T *)v.p, (const T *)v.Ap, partials_.p,
               ticket_.p, sc_.p);
            if (prof) MPS_CUDA(cudaEventRecord(e[2], st_));
            if (icc) sweep(true);
            if (prof) MPS_CUDA(cudaEventRecord(e[3], st_));
            if (icc) sweep(false);
            if (prof) MPS_CUDA(cudaEventRecord(e[4], st_));
            lk(4, k_cg_rz<T>, RB, CG_BLOCK, 0, n_eq, (const T *)v.r, (const T *)z, partials_.p, ticket_.p, sc_.p);
            lk(4, k_cg_update_p<T>, RB, CG_BLOCK, 0, n_eq, v.p, (const T *)z, sc_.p);
        }
        MPS_CUDA(cudaGetLastError());
        MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
        MPS_CUDA(cudaStreamSynchronize(st_));
        if (prof) {
            int worked = sc_host_->iter - iter_before;   // iterations that did work in this batch
            for (int it = 0; it < worked && it < CG_BATCH; it++) {
                cudaEvent_t *e = pev_ + it * PEV;
                float a = 0, b2 = 0, c2 = 0, d2 = 0;
                cudaEventElapsedTime(&a, e[0], e[1]);
                cudaEventElapsedTime(&b2, e[1], e[2]);
                cudaEventElapsedTime(&c2, e[2], e[3]);
                cudaEventElapsedTime(&d2, e[3], e[4]);
                met.prof_spmv_ms += a;
                met.prof_spmv_launches += 1;
                met.prof_vec_ms += b2;
                if (icc) {
                    met.prof_fwd_ms += c2;
                    met.prof_fwd_sweeps += 1;
                    met.prof_bwd_ms += d2;
                    met.prof_bwd_sweeps += 1;
                }
                met.prof_iterations += 1;
                met.prof_nnz_sum += nnz;
                met.prof_rows_sum += n_eq;
            }
        }
        iter_before = sc_host_->iter;
        if (sc_host_->done) break;
    }
}

// Phase times of the last k_pcg launch from its trace (CTA 0's global timer
// as it left each barrier), added to the profiling metrics: per iteration
// the SpMV phase, the forward phases (the last colour's fused backward
// in-cell product included) and the backward phases.
template <int D>
void Engine<D>::trace_phases(int iterations)
{
    int nc = 0;
    for (int c = 0; c < (1 << D); c++) nc += act_off_[c + 1] > act_off_[c];
    trace_host_.resize(PCG_TRACE + 2);
    MPS_CUDA(cudaMemcpy(trace_host_.data(), pcg_trace_.p, sizeof(unsigned long long) * (PCG_TRACE + 2),
                        cudaMemcpyDeviceToHost));
    long long nbar = (long long)trace_host_[PCG_TRACE + 1];
    const unsigned long long *t = trace_host_.data();
    int per = 2 * nc;   // barriers per iteration
    for (int it = 0; it < iterations; it++) {
        long long b0 = (long long)it * per;
        if (b0 + per > nbar || b0 + per > PCG_TRACE) break;
        met.prof_spmv_ms += 1e-6 * (double)(t[b0 + 1] - t[b0]);
        met.prof_spmv_launches += 1;
        met.prof_fwd_ms += 1e-6 * (double)(t[b0 + 1 + nc] - t[b0 + 1]);
        met.prof_fwd_sweeps += 1;
        met.prof_bwd_ms += 1e-6 * (double)(t[b0 + per] - t[b0 + 1 + nc]);
        met.prof_bwd_sweeps += 1;
    }
}

// Grid of k_pcg: every CTA must be resident at once (the grid barriers wait
// for all of them), so the grid is the occupancy, at most 2 CTAs per SM,
// times the SM count; a cooperative launch refuses anything larger.
template <int D>
int Engine<D>::pcg_grid(const void *kernel)
{
    int nb = 0;
    MPS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, PCG_THREADS, 0));
    nb = std::min(nb, 2);
    if (nb < 1) throw CudaError("the persistent PCG kernel cannot be resident", MPS_ERR_CUDA);
    return nb * num_sms_;
}

template <int D>
template <class TM>
void Engine<D>::launch_pcg(const PcgBufs<TM> &v, bool apply, int batch)
{
    PcgArgs<TM> a{};
    int nc = 0;
    for (int c = 0; c < (1 << D); c++)
        if (act_off_[c + 1] > act_off_[c]) {
            a.kb[nc] = act_off_[c];
            a.ke[nc] = act_off_[c + 1];
            nc++;
        }
    if (nc == 0) return;
    if (v.A64) throw CudaError("the persistent PCG kernel reads the matrix in its storage type only", MPS_ERR_UNSUPPORTED);
    a.n_eq = n_eq_;
    a.ncol = nc;
    a.row_ptr = row_ptr_.p;
    a.colidx = col_.p;
    a.A = v.A;
    a.dsum = v.dsum;
    a.desc = adesc_.p;
    a.inv_off = inv_off_.p;
    a.inv_cm = v.inv_cm;
    a.inv_rm = v.inv_rm;
    a.jdc_lo = jdc_lo_.p;
    a.jdp_lo = jdp_lo_.p;
    a.jdc_up = jdc_up_.p;
    a.jdp_up = jdp_up_.p;
    a.jperm_lo = jperm_lo_.p;
    a.jperm_up = jperm_up_.p;
    a.xc_lo = xc_lo_.p;
    a.xc_up = xc_up_.p;
    a.xf_lo = v.xf_lo;
    a.xf_up = v.xf_up;
    a.pk_off_lo = pk_off_lo_.p;
    a.pk_len_lo = pk_len_lo_.p;
    a.pk_off_up = pk_off_up_.p;
    a.pk_len_up = pk_len_up_.p;
    a.pkv_lo = v.pkv_lo;
    a.pkv_up = v.pkv_up;
    a.pkk_lo = pk_k_lo_.p;
    a.pkk_up = pk_k_up_.p;
    a.dinv = v.dinv;
    a.x = v.x;
    a.r = v.r;
    a.y = v.y;
    a.z = v.z;
    a.Ap = v.Ap;
    a.p = v.p;
    a.p2 = p2_.p;
    a.sc = sc_.p;
    a.partials = partials_.p;
    a.bar = pcg_bar_.p;
    a.err = err_.p;
    a.batch = batch;
    a.apply = apply ? 1 : 0;
    a.bar_polls = bar_polls_;
    a.trace = nullptr;
    if (profiling && !apply) {
        pcg_trace_.reserve(PCG_TRACE + 2);
        a.trace = pcg_trace_.p;
    }
    const void *k;
    int variant;
    if constexpr (sizeof(TM) == 8) {
        k = (const void *)k_pcg<TM, false>;
        variant = 0;
    } else {
        if (v.dsum) {
            k = (const void *)k_pcg<TM, true>;
            variant = 1;
        } else {
            k = (const void *)k_pcg<TM, false>;
            variant = 2;
        }
    }
    if (!pcg_grid_[variant]) pcg_grid_[variant] = pcg_grid(k);
    int grid = pcg_grid_[variant];
    if ((size_t)PCG_SLOTS * grid > partials_.n) throw CudaError("PCG partials too small", MPS_ERR_CUDA);
    MPS_CUDA(cudaMemsetAsync(pcg_bar_.p, 0, sizeof(unsigned), st_));
    void *args[] = {&a};
    MPS_CUDA(cudaLaunchCooperativeKernel(k, grid, PCG_THREADS, args, 0, st_));
    ++launch_counter();
}

// Window tables of the staged in-cell sweeps for the current factor: each
// colour's range of block inverses split into windows of win_ entries
// (MPS_CELL_WIN if set, else 8 KB of inverse entries in the precision the
// sweeps run in: 1,024 FP64, 2,048 FP32).
template <int D>
void Engine<D>::build_windows(bool fp32)
{
    int want = cell_win_ ? cell_win_ : (fp32 ? 2 * CELL_WIN : CELL_WIN);
    if (want == win_ && win_valid_) return;
    int ncol = (int)inv_col_off_.size() - 1;
    win_ = want;
    win_off_.assign(ncol + 1, 0);
    nwin_.assign(ncol, 0);
    for (int c = 0; c < ncol; c++) {
        int span = inv_col_off_[c + 1] - inv_col_off_[c];
        nwin_[c] = act_off_[c + 1] > act_off_[c] ? std::max(1, (span + win_ - 1) / win_) : 0;
        win_off_[c + 1] = win_off_[c] + nwin_[c] + 1;
    }
    wfirst_.reserve((size_t)win_off_[ncol] + 1);
    for (int c = 0; c < ncol; c++)
        if (nwin_[c])
            launch(k_inv_windows, nblk(nwin_[c] + 1, TPB), TPB, 0, st_, act_off_[c], act_off_[c + 1],
                   (const int *)inv_off_.p, win_, nwin_[c], wfirst_.p + win_off_[c]);
    win_valid_ = true;
}

// Mixed form: the ICCG with the matrix and the IC(0) factor stored in FP32
// (the SpMV in difference form, k_cg_spmv<.., true>) and FP64 vectors and
// arithmetic, with reliable updates.  Whenever the recursive residual has
// fallen by rel_delta_ since the last update, the true residual r = b - A x
// is recomputed with the FP64 matrix and the iteration resumes from it with
// its search direction kept.  Stops when ||b - A x|| <= max(cg_tolerance,
// refine_tolerance ||b||, kFloor u || |b| + |A| |x| ||), u the FP64 unit
// roundoff: kFloor times the rounding floor of an FP64 residual, where the
// FP64 form's own solve ends; or when the true residual stalls.
template <int D>
void Engine<D>::mixed_solve(int n_eq, long long nnz, bool icc, bool adjoint)
{
    const int RB = RED_BLOCKS;
    size_t nz = (size_t)nnz;
    // packed words for the launch-per-colour loop; the persistent and the
    // CTA-per-cell loops read the separate arrays
    const bool pk = pack_ && sweep_mode_ == 0 && head_batch_ == 4;
    const bool pk_spmv = pk && mixed_spmv_ == 2;
    for (auto *v : {&A32_, &pkv32_lo_, &pkv32_up_}) v->reserve(nz);
    xf32_lo_.reserve((size_t)nx_lo_ + 1);
    xf32_up_.reserve((size_t)nx_up_ + 1);
    for (auto *v : {&inv32_cm_, &inv32_rm_}) v->reserve((size_t)ninv_ + 1);
    dinv32_.reserve((size_t)cap_);
    zprev_.reserve((size_t)cap_);
    if (pk_spmv) {
        ac32_.reserve(nz);
        launch(k_pack_fc, RB, CG_BLOCK, 0, st_, nz, (const double *)A_.p, (const int *)col_.p, ac32_.p);
    } else
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, nz, (const double *)A_.p, A32_.p);
    if (icc && pk) {
        xfc32_lo_.reserve((size_t)nx_lo_ + 1);
        xfc32_up_.reserve((size_t)nx_up_ + 1);
        launch(k_pack_fc, RB, CG_BLOCK, 0, st_, (size_t)nx_lo_, (const double *)xf_lo_.p, (const int *)xc_lo_.p,
               xfc32_lo_.p);
        launch(k_pack_fc, RB, CG_BLOCK, 0, st_, (size_t)nx_up_, (const double *)xf_up_.p, (const int *)xc_up_.p,
               xfc32_up_.p);
    }
    packed_ = icc && pk;
    if (icc) {
        if (!pk) {
            launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, (size_t)nx_lo_, (const double *)xf_lo_.p,
                   xf32_lo_.p);
            launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, (size_t)nx_up_, (const double *)xf_up_.p,
                   xf32_up_.p);
        }
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, nz, (const double *)pk_val_lo_.p, pkv32_lo_.p);
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, nz, (const double *)pk_val_up_.p, pkv32_up_.p);
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, (size_t)n_eq, (const double *)dinv_.p, dinv32_.p);
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, (size_t)ninv_, (const double *)inv_cm_.p,
               inv32_cm_.p);
        launch(k_convert<double, float>, RB, CG_BLOCK, 0, st_, (size_t)ninv_, (const double *)inv_rm_.p,
               inv32_rm_.p);
    }
    CGScalars init{};
    MPS_CUDA(cudaMemcpyAsync(sc_.p, &init, sizeof(CGScalars), cudaMemcpyHostToDevice, st_));
    launch(k_refine_init, RB, CG_BLOCK, 0, st_, n_eq, x_.p, r_.p, (const double *)b_.p, partials_.p, ticket_.p,
           sc_.p);
    MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    double bnorm = std::sqrt(sc_host_->rr_outer);
    double target = adjoint ? kAdjRtol * bnorm
                            : std::max(prm_.cg_tolerance, std::max(prm_.refine_tolerance, 0.0) * bnorm);
    double rnorm = bnorm, rbest = bnorm, floor_norm = 0.0;
    int updates = 0, stalls = 0;
    PcgBufs<float> v{A32_.p,      xf32_lo_.p, xf32_up_.p, pkv32_lo_.p, pkv32_up_.p, dinv32_.p, inv32_cm_.p,
                     inv32_rm_.p, x_.p,       r_.p,       z_.p,        p_.p,        Ap_.p,     y_.p,
                     part_.p,     b_.p};
    if (mixed_spmv_ == 1 && sweep_mode_ != 2) v.A64 = A_.p;   // tuning alternatives of the inner SpMV
    if (pk_spmv) v.ac = ac32_.p;
    if (packed_) {
        v.xfc_lo = xfc32_lo_.p;
        v.xfc_up = xfc32_up_.p;
    }
    if (mixed_spmv_ == 2) {
        dsum_.reserve((size_t)cap_);
        launch(k_row_sum, nblk(n_eq, TPB), TPB, 0, st_, n_eq, (const int *)row_ptr_.p, (const double *)A_.p,
               dsum_.p);
        v.dsum = dsum_.p;
    }
    const double *zsrc = icc ? z_.p : r_.p;   // the preconditioned residual
    if (rnorm > target) {
        pcg_solve<float>(v, std::max(target, rel_delta_ * rnorm), prm_.cg_max_iter, icc, n_eq, nnz);
        double goal = target;
        for (;;) {
            MPS_CUDA(cudaMemcpyAsync(zprev_.p, zsrc, sizeof(double) * n_eq, cudaMemcpyDeviceToDevice, st_));
            launch(k_refine_residual, RB, CG_BLOCK, 0, st_, n_eq, (const int *)row_ptr_.p, (const int *)col_.p,
                   (const double *)A_.p, (const double *)x_.p, (const double *)b_.p, r_.p, partials_.p, ticket_.p,
                   sc_.p);
            MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
            MPS_CUDA(cudaStreamSynchronize(st_));
            rnorm = std::sqrt(sc_host_->rr_outer);
            floor_norm = kUnitRoundoff * std::sqrt(sc_host_->ff);
            updates++;
            // stagnation: the true residual has stopped falling
            if (rnorm < kStall * rbest) stalls = 0;
            else stalls++;
            rbest = std::min(rbest, rnorm);
            goal = std::max(target, kFloor * floor_norm);
            if (rnorm <= goal || sc_host_->iter >= prm_.cg_max_iter || sc_host_->breakdown ||
                updates >= kMaxUpdates || stalls >= kMaxStalls)
                break;
            // the next inner solve aims at most at the goal: its recursive
            // residual tracks the true one closely (FP64 vectors)
            pcg_solve<float>(v, std::max(goal, rel_delta_ * rnorm), prm_.cg_max_iter, icc, n_eq, nnz, zprev_.p);
        }
    }
    int inner = sc_host_->iter;
    if (adjoint) return;
    met.ppe_iterations = inner;
    met.ppe_outer = updates;
    met.ppe_residual = rnorm;
    met.ppe_true_residual = rnorm;
    met.ppe_bnorm = bnorm;
    met.ppe_rounding_floor = floor_norm;
    met.converged = rnorm <= std::max(target, kFloor * floor_norm);
    met.total_iterations += inner;
}

// ---- differentiation form ----------------------------------------------------
//
// A checkpoint is the current state buffer (positions, velocities,
// accelerations, sort keys, pressures, densities, types, flags, reference
// indices, cell indices) with the cell starts of its structure: everything
// the next step reads, so that loading it and stepping reproduces the step
// bit for bit.

// Drive values at time t: displacement A sin(w t) and velocity A w cos(w t),
// w = 2 pi f (the oracle's oracle_wall_drive_terms, the same expressions).
template <int D>
void Engine<D>::drive_terms(double t, double *dx, double *vel) const
{
    double w = 2.0 * 3.14159265358979323846 * prm_.wall_drive_freq;
    double ph = w * t;
    *dx = prm_.wall_drive_amp * std::sin(ph);
    *vel = prm_.wall_drive_amp * w * std::cos(ph);
}

namespace {
struct StateHeader {
    long long magic, n, cap, total, dim, tstep;
};
constexpr long long kStateMagic = 0x4d50535354415445LL;
}  // namespace

template <int D>
size_t Engine<D>::state_bytes() const
{
    size_t nd = (size_t)(4 * D + 2), ni = 5;
    return sizeof(StateHeader) + (nd * cap_) * sizeof(double) + (ni * cap_) * sizeof(int) +
           ((size_t)g_.total + 2) * sizeof(int);
}

template <int D>
void Engine<D>::state_save(void *dst)
{
    if (!structure_) throw CudaError("no neighbour structure to checkpoint", MPS_ERR_INVALID);
    if (!dst) throw CudaError("null checkpoint buffer", MPS_ERR_INVALID);
    size_t nd = (size_t)(4 * D + 2), ni = 5;
    StateHeader h{kStateMagic, n_, cap_, g_.total, D, tstep_};
    char *o = (char *)dst;
    MPS_CUDA(cudaMemcpyAsync(o, &h, sizeof h, cudaMemcpyDefault, st_));
    o += sizeof h;
    MPS_CUDA(cudaMemcpyAsync(o, dbuf_[cur_].p, nd * cap_ * sizeof(double), cudaMemcpyDefault, st_));
    o += nd * cap_ * sizeof(double);
    MPS_CUDA(cudaMemcpyAsync(o, ibuf_[cur_].p, ni * cap_ * sizeof(int), cudaMemcpyDefault, st_));
    o += ni * cap_ * sizeof(int);
    MPS_CUDA(cudaMemcpyAsync(o, start_.p, ((size_t)g_.total + 2) * sizeof(int), cudaMemcpyDefault, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::state_load(const void *src)
{
    if (!src) throw CudaError("null checkpoint buffer", MPS_ERR_INVALID);
    StateHeader h{};
    MPS_CUDA(cudaMemcpyAsync(&h, src, sizeof h, cudaMemcpyDefault, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    if (h.magic != kStateMagic || h.dim != D || h.cap != cap_ || h.total != g_.total || h.n < 0 || h.n > cap_)
        throw CudaError("checkpoint does not belong to this session", MPS_ERR_INVALID);
    size_t nd = (size_t)(4 * D + 2), ni = 5;
    const char *o = (const char *)src + sizeof h;
    MPS_CUDA(cudaMemcpyAsync(dbuf_[cur_].p, o, nd * cap_ * sizeof(double), cudaMemcpyDefault, st_));
    o += nd * cap_ * sizeof(double);
    MPS_CUDA(cudaMemcpyAsync(ibuf_[cur_].p, o, ni * cap_ * sizeof(int), cudaMemcpyDefault, st_));
    o += ni * cap_ * sizeof(int);
    MPS_CUDA(cudaMemcpyAsync(start_.p, o, ((size_t)g_.total + 2) * sizeof(int), cudaMemcpyDefault, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    n_ = (int)h.n;
    tstep_ = h.tstep;
    g_.start = start_.p;
    structure_ = true;
    ppe_valid_ = false;
}

template <int D>
void Engine<D>::ensure_adj()
{
    if (adj_cap_ == (size_t)cap_) return;
    size_t c = (size_t)cap_;
    adjd_.reserve((11 * D + 7) * c + (size_t)ADJ_MAXEV * 2 * D * c);
    adji_.reserve((2 + (size_t)ADJ_MAXEV) * c);
    adjsum_.reserve(D + 3);
    snap_.reserve(state_bytes());
    double *p = adjd_.p;
    auto take = [&](size_t m) {
        double *r = p;
        p += m;
        return r;
    };
    for (int d = 0; d < D; d++) {
        adj_.lx[d] = take(c);
        adj_.lu[d] = take(c);
        adj_.xs[d] = take(c);
        adj_.us[d] = take(c);
        adj_.lxc[d] = take(c);
        adj_.luc[d] = take(c);
        adj_.lxs[d] = take(c);
        adj_.lus[d] = take(c);
        adj_.lap[d] = take(c);
        adj_.la[d] = take(c);
        adj_.gv[d] = take(c);
    }
    adj_.pmv = take(c);
    adj_.psc = take(c);
    adj_.lp = take(c);
    adj_.mu = take(c);
    adj_.nv = take(c);
    adj_.dA = take(c);
    adj_.df = take(c);
    adj_.evd = take((size_t)ADJ_MAXEV * 2 * D * c);
    adj_.pmi = adji_.p;
    adj_.evn = adji_.p + c;
    adj_.evj = adji_.p + 2 * c;
    MPS_CUDA(cudaMemsetAsync(adjd_.p, 0, ((11 * D + 7) * c) * sizeof(double), st_));
    MPS_CUDA(cudaMemsetAsync(adji_.p, 0, 2 * c * sizeof(int), st_));
    MPS_CUDA(cudaMemsetAsync(adjsum_.p, 0, (D + 3) * sizeof(double), st_));
    adj_cap_ = c;
}

// Seeds (host, reference order, [n][D]; null = zero) of the adjoint of the
// state after the next step to be reversed; clears the parameter gradients.
template <int D>
void Engine<D>::adjoint_seed(const double *lam_pos, const double *lam_vel)
{
    ensure_adj();
    int n = n_;
    soa_in_.reserve((size_t)2 * D * cap_ + 2);
    double *dx = lam_pos ? soa_in_.p : nullptr, *du = lam_vel ? soa_in_.p + (size_t)D * cap_ : nullptr;
    if (lam_pos) MPS_CUDA(cudaMemcpyAsync(dx, lam_pos, sizeof(double) * D * n, cudaMemcpyHostToDevice, st_));
    if (lam_vel) MPS_CUDA(cudaMemcpyAsync(du, lam_vel, sizeof(double) * D * n, cudaMemcpyHostToDevice, st_));
    if (n) launch(k_adj_set<D>, nblk(n, TPB), TPB, 0, st_, n, (const double *)dx, (const double *)du, adj_);
    MPS_CUDA(cudaMemsetAsync(adjsum_.p, 0, (D + 3) * sizeof(double), st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    MPS_CUDA(cudaGetLastError());
}

template <int D>
void Engine<D>::adjoint_pressure_seed(const double *dLdP, int num)
{
    if (num != n_) throw CudaError("pressure seed size differs from the particle count", MPS_ERR_INVALID);
    if (!dLdP) {
        pseed_on_ = false;
        return;
    }
    pseed_.reserve((size_t)cap_ + 1);
    MPS_CUDA(cudaMemcpyAsync(pseed_.p, dLdP, sizeof(double) * num, cudaMemcpyHostToDevice, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    pseed_on_ = true;
}

template <int D>
void Engine<D>::adjoint_get(double *lam_pos, double *lam_vel, double *grad_gravity, double *grad_viscosity,
                            double *grad_drive)
{
    ensure_adj();
    int n = n_;
    soa_in_.reserve((size_t)2 * D * cap_ + 2);
    double *dx = soa_in_.p, *du = soa_in_.p + (size_t)D * cap_;
    if (n) launch(k_adj_get<D>, nblk(n, TPB), TPB, 0, st_, n, dx, du, adj_);
    if (lam_pos) MPS_CUDA(cudaMemcpyAsync(lam_pos, dx, sizeof(double) * D * n, cudaMemcpyDeviceToHost, st_));
    if (lam_vel) MPS_CUDA(cudaMemcpyAsync(lam_vel, du, sizeof(double) * D * n, cudaMemcpyDeviceToHost, st_));
    double sums[D + 3];
    MPS_CUDA(cudaMemcpyAsync(sums, adjsum_.p, sizeof(sums), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    if (grad_gravity)
        for (int d = 0; d < D; d++) grad_gravity[d] = sums[d];
    if (grad_viscosity) *grad_viscosity = sums[D];
    if (grad_drive) {
        grad_drive[0] = sums[D + 1];
        grad_drive[1] = sums[D + 2];
    }
}

// Adjoint of one step.  The session holds the step's input state; the
// adjoint seeds hold the adjoint of its output.  The step is recomputed
// (recording x*, u*), its implicit part is reversed on the fresh structure
// (correction, gradient, PPE by a second ICCG solve with the same matrix and
// IC(0) factor, density), the input state is restored and the explicit part
// is reversed on the previous step's structure (collision, explicit update,
// viscosity).  Afterwards the seeds hold the adjoint of the step's input,
// the parameter gradients have this step's terms added, and the session
// again holds the step's input state.
template <int D>
void Engine<D>::step_adjoint()
{
    require_ref();
    if (!structure_) throw CudaError("no neighbour structure: load a checkpoint first", MPS_ERR_INVALID);
    if (prm_.hs_mode != 0 || prm_.ppe_type != 0 || prm_.cmps_gradient != 0 || prm_.clamp_negative_pressure ||
        prm_.surface_tension_enabled || prm_.friction_enabled)
        throw CudaError("the adjoint supports hs_mode 0, ppe_type 0, cmps_gradient 0, no clamp, no surface tension "
                        "or friction",
                        MPS_ERR_UNSUPPORTED);
    ensure_adj();
    bool pseed = pseed_on_;   // consumed by this call
    pseed_on_ = false;
    int n = n_;
    if (!n) return;
    int nb = nblk(n, TPB);
    const int RB = RED_BLOCKS;
    state_save(snap_.p);
    // forward recompute
    adj_rec_ = true;
    try {
        explicit_stage(false);
    } catch (...) {
        adj_rec_ = false;
        throw;
    }
    adj_rec_ = false;
    sort();
    launch(k_density<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, err_.p, 1, 1);
    ppe(false);
    launch(k_pmin<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), n, pmin_.p);
    launch(k_gradient<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, (const double *)pmin_.p);
    check_err();
    // implicit part in reverse, on the fresh structure (state before the correction)
    launch(k_adj_seed<D>, nb, TPB, 0, st_, S(), k_, n, adj_);
    launch(k_adj_pmin<D>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_);
    launch(k_adj_gradient<D>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_);
    if (pseed) launch(k_adj_add, nb, TPB, 0, st_, n, (const double *)pseed_.p, adj_.lp);
    MPS_CUDA(cudaMemsetAsync(adj_.mu, 0, sizeof(double) * cap_, st_));
    int n_eq = n_eq_;
    if (n_eq > 0) {
        launch(k_adj_rhs, RB, CG_BLOCK, 0, st_, n_eq, (const int *)part_of_row_.p, (const int *)S().id,
               (const double *)adj_.lp, b_.p, partials_.p, ticket_.p, sc_.p);
        MPS_CUDA(cudaMemcpyAsync(sc_host_, sc_.p, sizeof(CGScalars), cudaMemcpyDeviceToHost, st_));
        MPS_CUDA(cudaStreamSynchronize(st_));
        double bnorm = std::sqrt(sc_host_->rr_outer);
        if (bnorm > 0.0) {
            launch(k_adj_scale, RB, CG_BLOCK, 0, st_, n_eq, b_.p, 1.0 / bnorm);
            bool icc = prm_.solver_type == 1;
            if (prm_.precision == MPS_PREC_MIXED) {
                // the mixed form's solve (FP32 matrix and factor, FP64
                // vectors, reliable updates) down to the same relative
                // residual, or to the FP64 rounding floor if that is higher
                if (icc && sweep_mode_ == 0) build_windows(true);
                mixed_solve(n_eq, nnz_, icc, true);
            } else {
                PcgBufs<double> v{A_.p,      xf_lo_.p, xf_up_.p, pk_val_lo_.p, pk_val_up_.p, dinv_.p, inv_cm_.p,
                                  inv_rm_.p, x_.p,     r_.p,     z_.p,         p_.p,         Ap_.p,   y_.p,
                                  part_.p,   b_.p};
                if (icc && sweep_mode_ == 0) build_windows(false);   // FP64 sweeps: FP64 windows
                pcg_solve<double>(v, kAdjRtol, prm_.cg_max_iter, icc, n_eq, nnz_);
            }
            launch(k_adj_mu, RB, CG_BLOCK, 0, st_, n_eq, (const int *)part_of_row_.p, (const int *)S().id,
                   (const double *)x_.p, bnorm, adj_.mu);
        }
    }
    launch(k_adj_ppe_pairs<D>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_, (const int *)row_of_.p);
    // explicit part in reverse, on the previous step's structure
    state_load(snap_.p);
    if (k_.collision_on) {
        if (D == 3) {
            launch(k_adj_collision<D, true>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_, err_.p);
            launch(k_adj_collision_gather<D>, nb, TPB, 0, st_, cells(), S(), n, adj_);
        } else {
            // the 2-D collision runs on a structure sorted after the explicit update
            launch(k_viscosity<D, CellSource<D>>, nb, TPB, 0, st_, cells(), S(), k_, n, 0);
            launch(k_explicit_update<D>, nb, TPB, 0, st_, S(), k_, n);
            sort();
            launch(k_adj_collision<D, false>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_, err_.p);
            launch(k_adj_collision_gather<D>, nb, TPB, 0, st_, cells(), S(), n, adj_);
            state_load(snap_.p);
        }
    } else {
        launch(k_adj_no_collision<D>, nb, TPB, 0, st_, S(), n, adj_);
    }
    launch(k_adj_accel<D>, nb, TPB, 0, st_, S(), k_, n, adj_);
    launch(k_adj_viscosity<D>, nb, TPB, 0, st_, cells(), S(), k_, n, adj_);
    {
        DriveT dv{};
        dv.A = prm_.wall_drive_amp;
        dv.w = 2.0 * 3.14159265358979323846 * prm_.wall_drive_freq;
        dv.t0 = (double)tstep_ * prm_.dt;
        dv.t1 = (double)(tstep_ + 1) * prm_.dt;
        dv.s0 = std::sin(dv.w * dv.t0);
        dv.c0 = std::cos(dv.w * dv.t0);
        dv.s1 = std::sin(dv.w * dv.t1);
        dv.c1 = std::cos(dv.w * dv.t1);
        dv.axis = prm_.wall_drive_axis;
        dv.first = tstep_ == 0;
        launch(k_adj_drive<D>, nb, TPB, 0, st_, S(), n, adj_, dv);
    }
    launch(k_adj_param_sum<D>, RB, CG_BLOCK, 0, st_, n, adj_, partials_.p, ticket_.p, adjsum_.p);
    MPS_CUDA(cudaGetLastError());
    unsigned e = 0;
    MPS_CUDA(cudaMemcpyAsync(int_host_, err_.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    std::memcpy(&e, int_host_, sizeof(unsigned));
    if (e & ERR_ADJ_EVENTS) {
        MPS_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(unsigned), st_));
        throw CudaError("more collision impulses on one particle than the adjoint records", MPS_ERR_UNSUPPORTED);
    }
    check_err();
}

// ---- introspection --------------------------------------------------------

// The current structure's list into the caller's reference-layout arrays:
// counts first, then the rows at a pitch of the longest row, copied out with
// one pitched copy.
template <int D>
void Engine<D>::get_neighbor_list(int *nb, int *cnt, int max_nb)
{
    if (!structure_) throw CudaError("no neighbour structure", MPS_ERR_INVALID);
    int n = n_;
    if (max_nb <= 0) throw CudaError("max_nb must be positive", MPS_ERR_INVALID);
    lcnt_.reserve((size_t)n + 1);
    std::vector<int> hc;
    int *hcnt = cnt;
    if (!hcnt) {
        hc.resize((size_t)n + 1);
        hcnt = hc.data();
    }
    if (n)
        launch(k_build_list<D>, nblk(n, TPB), TPB, 0, st_, cells(), (const int *)S().id, n, max_nb, 0,
               (int *)nullptr, lcnt_.p, err_.p);
    MPS_CUDA(cudaMemcpyAsync(hcnt, lcnt_.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st_));
    check_err();
    if (!nb || n == 0) return;
    int mc = 0;
    for (int i = 0; i < n; i++) mc = std::max(mc, hcnt[i]);
    if (mc == 0) return;
    lout_.reserve((size_t)n * mc);
    launch(k_build_list<D>, nblk(n, TPB), TPB, 0, st_, cells(), (const int *)S().id, n, max_nb, mc, lout_.p,
           lcnt_.p, err_.p);
    MPS_CUDA(cudaMemcpy2DAsync(nb, sizeof(int) * (size_t)max_nb, lout_.p, sizeof(int) * mc, sizeof(int) * mc, n,
                               cudaMemcpyDeviceToHost, st_));
    check_err();
}

template <int D>
void Engine<D>::get_cell_index(int *cell)
{
    if (!structure_) throw CudaError("no neighbour structure", MPS_ERR_INVALID);
    int n = n_;
    lcnt_.reserve((size_t)n + 1);
    if (n) launch(k_cell_ref_order<D>, nblk(n, TPB), TPB, 0, st_, S().cell, S().id, n, lcnt_.p);
    MPS_CUDA(cudaMemcpyAsync(cell, lcnt_.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::get_cell_links(int *head, int *next, int total)
{
    if (!structure_) throw CudaError("no neighbour structure", MPS_ERR_INVALID);
    if (total != g_.total) throw CudaError("cell count differs from the session grid", MPS_ERR_INVALID);
    int n = n_;
    link_head_.reserve((size_t)total + 1);
    link_next_.reserve((size_t)n + 1);
    int m = std::max(total, n);
    if (m)
        launch(k_cell_links, nblk(m, TPB), TPB, 0, st_, start_.p, S().id, S().cell, total, n, link_head_.p,
               link_next_.p);
    if (head) MPS_CUDA(cudaMemcpyAsync(head, link_head_.p, sizeof(int) * total, cudaMemcpyDeviceToHost, st_));
    if (next) MPS_CUDA(cudaMemcpyAsync(next, link_next_.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::get_ppe(int *eq_idx, int *row_ptr, int *col, double *val, double *b, int *n_eq, long long *nnz)
{
    if (!ppe_valid_) throw CudaError("no assembled PPE: run a step or the solve stage first", MPS_ERR_INVALID);
    if (n_eq) *n_eq = n_eq_;
    if (nnz) *nnz = nnz_;
    if (!row_ptr) return;
    int n = n_, ne = n_eq_;
    // reference numbering: unknowns in reference index order
    DevArray<int> by_id, eq_by_id, rp_ref, ccol;
    DevArray<double> cval, cb;
    by_id.reserve(n + 1);
    eq_by_id.reserve(n + 1);
    if (n) launch(k_ref_eq, nblk(n, TPB), TPB, 0, st_, row_of_.p, S().id, n, by_id.p);
    std::vector<int> h_by(n), h_eq(n);
    MPS_CUDA(cudaMemcpyAsync(h_by.data(), by_id.p, sizeof(int) * n, cudaMemcpyDeviceToHost, st_));
    std::vector<int> h_rp(ne + 1);
    MPS_CUDA(cudaMemcpyAsync(h_rp.data(), row_ptr_.p, sizeof(int) * (ne + 1), cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    int e = 0;
    std::vector<int> eng_row_of_ref(ne);
    for (int i = 0; i < n; i++) {
        if (h_by[i] >= 0) { eng_row_of_ref[e] = h_by[i]; h_eq[i] = e++; }
        else h_eq[i] = -1;
    }
    std::vector<int> ref_rp(ne + 1, 0);
    for (int r = 0; r < ne; r++) ref_rp[r + 1] = ref_rp[r] + (h_rp[eng_row_of_ref[r] + 1] - h_rp[eng_row_of_ref[r]]);
    MPS_CUDA(cudaMemcpyAsync(eq_by_id.p, h_eq.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st_));
    rp_ref.reserve(ne + 1);
    MPS_CUDA(cudaMemcpyAsync(rp_ref.p, ref_rp.data(), sizeof(int) * (ne + 1), cudaMemcpyHostToDevice, st_));
    ccol.reserve(nnz_ + 1);
    cval.reserve(nnz_ + 1);
    cb.reserve(ne + 1);
    if (ne)
        launch(k_ppe_to_ref, nblk(ne, TPB), TPB, 0, st_, ne, part_of_row_.p, S().id, eq_by_id.p, row_ptr_.p, col_.p,
                                                      A_.p, b_.p, part_of_row_.p, rp_ref.p, ccol.p, cval.p, cb.p);
    std::vector<int> hc(nnz_);
    std::vector<double> hv(nnz_);
    MPS_CUDA(cudaMemcpyAsync(hc.data(), ccol.p, sizeof(int) * nnz_, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaMemcpyAsync(hv.data(), cval.p, sizeof(double) * nnz_, cudaMemcpyDeviceToHost, st_));
    if (b) MPS_CUDA(cudaMemcpyAsync(b, cb.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    // sort each row by column (the reference's insertion sort, :536-551)
    std::vector<std::pair<int, double>> rowbuf;
    for (int r = 0; r < ne; r++) {
        rowbuf.clear();
        for (int q = ref_rp[r]; q < ref_rp[r + 1]; q++) rowbuf.push_back({hc[q], hv[q]});
        std::sort(rowbuf.begin(), rowbuf.end(),
                  [](const std::pair<int, double> &a, const std::pair<int, double> &b2) { return a.first < b2.first; });
        for (int q = ref_rp[r]; q < ref_rp[r + 1]; q++) {
            if (col) col[q] = rowbuf[q - ref_rp[r]].first;
            if (val) val[q] = rowbuf[q - ref_rp[r]].second;
        }
    }
    std::memcpy(row_ptr, ref_rp.data(), sizeof(int) * (ne + 1));
    if (eq_idx) std::memcpy(eq_idx, h_eq.data(), sizeof(int) * n);
}

template <int D>
void Engine<D>::get_ic0(int *row_ptr, int *col, double *A, double *F, double *b, int *n_eq, long long *nnz)
{
    if (!ppe_valid_ || !ic0_valid_) throw CudaError("no IC(0) factor: run an ICCG step first", MPS_ERR_INVALID);
    if (n_eq) *n_eq = n_eq_;
    if (nnz) *nnz = nnz_;
    if (!row_ptr) return;
    int ne = n_eq_;
    MPS_CUDA(cudaMemcpyAsync(row_ptr, row_ptr_.p, sizeof(int) * (ne + 1), cudaMemcpyDeviceToHost, st_));
    if (col) MPS_CUDA(cudaMemcpyAsync(col, col_.p, sizeof(int) * nnz_, cudaMemcpyDeviceToHost, st_));
    if (A) MPS_CUDA(cudaMemcpyAsync(A, A_.p, sizeof(double) * nnz_, cudaMemcpyDeviceToHost, st_));
    if (F) MPS_CUDA(cudaMemcpyAsync(F, F_.p, sizeof(double) * nnz_, cudaMemcpyDeviceToHost, st_));
    if (b) MPS_CUDA(cudaMemcpyAsync(b, b_.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::get_cell_blocks(int *cells, int *inv_off, double *inv, int *colour_rows, int *ncells,
                                long long *ninv)
{
    if (!ppe_valid_ || !ic0_valid_) throw CudaError("no IC(0) factor: run an ICCG step first", MPS_ERR_INVALID);
    int ncol = 1 << D;
    int nact = act_off_[ncol];
    if (ncells) *ncells = nact;
    if (ninv) *ninv = ninv_;
    if (colour_rows)
        for (int c = 0; c <= ncol; c++) colour_rows[c] = row_off_[c];
    if (cells && nact) MPS_CUDA(cudaMemcpyAsync(cells, adesc_.p, sizeof(int2) * nact, cudaMemcpyDeviceToHost, st_));
    if (inv_off) MPS_CUDA(cudaMemcpyAsync(inv_off, inv_off_.p, sizeof(int) * (nact + 1), cudaMemcpyDeviceToHost, st_));
    if (inv && ninv_) MPS_CUDA(cudaMemcpyAsync(inv, inv_cm_.p, sizeof(double) * ninv_, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
}

template <int D>
void Engine<D>::apply_preconditioner(const double *r, double *z)
{
    if (!ppe_valid_ || !ic0_valid_) throw CudaError("no IC(0) factor: run an ICCG step first", MPS_ERR_INVALID);
    if (!r || !z) throw CudaError("null vector", MPS_ERR_INVALID);
    int ne = n_eq_;
    MPS_CUDA(cudaMemcpyAsync(r_.p, r, sizeof(double) * ne, cudaMemcpyHostToDevice, st_));
    MPS_CUDA(cudaMemsetAsync(&sc_.p->done, 0, sizeof(int), st_));
    if (last_fp32_) {
        if (sweep_mode_ == 0) build_windows(true);
        PcgBufs<float> v{A32_.p,      xf32_lo_.p, xf32_up_.p, pkv32_lo_.p, pkv32_up_.p, dinv32_.p, inv32_cm_.p,
                         inv32_rm_.p, x_.p,       r_.p,       z_.p,        p_.p,        Ap_.p,     y_.p,
                         part_.p,     b_.p};
        if (packed_) {
            v.xfc_lo = xfc32_lo_.p;
            v.xfc_up = xfc32_up_.p;
        }
        if (sweep_mode_ == 2) launch_pcg<float>(v, true, 0);
        else {
            run_sweep<float>(v, true);
            run_sweep<float>(v, false);
        }
    } else {
        if (sweep_mode_ == 0) build_windows(false);
        PcgBufs<double> v{A_.p,      xf_lo_.p, xf_up_.p, pk_val_lo_.p, pk_val_up_.p, dinv_.p, inv_cm_.p,
                          inv_rm_.p, x_.p,     r_.p,     z_.p,         p_.p,         Ap_.p,   y_.p,
                          part_.p,   b_.p};
        if (sweep_mode_ == 2) launch_pcg<double>(v, true, 0);
        else {
            run_sweep<double>(v, true);
            run_sweep<double>(v, false);
        }
    }
    MPS_CUDA(cudaGetLastError());
    MPS_CUDA(cudaMemcpyAsync(z, z_.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, st_));
    MPS_CUDA(cudaStreamSynchronize(st_));
    check_err();
}

// ---- stages over a caller list (drop-in fine-grained functions) ----------------

template <int D>
void Engine<D>::run_stage(int stage, const int *nb, const int *cnt, int max_nb, double arg)
{
    int n = n_;
    bool needs_list = stage == MPS_STAGE_DENSITY || stage == MPS_STAGE_VISCOSITY || stage == MPS_STAGE_GRADIENT ||
                      stage == MPS_STAGE_NEIGHBOR_COUNT || stage == MPS_STAGE_SOLVE_PRESSURE ||
                      stage == MPS_STAGE_SURFACE_TENSION || stage == MPS_STAGE_SURFACE_TENSION_SL ||
                      (stage == MPS_STAGE_COLLISION && D == 3);
    bool needs_ref = stage == MPS_STAGE_VISCOSITY || stage == MPS_STAGE_GRADIENT ||
                     stage == MPS_STAGE_SOLVE_PRESSURE || stage == MPS_STAGE_SURFACE ||
                     stage == MPS_STAGE_SURFACE_BY_COUNT;
    if (needs_ref) require_ref();
    if (needs_list && (!nb || !cnt)) throw CudaError("stage needs a neighbour list", MPS_ERR_INVALID);
    if (structure_ && stage != MPS_STAGE_CLAMP && stage != MPS_STAGE_WALL && stage != MPS_STAGE_OUT_OF_BOUNDS &&
        stage != MPS_STAGE_SURFACE && stage != MPS_STAGE_SURFACE_BY_COUNT)
        unsort();
    if (needs_list) upload_list(nb, cnt, max_nb);
    int bl = nblk(n, TPB);
    if (n == 0) return;
    switch (stage) {
    case MPS_STAGE_DENSITY:
        launch(k_density<D, ListSource>, bl, TPB, 0, st_, list(), S(), k_, n, err_.p, 0, 0);
        break;
    case MPS_STAGE_VISCOSITY:
        launch(k_viscosity<D, ListSource>, bl, TPB, 0, st_, list(), S(), k_, n, 1);
        break;
    case MPS_STAGE_GRADIENT:
        if (k_.cmps != 2) launch(k_pmin<D, ListSource>, bl, TPB, 0, st_, list(), S(), n, pmin_.p);
        launch(k_gradient<D, ListSource>, bl, TPB, 0, st_, list(), S(), k_, n, k_.cmps != 2 ? pmin_.p : nullptr);
        break;
    case MPS_STAGE_NEIGHBOR_COUNT:
        launch(k_neighbor_count<D, ListSource>, bl, TPB, 0, st_, list(), S(), k_, n);
        break;
    case MPS_STAGE_COLLISION:
        if (D == 3) {
            launch(k_collision_list<D, ListSource>, bl, TPB, 0, st_, list(), S(), k_, n, vafter_.p);
        } else {
            sort();
            launch(k_collision_allpairs<D>, bl, TPB, 0, st_, cells(), S(), k_, n, vafter_.p);
        }
        launch(k_collision_apply<D>, bl, TPB, 0, st_, S(), k_, n, vafter_.p);
        break;
    case MPS_STAGE_SOLVE_PRESSURE: {
        // the block-colour solver needs the cell structure; the caller's
        // list must be the one that structure produces
        sort();
        launch(k_compare_list<D>, bl, TPB, 0, st_, cells(), S().id, n, lptr_.p, lidx_.p, err_.p);
        check_err();
        ppe(false);
        break;
    }
    case MPS_STAGE_SURFACE:
    case MPS_STAGE_SURFACE_BY_COUNT: {
        Consts k = k_;
        int by_count = stage == MPS_STAGE_SURFACE_BY_COUNT;
        if (by_count) k.count_thr = arg * n0_count_;
        else k.surf_thr = arg * n0_;
        launch(k_surface<D>, bl, TPB, 0, st_, S(), k, n, by_count);
        break;
    }
    case MPS_STAGE_SURFACE_TENSION:
    case MPS_STAGE_SURFACE_TENSION_SL: {
        // arg = C_LL or C_SL of the caller's particle system (operators.c:284, :326)
        Consts k = k_;
        double l0 = prm_.particle_distance;
        double c = (D == 3) ? arg / (prm_.density * l0 * l0 * l0) : arg / (prm_.density * l0 * l0);
        int which = stage == MPS_STAGE_SURFACE_TENSION ? 1 : 2;
        if (which == 1) k.st_ll = c;
        else {
            k.st_sl = c;
            k.st_sl_on = arg != 0.0;
        }
        launch(k_surface_tension<D, ListSource>, bl, TPB, 0, st_, list(), S(), k, n, which);
        break;
    }
    case MPS_STAGE_CLAMP:
        launch(k_clamp<D>, bl, TPB, 0, st_, S(), n);
        break;
    case MPS_STAGE_WALL:
        launch(k_correct<D>, bl, TPB, 0, st_, S(), k_, n, 0, 1, 0);
        break;
    case MPS_STAGE_OUT_OF_BOUNDS:
        launch(k_correct<D>, bl, TPB, 0, st_, S(), k_, n, 0, 0, 1);
        break;
    default:
        throw CudaError("unknown stage", MPS_ERR_INVALID);
    }
    MPS_CUDA(cudaGetLastError());
    check_err();
}

EngineBase *make_engine(const mps_params_t &p, int capacity)
{
    if (p.dim == 3) return new Engine<3>(p, capacity);
    if (p.dim == 2) return new Engine<2>(p, capacity);
    throw CudaError("dim must be 2 or 3", MPS_ERR_INVALID);
}

}  // namespace mps

// =============================================================================
// C ABI
// =============================================================================

struct mps_session {
    std::unique_ptr<mps::EngineBase> eng;
};

#define MPS_API_BODY(s, body)                                          \
    do {                                                               \
        if (!(s) || !(s)->eng) return MPS_ERR_INVALID;                 \
        try {                                                          \
            body;                                                      \
            return MPS_OK;                                             \
        } catch (const mps::CudaError &e) {                            \
            (s)->eng->last_error = e.what();                           \
            return e.code;                                             \
        } catch (const std::bad_alloc &) {                             \
            return MPS_ERR_OOM;                                        \
        } catch (const std::exception &e) {                            \
            (s)->eng->last_error = e.what();                           \
            return MPS_ERR_INVALID;                                    \
        }                                                              \
    } while (0)

extern "C" {

int mps_version(void) { return 10000; }

const char *mps_error_string(int code)
{
    switch (code) {
    case MPS_OK: return "ok";
    case MPS_ERR_INVALID: return "invalid argument or state";
    case MPS_ERR_CUDA: return "CUDA error";
    case MPS_ERR_OOM: return "out of device memory";
    case MPS_ERR_NEIGHBOR_OVERFLOW: return "neighbour count exceeded max_neighbors";
    case MPS_ERR_UNSUPPORTED: return "unsupported configuration";
    case MPS_ERR_NOT_CONVERGED: return "PPE solve did not converge";
    case MPS_ERR_NAN: return "non-finite value";
    default: return "unknown error";
    }
}

int mps_session_create(mps_session **out, const mps_params_t *params, int capacity)
{
    if (!out || !params) return MPS_ERR_INVALID;
    *out = nullptr;
    try {
        auto *s = new mps_session;
        s->eng.reset(mps::make_engine(*params, capacity));
        *out = s;
        return MPS_OK;
    } catch (const mps::CudaError &e) {
        std::fprintf(stderr, "mps_session_create: %s\n", e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        return MPS_ERR_OOM;
    }
}

int mps_session_destroy(mps_session *s)
{
    delete s;
    return MPS_OK;
}

int mps_update_params(mps_session *s, const mps_params_t *p)
{
    if (!p) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->update_params(*p));
}

int mps_set_precision(mps_session *s, int precision)
{
    if (precision != MPS_PREC_FP64 && precision != MPS_PREC_MIXED) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->set_precision(precision));
}

int mps_upload_particles(mps_session *s, const void *particles, int num)
{
    if (!particles && num) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->upload_aos(particles, num));
}

int mps_download_particles(mps_session *s, void *particles, int num)
{
    if (!particles && num) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->download_aos(particles, num));
}

int mps_upload_soa(mps_session *s, const double *pos, const double *vel, const int *type, int num)
{
    if ((!pos || !vel || !type) && num) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->upload_soa(pos, vel, type, num));
}

int mps_download_pressure(mps_session *s, double *pressure, int num)
{
    if (!pressure && num) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->download_pressure(pressure, num));
}

int mps_compute_initial_params(mps_session *s, double *n0, double *lambda, int *n0_count)
{
    MPS_API_BODY(s, s->eng->compute_initial_params(n0, lambda, n0_count));
}

int mps_set_initial_params(mps_session *s, double n0, double lambda, int n0_count)
{
    MPS_API_BODY(s, s->eng->set_initial_params(n0, lambda, n0_count));
}

int mps_neighbor_search(mps_session *s) { MPS_API_BODY(s, s->eng->neighbor_search()); }

int mps_step(mps_session *s, int nsteps)
{
    if (nsteps < 0) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->step(nsteps));
}

int mps_step_with_list(mps_session *s, const int *neighbors, const int *count, int max_nb)
{
    if (!neighbors || !count) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->step_with_list(neighbors, count, max_nb));
}

int mps_get_neighbor_list(mps_session *s, int *neighbors, int *count, int max_nb)
{
    MPS_API_BODY(s, s->eng->get_neighbor_list(neighbors, count, max_nb));
}

int mps_get_cell_index(mps_session *s, int *cell)
{
    if (!cell) return MPS_ERR_INVALID;
    MPS_API_BODY(s, s->eng->get_cell_index(cell));
}

int mps_get_cell_links(mps_session *s, int *head, int *next, int total_cells)
{
    MPS_API_BODY(s, s->eng->get_cell_links(head, next, total_cells));
}

int mps_get_ppe(mps_session *s, int *eq_idx, int *row_ptr, int *col_idx, double *val, double *b, int *n_eq,
                long long *nnz)
{
    MPS_API_BODY(s, s->eng->get_ppe(eq_idx, row_ptr, col_idx, val, b, n_eq, nnz));
}

int mps_get_ic0(mps_session *s, int *row_ptr, int *col, double *A, double *F, double *b, int *n_eq,
                long long *nnz)
{
    MPS_API_BODY(s, s->eng->get_ic0(row_ptr, col, A, F, b, n_eq, nnz));
}

int mps_get_cell_blocks(mps_session *s, int *cells, int *inv_off, double *inv, int *colour_rows, int *ncells,
                        long long *ninv)
{
    MPS_API_BODY(s, s->eng->get_cell_blocks(cells, inv_off, inv, colour_rows, ncells, ninv));
}

int mps_apply_preconditioner(mps_session *s, const double *r, double *z)
{
    MPS_API_BODY(s, s->eng->apply_preconditioner(r, z));
}

int mps_get_metrics(mps_session *s, mps_metrics_t *m)
{
    if (!m) return MPS_ERR_INVALID;
    MPS_API_BODY(s, *m = s->eng->met);
}

unsigned long long mps_launch_count(void) { return mps::launch_counter(); }

int mps_set_profiling(mps_session *s, int on) { MPS_API_BODY(s, s->eng->profiling = (on != 0)); }

int mps_reset_metrics(mps_session *s) { MPS_API_BODY(s, s->eng->met = mps_metrics_t{}); }

void *mps_get_stream(mps_session *s) { return (s && s->eng) ? (void *)s->eng->stream() : nullptr; }

const char *mps_last_error(mps_session *s)
{
    return (s && s->eng) ? s->eng->last_error.c_str() : "no session";
}

int mps_surface_tension_coeffs(const mps_params_t *params, double *c_ll, double *c_sl)
{
    if (!params || !c_ll || !c_sl) return MPS_ERR_INVALID;
    mps::surface_tension_coeffs(*params, c_ll, c_sl);
    return MPS_OK;
}

int mps_run_stage(mps_session *s, int stage, const int *neighbors, const int *count, int max_nb, double arg)
{
    MPS_API_BODY(s, s->eng->run_stage(stage, neighbors, count, max_nb, arg));
}

int mps_state_bytes(mps_session *s, size_t *bytes)
{
    if (!bytes) return MPS_ERR_INVALID;
    MPS_API_BODY(s, *bytes = s->eng->state_bytes());
}

int mps_state_save(mps_session *s, void *buf) { MPS_API_BODY(s, s->eng->state_save(buf)); }

int mps_state_load(mps_session *s, const void *buf) { MPS_API_BODY(s, s->eng->state_load(buf)); }

int mps_adjoint_pressure_seed(mps_session *s, const double *dLdP, int num)
{
    MPS_API_BODY(s, s->eng->adjoint_pressure_seed(dLdP, num));
}

int mps_adjoint_seed(mps_session *s, const double *lam_pos, const double *lam_vel)
{
    MPS_API_BODY(s, s->eng->adjoint_seed(lam_pos, lam_vel));
}

int mps_step_adjoint(mps_session *s) { MPS_API_BODY(s, s->eng->step_adjoint()); }

int mps_adjoint_get(mps_session *s, double *lam_pos, double *lam_vel, double *grad_gravity, double *grad_viscosity,
                    double *grad_drive)
{
    MPS_API_BODY(s, s->eng->adjoint_get(lam_pos, lam_vel, grad_gravity, grad_viscosity, grad_drive));
}

}  // extern "C"
