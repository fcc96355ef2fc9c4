// engine.cuh -- host-side engine of one device-resident particle system.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mps_b200.h"
#include "device.cuh"
#include "k_ppe.cuh"

namespace mps {

struct CudaError : std::runtime_error {
    int code;
    CudaError(const std::string &m, int c) : std::runtime_error(m), code(c) {}
};

#define MPS_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            throw ::mps::CudaError(std::string(#call) + ": " + cudaGetErrorString(e_),         \
                                   e_ == cudaErrorMemoryAllocation ? MPS_ERR_OOM : MPS_ERR_CUDA); \
    } while (0)

// Growable device array; contents are not preserved on growth.
template <class T>
struct DevArray {
    T *p = nullptr;
    size_t n = 0;
    DevArray() = default;
    DevArray(const DevArray &) = delete;
    DevArray &operator=(const DevArray &) = delete;
    ~DevArray() { if (p) cudaFree(p); }
    void reserve(size_t m)
    {
        if (m <= n) return;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        size_t want = m + m / 8 + 16;
        MPS_CUDA(cudaMalloc((void **)&p, want * sizeof(T)));
        n = want;
    }
    operator T *() const { return p; }
};

class EngineBase {
public:
    virtual ~EngineBase() = default;
    virtual int dim() const = 0;
    virtual void update_params(const mps_params_t &p) = 0;
    virtual void upload_aos(const void *aos, int num) = 0;
    virtual void download_aos(void *aos, int num) = 0;
    virtual void upload_soa(const double *pos, const double *vel, const int *type, int num) = 0;
    virtual void download_pressure(double *p, int num) = 0;
    virtual void compute_initial_params(double *n0, double *lambda, int *n0_count) = 0;
    virtual void set_initial_params(double n0, double lambda, int n0_count) = 0;
    virtual void neighbor_search() = 0;
    virtual void step(int nsteps) = 0;
    virtual void step_with_list(const int *nb, const int *cnt, int max_nb) = 0;
    virtual void get_neighbor_list(int *nb, int *cnt, int max_nb) = 0;
    virtual void get_cell_index(int *cell) = 0;
    virtual void get_cell_links(int *head, int *next, int total) = 0;
    virtual void set_precision(int precision) = 0;
    virtual void get_ppe(int *eq_idx, int *row_ptr, int *col, double *val, double *b, int *n_eq,
                         long long *nnz) = 0;
    virtual void run_stage(int stage, const int *nb, const int *cnt, int max_nb, double arg) = 0;
    // the last step's PPE and IC(0) preconditioner in the solver's numbering
    virtual void get_ic0(int *row_ptr, int *col, double *A, double *F, double *b, int *n_eq, long long *nnz) = 0;
    virtual void get_cell_blocks(int *cells, int *inv_off, double *inv, int *colour_rows, int *ncells,
                                 long long *ninv) = 0;
    virtual void apply_preconditioner(const double *r, double *z) = 0;
    virtual cudaStream_t stream() const = 0;
    // differentiation form: checkpoints and the adjoint of one step
    virtual size_t state_bytes() const = 0;
    virtual void state_save(void *dst) = 0;
    virtual void state_load(const void *src) = 0;
    virtual void adjoint_seed(const double *lam_pos, const double *lam_vel) = 0;
    virtual void adjoint_pressure_seed(const double *dLdP, int num) = 0;
    virtual void step_adjoint() = 0;
    virtual void adjoint_get(double *lam_pos, double *lam_vel, double *grad_gravity, double *grad_viscosity,
                             double *grad_drive) = 0;
    bool profiling = false;
    mps_metrics_t met{};
    std::string last_error;
};

EngineBase *make_engine(const mps_params_t &p, int capacity);

}  // namespace mps
