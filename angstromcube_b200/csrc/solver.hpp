// tfQMR solver of (H - E S) X = B on the device (B: unit blocks on the diagonal).
#pragma once

#include "device.cuh"
#include "../../include/a43g.h"

namespace a43g {

// device vectors of one precision for the tfQMR recurrences
struct TfqmrVectors {
    size_t elem = 0;             // bytes per real
    size_t n = 0;                // reals per vector (nnzb * 8192)
    DeviceBuffer X, W, U1, U2, V, D, AU1, AU2, Rt;
    bool alloc(size_t nreals, size_t elem_bytes);
    void release();
};

struct SolverWorkspace {
    TfqmrVectors v64, v32;
    DeviceBuffer X64, R64, AX64;     // refinement vectors (FP64)
    DeviceBuffer colstate;           // per-column scalars (double), see solver.cu
    DeviceBuffer counters;           // int32 [4]
    DeviceBuffer colnorm;            // double [nCols*64]
    int32_t *host_counters = nullptr; // pinned
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~SolverWorkspace();
};

int solve(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
          void *X, double *rho, a43g_solve_stats_t *stats, cudaStream_t st);

int solve_batched(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
                  int32_t n, double const *energies, double const *kpoints, double dVol,
                  double *rho, a43g_solve_stats_t *stats, cudaStream_t st);

} // namespace a43g
