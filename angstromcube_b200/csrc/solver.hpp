// tfQMR solver of (H - E S) X = B on the device (B: unit blocks on the diagonal).
#pragma once

#include "device.cuh"
#include "precond.hpp"
#include "../../include/a43g.h"

#include <memory>

namespace a43g {

// device vectors of one precision for the tfQMR recurrences
struct TfqmrVectors {
    size_t elem = 0;             // bytes per real
    size_t n = 0;                // reals per vector (nnzb * 8192)
    DeviceBuffer X, W, U1, U2, V, D, AU1, AU2;
    bool alloc(size_t nreals, size_t elem_bytes, bool with_x);
    void release();
};

struct SolverWorkspace {
    TfqmrVectors v64, v32;
    DeviceBuffer X64, AX64;          // FP64 solution, FP64 operator scratch of the FP32 recurrences
    DeviceBuffer state;              // per-column and per-source scalars, control block (solver.cu)
    DeviceBuffer part, tickets;      // fixed-order column reductions
    DeviceBuffer trace_sums;         // |X - Xref|^2 and |Xref|^2 of a traced solve
    BlockPreconditioner pc;          // cube-diagonal preconditioner (A43G_SOLVE_PRECONDITION)
    bool use_pc = false;
    DeviceBuffer PT64, PT32;         // M^-1 x ahead of the operator
    void *host_ctl = nullptr;        // pinned copy of the control block
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~SolverWorkspace();
};

// per-source results of a solve (batches report them per pair)
struct SourceStats {
    uint32_t live_sources = 0;       // sources beyond this are padding of a batch, retired at the start
    std::vector<int> iterations, updates, fallback;
    std::vector<double> residual;
};

// error of the solution against a given FP64 solution, sampled while the solve runs (the
// current solution: the FP64 solution plus the FP32 correction not yet added to it)
struct SolveTrace {
    double const *Xref = nullptr;    // device FP64 [nnzb][2][64][64]
    int every = 10;                  // iterations between samples
    std::vector<double> rows;        // per sample: iteration, |X - Xref| / |Xref|, active sources
};

// the batch plan and workspace of solve_batched, kept between calls
struct BatchCache {
    GreenPlan host;
    std::unique_ptr<DevicePlan> dev;
    std::unique_ptr<SolverWorkspace> ws;
    uint32_t npairs = 0;
};

// peak device bytes of the solver vectors of one solve of this plan in the given precision
size_t solve_bytes(DevicePlan const &dp, int precision, bool precondition = false);

int solve(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
          void *X, double *rho, a43g_solve_stats_t *stats, cudaStream_t st, SourceStats *per_source = nullptr,
          SolveTrace *trace = nullptr);

int solve_batched(GreenPlan &hp, DevicePlan &dp, BatchCache &bc, a43g_solve_options_t const &opt,
                  int32_t n, double const *energies, double const *kpoints, double dVol,
                  double *rho, a43g_solve_stats_t *stats, cudaStream_t st);

} // namespace a43g
