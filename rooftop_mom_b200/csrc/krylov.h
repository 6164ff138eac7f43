// Iterative solvers on the device (krylov.cu, mixed.cu).
#pragma once

#include <atomic>
#include <vector>

#include "ops.h"

namespace rtm {

struct SolveConfig {
    int method = RTM_METHOD_CG;
    double tolerance = 1e-6;
    const double* tolerances = nullptr;  // host, one per right-hand side: overrides `tolerance` when set
    int max_iterations = 1000;
    int restart = 50;
    int check_every = 0;
    double inner_tolerance = 1e-4;  // mixed: the tightest relative residual an inner FP32 solve aims at
    int max_refinements = 20;
    int right_preconditioned = 0;  // GMRES: 0 left (the reference's form), 1 right (flexible)
    const std::atomic<int>* cancel = nullptr;  // nonzero: stop at the next host check (unconverged result)
};

struct SolveResult {
    std::vector<double> history;  // [rhs][hist_stride], NaN after the last iteration
    int hist_stride = 0;
    std::vector<rtm_solve_stats> stats;
    int matvecs = 0;
};

// Solves A x = b for nrhs right-hand sides in the operator's precision (vectors on the device).
int solve(LinearOp* A, LinearOp* M, const SolveConfig& cfg, const void* b, const void* x0, void* x, int64_t n, int nrhs,
          SolveResult& res, cudaStream_t s);

// FP64 outer iterative refinement around FP32 inner flexible GMRES (A64 FP64, A32 / M32 FP32).
int solve_mixed(LinearOp* A64, LinearOp* A32, LinearOp* M32, const SolveConfig& cfg, const void* b, const void* x0,
                void* x, int64_t n, int nrhs, SolveResult& res, cudaStream_t s);

}  // namespace rtm
