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
    int inner_max_iterations = 0;  // mixed: iterations one inner FP32 solve may take (0: the remaining budget)
    int fallback_fp64 = 0;         // mixed: finish in FP64 when a refinement step does not halve the residual
    int gram_schmidt_passes = 2;   // GMRES: classical Gram-Schmidt passes per Arnoldi step (2: CGS2, or 1)
    int inner_gram_schmidt_passes = 1;  // mixed: the passes of the FP32 inner solves
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

// FP64 outer iterative refinement around FP32 inner flexible GMRES (A64 FP64, A32 / M32 FP32). With
// cfg.fallback_fp64, a refinement step that does not halve some right-hand side's FP64 residual (the FP32
// inner solve diverged or stalled) ends the refinement, and the solve finishes in FP64 (A64 and M64, which
// may be null) from the current iterate.
int solve_mixed(LinearOp* A64, LinearOp* A32, LinearOp* M32, const SolveConfig& cfg, const void* b, const void* x0,
                void* x, int64_t n, int nrhs, SolveResult& res, cudaStream_t s, LinearOp* M64 = nullptr);

}  // namespace rtm
