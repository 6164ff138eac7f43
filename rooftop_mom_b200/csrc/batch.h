// Plate batches: several plates of uneven size, one right-hand side each, solved together.
//
// The vectors of a batch hold `count` entries of `stride` elements (the largest plate's rooftops); entry k
// keeps its plate's n_k rooftops first and zeros after them. A batch operator applies every entry's own
// operator: split products that share their transform grid and precision on the power-of-two path run as
// one launch of each of their three kernels for the whole batch (grid_fast.cu reads each right-hand side's
// plate from a descriptor table), block-Jacobi preconditioners of one packed block size as one launch too;
// other operators (the circulant preconditioners among them) run one after another on their entries.
// Every apply zeroes the entries' tails, so the Krylov solvers run on the batch unchanged: the padding adds
// zeros to every sum.
#pragma once

#include <memory>
#include <vector>

#include "grid.h"

namespace rtm {

struct BatchOp : LinearOp {
    std::vector<LinearOp*> ops;          // per entry (borrowed; the handles outlive the batch)
    std::vector<int64_t> counts;         // per entry: unknowns
    int64_t max_tail = 0;                // stride minus the fewest unknowns of an entry
    int64_t stride = 0;                  // elements of an entry
    bool fused = false;                  // one launch per kernel for the whole batch
    std::vector<const GridApplicator*> plates;  // fused products: the entries' products
    bool fused_bj = false;               // fused block-Jacobi preconditioners
    int bj_blocks = 0, bj_S = 0;         // fused block-Jacobi: the most blocks of an entry, their packed size
    DeviceBuffer descs, tails, work;     // fused: plate or block-Jacobi table, per-entry unknowns (device), W
    int* fault = nullptr;

    int apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) override;
    int reserve(int nrhs) override;
    double working_bytes() const override { return (double)work.bytes; }
};

// A batch over the given per-entry operators (all of one precision, each of n_k <= stride unknowns).
// fuse: join split products of one transform grid into single launches when they allow it.
std::unique_ptr<BatchOp> make_batch(const std::vector<LinearOp*>& ops, int64_t stride, bool fuse, cudaStream_t s,
                                    int* status);

// Zeroes elements [counts[k], stride) of entry k of y (k < count, where the skip flag is zero); max_tail, the
// longest tail, sizes the launch.
int zero_tails(void* y, int precision, int64_t stride, const int64_t* counts_device, int count, int64_t max_tail,
               cudaStream_t s, SkipFlags skip);

}  // namespace rtm
