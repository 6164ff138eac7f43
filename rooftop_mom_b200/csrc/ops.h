// Linear operators on rooftop vectors, as the solvers see them.
#pragma once

#include <memory>

#include "internal.h"

namespace rtm {

// Per-right-hand-side skip flags: an operator skips the vectors whose flag is nonzero.
struct SkipFlags {
    const int* ptr = nullptr;  // device; flag of rhs r at ptr[r * stride]
    int stride = 1;
};

struct LinearOp {
    int64_t n = 0;
    int precision = RTM_FP64;
    virtual ~LinearOp() = default;
    // y = A x for nrhs vectors of length n in the operator's precision, both on the device.
    virtual int apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) = 0;
    // Makes room for nrhs vectors in one apply (outside of any stream capture).
    virtual int reserve(int nrhs) { (void)nrhs; return RTM_OK; }
    virtual double stored_bytes() const { return 0; }
    virtual double working_bytes() const { return 0; }
};

// Dense n x n complex FP64 matrix (column-major).
std::unique_ptr<LinearOp> make_dense_op(const double2* device_matrix, int64_t n, int* status);

struct DeviceGenerators;
// Block-Jacobi over blocks of bx x by faces, inverted on the device.
std::unique_ptr<LinearOp> make_block_jacobi(const DeviceGenerators& g, double size_x, double size_y, int bx, int by,
                                            int precision, cudaStream_t s, int* status);

// The device arrays of a block-Jacobi operator (make_block_jacobi), for batched applies: blocks, their
// packed size S, unknowns per block, rooftop indices [nblocks][S] and inverses [nblocks][S][S] (column-major).
struct BjEntry {
    int nblocks = 0, S = 0;
    const int* counts = nullptr;
    const int64_t* index = nullptr;
    const void* inv = nullptr;
};
// False when op is not a block-Jacobi operator.
bool block_jacobi_entry(const LinearOp* op, BjEntry* out);
// y = M_k x for count block-Jacobi operators at once (one launch; entry k's vectors start at k * stride),
// entries a device table; max_blocks the most blocks of an entry.
int apply_block_jacobi_batch(const BjEntry* entries, int count, int max_blocks, int S, int precision, const void* x,
                             void* y, int64_t stride, cudaStream_t s, SkipFlags skip);

// Precision conversion of complex vectors on the device.
void convert_to_fp32(const double2* in, float2* out, int64_t n, cudaStream_t s);
void convert_to_fp64(const float2* in, double2* out, int64_t n, cudaStream_t s);

}  // namespace rtm
