// Plate batches (batch.h): the batch operator and the zeroing of the entries' tails.
#include <algorithm>

#include "batch.h"

namespace rtm {
namespace {

template <typename T2>
__global__ void k_zero_tails(T2* __restrict__ y, int64_t stride, const int64_t* __restrict__ counts, const int* skip,
                             int skip_stride) {
    const int k = blockIdx.y;
    if (skip && skip[(int64_t)k * skip_stride]) return;
    T2* yk = y + (int64_t)k * stride;
    for (int64_t i = counts[k] + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < stride;
         i += (int64_t)gridDim.x * blockDim.x)
        yk[i] = T2{};
}

}  // namespace

int zero_tails(void* y, int precision, int64_t stride, const int64_t* counts_device, int count, int64_t max_tail,
               cudaStream_t s, SkipFlags skip) {
    if (max_tail <= 0) return RTM_OK;
    // about eight elements a thread: a CTA or a few per entry
    const dim3 grid((unsigned)std::min<int64_t>(64, (max_tail + 2047) / 2048), count);
    if (precision == RTM_FP64)
        k_zero_tails<double2><<<grid, 256, 0, s>>>(static_cast<double2*>(y), stride, counts_device, skip.ptr,
                                                   skip.stride);
    else
        k_zero_tails<float2><<<grid, 256, 0, s>>>(static_cast<float2*>(y), stride, counts_device, skip.ptr,
                                                  skip.stride);
    count_launch();
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

int BatchOp::reserve(int nrhs) {
    if (nrhs != (int)ops.size()) return fail(RTM_ERR_ARG, "a plate batch applies to one vector per entry");
    RTM_TRY(device_fault_word(&fault));
    if (fused) {
        const size_t need = plates[0]->work_bytes_per_rhs() * ops.size();
        if (work.bytes < need) RTM_TRY(work.alloc(need));
        // the entries' own reserve sets up the kernels' attributes and their fault word
        for (LinearOp* op : ops) RTM_TRY(op->reserve(1));
        return RTM_OK;
    }
    for (LinearOp* op : ops) RTM_TRY(op->reserve(1));
    return RTM_OK;
}

int BatchOp::apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) {
    if (nrhs != (int)ops.size()) return fail(RTM_ERR_ARG, "a plate batch applies to one vector per entry");
    if (fused) {
        if (work.bytes < plates[0]->work_bytes_per_rhs() * ops.size())
            return fail(RTM_ERR_ARG, "the plate batch was not reserved");
        RTM_TRY(apply_plate_batch(plates, descs.ptr, stride, work.ptr, fault, x, y, s, skip));
    } else if (fused_bj) {
        RTM_TRY(apply_block_jacobi_batch(descs.as<BjEntry>(), (int)ops.size(), bj_blocks, bj_S, precision, x, y, stride,
                                         s, skip));
    } else {
        const size_t elem = precision == RTM_FP64 ? sizeof(double2) : sizeof(float2);
        for (size_t k = 0; k < ops.size(); ++k) {
            const SkipFlags sk{skip.ptr ? skip.ptr + (int64_t)k * skip.stride : nullptr, skip.stride};
            RTM_TRY(ops[k]->apply(static_cast<const char*>(x) + k * stride * elem,
                                  static_cast<char*>(y) + k * stride * elem, 1, s, sk));
        }
    }
    return zero_tails(y, precision, stride, tails.as<int64_t>(), (int)ops.size(), max_tail, s, skip);
}

std::unique_ptr<BatchOp> make_batch(const std::vector<LinearOp*>& ops, int64_t stride, bool fuse, cudaStream_t s,
                                    int* status) {
    *status = RTM_OK;
    if (ops.empty() || ops.size() > 65535) {
        *status = fail(ops.empty() ? RTM_ERR_ARG : RTM_ERR_SIZE, "a plate batch holds 1 to 65535 entries");
        return nullptr;
    }
    auto b = std::make_unique<BatchOp>();
    b->precision = ops[0]->precision;
    b->stride = stride;
    b->n = stride;
    b->ops = ops;
    for (LinearOp* op : ops) {
        if (op->precision != b->precision) {
            *status = fail(RTM_ERR_ARG, "the entries of a plate batch have one precision");
            return nullptr;
        }
        if (op->n > stride) {
            *status = fail(RTM_ERR_SIZE, "an entry of a plate batch is longer than the batch's stride");
            return nullptr;
        }
        b->counts.push_back(op->n);
        b->max_tail = std::max(b->max_tail, stride - op->n);
    }
    if ((*status = b->tails.alloc(sizeof(int64_t) * ops.size())) != RTM_OK) return nullptr;
    if ((*status = check_cuda(cudaMemcpyAsync(b->tails.ptr, b->counts.data(), b->tails.bytes, cudaMemcpyHostToDevice, s),
                              "cudaMemcpyAsync")) != RTM_OK)
        return nullptr;
    if (fuse) {
        const auto* first = dynamic_cast<const GridApplicator*>(ops[0]);
        bool ok = first != nullptr;
        for (LinearOp* op : ops) {
            const auto* g = dynamic_cast<const GridApplicator*>(op);
            ok = ok && g && batchable(*g) && g->P == first->P && g->Q == first->Q;
            if (ok) b->plates.push_back(g);
        }
        if (ok) {
            if ((*status = plate_descs(b->plates, b->descs, s)) != RTM_OK) return nullptr;
            b->fused = true;
        } else {
            b->plates.clear();
        }
        std::vector<BjEntry> bj(ops.size());
        bool all_bj = !b->fused;
        for (size_t k = 0; k < ops.size() && all_bj; ++k)
            all_bj = block_jacobi_entry(ops[k], &bj[k]) && bj[k].S == bj[0].S;
        if (all_bj) {
            for (const BjEntry& e : bj) b->bj_blocks = std::max(b->bj_blocks, e.nblocks);
            b->bj_S = bj[0].S;
            if ((*status = b->descs.alloc(sizeof(BjEntry) * bj.size())) != RTM_OK) return nullptr;
            if ((*status = check_cuda(cudaMemcpyAsync(b->descs.ptr, bj.data(), b->descs.bytes, cudaMemcpyHostToDevice, s),
                                      "cudaMemcpyAsync")) != RTM_OK)
                return nullptr;
            b->fused_bj = true;
        }
    }
    if ((*status = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize")) != RTM_OK) return nullptr;
    return b;
}

}  // namespace rtm
