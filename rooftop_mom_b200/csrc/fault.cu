// The fault word: kernels whose waits are bounded (the pipelined x-mix of grid_fast.cu) record
// RTM_ERR_TIMEOUT here when a wait runs out, instead of hanging; the host reads it after a
// synchronisation. A file-scope device variable, so that no call allocates device memory for it (the
// fixed-scratch product, which must not allocate, reaches the same kernels).
#include "internal.h"

namespace rtm {

static __device__ int g_fault_word;

int device_fault_word(int** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_fault_word);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fault_word)");
    *out = static_cast<int*>(p);
    return RTM_OK;
}

int device_fault_check(cudaStream_t s) {
    int* w = nullptr;
    RTM_TRY(device_fault_word(&w));
    int v = 0;
    RTM_CUDA(cudaMemcpyAsync(&v, w, sizeof(int), cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    if (v == 0) return RTM_OK;
    RTM_CUDA(cudaMemsetAsync(w, 0, sizeof(int), s));
    RTM_CUDA(cudaStreamSynchronize(s));
    return fail(RTM_ERR_TIMEOUT, "a bounded wait of a product kernel ran out on the device; the result is invalid");
}

}  // namespace rtm
