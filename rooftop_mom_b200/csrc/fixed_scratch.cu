// The fixed scratch array of rtm_operator_apply_fixed_scratch: a working grid in a file-scope device
// array, for callers that must not allocate device memory per call. Such callers are the ones whose
// device memory is owned by someone else: a MATLAB MEX gateway whose gpuArray memory pool already
// holds the device, or a serving process whose admission ledger has handed out all of HBM and cannot
// let a call take more behind its back.
//
// The array sits alone in this file, so it belongs to a module of its own that no product kernel
// references (the kernels receive its address as an argument). Under CUDA's default lazy module
// loading the 32 MiB are therefore taken on a device only when the first fixed-scratch call looks the
// array up there, and then held until the process exits; with CUDA_MODULE_LOADING=EAGER every context
// of the process takes them at creation. They are outside the budget ledger (rtm_budget_*).
#include "internal.h"

namespace rtm {

constexpr size_t kFixedScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) unsigned char g_fixed_scratch[kFixedScratchBytes];

// The array's device address on the current device. Looked up on every call: after the module is
// loaded this is a table lookup, and a context torn down and re-created on the same device
// (cudaDeviceReset) is picked up instead of a stale cached pointer. The first call on a device loads
// the module, so make it before any stream capture.
int fixed_scratch_address(void** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_fixed_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fixed_scratch)");
    *out = p;
    return RTM_OK;
}

size_t fixed_scratch_bytes() { return kFixedScratchBytes; }

}  // namespace rtm
