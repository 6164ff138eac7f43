// Internal declarations shared by the CUDA and C++ sources of librtm.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/rtm.h"

namespace rtm {

// ---------------------------------------------------------------------------------------------
// Errors: every entry point returns a status and records a thread-local message.
void set_error(const std::string& msg);
int fail(int status, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);
inline int check_cuda(cudaError_t e, const char* what) { return e == cudaSuccess ? RTM_OK : cuda_fail(e, what); }

#define RTM_CUDA(call)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return ::rtm::cuda_fail(e_, #call); \
    } while (0)

#define RTM_TRY(call)                   \
    do {                                \
        int s_ = (call);                \
        if (s_ != RTM_OK) return s_;    \
    } while (0)

extern int64_t g_launches;  // launches of this library's kernels (incremented by the launchers)
inline void count_launch(int n = 1) { __atomic_fetch_add(&g_launches, (int64_t)n, __ATOMIC_RELAXED); }

// One-time set-up per device, such as kernel attributes, which belong to the device's context. Host
// threads that reach the same device's set-up together may both run it, so the set-up must be
// idempotent; the flags are atomic, so that race is well defined. The flag is set only when the
// set-up succeeds. Ordinals above 63 run the set-up on every call.
struct DeviceOnce {
    std::atomic<bool> done[64] = {};
    template <typename F> int operator()(F&& setup) {
        int dev = 0;
        RTM_CUDA(cudaGetDevice(&dev));
        const bool tracked = dev >= 0 && dev < 64;
        if (tracked && done[dev].load(std::memory_order_acquire)) return RTM_OK;
        RTM_TRY(setup());
        if (tracked) done[dev].store(true, std::memory_order_release);
        return RTM_OK;
    }
};

// ---------------------------------------------------------------------------------------------
// Budget ledger of device bytes (Budget.m). Thread-safe.
int budget_require(double bytes, const char* what);
// A byte count as the reference's messages write it (formatBytes.m): "512 B", "1.5 kB", "3.0 GB".
std::string format_bytes(double bytes);
void budget_hold(double bytes);
void budget_release(double bytes);
// Returns the cached idle blocks of the current device to the driver.
void release_cached_blocks();

// Device buffer owned by a handle; its bytes are held in the budget while it lives.
// Blocks come from a per-device cache of freed blocks (no cudaFree, whose implicit device-wide
// synchronisation would stall concurrent solves); the cache is emptied when cudaMalloc fails.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;     // requested (held in the budget)
    size_t capacity = 0;  // size of the cached block
    int device = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    ~DeviceBuffer() { reset(); }
    int alloc(size_t n);
    void reset();
    template <typename T> T* as() const { return reinterpret_cast<T*>(ptr); }
    // Moves another buffer's block into this one.
    void take(DeviceBuffer& o) {
        reset();
        ptr = o.ptr; bytes = o.bytes; capacity = o.capacity; device = o.device;
        o.ptr = nullptr; o.bytes = 0; o.capacity = 0;
    }
};

// Synchronises a stream when it leaves scope. Declared after a function's device buffers, it runs
// before their blocks return to the cache, on every path out of the function.
struct StreamSyncGuard {
    cudaStream_t s;
    explicit StreamSyncGuard(cudaStream_t st) : s(st) {}
    ~StreamSyncGuard() { cudaStreamSynchronize(s); }
};

// ---------------------------------------------------------------------------------------------
// FFT plans: a length n factorised into radices; twiddle tables exp(-2 pi i m / n), m < n, in
// FP64 and FP32, computed on the host in long double and kept on the device for the life of the
// process (one table per length and device).
constexpr int kMaxStages = 20;
constexpr int kMaxGenericRadix = 64;  // largest prime factor this build transforms

// A length whose factorisation needs a prime above kMaxGenericRadix runs as a Bluestein (chirp-z)
// convolution: m is then the power of two >= 2n - 1 that a line buffer must hold, the radices are those
// of m, and the plan points to the chirp, the convolution kernel's spectrum and the roots of length m.
// Otherwise m == n and the pointers are null.
struct FftPlan {
    int n;
    int nstages;
    int radix[kMaxStages];
    int m;
    const double2* chirp64;  // exp(-i pi (j^2 mod 2n) / n), j < n
    const float2* chirp32;
    const double2* kern64;   // DFT_m of exp(+i pi d^2 / n) wrapped to length m, divided by m
    const float2* kern32;
    const double2* twm64;    // exp(-2 pi i k / m), k < m
    const float2* twm32;
};

struct FftTables {
    FftPlan plan;
    const double2* tw64;   // n entries
    const float2* tw32;
    const double2* mod64;  // exp(-i pi d / n), d < n (the odd-subband modulation)
    const float2* mod32;
};

// Returns the cached tables of length n on the current device (a Bluestein plan when n has a prime
// factor above kMaxGenericRadix).
int fft_tables(int n, const FftTables** out);

// Shift-phase factors of generateShiftPhases.m: u(m) = 1 - exp(i pi (2m + parity) / n).
int shift_factors(int n, int parity, const double2** out64, const float2** out32);

template <typename T> struct Cx;
template <> struct Cx<double> { using T2 = double2; };
template <> struct Cx<float> { using T2 = float2; };

// Host FP64 helpers used by the assembler set-up.
void gauss_legendre(int order, double a, double b, std::vector<double>& points, std::vector<double>& weights);
void power_moments(double size_x, double size_y, int power, double out[7][4]);
void extracted_moments(double size_x, double size_y, double k, double out[7][4]);

int fast_fft_size(int count);

// The device's fault word, which kernels with bounded waits set to RTM_ERR_TIMEOUT when a wait runs
// out (a device variable: looking it up allocates nothing; the first lookup on a device loads its
// module, so it is made outside any stream capture), and its check: reads and clears the word after
// synchronising the stream, returning RTM_ERR_TIMEOUT if it was set.
int device_fault_word(int** out);
int device_fault_check(cudaStream_t s);

}  // namespace rtm
