// Autotuner of the split product (rtm_tune_product): for a face grid and precision it measures every
// candidate transform grid and kernel schedule and keeps the fastest, per device, for the products built
// afterwards (build_product reads the choice through tuned_choice).
//
// Candidates along each direction with more than one face: the reference's transform size, the smallest
// 7-smooth length >= the face count (generateFastFFTSize.m:11-15), and the smallest power of two >= the
// face count when it differs and the power-of-two kernels take it. Any length >= the face count gives the
// same product (the period of the subband embedding then holds the whole two-sided generator), so the
// choice changes rounding only. On a power-of-two grid the schedules of grid_fast.cu are swept too: the
// CTAs per SM of the y passes and the form of the x-mix.
//
// Each configuration is timed on the device over a few applies of a product built from zero generators
// (the timing does not depend on the values), each apply after a write of a buffer larger than L2 when
// RTM_TUNE_FLUSH_L2 is set, as in a solve whose other kernels evict the product's spectra between
// products; the median of the applies is the configuration's time.
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "grid.h"
#include "handles.h"

namespace rtm {
namespace {

struct TuneKey {
    int device, precision, count_x, count_y;
    bool operator<(const TuneKey& o) const {
        return std::tie(device, precision, count_x, count_y) < std::tie(o.device, o.precision, o.count_x, o.count_y);
    }
};

struct TuneChoice {
    int P = 0, Q = 0;
    FastSchedule sched;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tuned;

int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Device time of one apply of a product: the median over `reps` applies after two warm-up applies.
int time_product(GridApplicator& op, int nrhs, bool flush, DeviceBuffer& scratch, cudaStream_t s, double* seconds) {
    const size_t elem = op.precision == RTM_FP64 ? sizeof(double2) : sizeof(float2);
    DeviceBuffer x, y;
    RTM_TRY(x.alloc((size_t)op.n * nrhs * elem));
    RTM_TRY(y.alloc((size_t)op.n * nrhs * elem));
    RTM_CUDA(cudaMemsetAsync(x.ptr, 0, x.bytes, s));
    RTM_TRY(op.reserve(nrhs));
    for (int w = 0; w < 2; ++w) RTM_TRY(op.apply(x.ptr, y.ptr, nrhs, s, SkipFlags{}));
    constexpr int reps = 5;
    std::vector<cudaEvent_t> ev(2 * reps, nullptr);
    for (auto& e : ev) RTM_CUDA(cudaEventCreate(&e));
    int st = RTM_OK;
    for (int r = 0; r < reps && st == RTM_OK; ++r) {
        if (flush) st = check_cuda(cudaMemsetAsync(scratch.ptr, r & 0xff, scratch.bytes, s), "cudaMemsetAsync");
        if (st == RTM_OK) st = check_cuda(cudaEventRecord(ev[2 * r], s), "cudaEventRecord");
        if (st == RTM_OK) st = op.apply(x.ptr, y.ptr, nrhs, s, SkipFlags{});
        if (st == RTM_OK) st = check_cuda(cudaEventRecord(ev[2 * r + 1], s), "cudaEventRecord");
    }
    if (st == RTM_OK) st = check_cuda(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    std::vector<double> t;
    for (int r = 0; r < reps && st == RTM_OK; ++r) {
        float ms = 0;
        st = check_cuda(cudaEventElapsedTime(&ms, ev[2 * r], ev[2 * r + 1]), "cudaEventElapsedTime");
        t.push_back(ms * 1e-3);
    }
    for (auto& e : ev) cudaEventDestroy(e);
    RTM_TRY(st);
    std::sort(t.begin(), t.end());
    *seconds = t[t.size() / 2];
    return RTM_OK;
}

}  // namespace

bool tuned_choice(int count_x, int count_y, int precision, int* P, int* Q, FastSchedule* sched) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tuned.find({dev, precision, count_x, count_y});
    if (it == g_tuned.end()) return false;
    *P = it->second.P;
    *Q = it->second.Q;
    *sched = it->second.sched;
    return true;
}

void register_choice(int count_x, int count_y, int precision, int P, int Q) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    TuneChoice c;
    c.P = P;
    c.Q = Q;
    c.sched = default_fast_schedule(P, Q, precision == RTM_FP64);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[{dev, precision, count_x, count_y}] = c;
}

}  // namespace rtm

using namespace rtm;

extern "C" {

int rtm_tune_product(int count_x, int count_y, int precision, int nrhs, int flags, rtm_tune_result* out) {
    if (!out) return fail(RTM_ERR_ARG, "null output");
    if (count_x < 2 || count_y < 2) return fail(RTM_ERR_ARG, "the autotuner takes plates of at least 2 x 2 faces");
    if (precision != RTM_FP64 && precision != RTM_FP32) return fail(RTM_ERR_ARG, "unknown precision");
    if (nrhs < 1 || nrhs > 65535) return fail(nrhs < 1 ? RTM_ERR_ARG : RTM_ERR_SIZE, "nrhs must lie in 1..65535");
    int dev = 0;
    RTM_CUDA(cudaGetDevice(&dev));
    const bool fp64 = precision == RTM_FP64;
    std::vector<int> Ps{fast_fft_size(count_x)}, Qs{fast_fft_size(count_y)};
    if (!(flags & RTM_TUNE_REFERENCE_SIZES)) {
        if (next_pow2(count_x) != Ps[0]) Ps.push_back(next_pow2(count_x));
        if (next_pow2(count_y) != Qs[0]) Qs.push_back(next_pow2(count_y));
    }
    cudaStream_t s = nullptr;
    RTM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } sg{s};
    DeviceGenerators g;
    g.count_x = count_x;
    g.count_y = count_y;
    g.content = RTM_BOTH;
    DeviceBuffer scratch;
    {
        const size_t gx = (size_t)(count_x - 1) * count_y, gy = (size_t)count_x * (count_y - 1),
                     ge = (size_t)count_x * count_y;
        RTM_TRY(g.xx.alloc(gx * sizeof(double2)));
        RTM_TRY(g.yy.alloc(gy * sizeof(double2)));
        RTM_TRY(g.e.alloc(ge * sizeof(double2)));
        RTM_CUDA(cudaMemsetAsync(g.xx.ptr, 0, g.xx.bytes, s));
        RTM_CUDA(cudaMemsetAsync(g.yy.ptr, 0, g.yy.bytes, s));
        RTM_CUDA(cudaMemsetAsync(g.e.ptr, 0, g.e.bytes, s));
        if (flags & RTM_TUNE_FLUSH_L2) RTM_TRY(scratch.alloc(size_t(256) << 20));
    }
    const double h = 1.0;  // the face size does not change the work
    double best = 0, ref = 0;
    TuneChoice choice;
    int measured = 0;
    for (int P : Ps)
        for (int Q : Qs) {
            std::vector<FastSchedule> scheds;
            if (fast_split_eligible(P, Q, fp64)) {
                const int ymax = fp64 ? 3 : 2;
                for (int yb = 1; yb <= ymax; ++yb)
                    for (int xk : {kMixDirect1, kMixDirect2, kMixDirect3, kMixPipelined}) {
                        if (xk == kMixDirect3 && !fp64) continue;
                        FastSchedule f;
                        f.y_blocks = yb;
                        f.x_kind = xk;
                        scheds.push_back(f);
                    }
            } else {
                scheds.push_back(default_fast_schedule(P, Q, fp64));  // unused off the power-of-two path
            }
            for (const FastSchedule& f : scheds) {
                GridApplicator op;
                RTM_TRY(build_product(g, h, h, RTM_PRODUCT_SPLIT, precision, nrhs, op, s, P, Q, &f));
                double t = 0;
                RTM_TRY(time_product(op, nrhs, (flags & RTM_TUNE_FLUSH_L2) != 0, scratch, s, &t));
                ++measured;
                if (flags & RTM_TUNE_VERBOSE)
                    std::fprintf(stderr, "rtm_tune %dx%d %s nrhs %d: P %d Q %d y_blocks %d mix %d: %.2f us\n", count_x,
                                 count_y, fp64 ? "fp64" : "fp32", nrhs, P, Q, f.y_blocks, f.x_kind, t * 1e6);
                const FastSchedule d = default_fast_schedule(P, Q, fp64);
                if (P == Ps[0] && Q == Qs[0] && (!fast_split_eligible(P, Q, fp64) ||
                                                 (f.y_blocks == d.y_blocks && f.x_kind == d.x_kind)))
                    ref = t;
                if (measured == 1 || t < best) {
                    best = t;
                    choice.P = P;
                    choice.Q = Q;
                    choice.sched = f;
                }
            }
        }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[{dev, precision, count_x, count_y}] = choice;
    }
    out->fft_x = choice.P;
    out->fft_y = choice.Q;
    const bool fast = fast_split_eligible(choice.P, choice.Q, fp64);
    out->y_blocks = fast ? choice.sched.y_blocks : 0;
    out->mix_kind = fast ? choice.sched.x_kind : -1;
    out->seconds = best;
    out->reference_seconds = ref;
    out->candidates = measured;
    return RTM_OK;
}

int rtm_tune_set(int count_x, int count_y, int precision, int fft_x, int fft_y) {
    if (count_x < 2 || count_y < 2) return fail(RTM_ERR_ARG, "transform grids are set for plates of at least 2 x 2 faces");
    if (precision != RTM_FP64 && precision != RTM_FP32) return fail(RTM_ERR_ARG, "unknown precision");
    if (fft_x < count_x || fft_y < count_y) return fail(RTM_ERR_ARG, "a transform grid smaller than the face grid");
    if (fft_x > (1 << 16) || fft_y > (1 << 16)) return fail(RTM_ERR_SIZE, "transform lengths up to 65536");
    register_choice(count_x, count_y, precision, fft_x, fft_y);
    return RTM_OK;
}

int rtm_tune_clear(void) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned.clear();
    return RTM_OK;
}

}  // extern "C"
