// The C ABI of librtm.so (include/rtm.h): handles, argument checks, host <-> device staging.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "batch.h"
#include "excitation.h"
#include "handles.h"
#include "krylov.h"

using namespace rtm;

namespace rtm {
int middle_port(int count_x, int count_y, int direction, std::vector<int64_t>& p) {
    // generateMiddlePort.m:14-28
    const int64_t nx = (int64_t)(count_x - 1) * count_y, n = nx + (int64_t)count_x * (count_y - 1);
    p.clear();
    if (direction == 0) {
        if (nx == 0) return fail(RTM_ERR_ARG, "The mesh has no x-directed rooftops.");
        const int row = count_x / 2 - 1;
        for (int c = 0; c < count_y; ++c) p.push_back(row + (int64_t)c * (count_x - 1));
    } else {
        if (n - nx == 0) return fail(RTM_ERR_ARG, "The mesh has no y-directed rooftops.");
        const int col = count_y / 2 - 1;
        for (int r = 0; r < count_x; ++r) p.push_back(nx + r + (int64_t)col * count_x);
    }
    return RTM_OK;
}

int check_plane_wave(const double* d, const double* p) {
    double dd = 0, pp = 0, dp = 0;
    for (int i = 0; i < 3; ++i) {
        dd += d[i] * d[i];
        pp += p[i] * p[i];
        dp += d[i] * p[i];
    }
    constexpr double kTol = 1e-9;
    if (!(std::fabs(std::sqrt(dd) - 1) <= kTol) || !(std::fabs(std::sqrt(pp) - 1) <= kTol) || !(std::fabs(dp) <= kTol))
        return fail(RTM_ERR_ARG, "The direction and polarization of a plane wave must be perpendicular unit vectors.");
    return RTM_OK;
}
}  // namespace rtm

namespace {

int make_stream(cudaStream_t* s) {
    RTM_CUDA(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking));
    return RTM_OK;
}

// A stream made for one call; declared before the call's staging buffers, it outlives them.
struct CallStream {
    cudaStream_t s = nullptr;
    ~CallStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

cudaStream_t pick(void* user, cudaStream_t own) { return user ? static_cast<cudaStream_t>(user) : own; }

int check_where(int where) {
    if (where != RTM_HOST && where != RTM_DEVICE) return fail(RTM_ERR_ARG, "where must be RTM_HOST or RTM_DEVICE");
    return RTM_OK;
}

// Right-hand sides of one call: the batched launches span them in a grid's y or z dimension.
constexpr int kMaxRhs = 65535;
int check_rhs(int nrhs) {
    if (nrhs < 1) return fail(RTM_ERR_ARG, "nrhs must be positive");
    if (nrhs > kMaxRhs) return fail(RTM_ERR_SIZE, "at most 65535 right-hand sides in one call");
    return RTM_OK;
}

// Input vectors of an operator call as device pointers in the operator's precision.
// Staging blocks go back to the allocator's cache when these leave scope, so any copy or kernel
// still using them on the call's stream is waited for first.
struct Staged {
    DeviceBuffer buf64, buf32;
    const void* ptr = nullptr;
    cudaStream_t stream = nullptr;
    ~Staged() {
        if (buf64.ptr || buf32.ptr) cudaStreamSynchronize(stream);
    }
};

int stage_in(const void* src, int64_t count, int precision, int where, Staged& st, cudaStream_t s) {
    if (where == RTM_DEVICE) {
        st.ptr = src;
        return RTM_OK;
    }
    if (!src) {
        st.ptr = nullptr;
        return RTM_OK;
    }
    st.stream = s;
    RTM_TRY(st.buf64.alloc((size_t)count * sizeof(double2)));
    RTM_CUDA(cudaMemcpyAsync(st.buf64.ptr, src, (size_t)count * sizeof(double2), cudaMemcpyHostToDevice, s));
    if (precision == RTM_FP64) {
        st.ptr = st.buf64.ptr;
        return RTM_OK;
    }
    RTM_TRY(st.buf32.alloc((size_t)count * sizeof(float2)));
    convert_to_fp32(st.buf64.as<double2>(), st.buf32.as<float2>(), count, s);
    st.ptr = st.buf32.ptr;
    return RTM_OK;
}

// An output buffer on the device; stage_out copies it to the host (as complex doubles) if needed.
struct Out {
    DeviceBuffer buf64, buf32;
    void* ptr = nullptr;
    cudaStream_t stream = nullptr;
    ~Out() {
        if (buf64.ptr || buf32.ptr) cudaStreamSynchronize(stream);
    }
};

int out_prepare(void* dst, int64_t count, int precision, int where, Out& o, cudaStream_t s) {
    if (where == RTM_DEVICE) {
        o.ptr = dst;
        return RTM_OK;
    }
    o.stream = s;
    if (precision == RTM_FP64) {
        RTM_TRY(o.buf64.alloc((size_t)count * sizeof(double2)));
        o.ptr = o.buf64.ptr;
    } else {
        RTM_TRY(o.buf32.alloc((size_t)count * sizeof(float2)));
        o.ptr = o.buf32.ptr;
    }
    return RTM_OK;
}

int out_finish(void* dst, int64_t count, int precision, int where, Out& o, cudaStream_t s) {
    if (where == RTM_DEVICE) return RTM_OK;
    if (precision == RTM_FP32) {
        RTM_TRY(o.buf64.alloc((size_t)count * sizeof(double2)));
        convert_to_fp64(o.buf32.as<float2>(), o.buf64.as<double2>(), count, s);
    }
    RTM_CUDA(cudaMemcpyAsync(dst, o.buf64.ptr, (size_t)count * sizeof(double2), cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

int copy_generator(DeviceBuffer& dst, const double* src, int64_t count, int where, cudaStream_t s) {
    if (count <= 0) return RTM_OK;
    if (!src) return fail(RTM_ERR_ARG, "a generator of a present rooftop direction is missing");
    RTM_TRY(dst.alloc((size_t)count * sizeof(double2)));
    RTM_CUDA(cudaMemcpyAsync(dst.ptr, src, (size_t)count * sizeof(double2),
                             where == RTM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, s));
    return RTM_OK;
}

}  // namespace

extern "C" {

int rtm_version(int* major, int* minor, int* patch) {
    if (major) *major = RTM_VERSION_MAJOR;
    if (minor) *minor = RTM_VERSION_MINOR;
    if (patch) *patch = RTM_VERSION_PATCH;
    return RTM_OK;
}

int rtm_set_device(int device) {
    RTM_CUDA(cudaSetDevice(device));
    return RTM_OK;
}

int rtm_launch_count(int64_t* count) {
    if (!count) return fail(RTM_ERR_ARG, "null count");
    *count = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
    return RTM_OK;
}

int rtm_budget_require(double bytes) { return budget_require(bytes, "The request"); }

int rtm_estimate_bytes(int count_x, int count_y, int product, int method, int preconditioned, int restart,
                       int max_iterations, double out[6]) {
    // src/+rooftopMoM/+resources/estimate{Generators,Product,Preconditioner,Solver}.m
    if (!out || count_x < 1 || count_y < 1) return fail(RTM_ERR_ARG, "invalid grid");
    const double nx = (double)(count_x - 1) * count_y, ny = (double)count_x * (count_y - 1), N = nx + ny;
    const bool both = nx > 0 && ny > 0;
    const double blocks = both ? 4 : 1;
    out[0] = 16 * (N + (double)count_x * count_y);
    double sx, sy, sub;
    if (product == RTM_PRODUCT_FFT) {
        sx = std::max(2 * count_x - 2, 1);
        sy = std::max(2 * count_y - 2, 1);
        sub = 1;
    } else {
        sx = count_x > 1 ? fast_fft_size(count_x) : 1;
        sy = count_y > 1 ? fast_fft_size(count_y) : 1;
        sub = (count_x > 1 ? 2 : 1) * (count_y > 1 ? 2 : 1);
    }
    out[1] = 16 * blocks * sub * sx * sy;
    const double grid = 16 * sx * sy;
    if (product == RTM_PRODUCT_FFT) out[2] = both ? 3 * grid + 16 * ny : 2.5 * grid;
    else if (product == RTM_PRODUCT_SPLIT) out[2] = both ? 8 * grid : 3 * grid;
    else {
        if (!both) out[2] = 3 * grid;
        else {
            const int rows[2] = {count_x - 1, count_x}, cols[2] = {count_y, count_y - 1};
            double chunk = 0;
            for (int c = 0; c < 2; ++c)
                chunk = std::max(chunk, (double)rows[c] * std::ceil((double)cols[c] / std::min(32, cols[c])));
            out[2] = 16 * (N + sx * sy + 3 * chunk);
        }
    }
    const double face = 16 * (double)count_x * count_y;
    out[3] = blocks * face;
    out[4] = both ? 3 * face + 16 * ny : 2.5 * face;
    double vectors;
    if (method == RTM_METHOD_CG) vectors = 5 + (preconditioned ? 1 : 0);
    else {
        const double basis = std::min({(double)restart, N, (double)max_iterations}) + 1;
        vectors = 1.5 * basis + 2 + (preconditioned ? 1 : 0);
    }
    out[5] = 16 * N * vectors;
    return RTM_OK;
}

int rtm_generators_assemble(int count_x, int count_y, double size_x, double size_y, double wavenumber, int near_order,
                            int far_order, void* stream, rtm_generators** out) {
    if (!out) return fail(RTM_ERR_ARG, "null output handle");
    *out = nullptr;
    if (count_x < 1 || count_y < 1) return fail(RTM_ERR_ARG, "invalid grid");
    // Problem.m:210-219 (requireAssembly_): the generators and the assembly's working arrays, here the 28
    // lattice-block sums and the 7 moment terms of every block, must fit before anything is built
    const double rooftops = (double)(count_x - 1) * count_y + (double)count_x * (count_y - 1);
    const double gen_bytes = 16.0 * (rooftops + (double)count_x * count_y);
    const double work_bytes = 16.0 * 35 * (count_x + 1.0) * (count_y + 1.0);
    const std::string subject = "The assembly of " + std::to_string((long long)rooftops) + " rooftops (generators " +
                                format_bytes(gen_bytes) + ", chunk " + format_bytes(work_bytes) + ")";
    RTM_TRY(budget_require(gen_bytes + work_bytes, subject.c_str()));
    auto h = std::make_unique<rtm_generators>();
    RTM_CUDA(cudaGetDevice(&h->device));
    RTM_TRY(make_stream(&h->stream));
    RTM_TRY(assemble_generators(count_x, count_y, size_x, size_y, wavenumber, near_order, far_order, h->g,
                                pick(stream, h->stream)));
    if (stream) RTM_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    *out = h.release();
    return RTM_OK;
}

int rtm_generators_create(int count_x, int count_y, const double* magnetic_xx, const double* magnetic_yy,
                          const double* electric, int where, rtm_generators** out) {
    if (!out) return fail(RTM_ERR_ARG, "null output handle");
    *out = nullptr;
    RTM_TRY(check_where(where));
    if (count_x < 1 || count_y < 1 || (count_x == 1 && count_y == 1))
        return fail(RTM_ERR_ARG, "A single face has no interior edge, so it carries no rooftop.");
    auto h = std::make_unique<rtm_generators>();
    RTM_CUDA(cudaGetDevice(&h->device));
    RTM_TRY(make_stream(&h->stream));
    const int64_t nx = (int64_t)(count_x - 1) * count_y, ny = (int64_t)count_x * (count_y - 1);
    h->g.count_x = count_x;
    h->g.count_y = count_y;
    h->g.content = (nx > 0 && ny > 0) ? RTM_BOTH : nx > 0 ? RTM_XONLY : RTM_YONLY;
    RTM_TRY(copy_generator(h->g.e, electric, (int64_t)count_x * count_y, where, h->stream));
    RTM_TRY(copy_generator(h->g.xx, magnetic_xx, nx, where, h->stream));
    RTM_TRY(copy_generator(h->g.yy, magnetic_yy, ny, where, h->stream));
    RTM_CUDA(cudaStreamSynchronize(h->stream));
    *out = h.release();
    return RTM_OK;
}

int rtm_generators_modify(const rtm_generators* g, int modifier, rtm_generators** out) {
    if (!g || !out) return fail(RTM_ERR_ARG, "null handle");
    if (modifier < RTM_MODIFY_NONE || modifier > RTM_MODIFY_IMAG) return fail(RTM_ERR_ARG, "unknown modifier");
    auto h = std::make_unique<rtm_generators>();
    h->device = g->device;
    RTM_TRY(make_stream(&h->stream));
    RTM_TRY(modify_generators(g->g, modifier, h->g, h->stream));
    *out = h.release();
    return RTM_OK;
}

int rtm_generators_read(const rtm_generators* g, double* magnetic_xx, double* magnetic_yy, double* electric,
                        int where) {
    if (!g) return fail(RTM_ERR_ARG, "null handle");
    RTM_TRY(check_where(where));
    const cudaMemcpyKind kind = where == RTM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (magnetic_xx && g->g.xx.ptr) RTM_CUDA(cudaMemcpyAsync(magnetic_xx, g->g.xx.ptr, g->g.xx.bytes, kind, g->stream));
    if (magnetic_yy && g->g.yy.ptr) RTM_CUDA(cudaMemcpyAsync(magnetic_yy, g->g.yy.ptr, g->g.yy.bytes, kind, g->stream));
    if (electric) RTM_CUDA(cudaMemcpyAsync(electric, g->g.e.ptr, g->g.e.bytes, kind, g->stream));
    RTM_CUDA(cudaStreamSynchronize(g->stream));
    return RTM_OK;
}

int rtm_generators_info(const rtm_generators* g, int* count_x, int* count_y, int* content) {
    if (!g) return fail(RTM_ERR_ARG, "null handle");
    if (count_x) *count_x = g->g.count_x;
    if (count_y) *count_y = g->g.count_y;
    if (content) *content = g->g.content;
    return RTM_OK;
}

int rtm_generators_destroy(rtm_generators* g) {
    delete g;
    return RTM_OK;
}

int rtm_operator_create(const rtm_generators* g, double size_x, double size_y, int product, int precision, int max_rhs,
                        rtm_operator** out) {
    if (!g || !out) return fail(RTM_ERR_ARG, "null handle");
    *out = nullptr;
    if (product < RTM_PRODUCT_FFT || product > RTM_PRODUCT_LEAN) return fail(RTM_ERR_ARG, "unknown product");
    if (precision != RTM_FP64 && precision != RTM_FP32) return fail(RTM_ERR_ARG, "unknown precision");
    if (!(size_x > 0) || !(size_y > 0)) return fail(RTM_ERR_ARG, "face sizes must be positive");
    double est[6];
    RTM_TRY(rtm_estimate_bytes(g->g.count_x, g->g.count_y, product, RTM_METHOD_CG, 0, 50, 1000, est));
    const double scale = precision == RTM_FP32 ? 0.5 : 1.0;
    RTM_TRY(budget_require(scale * (est[1] + est[2] * std::max(1, max_rhs)), "The product"));
    auto h = std::make_unique<rtm_operator>();
    h->device = g->device;
    h->kind = product;
    RTM_TRY(make_stream(&h->stream));
    auto grid = std::make_unique<GridApplicator>();
    RTM_TRY(build_product(g->g, size_x, size_y, product, precision, max_rhs, *grid, h->stream));
    h->grid = grid.get();
    h->op = std::move(grid);
    *out = h.release();
    return RTM_OK;
}

int rtm_operator_create_dense(const double* matrix, int64_t n, int where, rtm_operator** out) {
    if (!matrix || !out || n < 1) return fail(RTM_ERR_ARG, "invalid dense matrix");
    *out = nullptr;
    RTM_TRY(check_where(where));
    auto h = std::make_unique<rtm_operator>();
    RTM_CUDA(cudaGetDevice(&h->device));
    h->kind = -1;
    RTM_TRY(make_stream(&h->stream));
    DeviceBuffer tmp;
    const double2* src = reinterpret_cast<const double2*>(matrix);
    if (where == RTM_HOST) {
        RTM_TRY(tmp.alloc((size_t)n * n * sizeof(double2)));
        RTM_CUDA(cudaMemcpy(tmp.ptr, matrix, tmp.bytes, cudaMemcpyHostToDevice));
        src = tmp.as<double2>();
    }
    int st = RTM_OK;
    h->op = make_dense_op(src, n, &st);
    if (st != RTM_OK) return st;
    *out = h.release();
    return RTM_OK;
}

int rtm_operator_apply(rtm_operator* op, const void* x, void* y, int64_t n, int nrhs, int where, void* stream) {
    if (!op || !x || !y) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_where(where));
    if (n != op->op->n) return fail(RTM_ERR_SIZE, "The input must be a numeric " + std::to_string(op->op->n) + "x1 vector.");
    RTM_TRY(check_rhs(nrhs));
    cudaStream_t s = pick(stream, op->stream);
    RTM_TRY(op->op->reserve(nrhs));
    Staged in;
    Out o;
    const int prec = op->op->precision;
    RTM_TRY(stage_in(x, n * nrhs, prec, where, in, s));
    RTM_TRY(out_prepare(y, n * nrhs, prec, where, o, s));
    RTM_TRY(op->op->apply(in.ptr, o.ptr, nrhs, s, SkipFlags{}));
    RTM_TRY(out_finish(y, n * nrhs, prec, where, o, s));
    if (where == RTM_HOST || !stream) RTM_TRY(device_fault_check(s));
    return RTM_OK;
}

int rtm_operator_apply_fixed_scratch(const rtm_operator* op, const void* x, void* y, int64_t n, int nrhs,
                                     void* stream) {
    if (!op || !x || !y) return fail(RTM_ERR_ARG, "null argument");
    if (!op->grid) return fail(RTM_ERR_UNSUPPORTED, "the fixed scratch serves FFT products only");
    if (n != op->op->n) return fail(RTM_ERR_SIZE, "The input must be a numeric " + std::to_string(op->op->n) + "x1 vector.");
    RTM_TRY(check_rhs(nrhs));
    cudaStream_t s = pick(stream, op->stream);
    RTM_TRY(apply_fixed_scratch(*op->grid, x, y, nrhs, s));
    if (!stream) RTM_TRY(device_fault_check(s));
    return RTM_OK;
}

int rtm_fixed_scratch_bytes(double* bytes) {
    if (!bytes) return fail(RTM_ERR_ARG, "null argument");
    *bytes = (double)fixed_scratch_bytes();
    return RTM_OK;
}

int rtm_operator_info(const rtm_operator* op, int64_t* n, int* fft_x, int* fft_y, double* spectra_bytes,
                      double* working_bytes) {
    if (!op) return fail(RTM_ERR_ARG, "null handle");
    if (n) *n = op->op->n;
    if (fft_x) *fft_x = op->grid ? op->grid->P : 0;
    if (fft_y) *fft_y = op->grid ? op->grid->Q : 0;
    if (spectra_bytes) *spectra_bytes = op->op->stored_bytes();
    if (working_bytes) *working_bytes = op->op->working_bytes();
    return RTM_OK;
}

int rtm_operator_read_spectra(const rtm_operator* op, double* out, int* count) {
    if (!op || !op->grid) return fail(RTM_ERR_ARG, "not an FFT product");
    const GridApplicator& g = *op->grid;
    if (count) *count = g.spec_blocks;
    if (!out) return RTM_OK;
    const int64_t elems = (int64_t)(g.spec.bytes / (g.precision == RTM_FP64 ? sizeof(double2) : sizeof(float2)));
    if (g.precision == RTM_FP64) {
        RTM_CUDA(cudaMemcpy(out, g.spec.ptr, g.spec.bytes, cudaMemcpyDeviceToHost));
    } else {
        DeviceBuffer tmp;
        RTM_TRY(tmp.alloc((size_t)elems * sizeof(double2)));
        convert_to_fp64(g.spec.as<float2>(), tmp.as<double2>(), elems, op->stream);
        RTM_CUDA(cudaStreamSynchronize(op->stream));
        RTM_CUDA(cudaMemcpy(out, tmp.ptr, tmp.bytes, cudaMemcpyDeviceToHost));
    }
    return RTM_OK;
}

int rtm_operator_destroy(rtm_operator* op) {
    delete op;
    return RTM_OK;
}

int rtm_preconditioner_create(const rtm_generators* g, double size_x, double size_y, int kernel, int builder,
                              const int* bandwidth, int precision, rtm_preconditioner** out) {
    if (!g || !out) return fail(RTM_ERR_ARG, "null handle");
    *out = nullptr;
    if (kernel < RTM_KERNEL_STRANG || kernel > RTM_KERNEL_SUPEROPTIMAL) return fail(RTM_ERR_ARG, "unknown kernel");
    if (builder < RTM_BUILDER_PARTWISE || builder > RTM_BUILDER_HYBRID) return fail(RTM_ERR_ARG, "unknown builder");
    if (bandwidth && (bandwidth[0] < 1 || bandwidth[1] < 1))
        return fail(RTM_ERR_ARG, "The bandwidth is a pair [bandwidthX, bandwidthY].");
    double est[6];
    RTM_TRY(rtm_estimate_bytes(g->g.count_x, g->g.count_y, RTM_PRODUCT_SPLIT, RTM_METHOD_CG, 1, 50, 1000, est));
    RTM_TRY(budget_require(est[3] + est[4], "The circulant preconditioner"));
    auto h = std::make_unique<rtm_preconditioner>();
    h->device = g->device;
    RTM_TRY(make_stream(&h->stream));
    auto grid = std::make_unique<GridApplicator>();
    RTM_TRY(build_circulant(g->g, size_x, size_y, kernel, builder, bandwidth, precision, *grid, h->stream));
    h->op = std::move(grid);
    *out = h.release();
    return RTM_OK;
}

int rtm_preconditioner_create_block_jacobi(const rtm_generators* g, double size_x, double size_y, int block_x,
                                           int block_y, int precision, rtm_preconditioner** out) {
    if (!g || !out) return fail(RTM_ERR_ARG, "null handle");
    *out = nullptr;
    auto h = std::make_unique<rtm_preconditioner>();
    h->device = g->device;
    RTM_TRY(make_stream(&h->stream));
    int st = RTM_OK;
    h->op = make_block_jacobi(g->g, size_x, size_y, block_x, block_y, precision, h->stream, &st);
    if (st != RTM_OK) return st;
    *out = h.release();
    return RTM_OK;
}

int rtm_preconditioner_apply(rtm_preconditioner* pc, const void* x, void* y, int64_t n, int nrhs, int where,
                             void* stream) {
    if (!pc || !x || !y) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_where(where));
    if (n != pc->op->n) return fail(RTM_ERR_SIZE, "The input must be a numeric " + std::to_string(pc->op->n) + "x1 vector.");
    RTM_TRY(check_rhs(nrhs));
    cudaStream_t s = pick(stream, pc->stream);
    RTM_TRY(pc->op->reserve(nrhs));
    Staged in;
    Out o;
    const int prec = pc->op->precision;
    RTM_TRY(stage_in(x, n * nrhs, prec, where, in, s));
    RTM_TRY(out_prepare(y, n * nrhs, prec, where, o, s));
    RTM_TRY(pc->op->apply(in.ptr, o.ptr, nrhs, s, SkipFlags{}));
    RTM_TRY(out_finish(y, n * nrhs, prec, where, o, s));
    if (where == RTM_HOST || !stream) RTM_TRY(device_fault_check(s));
    return RTM_OK;
}

int rtm_preconditioner_destroy(rtm_preconditioner* pc) {
    delete pc;
    return RTM_OK;
}

static int check_config(const rtm_solve_config* c) {
    if (!c) return fail(RTM_ERR_ARG, "null config");
    if (!(c->tolerance > 0) || !(c->tolerance < 1)) return fail(RTM_ERR_ARG, "tolerance must lie in (0, 1)");
    if (c->max_iterations < 1) return fail(RTM_ERR_ARG, "maxIterationCount must be positive");
    if (c->method == RTM_METHOD_GMRES && c->restart < 1) return fail(RTM_ERR_ARG, "The restart is a positive integer.");
    if (c->gram_schmidt_passes < 0 || c->gram_schmidt_passes > 2)
        return fail(RTM_ERR_ARG, "gram_schmidt_passes is 0 (the default), 1 or 2");
    return RTM_OK;
}

static void copy_out_stats(const SolveResult& r, double* history, rtm_solve_stats* stats, int nrhs, int max_iterations,
                           float ms) {
    for (int k = 0; k < nrhs; ++k) {
        if (stats) {
            stats[k] = r.stats[k];
            stats[k].time_s = ms * 1e-3;
        }
        if (history)
            for (int i = 0; i <= max_iterations; ++i)
                history[(size_t)k * (max_iterations + 1) + i] =
                    i < r.hist_stride ? r.history[(size_t)k * r.hist_stride + i] : NAN;
    }
}

int rtm_solve(rtm_operator* op, rtm_preconditioner* pc, const rtm_solve_config* config, const void* b, const void* x0,
              void* x, int64_t n, int nrhs, int where, double* history, rtm_solve_stats* stats, void* stream) {
    if (!op || !b || !x) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_config(config));
    RTM_TRY(check_where(where));
    RTM_TRY(check_rhs(nrhs));
    if (n != op->op->n) return fail(RTM_ERR_SIZE, "The operator does not match the " + std::to_string(n) +
                                                      " unknowns of the right-hand side.");
    if (pc && pc->op->n != n) return fail(RTM_ERR_SIZE, "The preconditioner does not match the " + std::to_string(n) +
                                                            " unknowns of the right-hand side.");
    if (pc && pc->op->precision != op->op->precision)
        return fail(RTM_ERR_ARG, "operator and preconditioner must have one precision");
    if (config->method == RTM_METHOD_FGMRES_IR) return fail(RTM_ERR_ARG, "use rtm_solve_mixed for FGMRES_IR");
    double est[6];
    if (op->grid) {
        RTM_TRY(rtm_estimate_bytes(op->grid->count_x, op->grid->count_y, op->kind, config->method, pc != nullptr,
                                   config->restart, config->max_iterations, est));
        RTM_TRY(budget_require(est[5] * nrhs * (op->op->precision == RTM_FP32 ? 0.5 : 1.0), "The solve"));
    }
    cudaStream_t s = pick(stream, op->stream);
    const int prec = op->op->precision;
    Staged sb, sx0;
    Out o;
    RTM_TRY(stage_in(b, n * nrhs, prec, where, sb, s));
    RTM_TRY(stage_in(x0, n * nrhs, prec, where, sx0, s));
    RTM_TRY(out_prepare(x, n * nrhs, prec, where, o, s));
    SolveConfig cfg;
    cfg.method = config->method;
    cfg.tolerance = config->tolerance;
    cfg.max_iterations = config->max_iterations;
    cfg.restart = config->restart;
    cfg.check_every = config->check_every;
    cfg.right_preconditioned = config->right_preconditioned;
    cfg.gram_schmidt_passes = config->gram_schmidt_passes == 0 ? 2 : config->gram_schmidt_passes;
    cudaEvent_t e0, e1;
    RTM_CUDA(cudaEventCreate(&e0));
    RTM_CUDA(cudaEventCreate(&e1));
    RTM_CUDA(cudaEventRecord(e0, s));
    SolveResult res;
    int st = rtm::solve(op->op.get(), pc ? pc->op.get() : nullptr, cfg, sb.ptr, x0 ? sx0.ptr : nullptr, o.ptr, n, nrhs,
                        res, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RTM_OK) return st;
    RTM_TRY(out_finish(x, n * nrhs, prec, where, o, s));
    copy_out_stats(res, history, stats, nrhs, config->max_iterations, ms);
    return RTM_OK;
}

int rtm_solve_mixed(rtm_operator* op, rtm_operator* inner_op, rtm_preconditioner* inner_pc,
                    const rtm_solve_config* config, const void* b, const void* x0, void* x, int64_t n, int nrhs,
                    int where, double* history, rtm_solve_stats* stats, void* stream) {
    if (!op || !inner_op || !b || !x) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_config(config));
    RTM_TRY(check_where(where));
    RTM_TRY(check_rhs(nrhs));
    if (op->op->precision != RTM_FP64 || inner_op->op->precision != RTM_FP32)
        return fail(RTM_ERR_ARG, "the outer operator is FP64 and the inner one FP32");
    if (inner_pc && inner_pc->op->precision != RTM_FP32) return fail(RTM_ERR_ARG, "the inner preconditioner is FP32");
    if (n != op->op->n || n != inner_op->op->n || (inner_pc && inner_pc->op->n != n))
        return fail(RTM_ERR_SIZE, "operator sizes do not match the right-hand side");
    cudaStream_t s = pick(stream, op->stream);
    Staged sb, sx0;
    Out o;
    RTM_TRY(stage_in(b, n * nrhs, RTM_FP64, where, sb, s));
    RTM_TRY(stage_in(x0, n * nrhs, RTM_FP64, where, sx0, s));
    RTM_TRY(out_prepare(x, n * nrhs, RTM_FP64, where, o, s));
    SolveConfig cfg;
    cfg.method = config->method;
    cfg.tolerance = config->tolerance;
    cfg.max_iterations = config->max_iterations;
    cfg.restart = config->restart;
    cfg.check_every = config->check_every;
    cfg.inner_tolerance = config->inner_tolerance > 0 ? config->inner_tolerance : 1e-4;
    cfg.max_refinements = config->max_refinements > 0 ? config->max_refinements : 20;
    cfg.inner_gram_schmidt_passes = config->gram_schmidt_passes == 0 ? 1 : config->gram_schmidt_passes;
    cudaEvent_t e0, e1;
    RTM_CUDA(cudaEventCreate(&e0));
    RTM_CUDA(cudaEventCreate(&e1));
    RTM_CUDA(cudaEventRecord(e0, s));
    SolveResult res;
    int st = rtm::solve_mixed(op->op.get(), inner_op->op.get(), inner_pc ? inner_pc->op.get() : nullptr, cfg, sb.ptr,
                              x0 ? sx0.ptr : nullptr, o.ptr, n, nrhs, res, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RTM_OK) return st;
    RTM_TRY(out_finish(x, n * nrhs, RTM_FP64, where, o, s));
    copy_out_stats(res, history, stats, nrhs, config->max_iterations, ms);
    return RTM_OK;
}

int rtm_plane_wave(int count_x, int count_y, double size_x, double size_y, int order, double wavenumber,
                   const double* directions, const double* polarizations, const double* intensities, int nrhs,
                   void* out, int where, void* stream) {
    if (!directions || !polarizations || !intensities || !out) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_rhs(nrhs));
    RTM_TRY(check_where(where));
    for (int k = 0; k < nrhs; ++k) RTM_TRY(check_plane_wave(directions + 3 * k, polarizations + 3 * k));
    if (count_x < 1 || count_y < 1 || order < 1) return fail(RTM_ERR_ARG, "invalid grid or order");
    CallStream own;
    RTM_TRY(make_stream(&own.s));
    cudaStream_t s = pick(stream, own.s);
    const int64_t n = (int64_t)(count_x - 1) * count_y + (int64_t)count_x * (count_y - 1);
    Out o;
    int st = out_prepare(out, n * nrhs, RTM_FP64, where, o, s);
    if (st == RTM_OK)
        st = plane_wave(count_x, count_y, size_x, size_y, order, wavenumber, directions, polarizations, intensities,
                        nrhs, static_cast<double2*>(o.ptr), s);
    if (st == RTM_OK) st = out_finish(out, n * nrhs, RTM_FP64, where, o, s);
    cudaStreamSynchronize(s);
    return st;
}

int rtm_delta_gap(int count_x, int count_y, double size_x, double size_y, const int64_t* port, int port_count,
                  int direction, double voltage, void* out, int where) {
    if (!out) return fail(RTM_ERR_ARG, "null output");
    RTM_TRY(check_where(where));
    const int64_t nx = (int64_t)(count_x - 1) * count_y, n = nx + (int64_t)count_x * (count_y - 1);
    std::vector<int64_t> p;
    if (port && port_count > 0) {
        p.assign(port, port + port_count);
        std::vector<int64_t> sorted(p);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end() || sorted.front() < 0 || sorted.back() >= n)
            return fail(RTM_ERR_ARG, "The port must hold distinct rooftop indices up to " + std::to_string(n) + ".");
    } else {
        RTM_TRY(middle_port(count_x, count_y, direction, p));
    }
    std::vector<double2> v((size_t)n, make_double2(0, 0));
    for (int64_t i : p) v[(size_t)i] = make_double2(voltage * (i < nx ? size_y : size_x), 0.0);
    if (where == RTM_HOST) std::memcpy(out, v.data(), v.size() * sizeof(double2));
    else RTM_CUDA(cudaMemcpy(out, v.data(), v.size() * sizeof(double2), cudaMemcpyHostToDevice));
    return RTM_OK;
}

int rtm_radar_cross_section(double wavenumber, const void* excitation, const void* current, int64_t n,
                            double intensity, int where, double* out) {
    if (!excitation || !current || !out || n < 1) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_where(where));
    CallStream own;
    RTM_TRY(make_stream(&own.s));
    cudaStream_t s = own.s;
    Staged e, j;
    int st = stage_in(excitation, n, RTM_FP64, where, e, s);
    if (st == RTM_OK) st = stage_in(current, n, RTM_FP64, where, j, s);
    if (st == RTM_OK)
        st = radar_cross_section(wavenumber, static_cast<const double2*>(e.ptr), static_cast<const double2*>(j.ptr), n,
                                 intensity, out, s);
    return st;
}

int rtm_input_impedance(int count_x, int count_y, double size_x, double size_y, const void* current,
                        const int64_t* port, int port_count, double voltage, int where, double* out) {
    if (!current || !port || port_count < 1 || !out) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_where(where));
    if (count_x < 1 || count_y < 1) return fail(RTM_ERR_ARG, "invalid grid");
    const int64_t n = (int64_t)(count_x - 1) * count_y + (int64_t)count_x * (count_y - 1);
    // the port's currents are gathered on the device: every index must name a rooftop
    for (int i = 0; i < port_count; ++i)
        if (port[i] < 0 || port[i] >= n)
            return fail(RTM_ERR_ARG, "The port must hold rooftop indices below " + std::to_string(n) + ".");
    CallStream own;
    RTM_TRY(make_stream(&own.s));
    cudaStream_t s = own.s;
    Staged j;
    int st = stage_in(current, n, RTM_FP64, where, j, s);
    if (st == RTM_OK)
        st = input_impedance(count_x, count_y, size_x, size_y, static_cast<const double2*>(j.ptr), port, port_count,
                             voltage, out, s);
    return st;
}

struct rtm_plate_batch {
    std::unique_ptr<rtm::BatchOp> op, pc;
    int device = 0;
    cudaStream_t stream = nullptr;
    ~rtm_plate_batch() {
        if (stream) cudaStreamSynchronize(stream);
        op.reset();
        pc.reset();
        if (stream) cudaStreamDestroy(stream);
    }
};

int rtm_plate_batch_create(rtm_operator* const* ops, rtm_preconditioner* const* pcs, int count,
                           rtm_plate_batch** out) {
    if (!ops || !out) return fail(RTM_ERR_ARG, "null argument");
    *out = nullptr;
    RTM_TRY(check_rhs(count));
    std::vector<LinearOp*> o(count), p;
    int64_t stride = 0;
    for (int k = 0; k < count; ++k) {
        if (!ops[k]) return fail(RTM_ERR_ARG, "null operator in a plate batch");
        o[k] = ops[k]->op.get();
        stride = std::max(stride, o[k]->n);
    }
    if (pcs) {
        p.resize(count);
        for (int k = 0; k < count; ++k) {
            if (!pcs[k]) return fail(RTM_ERR_ARG, "null preconditioner in a plate batch");
            if (pcs[k]->op->n != o[k]->n)
                return fail(RTM_ERR_SIZE, "The preconditioner does not match the " + std::to_string(o[k]->n) +
                                              " unknowns of its plate.");
            if (pcs[k]->op->precision != o[k]->precision)
                return fail(RTM_ERR_ARG, "operator and preconditioner must have one precision");
            p[k] = pcs[k]->op.get();
        }
    }
    auto h = std::make_unique<rtm_plate_batch>();
    h->device = ops[0]->device;
    RTM_TRY(make_stream(&h->stream));
    int st = RTM_OK;
    h->op = make_batch(o, stride, true, h->stream, &st);
    RTM_TRY(st);
    if (pcs) {
        h->pc = make_batch(p, stride, true, h->stream, &st);
        RTM_TRY(st);
    }
    *out = h.release();
    return RTM_OK;
}

int rtm_plate_batch_info(const rtm_plate_batch* b, int64_t* stride, int* count, int* fused, int* fused_preconditioner) {
    if (!b) return fail(RTM_ERR_ARG, "null handle");
    if (stride) *stride = b->op->stride;
    if (count) *count = (int)b->op->ops.size();
    if (fused) *fused = b->op->fused ? 1 : 0;
    if (fused_preconditioner) *fused_preconditioner = b->pc && b->pc->fused_bj ? 1 : 0;
    return RTM_OK;
}

int rtm_plate_batch_apply(rtm_plate_batch* b, int preconditioner, const void* x, void* y, int where, void* stream) {
    if (!b || !x || !y) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_where(where));
    if (preconditioner != 0 && preconditioner != 1) return fail(RTM_ERR_ARG, "preconditioner is 0 or 1");
    if (preconditioner && !b->pc) return fail(RTM_ERR_ARG, "the batch has no preconditioners");
    BatchOp* op = preconditioner ? b->pc.get() : b->op.get();
    cudaStream_t s = pick(stream, b->stream);
    const int count = (int)op->ops.size();
    const int64_t total = op->stride * count;
    const int prec = op->precision;
    Staged in;
    Out o;
    RTM_TRY(stage_in(x, total, prec, where, in, s));
    RTM_TRY(out_prepare(y, total, prec, where, o, s));
    RTM_TRY(op->reserve(count));
    RTM_TRY(op->apply(in.ptr, o.ptr, count, s, SkipFlags{}));
    RTM_TRY(out_finish(y, total, prec, where, o, s));
    if (where == RTM_HOST || !stream) RTM_CUDA(cudaStreamSynchronize(s));
    return device_fault_check(s);
}

int rtm_plate_batch_solve(rtm_plate_batch* b, const rtm_solve_config* config, const void* rhs, const void* x0,
                          void* x, int where, double* history, rtm_solve_stats* stats, void* stream) {
    if (!b || !rhs || !x) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_config(config));
    RTM_TRY(check_where(where));
    if (config->method == RTM_METHOD_FGMRES_IR) return fail(RTM_ERR_ARG, "a plate batch solves by COCG or GMRES");
    const int count = (int)b->op->ops.size();
    const int64_t stride = b->op->stride, total = stride * count;
    const int prec = b->op->precision;
    const size_t elem = prec == RTM_FP64 ? sizeof(double2) : sizeof(float2);
    // the solver's vectors: GMRES the basis and three more, COCG six
    const int m = (int)std::max<int64_t>(1, std::min<int64_t>(config->restart, stride));
    const double vectors = config->method == RTM_METHOD_GMRES ? m + 4.0 : 6.0;
    RTM_TRY(budget_require(vectors * (double)total * elem, "The solve"));
    cudaStream_t s = pick(stream, b->stream);
    Staged sb, sx0;
    Out o;
    RTM_TRY(stage_in(rhs, total, prec, where, sb, s));
    RTM_TRY(stage_in(x0, total, prec, where, sx0, s));
    RTM_TRY(out_prepare(x, total, prec, where, o, s));
    // the solver reads the right-hand sides and the initial guesses with their tails zeroed
    DeviceBuffer bz, xz;
    RTM_TRY(bz.alloc(total * elem));
    RTM_CUDA(cudaMemcpyAsync(bz.ptr, sb.ptr, total * elem, cudaMemcpyDeviceToDevice, s));
    RTM_TRY(zero_tails(bz.ptr, prec, stride, b->op->tails.as<int64_t>(), count, b->op->max_tail, s, SkipFlags{}));
    if (x0) {
        RTM_TRY(xz.alloc(total * elem));
        RTM_CUDA(cudaMemcpyAsync(xz.ptr, sx0.ptr, total * elem, cudaMemcpyDeviceToDevice, s));
        RTM_TRY(zero_tails(xz.ptr, prec, stride, b->op->tails.as<int64_t>(), count, b->op->max_tail, s,
                           SkipFlags{}));
    }
    SolveConfig cfg;
    cfg.method = config->method;
    cfg.tolerance = config->tolerance;
    cfg.max_iterations = config->max_iterations;
    cfg.restart = config->restart;
    cfg.check_every = config->check_every;
    cfg.right_preconditioned = config->right_preconditioned;
    cfg.gram_schmidt_passes = config->gram_schmidt_passes == 0 ? 2 : config->gram_schmidt_passes;
    cudaEvent_t e0, e1;
    RTM_CUDA(cudaEventCreate(&e0));
    RTM_CUDA(cudaEventCreate(&e1));
    RTM_CUDA(cudaEventRecord(e0, s));
    SolveResult res;
    int st = rtm::solve(b->op.get(), b->pc.get(), cfg, bz.ptr, x0 ? xz.ptr : nullptr, o.ptr, stride, count, res, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != RTM_OK) return st;
    RTM_TRY(out_finish(x, total, prec, where, o, s));
    copy_out_stats(res, history, stats, count, config->max_iterations, ms);
    return RTM_OK;
}

int rtm_plate_batch_destroy(rtm_plate_batch* b) {
    delete b;
    return RTM_OK;
}

}  // extern "C"
