// The serving form: a request loop of plate solves (include/rtm.h, rtm_server_*).
//
// Admission follows the reference's memory ledger (src/+rooftopMoM/+resources/Budget.m:82-106): a
// request is admitted only when its estimated device bytes (the byte models of
// estimateGenerators.m:11, estimateProduct.m:13-37 and estimateSolver.m:19-26, as rtm_estimate_bytes)
// fit under what the admitted requests leave of the budget. Admission scans the queue in arrival
// order and takes every request that fits while a slot is free, so a large request at the head does
// not hold back small ones behind it.
//
// Each slot is a host worker thread. An admitted request runs its whole pipeline on that thread with
// the handles' own non-blocking streams: assembly, split-FFT product, preconditioner (block-Jacobi or rChan),
// excitation on the device, the solve, the RCS or input impedance. Device work of different requests
// overlaps; no call here synchronises the whole device. Results depend on the request alone, since
// every launch shape follows from the request's sizes. With max_batch > 1 a worker takes several admitted
// requests of one batch key and solves them as one plate batch (batch.h); their results then agree with
// the same requests solved alone to their tolerances, and a batch that fails runs its requests alone.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "grid.h"
#include "handles.h"
#include "krylov.h"

using namespace rtm;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kBlockJacobiUnknowns = 8;  // packed unknowns a 2 x 2-face block of the block-Jacobi inverse (ops.cu)
constexpr int kPcBlockJacobi = 1, kPcCirculant = 2;  // rtm_request.preconditioner
constexpr int kInnerCap = 3000;  // iterations of one inner FP32 solve of the mixed server

struct Record {
    uint64_t id = 0;
    rtm_request req{};
    rtm_request_result res{};
    std::vector<double> current;  // interleaved complex
    std::atomic<int> cancel{0};  // set by rtm_server_cancel / destroy, read by the worker and the solver
};

// What a request's pipeline produces: the result fields it fills and the current it keeps.
struct Outcome {
    rtm_request_result res{};
    std::vector<double> current;
    void commit(rtm_request_result& to) const {
        to.unknowns = res.unknowns;
        to.solve_s = res.solve_s;
        to.converged = res.converged;
        to.iteration_count = res.iteration_count;
        to.residual_norm = res.residual_norm;
        to.rcs = res.rcs;
        to.impedance[0] = res.impedance[0];
        to.impedance[1] = res.impedance[1];
    }
};

double seconds_since(Clock::time_point t0) {
    return std::chrono::duration<double>(Clock::now() - t0).count();
}

int check_request(const rtm_request& q) {
    if (q.count_x < 1 || q.count_y < 1) return fail(RTM_ERR_ARG, "The face counts must be positive.");
    if ((int64_t)(q.count_x - 1) * q.count_y + (int64_t)q.count_x * (q.count_y - 1) < 1)
        return fail(RTM_ERR_ARG, "The plate is a single face, which carries no rooftop.");
    if (!(q.size_x > 0) || !(q.size_y > 0) || !(q.wavenumber > 0)) return fail(RTM_ERR_ARG, "invalid sizes");
    if (q.excitation != RTM_EXCITE_PLANE_WAVE && q.excitation != RTM_EXCITE_DELTA_GAP)
        return fail(RTM_ERR_ARG, "unknown excitation");
    if (q.excitation == RTM_EXCITE_PLANE_WAVE) RTM_TRY(check_plane_wave(q.direction, q.polarization));
    if (q.method != RTM_METHOD_CG && q.method != RTM_METHOD_GMRES) return fail(RTM_ERR_ARG, "unknown method");
    if (!(q.tolerance > 0) || q.max_iterations < 1 || q.restart < 1) return fail(RTM_ERR_ARG, "invalid solver");
    if (q.preconditioner < 0 || q.preconditioner > kPcCirculant) return fail(RTM_ERR_ARG, "unknown preconditioner");
    return RTM_OK;
}

int next_pow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Device bytes of a request's pipeline (generators, product spectra and working grids, preconditioner,
// solver vectors, excitation and solution), in the server's precision. Under a power-of-two or autotuned
// size policy a plate's product is counted at the power-of-two grid where the power-of-two kernels take it
// (the larger of the candidates).
int request_bytes(const rtm_request& q, int precision, int sizes, double* bytes) {
    double est[6];
    RTM_TRY(rtm_estimate_bytes(q.count_x, q.count_y, RTM_PRODUCT_SPLIT, q.method, q.preconditioner != 0, q.restart,
                               q.max_iterations, est));
    if (sizes != RTM_SIZES_REFERENCE && q.count_x > 1 && q.count_y > 1) {
        const int P = next_pow2(q.count_x), Q = next_pow2(q.count_y);
        if (fast_split_eligible(P, Q, precision == RTM_FP64)) {
            const double grow = (double)P * Q / ((double)fast_fft_size(q.count_x) * fast_fft_size(q.count_y));
            est[1] *= grow;
            est[2] *= grow;
        }
    }
    const double n = (double)(q.count_x - 1) * q.count_y + (double)q.count_x * (q.count_y - 1);
    const double blocks = (double)((q.count_x + 1) / 2) * ((q.count_y + 1) / 2);
    double pc = 0;
    if (q.preconditioner == kPcBlockJacobi)
        pc = blocks * (kBlockJacobiUnknowns * kBlockJacobiUnknowns * 16.0 + kBlockJacobiUnknowns * 8.0 + 4);
    else if (q.preconditioner == kPcCirculant)
        pc = est[3] + est[4];
    double total = est[0] + est[1] + est[2] + pc + est[5] + 2 * 16 * n;
    // inner FP32 copies, and the FP32 preconditioner beside the FP64 one of the FP64 finish
    if (precision == RTM_FP32) total += 0.5 * (est[1] + est[2] + est[5] + pc) + 4 * 16 * n;
    *bytes = total;
    return RTM_OK;
}

}  // namespace

struct rtm_server {
    rtm_server_config cfg{};
    Clock::time_point epoch;
    std::mutex mu;
    std::condition_variable work_cv, done_cv;
    std::deque<uint64_t> queue;  // waiting, in arrival order
    std::deque<uint64_t> ready;  // admitted, not yet taken by a worker
    std::map<uint64_t, std::unique_ptr<Record>> records;
    double held = 0;
    int admitted = 0;
    uint64_t next_id = 1;
    bool stopping = false;
    std::atomic<int> stop_flag{0};  // the cancel flag of batched solves: set when the server stops
    std::vector<std::thread> workers;

    // Requests that may share one plate batch: 2-D plates whose split products take one power-of-two
    // transform grid under the power-of-two policy, with one method, preconditioner, restart and iteration
    // bound (each keeps its own tolerance). False when the request solves alone.
    bool batch_key(const rtm_request& q, std::vector<int>& key) const {
        if (cfg.max_batch < 2 || cfg.precision != RTM_FP64 || cfg.transform_sizes != RTM_SIZES_POWER_OF_TWO ||
            q.count_x < 2 || q.count_y < 2)
            return false;
        const int P = next_pow2(q.count_x), Q = next_pow2(q.count_y);
        if (!fast_split_eligible(P, Q, true)) return false;
        key = {P, Q, q.method, q.preconditioner, q.restart, q.max_iterations};
        return true;
    }

    void admit_locked() {
        for (auto it = queue.begin(); it != queue.end() && admitted < cfg.max_active;) {
            Record& r = *records.at(*it);
            if (held + r.res.bytes <= cfg.budget_bytes) {
                held += r.res.bytes;
                ++admitted;
                ready.push_back(*it);
                it = queue.erase(it);
                work_cv.notify_one();
            } else {
                ++it;
            }
        }
    }

    void worker() {
        cudaSetDevice(cfg.device);
        while (true) {
            std::vector<Record*> group;
            {
                std::unique_lock<std::mutex> lk(mu);
                work_cv.wait(lk, [&] { return stopping || !ready.empty(); });
                if (ready.empty()) return;  // stopping
                Record* r = records.at(ready.front()).get();
                ready.pop_front();
                if (r->cancel) {
                    // Cancelled while admitted: give its bytes and slot back in this same critical
                    // section. Once the state reads CANCELLED a poll with release may erase the
                    // record, so nothing touches r after the lock is dropped.
                    r->res.state = RTM_REQUEST_CANCELLED;
                    r->res.finished_s = seconds_since(epoch);
                    held -= r->res.bytes;
                    --admitted;
                    admit_locked();
                    lk.unlock();
                    done_cv.notify_all();
                    continue;
                }
                group.push_back(r);
                std::vector<int> key, other;
                if (batch_key(r->req, key))
                    for (auto it = ready.begin(); it != ready.end() && (int)group.size() < cfg.max_batch;) {
                        Record* o = records.at(*it).get();
                        if (!o->cancel && batch_key(o->req, other) && other == key) {
                            group.push_back(o);
                            it = ready.erase(it);
                        } else {
                            ++it;
                        }
                    }
                const double now = seconds_since(epoch);  // a batch's requests start together
                for (Record* g : group) {
                    g->res.state = RTM_REQUEST_RUNNING;
                    g->res.started_s = now;
                }
            }
            // RUNNING is not a finished state, so no poll releases the records while they run.
            std::vector<Outcome> outs(group.size());
            std::vector<int> sts(group.size());
            if (group.size() == 1) {
                sts[0] = run(*group[0], outs[0]);
            } else if (run_batch(group, outs) == RTM_OK) {
                std::fill(sts.begin(), sts.end(), RTM_OK);
            } else {
                // the batch failed (one request's set-up, or the batch's own memory): each request runs alone,
                // so one that cannot run fails without the others
                for (size_t k = 0; k < group.size(); ++k) {
                    outs[k] = Outcome{};
                    sts[k] = run(*group[k], outs[k]);
                }
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                const double now = seconds_since(epoch);  // and finish together
                for (size_t k = 0; k < group.size(); ++k) {
                    Record* r = group[k];
                    const int st = sts[k];
                    outs[k].commit(r->res);
                    r->current = std::move(outs[k].current);
                    r->res.finished_s = now;
                    r->res.status = st;
                    held -= r->res.bytes;
                    --admitted;
                    r->res.state = r->cancel ? RTM_REQUEST_CANCELLED
                                             : (st == RTM_OK ? RTM_REQUEST_DONE : RTM_REQUEST_FAILED);
                }
                admit_locked();
            }
            done_cv.notify_all();
        }
    }

    // The transform grid of a plate's split products under the server's policy (strips keep the
    // reference's sizes). Choices are per device and face grid, shared by all requests of that grid.
    int choose_sizes(int cx, int cy, int precision) {
        if (cfg.transform_sizes == RTM_SIZES_REFERENCE || cx < 2 || cy < 2) return RTM_OK;
        int P = 0, Q = 0;
        FastSchedule f;
        if (tuned_choice(cx, cy, precision, &P, &Q, &f)) return RTM_OK;
        if (cfg.transform_sizes == RTM_SIZES_AUTOTUNE) {
            rtm_tune_result r{};
            return rtm_tune_product(cx, cy, precision, 1, RTM_TUNE_FLUSH_L2, &r);
        }
        if (fast_split_eligible(next_pow2(cx), next_pow2(cy), precision == RTM_FP64))
            register_choice(cx, cy, precision, next_pow2(cx), next_pow2(cy));
        return RTM_OK;
    }

    // A request's device state between the stages of its pipeline.
    struct Prepared {
        rtm_generators* g = nullptr;
        rtm_operator* op = nullptr;
        rtm_operator* op32 = nullptr;
        rtm_preconditioner* pc = nullptr;
        rtm_preconditioner* pc64 = nullptr;  // mixed: the FP64 preconditioner of the FP64 finish
        DeviceBuffer b, x;
        std::vector<int64_t> port;
        int64_t n = 0;
        cudaStream_t s = nullptr;
        Prepared() = default;
        Prepared(const Prepared&) = delete;
        Prepared& operator=(const Prepared&) = delete;
        ~Prepared() {
            if (s) cudaStreamSynchronize(s);
            b.reset();
            x.reset();
            rtm_preconditioner_destroy(pc64);
            rtm_preconditioner_destroy(pc);
            rtm_operator_destroy(op32);
            rtm_operator_destroy(op);
            rtm_generators_destroy(g);
        }
    };

    // Assembly, split-FFT product(s), preconditioner(s) and the excitation on the device.
    int prepare(const rtm_request& q, Prepared& h) {
        const bool mixed = cfg.precision == RTM_FP32;
        RTM_TRY(choose_sizes(q.count_x, q.count_y, RTM_FP64));
        if (mixed) RTM_TRY(choose_sizes(q.count_x, q.count_y, RTM_FP32));
        RTM_TRY(rtm_generators_assemble(q.count_x, q.count_y, q.size_x, q.size_y, q.wavenumber, 16, 8, nullptr, &h.g));
        RTM_TRY(rtm_operator_create(h.g, q.size_x, q.size_y, RTM_PRODUCT_SPLIT, RTM_FP64, 1, &h.op));
        if (mixed) RTM_TRY(rtm_operator_create(h.g, q.size_x, q.size_y, RTM_PRODUCT_SPLIT, RTM_FP32, 1, &h.op32));
        if (q.preconditioner == kPcBlockJacobi)
            RTM_TRY(rtm_preconditioner_create_block_jacobi(h.g, q.size_x, q.size_y, 2, 2, mixed ? RTM_FP32 : RTM_FP64,
                                                           &h.pc));
        else if (q.preconditioner == kPcCirculant)
            RTM_TRY(rtm_preconditioner_create(h.g, q.size_x, q.size_y, RTM_KERNEL_RCHAN, RTM_BUILDER_PARTWISE, nullptr,
                                              mixed ? RTM_FP32 : RTM_FP64, &h.pc));
        if (mixed && q.preconditioner == kPcBlockJacobi)
            RTM_TRY(rtm_preconditioner_create_block_jacobi(h.g, q.size_x, q.size_y, 2, 2, RTM_FP64, &h.pc64));
        else if (mixed && q.preconditioner == kPcCirculant)
            RTM_TRY(rtm_preconditioner_create(h.g, q.size_x, q.size_y, RTM_KERNEL_RCHAN, RTM_BUILDER_PARTWISE, nullptr,
                                              RTM_FP64, &h.pc64));
        h.n = h.op->op->n;
        h.s = h.op->stream;
        RTM_TRY(h.b.alloc((size_t)h.n * sizeof(double2)));
        RTM_TRY(h.x.alloc((size_t)h.n * sizeof(double2)));
        if (q.excitation == RTM_EXCITE_PLANE_WAVE) {
            const double one = 1.0;
            RTM_TRY(rtm_plane_wave(q.count_x, q.count_y, q.size_x, q.size_y, 8, q.wavenumber, q.direction,
                                   q.polarization, &one, 1, h.b.ptr, RTM_DEVICE, h.s));
        } else {
            RTM_TRY(middle_port(q.count_x, q.count_y, q.port_direction, h.port));
            RTM_TRY(rtm_delta_gap(q.count_x, q.count_y, q.size_x, q.size_y, h.port.data(), (int)h.port.size(), 0,
                                  q.voltage, h.b.ptr, RTM_DEVICE));
        }
        return RTM_OK;
    }

    SolveConfig solve_config(const Record& r) const {
        const rtm_request& q = r.req;
        SolveConfig sc;
        sc.method = q.method;
        sc.tolerance = q.tolerance;
        sc.max_iterations = q.max_iterations;
        sc.restart = q.restart;
        sc.right_preconditioned = 1;
        sc.cancel = &r.cancel;
        return sc;
    }

    // The stats of right-hand side k of a solve, the RCS or input impedance, and the current if kept.
    int finish(const rtm_request& q, Prepared& h, const SolveResult& res, int k, float solve_ms, Outcome& out) {
        out.res.unknowns = h.n;
        out.res.solve_s = solve_ms * 1e-3;
        if ((int)res.stats.size() > k) {
            out.res.converged = res.stats[k].converged;
            out.res.iteration_count = res.stats[k].iteration_count;
            out.res.residual_norm = res.stats[k].residual_norm;
        }
        if (q.excitation == RTM_EXCITE_PLANE_WAVE)
            RTM_TRY(rtm_radar_cross_section(q.wavenumber, h.b.ptr, h.x.ptr, h.n, 1.0, RTM_DEVICE, &out.res.rcs));
        else
            RTM_TRY(rtm_input_impedance(q.count_x, q.count_y, q.size_x, q.size_y, h.x.ptr, h.port.data(),
                                        (int)h.port.size(), q.voltage, RTM_DEVICE, out.res.impedance));
        if (q.keep_current) {
            out.current.resize((size_t)2 * h.n);
            RTM_CUDA(cudaMemcpyAsync(out.current.data(), h.x.ptr, (size_t)h.n * sizeof(double2), cudaMemcpyDeviceToHost,
                                     h.s));
            RTM_CUDA(cudaStreamSynchronize(h.s));
        }
        return RTM_OK;
    }

    // The whole pipeline of one request on this thread. Its results go to `out`, which the worker
    // copies into the record under the lock, so a concurrent poll never sees them half written.
    int run(const Record& r, Outcome& out) {
        const rtm_request& q = r.req;
        Prepared h;
        RTM_TRY(prepare(q, h));
        const cudaStream_t s = h.s;
        SolveConfig sc = solve_config(r);
        SolveResult res;
        cudaEvent_t e0, e1;
        RTM_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDefault));
        RTM_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDefault));
        cudaEventRecord(e0, s);
        int st;
        if (cfg.precision == RTM_FP32) {
            // FP32 inner solves of at most kInnerCap iterations inside FP64 refinement; a refinement step that does
            // not halve the FP64 residual (FP32 COCG can diverge on large plates: its short recurrence loses
            // accuracy in FP32) hands the solve to the FP64 method from the current iterate
            sc.inner_tolerance = 1e-4;
            sc.inner_max_iterations = kInnerCap;
            sc.fallback_fp64 = 1;
            st = solve_mixed(h.op->op.get(), h.op32->op.get(), h.pc ? h.pc->op.get() : nullptr, sc, h.b.ptr, nullptr,
                             h.x.ptr, h.n, 1, res, s, h.pc64 ? h.pc64->op.get() : nullptr);
        } else {
            st = solve(h.op->op.get(), h.pc ? h.pc->op.get() : nullptr, sc, h.b.ptr, nullptr, h.x.ptr, h.n, 1, res, s);
        }
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (st != RTM_OK) return st;
        return finish(q, h, res, 0, ms, out);
    }

    // Several requests of one batch key (batch_key) solved as one plate batch: each is prepared on its own,
    // then one solve takes them all, every right-hand side on its own tolerance, and each is finished.
    int run_batch(const std::vector<Record*>& rs, std::vector<Outcome>& outs) {
        const int count = (int)rs.size();
        std::vector<std::unique_ptr<Prepared>> hs;
        for (Record* r : rs) {
            hs.push_back(std::make_unique<Prepared>());
            RTM_TRY(prepare(r->req, *hs.back()));
        }
        for (auto& h : hs) RTM_CUDA(cudaStreamSynchronize(h->s));
        std::vector<LinearOp*> ops, pcs;
        int64_t stride = 0;
        for (auto& h : hs) {
            ops.push_back(h->op->op.get());
            if (h->pc) pcs.push_back(h->pc->op.get());
            stride = std::max(stride, h->n);
        }
        const cudaStream_t s = hs[0]->s;
        int st = RTM_OK;
        std::unique_ptr<BatchOp> A = make_batch(ops, stride, true, s, &st), M;
        RTM_TRY(st);
        if (!pcs.empty()) {
            M = make_batch(pcs, stride, true, s, &st);
            RTM_TRY(st);
        }
        const size_t vec = (size_t)stride * sizeof(double2);
        DeviceBuffer b, x;
        StreamSyncGuard guard(s);
        RTM_TRY(b.alloc(vec * count));
        RTM_TRY(x.alloc(vec * count));
        RTM_CUDA(cudaMemsetAsync(b.ptr, 0, b.bytes, s));
        for (int k = 0; k < count; ++k)
            RTM_CUDA(cudaMemcpyAsync(b.as<double2>() + k * stride, hs[k]->b.ptr, hs[k]->n * sizeof(double2),
                                     cudaMemcpyDeviceToDevice, s));
        SolveConfig sc = solve_config(*rs[0]);
        std::vector<double> tol(count);
        for (int k = 0; k < count; ++k) tol[k] = rs[k]->req.tolerance;
        sc.tolerances = tol.data();
        // a request cancelled while its batch runs is discarded when the batch ends; the batch itself stops
        // at its next host check when the server stops
        sc.cancel = &stop_flag;
        SolveResult res;
        cudaEvent_t e0, e1;
        RTM_CUDA(cudaEventCreateWithFlags(&e0, cudaEventDefault));
        RTM_CUDA(cudaEventCreateWithFlags(&e1, cudaEventDefault));
        cudaEventRecord(e0, s);
        st = solve(A.get(), M.get(), sc, b.ptr, nullptr, x.ptr, stride, count, res, s);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        RTM_TRY(st);
        for (int k = 0; k < count; ++k)
            RTM_CUDA(cudaMemcpyAsync(hs[k]->x.ptr, x.as<double2>() + k * stride, hs[k]->n * sizeof(double2),
                                     cudaMemcpyDeviceToDevice, s));
        RTM_CUDA(cudaStreamSynchronize(s));
        for (int k = 0; k < count; ++k) RTM_TRY(finish(rs[k]->req, *hs[k], res, k, ms, outs[k]));
        return RTM_OK;
    }
};

extern "C" {

int rtm_server_create(const rtm_server_config* config, rtm_server** out) {
    if (!out) return fail(RTM_ERR_ARG, "null argument");
    *out = nullptr;
    auto srv = std::make_unique<rtm_server>();
    if (config) srv->cfg = *config;
    if (!(srv->cfg.budget_bytes > 0)) srv->cfg.budget_bytes = 150e9;
    if (srv->cfg.max_active <= 0) srv->cfg.max_active = 8;
    if (srv->cfg.precision != RTM_FP64 && srv->cfg.precision != RTM_FP32)
        return fail(RTM_ERR_ARG, "precision must be RTM_FP64 or RTM_FP32");
    if (srv->cfg.max_active > 256) return fail(RTM_ERR_ARG, "at most 256 active requests");
    if (srv->cfg.transform_sizes < RTM_SIZES_REFERENCE || srv->cfg.transform_sizes > RTM_SIZES_AUTOTUNE)
        return fail(RTM_ERR_ARG, "unknown transform size policy");
    if (srv->cfg.max_batch < 0 || srv->cfg.max_batch > 256) return fail(RTM_ERR_ARG, "max_batch lies in 0..256");
    srv->epoch = Clock::now();
    rtm_server* p = srv.get();
    // with batches, a worker takes up to max_batch admitted requests at once
    const int workers = srv->cfg.max_batch > 1 ? std::max(1, srv->cfg.max_active / srv->cfg.max_batch)
                                               : srv->cfg.max_active;
    for (int i = 0; i < workers; ++i) srv->workers.emplace_back([p] { p->worker(); });
    *out = srv.release();
    return RTM_OK;
}

int rtm_server_submit(rtm_server* srv, const rtm_request* request, uint64_t* id) {
    if (!srv || !request || !id) return fail(RTM_ERR_ARG, "null argument");
    RTM_TRY(check_request(*request));
    auto rec = std::make_unique<Record>();
    rec->req = *request;
    RTM_TRY(request_bytes(*request, srv->cfg.precision, srv->cfg.transform_sizes, &rec->res.bytes));
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return fail(RTM_ERR_ARG, "the server is stopping");
    rec->id = srv->next_id++;
    rec->res.submitted_s = seconds_since(srv->epoch);
    *id = rec->id;
    if (rec->res.bytes > srv->cfg.budget_bytes) {
        rec->res.state = RTM_REQUEST_FAILED;
        rec->res.status = RTM_ERR_OOM_BUDGET;
        rec->res.finished_s = rec->res.submitted_s;
        srv->records.emplace(rec->id, std::move(rec));
        srv->done_cv.notify_all();
        return RTM_OK;
    }
    rec->res.state = RTM_REQUEST_QUEUED;
    srv->queue.push_back(rec->id);
    srv->records.emplace(rec->id, std::move(rec));
    srv->admit_locked();
    return RTM_OK;
}

int rtm_server_poll(rtm_server* srv, uint64_t id, int wait_ms, rtm_request_result* out, double* current, int64_t n,
                    int release) {
    if (!srv || !out) return fail(RTM_ERR_ARG, "null argument");
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->records.find(id);
    if (it == srv->records.end()) return fail(RTM_ERR_ARG, "unknown request " + std::to_string(id));
    Record* r = it->second.get();
    auto finished = [&] { return r->res.state >= RTM_REQUEST_DONE; };
    if (wait_ms < 0) srv->done_cv.wait(lk, finished);
    else if (wait_ms > 0) srv->done_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), finished);
    *out = r->res;
    if (current && finished() && !r->current.empty()) {
        if ((int64_t)r->current.size() != 2 * n)
            return fail(RTM_ERR_SIZE, "The request has " + std::to_string(r->current.size() / 2) + " unknowns.");
        std::memcpy(current, r->current.data(), r->current.size() * sizeof(double));
    }
    if (release && finished()) srv->records.erase(it);
    return RTM_OK;
}

int rtm_server_cancel(rtm_server* srv, uint64_t id) {
    if (!srv) return fail(RTM_ERR_ARG, "null argument");
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->records.find(id);
    if (it == srv->records.end()) return fail(RTM_ERR_ARG, "unknown request " + std::to_string(id));
    Record* r = it->second.get();
    r->cancel = 1;
    if (r->res.state == RTM_REQUEST_QUEUED) {
        for (auto q = srv->queue.begin(); q != srv->queue.end(); ++q)
            if (*q == id) {
                srv->queue.erase(q);
                r->res.state = RTM_REQUEST_CANCELLED;
                r->res.finished_s = seconds_since(srv->epoch);
                srv->done_cv.notify_all();
                break;
            }
    }
    return RTM_OK;
}

int rtm_server_destroy(rtm_server* srv) {
    if (!srv) return RTM_OK;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
        srv->stop_flag = 1;
        for (uint64_t id : srv->queue) {
            Record& r = *srv->records.at(id);
            r.res.state = RTM_REQUEST_CANCELLED;
            r.res.finished_s = seconds_since(srv->epoch);
        }
        srv->queue.clear();
        for (auto& kv : srv->records) kv.second->cancel = 1;
    }
    srv->work_cv.notify_all();
    for (auto& t : srv->workers) t.join();
    delete srv;
    return RTM_OK;
}

}  // extern "C"
