// COCG, preconditioned COCG and restarted left-preconditioned GMRES on the device.
//
// Follows the reference's
//   src/+rooftopMoM/+solver/IterativeMethod.m:27-70        (zero right-hand side, true residual)
//   src/+rooftopMoM/+solver/ConjugateGradient.m:12-62       (COCG: r^T z, alpha = rho / d^T A d)
//   src/+rooftopMoM/+solver/PreconditionedConjugateGradient.m:18-23
//   src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/iterate_.m:1-85
//   src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/private/orthogonalize_.m:15-23 (CGS2)
//   src/+rooftopMoM/+solver/@GeneralizedMinimumResidual/private/generateRotation_.m:11-18
//
// Every scalar of an iteration lives on the device. Each reduction is one kernel whose last CTA to
// arrive (atomic counter, no waiting) sums the per-CTA partials in a fixed order and updates the
// solver state, so results do not depend on scheduling. Every kernel of an iteration first reads
// the state of its right-hand side and does nothing once that solve is done; the host launches
// `check_every` iterations, then reads the done flags once. Converged systems thus stop exactly at
// the reference's iteration, and the extra launched iterations are no-ops.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "fft.cuh"
#include "krylov.h"

namespace rtm {

constexpr int kRT = 256;  // threads of the vector kernels
static int reduce_blocks(int64_t n);

__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2(v.x, v.y); }
template <typename T2> __device__ __forceinline__ T2 from_d2(double2 v);
template <> __device__ __forceinline__ double2 from_d2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 from_d2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double2 dmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ double2 dmulc(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 ddiv(double2 a, double2 b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double dabs(double2 a) { return hypot(a.x, a.y); }

// Sums K double2 values over the CTA into out[0..K-1] (thread 0..K-1 write).
template <int K> __device__ __forceinline__ void block_sum(double2 (&v)[K], double2* out) {
    __shared__ double2 sm[K][kRT / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double r = v[k].x, i = v[k].y;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
            i += __shfl_down_sync(0xffffffffu, i, o);
        }
        if (lane == 0) sm[k][warp] = make_double2(r, i);
    }
    __syncthreads();
    if (threadIdx.x < K) {
        double2 s = make_double2(0, 0);
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s = dadd(s, sm[threadIdx.x][w]);
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// Returns true in the last CTA of this right-hand side to arrive; its partials are then visible.
__device__ __forceinline__ bool arrive(unsigned int* counter) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned int prev = atomicAdd(counter, 1u);
        last = prev == gridDim.x - 1;
        if (last) *counter = 0;  // ready for the next reduction
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

// Sum of nb partials by the whole CTA in a fixed order (every thread gets the total).
__device__ __forceinline__ double2 cta_total(const double2* p, int nb) {
    __shared__ double2 total;
    double2 v[1] = {make_double2(0, 0)};
    for (int b = threadIdx.x; b < nb; b += blockDim.x) v[0] = dadd(v[0], p[b]);
    block_sum<1>(v, &total);
    return total;
}

// ============================================================================================
// COCG
struct CgState {
    double2 rho, beta, alpha;
    double bnorm, tol;
    int iteration, max_iterations;
    int done;        // nonzero: this solve is finished (also the operators' skip flag)
    int converged;
    int zero_rhs;
    unsigned int counter;
};

template <typename T2>
__global__ void __launch_bounds__(kRT) k_cg_start(const T2* __restrict__ b, const T2* __restrict__ r, int64_t n,
                                                  CgState* st, double2* part, double* hist, int hist_stride) {
    const int rhs = blockIdx.y;
    const T2* br = b + rhs * n;
    const T2* rr = r + rhs * n;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 bv = to_d2(br[i]), rv = to_d2(rr[i]);
        acc[0].x += bv.x * bv.x + bv.y * bv.y;
        acc[0].y += rv.x * rv.x + rv.y * rv.y;
    }
    double2* mine = part + ((int64_t)rhs * gridDim.x + blockIdx.x);
    block_sum<1>(acc, mine);
    if (!arrive(&st[rhs].counter)) return;
    const double2 s = cta_total(part + (int64_t)rhs * gridDim.x, gridDim.x);
    if (threadIdx.x == 0) {
        CgState& S = st[rhs];
        S.bnorm = sqrt(s.x);
        S.iteration = 0;
        S.rho = S.beta = S.alpha = make_double2(0, 0);
        if (S.bnorm == 0.0) {
            // IterativeMethod.m:53-56: the solution of a zero right-hand side is zero.
            S.zero_rhs = 1;
            S.converged = 1;
            S.done = 1;
            hist[(int64_t)rhs * hist_stride] = 0.0;
            return;
        }
        S.zero_rhs = 0;
        const double h0 = sqrt(s.y) / S.bnorm;
        hist[(int64_t)rhs * hist_stride] = h0;
        S.converged = h0 < S.tol;
        S.done = S.converged || S.max_iterations <= 0;
    }
}

// rho = r^T z (no conjugate); beta = rho / rho_previous from the second iteration on.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_cg_rz(const T2* __restrict__ r, const T2* __restrict__ z, int64_t n,
                                               CgState* st, double2* part) {
    const int rhs = blockIdx.y;
    if (st[rhs].done) return;
    const T2* rr = r + rhs * n;
    const T2* zr = z + rhs * n;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] = dadd(acc[0], dmul(to_d2(rr[i]), to_d2(zr[i])));
    block_sum<1>(acc, part + ((int64_t)rhs * gridDim.x + blockIdx.x));
    if (!arrive(&st[rhs].counter)) return;
    const double2 s = cta_total(part + (int64_t)rhs * gridDim.x, gridDim.x);
    if (threadIdx.x == 0) {
        CgState& S = st[rhs];
        S.beta = S.iteration == 0 ? make_double2(0, 0) : ddiv(s, S.rho);
        S.rho = s;
    }
}

// d = z + beta d (d = z in the first iteration).
template <typename T2>
__global__ void __launch_bounds__(kRT) k_cg_dir(const T2* __restrict__ z, T2* __restrict__ d, int64_t n,
                                                const CgState* st) {
    const int rhs = blockIdx.y;
    const CgState& S = st[rhs];
    if (S.done) return;
    const T2* zr = z + rhs * n;
    T2* dr = d + rhs * n;
    const bool first = S.iteration == 0;
    const double2 beta = S.beta;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 zv = to_d2(zr[i]);
        dr[i] = first ? zr[i] : from_d2<T2>(dadd(zv, dmul(beta, to_d2(dr[i]))));
    }
}

// alpha = rho / (d^T q).
template <typename T2>
__global__ void __launch_bounds__(kRT) k_cg_dq(const T2* __restrict__ d, const T2* __restrict__ q, int64_t n,
                                               CgState* st, double2* part) {
    const int rhs = blockIdx.y;
    if (st[rhs].done) return;
    const T2* dr = d + rhs * n;
    const T2* qr = q + rhs * n;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        acc[0] = dadd(acc[0], dmul(to_d2(dr[i]), to_d2(qr[i])));
    block_sum<1>(acc, part + ((int64_t)rhs * gridDim.x + blockIdx.x));
    if (!arrive(&st[rhs].counter)) return;
    const double2 s = cta_total(part + (int64_t)rhs * gridDim.x, gridDim.x);
    if (threadIdx.x == 0) st[rhs].alpha = ddiv(st[rhs].rho, s);
}

// x += alpha d, r -= alpha q, then the relative residual, the history and the stopping tests.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_cg_update(T2* __restrict__ x, T2* __restrict__ r, const T2* __restrict__ d,
                                                   const T2* __restrict__ q, int64_t n, CgState* st, double2* part,
                                                   double* hist, int hist_stride) {
    const int rhs = blockIdx.y;
    if (st[rhs].done) return;
    const double2 alpha = st[rhs].alpha;
    T2* xr = x + rhs * n;
    T2* rr = r + rhs * n;
    const T2* dr = d + rhs * n;
    const T2* qr = q + rhs * n;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 xv = dadd(to_d2(xr[i]), dmul(alpha, to_d2(dr[i])));
        const double2 aq = dmul(alpha, to_d2(qr[i]));
        const double2 rv0 = to_d2(rr[i]);
        const double2 rv = make_double2(rv0.x - aq.x, rv0.y - aq.y);
        const T2 rs = from_d2<T2>(rv);
        xr[i] = from_d2<T2>(xv);
        rr[i] = rs;
        const double2 rd = to_d2(rs);
        acc[0].x += rd.x * rd.x + rd.y * rd.y;
    }
    block_sum<1>(acc, part + ((int64_t)rhs * gridDim.x + blockIdx.x));
    if (!arrive(&st[rhs].counter)) return;
    const double s = cta_total(part + (int64_t)rhs * gridDim.x, gridDim.x).x;
    if (threadIdx.x == 0) {
        CgState& S = st[rhs];
        S.iteration += 1;
        const double h = sqrt(s) / S.bnorm;
        hist[(int64_t)rhs * hist_stride + S.iteration] = h;
        S.converged = h < S.tol;
        // A breakdown (d^T A d = 0) leaves Inf or NaN (ConjugateGradient.m:55-58).
        S.done = S.converged || !isfinite(h) || S.iteration >= S.max_iterations;
    }
}

// ============================================================================================
// GMRES
struct GmState {
    double ref;       // || P b ||
    double rn;        // norm of the residual a cycle starts from
    double tol;
    double inv_sub;
    int iteration, max_iterations, m, step;
    int active;       // inside a cycle
    int skip_step;    // = !active: the operators' skip flag within a cycle
    int done;         // converged or out of iterations: the skip flag of the restart
    int converged;
    int zero_rhs;
    int cycle_ran;
    int skip_update;  // = !cycle_ran: the preconditioner's skip flag for the right-preconditioned update
    unsigned int counter;
};

struct GmArrays {
    double2* H;      // [rhs][(m+1) * m], column-major
    double2* g;      // [rhs][m+1]
    double2* cs;     // [rhs][m]
    double2* sn;     // [rhs][m]
    double2* h;      // [rhs][m+1] accumulated Gram-Schmidt coefficients
    double2* c;      // [rhs][m+1] coefficients of the current pass
    double2* y;      // [rhs][m]
    double2* part;   // [rhs][blocks][m+1]
    double* hist;
    int hist_stride;
    int m;
};

// ||w||: mode 0 sets ref = ||P b||; mode 1 starts a cycle from w (first: the history's first entry).
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_norm(const T2* __restrict__ w, int64_t n, GmState* st, GmArrays ar,
                                                 int mode, int first) {
    const int rhs = blockIdx.y;
    GmState& S = st[rhs];
    if (mode == 1 && S.done) return;
    const T2* wr = w + rhs * n;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = to_d2(wr[i]);
        acc[0].x += v.x * v.x + v.y * v.y;
    }
    double2* part = ar.part + (int64_t)rhs * gridDim.x * (ar.m + 1);
    block_sum<1>(acc, part + blockIdx.x);
    if (!arrive(&S.counter)) return;
    const double s = cta_total(part, gridDim.x).x;
    if (threadIdx.x == 0) {
        const double nrm = sqrt(s);
        if (mode == 0) {
            S.ref = nrm;
            S.iteration = 0;
            S.zero_rhs = nrm == 0.0;
            S.done = S.zero_rhs;
            S.converged = S.zero_rhs;
            S.active = 0;
            S.skip_step = 1;
            if (S.zero_rhs) ar.hist[(int64_t)rhs * ar.hist_stride] = 0.0;
            return;
        }
        S.rn = nrm;
        if (first) {
            const double h0 = nrm / S.ref;
            ar.hist[(int64_t)rhs * ar.hist_stride] = h0;
            S.converged = h0 < S.tol;
            S.done = S.converged || S.max_iterations <= 0;
        }
        double2* g = ar.g + (int64_t)rhs * (ar.m + 1);
        for (int k = 0; k <= ar.m; ++k) g[k] = make_double2(0, 0);
        g[0] = make_double2(nrm, 0);
        S.step = 0;
        S.active = !S.done;
        S.skip_step = !S.active;
        S.cycle_ran = S.active;
        S.skip_update = !S.cycle_ran;
    }
}

// V[:, 0] = w / rn.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_v0(const T2* __restrict__ w, T2* __restrict__ V, int64_t n, int nrhs,
                                               const GmState* st) {
    const int rhs = blockIdx.y;
    const GmState& S = st[rhs];
    if (!S.active) return;
    const double inv = 1.0 / S.rn;
    const T2* wr = w + rhs * n;
    T2* v0 = V + (int64_t)rhs * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = to_d2(wr[i]);
        v0[i] = from_d2<T2>(make_double2(v.x * inv, v.y * inv));
    }
}

// The rest of an Arnoldi step once ||w|| is known: the Hessenberg column, its previous rotations,
// the new rotation, the rotated right-hand side, the history and the stopping tests (one thread).
// col, cs, sn: the Hessenberg column being formed and the rotations, in global memory or staged in
// shared memory by the caller with col already holding h (the rotation chain is sequential; staged, each
// step costs a shared-memory access instead of a global one).
__device__ void arnoldi_finish(GmState& S, GmArrays& ar, int rhs, double s, double2* col, double2* cs, double2* sn,
                               bool staged) {
    const double sub = sqrt(s);
    const int m = ar.m, j = S.step;
    double2* g = ar.g + (int64_t)rhs * (m + 1);
    const double2* h = ar.h + (int64_t)rhs * (m + 1);
    if (!staged)
        for (int k = 0; k <= j; ++k) col[k] = h[k];
    col[j + 1] = make_double2(sub, 0);
    for (int k = 0; k < j; ++k) {
        const double2 a0 = col[k], a1 = col[k + 1];
        col[k] = dadd(dmulc(cs[k], a0), dmulc(sn[k], a1));
        const double2 t = dmul(sn[k], a0);
        const double2 u = dmul(cs[k], a1);
        col[k + 1] = make_double2(u.x - t.x, u.y - t.y);
    }
    // generateRotation_.m:11-18
    const double2 a = col[j], bsub = col[j + 1];
    const double radius = sqrt(a.x * a.x + a.y * a.y + bsub.x * bsub.x + bsub.y * bsub.y);
    double2 cj = make_double2(1, 0), sj = make_double2(0, 0);
    if (radius > 0) {
        cj = make_double2(a.x / radius, a.y / radius);
        sj = make_double2(bsub.x / radius, bsub.y / radius);
    }
    cs[j] = cj;
    sn[j] = sj;
    col[j] = dadd(dmulc(cj, a), dmulc(sj, bsub));
    col[j + 1] = make_double2(0, 0);
    const double2 gj = g[j];
    const double2 t = dmul(sj, gj);
    g[j + 1] = make_double2(-t.x, -t.y);
    g[j] = dmulc(cj, gj);
    S.iteration += 1;
    const double hres = dabs(g[j + 1]) / S.ref;
    ar.hist[(int64_t)rhs * ar.hist_stride + S.iteration] = hres;
    S.converged = hres < S.tol;
    S.step = j + 1;
    S.inv_sub = sub != 0 ? 1.0 / sub : 0.0;
    const bool more = !S.converged && sub != 0 && S.step < m && S.iteration < S.max_iterations;
    // A zero subdiagonal means the basis spans the solution (iterate_.m:65-68).
    S.active = more;
    S.skip_step = !more;
    S.done = S.converged || S.iteration >= S.max_iterations;
}

// Asynchronous global -> shared copies (cp.async, sm_80 and later): a thread issues all the copies
// of a tile without waiting, then waits for its groups before the CTA barrier.
template <int BYTES> __device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    if constexpr (BYTES == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

// One pass of the classical Gram-Schmidt run twice (orthogonalize_.m:15-23) over tiles of TR rows:
//   mode 0: c = V^H w                       (h = c)
//   mode 1: w -= V h, then c = V^H w        (h += c)
//   mode 2: w -= V c, then ||w|| and the end of the Arnoldi step.
// Every CTA streams its tiles of the basis (columns 0..step) and of w through two shared buffers
// with asynchronous copies: the next tile is in flight while the current one is reduced, and each
// pass reads the basis once. Column partials accumulate in shared memory over the CTA's tiles; the
// last CTA sums the per-CTA partials in a fixed order.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_orth(const T2* __restrict__ V, T2* __restrict__ w, int64_t n, int nrhs,
                                                 GmState* st, GmArrays ar, int mode, int TR) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int rhs = blockIdx.y;
    GmState& S = st[rhs];
    if (!S.active) return;
    const int cols = S.step + 1;
    const int ld = TR + 1;
    const int mc = ar.m + 1;
    double2* colacc = reinterpret_cast<double2*>(smem_raw);  // [m + 1]
    double2* coef = colacc + mc;                               // [m + 1]
    double2* scratch = coef + mc;                              // [max(kRT, m + 1)]
    T2* wsb = reinterpret_cast<T2*>(scratch + (kRT > mc ? kRT : mc));  // [2][TR]
    T2* Vsb = wsb + 2 * TR;                                    // [2][m + 1][ld]
    const double2* cf = mode == 1 ? ar.h + (int64_t)rhs * mc : ar.c + (int64_t)rhs * mc;
    for (int k = threadIdx.x; k < cols; k += blockDim.x) {
        colacc[k] = make_double2(0, 0);
        if (mode) coef[k] = cf[k];
    }
    const int G = kRT / cols > 0 ? kRT / cols : 1;  // row groups of the column sums
    T2* wr = w + rhs * n;
    double nrm = 0;
    const int64_t tiles = (n + TR - 1) / TR;
    const T2 zero = from_d2<T2>(make_double2(0, 0));
    auto stage = [&](int64_t tile, int buf) {
        const int64_t r0 = tile * TR;
        T2* Vs = Vsb + (size_t)buf * mc * ld;
        T2* ws = wsb + (size_t)buf * TR;
        for (int t = threadIdx.x; t < cols * TR; t += blockDim.x) {
            const int k = t / TR, r = t - k * TR;
            const int64_t row = r0 + r;
            if (row < n) cp_async<sizeof(T2)>(&Vs[k * ld + r], &V[((int64_t)k * nrhs + rhs) * n + row]);
            else Vs[k * ld + r] = zero;
        }
        for (int r = threadIdx.x; r < TR; r += blockDim.x) {
            const int64_t row = r0 + r;
            if (row < n) cp_async<sizeof(T2)>(&ws[r], &wr[row]);
            else ws[r] = zero;
        }
        cp_async_commit();
    };
    int buf = 0;
    if ((int64_t)blockIdx.x < tiles) stage(blockIdx.x, 0);
    for (int64_t tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int64_t next = tile + gridDim.x;
        if (next < tiles) {
            stage(next, buf ^ 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();  // this tile's copies (and coef, colacc) are visible
        const int64_t r0 = tile * TR;
        T2* Vs = Vsb + (size_t)buf * mc * ld;
        T2* ws = wsb + (size_t)buf * TR;
        if (mode) {
            for (int r = threadIdx.x; r < TR; r += blockDim.x) {
                double2 v = to_d2(ws[r]);
                for (int k = 0; k < cols; ++k) {
                    const double2 p = dmul(to_d2(Vs[k * ld + r]), coef[k]);
                    v.x -= p.x;
                    v.y -= p.y;
                }
                const T2 vs = from_d2<T2>(v);
                ws[r] = vs;
                const int64_t row = r0 + r;
                if (row < n) {
                    wr[row] = vs;
                    const double2 vd = to_d2(vs);
                    nrm += vd.x * vd.x + vd.y * vd.y;
                }
            }
            __syncthreads();
        }
        if (mode < 2) {
            for (int t = threadIdx.x; t < cols * G; t += blockDim.x) {
                const int k = t % cols, g = t / cols;
                double2 acc = make_double2(0, 0);
                for (int r = g; r < TR; r += G) acc = dadd(acc, dmulc(to_d2(Vs[k * ld + r]), to_d2(ws[r])));
                scratch[t] = acc;
            }
            __syncthreads();
            for (int k = threadIdx.x; k < cols; k += blockDim.x) {
                double2 acc = colacc[k];
                for (int g = 0; g < G; ++g) acc = dadd(acc, scratch[k + g * cols]);
                colacc[k] = acc;
            }
        }
        __syncthreads();  // the buffer is free for the stage after next
        buf ^= 1;
    }
    double2* part = ar.part + (int64_t)rhs * gridDim.x * mc;
    if (mode < 2) {
        for (int k = threadIdx.x; k < cols; k += blockDim.x) part[(int64_t)k * gridDim.x + blockIdx.x] = colacc[k];
    } else {
        double2 v[1] = {make_double2(nrm, 0)};
        block_sum<1>(v, part + blockIdx.x);
    }
    if (!arrive(&S.counter)) return;
    if (mode == 2) {
        const double tot = cta_total(part, gridDim.x).x;
        if (threadIdx.x == 0) {
            const int m = ar.m;
            arnoldi_finish(S, ar, rhs, tot, ar.H + ((int64_t)rhs * m + S.step) * (m + 1), ar.cs + (int64_t)rhs * m,
                           ar.sn + (int64_t)rhs * m, false);
        }
        return;
    }
    // One warp per column: lanes sum strided partials, then a shuffle tree (fixed order).
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = warp; k < cols; k += nw) {
        double2 v = make_double2(0, 0);
        const double2* pk = part + (int64_t)k * gridDim.x;
        for (int b = lane; b < (int)gridDim.x; b += 32) v = dadd(v, pk[b]);
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_down_sync(0xffffffffu, v.x, o);
            v.y += __shfl_down_sync(0xffffffffu, v.y, o);
        }
        if (lane == 0) {
            double2* h = ar.h + (int64_t)rhs * mc;
            ar.c[(int64_t)rhs * mc + k] = v;
            h[k] = mode == 0 ? v : dadd(h[k], v);
        }
    }
}

constexpr int kOrthSmemMax = 200 * 1024;  // dynamic shared memory k_gm_orth may take

// Rows per tile and shared bytes of k_gm_orth (two buffers) for a basis of up to m + 1 columns.
template <typename T2> static void orth_config(int m, int* TR, size_t* smem) {
    const size_t fixed = (size_t)(2 * (m + 1) + std::max(kRT, m + 1)) * sizeof(double2);
    auto bytes = [&](int tr) { return fixed + 2 * ((size_t)tr + (size_t)(m + 1) * (tr + 1)) * sizeof(T2); };
    int tr = 128;
    while (tr > 16 && bytes(tr) > 100 * 1024) tr -= 16;
    *TR = tr;
    *smem = bytes(tr);
}

// --------------------------------------------------------------------------------------------
// The same three passes, streamed from global memory with no per-tile barriers. Each CTA owns one
// contiguous chunk of rows. The update w -= V c runs one thread per row, loading eight basis entries
// before using them (coalesced across the warp), in the column order of k_gm_orth. The dots run one
// warp per column: lanes stride the chunk's rows and keep the column's sum in registers until the
// chunk ends; the chunk of w sits in shared memory. With fewer columns than warps, the rows of a
// column are split between warps. Mode 1 reads the basis twice (the second read mostly from L2).
// Serves bases of up to kStreamCols columns.
constexpr int kStreamCols = 64;
constexpr int kStreamRows = 3072;  // rows per CTA chunk the launcher aims at (bounds the shared w chunk)

// Arithmetic type of the Gram-Schmidt passes: a basis kept in FP32 (the precision form's inner solves) is
// updated and multiplied in FP32, with the sums over lanes, CTAs and chunks in FP64; an FP64 basis in FP64.
// (Converting every FP32 element to FP64 made the FP32 passes slower than the FP64 ones.)
template <typename T2> struct OrthAcc { using type = double2; };
template <> struct OrthAcc<float2> { using type = float2; };
__device__ __forceinline__ double2 amul(double2 a, double2 b) { return dmul(a, b); }
__device__ __forceinline__ float2 amul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 amulc(double2 a, double2 b) { return dmulc(a, b); }
__device__ __forceinline__ float2 amulc(float2 a, float2 b) {  // conj(a) * b
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}

// RL consecutive rows of one basis column, read with one load where RL = 2 (two FP32 complex values in 16
// bytes): FP32 threads then keep as many bytes in flight as FP64 ones, which the passes' throughput
// follows (they are bound by the memory requests in flight, not by arithmetic).
template <typename T2, int RL> struct RowPack {
    T2 v[RL];
};
template <typename T2, int RL>
__device__ __forceinline__ RowPack<T2, RL> load_rows(const T2* __restrict__ p, int valid) {
    RowPack<T2, RL> r;
    if constexpr (RL == 2) {
        if (valid == 2) {
            const float4 f = *reinterpret_cast<const float4*>(p);
            r.v[0] = make_float2(f.x, f.y);
            r.v[1] = make_float2(f.z, f.w);
            return r;
        }
    }
#pragma unroll
    for (int q = 0; q < RL; ++q) r.v[q] = q < valid ? p[q] : from_d2<T2>(make_double2(0, 0));
    return r;
}

// KQE: the basis columns a warp takes at once in the dots (1, 2, 4 or 8; the launcher picks the fewest that
// cover the step's columns); each lane then keeps KQ / KQE groups of rows in flight, so a dot pass over few
// columns takes as many loads per round as one over many, in fewer rounds.
template <typename T2, int RL, int KQE>
__global__ void __launch_bounds__(kRT, 2) k_gm_orth_stream(const T2* __restrict__ V, T2* __restrict__ w, int64_t n,
                                                           int nrhs, GmState* st, GmArrays ar, int mode, int chunk) {
    // (two-row FP32 loads over one or two columns hold half the groups: the registers of two CTAs an SM
    // spill otherwise)
    constexpr int NW = kRT / 32, KQ = kStreamCols / NW, RU = (RL == 2 && KQE <= 2) ? KQ / KQE / 2 : KQ / KQE;
    using A2 = typename OrthAcc<T2>::type;  // arithmetic of the passes: FP64 for an FP64 basis, FP32 for FP32
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ A2 coef[kStreamCols];
    __shared__ double2 red[NW][KQ];
    T2* ws = reinterpret_cast<T2*>(smem_raw);  // [chunk]
    const int rhs = blockIdx.y;
    GmState& S = st[rhs];
    if (!S.active) return;
    const int cols = S.step + 1;
    const int mc = ar.m + 1;
    const int64_t c0 = (int64_t)blockIdx.x * chunk < n ? (int64_t)blockIdx.x * chunk : n;
    const int len = (int)(n - c0 < (int64_t)chunk ? n - c0 : (int64_t)chunk);
    const double2* cf = mode == 1 ? ar.h + (int64_t)rhs * mc : ar.c + (int64_t)rhs * mc;
    for (int k = threadIdx.x; k < cols; k += kRT) coef[k] = from_d2<A2>(mode ? cf[k] : make_double2(0, 0));
    T2* wr = w + (int64_t)rhs * n + c0;
    const T2* Vr = V + (int64_t)rhs * n + c0;        // column k at Vr + k * col
    const int64_t col = (int64_t)nrhs * n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double nrm = 0;
    __syncthreads();  // coef
    if (mode) {
        // two groups of RL rows a thread at once (r and r + RL kRT): twice the loads in flight per batch
        // of columns; every row takes its columns in order, as in k_gm_orth
        for (int r = RL * threadIdx.x; r < len; r += 2 * RL * kRT) {
            const int r2 = r + RL * kRT;
            const int n0 = min(RL, len - r), n1 = max(0, min(RL, len - r2));
            A2 v[RL], v2[RL];
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                v[q] = q < n0 ? wr[r + q] : from_d2<A2>(make_double2(0, 0));
                v2[q] = q < n1 ? wr[r2 + q] : from_d2<A2>(make_double2(0, 0));
            }
            constexpr int UB = 8;  // columns a batch: 16-byte loads, the same bytes in flight for every RL
            int k = 0;
            for (; k + UB <= cols; k += UB) {
                RowPack<T2, RL> t[UB], t2[UB];
#pragma unroll
                for (int u = 0; u < UB; ++u) {
                    t[u] = load_rows<T2, RL>(Vr + (k + u) * col + r, n0);
                    t2[u] = load_rows<T2, RL>(Vr + (k + u) * col + r2, n1);
                }
#pragma unroll
                for (int u = 0; u < UB; ++u)
#pragma unroll
                    for (int q = 0; q < RL; ++q) {
                        const A2 p = amul(t[u].v[q], coef[k + u]);
                        v[q].x -= p.x;
                        v[q].y -= p.y;
                        const A2 p2 = amul(t2[u].v[q], coef[k + u]);
                        v2[q].x -= p2.x;
                        v2[q].y -= p2.y;
                    }
            }
            for (; k < cols; ++k) {
                const RowPack<T2, RL> t = load_rows<T2, RL>(Vr + k * col + r, n0);
                const RowPack<T2, RL> t2 = load_rows<T2, RL>(Vr + k * col + r2, n1);
#pragma unroll
                for (int q = 0; q < RL; ++q) {
                    const A2 p = amul(t.v[q], coef[k]);
                    v[q].x -= p.x;
                    v[q].y -= p.y;
                    const A2 p2 = amul(t2.v[q], coef[k]);
                    v2[q].x -= p2.x;
                    v2[q].y -= p2.y;
                }
            }
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                if (q < n0) {
                    const T2 vs = v[q];
                    wr[r + q] = vs;
                    if (mode == 1) ws[r + q] = vs;
                    const double2 vd = to_d2(vs);
                    nrm += vd.x * vd.x + vd.y * vd.y;
                }
                if (q < n1) {
                    const T2 vs2 = v2[q];
                    wr[r2 + q] = vs2;
                    if (mode == 1) ws[r2 + q] = vs2;
                    const double2 vd2 = to_d2(vs2);
                    nrm += vd2.x * vd2.x + vd2.y * vd2.y;
                }
            }
        }
    } else {
        for (int r = threadIdx.x; r < len; r += kRT) ws[r] = wr[r];
    }
    double2* part = ar.part + (int64_t)rhs * gridDim.x * mc;
    if (mode < 2) {
        __syncthreads();  // the chunk of w
        const bool wide = cols >= NW;
        const int G = wide ? 1 : NW / cols;  // warps per column
        const bool on = wide || warp < G * cols;
        const int kw = wide ? warp : warp % cols;
        const int slice = wide ? 0 : warp / cols;
        // slices start on multiples of RL (the packed loads' alignment)
        const int rs = (int)((int64_t)len * slice / G) / RL * RL;
        const int re = slice + 1 == G ? len : (int)((int64_t)len * (slice + 1) / G) / RL * RL;
        // groups of KQE columns (one group when the launcher's KQE covers the step's columns)
        for (int q0 = 0; q0 < KQ; q0 += KQE) {
            if (q0 > 0 && !(wide && kw + NW * q0 < cols)) {
                // no column of this warp left: the group's sums are zero
#pragma unroll
                for (int q = 0; q < KQE; ++q)
                    if (lane == 0) red[warp][q0 + q] = make_double2(0, 0);
                continue;
            }
            A2 acc[KQE];
#pragma unroll
            for (int q = 0; q < KQE; ++q) acc[q] = from_d2<A2>(make_double2(0, 0));
            if (on) {
                // RU steps of two groups of RL rows a lane at once: 2 KQE RU loads in flight (2 KQ but in one case)
                for (int r0 = rs + RL * lane; r0 < re; r0 += 64 * RL * RU) {
                    RowPack<T2, RL> t[RU][KQE], u[RU][KQE];
                    T2 x[RU][RL], x2[RU][RL];  // kept in the stored precision until used (registers)
#pragma unroll
                    for (int g = 0; g < RU; ++g) {
                        const int r = r0 + 64 * RL * g, r2 = r + 32 * RL;
                        const int n0 = max(0, min(RL, re - r)), n1 = max(0, min(RL, re - r2));
#pragma unroll
                        for (int q = 0; q < KQE; ++q) {
                            const int k = kw + NW * (q0 + q);
                            const bool use = (wide || q0 + q == 0) && k < cols;
                            t[g][q] = load_rows<T2, RL>(Vr + k * col + r, use ? n0 : 0);
                            u[g][q] = load_rows<T2, RL>(Vr + k * col + r2, use ? n1 : 0);
                        }
#pragma unroll
                        for (int e = 0; e < RL; ++e) {
                            x[g][e] = e < n0 ? ws[r + e] : from_d2<T2>(make_double2(0, 0));
                            x2[g][e] = e < n1 ? ws[r2 + e] : from_d2<T2>(make_double2(0, 0));
                        }
                    }
#pragma unroll
                    for (int g = 0; g < RU; ++g)
#pragma unroll
                        for (int q = 0; q < KQE; ++q)
#pragma unroll
                            for (int e = 0; e < RL; ++e) {
                                const A2 a = amulc(t[g][q].v[e], x[g][e]), b = amulc(u[g][q].v[e], x2[g][e]);
                                acc[q].x += a.x;
                                acc[q].y += a.y;
                                acc[q].x += b.x;
                                acc[q].y += b.y;
                            }
                }
            }
#pragma unroll
            for (int q = 0; q < KQE; ++q) {
                double2 v = to_d2(acc[q]);  // the sums over lanes, CTAs and chunks in FP64
                for (int o = 16; o > 0; o >>= 1) {
                    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
                    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
                }
                if (lane == 0) red[warp][q0 + q] = v;
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < cols; k += kRT) {
            double2 v;
            if (wide) {
                v = red[k % NW][k / NW];
            } else {
                v = make_double2(0, 0);
                for (int g = 0; g < G; ++g) v = dadd(v, red[k + g * cols][0]);
            }
            part[(int64_t)k * gridDim.x + blockIdx.x] = v;
        }
    } else {
        double2 v[1] = {make_double2(nrm, 0)};
        block_sum<1>(v, part + blockIdx.x);
    }
    if (!arrive(&S.counter)) return;
    if (mode == 2) {
        const double tot = cta_total(part, gridDim.x).x;
        // stage h, the rotations and the column in shared memory; thread 0 runs the chain there
        __shared__ double2 scol[kStreamCols + 1], scs[kStreamCols], ssn[kStreamCols];
        const int m = ar.m, j = S.step;
        const double2* h = ar.h + (int64_t)rhs * mc;
        double2* cs = ar.cs + (int64_t)rhs * m;
        double2* sn = ar.sn + (int64_t)rhs * m;
        for (int k = threadIdx.x; k <= j; k += kRT) scol[k] = h[k];
        for (int k = threadIdx.x; k < j; k += kRT) {
            scs[k] = cs[k];
            ssn[k] = sn[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) arnoldi_finish(S, ar, rhs, tot, scol, scs, ssn, true);
        __syncthreads();
        double2* col = ar.H + ((int64_t)rhs * m + j) * mc;
        for (int k = threadIdx.x; k <= j + 1; k += kRT) col[k] = scol[k];
        if (threadIdx.x == 0) {
            cs[j] = scs[j];
            sn[j] = ssn[j];
        }
        return;
    }
    for (int k = warp; k < cols; k += NW) {
        double2 v = make_double2(0, 0);
        const double2* pk = part + (int64_t)k * gridDim.x;
        for (int b = lane; b < (int)gridDim.x; b += 32) v = dadd(v, pk[b]);
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_down_sync(0xffffffffu, v.x, o);
            v.y += __shfl_down_sync(0xffffffffu, v.y, o);
        }
        if (lane == 0) {
            double2* h = ar.h + (int64_t)rhs * mc;
            ar.c[(int64_t)rhs * mc + k] = v;
            h[k] = mode == 0 ? v : dadd(h[k], v);
        }
    }
}

// CTAs and rows per CTA of k_gm_orth_stream: at least two CTAs per SM, chunks of at most about
// kStreamRows rows, no more CTAs than the partial buffers hold.
static void stream_config(int64_t n, int* blocks, int* chunk) {
    const int64_t want = std::max<int64_t>(2 * 148, (n + kStreamRows - 1) / kStreamRows);
    const int64_t b = std::max<int64_t>(1, std::min<int64_t>(want, reduce_blocks(n)));
    int64_t c = (n + b - 1) / b;
    c = (c + 31) / 32 * 32;
    *chunk = (int)c;
    *blocks = (int)((n + c - 1) / c);
}

// (the dynamic shared-memory attributes are set before any capture, in gmres())
template <typename T2, int KQE>
static void launch_orth_stream(const T2* V, T2* w, int64_t n, int nrhs, GmState* st, const GmArrays& ar, int mode,
                               cudaStream_t s) {
    int blocks, chunk;
    stream_config(n, &blocks, &chunk);
    // FP32 reads two rows a load where every column starts on 16 bytes (an even length)
    if (sizeof(T2) == 8 && n % 2 == 0)
        k_gm_orth_stream<T2, (sizeof(T2) == 8 ? 2 : 1), KQE><<<dim3(blocks, nrhs), kRT, (size_t)chunk * sizeof(T2), s>>>(
            V, w, n, nrhs, st, ar, mode, chunk);
    else
        k_gm_orth_stream<T2, 1, KQE><<<dim3(blocks, nrhs), kRT, (size_t)chunk * sizeof(T2), s>>>(V, w, n, nrhs, st, ar,
                                                                                                 mode, chunk);
    count_launch();
}

// The shared-memory attribute of every form of k_gm_orth_stream (set before any capture).
template <typename T2> static int stream_attrs(int bytes) {
    const int b = std::max(bytes, 48 * 1024);
    constexpr int RL = sizeof(T2) == 8 ? 2 : 1;
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, 1, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, 1, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, 1, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, RL, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, RL, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, RL, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth_stream<T2, RL, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    return RTM_OK;
}

// cols: the basis columns of this Arnoldi step (the dots' column groups follow it).
template <typename T2> static void launch_orth(const T2* V, T2* w, int64_t n, int nrhs, GmState* st, const GmArrays& ar,
                                               int mode, int cols, cudaStream_t s) {
    if (ar.m + 1 <= kStreamCols) {
        constexpr int NW = kRT / 32;
        if (mode == 2 || cols > 4 * NW) launch_orth_stream<T2, 8>(V, w, n, nrhs, st, ar, mode, s);
        else if (cols > 2 * NW) launch_orth_stream<T2, 4>(V, w, n, nrhs, st, ar, mode, s);
        else if (cols > NW) launch_orth_stream<T2, 2>(V, w, n, nrhs, st, ar, mode, s);
        else launch_orth_stream<T2, 1>(V, w, n, nrhs, st, ar, mode, s);
        return;
    }
    int TR;
    size_t smem;
    orth_config<T2>(ar.m, &TR, &smem);
    const int64_t tiles = (n + TR - 1) / TR;
    const int blocks = (int)std::min<int64_t>({tiles, (int64_t)reduce_blocks(n), 2 * 148});
    k_gm_orth<T2><<<dim3(blocks, nrhs), kRT, smem, s>>>(V, w, n, nrhs, st, ar, mode, TR);
    count_launch();
}

// V[:, step] = w / H(step, step - 1) while the cycle goes on.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_next(const T2* __restrict__ w, T2* __restrict__ V, int64_t n, int nrhs,
                                                 const GmState* st) {
    const int rhs = blockIdx.y;
    const GmState& S = st[rhs];
    if (!S.active) return;
    const double inv = S.inv_sub;
    const T2* wr = w + rhs * n;
    T2* v = V + ((int64_t)S.step * nrhs + rhs) * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 x = to_d2(wr[i]);
        v[i] = from_d2<T2>(make_double2(x.x * inv, x.y * inv));
    }
}

// y = H(1:step, 1:step) \ g(1:step) (upper triangular after the rotations; iterate_.m:73-74).
// One CTA per right-hand side: H and g are staged in shared memory, then column-oriented back
// substitution (y_c = g_c / H_cc; g_i -= H_ic y_c for i < c, in parallel over i).
__global__ void k_gm_solve(GmState* st, GmArrays ar, int staged) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int rhs = blockIdx.x;
    GmState& S = st[rhs];
    if (!S.cycle_ran) return;
    const int m = ar.m, k = S.step;
    const double2* H = ar.H + (int64_t)rhs * (m + 1) * m;
    const double2* g = ar.g + (int64_t)rhs * (m + 1);
    double2* y = ar.y + (int64_t)rhs * m;
    // staged: H (k x k, leading dimension k) and g in shared memory; otherwise read H in place and
    // run the substitution in y.
    const double2* Hs = H;
    int ld = m + 1;
    double2* gs = y;
    if (staged) {
        double2* hs = reinterpret_cast<double2*>(smem_raw);
        for (int t = threadIdx.x; t < k * k; t += blockDim.x) {
            const int r = t % k, c = t / k;
            hs[t] = H[(int64_t)c * (m + 1) + r];
        }
        Hs = hs;
        ld = k;
        gs = hs + (int64_t)k * k;
    }
    for (int t = threadIdx.x; t < k; t += blockDim.x) gs[t] = g[t];
    __syncthreads();
    for (int c = k - 1; c >= 0; --c) {
        const double2 yc = ddiv(gs[c], Hs[(int64_t)c * ld + c]);
        for (int i = threadIdx.x; i < c; i += blockDim.x) {
            const double2 p = dmul(Hs[(int64_t)c * ld + i], yc);
            gs[i].x -= p.x;
            gs[i].y -= p.y;
        }
        __syncthreads();
        if (threadIdx.x == 0) gs[c] = yc;
        __syncthreads();
    }
    if (staged)
        for (int t = threadIdx.x; t < k; t += blockDim.x) y[t] = gs[t];
}

static void launch_gm_solve(GmState* st, const GmArrays& ar, int nrhs, cudaStream_t s) {
    const size_t bytes = ((size_t)ar.m * ar.m + ar.m) * sizeof(double2);
    const bool staged = bytes <= 200 * 1024;
    k_gm_solve<<<nrhs, 128, staged ? bytes : 0, s>>>(st, ar, staged ? 1 : 0);
    count_launch();
}

// x += V(:, 1:step) y.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_xupdate(T2* __restrict__ x, const T2* __restrict__ V, int64_t n, int nrhs,
                                                    GmState* st, GmArrays ar) {
    const int rhs = blockIdx.y;
    const GmState& S = st[rhs];
    if (!S.cycle_ran) return;
    const int k = S.step;
    const double2* y = ar.y + (int64_t)rhs * ar.m;
    T2* xr = x + rhs * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 v = to_d2(xr[i]);
        for (int l = 0; l < k; ++l) v = dadd(v, dmul(to_d2(V[((int64_t)l * nrhs + rhs) * n + i]), y[l]));
        xr[i] = from_d2<T2>(v);
    }
}

// u = V(:, 1:step) y (right preconditioning: x += M u follows).
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_vy(T2* __restrict__ u, const T2* __restrict__ V, int64_t n, int nrhs,
                                               GmState* st, GmArrays ar) {
    const int rhs = blockIdx.y;
    const GmState& S = st[rhs];
    if (!S.cycle_ran) return;
    const int k = S.step;
    const double2* y = ar.y + (int64_t)rhs * ar.m;
    T2* ur = u + rhs * n;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double2 v = make_double2(0, 0);
        for (int l = 0; l < k; ++l) v = dadd(v, dmul(to_d2(V[((int64_t)l * nrhs + rhs) * n + i]), y[l]));
        ur[i] = from_d2<T2>(v);
    }
}

// x += w where the cycle ran.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_gm_addx(T2* __restrict__ x, const T2* __restrict__ w, int64_t n,
                                                 const GmState* st) {
    const int rhs = blockIdx.y;
    if (!st[rhs].cycle_ran) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 a = to_d2(x[rhs * n + i]), b = to_d2(w[rhs * n + i]);
        x[rhs * n + i] = from_d2<T2>(make_double2(a.x + b.x, a.y + b.y));
    }
}

__global__ void k_gm_cycle_end(GmState* st, int nrhs) {
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs) return;
    st[rhs].cycle_ran = 0;
    st[rhs].skip_update = 1;
    st[rhs].active = 0;
    st[rhs].skip_step = 1;
}

// ============================================================================================
// Shared helpers
// out = b - t where flag (stride) is zero.
template <typename T2>
__global__ void __launch_bounds__(kRT) k_residual(const T2* __restrict__ b, const T2* __restrict__ t, T2* __restrict__ out,
                                                  int64_t n, const int* skip, int stride) {
    const int rhs = blockIdx.y;
    if (skip && skip[(int64_t)rhs * stride]) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 bv = to_d2(b[rhs * n + i]), tv = to_d2(t[rhs * n + i]);
        out[rhs * n + i] = from_d2<T2>(make_double2(bv.x - tv.x, bv.y - tv.y));
    }
}

// ||b - t||^2 and ||b||^2 per right-hand side into res[rhs] = (||b - t||, ||b||).
template <typename T2>
__global__ void __launch_bounds__(kRT) k_true_residual(const T2* __restrict__ b, const T2* __restrict__ t, int64_t n,
                                                       double2* part, unsigned int* counters, double2* res) {
    const int rhs = blockIdx.y;
    double2 acc[1] = {make_double2(0, 0)};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 bv = to_d2(b[rhs * n + i]), tv = to_d2(t[rhs * n + i]);
        const double dx = bv.x - tv.x, dy = bv.y - tv.y;
        acc[0].x += dx * dx + dy * dy;
        acc[0].y += bv.x * bv.x + bv.y * bv.y;
    }
    block_sum<1>(acc, part + ((int64_t)rhs * gridDim.x + blockIdx.x));
    if (!arrive(&counters[rhs])) return;
    const double2 s = cta_total(part + (int64_t)rhs * gridDim.x, gridDim.x);
    if (threadIdx.x == 0) res[rhs] = make_double2(sqrt(s.x), sqrt(s.y));
}

template <typename T2>
__global__ void k_zero_where(T2* __restrict__ x, int64_t n, const int* flag, int stride) {
    const int rhs = blockIdx.y;
    if (!flag[(int64_t)rhs * stride]) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[rhs * n + i] = from_d2<T2>(make_double2(0, 0));
}

__global__ void k_fill(double* p, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_d2f(const double2* __restrict__ in, float2* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}
__global__ void k_f2d(const float2* __restrict__ in, double2* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_double2(in[i].x, in[i].y);
}

void convert_to_fp32(const double2* in, float2* out, int64_t n, cudaStream_t s) {
    k_d2f<<<592, 256, 0, s>>>(in, out, n);
    count_launch();
}
void convert_to_fp64(const float2* in, double2* out, int64_t n, cudaStream_t s) {
    k_f2d<<<592, 256, 0, s>>>(in, out, n);
    count_launch();
}

// CTAs of the vector kernels: about two elements per thread, at most 4 waves of the 148 SMs.
static int reduce_blocks(int64_t n) {
    const int64_t b = (n + (int64_t)kRT * 2 - 1) / ((int64_t)kRT * 2);
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 592));
}

// A CUDA graph of a fixed launch sequence: captured once from the stream, replayed per chunk.
struct GraphRunner {
    cudaGraphExec_t exec = nullptr;
    int64_t kernels = 0;
    GraphRunner() = default;
    GraphRunner(const GraphRunner&) = delete;
    GraphRunner& operator=(const GraphRunner&) = delete;
    ~GraphRunner() {
        if (exec) cudaGraphExecDestroy(exec);
    }
    template <class F> int capture(cudaStream_t s, F&& body) {
        const int64_t before = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
        RTM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
        const int st = body();
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        // the captured launches have not run yet; they are counted at every replay
        kernels = __atomic_load_n(&g_launches, __ATOMIC_RELAXED) - before;
        __atomic_fetch_sub(&g_launches, kernels, __ATOMIC_RELAXED);
        if (st != RTM_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (ei != cudaSuccess) return cuda_fail(ei, "cudaGraphInstantiate");
        return RTM_OK;
    }
    // Captures once; if the capture fails the sequence runs as plain launches from then on (the
    // same kernels, only without the graph).
    template <class F> int run(cudaStream_t s, F&& body) {
        if (!exec && !eager) {
            if (capture(s, body) != RTM_OK) {
                cudaGetLastError();
                eager = true;
                if (getenv("RTM_DEBUG")) fprintf(stderr, "librtm: graph capture failed, launching eagerly\n");
            }
        }
        if (eager) return body();
        return launch(s);
    }
    bool eager = false;
    int launch(cudaStream_t s) {
        RTM_CUDA(cudaGraphLaunch(exec, s));
        count_launch((int)kernels);
        return RTM_OK;
    }
};

// ============================================================================================
template <typename T>
static int cocg(LinearOp* A, LinearOp* M, const SolveConfig& cfg, const void* bv, const void* x0v, void* xv, int64_t n,
                int nrhs, SolveResult& res, cudaStream_t s) {
    using T2 = typename Cx<T>::T2;
    const T2* b = static_cast<const T2*>(bv);
    const T2* x0 = static_cast<const T2*>(x0v);
    T2* x = static_cast<T2*>(xv);
    const int nb = reduce_blocks(n);
    const size_t vec = (size_t)n * nrhs * sizeof(T2);
    DeviceBuffer r, z, d, q, stb, part, hist, resb, cnt;
    StreamSyncGuard guard(s);
    RTM_TRY(r.alloc(vec));
    if (M) RTM_TRY(z.alloc(vec));
    RTM_TRY(d.alloc(vec));
    RTM_TRY(q.alloc(vec));
    RTM_TRY(stb.alloc(sizeof(CgState) * nrhs));
    RTM_TRY(part.alloc(sizeof(double2) * nb * nrhs));
    const int hs = cfg.max_iterations + 1;
    RTM_TRY(hist.alloc(sizeof(double) * hs * nrhs));
    RTM_TRY(resb.alloc(sizeof(double2) * nrhs));
    RTM_TRY(cnt.alloc(sizeof(unsigned int) * nrhs));
    std::vector<CgState> init(nrhs);
    for (int k = 0; k < nrhs; ++k) {
        CgState& st = init[k];
        memset(&st, 0, sizeof st);
        st.tol = cfg.tolerances ? cfg.tolerances[k] : cfg.tolerance;
        st.max_iterations = cfg.max_iterations;
    }
    RTM_CUDA(cudaMemcpyAsync(stb.ptr, init.data(), sizeof(CgState) * nrhs, cudaMemcpyHostToDevice, s));
    RTM_CUDA(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, s));
    k_fill<<<64, 256, 0, s>>>(hist.as<double>(), (int64_t)hs * nrhs, NAN);
    count_launch();
    RTM_TRY(A->reserve(nrhs));
    if (M) RTM_TRY(M->reserve(nrhs));
    CgState* st = stb.as<CgState>();
    SkipFlags skip{&st[0].done, (int)(sizeof(CgState) / sizeof(int))};
    const dim3 grid(nb, nrhs);
    if (x0) {
        RTM_CUDA(cudaMemcpyAsync(x, x0, vec, cudaMemcpyDeviceToDevice, s));
        RTM_TRY(A->apply(x, q.ptr, nrhs, s, SkipFlags{}));
        k_residual<T2><<<grid, kRT, 0, s>>>(b, q.as<T2>(), r.as<T2>(), n, nullptr, 0);
        count_launch();
    } else {
        RTM_CUDA(cudaMemsetAsync(x, 0, vec, s));
        RTM_CUDA(cudaMemcpyAsync(r.ptr, b, vec, cudaMemcpyDeviceToDevice, s));
    }
    k_cg_start<T2><<<grid, kRT, 0, s>>>(b, r.as<T2>(), n, st, part.as<double2>(), hist.as<double>(), hs);
    count_launch();
    T2* zp = M ? z.as<T2>() : r.as<T2>();
    const int every = cfg.check_every > 0 ? cfg.check_every : 16;
    std::vector<CgState> host(nrhs);
    int launched = 0;
    res.matvecs = x0 ? 1 : 0;
    // `every` iterations as one graph; iterations past the stopping test are no-ops on the device.
    auto chunk_body = [&]() -> int {
        for (int it = 0; it < every; ++it) {
            if (M) RTM_TRY(M->apply(r.ptr, z.ptr, nrhs, s, skip));
            k_cg_rz<T2><<<grid, kRT, 0, s>>>(r.as<T2>(), zp, n, st, part.as<double2>());
            k_cg_dir<T2><<<grid, kRT, 0, s>>>(zp, d.as<T2>(), n, st);
            RTM_TRY(A->apply(d.ptr, q.ptr, nrhs, s, skip));
            k_cg_dq<T2><<<grid, kRT, 0, s>>>(d.as<T2>(), q.as<T2>(), n, st, part.as<double2>());
            k_cg_update<T2><<<grid, kRT, 0, s>>>(x, r.as<T2>(), d.as<T2>(), q.as<T2>(), n, st, part.as<double2>(),
                                                 hist.as<double>(), hs);
            count_launch(4);
        }
        RTM_CUDA(cudaGetLastError());
        return RTM_OK;
    };
    GraphRunner graph;
    while (true) {
        RTM_CUDA(cudaMemcpyAsync(host.data(), stb.ptr, sizeof(CgState) * nrhs, cudaMemcpyDeviceToHost, s));
        RTM_CUDA(cudaStreamSynchronize(s));
        bool all = true;
        for (auto& h : host) all = all && h.done;
        if (all || launched >= cfg.max_iterations || (cfg.cancel && *cfg.cancel)) break;
        RTM_TRY(graph.run(s, chunk_body));
        launched += every;
    }
    // IterativeMethod.m:52: the true residual costs one more product.
    RTM_TRY(A->apply(x, q.ptr, nrhs, s, SkipFlags{}));
    k_zero_where<T2><<<grid, kRT, 0, s>>>(x, n, &st[0].zero_rhs, (int)(sizeof(CgState) / sizeof(int)));
    k_true_residual<T2><<<grid, kRT, 0, s>>>(b, q.as<T2>(), n, part.as<double2>(), cnt.as<unsigned int>(),
                                             resb.as<double2>());
    count_launch(2);
    std::vector<double2> rb(nrhs);
    RTM_CUDA(cudaMemcpyAsync(rb.data(), resb.ptr, sizeof(double2) * nrhs, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaMemcpyAsync(host.data(), stb.ptr, sizeof(CgState) * nrhs, cudaMemcpyDeviceToHost, s));
    res.history.resize((size_t)hs * nrhs);
    RTM_CUDA(cudaMemcpyAsync(res.history.data(), hist.ptr, hist.bytes, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    RTM_TRY(device_fault_check(s));
    res.hist_stride = hs;
    res.stats.resize(nrhs);
    for (int k = 0; k < nrhs; ++k) {
        rtm_solve_stats& o = res.stats[k];
        o.converged = host[k].converged;
        o.iteration_count = host[k].zero_rhs ? 0 : host[k].iteration;
        o.residual_norm = host[k].zero_rhs ? 0.0 : rb[k].x / rb[k].y;
        o.refinements = 0;
        o.matvecs = res.matvecs + host[k].iteration + 1;
    }
    return RTM_OK;
}

template <typename T>
static int gmres(LinearOp* A, LinearOp* M, const SolveConfig& cfg, const void* bv, const void* x0v, void* xv, int64_t n,
                 int nrhs, SolveResult& res, cudaStream_t s) {
    using T2 = typename Cx<T>::T2;
    const T2* b = static_cast<const T2*>(bv);
    const T2* x0 = static_cast<const T2*>(x0v);
    T2* x = static_cast<T2*>(xv);
    const int m = (int)std::max<int64_t>(1, std::min<int64_t>({(int64_t)cfg.restart, n, (int64_t)cfg.max_iterations}));
    if (m + 1 > kStreamCols) {
        // bases above kStreamCols columns run k_gm_orth, whose tile of the basis sits in shared memory
        int TR;
        size_t smem;
        orth_config<T2>(m, &TR, &smem);
        if (smem > (size_t)kOrthSmemMax)
            return fail(RTM_ERR_UNSUPPORTED, "a GMRES restart of " + std::to_string(m) +
                                                 " is longer than this build's orthogonalisation holds in shared memory");
    }
    const int nb = reduce_blocks(n);
    const size_t vec = (size_t)n * nrhs * sizeof(T2);
    // Right preconditioning solves A M u = b with x = x0 + M (V y) at the end of each cycle: the
    // monitored residual is the residual of A x = b itself. The preconditioners here are fixed linear
    // operators, so M (V y) equals the flexible form's sum of the z_j = M v_j y_j, and no basis of the
    // z_j is kept. Left preconditioning is the reference's form.
    const bool right = M != nullptr && cfg.right_preconditioned;
    DeviceBuffer V, w, t, stb, H, g, cs, sn, h, c, y, part, hist, resb, cnt;
    StreamSyncGuard guard(s);
    RTM_TRY(V.alloc(vec * (m + 1)));
    RTM_TRY(w.alloc(vec));
    RTM_TRY(t.alloc(vec));
    RTM_TRY(stb.alloc(sizeof(GmState) * nrhs));
    RTM_TRY(H.alloc(sizeof(double2) * (m + 1) * m * nrhs));
    RTM_TRY(g.alloc(sizeof(double2) * (m + 1) * nrhs));
    RTM_TRY(cs.alloc(sizeof(double2) * m * nrhs));
    RTM_TRY(sn.alloc(sizeof(double2) * m * nrhs));
    RTM_TRY(h.alloc(sizeof(double2) * (m + 1) * nrhs));
    RTM_TRY(c.alloc(sizeof(double2) * (m + 1) * nrhs));
    RTM_TRY(y.alloc(sizeof(double2) * m * nrhs));
    RTM_TRY(part.alloc(sizeof(double2) * (size_t)nb * (m + 1) * nrhs));
    const int hs = cfg.max_iterations + 1;
    RTM_TRY(hist.alloc(sizeof(double) * hs * nrhs));
    RTM_TRY(resb.alloc(sizeof(double2) * nrhs));
    RTM_TRY(cnt.alloc(sizeof(unsigned int) * nrhs));
    RTM_CUDA(cudaMemsetAsync(H.ptr, 0, H.bytes, s));
    RTM_CUDA(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, s));
    std::vector<GmState> init(nrhs);
    for (int k = 0; k < nrhs; ++k) {
        GmState& st = init[k];
        memset(&st, 0, sizeof st);
        st.tol = cfg.tolerances ? cfg.tolerances[k] : cfg.tolerance;
        st.max_iterations = cfg.max_iterations;
        st.m = m;
        st.skip_step = 1;
        st.skip_update = 1;
    }
    RTM_CUDA(cudaMemcpyAsync(stb.ptr, init.data(), sizeof(GmState) * nrhs, cudaMemcpyHostToDevice, s));
    k_fill<<<64, 256, 0, s>>>(hist.as<double>(), (int64_t)hs * nrhs, NAN);
    count_launch();
    RTM_TRY(A->reserve(nrhs));
    if (M) RTM_TRY(M->reserve(nrhs));
    GmState* st = stb.as<GmState>();
    GmArrays ar{H.as<double2>(), g.as<double2>(), cs.as<double2>(), sn.as<double2>(), h.as<double2>(),
                c.as<double2>(), y.as<double2>(), part.as<double2>(), hist.as<double>(), hs, m};
    const int stride = (int)(sizeof(GmState) / sizeof(int));
    SkipFlags skip_step{&st[0].skip_step, stride};
    SkipFlags skip_done{&st[0].done, stride};
    SkipFlags skip_update{&st[0].skip_update, stride};
    const dim3 grid(nb, nrhs);
    // reference = ||P b|| (iterate_.m:9); ||b|| with right preconditioning
    if (M && !right) RTM_TRY(M->apply(b, w.ptr, nrhs, s, SkipFlags{}));
    else RTM_CUDA(cudaMemcpyAsync(w.ptr, b, vec, cudaMemcpyDeviceToDevice, s));
    k_gm_norm<T2><<<grid, kRT, 0, s>>>(w.as<T2>(), n, st, ar, 0, 0);
    count_launch();
    res.matvecs = 0;
    if (x0) {
        RTM_CUDA(cudaMemcpyAsync(x, x0, vec, cudaMemcpyDeviceToDevice, s));
        RTM_TRY(A->apply(x, t.ptr, nrhs, s, skip_done));
        k_residual<T2><<<grid, kRT, 0, s>>>(b, t.as<T2>(), t.as<T2>(), n, &st[0].done, stride);
        count_launch();
        if (M && !right) RTM_TRY(M->apply(t.ptr, w.ptr, nrhs, s, skip_done));
        else RTM_CUDA(cudaMemcpyAsync(w.ptr, t.ptr, vec, cudaMemcpyDeviceToDevice, s));
        res.matvecs += 1;
    } else {
        RTM_CUDA(cudaMemsetAsync(x, 0, vec, s));
    }
    k_gm_norm<T2><<<grid, kRT, 0, s>>>(w.as<T2>(), n, st, ar, 1, 1);
    count_launch();
    // function attributes are set before the capture
    RTM_CUDA(cudaFuncSetAttribute(k_gm_orth<T2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kOrthSmemMax));
    {
        int sb, sc;
        stream_config(n, &sb, &sc);
        RTM_TRY(stream_attrs<T2>(sc * (int)sizeof(T2)));
    }
    RTM_CUDA(cudaFuncSetAttribute(k_gm_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    std::vector<GmState> host(nrhs);
    T2* Vp = V.as<T2>();
    // One restart cycle as a graph: the m Arnoldi steps, the least-squares solve, the update of x and
    // the true residual the next cycle starts from (iterate_.m:30-82). Steps after the stopping test
    // and the restart of a finished system are no-ops on the device.
    auto cycle_body = [&]() -> int {
        k_gm_v0<T2><<<grid, kRT, 0, s>>>(w.as<T2>(), Vp, n, nrhs, st);
        count_launch();
        for (int j = 0; j < m; ++j) {
            T2* vj = Vp + (int64_t)j * nrhs * n;
            if (right) {
                RTM_TRY(M->apply(vj, t.ptr, nrhs, s, skip_step));
                RTM_TRY(A->apply(t.ptr, w.ptr, nrhs, s, skip_step));
            } else if (M) {
                RTM_TRY(A->apply(vj, t.ptr, nrhs, s, skip_step));
                RTM_TRY(M->apply(t.ptr, w.ptr, nrhs, s, skip_step));
            } else {
                RTM_TRY(A->apply(vj, w.ptr, nrhs, s, skip_step));
            }
            // CGS2: project (mode 0), subtract and project again (1), subtract the correction and take the
            // norm (2). One pass skips mode 1: mode 2 then subtracts the first projection, which mode 0
            // left in the coefficients it reads.
            launch_orth<T2>(Vp, w.as<T2>(), n, nrhs, st, ar, 0, j + 1, s);
            if (cfg.gram_schmidt_passes != 1) launch_orth<T2>(Vp, w.as<T2>(), n, nrhs, st, ar, 1, j + 1, s);
            launch_orth<T2>(Vp, w.as<T2>(), n, nrhs, st, ar, 2, j + 1, s);
            k_gm_next<T2><<<grid, kRT, 0, s>>>(w.as<T2>(), Vp, n, nrhs, st);
            count_launch(1);
        }
        launch_gm_solve(st, ar, nrhs, s);
        if (right) {
            k_gm_vy<T2><<<grid, kRT, 0, s>>>(t.as<T2>(), Vp, n, nrhs, st, ar);
            count_launch();
            RTM_TRY(M->apply(t.ptr, w.ptr, nrhs, s, skip_update));
            k_gm_addx<T2><<<grid, kRT, 0, s>>>(x, w.as<T2>(), n, st);
            count_launch();
        } else {
            k_gm_xupdate<T2><<<grid, kRT, 0, s>>>(x, Vp, n, nrhs, st, ar);
            count_launch();
        }
        k_gm_cycle_end<<<(nrhs + 31) / 32, 32, 0, s>>>(st, nrhs);
        count_launch();
        RTM_TRY(A->apply(x, t.ptr, nrhs, s, skip_done));
        k_residual<T2><<<grid, kRT, 0, s>>>(b, t.as<T2>(), t.as<T2>(), n, &st[0].done, stride);
        count_launch();
        if (M && !right) RTM_TRY(M->apply(t.ptr, w.ptr, nrhs, s, skip_done));
        else RTM_CUDA(cudaMemcpyAsync(w.ptr, t.ptr, vec, cudaMemcpyDeviceToDevice, s));
        k_gm_norm<T2><<<grid, kRT, 0, s>>>(w.as<T2>(), n, st, ar, 1, 0);
        count_launch();
        RTM_CUDA(cudaGetLastError());
        return RTM_OK;
    };
    GraphRunner graph;
    int cycles = 0;
    while (true) {
        RTM_CUDA(cudaMemcpyAsync(host.data(), stb.ptr, sizeof(GmState) * nrhs, cudaMemcpyDeviceToHost, s));
        RTM_CUDA(cudaStreamSynchronize(s));
        bool all = true;
        for (auto& hh : host) all = all && hh.done;
        if (all || cycles > cfg.max_iterations || (cfg.cancel && *cfg.cancel)) break;
        RTM_TRY(graph.run(s, cycle_body));
        ++cycles;
        res.matvecs += 1;
    }
    RTM_TRY(A->apply(x, t.ptr, nrhs, s, SkipFlags{}));
    k_zero_where<T2><<<grid, kRT, 0, s>>>(x, n, &st[0].zero_rhs, stride);
    k_true_residual<T2><<<grid, kRT, 0, s>>>(b, t.as<T2>(), n, part.as<double2>(), cnt.as<unsigned int>(),
                                             resb.as<double2>());
    count_launch(2);
    std::vector<double2> rb(nrhs);
    RTM_CUDA(cudaMemcpyAsync(rb.data(), resb.ptr, sizeof(double2) * nrhs, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaMemcpyAsync(host.data(), stb.ptr, sizeof(GmState) * nrhs, cudaMemcpyDeviceToHost, s));
    res.history.resize((size_t)hs * nrhs);
    RTM_CUDA(cudaMemcpyAsync(res.history.data(), hist.ptr, hist.bytes, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    RTM_TRY(device_fault_check(s));
    res.hist_stride = hs;
    res.stats.resize(nrhs);
    for (int k = 0; k < nrhs; ++k) {
        rtm_solve_stats& o = res.stats[k];
        o.converged = host[k].converged;
        o.iteration_count = host[k].zero_rhs ? 0 : host[k].iteration;
        o.residual_norm = host[k].zero_rhs ? 0.0 : rb[k].x / rb[k].y;
        o.refinements = 0;
        o.matvecs = res.matvecs + host[k].iteration + 1;
    }
    return RTM_OK;
}

// ============================================================================================
// Mixed precision: FP64 iterative refinement around an FP32 inner solve.
//   r = b - A64 x (FP64); r32 = r / ||r||; d32 ~ A32^-1 r32 (FP32 flexible GMRES, or FP32 COCG);
//   x += ||r|| d32; repeat until ||b - A64 x|| / ||b|| < tolerance. The outer residual is always
//   the true FP64 residual, so the stopping test holds for the FP64 operator.
// Each right-hand side's inner solve stops at the relative residual that meets the outer tolerance
// in this step, 0.5 tolerance ||b|| / ||r|| (an inner residual eps leaves an outer one of about
// eps ||r|| plus the FP32 operator's error), but never aims below inner_tolerance, the accuracy an
// FP32 solve reaches safely; a step that stops there leaves the rest to the next refinement.

__global__ void k_ir_to32(const double2* __restrict__ r, float2* __restrict__ r32, int64_t n, const double2* res,
                          const int* done) {
    const int rhs = blockIdx.y;
    const bool off = done[rhs] != 0;
    const double inv = off ? 0.0 : 1.0 / res[rhs].x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = r[rhs * n + i];
        r32[rhs * n + i] = make_float2((float)(v.x * inv), (float)(v.y * inv));
    }
}

__global__ void k_ir_update(double2* __restrict__ x, const float2* __restrict__ d, int64_t n, const double2* res,
                            const int* done) {
    const int rhs = blockIdx.y;
    if (done[rhs]) return;
    const double s = res[rhs].x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = d[rhs * n + i];
        double2 xv = x[rhs * n + i];
        xv.x += s * v.x;
        xv.y += s * v.y;
        x[rhs * n + i] = xv;
    }
}

// res = (||r||, ||b||): history entry and stopping test of refinement step `step`.
__global__ void k_ir_check(const double2* res, int* done, int* converged, double* hist, int hist_stride, int step,
                           double tol, int nrhs) {
    const int rhs = blockIdx.x * blockDim.x + threadIdx.x;
    if (rhs >= nrhs || done[rhs]) return;
    const double2 v = res[rhs];
    const double rel = v.y == 0.0 ? 0.0 : v.x / v.y;
    if (step < hist_stride) hist[(int64_t)rhs * hist_stride + step] = rel;
    converged[rhs] = rel < tol;
    done[rhs] = converged[rhs] || !isfinite(rel);
}

template <typename T>
static int gmres(LinearOp* A, LinearOp* M, const SolveConfig& cfg, const void* bv, const void* x0v, void* xv, int64_t n,
                 int nrhs, SolveResult& res, cudaStream_t s);

int solve_mixed(LinearOp* A64, LinearOp* A32, LinearOp* M32, const SolveConfig& cfg, const void* bv, const void* x0v,
                void* xv, int64_t n, int nrhs, SolveResult& res, cudaStream_t s, LinearOp* M64) {
    const double2* b = static_cast<const double2*>(bv);
    const double2* x0 = static_cast<const double2*>(x0v);
    double2* x = static_cast<double2*>(xv);
    const int nb = reduce_blocks(n);
    const dim3 grid(nb, nrhs);
    const size_t vec64 = (size_t)n * nrhs * sizeof(double2), vec32 = (size_t)n * nrhs * sizeof(float2);
    const int m = (int)std::max<int64_t>(1, std::min<int64_t>((int64_t)cfg.restart, n));
    DeviceBuffer r64, t64, r32, d32, part, resb, cnt, done, conv, hist;
    StreamSyncGuard guard(s);
    RTM_TRY(r64.alloc(vec64));
    RTM_TRY(t64.alloc(vec64));
    RTM_TRY(r32.alloc(vec32));
    RTM_TRY(d32.alloc(vec32));
    RTM_TRY(part.alloc(sizeof(double2) * (size_t)nb * (m + 1) * nrhs));
    RTM_TRY(resb.alloc(sizeof(double2) * nrhs));
    RTM_TRY(cnt.alloc(sizeof(unsigned int) * nrhs));
    RTM_TRY(done.alloc(sizeof(int) * nrhs));
    RTM_TRY(conv.alloc(sizeof(int) * nrhs));
    const int hs = cfg.max_iterations + 1;
    RTM_TRY(hist.alloc(sizeof(double) * hs * nrhs));
    RTM_CUDA(cudaMemsetAsync(cnt.ptr, 0, cnt.bytes, s));
    RTM_CUDA(cudaMemsetAsync(done.ptr, 0, done.bytes, s));
    RTM_CUDA(cudaMemsetAsync(conv.ptr, 0, conv.bytes, s));
    k_fill<<<64, 256, 0, s>>>(hist.as<double>(), (int64_t)hs * nrhs, NAN);
    count_launch();
    RTM_TRY(A64->reserve(nrhs));
    RTM_TRY(A32->reserve(nrhs));
    if (M32) RTM_TRY(M32->reserve(nrhs));
    const bool inner_cg = cfg.method == RTM_METHOD_CG;
    if (x0) RTM_CUDA(cudaMemcpyAsync(x, x0, vec64, cudaMemcpyDeviceToDevice, s));
    else RTM_CUDA(cudaMemsetAsync(x, 0, vec64, s));
    int inner_total = 0, steps = 0;
    res.matvecs = 0;
    std::vector<int> hd(nrhs);
    std::vector<double2> hr(nrhs), hr_prev(nrhs);
    std::vector<double> inner_tol(nrhs);
    bool fallback = false;
    for (int step = 0;; ++step) {
        RTM_TRY(A64->apply(x, t64.ptr, nrhs, s, SkipFlags{}));
        k_residual<double2><<<grid, kRT, 0, s>>>(b, t64.as<double2>(), r64.as<double2>(), n, nullptr, 0);
        k_true_residual<double2><<<grid, kRT, 0, s>>>(b, t64.as<double2>(), n, part.as<double2>(),
                                                      cnt.as<unsigned int>(), resb.as<double2>());
        k_ir_check<<<(nrhs + 31) / 32, 32, 0, s>>>(resb.as<double2>(), done.as<int>(), conv.as<int>(),
                                                   hist.as<double>(), hs, step, cfg.tolerance, nrhs);
        count_launch(3);
        res.matvecs += 1;
        RTM_CUDA(cudaMemcpyAsync(hd.data(), done.ptr, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, s));
        RTM_CUDA(cudaMemcpyAsync(hr.data(), resb.ptr, sizeof(double2) * nrhs, cudaMemcpyDeviceToHost, s));
        RTM_CUDA(cudaStreamSynchronize(s));
        steps = step;
        bool all = true, stalled = false;
        for (int k = 0; k < nrhs; ++k) {
            all = all && hd[k];
            // a step that leaves a right-hand side's FP64 residual above half of what it was
            if (step > 0 && !hd[k] && hr[k].x > 0.5 * hr_prev[k].x) stalled = true;
        }
        hr_prev = hr;
        if (all || (cfg.cancel && *cfg.cancel)) break;
        if (cfg.fallback_fp64 && stalled) {
            fallback = true;
            break;
        }
        if (step >= cfg.max_refinements || inner_total >= cfg.max_iterations) break;
        k_ir_to32<<<grid, kRT, 0, s>>>(r64.as<double2>(), r32.as<float2>(), n, resb.as<double2>(), done.as<int>());
        count_launch();
        // The inner FP32 solve of A32 d = r / ||r||: COCG, or restarted flexible GMRES(m).
        for (int k = 0; k < nrhs; ++k) {
            const double need = hr[k].x > 0 ? 0.5 * cfg.tolerance * hr[k].y / hr[k].x : 0.5;
            inner_tol[k] = std::max(cfg.inner_tolerance, std::min(0.5, need));
        }
        SolveConfig ic;
        ic.method = inner_cg ? RTM_METHOD_CG : RTM_METHOD_GMRES;
        ic.tolerance = cfg.inner_tolerance;
        ic.tolerances = inner_tol.data();
        ic.max_iterations = std::max(1, cfg.max_iterations - inner_total);
        if (cfg.inner_max_iterations > 0) ic.max_iterations = std::min(ic.max_iterations, cfg.inner_max_iterations);
        ic.restart = m;
        ic.check_every = cfg.check_every;
        ic.right_preconditioned = 1;
        ic.gram_schmidt_passes = cfg.inner_gram_schmidt_passes;
        ic.cancel = cfg.cancel;
        SolveResult ir;
        if (inner_cg) RTM_TRY(cocg<float>(A32, M32, ic, r32.ptr, nullptr, d32.ptr, n, nrhs, ir, s));
        else RTM_TRY(gmres<float>(A32, M32, ic, r32.ptr, nullptr, d32.ptr, n, nrhs, ir, s));
        int most = 0;
        for (auto& st : ir.stats) most = std::max(most, st.iteration_count);
        inner_total += most;
        res.matvecs += ir.matvecs + most + 1;
        k_ir_update<<<grid, kRT, 0, s>>>(x, d32.as<float2>(), n, resb.as<double2>(), done.as<int>());
        count_launch();
    }
    if (fallback) {
        // the FP32 inner solves stopped making progress: finish every right-hand side in FP64 from the current
        // iterate (those already converged stop at once, their first residual meeting the tolerance)
        DeviceBuffer xs;
        RTM_TRY(xs.alloc(vec64));
        RTM_CUDA(cudaMemcpyAsync(xs.ptr, x, vec64, cudaMemcpyDeviceToDevice, s));
        SolveConfig fc = cfg;
        fc.method = inner_cg ? RTM_METHOD_CG : RTM_METHOD_GMRES;
        fc.tolerances = nullptr;
        fc.max_iterations = std::max(1, cfg.max_iterations - inner_total);
        fc.restart = m;
        fc.right_preconditioned = 1;
        SolveResult fr;
        RTM_TRY(solve(A64, M64, fc, b, xs.ptr, x, n, nrhs, fr, s));
        res.history = fr.history;
        res.hist_stride = fr.hist_stride;
        res.matvecs += fr.matvecs;
        res.stats = fr.stats;
        for (auto& o : res.stats) {
            o.iteration_count += inner_total;
            o.refinements = steps;
            o.matvecs = res.matvecs;
        }
        return RTM_OK;
    }
    std::vector<double2> rb(nrhs);
    std::vector<int> hc(nrhs);
    RTM_CUDA(cudaMemcpyAsync(rb.data(), resb.ptr, sizeof(double2) * nrhs, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaMemcpyAsync(hc.data(), conv.ptr, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, s));
    res.history.resize((size_t)hs * nrhs);
    RTM_CUDA(cudaMemcpyAsync(res.history.data(), hist.ptr, hist.bytes, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    // IterativeMethod.m:53-56: the solution of a zero right-hand side is zero, whatever the initial guess
    std::vector<int> zero(nrhs);
    bool any_zero = false;
    for (int k = 0; k < nrhs; ++k) any_zero |= (zero[k] = rb[k].y == 0.0) != 0;
    if (any_zero) {
        RTM_CUDA(cudaMemcpyAsync(done.ptr, zero.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, s));
        k_zero_where<double2><<<grid, kRT, 0, s>>>(x, n, done.as<int>(), 1);
        count_launch();
        RTM_CUDA(cudaStreamSynchronize(s));
    }
    RTM_TRY(device_fault_check(s));
    res.hist_stride = hs;
    res.stats.resize(nrhs);
    for (int k = 0; k < nrhs; ++k) {
        rtm_solve_stats& o = res.stats[k];
        o.converged = hc[k];
        o.iteration_count = zero[k] ? 0 : inner_total;
        o.residual_norm = rb[k].y == 0 ? 0.0 : rb[k].x / rb[k].y;
        o.refinements = zero[k] ? 0 : steps;
        o.matvecs = res.matvecs;
    }
    return RTM_OK;
}

int solve(LinearOp* A, LinearOp* M, const SolveConfig& cfg, const void* b, const void* x0, void* x, int64_t n, int nrhs,
          SolveResult& res, cudaStream_t s) {
    if (cfg.method == RTM_METHOD_CG)
        return A->precision == RTM_FP64 ? cocg<double>(A, M, cfg, b, x0, x, n, nrhs, res, s)
                                        : cocg<float>(A, M, cfg, b, x0, x, n, nrhs, res, s);
    if (cfg.method == RTM_METHOD_GMRES)
        return A->precision == RTM_FP64 ? gmres<double>(A, M, cfg, b, x0, x, n, nrhs, res, s)
                                        : gmres<float>(A, M, cfg, b, x0, x, n, nrhs, res, s);
    return fail(RTM_ERR_ARG, "unknown solver method");
}

}  // namespace rtm
