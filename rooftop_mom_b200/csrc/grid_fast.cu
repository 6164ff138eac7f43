// Power-of-two split products with register-resident line transforms.
//
// The same product as k_grid_y_fwd / k_grid_x_mix / k_grid_y_inv in grid.cu (the reference's
// src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/applyBothDirections_.m:14-85) for
// transform sizes that are powers of two. A line of n = R1 R2 points is transformed by a group of R2
// threads, each holding R1 values in registers (four-step form, decimation in time):
//   thread m2 holds x[R2 m1 + m2], m1 < R1
//   -> R1-point DFT over m1 in registers -> twiddle w_n^(m2 k1)
//   -> one exchange through shared memory
//   -> R1 / R2 DFTs of R2 points over m2 -> X[k1 + R1 k2], thread t holding k1 = t + R2 s (s < R1 / R2)
//      for every k2, at register s R2 + k2.
// The inverse runs the same steps backwards from that layout. The x-mix multiplies the spectra in this
// layout without reordering; every global load and store is coalesced (consecutive threads touch
// consecutive elements). The line buffers are padded (row stride R2 + 1) against bank conflicts.
#include <algorithm>

#include "grid.h"
#include "grid_args.cuh"
#include "bulk.cuh"
#include "pdl.cuh"

namespace rtm {
namespace {

// CTA size: FP32 256 threads, FP64 128. How many CTAs an SM holds (the launch bound, which sets the
// registers a thread may use) is part of the schedule a product runs with (FastSchedule, grid.h).
template <typename T> struct Fast {
    static constexpr int threads = sizeof(T) == 8 ? 128 : 256;
};

template <int N> struct Shape;
template <> struct Shape<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Shape<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Shape<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Shape<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Shape<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Shape<1024> { static constexpr int R1 = 32, R2 = 32; };

// cos(pi k / 16) for k = 0 .. 8 (the real parts of the 32nd roots of unity).
__host__ __device__ constexpr double cos_pi16(int k) {
    return k == 0 ? 1.0 : k == 1 ? 0.980785280403230449126182236134239 : k == 2 ? 0.923879532511286756128183189396788
         : k == 3 ? 0.831469612302545237078788377617906 : k == 4 ? 0.707106781186547524400844362104849
         : k == 5 ? 0.555570233019602224742830813948533 : k == 6 ? 0.382683432365089771728459984030399
         : k == 7 ? 0.195090322016128267848284868477022 : 0.0;
}
// The forward root w_32^k = exp(-i pi k / 16) = (cos, -sin), k < 16, as compile-time constants.
__host__ __device__ constexpr double root32_re(int k) { return k <= 8 ? cos_pi16(k) : -cos_pi16(16 - k); }
__host__ __device__ constexpr double root32_im(int k) { return k <= 8 ? -cos_pi16(8 - k) : -cos_pi16(k - 8); }

// In-register DFT of R points, natural order in and out. R = 32 splits by decimation in frequency
// into two 16-point transforms with the roots w_32^k (constants, no table reads).
template <int R, bool INV, typename T2>
__device__ __forceinline__ void dft_reg(T2 (&v)[R], const T2* __restrict__ tw, int n) {
    if constexpr (R == 4) {
        dft4<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (R == 8) {
        dft8<INV>(v);
    } else if constexpr (R == 16) {
        dft16<INV>(v);
    } else {
        static_assert(R == 32, "radix");
        using S = decltype(v[0].x);
        T2 a[16], b[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            a[k] = cadd(v[k], v[k + 16]);
            b[k] = csub(v[k], v[k + 16]);
            if (k) b[k] = twc<INV>(b[k], (S)root32_re(k), (S)root32_im(k));
        }
        dft16<INV>(a);
        dft16<INV>(b);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            v[2 * k] = a[k];
            v[2 * k + 1] = b[k];
        }
    }
}

template <typename T2> __device__ __forceinline__ T2 make_vec2(decltype(T2{}.x) x, decltype(T2{}.x) y) {
    T2 r;
    r.x = x;
    r.y = y;
    return r;
}

// Element (r, c) of a line buffer at base[r * RS + c * CS].
template <typename T2> struct LineBuf {
    T2* base;
    int RS, CS;
    __device__ __forceinline__ T2& at(int r, int c) const { return base[r * RS + c * CS]; }
};

// Forward transform of the group's line, steps before the exchange: v[m1] = x[R2 m1 + t] in,
// written to buf(k1, t).
template <int N, typename T2>
__device__ __forceinline__ void fwd_first(T2 (&v)[Shape<N>::R1], int t, const T2* __restrict__ tw,
                                          const LineBuf<T2>& buf) {
    constexpr int R1 = Shape<N>::R1;
    dft_reg<R1, false>(v, tw, N);
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        const T2 w = k1 ? cmul(v[k1], __ldg(&tw[t * k1])) : v[k1];
        buf.at(k1, t) = w;
    }
}

// After the exchange: v[s R2 + k2] = X[(t + R2 s) + R1 k2].
template <int N, typename T2>
__device__ __forceinline__ void fwd_second(T2 (&v)[Shape<N>::R1], int t, const T2* __restrict__ tw,
                                           const LineBuf<T2>& buf) {
    constexpr int R1 = Shape<N>::R1, R2 = Shape<N>::R2, S = R1 / R2;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        T2 u[R2];
#pragma unroll
        for (int m2 = 0; m2 < R2; ++m2) u[m2] = buf.at(t + R2 * s, m2);
        dft_reg<R2, false>(u, tw, N);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[s * R2 + k2] = u[k2];
    }
}

// Inverse from the transformed layout, steps before the exchange: written to buf(k1, m2) twiddled.
template <int N, typename T2>
__device__ __forceinline__ void inv_first(T2 (&v)[Shape<N>::R1], int t, const T2* __restrict__ tw,
                                          const LineBuf<T2>& buf) {
    constexpr int R1 = Shape<N>::R1, R2 = Shape<N>::R2, S = R1 / R2;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        T2 u[R2];
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) u[k2] = v[s * R2 + k2];
        dft_reg<R2, true>(u, tw, N);
        const int k1 = t + R2 * s;
#pragma unroll
        for (int m2 = 0; m2 < R2; ++m2) buf.at(k1, m2) = (m2 && k1) ? cmulc(u[m2], __ldg(&tw[m2 * k1])) : u[m2];
    }
}

// After the exchange: v[m1] = N x[R2 m1 + t] (unnormalised).
template <int N, typename T2>
__device__ __forceinline__ void inv_second(T2 (&v)[Shape<N>::R1], int t, const T2* __restrict__ tw,
                                           const LineBuf<T2>& buf) {
    constexpr int R1 = Shape<N>::R1;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) v[k1] = buf.at(k1, t);
    dft_reg<R1, true>(v, tw, N);
}

// --------------------------------------------------------------------------------------------
// y-forward: TI x-columns of one component; a group per (column, y subband). Thread index
// l + TI (py + 2 t): consecutive threads take consecutive columns, so rows of TI elements are read
// and written at once. W[py][c][k][i] = FFT_y(x_c(i, j) mod_y(j)^py).
template <typename T, int NQ, int MINB>
__global__ void __launch_bounds__(Fast<T>::threads, MINB) k_fast_y_fwd(const GridArgs<T> a, const typename Cx<T>::T2* __restrict__ x) {
    using T2 = typename Cx<T>::T2;
    constexpr int R1 = Shape<NQ>::R1, R2 = Shape<NQ>::R2, TI = Fast<T>::threads / (2 * R2), G = 2 * TI;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* sm = reinterpret_cast<T2*>(smem_raw);
    griddep_wait();
    griddep_launch_dependents();
    const int c = blockIdx.y, rhs = blockIdx.z;
    if (skipped(a, rhs)) return;
    const PlateDesc<T> pd = plate_of(a, rhs);
    const int rows = pd.rows[c], cols = pd.cols[c];
    if ((int)blockIdx.x * TI >= rows) return;  // a smaller plate of a batch
    const int l = threadIdx.x % TI, py = (threadIdx.x / TI) % 2, t = threadIdx.x / (2 * TI);
    const int g = l + TI * py;
    const int i = blockIdx.x * TI + l;
    const bool on = i < rows;
    const LineBuf<T2> buf{sm + g, (R2 + 1) * G, G};
    const T2* xr = x + (int64_t)rhs * a.n + pd.off[c];
    T2 v[R1];
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
        const int j = R2 * m1 + t;
        T2 e = (on && j < cols) ? xr[i + (int64_t)j * rows] : czero<T2>();
        if (py) e = cmul(e, __ldg(&a.modQ[j]));
        v[m1] = e;
    }
    fwd_first<NQ>(v, t, a.twQ, buf);
    __syncthreads();
    fwd_second<NQ>(v, t, a.twQ, buf);
    if (!on) return;
    T2* dst = a.work + (int64_t)rhs * a.work_rhs + (int64_t)(py * a.ncomp + c) * NQ * a.P + i;
#pragma unroll
    for (int s = 0; s < R1 / R2; ++s)
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) dst[(int64_t)((t + R2 * s) + R1 * k2) * a.P] = v[s * R2 + k2];
}

// x-mix, direct form (one CTA per TEAMS y frequencies; inputs loaded straight into registers, the spectra
// read in the mix): teams of four groups (component c, x subband px) per y frequency j of subband py. Thread
// index t + R2 (team * 4 + 2 px + c). Forward transform along x of W mod_x^px, the 2x2 block mix
// with the subband spectra (the two components of a group pair meet through shared memory), inverse
// transform, demodulation, the sum over px, scaled by 1 / (PQ), in place in W.
template <typename T, int NP, int MINB>
__global__ void __launch_bounds__(Fast<T>::threads, MINB) k_fast_x_mix_direct(const GridArgs<T> a) {
    using T2 = typename Cx<T>::T2;
    constexpr int R1 = Shape<NP>::R1, R2 = Shape<NP>::R2, S = R1 / R2;
    constexpr int TEAMS = Fast<T>::threads / (4 * R2), LB = R1 * (R2 + 1);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* sm = reinterpret_cast<T2*>(smem_raw);
    griddep_wait();
    griddep_launch_dependents();
    const int py = blockIdx.y, rhs = blockIdx.z;
    if (skipped(a, rhs)) return;
    const PlateDesc<T> pd = plate_of(a, rhs);
    const int t = threadIdx.x % R2, gid = threadIdx.x / R2;
    const int team = gid / 4, c = gid % 2, px = (gid / 2) % 2;
    const int j = blockIdx.x * TEAMS + team;
    const bool on = j < a.Q;
    const int Q = a.Q;
    const int64_t QP = (int64_t)Q * NP;
    const LineBuf<T2> buf{sm + gid * LB, R2 + 1, 1};
    T2* own = sm + gid * LB;
    const T2* partner = sm + (gid ^ 1) * LB;
    const int rows = pd.rows[c];
    T2* row = a.work + (int64_t)rhs * a.work_rhs + (int64_t)(py * a.ncomp + c) * QP + (int64_t)(on ? j : 0) * NP;
    T2 v[R1];
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
        const int i = R2 * m1 + t;
        T2 e = (on && i < rows) ? row[i] : czero<T2>();
        if (px) e = cmul(e, __ldg(&a.modP[i]));
        v[m1] = e;
    }
    fwd_first<NP>(v, t, a.twP, buf);
    __syncthreads();
    fwd_second<NP>(v, t, a.twP, buf);
    __syncthreads();  // the buffers are read; they now carry the spectra values to the partner
#pragma unroll
    for (int r = 0; r < R1; ++r) own[r * R2 + t] = v[r];
    __syncthreads();
    if (on) {
        const int sub = px + 2 * py;
        const T2* spec = pd.spec + (int64_t)(sub * 3) * QP + (int64_t)j * NP;
        const T2* ux = px ? a.ux1 : a.ux0;
        const T2 vv = __ldg(&(py ? a.vy1 : a.vy0)[j]);
        const T cv = (vv.x * vv.x + vv.y * vv.y) * pd.inv_b2;
#pragma unroll
        for (int s = 0; s < S; ++s)
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) {
                const int k = (t + R2 * s) + R1 * k2;
                const T2 E = __ldg(&spec[k]);
                const T2 M = __ldg(&spec[(1 + c) * QP + k]);
                const T2 uu = __ldg(&ux[k]);
                const T cu = (uu.x * uu.x + uu.y * uu.y) * pd.inv_a2;
                // qc = -u conj(v) / (ab): XY = qc E, YX = conj(qc) E
                T2 qc = cmulc(uu, vv);
                qc.x = -qc.x * pd.inv_ab;
                qc.y = -qc.y * pd.inv_ab;
                const T2 coupling = c ? cconj(qc) : qc;
                const T cself = c ? cv : cu;
                const T2 me = v[s * R2 + k2], other = partner[(s * R2 + k2) * R2 + t];
                // M me - cself E me + coupling E other = M me + E (coupling other - cself me)
                const T2 cp = cmul(coupling, other);
                const T2 d = make_vec2<T2>(cp.x - cself * me.x, cp.y - cself * me.y);
                v[s * R2 + k2] = cadd(cmul(M, me), cmul(E, d));
            }
    }
    __syncthreads();  // the partner values are read
    inv_first<NP>(v, t, a.twP, buf);
    __syncthreads();
    inv_second<NP>(v, t, a.twP, buf);
    __syncthreads();
    if (px) {
#pragma unroll
        for (int m1 = 0; m1 < R1; ++m1) own[m1 * R2 + t] = cmulc(v[m1], __ldg(&a.modP[R2 * m1 + t]));
    }
    __syncthreads();
    if (px || !on) return;
    const T2* odd = sm + (gid + 2) * LB;
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
        const int i = R2 * m1 + t;
        if (i < rows) row[i] = cscale(cadd(v[m1], odd[m1 * R2 + t]), a.scale);
    }
}

// x-mix, pipelined form: persistent CTAs. A CTA takes the iterations it = blockIdx.x, blockIdx.x + gridDim.x, ...; an
// iteration is TEAMS consecutive y frequencies j of one (right-hand side, y subband py). Its inputs are
// copied into shared memory one iteration ahead by bulk asynchronous copies (one thread issues them): the
// W rows of both components (contiguous for consecutive j) as soon as the current ones are in registers,
// and the subband spectra rows (E, MXX, MYY of both x subbands) as soon as the current mix has read them,
// so the global-memory latency of both overlaps the transforms. Per y frequency, a team of four groups
// (component c, x subband px), thread index t + R2 (team * 4 + 2 px + c): forward transform along x of
// W mod_x^px, the 2x2 block mix with the subband spectra (the two components of a group pair meet through
// shared memory), inverse transform, demodulation, the sum over px, scaled by 1 / (PQ), in place in W.
// A bulk-copy wait that runs out records RTM_ERR_TIMEOUT in the fault word and ends the CTA.
template <typename T, int NP> struct MixShape {
    static constexpr int R1 = Shape<NP>::R1, R2 = Shape<NP>::R2;
    static constexpr int TEAMS = Fast<T>::threads / (4 * R2), LB = R1 * (R2 + 1);
    using T2 = typename Cx<T>::T2;
    // line buffers [4 TEAMS][LB], W rows [2 c][TEAMS][NP], spectra rows [2 px][3 kind][TEAMS][NP]
    static constexpr size_t lines = (size_t)4 * TEAMS * LB * sizeof(T2);
    static constexpr size_t wrows = (size_t)2 * TEAMS * NP * sizeof(T2);
    static constexpr size_t srows = (size_t)6 * TEAMS * NP * sizeof(T2);
    static constexpr size_t smem = lines + wrows + srows;
    static constexpr int blocks = 2 * smem <= 220 * 1024 ? 2 : 1;  // CTAs per SM the registers are sized for
};

template <typename T, int NP>
__global__ void __launch_bounds__(Fast<T>::threads, (MixShape<T, NP>::blocks)) k_fast_x_mix_pipe(const GridArgs<T> a, int iters) {
    using M = MixShape<T, NP>;
    using T2 = typename Cx<T>::T2;
    constexpr int R1 = M::R1, R2 = M::R2, S = R1 / R2, TEAMS = M::TEAMS, LB = M::LB;
    constexpr unsigned BLOCK = TEAMS * NP * sizeof(T2);  // TEAMS consecutive rows of one grid
    static_assert(BLOCK % 16 == 0 && M::lines % 16 == 0 && M::wrows % 16 == 0, "bulk copies need 16-byte units");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* sm = reinterpret_cast<T2*>(smem_raw);
    T2* wst = reinterpret_cast<T2*>(smem_raw + M::lines);
    T2* sst = reinterpret_cast<T2*>(smem_raw + M::lines + M::wrows);
    __shared__ __align__(8) uint64_t bar[2];  // 0: W rows, 1: spectra rows
    griddep_wait();
    griddep_launch_dependents();
    const int Q = a.Q, per_py = Q / TEAMS, per_rhs = 2 * per_py;
    const int64_t QP = (int64_t)Q * NP;
    const int tid = threadIdx.x;
    const int t = tid % R2, gid = tid / R2;
    const int team = gid / 4, c = gid % 2, px = (gid / 2) % 2;
    auto live = [&](int it) {
        while (it < iters && skipped(a, it / per_rhs)) it += gridDim.x;
        return it;
    };
    // copies issued (thread 0) and barrier phases completed (every thread), per barrier
    unsigned issued[2] = {0, 0}, done[2] = {0, 0};
    auto issue = [&](int it, bool w, bool spectra) {
        const int rhs = it / per_rhs, r = it % per_rhs, py = r / per_py, j0 = (r % per_py) * TEAMS;
        if (w) {
            ++issued[0];
            mbar_expect_tx(&bar[0], 2 * BLOCK);
            for (int cc = 0; cc < 2; ++cc)
                bulk_load(wst + cc * TEAMS * NP,
                          a.work + rhs * a.work_rhs + (int64_t)(py * a.ncomp + cc) * QP + (int64_t)j0 * NP, BLOCK,
                          &bar[0]);
        }
        if (spectra) {
            ++issued[1];
            mbar_expect_tx(&bar[1], 6 * BLOCK);
            const T2* sp = a.plates ? a.plates[rhs].spec : a.spec;
            for (int q = 0; q < 2; ++q)
                for (int kind = 0; kind < 3; ++kind)
                    bulk_load(sst + (q * 3 + kind) * TEAMS * NP,
                              sp + (int64_t)((q + 2 * py) * 3 + kind) * QP + (int64_t)j0 * NP, BLOCK, &bar[1]);
        }
    };
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_fence_init();
    }
    __syncthreads();
    int it = live(blockIdx.x);
    if (tid == 0 && it < iters) issue(it, true, true);
    const LineBuf<T2> buf{sm + gid * LB, R2 + 1, 1};
    T2* own = sm + gid * LB;
    const T2* partner = sm + (gid ^ 1) * LB;
    const T2* odd = sm + (gid + 2) * LB;
    const T2* ux = px ? a.ux1 : a.ux0;
    while (it < iters) {
        const int nxt = live(it + gridDim.x);
        const int rhs = it / per_rhs, r = it % per_rhs, py = r / per_py, j = (r % per_py) * TEAMS + team;
        const PlateDesc<T> pd = plate_of(a, rhs);
        const int rows = pd.rows[c];
        if (__syncthreads_or(!mbar_wait(&bar[0], done[0] & 1, a.fault))) break;
        ++done[0];
        T2 v[R1];
        const T2* wrow = wst + (c * TEAMS + team) * NP;
#pragma unroll
        for (int m1 = 0; m1 < R1; ++m1) {
            const int i = R2 * m1 + t;
            T2 e = i < rows ? wrow[i] : czero<T2>();
            if (px) e = cmul(e, __ldg(&a.modP[i]));
            v[m1] = e;
        }
        __syncthreads();  // the W rows are in registers: the next iteration's may come in
        if (tid == 0 && nxt < iters) issue(nxt, true, false);
        fwd_first<NP>(v, t, a.twP, buf);
        __syncthreads();
        fwd_second<NP>(v, t, a.twP, buf);
        __syncthreads();  // the buffers are read; they now carry the spectra values to the partner
#pragma unroll
        for (int q = 0; q < R1; ++q) own[q * R2 + t] = v[q];
        if (__syncthreads_or(!mbar_wait(&bar[1], done[1] & 1, a.fault))) break;
        ++done[1];
        {
            const T2* Es = sst + (px * 3 * TEAMS + team) * NP;
            const T2* Ms = sst + ((px * 3 + 1 + c) * TEAMS + team) * NP;
            const T2 vv = __ldg(&(py ? a.vy1 : a.vy0)[j]);
            const T cv = (vv.x * vv.x + vv.y * vv.y) * pd.inv_b2;
#pragma unroll
            for (int s = 0; s < S; ++s)
#pragma unroll
                for (int k2 = 0; k2 < R2; ++k2) {
                    const int k = (t + R2 * s) + R1 * k2;
                    const T2 E = Es[k];
                    const T2 Mk = Ms[k];
                    const T2 uu = __ldg(&ux[k]);
                    const T cu = (uu.x * uu.x + uu.y * uu.y) * pd.inv_a2;
                    // qc = -u conj(v) / (ab): XY = qc E, YX = conj(qc) E
                    T2 qc = cmulc(uu, vv);
                    qc.x = -qc.x * pd.inv_ab;
                    qc.y = -qc.y * pd.inv_ab;
                    const T2 coupling = c ? cconj(qc) : qc;
                    const T cself = c ? cv : cu;
                    const T2 me = v[s * R2 + k2], other = partner[(s * R2 + k2) * R2 + t];
                    // Mk me - cself E me + coupling E other = Mk me + E (coupling other - cself me)
                    const T2 cp = cmul(coupling, other);
                    const T2 d = make_vec2<T2>(cp.x - cself * me.x, cp.y - cself * me.y);
                    v[s * R2 + k2] = cadd(cmul(Mk, me), cmul(E, d));
                }
        }
        __syncthreads();  // the spectra and the partner values are read
        if (tid == 0 && nxt < iters) issue(nxt, false, true);
        inv_first<NP>(v, t, a.twP, buf);
        __syncthreads();
        inv_second<NP>(v, t, a.twP, buf);
        __syncthreads();
        if (px) {
#pragma unroll
            for (int m1 = 0; m1 < R1; ++m1) own[m1 * R2 + t] = cmulc(v[m1], __ldg(&a.modP[R2 * m1 + t]));
        }
        __syncthreads();
        if (!px) {
            T2* row = a.work + rhs * a.work_rhs + (int64_t)(py * a.ncomp + c) * QP + (int64_t)j * NP;
#pragma unroll
            for (int m1 = 0; m1 < R1; ++m1) {
                const int i = R2 * m1 + t;
                if (i < rows) row[i] = cscale(cadd(v[m1], odd[m1 * R2 + t]), a.scale);
            }
        }
        it = nxt;
    }
    // A wait ran out: let the copies still in flight into this CTA's shared memory land (each wait
    // bounded) before the CTA ends.
    if (tid == 0)
        for (int q = 0; q < 2; ++q)
            for (; done[q] < issued[q]; ++done[q]) mbar_wait(&bar[q], done[q] & 1, nullptr);
}

// y-inverse: TI columns of one component, a group per (column, y subband); inverse transform along y,
// demodulation, the sum over py through shared memory, cropped into y.
template <typename T, int NQ, int MINB>
__global__ void __launch_bounds__(Fast<T>::threads, MINB) k_fast_y_inv(const GridArgs<T> a, typename Cx<T>::T2* __restrict__ y) {
    using T2 = typename Cx<T>::T2;
    constexpr int R1 = Shape<NQ>::R1, R2 = Shape<NQ>::R2, TI = Fast<T>::threads / (2 * R2), G = 2 * TI;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* sm = reinterpret_cast<T2*>(smem_raw);
    griddep_wait();
    griddep_launch_dependents();
    const int c = blockIdx.y, rhs = blockIdx.z;
    if (skipped(a, rhs)) return;
    const PlateDesc<T> pd = plate_of(a, rhs);
    const int rows = pd.rows[c], cols = pd.cols[c];
    if ((int)blockIdx.x * TI >= rows) return;  // a smaller plate of a batch
    const int l = threadIdx.x % TI, py = (threadIdx.x / TI) % 2, t = threadIdx.x / (2 * TI);
    const int g = l + TI * py;
    const int i = blockIdx.x * TI + l;
    const bool on = i < rows;
    const LineBuf<T2> buf{sm + g, (R2 + 1) * G, G};
    const T2* src = a.work + (int64_t)rhs * a.work_rhs + (int64_t)(py * a.ncomp + c) * NQ * a.P + (on ? i : 0);
    T2 v[R1];
#pragma unroll
    for (int s = 0; s < R1 / R2; ++s)
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2)
            v[s * R2 + k2] = on ? src[(int64_t)((t + R2 * s) + R1 * k2) * a.P] : czero<T2>();
    inv_first<NQ>(v, t, a.twQ, buf);
    __syncthreads();
    inv_second<NQ>(v, t, a.twQ, buf);
    __syncthreads();
    if (py) {
#pragma unroll
        for (int m1 = 0; m1 < R1; ++m1) buf.at(m1, t) = cmulc(v[m1], __ldg(&a.modQ[R2 * m1 + t]));
    }
    __syncthreads();
    if (py || !on) return;
    const LineBuf<T2> odd{sm + g + TI, (R2 + 1) * G, G};
    T2* yr = y + (int64_t)rhs * a.n + pd.off[c];
#pragma unroll
    for (int m1 = 0; m1 < R1; ++m1) {
        const int j = R2 * m1 + t;
        if (j < cols) yr[i + (int64_t)j * rows] = cadd(v[m1], odd.at(m1, t));
    }
}

template <typename T, int NQ> size_t y_smem() {
    constexpr int R1 = Shape<NQ>::R1, R2 = Shape<NQ>::R2, TI = Fast<T>::threads / (2 * R2);
    return (size_t)2 * TI * R1 * (R2 + 1) * sizeof(typename Cx<T>::T2);
}
template <typename T, int NQ, int MINB> int launch_y_b(const GridArgs<T>& a, int nrhs, const void* x, void* y,
                                                       bool fwd, cudaStream_t s) {
    using T2 = typename Cx<T>::T2;
    constexpr int TI = Fast<T>::threads / (2 * Shape<NQ>::R2);
    const size_t smem = y_smem<T, NQ>();
    static DeviceOnce once;
    RTM_TRY(once([smem]() -> int {
        RTM_CUDA(cudaFuncSetAttribute(k_fast_y_fwd<T, NQ, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        RTM_CUDA(cudaFuncSetAttribute(k_fast_y_inv<T, NQ, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        return RTM_OK;
    }));
    const int rows_max = a.rows[0] > a.rows[1] ? a.rows[0] : a.rows[1];
    const dim3 grid((rows_max + TI - 1) / TI, 2, nrhs);
    if (fwd)
        k_fast_y_fwd<T, NQ, MINB><<<grid, Fast<T>::threads, smem, s>>>(a, static_cast<const T2*>(x));
    else
        RTM_CUDA(launch_dependent(k_fast_y_inv<T, NQ, MINB>, grid, dim3(Fast<T>::threads), smem, s, a,
                                  static_cast<T2*>(y)));
    count_launch();
    return RTM_OK;
}

template <typename T, int NQ> int launch_y(const GridArgs<T>& a, int nrhs, const void* x, void* y, bool fwd,
                                           int minb, cudaStream_t s) {
    if (minb <= 1) return launch_y_b<T, NQ, 1>(a, nrhs, x, y, fwd, s);
    if constexpr (sizeof(T) == 8) {
        if (minb >= 3) return launch_y_b<T, NQ, 3>(a, nrhs, x, y, fwd, s);
    }
    return launch_y_b<T, NQ, 2>(a, nrhs, x, y, fwd, s);
}

template <typename T, int NP> size_t x_direct_smem() {
    constexpr int R1 = Shape<NP>::R1, R2 = Shape<NP>::R2, TEAMS = Fast<T>::threads / (4 * R2);
    return (size_t)4 * TEAMS * R1 * (R2 + 1) * sizeof(typename Cx<T>::T2);
}

template <typename T, int NP, int MINB> int launch_x_direct(const GridArgs<T>& a, int nrhs, cudaStream_t s) {
    constexpr int TEAMS = Fast<T>::threads / (4 * Shape<NP>::R2);
    const size_t smem = x_direct_smem<T, NP>();
    static DeviceOnce once;
    RTM_TRY(once([smem]() -> int {
        RTM_CUDA(cudaFuncSetAttribute(k_fast_x_mix_direct<T, NP, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        return RTM_OK;
    }));
    const dim3 grid((a.Q + TEAMS - 1) / TEAMS, 2, nrhs);
    RTM_CUDA(launch_dependent(k_fast_x_mix_direct<T, NP, MINB>, grid, dim3(Fast<T>::threads), smem, s, a));
    count_launch();
    return RTM_OK;
}

template <typename T, int NP> int launch_x_pipe(const GridArgs<T>& a, int nrhs, cudaStream_t s) {
    using M = MixShape<T, NP>;
    static DeviceOnce once;
    static int per_sm[64] = {};
    int dev = 0;
    RTM_CUDA(cudaGetDevice(&dev));
    RTM_TRY(once([dev]() -> int {
        RTM_CUDA(cudaFuncSetAttribute(k_fast_x_mix_pipe<T, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)M::smem));
        int blocks = 0, sms = 0;
        RTM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_fast_x_mix_pipe<T, NP>, Fast<T>::threads,
                                                               M::smem));
        RTM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        if (dev >= 0 && dev < 64) per_sm[dev] = std::max(1, blocks) * sms;
        return RTM_OK;
    }));
    const int iters = nrhs * 2 * (a.Q / M::TEAMS);
    const int resident = dev >= 0 && dev < 64 && per_sm[dev] > 0 ? per_sm[dev] : 148;
    const int grid = std::max(1, std::min(iters, resident));
    RTM_CUDA(launch_dependent(k_fast_x_mix_pipe<T, NP>, dim3(grid), dim3(Fast<T>::threads), M::smem, s, a, iters));
    count_launch();
    return RTM_OK;
}

template <typename T, int NP> int launch_x(const GridArgs<T>& a, int nrhs, int kind, cudaStream_t s) {
    if (kind == kMixPipelined) return launch_x_pipe<T, NP>(a, nrhs, s);
    if (kind == kMixDirect2) return launch_x_direct<T, NP, 2>(a, nrhs, s);
    if constexpr (sizeof(T) == 8) {
        if (kind == kMixDirect3) return launch_x_direct<T, NP, 3>(a, nrhs, s);
    }
    return launch_x_direct<T, NP, 1>(a, nrhs, s);
}

template <typename T> int dispatch_y(const GridArgs<T>& a, int nrhs, const void* x, void* y, bool fwd, int minb,
                                     cudaStream_t s) {
    switch (a.Q) {
        case 32: return launch_y<T, 32>(a, nrhs, x, y, fwd, minb, s);
        case 64: return launch_y<T, 64>(a, nrhs, x, y, fwd, minb, s);
        case 128: return launch_y<T, 128>(a, nrhs, x, y, fwd, minb, s);
        case 256: return launch_y<T, 256>(a, nrhs, x, y, fwd, minb, s);
        case 512: return launch_y<T, 512>(a, nrhs, x, y, fwd, minb, s);
        default:
            if constexpr (sizeof(T) == 4) return launch_y<T, 1024>(a, nrhs, x, y, fwd, minb, s);
            return fail(RTM_ERR_UNSUPPORTED, "transform size");
    }
}

template <typename T> int dispatch_x(const GridArgs<T>& a, int nrhs, int kind, cudaStream_t s) {
    switch (a.P) {
        case 32: return launch_x<T, 32>(a, nrhs, kind, s);
        case 64: return launch_x<T, 64>(a, nrhs, kind, s);
        case 128: return launch_x<T, 128>(a, nrhs, kind, s);
        case 256: return launch_x<T, 256>(a, nrhs, kind, s);
        case 512: return launch_x<T, 512>(a, nrhs, kind, s);
        default:
            if constexpr (sizeof(T) == 4) return launch_x<T, 1024>(a, nrhs, kind, s);
            return fail(RTM_ERR_UNSUPPORTED, "transform size");
    }
}

}  // namespace

bool fast_split_eligible(int P, int Q, bool fp64) {
    auto ok = [&](int n) { return n >= 32 && n <= (fp64 ? 512 : 1024) && (n & (n - 1)) == 0; };
    return ok(P) && ok(Q);
}

FastSchedule default_fast_schedule(int P, int Q, bool fp64) {
    FastSchedule f;
    // y passes: FP32 two CTAs of 256 threads an SM (128 registers, no spills up to lines of 1024); FP64
    // three CTAs of 128 threads below lines of 512, two at 512 (up to 255 registers).
    f.y_blocks = fp64 ? (Q >= 512 ? 2 : 3) : 2;
    // x-mix: the pipelined form at FP32 1024 (one CTA of 256 threads an SM either way, and 100 MB of spectra
    // that do not stay in L2 between products); elsewhere the direct form, which keeps more warps resident.
    if (!fp64 && P >= 1024) f.x_kind = kMixPipelined;
    else if (fp64) f.x_kind = P >= 512 ? kMixDirect1 : kMixDirect3;
    else f.x_kind = kMixDirect2;
    return f;
}

template <typename T>
int launch_fast_split(const GridArgs<T>& a, int nrhs, const void* x, void* y, const FastSchedule& f, cudaStream_t s) {
    RTM_TRY(dispatch_y<T>(a, nrhs, x, y, true, f.y_blocks, s));
    RTM_TRY(dispatch_x<T>(a, nrhs, f.x_kind, s));
    RTM_TRY(dispatch_y<T>(a, nrhs, x, y, false, f.y_blocks, s));
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

template int launch_fast_split<float>(const GridArgs<float>&, int, const void*, void*, const FastSchedule&,
                                      cudaStream_t);
template int launch_fast_split<double>(const GridArgs<double>&, int, const void*, void*, const FastSchedule&,
                                       cudaStream_t);

}  // namespace rtm
