// FFT products on the rooftop grid and the on-device spectra builders (see grid.h).
//
// Follows the reference's
//   src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/applyBothDirections_.m:14-85
//   src/+rooftopMoM/+assembler/+greensMatrix/@SplitFFTApplicator/applySingleDirection_.m:14-26
//   src/+rooftopMoM/+assembler/+greensMatrix/@LeanSplitFFTApplicator/applyBothDirections_.m:13-91
//   src/+rooftopMoM/+assembler/+greensMatrix/FFTApplicator.m:52-87
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateSubbandSpectra.m:20-77
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateEmbeddingSpectra.m:15-40
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateBlockSpectra.m:19-50
//   src/+rooftopMoM/+assembler/+preconditioner/generatePartwiseSpectra.m:16-30 (+ kernels, foldGenerator.m)
//   src/+rooftopMoM/+assembler/+greensMatrix/@Spectra/invert.m:12-20
//
// The subband spectra are computed as P x Q transforms of the folded, modulated embedding:
// frequency 2m + p of a period-2P sequence e is the length-P DFT of (e(d) + (-1)^p e(d + P)) w^(p d),
// w = exp(-i pi / P), which is the same number as subsampling the 2P x 2Q transform.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "fft.cuh"
#include "grid.h"
#include "grid_args.cuh"

namespace rtm {

static constexpr int kSmemBudget = 200 * 1024;
static constexpr int kMaxThreads = 256;  // CTA size of the FFT kernels (up to 255 registers a thread)

// GridArgs and skipped(): grid_args.cuh

// Copies the n roots of unity into shared memory (ordered before use by the caller's barrier).
template <typename T2> __device__ __forceinline__ void stage_roots(T2* dst, const T2* __restrict__ src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

constexpr int kBatch = 8;  // independent global loads a thread issues before it uses them

// --------------------------------------------------------------------------------------------
// y-forward: for a tile of TI x columns of component c, both y subbands at once:
// W[py][c][j][i] = FFT_y( x_c(i, j) mody(j)^py ). Shared tile A[sk(j)][L], L = npy TI lines,
// line pyi TI + l (grid: tiles x components x right-hand sides).
template <typename T, bool POW2>
__global__ void __launch_bounds__(kMaxThreads, sizeof(T) == 8 ? 1 : 2) k_grid_y_fwd(const GridArgs<T> a, const typename Cx<T>::T2* __restrict__ x) {
    using T2 = typename Cx<T>::T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TI = a.ti, Q = a.Q, L = a.npy * TI;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* tws = A + (size_t)L * fft_span(a.planQ);
    const int c = blockIdx.y, rhs = blockIdx.z;
    const int rows = a.rows[c], cols = a.cols[c];
    const int i0 = blockIdx.x * TI;
    if (i0 >= rows || skipped(a, rhs)) return;
    stage_roots(tws, a.twQ, Q);
    const T2* xr = x + (int64_t)rhs * a.n + a.off[c];
    const int total = TI * Q;
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
        T2 v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            const int l = it % TI, j = it / TI, i = i0 + l;
            v[u] = (it < total && i < rows && j < cols) ? xr[i + (int64_t)j * rows] : czero<T2>();
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            if (it >= total) break;
            const int l = it % TI, j = it / TI;
            T2* row = A + (size_t)sk(j) * L + l;
            if (a.npy == 2) {
                row[0] = v[u];
                row[TI] = cmul(v[u], __ldg(&a.modQ[j]));
            } else {
                row[0] = a.py0 ? cmul(v[u], __ldg(&a.modQ[j])) : v[u];
            }
        }
    }
    __syncthreads();
    fft_inplace<false, POW2>(A, L, 1, L, a.planQ, tws);
    T2* dst = a.work + (int64_t)rhs * a.work_rhs;
    for (int it = threadIdx.x; it < L * Q; it += blockDim.x) {
        const int l = it % L, j = it / L;
        const int pyi = l / TI, i = i0 + (l - pyi * TI);
        if (i < rows) dst[((int64_t)(pyi * a.ncomp + c) * Q + j) * a.P + i] = A[(size_t)sk(j) * L + l];
    }
}

// --------------------------------------------------------------------------------------------
// x-mix: CB y frequencies j of the y subband py; for both components and both x subbands at once
// (line (jj nsx + px) nc + c): sum over px of demod_x^px IFFT_x( B(px, py) FFT_x( W mod_x^px ) ),
// scaled by 1/(PQ), in place in W. Line stride a.ls spreads the lines of a warp over the banks.
template <typename T, bool POW2>
__global__ void __launch_bounds__(kMaxThreads, sizeof(T) == 8 ? 1 : 2) k_grid_x_mix(const GridArgs<T> a) {
    using T2 = typename Cx<T>::T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P = a.P, Q = a.Q, nc = a.ncomp, CB = a.cb, ls = a.ls, nsx = a.nsx;
    const int lines = CB * nsx * nc;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* tws = A + (size_t)lines * ls;
    const int j0 = blockIdx.x * CB;
    const int pyi = blockIdx.y;
    const int py = a.py0 + pyi;
    const int rhs = blockIdx.z;
    if (skipped(a, rhs)) return;
    stage_roots(tws, a.twP, P);
    T2* wr = a.work + (int64_t)rhs * a.work_rhs + (int64_t)pyi * nc * Q * P;
    const int total = CB * nc * P;
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
        T2 v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            const int jc = it / P, i = it - jc * P;
            const int jj = jc / nc, c = jc - jj * nc, j = j0 + jj;
            v[u] = (it < total && i < a.rows[c] && j < Q) ? wr[((int64_t)c * Q + j) * P + i] : czero<T2>();
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            if (it >= total) break;
            const int jc = it / P, i = it - jc * P;
            const int jj = jc / nc, c = jc - jj * nc;
            A[(size_t)((jj * nsx) * nc + c) * ls + sk(i)] = v[u];
            if (nsx == 2) A[(size_t)((jj * nsx + 1) * nc + c) * ls + sk(i)] = cmul(v[u], __ldg(&a.modP[i]));
        }
    }
    __syncthreads();
    fft_inplace<false, POW2>(A, lines, ls, 1, a.planP, tws);
    const T2* vy = py ? a.vy1 : a.vy0;
    constexpr int kMix = 4;
    const int mtotal = CB * nsx * P;
    for (int base = threadIdx.x; base < mtotal; base += kMix * blockDim.x) {
        T2 e3[kMix][3];
#pragma unroll
        for (int u = 0; u < kMix; ++u) {
            const int it = base + u * blockDim.x;
            const int jp = it / P, i = it - jp * P;
            const int jj = jp / nsx, px = jp - jj * nsx, j = j0 + jj;
            const int sub = px + nsx * py;
            if (it < mtotal && j < Q) {
                if (a.mode == kGen3) {
                    const int64_t sb = ((int64_t)(sub * 3) * Q + j) * P + i;
                    e3[u][0] = __ldg(&a.spec[sb]);
                    e3[u][1] = __ldg(&a.spec[sb + (int64_t)Q * P]);
                    e3[u][2] = __ldg(&a.spec[sb + 2 * (int64_t)Q * P]);
                } else {
                    e3[u][0] = e3[u][1] = e3[u][2] = czero<T2>();
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kMix; ++u) {
            const int it = base + u * blockDim.x;
            if (it >= mtotal) break;
            const int jp = it / P, i = it - jp * P;
            const int jj = jp / nsx, px = jp - jj * nsx, j = j0 + jj;
            if (j >= Q) continue;
            T2* lx = A + (size_t)(jp * nc) * ls + sk(i);
            T2* ly = lx + ls;
            const T2 sx = *lx, sy = *ly;
            T2 ox, oy;
            if (a.mode == kGen3) {
                const T2 E = e3[u][0], Mx = e3[u][1], My = e3[u][2];
                const T2 uu = __ldg(&(px ? a.ux1 : a.ux0)[i]);
                const T2 vv = __ldg(&vy[j]);
                const T cu = (uu.x * uu.x + uu.y * uu.y) * a.inv_a2;
                const T cv = (vv.x * vv.x + vv.y * vv.y) * a.inv_b2;
                // qc = -u conj(v) / (ab): XY = qc E, YX = conj(qc) E.
                T2 qc = cmulc(uu, vv);
                qc.x = -qc.x * a.inv_ab;
                qc.y = -qc.y * a.inv_ab;
                const T2 Ex = cmul(E, sx), Ey = cmul(E, sy);
                ox = csub(cmul(Mx, sx), cscale(Ex, cu));
                ox = cadd(ox, cmul(qc, Ey));
                oy = csub(cmul(My, sy), cscale(Ey, cv));
                oy = cadd(oy, cmul(cconj(qc), Ex));
            } else {
                const int64_t sb = (int64_t)j * P + i, blk = (int64_t)Q * P;
                const T2 XX = __ldg(&a.spec[sb]), XY = __ldg(&a.spec[sb + blk]);
                const T2 YX = __ldg(&a.spec[sb + 2 * blk]), YY = __ldg(&a.spec[sb + 3 * blk]);
                ox = cadd(cmul(XX, sx), cmul(XY, sy));
                oy = cadd(cmul(YX, sx), cmul(YY, sy));
            }
            *lx = ox;
            *ly = oy;
        }
    }
    __syncthreads();
    fft_inplace<true, POW2>(A, lines, ls, 1, a.planP, tws);
    for (int it = threadIdx.x; it < CB * nc * P; it += blockDim.x) {
        const int jc = it / P, i = it - jc * P;
        const int jj = jc / nc, c = jc - jj * nc, j = j0 + jj;
        if (i >= a.rows[c] || j >= Q) continue;
        T2 v = A[(size_t)((jj * nsx) * nc + c) * ls + sk(i)];
        if (nsx == 2) v = cadd(v, cmulc(A[(size_t)((jj * nsx + 1) * nc + c) * ls + sk(i)], __ldg(&a.modP[i])));
        wr[((int64_t)c * Q + j) * P + i] = cscale(v, a.scale);
    }
}

// --------------------------------------------------------------------------------------------
// y-inverse: y_c(i, j) = sum_py demod_y^py IFFT_y(W[py][c][:, i]) for a tile of TI columns of one
// component, both y subbands at once (tile A[sk(j)][L] as in the y-forward), cropped.
template <typename T, bool POW2>
__global__ void __launch_bounds__(kMaxThreads, sizeof(T) == 8 ? 1 : 2) k_grid_y_inv(const GridArgs<T> a, typename Cx<T>::T2* __restrict__ y) {
    using T2 = typename Cx<T>::T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TI = a.ti, Q = a.Q, L = a.npy * TI;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* tws = A + (size_t)L * fft_span(a.planQ);
    const int c = blockIdx.y, rhs = blockIdx.z;
    const int rows = a.rows[c], cols = a.cols[c];
    const int i0 = blockIdx.x * TI;
    if (i0 >= rows || skipped(a, rhs)) return;
    stage_roots(tws, a.twQ, Q);
    const T2* wr = a.work + (int64_t)rhs * a.work_rhs;
    const int total = L * Q;
    for (int base = threadIdx.x; base < total; base += kBatch * blockDim.x) {
        T2 v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            const int l = it % L, j = it / L;
            const int pyi = l / TI, i = i0 + (l - pyi * TI);
            v[u] = (it < total && i < rows) ? wr[((int64_t)(pyi * a.ncomp + c) * Q + j) * a.P + i] : czero<T2>();
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const int it = base + u * blockDim.x;
            if (it >= total) break;
            const int l = it % L, j = it / L;
            A[(size_t)sk(j) * L + l] = v[u];
        }
    }
    __syncthreads();
    fft_inplace<true, POW2>(A, L, 1, L, a.planQ, tws);
    T2* yr = y + (int64_t)rhs * a.n + a.off[c];
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI, i = i0 + l;
        if (i >= rows || j >= cols) continue;
        const T2* row = A + (size_t)sk(j) * L + l;
        T2 v;
        if (a.npy == 2) v = cadd(row[0], cmulc(row[TI], __ldg(&a.modQ[j])));
        else v = a.py0 ? cmulc(row[0], __ldg(&a.modQ[j])) : row[0];
        const int64_t idx = i + (int64_t)j * rows;
        yr[idx] = a.accumulate ? cadd(yr[idx], v) : v;
    }
}

// --------------------------------------------------------------------------------------------
// Strip: y = sum_s demod^s IFFT( B_s FFT( x mod^s ) ) / L, the subbands as lines of one transform.
template <typename T, bool POW2>
__global__ void __launch_bounds__(kMaxThreads, sizeof(T) == 8 ? 1 : 2) k_strip(const GridArgs<T> a, const typename Cx<T>::T2* __restrict__ x,
                                                         typename Cx<T>::T2* __restrict__ y) {
    using T2 = typename Cx<T>::T2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = a.P, ls = a.ls, ns = a.nsx;
    const int count = (int)a.n;
    T2* A = reinterpret_cast<T2*>(smem_raw);
    T2* tws = A + (size_t)ns * ls;
    const int rhs = blockIdx.x;
    if (skipped(a, rhs)) return;
    stage_roots(tws, a.twP, L);
    const T2* xr = x + (int64_t)rhs * a.n;
    T2* yr = y + (int64_t)rhs * a.n;
    for (int i = threadIdx.x; i < L; i += blockDim.x) {
        const T2 v = i < count ? xr[i] : czero<T2>();
        A[sk(i)] = v;
        if (ns == 2) A[ls + sk(i)] = cmul(v, __ldg(&a.modP[i]));
    }
    __syncthreads();
    fft_inplace<false, POW2>(A, ns, ls, 1, a.planP, tws);
    for (int it = threadIdx.x; it < ns * L; it += blockDim.x) {
        const int s = it / L, i = it - s * L;
        A[s * ls + sk(i)] = cmul(A[s * ls + sk(i)], __ldg(&a.spec[(int64_t)s * L + i]));
    }
    __syncthreads();
    fft_inplace<true, POW2>(A, ns, ls, 1, a.planP, tws);
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        T2 v = A[sk(i)];
        if (ns == 2) v = cadd(v, cmulc(A[ls + sk(i)], __ldg(&a.modP[i])));
        yr[i] = cscale(v, a.scale);
    }
}

// --------------------------------------------------------------------------------------------
template <typename T, bool POW2> static int set_attrs_one() {
    RTM_CUDA(cudaFuncSetAttribute(k_grid_y_fwd<T, POW2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    RTM_CUDA(cudaFuncSetAttribute(k_grid_x_mix<T, POW2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    RTM_CUDA(cudaFuncSetAttribute(k_grid_y_inv<T, POW2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    RTM_CUDA(cudaFuncSetAttribute(k_strip<T, POW2>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    return RTM_OK;
}

template <typename T> static int set_smem_attrs() {
    static DeviceOnce once;
    return once([]() -> int {
        RTM_TRY((set_attrs_one<T, true>()));
        return set_attrs_one<T, false>();
    });
}

// Shared stride of the lines of a CTA that transforms `lines` lines of length n in place: room for
// the skewed positions sk(e), and a remainder modulo the elements of 128 bytes chosen so that the
// lines touched by one warp start on different banks.
static int line_stride(int n, int lines, size_t elem) {
    const int W = (int)(128 / elem);
    const int per = 32 / std::max(1, std::min(lines, 32));
    const int target = per % W;
    int ls = sk(n - 1) + 1;
    while (ls % W != target) ++ls;
    return ls;
}

size_t GridApplicator::work_bytes_per_rhs() const {
    if (mode == kStrip) return 0;
    const size_t elem = precision == RTM_FP64 ? sizeof(double2) : sizeof(float2);
    const int npy = lean ? 1 : nsy;
    return (size_t)npy * 2 * P * Q * elem;
}

// The launch arguments of a product (the transform grid's tables, the face grid, the spectra).
template <typename T> static GridArgs<T> product_args(const GridApplicator& g, SkipFlags skip) {
    using T2 = typename Cx<T>::T2;
    GridArgs<T> a{};
    a.skip = skip.ptr;
    a.skip_stride = skip.stride;
    a.P = g.P;
    a.Q = g.Q;
    a.nsx = g.nsx;
    a.nsy = g.nsy;
    for (int c = 0; c < 2; ++c) {
        a.rows[c] = g.rows[c];
        a.cols[c] = g.cols[c];
        a.off[c] = g.off[c];
    }
    a.n = g.n;
    a.ncomp = 2;
    a.planP = g.tP->plan;
    a.planQ = g.tQ->plan;
    if constexpr (sizeof(T) == 8) {
        a.twP = g.tP->tw64; a.twQ = g.tQ->tw64; a.modP = g.tP->mod64; a.modQ = g.tQ->mod64;
    } else {
        a.twP = g.tP->tw32; a.twQ = g.tQ->tw32; a.modP = g.tP->mod32; a.modQ = g.tQ->mod32;
    }
    a.spec = g.spec.as<T2>();
    a.mode = g.mode;
    a.ux0 = static_cast<const T2*>(g.ux[0]);
    a.ux1 = static_cast<const T2*>(g.ux[1]);
    a.vy0 = static_cast<const T2*>(g.vy[0]);
    a.vy1 = static_cast<const T2*>(g.vy[1]);
    a.inv_a2 = (T)(1.0 / (g.size_x * g.size_x));
    a.inv_b2 = (T)(1.0 / (g.size_y * g.size_y));
    a.inv_ab = (T)(1.0 / (g.size_x * g.size_y));
    return a;
}

template <typename T>
static int apply_t(const GridApplicator& g, const void* xv, void* yv, int nrhs, cudaStream_t s, SkipFlags skip,
                   void* work, int* fault) {
    using T2 = typename Cx<T>::T2;
    RTM_TRY(set_smem_attrs<T>());
    const T2* x = static_cast<const T2*>(xv);
    T2* y = static_cast<T2*>(yv);
    GridArgs<T> a = product_args<T>(g, skip);
    const size_t elem = sizeof(T2);
    if (g.mode == kStrip) {
        a.scale = (T)(1.0 / g.P);
        a.ls = line_stride(g.tP->plan.m, g.nsx, elem);
        const size_t smem = ((size_t)g.nsx * a.ls + g.P) * elem;
        const int thr = fft_threads(g.nsx, g.tP->plan);
        if (smem > (size_t)kSmemBudget || thr > kMaxThreads)
            return fail(RTM_ERR_UNSUPPORTED, "strip too long for this build");
        if (fft_pow2(g.tP->plan)) k_strip<T, true><<<nrhs, thr, smem, s>>>(a, x, y);
        else k_strip<T, false><<<nrhs, thr, smem, s>>>(a, x, y);
        count_launch();
        RTM_CUDA(cudaGetLastError());
        return RTM_OK;
    }
    a.scale = (T)(1.0 / ((double)g.P * g.Q));
    a.fault = fault;
    a.work = static_cast<T2*>(work);
    a.work_rhs = (int64_t)g.work_bytes_per_rhs() / (int64_t)elem;
    if (g.mode == kGen3 && g.nsx == 2 && g.nsy == 2 && !g.lean && fast_split_eligible(g.P, g.Q, sizeof(T) == 8)) {
        a.py0 = 0;
        a.npy = 2;
        a.accumulate = 0;
        return launch_fast_split<T>(a, nrhs, x, y, g.sched, s);
    }
    const int passes = g.lean ? g.nsy : 1;
    const int npy = g.lean ? 1 : g.nsy;
    // y passes: TI x columns per CTA (rows of 64 bytes) for every y subband at once; fewer columns
    // while the tile (plus the roots) would not fit or would need more than kMaxThreads threads.
    int ti = sizeof(T) == 8 ? 4 : 8;
    auto y_smem = [&](int t) { return ((size_t)npy * t * fft_span(g.tQ->plan) + g.Q) * elem; };
    while (ti > 1 && (y_smem(ti) > (size_t)kSmemBudget || fft_threads(npy * ti, g.tQ->plan) > kMaxThreads)) ti /= 2;
    const int thr_y = fft_threads(npy * ti, g.tQ->plan);
    // x-mix: CB y frequencies per CTA, every x subband and component at once (CB nsx 2 lines).
    auto x_smem = [&](int c) { return ((size_t)c * g.nsx * 2 * line_stride(g.tP->plan.m, c * g.nsx * 2, elem) + g.P) * elem; };
    int cb = 8;
    while (cb > 1 && (x_smem(cb) > (size_t)kSmemBudget || fft_threads(cb * g.nsx * 2, g.tP->plan) > kMaxThreads))
        cb /= 2;
    while (cb > 1 && (int64_t)((g.Q + cb - 1) / cb) * npy * nrhs < 148) cb /= 2;
    const int ls = line_stride(g.tP->plan.m, cb * g.nsx * 2, elem);
    const int thr_x = fft_threads(cb * g.nsx * 2, g.tP->plan);
    if (y_smem(ti) > (size_t)kSmemBudget || x_smem(cb) > (size_t)kSmemBudget || thr_y > kMaxThreads ||
        thr_x > kMaxThreads)
        return fail(RTM_ERR_UNSUPPORTED, "FFT grid too large for this build");
    a.ti = ti;
    a.cb = cb;
    a.ls = ls;
    const bool p2x = fft_pow2(g.tP->plan), p2y = fft_pow2(g.tQ->plan);
    const int rows_max = std::max(g.rows[0], g.rows[1]);
    const unsigned tiles = (unsigned)((rows_max + ti - 1) / ti);
    for (int pass = 0; pass < passes; ++pass) {
        a.py0 = g.lean ? pass : 0;
        a.npy = npy;
        a.accumulate = g.lean && pass > 0;
        const dim3 gy(tiles, 2, nrhs), gx((g.Q + cb - 1) / cb, npy, nrhs);
        if (p2y) k_grid_y_fwd<T, true><<<gy, thr_y, y_smem(ti), s>>>(a, x);
        else k_grid_y_fwd<T, false><<<gy, thr_y, y_smem(ti), s>>>(a, x);
        if (p2x) k_grid_x_mix<T, true><<<gx, thr_x, x_smem(cb), s>>>(a);
        else k_grid_x_mix<T, false><<<gx, thr_x, x_smem(cb), s>>>(a);
        if (p2y) k_grid_y_inv<T, true><<<gy, thr_y, y_smem(ti), s>>>(a, y);
        else k_grid_y_inv<T, false><<<gy, thr_y, y_smem(ti), s>>>(a, y);
        count_launch(3);
        RTM_CUDA(cudaGetLastError());
    }
    return RTM_OK;
}

int GridApplicator::reserve(int nrhs) {
    // kernel attributes and the fault word are set up here, outside of any stream capture
    RTM_TRY(precision == RTM_FP64 ? set_smem_attrs<double>() : set_smem_attrs<float>());
    RTM_TRY(device_fault_word(&fault));
    if (nrhs <= max_rhs && (mode == kStrip || work.bytes >= work_bytes_per_rhs() * (size_t)nrhs)) return RTM_OK;
    if (mode != kStrip) RTM_TRY(work.alloc(work_bytes_per_rhs() * (size_t)nrhs));
    max_rhs = std::max(max_rhs, nrhs);
    return RTM_OK;
}

bool batchable(const GridApplicator& g) {
    return g.mode == kGen3 && g.nsx == 2 && g.nsy == 2 && !g.lean &&
           fast_split_eligible(g.P, g.Q, g.precision == RTM_FP64);
}

template <typename T>
static int plate_descs_t(const std::vector<const GridApplicator*>& plates, DeviceBuffer& out, cudaStream_t s) {
    std::vector<PlateDesc<T>> d(plates.size());
    for (size_t k = 0; k < plates.size(); ++k) {
        const GridApplicator& g = *plates[k];
        for (int c = 0; c < 2; ++c) {
            d[k].rows[c] = g.rows[c];
            d[k].cols[c] = g.cols[c];
            d[k].off[c] = g.off[c];
        }
        d[k].spec = g.spec.as<typename Cx<T>::T2>();
        d[k].inv_a2 = (T)(1.0 / (g.size_x * g.size_x));
        d[k].inv_b2 = (T)(1.0 / (g.size_y * g.size_y));
        d[k].inv_ab = (T)(1.0 / (g.size_x * g.size_y));
    }
    RTM_TRY(out.alloc(sizeof(PlateDesc<T>) * d.size()));
    RTM_CUDA(cudaMemcpyAsync(out.ptr, d.data(), out.bytes, cudaMemcpyHostToDevice, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

int plate_descs(const std::vector<const GridApplicator*>& plates, DeviceBuffer& out, cudaStream_t s) {
    if (plates.empty()) return fail(RTM_ERR_ARG, "an empty plate batch");
    return plates[0]->precision == RTM_FP64 ? plate_descs_t<double>(plates, out, s)
                                            : plate_descs_t<float>(plates, out, s);
}

template <typename T>
static int apply_batch_t(const std::vector<const GridApplicator*>& plates, const void* descs, int64_t stride,
                         void* work, int* fault, const void* xv, void* yv, cudaStream_t s, SkipFlags skip) {
    const GridApplicator& g = *plates[0];
    RTM_TRY(set_smem_attrs<T>());
    GridArgs<T> a = product_args<T>(g, skip);
    a.plates = static_cast<const PlateDesc<T>*>(descs);
    a.n = stride;
    for (const GridApplicator* p : plates)  // the launch grids span the largest plate
        for (int c = 0; c < 2; ++c) {
            a.rows[c] = std::max(a.rows[c], p->rows[c]);
            a.cols[c] = std::max(a.cols[c], p->cols[c]);
        }
    a.scale = (T)(1.0 / ((double)g.P * g.Q));
    a.fault = fault;
    a.work = static_cast<typename Cx<T>::T2*>(work);
    a.work_rhs = (int64_t)g.work_bytes_per_rhs() / (int64_t)sizeof(typename Cx<T>::T2);
    a.py0 = 0;
    a.npy = 2;
    a.accumulate = 0;
    return launch_fast_split<T>(a, (int)plates.size(), xv, yv, g.sched, s);
}

int apply_plate_batch(const std::vector<const GridApplicator*>& plates, const void* descs, int64_t stride, void* work,
                      int* fault, const void* x, void* y, cudaStream_t s, SkipFlags skip) {
    return plates[0]->precision == RTM_FP64
               ? apply_batch_t<double>(plates, descs, stride, work, fault, x, y, s, skip)
               : apply_batch_t<float>(plates, descs, stride, work, fault, x, y, s, skip);
}

int GridApplicator::apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) {
    if (nrhs < 1 || nrhs > max_rhs) return fail(RTM_ERR_ARG, "more right-hand sides than the product reserved");
    if (!fault) RTM_TRY(device_fault_word(&fault));
    return precision == RTM_FP64 ? apply_t<double>(*this, x, y, nrhs, s, skip, work.ptr, fault)
                                 : apply_t<float>(*this, x, y, nrhs, s, skip, work.ptr, fault);
}

// ---------------------------------------------------------------------------------------------
// Fixed scratch: the working grid W in the library's fixed device array (fixed_scratch.cu) instead of
// the product's own buffer. Every call on a device shares the one array, so calls that may overlap in
// time (other streams, other host threads) race on it: the caller serialises them. Nothing in it has
// to start at zero: the y-forward pass writes every entry of W that the later passes read.
int fixed_scratch_address(void** out);

int apply_fixed_scratch(const GridApplicator& g, const void* x, void* y, int nrhs, cudaStream_t s) {
    if (nrhs < 1) return fail(RTM_ERR_ARG, "nrhs must be positive");
    const size_t need = g.work_bytes_per_rhs() * (size_t)nrhs;
    const size_t cap = fixed_scratch_bytes();
    if (need > cap)
        return fail(RTM_ERR_SIZE, "the working grid of " + std::to_string(nrhs) + " right-hand sides needs " +
                                      std::to_string(need) + " bytes, above the fixed scratch of " +
                                      std::to_string(cap) + " bytes");
    void* work = nullptr;
    if (g.mode != kStrip) RTM_TRY(fixed_scratch_address(&work));
    int* fault = nullptr;
    RTM_TRY(device_fault_word(&fault));
    return g.precision == RTM_FP64 ? apply_t<double>(g, x, y, nrhs, s, SkipFlags{}, work, fault)
                                   : apply_t<float>(g, x, y, nrhs, s, SkipFlags{}, work, fault);
}

// ============================================================================================
// Spectra builders: 2-D DFTs (P x Q) of generated inputs, in FP64.
enum SourceKind { kSrcEmbed = 0, kSrcCirculant = 1, kSrcTwoSided = 2, kSrcPart = 3 };
enum Window { kWinStrang = 0, kWinTChan = 1, kWinRChan = 2, kWinHuckle = 3 };
constexpr int kMaxItems = 12;

struct GenItem {
    const double2* g;  // generator, column-major rows x cols (two-sided sources: (2P - 1) x (2Q - 1))
    int rows, cols;
    int px, py;        // subband parities; part (m, n) of kSrcPart
    double2* dst;      // P x Q output (column-major, x fastest)
};

struct GenArgs {
    int P, Q;
    int kind;
    int Lx, Ly;        // mirror periods of the embedding
    int nsx, nsy;      // folded copies (2 for split directions)
    double scale;
    int window, bw_x, bw_y;
    int realify;
    int ti;
    FftPlan planP, planQ;
    const double2* twP;
    const double2* twQ;
    const double2* modP;
    const double2* modQ;
    int nitems;
    GenItem items[kMaxItems];
};

__device__ __forceinline__ int mirror_index(int i, int rows, int L) {
    if (i < rows) return i;
    const int m = L - i;
    return (m >= 0 && m < rows) ? m : -1;
}

__device__ __forceinline__ double window_weight(int w, int o, int n, int bw) {
    const int ao = o < 0 ? -o : o;
    switch (w) {
        case kWinStrang: return (2 * ao < n) ? 1.0 : (2 * ao == n ? 0.5 : 0.0);
        case kWinTChan: return (double)(n - ao) / (double)n;
        case kWinRChan: return 1.0;
        default: return fmax(0.0, 1.0 - (double)ao / (double)bw);
    }
}

__device__ double2 gen_value(const GenArgs& a, const GenItem& it, int i, int j) {
    double re = 0, im = 0;
    if (a.kind == kSrcEmbed) {
        for (int ca = 0; ca < a.nsx; ++ca) {
            const int mx = mirror_index(i + ca * a.P, it.rows, a.Lx);
            if (mx < 0) continue;
            const double sa = (it.px && ca) ? -1.0 : 1.0;
            for (int cb = 0; cb < a.nsy; ++cb) {
                const int my = mirror_index(j + cb * a.Q, it.cols, a.Ly);
                if (my < 0) continue;
                const double sb = (it.py && cb) ? -1.0 : 1.0;
                const double2 g = it.g[mx + (int64_t)my * it.rows];
                re += sa * sb * g.x;
                im += sa * sb * g.y;
            }
        }
        double2 v = make_double2(re * a.scale, im * a.scale);
        if (it.px) v = cmul(v, a.modP[i]);
        if (it.py) v = cmul(v, a.modQ[j]);
        return v;
    }
    if (a.kind == kSrcTwoSided || a.kind == kSrcPart) {
        // A two-sided source, offsets -(P-1)..P-1 by -(Q-1)..Q-1. kSrcTwoSided: the windowed fold onto the
        // face grid (foldGenerator.m:47-60). kSrcPart: part (m, n) of generatePartSpectra.m:15-49, the
        // halved sum (m = 0) or difference (m = 1) of the offsets i and i - P, likewise along y, times
        // exp(i pi i / P) for m = 1 and exp(i pi j / Q) for n = 1.
        const bool part = a.kind == kSrcPart;
        for (int ca = 0; ca < 2; ++ca) {
            if (ca == 1 && i == 0) continue;
            const int ox = ca ? i - a.P : i;
            const double wa = part ? ((it.px && ca) ? -0.5 : 0.5) : window_weight(a.window, ox, a.P, a.bw_x);
            for (int cb = 0; cb < 2; ++cb) {
                if (cb == 1 && j == 0) continue;
                const int oy = cb ? j - a.Q : j;
                const double wb = part ? ((it.py && cb) ? -0.5 : 0.5) : window_weight(a.window, oy, a.Q, a.bw_y);
                const double2 g = it.g[(ox + a.P - 1) + (int64_t)(oy + a.Q - 1) * it.rows];
                re += wa * wb * g.x;
                im += wa * wb * g.y;
            }
        }
        double2 v = make_double2(re, im);
        if (part && it.px) v = cmulc(v, a.modP[i]);
        if (part && it.py) v = cmulc(v, a.modQ[j]);
        return v;
    }
    // Circulant fold of the even generator onto the face grid (foldGenerator.m:38-45).
    for (int ca = 0; ca < 2; ++ca) {
        if (ca == 1 && i == 0) continue;
        const int mx = ca ? a.P - i : i;
        if (mx >= it.rows) continue;
        const double wa = window_weight(a.window, ca ? i - a.P : i, a.P, a.bw_x);
        for (int cb = 0; cb < 2; ++cb) {
            if (cb == 1 && j == 0) continue;
            const int my = cb ? a.Q - j : j;
            if (my >= it.cols) continue;
            const double wb = window_weight(a.window, cb ? j - a.Q : j, a.Q, a.bw_y);
            const double2 g = it.g[mx + (int64_t)my * it.rows];
            re += wa * wb * g.x;
            im += wa * wb * g.y;
        }
    }
    return make_double2(re, im);
}

__global__ void __launch_bounds__(kMaxThreads, 1) k_gen_y(const GenArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TI = a.ti, Q = a.Q;
    double2* A = reinterpret_cast<double2*>(smem_raw);
    const GenItem& item = a.items[blockIdx.y];
    const int i0 = blockIdx.x * TI;
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI, i = i0 + l;
        A[sk(j) * TI + l] = (i < a.P) ? gen_value(a, item, i, j) : make_double2(0, 0);
    }
    __syncthreads();
    fft_inplace<false, false>(A, TI, 1, TI, a.planQ, a.twQ);
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI, i = i0 + l;
        if (i < a.P) item.dst[(int64_t)j * a.P + i] = A[sk(j) * TI + l];
    }
}

__global__ void __launch_bounds__(kMaxThreads, 1) k_gen_x(const GenArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int P = a.P;
    double2* A = reinterpret_cast<double2*>(smem_raw);
    const GenItem& item = a.items[blockIdx.y];
    const int j = blockIdx.x;
    double2* col = item.dst + (int64_t)j * P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) A[sk(i)] = col[i];
    __syncthreads();
    fft_inplace<false, false>(A, 1, P, 1, a.planP, a.twP);
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        double2 v = A[sk(i)];
        if (a.realify) v.y = 0.0;
        col[i] = v;
    }
}

static int run_gen(GenArgs& a, cudaStream_t s) {
    static DeviceOnce once;
    RTM_TRY(once([]() -> int {
        RTM_CUDA(cudaFuncSetAttribute(k_gen_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        RTM_CUDA(cudaFuncSetAttribute(k_gen_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        return RTM_OK;
    }));
    if (a.nitems == 0) return RTM_OK;
    a.ti = 4;
    while (a.ti > 1 && ((size_t)a.ti * fft_span(a.planQ) * sizeof(double2) > (size_t)kSmemBudget ||
                        fft_threads(a.ti, a.planQ) > kMaxThreads))
        a.ti /= 2;
    const int thr_y = fft_threads(a.ti, a.planQ), thr_x = fft_threads(1, a.planP);
    const size_t smem_y = (size_t)a.ti * fft_span(a.planQ) * sizeof(double2);
    const size_t smem_x = (size_t)fft_span(a.planP) * sizeof(double2);
    if (smem_y > (size_t)kSmemBudget || smem_x > (size_t)kSmemBudget || thr_y > kMaxThreads || thr_x > kMaxThreads)
        return fail(RTM_ERR_UNSUPPORTED, "spectra grid too large for this build");
    dim3 gy((a.P + a.ti - 1) / a.ti, a.nitems);
    k_gen_y<<<gy, thr_y, smem_y, s>>>(a);
    dim3 gx(a.Q, a.nitems);
    k_gen_x<<<gx, thr_x, smem_x, s>>>(a);
    count_launch(2);
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

// Explicit strip blocks B_s = M_s - |u_s|^2 / h^2 E_s on a line of length L (generateBlockSpectra.m:36-42).
__global__ void k_strip_blocks(int L, int nsub, const double2* __restrict__ raw, const double2* __restrict__ u0,
                               const double2* __restrict__ u1, double inv_h2, double2* __restrict__ out) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= L * nsub) return;
    const int s = idx / L, i = idx - s * L;
    const double2 E = raw[(int64_t)(s * 2 + 0) * L + i];
    const double2 M = raw[(int64_t)(s * 2 + 1) * L + i];
    const double2 u = (s ? u1 : u0)[i];
    const double c = (u.x * u.x + u.y * u.y) * inv_h2;
    out[idx] = make_double2(M.x - c * E.x, M.y - c * E.y);
}

// Circulant blocks and their 2x2 inverse (generateBlockSpectra.m + Spectra.invert), flags any
// non-finite value. raw: [E, MXX, MYY] on the face grid; out: [XX, XY, YX, YY].
__global__ void k_circulant_invert(int P, int Q, int content, const double2* __restrict__ raw,
                                   const double2* __restrict__ u, const double2* __restrict__ v, double inv_a2,
                                   double inv_b2, double inv_ab, double2* __restrict__ out, int* __restrict__ bad) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t G = (int64_t)P * Q;
    if (idx >= G) return;
    const int i = (int)(idx % P), j = (int)(idx / P);
    const double2 E = raw[idx], Mx = raw[G + idx], My = raw[2 * G + idx];
    const double2 uu = u[i], vv = v[j];
    const double cu = (uu.x * uu.x + uu.y * uu.y) * inv_a2;
    const double cv = (vv.x * vv.x + vv.y * vv.y) * inv_b2;
    double2 XX = make_double2(Mx.x - cu * E.x, Mx.y - cu * E.y);
    double2 YY = make_double2(My.x - cv * E.x, My.y - cv * E.y);
    double2 qc = cmulc(uu, vv);
    qc.x = -qc.x * inv_ab;
    qc.y = -qc.y * inv_ab;
    double2 XY = cmul(qc, E), YX = cmul(cconj(qc), E);
    double2 r[4];
    if (content == RTM_XONLY) {
        const double d = XX.x * XX.x + XX.y * XX.y;
        r[0] = make_double2(XX.x / d, -XX.y / d);
        r[1] = r[2] = r[3] = make_double2(0, 0);
    } else if (content == RTM_YONLY) {
        const double d = YY.x * YY.x + YY.y * YY.y;
        r[3] = make_double2(YY.x / d, -YY.y / d);
        r[0] = r[1] = r[2] = make_double2(0, 0);
    } else {
        const double2 det = csub(cmul(XX, YY), cmul(XY, YX));
        const double dd = det.x * det.x + det.y * det.y;
        const double2 inv = make_double2(det.x / dd, -det.y / dd);
        r[0] = cmul(YY, inv);
        r[1] = cmul(make_double2(-XY.x, -XY.y), inv);
        r[2] = cmul(make_double2(-YX.x, -YX.y), inv);
        r[3] = cmul(XX, inv);
    }
    for (int b = 0; b < 4; ++b) {
        if (!isfinite(r[b].x) || !isfinite(r[b].y)) atomicExch(bad, 1);
        out[b * G + idx] = r[b];
    }
}

__global__ void k_to_fp32(int64_t n, const double2* __restrict__ in, float2* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

static int convert_spectra(const DeviceBuffer& src64, int precision, DeviceBuffer& dst, cudaStream_t s) {
    const int64_t n = (int64_t)(src64.bytes / sizeof(double2));
    if (precision == RTM_FP64) {
        RTM_TRY(dst.alloc(src64.bytes));
        RTM_CUDA(cudaMemcpyAsync(dst.ptr, src64.ptr, src64.bytes, cudaMemcpyDeviceToDevice, s));
        return RTM_OK;
    }
    RTM_TRY(dst.alloc((size_t)n * sizeof(float2)));
    k_to_fp32<<<592, 256, 0, s>>>(n, src64.as<double2>(), dst.as<float2>());
    count_launch();
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

static void fill_shift(GridApplicator& out, int n, int parity, bool x_dir, int slot) {
    const double2* s64 = nullptr;
    const float2* s32 = nullptr;
    shift_factors(n, parity, &s64, &s32);
    const void* p = out.precision == RTM_FP64 ? (const void*)s64 : (const void*)s32;
    if (x_dir) out.ux[slot] = p; else out.vy[slot] = p;
}

static void layout(GridApplicator& o, int cx, int cy) {
    o.count_x = cx;
    o.count_y = cy;
    o.rows[0] = cx - 1; o.cols[0] = cy;
    o.rows[1] = cx;     o.cols[1] = cy - 1;
    const int64_t nx = (int64_t)(cx - 1) * cy, ny = (int64_t)cx * (cy - 1);
    o.off[0] = 0;
    o.off[1] = nx;
    o.n = nx + ny;
    o.content = (nx > 0 && ny > 0) ? RTM_BOTH : nx > 0 ? RTM_XONLY : ny > 0 ? RTM_YONLY : RTM_NONE;
}

int build_product(const DeviceGenerators& g, double size_x, double size_y, int product, int precision, int max_rhs,
                  GridApplicator& out, cudaStream_t s, int force_P, int force_Q, const FastSchedule* force_sched) {
    const int cx = g.count_x, cy = g.count_y;
    layout(out, cx, cy);
    out.precision = precision;
    out.size_x = size_x;
    out.size_y = size_y;
    out.max_rhs = std::max(1, max_rhs);
    out.lean = product == RTM_PRODUCT_LEAN;
    if (out.content == RTM_NONE) return fail(RTM_ERR_ARG, "a single face carries no rooftop");
    GenArgs a{};
    a.kind = kSrcEmbed;
    if (product == RTM_PRODUCT_FFT) {
        // generateEmbeddingSpectra.m: period 2n - 2 along every direction with more than one face.
        out.P = cx > 1 ? 2 * cx - 2 : 1;
        out.Q = cy > 1 ? 2 * cy - 2 : 1;
        out.nsx = out.nsy = 1;
        a.Lx = out.P;
        a.Ly = out.Q;
        a.nsx = a.nsy = 1;
        a.scale = 1.0;
    } else {
        // generateSubbandSpectra.m: fast FFT size and 2 subbands along every direction with more than one face.
        // Any P >= countX gives the same product (the period 2P holds the whole two-sided generator), so the
        // autotuner may pick another size for speed; the result differs by rounding only.
        out.P = cx > 1 ? fast_fft_size(cx) : 1;
        out.Q = cy > 1 ? fast_fft_size(cy) : 1;
        out.sched = default_fast_schedule(out.P, out.Q, precision == RTM_FP64);
        int tp = 0, tq = 0;
        FastSchedule ts;
        if (force_P > 0 || force_Q > 0) {
            if (force_P > 0 && cx > 1) out.P = force_P;
            if (force_Q > 0 && cy > 1) out.Q = force_Q;
            out.sched = default_fast_schedule(out.P, out.Q, precision == RTM_FP64);
        } else if (product == RTM_PRODUCT_SPLIT && tuned_choice(cx, cy, precision, &tp, &tq, &ts)) {
            out.P = tp;
            out.Q = tq;
            out.sched = ts;
        }
        if (force_sched) out.sched = *force_sched;
        if (out.P < cx || out.Q < cy) return fail(RTM_ERR_ARG, "a transform grid smaller than the face grid");
        out.nsx = cx > 1 ? 2 : 1;
        out.nsy = cy > 1 ? 2 : 1;
        a.Lx = out.nsx * out.P;
        a.Ly = out.nsy * out.Q;
        a.nsx = out.nsx;
        a.nsy = out.nsy;
        a.scale = 1.0 / (out.nsx * out.nsy);
    }
    const FftTables* tP = nullptr;
    const FftTables* tQ = nullptr;
    RTM_TRY(fft_tables(out.P, &tP));
    RTM_TRY(fft_tables(out.Q, &tQ));
    out.tP = tP;
    out.tQ = tQ;
    a.P = out.P;
    a.Q = out.Q;
    a.planP = tP->plan;
    a.planQ = tQ->plan;
    a.twP = tP->tw64;
    a.twQ = tQ->tw64;
    a.modP = tP->mod64;
    a.modQ = tQ->mod64;
    a.realify = g.is_real ? 1 : 0;
    const int nsub = out.nsx * out.nsy;
    const int64_t G = (int64_t)out.P * out.Q;
    const double2* gens[3] = {g.e.as<double2>(), g.xx.as<double2>(), g.yy.as<double2>()};
    const int grows[3] = {cx, cx - 1, cx};
    const int gcols[3] = {cy, cy, cy - 1};

    if (out.content == RTM_BOTH) {
        out.mode = kGen3;
        DeviceBuffer raw;
        StreamSyncGuard guard(s);
        RTM_TRY(raw.alloc((size_t)nsub * 3 * G * sizeof(double2)));
        RTM_CUDA(cudaMemsetAsync(raw.ptr, 0, raw.bytes, s));
        for (int sub = 0; sub < nsub; ++sub) {
            for (int k = 0; k < 3; ++k) {
                GenItem& it = a.items[a.nitems++];
                it.g = gens[k];
                it.rows = grows[k];
                it.cols = gcols[k];
                it.px = sub % out.nsx;
                it.py = sub / out.nsx;
                it.dst = raw.as<double2>() + (int64_t)(sub * 3 + k) * G;
            }
        }
        RTM_TRY(run_gen(a, s));
        RTM_TRY(convert_spectra(raw, precision, out.spec, s));
        out.spec_blocks = nsub * 3;
        for (int p = 0; p < out.nsx; ++p) fill_shift(out, out.P, p, true, p);
        for (int p = 0; p < out.nsy; ++p) fill_shift(out, out.Q, p, false, p);
        if (out.nsx == 1) fill_shift(out, out.P, 0, true, 1);
        if (out.nsy == 1) fill_shift(out, out.Q, 0, false, 1);
        RTM_TRY(out.work.alloc(out.work_bytes_per_rhs() * out.max_rhs));
        RTM_CUDA(cudaStreamSynchronize(s));
        return RTM_OK;
    }
    // Strips: a line along the direction with rooftops; subbands along it (x strip: Q = 1).
    out.mode = kStrip;
    const bool xs = out.content == RTM_XONLY;
    const int L = xs ? out.P : out.Q;
    const int ns = xs ? out.nsx : out.nsy;
    DeviceBuffer raw, blocks64;
    StreamSyncGuard guard(s);
    RTM_TRY(raw.alloc((size_t)ns * 2 * G * sizeof(double2)));
    RTM_CUDA(cudaMemsetAsync(raw.ptr, 0, raw.bytes, s));
    for (int sub = 0; sub < ns; ++sub) {
        for (int k = 0; k < 2; ++k) {
            GenItem& it = a.items[a.nitems++];
            const int gi = k == 0 ? 0 : (xs ? 1 : 2);
            it.g = gens[gi];
            it.rows = grows[gi];
            it.cols = gcols[gi];
            it.px = xs ? sub : 0;
            it.py = xs ? 0 : sub;
            it.dst = raw.as<double2>() + (int64_t)(sub * 2 + k) * G;
        }
    }
    RTM_TRY(run_gen(a, s));
    RTM_TRY(blocks64.alloc((size_t)ns * L * sizeof(double2)));
    const double2* u0 = nullptr;
    const double2* u1 = nullptr;
    const float2* f = nullptr;
    RTM_TRY(shift_factors(L, 0, &u0, &f));
    if (ns > 1) RTM_TRY(shift_factors(L, 1, &u1, &f));
    const double h = xs ? size_x : size_y;
    k_strip_blocks<<<(ns * L + 255) / 256, 256, 0, s>>>(L, ns, raw.as<double2>(), u0, u1 ? u1 : u0, 1.0 / (h * h),
                                                         blocks64.as<double2>());
    count_launch();
    RTM_CUDA(cudaGetLastError());
    RTM_TRY(convert_spectra(blocks64, precision, out.spec, s));
    out.spec_blocks = ns;
    // The strip kernel runs on P (line length) with nsx subbands.
    out.P = L;
    out.Q = 1;
    out.nsx = ns;
    out.nsy = 1;
    RTM_TRY(fft_tables(L, &out.tP));
    RTM_TRY(fft_tables(1, &out.tQ));
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

// --------------------------------------------------------------------------------------------
// Superoptimal kernel and the blockwise / hybrid builders (generateSuperoptimal.m:14-25,
// generateOptimalOfProduct.m:18-62, generateSpatialBlocks.m:19-61, generateBlockwiseSpectra.m:17-33,
// generateHybridSpectra.m:16-26). Sources are two-sided arrays of (2P - 1) x (2Q - 1) offsets on the
// P x Q face grid; everything runs in FP64 at set-up.

// Two-sided even extension of a generator padded to P x Q (extendEvenly.m:12-13 of the padded array).
__global__ void k_two_sided_even(int P, int Q, const double2* __restrict__ g, int rows, int cols,
                                 double2* __restrict__ out) {
    const int64_t W = 2 * P - 1, n = W * (2 * Q - 1);
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int ox = abs((int)(t % W) - (P - 1)), oy = abs((int)(t / W) - (Q - 1));
        out[t] = (ox < rows && oy < cols) ? g[ox + (int64_t)oy * rows] : make_double2(0, 0);
    }
}

// Spatial blocks of the Green's matrix by offset between first faces (generateSpatialBlocks.m:19-61):
// XX = MXX - (2E - E(-1,0) - E(1,0)) / a^2, YY likewise along y, XY = -(E - E(0,-1) - E(1,0) + E(1,-1)) / ab,
// with E evenly extended and zero outside the offsets, and the offsets no rooftop pair has set to zero.
__global__ void k_spatial_blocks(int P, int Q, const double2* __restrict__ E, const double2* __restrict__ mxx,
                                 const double2* __restrict__ myy, double inv_a2, double inv_b2, double inv_ab,
                                 double2* __restrict__ bxx, double2* __restrict__ bxy, double2* __restrict__ byy) {
    const int64_t W = 2 * P - 1, n = W * (2 * Q - 1);
    auto e2 = [&](int ox, int oy) -> double2 {
        if (ox < -(P - 1) || ox > P - 1 || oy < -(Q - 1) || oy > Q - 1) return make_double2(0, 0);
        return E[abs(ox) + (int64_t)abs(oy) * P];
    };
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int ox = (int)(t % W) - (P - 1), oy = (int)(t / W) - (Q - 1);
        const double2 c = e2(ox, oy);
        if (bxx) {
            double2 v = make_double2(0, 0);
            if (abs(ox) <= P - 2) {
                const double2 l = e2(ox - 1, oy), r = e2(ox + 1, oy);
                const double2 m = abs(ox) < P - 1 ? mxx[abs(ox) + (int64_t)abs(oy) * (P - 1)] : make_double2(0, 0);
                v = make_double2(m.x - (2 * c.x - l.x - r.x) * inv_a2, m.y - (2 * c.y - l.y - r.y) * inv_a2);
            }
            bxx[t] = v;
        }
        if (byy) {
            double2 v = make_double2(0, 0);
            if (abs(oy) <= Q - 2) {
                const double2 d = e2(ox, oy - 1), u = e2(ox, oy + 1);
                const double2 m = abs(oy) < Q - 1 ? myy[abs(ox) + (int64_t)abs(oy) * P] : make_double2(0, 0);
                v = make_double2(m.x - (2 * c.x - d.x - u.x) * inv_b2, m.y - (2 * c.y - d.y - u.y) * inv_b2);
            }
            byy[t] = v;
        }
        if (bxy) {
            double2 v = make_double2(0, 0);
            if (ox <= P - 2 && oy >= -(Q - 2)) {
                const double2 a1 = e2(ox, oy - 1), a2 = e2(ox + 1, oy), a3 = e2(ox + 1, oy - 1);
                v = make_double2(-(c.x - a1.x - a2.x + a3.x) * inv_ab, -(c.y - a1.y - a2.y + a3.y) * inv_ab);
            }
            bxy[t] = v;
        }
    }
}

// Circular convolution along x (dim 0) or y (dim 1) of a P x Q array in place:
// ifft(K fft(values)) with K the kernel's spectrum (generateOptimalOfProduct.m:52-62). One CTA per line
// along x; TI lines per CTA along y.
__global__ void __launch_bounds__(kMaxThreads, 1) k_line_conv_x(int P, int Q, FftPlan plan, const double2* tw,
                                                                const double2* __restrict__ K, double2* v) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* A = reinterpret_cast<double2*>(smem_raw);
    double2* line = v + (int64_t)blockIdx.x * P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) A[sk(i)] = line[i];
    __syncthreads();
    fft_inplace<false, false>(A, 1, P, 1, plan, tw);
    for (int i = threadIdx.x; i < P; i += blockDim.x) A[sk(i)] = cmul(A[sk(i)], K[i]);
    __syncthreads();
    fft_inplace<true, false>(A, 1, P, 1, plan, tw);
    const double sc = 1.0 / P;
    for (int i = threadIdx.x; i < P; i += blockDim.x) line[i] = cscale(A[sk(i)], sc);
}

__global__ void __launch_bounds__(kMaxThreads, 1) k_line_conv_y(int P, int Q, int TI, FftPlan plan, const double2* tw,
                                                                const double2* __restrict__ K, double2* v) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* A = reinterpret_cast<double2*>(smem_raw);
    const int i0 = blockIdx.x * TI;
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI, i = i0 + l;
        A[sk(j) * TI + l] = i < P ? v[(int64_t)j * P + i] : make_double2(0, 0);
    }
    __syncthreads();
    fft_inplace<false, false>(A, TI, 1, TI, plan, tw);
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI;
        A[sk(j) * TI + l] = cmul(A[sk(j) * TI + l], K[j]);
    }
    __syncthreads();
    fft_inplace<true, false>(A, TI, 1, TI, plan, tw);
    const double sc = 1.0 / Q;
    for (int it = threadIdx.x; it < TI * Q; it += blockDim.x) {
        const int l = it % TI, j = it / TI, i = i0 + l;
        if (i < P) v[(int64_t)j * P + i] = cscale(A[sk(j) * TI + l], sc);
    }
}

// op 0: out = a conj(b); op 1: out += a; op 2: out = a / conj(b).
__global__ void k_spectra_arith(int op, int64_t n, const double2* __restrict__ a, const double2* __restrict__ b,
                                double2* __restrict__ out) {
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        if (op == 0) {
            out[t] = cmulc(a[t], b[t]);
        } else if (op == 1) {
            out[t] = cadd(out[t], a[t]);
        } else {
            const double2 d = cconj(b[t]);
            const double m = d.x * d.x + d.y * d.y;
            const double2 q = cmulc(a[t], d);
            out[t] = make_double2(q.x / m, q.y / m);
        }
    }
}

// Explicit 2x2 blocks and their inverse per frequency (Spectra.invert, invert.m:12-20). XX, YY given;
// mode 0 (blockwise): XY given, YX(i, j) = XY(-i, -j); mode 1 (hybrid): XY = qc E, YX = conj(qc) E with
// qc = -(1 - s_x) conj(1 - s_y) / ab (generateBlockSpectra.m:43-47). Flags any non-finite value.
__global__ void k_blocks_invert(int P, int Q, int content, int mode, const double2* __restrict__ xx,
                                const double2* __restrict__ xy, const double2* __restrict__ yy,
                                const double2* __restrict__ u, const double2* __restrict__ v, double inv_ab,
                                double2* __restrict__ out, int* __restrict__ bad) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t G = (int64_t)P * Q;
    if (idx >= G) return;
    const int i = (int)(idx % P), j = (int)(idx / P);
    double2 r[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    if (content == RTM_XONLY) {
        const double2 XX = xx[idx];
        const double d = XX.x * XX.x + XX.y * XX.y;
        r[0] = make_double2(XX.x / d, -XX.y / d);
    } else if (content == RTM_YONLY) {
        const double2 YY = yy[idx];
        const double d = YY.x * YY.x + YY.y * YY.y;
        r[3] = make_double2(YY.x / d, -YY.y / d);
    } else {
        const double2 XX = xx[idx], YY = yy[idx];
        double2 XY, YX;
        if (mode == 0) {
            XY = xy[idx];
            YX = xy[(i ? P - i : 0) + (int64_t)(j ? Q - j : 0) * P];
        } else {
            const double2 E = xy[idx];
            double2 qc = cmulc(u[i], v[j]);
            qc.x = -qc.x * inv_ab;
            qc.y = -qc.y * inv_ab;
            XY = cmul(qc, E);
            YX = cmul(cconj(qc), E);
        }
        const double2 det = csub(cmul(XX, YY), cmul(XY, YX));
        const double dd = det.x * det.x + det.y * det.y;
        const double2 inv = make_double2(det.x / dd, -det.y / dd);
        r[0] = cmul(YY, inv);
        r[1] = cmul(make_double2(-XY.x, -XY.y), inv);
        r[2] = cmul(make_double2(-YX.x, -YX.y), inv);
        r[3] = cmul(XX, inv);
    }
    for (int b = 0; b < 4; ++b) {
        if (!isfinite(r[b].x) || !isfinite(r[b].y)) atomicExch(bad, 1);
        out[b * G + idx] = r[b];
    }
}

// Spectrum of 1 / (n^2 sin^2(pi (2d + 1) / (2n))), d < n (generateOptimalOfProduct.m:52-55), by a direct
// DFT in long double on the host.
static std::vector<double2> convolution_kernel(int n) {
    const long double pi = 3.141592653589793238462643383279502884L;
    std::vector<long double> k(n);
    for (int d = 0; d < n; ++d) {
        const long double sn = sinl(pi * (2 * d + 1) / (2.0L * n));
        k[d] = 1.0L / ((long double)n * n * sn * sn);
    }
    std::vector<double2> out(n);
    for (int f = 0; f < n; ++f) {
        long double re = 0, im = 0;
        for (int d = 0; d < n; ++d) {
            const long double ang = -2 * pi * (long double)(((int64_t)f * d) % n) / n;
            re += k[d] * cosl(ang);
            im += k[d] * sinl(ang);
        }
        out[f] = make_double2((double)re, (double)im);
    }
    return out;
}

struct TwoSidedSpectra {
    int P, Q;
    int window;
    int bw_x, bw_y;
    const FftTables* tP;
    const FftTables* tQ;
};

static int line_conv(const TwoSidedSpectra& t, int dim, const double2* K, double2* v, cudaStream_t s) {
    static DeviceOnce once;
    RTM_TRY(once([]() -> int {
        RTM_CUDA(cudaFuncSetAttribute(k_line_conv_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        RTM_CUDA(cudaFuncSetAttribute(k_line_conv_y, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        return RTM_OK;
    }));
    if (dim == 0) {
        const size_t smem = (size_t)fft_span(t.tP->plan) * sizeof(double2);
        const int thr = fft_threads(1, t.tP->plan);
        if (smem > (size_t)kSmemBudget || thr > kMaxThreads) return fail(RTM_ERR_UNSUPPORTED, "grid too large");
        k_line_conv_x<<<t.Q, thr, smem, s>>>(t.P, t.Q, t.tP->plan, t.tP->tw64, K, v);
    } else {
        int ti = 4;
        while (ti > 1 && ((size_t)ti * fft_span(t.tQ->plan) * sizeof(double2) > (size_t)kSmemBudget ||
                          fft_threads(ti, t.tQ->plan) > kMaxThreads))
            ti /= 2;
        const size_t smem = (size_t)ti * fft_span(t.tQ->plan) * sizeof(double2);
        const int thr = fft_threads(ti, t.tQ->plan);
        if (smem > (size_t)kSmemBudget || thr > kMaxThreads) return fail(RTM_ERR_UNSUPPORTED, "grid too large");
        k_line_conv_y<<<(t.P + ti - 1) / ti, thr, smem, s>>>(t.P, t.Q, ti, t.tQ->plan, t.tQ->tw64, K, v);
    }
    count_launch();
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

static int run_two_sided(const TwoSidedSpectra& t, int kind, int window, const double2* src, int px, int py,
                         double2* dst, cudaStream_t s) {
    GenArgs a{};
    a.kind = kind;
    a.P = t.P;
    a.Q = t.Q;
    a.window = window;
    a.bw_x = t.bw_x;
    a.bw_y = t.bw_y;
    a.planP = t.tP->plan;
    a.planQ = t.tQ->plan;
    a.twP = t.tP->tw64;
    a.twQ = t.tQ->tw64;
    a.modP = t.tP->mod64;
    a.modQ = t.tQ->mod64;
    GenItem& it = a.items[a.nitems++];
    it.g = src;
    it.rows = 2 * t.P - 1;
    it.cols = 2 * t.Q - 1;
    it.px = px;
    it.py = py;
    it.dst = dst;
    return run_gen(a, s);
}

// Spectrum (P x Q) of the kernel applied to a two-sided source: the windowed fold for strang, tChan,
// rChan and huckle; for superoptimal c(T T^H) / conj(c(T)) with c the T. Chan approximation.
static int two_sided_spectrum(const TwoSidedSpectra& t, int kernel, const double2* src, double2* dst, cudaStream_t s) {
    if (kernel != RTM_KERNEL_SUPEROPTIMAL) return run_two_sided(t, kSrcTwoSided, t.window, src, 0, 0, dst, s);
    const int64_t G = (int64_t)t.P * t.Q;
    DeviceBuffer parts, tmp, kx, ky;
    StreamSyncGuard guard(s);
    RTM_TRY(parts.alloc(4 * (size_t)G * sizeof(double2)));  // part (m, n) at m + 2 n
    RTM_TRY(tmp.alloc(4 * (size_t)G * sizeof(double2)));    // va, vb, product, T. Chan spectrum
    double2* P4 = parts.as<double2>();
    double2* va = tmp.as<double2>();
    double2* vb = va + G;
    double2* pr = vb + G;
    double2* opt = pr + G;
    for (int q = 0; q < 4; ++q) RTM_TRY(run_two_sided(t, kSrcPart, 0, src, q & 1, q >> 1, P4 + q * G, s));
    RTM_TRY(run_two_sided(t, kSrcTwoSided, kWinTChan, src, 0, 0, opt, s));
    const std::vector<double2> hx = convolution_kernel(t.P), hy = convolution_kernel(t.Q);
    RTM_TRY(kx.alloc(hx.size() * sizeof(double2)));
    RTM_TRY(ky.alloc(hy.size() * sizeof(double2)));
    RTM_CUDA(cudaMemcpyAsync(kx.ptr, hx.data(), kx.bytes, cudaMemcpyHostToDevice, s));
    RTM_CUDA(cudaMemcpyAsync(ky.ptr, hy.data(), ky.bytes, cudaMemcpyHostToDevice, s));
    const double2* K[2] = {kx.as<double2>(), ky.as<double2>()};
    RTM_CUDA(cudaMemsetAsync(dst, 0, (size_t)G * sizeof(double2), s));
    const unsigned blocks = (unsigned)std::min<int64_t>((G + 255) / 256, 1184);
    // generateOptimalOfProduct.m:34-49: sum over the part types of a and b
    for (int ta = 0; ta < 4; ++ta)
        for (int tb = 0; tb < 4; ++tb) {
            const int a2[2] = {ta & 1, ta >> 1}, b2[2] = {tb & 1, tb >> 1};
            RTM_CUDA(cudaMemcpyAsync(va, P4 + ta * G, G * sizeof(double2), cudaMemcpyDeviceToDevice, s));
            RTM_CUDA(cudaMemcpyAsync(vb, P4 + tb * G, G * sizeof(double2), cudaMemcpyDeviceToDevice, s));
            for (int d = 0; d < 2; ++d)
                if (a2[d] == 1 && b2[d] == 0) RTM_TRY(line_conv(t, d, K[d], va, s));
            for (int d = 0; d < 2; ++d)
                if (a2[d] == 0 && b2[d] == 1) RTM_TRY(line_conv(t, d, K[d], vb, s));
            k_spectra_arith<<<blocks, 256, 0, s>>>(0, G, va, vb, pr);
            count_launch();
            for (int d = 0; d < 2; ++d)
                if (a2[d] == 1 && b2[d] == 1) RTM_TRY(line_conv(t, d, K[d], pr, s));
            k_spectra_arith<<<blocks, 256, 0, s>>>(1, G, pr, nullptr, dst);
            count_launch();
        }
    k_spectra_arith<<<blocks, 256, 0, s>>>(2, G, dst, opt, dst);
    count_launch();
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

int build_circulant(const DeviceGenerators& g, double size_x, double size_y, int kernel, int builder,
                    const int* bandwidth, int precision, GridApplicator& out, cudaStream_t s) {
    const int cx = g.count_x, cy = g.count_y;
    layout(out, cx, cy);
    out.precision = precision;
    out.size_x = size_x;
    out.size_y = size_y;
    out.max_rhs = 1;
    out.P = cx;
    out.Q = cy;
    out.nsx = out.nsy = 1;
    RTM_TRY(fft_tables(out.P, &out.tP));
    RTM_TRY(fft_tables(out.Q, &out.tQ));
    GenArgs a{};
    a.kind = kSrcCirculant;
    a.P = cx;
    a.Q = cy;
    a.window = kernel == RTM_KERNEL_STRANG ? kWinStrang : kernel == RTM_KERNEL_TCHAN ? kWinTChan
               : kernel == RTM_KERNEL_RCHAN ? kWinRChan : kWinHuckle;
    a.bw_x = bandwidth ? bandwidth[0] : cx;
    a.bw_y = bandwidth ? bandwidth[1] : cy;
    a.planP = out.tP->plan;
    a.planQ = out.tQ->plan;
    a.twP = out.tP->tw64;
    a.twQ = out.tQ->tw64;
    a.realify = 0;
    const int64_t G = (int64_t)cx * cy;
    DeviceBuffer raw, inv, flag;
    StreamSyncGuard guard(s);
    RTM_TRY(raw.alloc(3 * (size_t)G * sizeof(double2)));
    RTM_CUDA(cudaMemsetAsync(raw.ptr, 0, raw.bytes, s));
    RTM_TRY(inv.alloc(4 * (size_t)G * sizeof(double2)));
    RTM_TRY(flag.alloc(sizeof(int)));
    RTM_CUDA(cudaMemsetAsync(flag.ptr, 0, sizeof(int), s));
    const double2* u = nullptr;
    const double2* v = nullptr;
    const float2* f = nullptr;
    RTM_TRY(shift_factors(cx, 0, &u, &f));
    RTM_TRY(shift_factors(cy, 0, &v, &f));
    const double2* gens[3] = {g.e.as<double2>(), g.xx.as<double2>(), g.yy.as<double2>()};
    const int grows[3] = {cx, cx - 1, cx};
    const int gcols[3] = {cy, cy, cy - 1};
    if (builder == RTM_BUILDER_PARTWISE && kernel != RTM_KERNEL_SUPEROPTIMAL) {
        for (int k = 0; k < 3; ++k) {
            if (!gens[k]) continue;
            GenItem& it = a.items[a.nitems++];
            it.g = gens[k];
            it.rows = grows[k];
            it.cols = gcols[k];
            it.px = it.py = 0;
            it.dst = raw.as<double2>() + k * G;
        }
        RTM_TRY(run_gen(a, s));
    } else {
        TwoSidedSpectra t{cx, cy, a.window, a.bw_x, a.bw_y, out.tP, out.tQ};
        const int64_t T = (int64_t)(2 * cx - 1) * (2 * cy - 1);
        const unsigned tb = (unsigned)std::min<int64_t>((T + 255) / 256, 1184);
        DeviceBuffer two;
        StreamSyncGuard two_guard(s);
        RTM_TRY(two.alloc(3 * (size_t)T * sizeof(double2)));
        RTM_CUDA(cudaMemsetAsync(two.ptr, 0, two.bytes, s));
        double2* S0 = two.as<double2>();
        if (builder == RTM_BUILDER_PARTWISE) {
            // generatePartwiseSpectra.m:16-30 with the superoptimal kernel: E, MXX, MYY one by one
            for (int k = 0; k < 3; ++k) {
                if (!gens[k]) continue;
                k_two_sided_even<<<tb, 256, 0, s>>>(cx, cy, gens[k], grows[k], gcols[k], S0);
                count_launch();
                RTM_TRY(two_sided_spectrum(t, kernel, S0, raw.as<double2>() + k * G, s));
            }
        } else {
            const bool has_x = out.content != RTM_YONLY, has_y = out.content != RTM_XONLY;
            double2* bxx = has_x ? S0 : nullptr;
            double2* bxy = has_x && has_y ? S0 + T : nullptr;
            double2* byy = has_y ? S0 + 2 * T : nullptr;
            k_spatial_blocks<<<tb, 256, 0, s>>>(cx, cy, gens[0], gens[1], gens[2], 1.0 / (size_x * size_x),
                                                 1.0 / (size_y * size_y), 1.0 / (size_x * size_y), bxx, bxy, byy);
            count_launch();
            double2* sxx = raw.as<double2>();  // reuse of raw: XX, coupling (XY or E), YY
            double2* sxy = sxx + G;
            double2* syy = sxy + G;
            if (bxx) RTM_TRY(two_sided_spectrum(t, kernel, bxx, sxx, s));
            if (byy) RTM_TRY(two_sided_spectrum(t, kernel, byy, syy, s));
            if (bxy) {
                if (builder == RTM_BUILDER_BLOCKWISE) {
                    RTM_TRY(two_sided_spectrum(t, kernel, bxy, sxy, s));
                } else {
                    // generateHybridSpectra.m:16-26: the coupling from the electric generator alone
                    k_two_sided_even<<<tb, 256, 0, s>>>(cx, cy, gens[0], cx, cy, bxy);
                    count_launch();
                    RTM_TRY(two_sided_spectrum(t, kernel, bxy, sxy, s));
                }
            }
            k_blocks_invert<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(
                cx, cy, out.content, builder == RTM_BUILDER_BLOCKWISE ? 0 : 1, sxx, sxy, syy, u, v,
                1.0 / (size_x * size_y), inv.as<double2>(), flag.as<int>());
            count_launch();
        }
        RTM_CUDA(cudaGetLastError());
    }
    if (builder == RTM_BUILDER_PARTWISE) {
        k_circulant_invert<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(cx, cy, out.content, raw.as<double2>(), u, v,
                                                                       1.0 / (size_x * size_x), 1.0 / (size_y * size_y),
                                                                       1.0 / (size_x * size_y), inv.as<double2>(),
                                                                       flag.as<int>());
        count_launch();
    }
    RTM_CUDA(cudaGetLastError());
    int bad = 0;
    RTM_CUDA(cudaMemcpyAsync(&bad, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    if (bad)
        return fail(RTM_ERR_SINGULAR, "The circulant approximation is singular at some frequency. Use another kernel "
                                      "or builder.");
    if (out.content == RTM_BOTH) {
        out.mode = kBlock4;
        RTM_TRY(convert_spectra(inv, precision, out.spec, s));
        out.spec_blocks = 4;
        out.max_rhs = 0;
        RTM_TRY(out.reserve(1));
    } else {
        // A strip: 1-D FFT of the face line with the single inverted block (FFTApplicator.m:52-59).
        out.mode = kStrip;
        const bool xs = out.content == RTM_XONLY;
        const int L = xs ? cx : cy;
        DeviceBuffer line;
        StreamSyncGuard line_guard(s);
        RTM_TRY(line.alloc((size_t)L * sizeof(double2)));
        RTM_CUDA(cudaMemcpyAsync(line.ptr, inv.as<double2>() + (xs ? 0 : 3 * G), L * sizeof(double2),
                                 cudaMemcpyDeviceToDevice, s));
        RTM_TRY(convert_spectra(line, precision, out.spec, s));
        out.spec_blocks = 1;
        out.P = L;
        out.Q = 1;
        out.nsx = 1;
        out.nsy = 1;
        RTM_TRY(fft_tables(L, &out.tP));
        RTM_TRY(fft_tables(1, &out.tQ));
        out.max_rhs = 1 << 20;  // a strip needs no working grid
    }
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

__global__ void k_modify(int64_t n, const double2* __restrict__ in, double2* __restrict__ out, int modifier) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = in[i];
        out[i] = modifier == RTM_MODIFY_REAL ? make_double2(v.x, 0.0)
                 : modifier == RTM_MODIFY_IMAG ? make_double2(v.y, 0.0) : v;
    }
}

int modify_generators(const DeviceGenerators& in, int modifier, DeviceGenerators& out, cudaStream_t s) {
    out.count_x = in.count_x;
    out.count_y = in.count_y;
    out.content = in.content;
    out.is_real = in.is_real || modifier != RTM_MODIFY_NONE;
    const DeviceBuffer* src[3] = {&in.xx, &in.yy, &in.e};
    DeviceBuffer* dst[3] = {&out.xx, &out.yy, &out.e};
    for (int k = 0; k < 3; ++k) {
        if (!src[k]->ptr) continue;
        RTM_TRY(dst[k]->alloc(src[k]->bytes));
        const int64_t n = (int64_t)(src[k]->bytes / sizeof(double2));
        k_modify<<<256, 256, 0, s>>>(n, src[k]->as<double2>(), dst[k]->as<double2>(), modifier);
        count_launch();
        RTM_CUDA(cudaGetLastError());
    }
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

}  // namespace rtm
