// Dense operator and block-Jacobi preconditioner.
//
// The Green's-matrix entry between rooftops p and q follows the definition the reference's tests use
// (tests/+unit/Base.m:83-113): the magnetic generator of their direction at the offset of their first
// faces, minus sum over the two faces of each of div_p(f) E(f - f') div_q(f'), with the divergence
// +1/h on the first face and -1/h on the second (h the face size along the rooftop).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "fft.cuh"
#include "grid.h"
#include "ops.h"

namespace rtm {

__global__ void k_dense(const double2* __restrict__ A, const double2* __restrict__ x, double2* __restrict__ y, int64_t n,
                        const int* skip, int stride) {
    const int rhs = blockIdx.y;
    if (skip && skip[(int64_t)rhs * stride]) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2* xr = x + rhs * n;
    double re = 0, im = 0;
    for (int64_t j = 0; j < n; ++j) {
        const double2 a = A[i + j * n], v = xr[j];
        re += a.x * v.x - a.y * v.y;
        im += a.x * v.y + a.y * v.x;
    }
    y[rhs * n + i] = make_double2(re, im);
}

struct DenseOp : LinearOp {
    DeviceBuffer A;
    int apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) override {
        dim3 g((unsigned)((n + 127) / 128), nrhs);
        k_dense<<<g, 128, 0, s>>>(A.as<double2>(), static_cast<const double2*>(x), static_cast<double2*>(y), n,
                                  skip.ptr, skip.stride);
        count_launch();
        RTM_CUDA(cudaGetLastError());
        return RTM_OK;
    }
    double stored_bytes() const override { return (double)A.bytes; }
};

std::unique_ptr<LinearOp> make_dense_op(const double2* device_matrix, int64_t n, int* status) {
    auto op = std::make_unique<DenseOp>();
    op->n = n;
    op->precision = RTM_FP64;
    *status = op->A.alloc((size_t)n * n * sizeof(double2));
    if (*status != RTM_OK) return nullptr;
    if (cudaMemcpy(op->A.ptr, device_matrix, (size_t)n * n * sizeof(double2), cudaMemcpyDeviceToDevice) != cudaSuccess) {
        *status = fail(RTM_ERR_CUDA, "copy of the dense matrix failed");
        return nullptr;
    }
    return op;
}

// ---------------------------------------------------------------------------------------------
constexpr int kMaxBlockUnknowns = 16;

struct BjArgs {
    int cx, cy, bx, by, nbx, nby;
    double a, b;
    const double2* E;
    const double2* XX;
    const double2* YY;
    int64_t nx_roof;             // x-directed rooftops (offset of the y-directed ones)
    int* counts;                 // [blocks]
    int64_t* index;              // [blocks][kMaxBlockUnknowns]
    double2* inv;                // [blocks][kMaxBlockUnknowns^2], row-major
    int* singular;
};

__device__ double2 green_entry(const BjArgs& g, int dp, int ip, int jp, int dq, int iq, int jq) {
    double re = 0, im = 0;
    if (dp == dq) {
        const int dx = abs(ip - iq), dy = abs(jp - jq);
        const double2 m = dp == 0 ? g.XX[dx + (int64_t)(g.cx - 1) * dy] : g.YY[dx + (int64_t)g.cx * dy];
        re = m.x;
        im = m.y;
    }
    const double hp = dp == 0 ? g.a : g.b, hq = dq == 0 ? g.a : g.b;
    for (int s = 0; s < 2; ++s) {
        const int fi = ip + (s && dp == 0), fj = jp + (s && dp == 1);
        for (int t = 0; t < 2; ++t) {
            const int gi = iq + (t && dq == 0), gj = jq + (t && dq == 1);
            const double2 e = g.E[abs(fi - gi) + (int64_t)g.cx * abs(fj - gj)];
            const double w = ((s == t) ? 1.0 : -1.0) / (hp * hq);
            re -= w * e.x;
            im -= w * e.y;
        }
    }
    return make_double2(re, im);
}

// One thread per block: gather its rooftops, form the block of the Green's matrix, invert it by
// Gauss-Jordan elimination with partial pivoting.
__global__ void k_bj_build(const BjArgs g) {
    const int blk = blockIdx.x * blockDim.x + threadIdx.x;
    if (blk >= g.nbx * g.nby) return;
    const int I = blk % g.nbx, J = blk / g.nbx;
    int dir[kMaxBlockUnknowns], fi[kMaxBlockUnknowns], fj[kMaxBlockUnknowns];
    int64_t* idx = g.index + (int64_t)blk * kMaxBlockUnknowns;
    int cnt = 0;
    for (int d = 0; d < 2; ++d)
        for (int j = J * g.by; j < min((J + 1) * g.by, g.cy); ++j)
            for (int i = I * g.bx; i < min((I + 1) * g.bx, g.cx); ++i) {
                if (d == 0 && i > g.cx - 2) continue;
                if (d == 1 && j > g.cy - 2) continue;
                dir[cnt] = d;
                fi[cnt] = i;
                fj[cnt] = j;
                idx[cnt] = d == 0 ? i + (int64_t)(g.cx - 1) * j : g.nx_roof + i + (int64_t)g.cx * j;
                ++cnt;
            }
    g.counts[blk] = cnt;
    double2 A[kMaxBlockUnknowns][kMaxBlockUnknowns], B[kMaxBlockUnknowns][kMaxBlockUnknowns];
    for (int r = 0; r < cnt; ++r)
        for (int c = 0; c < cnt; ++c) {
            A[r][c] = green_entry(g, dir[r], fi[r], fj[r], dir[c], fi[c], fj[c]);
            B[r][c] = make_double2(r == c ? 1.0 : 0.0, 0.0);
        }
    for (int col = 0; col < cnt; ++col) {
        int piv = col;
        double best = -1;
        for (int r = col; r < cnt; ++r) {
            const double v = A[r][col].x * A[r][col].x + A[r][col].y * A[r][col].y;
            if (v > best) { best = v; piv = r; }
        }
        if (!(best > 0)) { atomicExch(g.singular, 1); return; }
        if (piv != col)
            for (int c = 0; c < cnt; ++c) {
                double2 t = A[col][c]; A[col][c] = A[piv][c]; A[piv][c] = t;
                t = B[col][c]; B[col][c] = B[piv][c]; B[piv][c] = t;
            }
        const double2 p = A[col][col];
        const double d = p.x * p.x + p.y * p.y;
        const double2 inv = make_double2(p.x / d, -p.y / d);
        for (int c = 0; c < cnt; ++c) { A[col][c] = cmul(A[col][c], inv); B[col][c] = cmul(B[col][c], inv); }
        for (int r = 0; r < cnt; ++r) {
            if (r == col) continue;
            const double2 f = A[r][col];
            for (int c = 0; c < cnt; ++c) {
                A[r][c] = csub(A[r][c], cmul(f, A[col][c]));
                B[r][c] = csub(B[r][c], cmul(f, B[col][c]));
            }
        }
    }
    double2* out = g.inv + (int64_t)blk * kMaxBlockUnknowns * kMaxBlockUnknowns;
    for (int r = 0; r < cnt; ++r)
        for (int c = 0; c < cnt; ++c) out[r * kMaxBlockUnknowns + c] = B[r][c];
}

// The inverses packed to S = 2 bx by unknowns a block, column-major inside the block (entry (r, c) at
// blk S^2 + c S + r), so the S threads of a block read S consecutive entries per column.
template <typename T2>
__global__ void k_bj_pack(int nblocks, int S, const double2* __restrict__ inv64, const int64_t* __restrict__ index,
                          T2* __restrict__ out, int64_t* __restrict__ packed_index) {
    const int64_t total = (int64_t)nblocks * S * S;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t blk = t / ((int64_t)S * S);
        const int e = (int)(t - blk * S * S), c = e / S, r = e % S;
        const double2 v = inv64[(blk * kMaxBlockUnknowns + r) * kMaxBlockUnknowns + c];
        out[t] = cmake<T2>(v.x, v.y);
        if (e < S) packed_index[blk * S + e] = index[blk * kMaxBlockUnknowns + e];
    }
}

// y(idx_r) = sum_c inv(r, c) x(idx_c) over the block's unknowns, one thread per (block, row). Where S divides
// the warp (blocks of 1, 2, 4, 8 or 16 unknowns, 2 x 2 faces among them), the S threads of a block each gather
// their own x(idx_r) and pass it to the others by warp shuffles, so a thread issues one index and one vector
// load instead of S of each; the sum runs over c in the same order either way.
template <typename T2, int SC>  // SC: S as a compile-time constant (the loops unroll), or 0
__device__ __forceinline__ void bj_rows(int nblocks, int S_, const int* __restrict__ counts,
                                        const int64_t* __restrict__ index, const T2* __restrict__ inv,
                                        const T2* __restrict__ xr, T2* __restrict__ yr, int64_t t) {
    const int S = SC ? SC : S_;
    const int blk = (int)(t / S), r = (int)(t % S);
    if ((32 % S) == 0) {
        // every lane reaches the shuffles: blocks past the end and rows past a block's count carry zeros
        const bool in = blk < nblocks;
        const int cnt = in ? counts[blk] : 0;
        const int64_t* idx = index + (int64_t)blk * S;
        const bool row = in && r < cnt;
        const T2 mine = row ? xr[idx[r]] : czero<T2>();
        const T2* col = inv + (int64_t)blk * S * S + r;
        const int base = (int)(threadIdx.x & 31) - r;  // the block's first lane (blocks align with warps)
        T2 acc = czero<T2>();
#pragma unroll 16
        for (int c = 0; c < S; ++c) {
            T2 v;
            v.x = __shfl_sync(0xffffffffu, mine.x, base + c);
            v.y = __shfl_sync(0xffffffffu, mine.y, base + c);
            if (c < cnt && row) acc = cadd(acc, cmul(col[c * S], v));
        }
        if (row) yr[idx[r]] = acc;
        return;
    }
    if (blk >= nblocks) return;
    const int cnt = counts[blk];
    if (r >= cnt) return;
    const int64_t* idx = index + (int64_t)blk * S;
    const T2* col = inv + (int64_t)blk * S * S + r;
    T2 acc = czero<T2>();
    // unrolled so that the loads of all columns are in flight together (the order of the sum is unchanged)
#pragma unroll 8
    for (int c = 0; c < cnt; ++c) acc = cadd(acc, cmul(col[c * S], xr[idx[c]]));
    yr[idx[r]] = acc;
}

template <typename T2>
__global__ void k_bj_apply(int nblocks, int S, const int* __restrict__ counts, const int64_t* __restrict__ index,
                           const T2* __restrict__ inv, const T2* __restrict__ x, T2* __restrict__ y, int64_t n,
                           const int* skip, int stride) {
    const int rhs = blockIdx.y;
    if (skip && skip[(int64_t)rhs * stride]) return;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (S == 8) bj_rows<T2, 8>(nblocks, S, counts, index, inv, x + rhs * n, y + rhs * n, t);
    else bj_rows<T2, 0>(nblocks, S, counts, index, inv, x + rhs * n, y + rhs * n, t);
}

// k_bj_apply for a batch of block-Jacobi operators: right-hand side k takes entry k's blocks.
template <typename T2>
__global__ void k_bj_apply_batch(const BjEntry* __restrict__ entries, const T2* __restrict__ x, T2* __restrict__ y,
                                 int64_t stride, const int* skip, int skip_stride) {
    const int rhs = blockIdx.y;
    if (skip && skip[(int64_t)rhs * skip_stride]) return;
    const BjEntry e = entries[rhs];
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (e.S == 8)
        bj_rows<T2, 8>(e.nblocks, e.S, e.counts, e.index, static_cast<const T2*>(e.inv), x + rhs * stride,
                       y + rhs * stride, t);
    else
        bj_rows<T2, 0>(e.nblocks, e.S, e.counts, e.index, static_cast<const T2*>(e.inv), x + rhs * stride,
                       y + rhs * stride, t);
}

int apply_block_jacobi_batch(const BjEntry* entries, int count, int max_blocks, int S, int precision, const void* x,
                             void* y, int64_t stride, cudaStream_t s, SkipFlags skip) {
    const int64_t threads = (int64_t)max_blocks * S;
    const dim3 g((unsigned)((threads + 255) / 256), count);
    if (precision == RTM_FP64)
        k_bj_apply_batch<double2><<<g, 256, 0, s>>>(entries, static_cast<const double2*>(x), static_cast<double2*>(y),
                                                    stride, skip.ptr, skip.stride);
    else
        k_bj_apply_batch<float2><<<g, 256, 0, s>>>(entries, static_cast<const float2*>(x), static_cast<float2*>(y),
                                                   stride, skip.ptr, skip.stride);
    count_launch();
    RTM_CUDA(cudaGetLastError());
    return RTM_OK;
}

struct BlockJacobi : LinearOp {
    int nblocks = 0;
    int S = kMaxBlockUnknowns;  // unknowns a block at most (packed stride)
    DeviceBuffer counts, index, inv;
    int apply(const void* x, void* y, int nrhs, cudaStream_t s, SkipFlags skip) override {
        const int64_t threads = (int64_t)nblocks * S;
        dim3 g((unsigned)((threads + 255) / 256), nrhs);
        if (precision == RTM_FP64)
            k_bj_apply<double2><<<g, 256, 0, s>>>(nblocks, S, counts.as<int>(), index.as<int64_t>(), inv.as<double2>(),
                                                  static_cast<const double2*>(x), static_cast<double2*>(y), n, skip.ptr,
                                                  skip.stride);
        else
            k_bj_apply<float2><<<g, 256, 0, s>>>(nblocks, S, counts.as<int>(), index.as<int64_t>(), inv.as<float2>(),
                                                 static_cast<const float2*>(x), static_cast<float2*>(y), n, skip.ptr,
                                                 skip.stride);
        count_launch();
        RTM_CUDA(cudaGetLastError());
        return RTM_OK;
    }
    double stored_bytes() const override { return (double)(counts.bytes + index.bytes + inv.bytes); }
};

bool block_jacobi_entry(const LinearOp* op, BjEntry* out) {
    const auto* bj = dynamic_cast<const BlockJacobi*>(op);
    if (!bj) return false;
    out->nblocks = bj->nblocks;
    out->S = bj->S;
    out->counts = bj->counts.as<int>();
    out->index = bj->index.as<int64_t>();
    out->inv = bj->inv.ptr;
    return true;
}

std::unique_ptr<LinearOp> make_block_jacobi(const DeviceGenerators& gen, double size_x, double size_y, int bx, int by,
                                            int precision, cudaStream_t s, int* status) {
    if (bx < 1 || by < 1 || 2 * bx * by > kMaxBlockUnknowns) {
        *status = fail(RTM_ERR_UNSUPPORTED, "block-Jacobi blocks hold at most 8 faces in this build");
        return nullptr;
    }
    auto op = std::make_unique<BlockJacobi>();
    const int cx = gen.count_x, cy = gen.count_y;
    const int64_t nx_roof = (int64_t)(cx - 1) * cy, ny_roof = (int64_t)cx * (cy - 1);
    op->n = nx_roof + ny_roof;
    op->precision = precision;
    BjArgs g{};
    g.cx = cx;
    g.cy = cy;
    g.bx = bx;
    g.by = by;
    g.nbx = (cx + bx - 1) / bx;
    g.nby = (cy + by - 1) / by;
    g.a = size_x;
    g.b = size_y;
    g.E = gen.e.as<double2>();
    g.XX = gen.xx.as<double2>();
    g.YY = gen.yy.as<double2>();
    g.nx_roof = nx_roof;
    op->nblocks = g.nbx * g.nby;
    const size_t nb = (size_t)op->nblocks;
    DeviceBuffer inv64, index16, flag;
    StreamSyncGuard guard(s);
    if ((*status = op->counts.alloc(nb * sizeof(int))) != RTM_OK) return nullptr;
    if ((*status = index16.alloc(nb * kMaxBlockUnknowns * sizeof(int64_t))) != RTM_OK) return nullptr;
    if ((*status = inv64.alloc(nb * kMaxBlockUnknowns * kMaxBlockUnknowns * sizeof(double2))) != RTM_OK) return nullptr;
    if ((*status = flag.alloc(sizeof(int))) != RTM_OK) return nullptr;
    if ((*status = check_cuda(cudaMemsetAsync(flag.ptr, 0, sizeof(int), s), "block-Jacobi flag")) != RTM_OK)
        return nullptr;
    g.counts = op->counts.as<int>();
    g.index = index16.as<int64_t>();
    g.inv = inv64.as<double2>();
    g.singular = flag.as<int>();
    // a preference only: a device that declines it runs the build all the same
    if (cudaFuncSetAttribute(k_bj_build, cudaFuncAttributePreferredSharedMemoryCarveout, 0) != cudaSuccess)
        (void)cudaGetLastError();
    k_bj_build<<<(unsigned)((nb + 63) / 64), 64, 0, s>>>(g);
    count_launch();
    if ((*status = check_cuda(cudaGetLastError(), "block-Jacobi build launch")) != RTM_OK) return nullptr;
    int bad = 0;
    if ((*status = check_cuda(cudaMemcpyAsync(&bad, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, s),
                              "block-Jacobi flag")) != RTM_OK)
        return nullptr;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        *status = cuda_fail(e, "block-Jacobi build");
        return nullptr;
    }
    if (bad) {
        *status = fail(RTM_ERR_SINGULAR, "a block of the block-Jacobi preconditioner is singular");
        return nullptr;
    }
    const int S = 2 * bx * by;
    op->S = S;
    const int64_t cnt = (int64_t)nb * S * S;
    if ((*status = op->index.alloc(nb * S * sizeof(int64_t))) != RTM_OK) return nullptr;
    if ((*status = op->inv.alloc(cnt * (precision == RTM_FP64 ? sizeof(double2) : sizeof(float2)))) != RTM_OK)
        return nullptr;
    const unsigned pb = (unsigned)std::min<int64_t>((cnt + 255) / 256, 2368);
    if (precision == RTM_FP64)
        k_bj_pack<double2><<<pb, 256, 0, s>>>(op->nblocks, S, inv64.as<double2>(), index16.as<int64_t>(),
                                              op->inv.as<double2>(), op->index.as<int64_t>());
    else
        k_bj_pack<float2><<<pb, 256, 0, s>>>(op->nblocks, S, inv64.as<double2>(), index16.as<int64_t>(),
                                             op->inv.as<float2>(), op->index.as<int64_t>());
    count_launch();
    if ((e = cudaGetLastError()) == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        *status = cuda_fail(e, "block-Jacobi packing");
        return nullptr;
    }
    *status = RTM_OK;
    return op;
}

}  // namespace rtm
