// Green's-matrix generator assembly on the device.
//
// Follows the reference's
//   src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/generate.m:10-59
//   src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/private/integrateLattice_.m:17-127
//   src/+rooftopMoM/+assembler/+greensMatrix/@MomentAssembler/private/countNearOffsets_.m:1-11
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/generateReducedRule.m:21-66
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/integrateMoments.m:17-39
//   src/+rooftopMoM/+assembler/+greensMatrix/+utils/accumulateMoments.m:27-133
//   src/+rooftopMoM/+assembler/+singularIntegrals/evaluateRemainder.m:13-14
//
// Kernels:
//   k_far_blocks  - the kernel exp(-ikR)/R on the far lattice: block (m, n) holds the order^2
//                   points x = a (p - m), y = b (p - n); each block's four quadrant sums of the 7
//                   moment weights (28 complex numbers) are written out. FP64 sincos/sqrt/div bound.
//   k_near        - one CTA per near offset: 7 weighted sums over the near rule, the remainder of
//                   the singularity extraction on the touching offsets plus their closed form.
//   k_terms       - per offset: the moments (near, or four quadrant sums of the far blocks) and
//                   the 7 scaled combinations of accumulateMoments.m:43-49.
//   k_gather      - per generator entry: E at e; XX at e from e, e + u (rising, doubled at
//                   dX = 1), e - u (falling); YY likewise along y.
#include <cmath>
#include <vector>

#include "fft.cuh"
#include "grid.h"

namespace rtm {

static constexpr double kZ0 = 376.730313668;  // Constants.m:11
static constexpr double kPi = 3.141592653589793238462643383279502884;

constexpr int kBlocksPerCta = 32;
constexpr int kPointChunk = 64;

struct FarArgs {
    int cx, cy;        // faces; blocks are 0..cx x 0..cy
    int order;
    double a, b, k;
    const double* points;   // order far points p in (0, 1)
    const double* weights;  // [4 quadrants][7][order^2], point index px + order * py
    double2* sums;          // [28][(cx+1)(cy+1)], block index m + (cx+1) n
};

__global__ void __launch_bounds__(128) k_far_blocks(const FarArgs f) {
    __shared__ double2 K[kPointChunk][kBlocksPerCta];
    __shared__ double W[4][7][kPointChunk];
    const int64_t nblocks = (int64_t)(f.cx + 1) * (f.cy + 1);
    const int64_t first = (int64_t)blockIdx.x * kBlocksPerCta;
    const int tb = threadIdx.x % kBlocksPerCta;  // block within the CTA (lane)
    const int q = threadIdx.x / kBlocksPerCta;   // quadrant (warp)
    const int npts = f.order * f.order;
    double re[7], im[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) re[m] = im[m] = 0.0;
    for (int p0 = 0; p0 < npts; p0 += kPointChunk) {
        const int np = min(kPointChunk, npts - p0);
        for (int t = threadIdx.x; t < kPointChunk * kBlocksPerCta; t += blockDim.x) {
            const int bl = t % kBlocksPerCta, pt = t / kBlocksPerCta;
            const int64_t blk = first + bl;
            double2 v = make_double2(0.0, 0.0);
            if (pt < np && blk < nblocks) {
                const int m = (int)(blk % (f.cx + 1)), n = (int)(blk / (f.cx + 1));
                const int gp = p0 + pt;
                const int px = gp % f.order, py = gp / f.order;
                const double x = f.a * (f.points[px] - m);
                const double y = f.b * (f.points[py] - n);
                const double R = sqrt(x * x + y * y);
                double s, c;
                sincos(f.k * R, &s, &c);
                const double inv = 1.0 / R;
                v = make_double2(c * inv, -s * inv);
            }
            K[pt][bl] = v;
        }
        for (int t = threadIdx.x; t < 4 * 7 * kPointChunk; t += blockDim.x) {
            const int pt = t % kPointChunk, r = t / kPointChunk;
            (&W[0][0][0])[t] = pt < np ? f.weights[(int64_t)r * npts + p0 + pt] : 0.0;
        }
        __syncthreads();
        for (int pt = 0; pt < np; ++pt) {
            const double2 kv = K[pt][tb];
#pragma unroll
            for (int m = 0; m < 7; ++m) {
                const double w = W[q][m][pt];
                re[m] = fma(w, kv.x, re[m]);
                im[m] = fma(w, kv.y, im[m]);
            }
        }
        __syncthreads();
    }
    const int64_t blk = first + tb;
    if (blk < nblocks) {
#pragma unroll
        for (int m = 0; m < 7; ++m) f.sums[(int64_t)(q * 7 + m) * nblocks + blk] = make_double2(re[m], im[m]);
    }
}

struct NearArgs {
    int near_x, near_y;
    int px_count, py_count;   // nodes of the near rule along x and y
    double a, b, k;
    const double* nodes_x;
    const double* nodes_y;
    const double* weights;    // [7][px_count * py_count], nu fastest
    const double* extracted;  // [7][4] closed-form moments at (0,0), (1,0), (0,1), (1,1)
    int count_x, count_y;
    double2* moments;         // [near_x * near_y][7], offset dX + near_x dY
};

__device__ __forceinline__ double2 remainder_kernel(double R, double k) {
    // exp(-ikR)/R - (1/R - k^2 R / 2 + k^4 R^3 / 24), with exp(-ikR) - 1 = -2 sin^2(kR/2) - i sin(kR).
    double sh, ch;
    sincos(0.5 * k * R, &sh, &ch);
    const double em1_re = -2.0 * sh * sh;
    const double em1_im = -2.0 * sh * ch;
    const double k2 = k * k;
    return make_double2(em1_re / R + 0.5 * k2 * R - k2 * k2 / 24.0 * R * R * R, em1_im / R);
}

__global__ void __launch_bounds__(256) k_near(const NearArgs f) {
    const int off = blockIdx.x;
    const int dX = off % f.near_x, dY = off / f.near_x;
    const bool touching = dX <= 1 && dY <= 1;
    const int npts = f.px_count * f.py_count;
    double re[7], im[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) re[m] = im[m] = 0.0;
    for (int p = threadIdx.x; p < npts; p += blockDim.x) {
        const int ix = p % f.px_count, iy = p / f.px_count;
        const double x = f.a * (f.nodes_x[ix] - dX);
        const double y = f.b * (f.nodes_y[iy] - dY);
        const double R = sqrt(x * x + y * y);
        double2 kv;
        if (touching) {
            kv = remainder_kernel(R, f.k);
        } else {
            double s, c;
            sincos(f.k * R, &s, &c);
            kv = make_double2(c / R, -s / R);
        }
#pragma unroll
        for (int m = 0; m < 7; ++m) {
            const double w = f.weights[(int64_t)m * npts + p];
            re[m] = fma(w, kv.x, re[m]);
            im[m] = fma(w, kv.y, im[m]);
        }
    }
    __shared__ double red[7][2][8];
    const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
#pragma unroll
    for (int m = 0; m < 7; ++m) {
        double r = re[m], i = im[m];
        for (int o = 16; o > 0; o >>= 1) {
            r += __shfl_down_sync(0xffffffffu, r, o);
            i += __shfl_down_sync(0xffffffffu, i, o);
        }
        if (lane == 0) {
            red[m][0][warp] = r;
            red[m][1][warp] = i;
        }
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        const int m = threadIdx.x;
        double r = 0, i = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) {
            r += red[m][0][w];
            i += red[m][1][w];
        }
        // The closed-form moments of the extracted part on the touching pairs (generate.m:45-52);
        // only offsets inside the grid exist here.
        if (touching && dX < f.count_x && dY < f.count_y) r += f.extracted[m * 4 + dX + 2 * dY];
        f.moments[(int64_t)off * 7 + m] = make_double2(r, i);
    }
}

struct TermArgs {
    int cx, cy;
    int near_x, near_y;
    const double2* near;     // [near_x*near_y][7]
    const double2* sums;     // [28][(cx+1)(cy+1)]
    double2 scale_e, scale_m;
    double2* terms;          // [7][cx*cy], offset dX + cx dY
};

// accumulateMoments.m:43-49: E; XX at e, e - u, e + u; YY at e, e - u, e + u.
__constant__ double c_combine[7][7] = {
    {1, 0, 0, 0, 0, 0, 0},  {1, -1, -1, 2, 0, 0, 0}, {0, 1, 0, -1, 0, 0, 0}, {0, 0, 1, -1, 0, 0, 0},
    {1, 0, 0, 0, -1, -1, 2}, {0, 0, 0, 0, 1, 0, -1}, {0, 0, 0, 0, 0, 1, -1}};

__global__ void k_terms(const TermArgs t) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t G = (int64_t)t.cx * t.cy;
    if (idx >= G) return;
    const int dX = (int)(idx % t.cx), dY = (int)(idx / t.cx);
    double2 M[7];
    if (dX < t.near_x && dY < t.near_y) {
#pragma unroll
        for (int m = 0; m < 7; ++m) M[m] = t.near[(int64_t)(dX + t.near_x * dY) * 7 + m];
    } else {
        const int64_t nb = (int64_t)(t.cx + 1) * (t.cy + 1);
#pragma unroll
        for (int m = 0; m < 7; ++m) M[m] = make_double2(0, 0);
        // Quadrant (hx, hy) takes the block of the offset plus (hx == 0, hy == 0).
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int sx = (q % 2) == 0 ? 1 : 0, sy = (q / 2) == 0 ? 1 : 0;
            const int64_t blk = (dX + sx) + (int64_t)(t.cx + 1) * (dY + sy);
#pragma unroll
            for (int m = 0; m < 7; ++m) {
                const double2 v = t.sums[(int64_t)(q * 7 + m) * nb + blk];
                M[m].x += v.x;
                M[m].y += v.y;
            }
        }
    }
#pragma unroll
    for (int r = 0; r < 7; ++r) {
        double sr = 0, si = 0;
#pragma unroll
        for (int m = 0; m < 7; ++m) {
            sr += c_combine[r][m] * M[m].x;
            si += c_combine[r][m] * M[m].y;
        }
        const double2 sc = r == 0 ? t.scale_e : t.scale_m;
        t.terms[(int64_t)r * G + idx] = make_double2(sc.x * sr - sc.y * si, sc.x * si + sc.y * sr);
    }
}

__global__ void k_gather(int cx, int cy, const double2* __restrict__ terms, double2* __restrict__ E,
                         double2* __restrict__ XX, double2* __restrict__ YY) {
    const int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t G = (int64_t)cx * cy;
    if (idx >= G) return;
    const int r = (int)(idx % cx), c = (int)(idx / cx);
    auto T = [&](int k, int rr, int cc) { return terms[(int64_t)k * G + rr + (int64_t)cx * cc]; };
    E[idx] = T(0, r, c);
    if (XX && r <= cx - 2) {
        double2 v = T(1, r, c);
        const double f = (r + 1 == 1) ? 2.0 : 1.0;  // the reflected pair at dX = -1
        const double2 rising = T(2, r + 1, c);
        v.x += f * rising.x;
        v.y += f * rising.y;
        if (r >= 1) {
            const double2 falling = T(3, r - 1, c);
            v.x += falling.x;
            v.y += falling.y;
        }
        XX[r + (int64_t)(cx - 1) * c] = v;
    }
    if (YY && c <= cy - 2) {
        double2 v = T(4, r, c);
        const double f = (c + 1 == 1) ? 2.0 : 1.0;
        const double2 rising = T(5, r, c + 1);
        v.x += f * rising.x;
        v.y += f * rising.y;
        if (c >= 1) {
            const double2 falling = T(6, r, c - 1);
            v.x += falling.x;
            v.y += falling.y;
        }
        YY[r + (int64_t)cx * c] = v;
    }
}

// generateReducedRule.m:36-66 along one axis: nodes and the columns W00, W10, W01, W11.
static void reduced_axis(int order, int parts, std::vector<double>& nodes, std::vector<double>& w /* P x 4 */) {
    std::vector<double> pts, pw;
    gauss_legendre(order, 0.0, 1.0, pts, pw);
    const int P = 2 * order * parts;
    nodes.resize(P);
    w.resize((size_t)P * 4);
    for (int half = 0; half < 2; ++half)
        for (int p = 0; p < parts; ++p)
            for (int i = 0; i < order; ++i) {
                const int idx = half * order * parts + p * order + i;
                const double right = (pts[i] + p) / parts;
                const double nu = half == 0 ? right - 1.0 : right;
                nodes[idx] = nu;
                const double g = pw[i] / parts;
                const bool left = nu < 0;
                const double d = std::fabs(nu);
                const double w10 = left ? (1 + nu) * (1 + nu) / 2 : (1 - nu * nu) / 2;
                const double w01 = left ? (1 - nu * nu) / 2 : (1 - nu) * (1 - nu) / 2;
                w[(size_t)idx * 4 + 0] = g * (1 - d);
                w[(size_t)idx * 4 + 1] = g * w10;
                w[(size_t)idx * 4 + 2] = g * w01;
                w[(size_t)idx * 4 + 3] = g * (1 - d) * (1 - d) * (2 + d) / 6;
            }
}

// 7 x (Px*Py) weights, nu fastest: rows M00, M10, M01, M11 = W00(eta) W..(nu), rows N10, N01, N11
// = W..(eta) W00(nu) (generateReducedRule.m:33).
static void reduced_rule(int order, int parts_x, int parts_y, std::vector<double>& nx, std::vector<double>& ny,
                         std::vector<double>& weights) {
    std::vector<double> wx, wy;
    reduced_axis(order, parts_x, nx, wx);
    reduced_axis(order, parts_y, ny, wy);
    const int Px = (int)nx.size(), Py = (int)ny.size();
    weights.assign((size_t)7 * Px * Py, 0.0);
    for (int iy = 0; iy < Py; ++iy)
        for (int ix = 0; ix < Px; ++ix) {
            const size_t col = (size_t)iy * Px + ix;
            for (int r = 0; r < 4; ++r) weights[(size_t)r * Px * Py + col] = wy[(size_t)iy * 4] * wx[(size_t)ix * 4 + r];
            for (int r = 1; r < 4; ++r) weights[(size_t)(3 + r) * Px * Py + col] = wy[(size_t)iy * 4 + r] * wx[(size_t)ix * 4];
        }
}

static int count_near(int count, double size, double longest) {
    int n = 0;
    for (int d = 0; d < count; ++d)
        if (std::max(d - 1, 0) * size < 3 * longest) ++n;
    return n;
}

template <typename V> static int upload(DeviceBuffer& buf, const std::vector<V>& v, cudaStream_t s) {
    RTM_TRY(buf.alloc(v.size() * sizeof(V)));
    RTM_CUDA(cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, s));
    return RTM_OK;
}

int assemble_generators(int cx, int cy, double a, double b, double k, int near_order, int far_order,
                        DeviceGenerators& out, cudaStream_t s) {
    if (cx < 1 || cy < 1 || (cx == 1 && cy == 1)) return fail(RTM_ERR_ARG, "A single face carries no rooftop.");
    if (!(a > 0) || !(b > 0) || !(k > 0) || !std::isfinite(a) || !std::isfinite(b) || !std::isfinite(k))
        return fail(RTM_ERR_ARG, "face sizes and the wavenumber must be positive and finite");
    if (near_order < 1 || far_order < 1) return fail(RTM_ERR_ARG, "quadrature orders must be positive");
    out.count_x = cx;
    out.count_y = cy;
    const int64_t nxr = (int64_t)(cx - 1) * cy, nyr = (int64_t)cx * (cy - 1);
    out.content = (nxr > 0 && nyr > 0) ? RTM_BOTH : nxr > 0 ? RTM_XONLY : RTM_YONLY;
    out.is_real = false;
    const int64_t G = (int64_t)cx * cy;
    RTM_TRY(out.e.alloc(G * sizeof(double2)));
    if (nxr > 0) RTM_TRY(out.xx.alloc(nxr * sizeof(double2)));
    if (nyr > 0) RTM_TRY(out.yy.alloc(nyr * sizeof(double2)));

    // generate.m:20: i Z0 / (4 pi) (ab)^2 [1/k, k].
    const double base = kZ0 / (4 * kPi) * (a * b) * (a * b);
    const double2 scale_e = make_double2(0.0, base / k), scale_m = make_double2(0.0, base * k);
    const double longest = std::max(a, b);
    const int near_x = count_near(cx, a, longest), near_y = count_near(cy, b, longest);
    const double shortest = std::min(a, b);
    const int parts_x = (int)std::floor(a / shortest + 0.5), parts_y = (int)std::floor(b / shortest + 0.5);

    // Near pass.
    std::vector<double> nnx, nny, nw;
    reduced_rule(near_order, parts_x, parts_y, nnx, nny, nw);
    double ext[7][4];
    extracted_moments(a, b, k, ext);
    std::vector<double> extv(28);
    for (int r = 0; r < 7; ++r)
        for (int c = 0; c < 4; ++c) extv[r * 4 + c] = ext[r][c];
    DeviceBuffer d_nx, d_ny, d_nw, d_ext, d_near, d_pts, d_qw, d_sums, d_terms;
    StreamSyncGuard guard(s);
    RTM_TRY(upload(d_nx, nnx, s));
    RTM_TRY(upload(d_ny, nny, s));
    RTM_TRY(upload(d_nw, nw, s));
    RTM_TRY(upload(d_ext, extv, s));
    RTM_TRY(d_near.alloc((size_t)near_x * near_y * 7 * sizeof(double2)));
    NearArgs na{};
    na.near_x = near_x;
    na.near_y = near_y;
    na.px_count = (int)nnx.size();
    na.py_count = (int)nny.size();
    na.a = a;
    na.b = b;
    na.k = k;
    na.nodes_x = d_nx.as<double>();
    na.nodes_y = d_ny.as<double>();
    na.weights = d_nw.as<double>();
    na.extracted = d_ext.as<double>();
    na.count_x = cx;
    na.count_y = cy;
    na.moments = d_near.as<double2>();
    k_near<<<near_x * near_y, 256, 0, s>>>(na);
    count_launch();
    RTM_CUDA(cudaGetLastError());

    // Far lattice (quadrant weights of the far rule, one part per direction).
    std::vector<double> fnx, fny, fw;
    reduced_rule(far_order, 1, 1, fnx, fny, fw);
    const int o = far_order, P2 = 2 * o;
    std::vector<double> points(fnx.begin() + o, fnx.end());
    std::vector<double> qw((size_t)4 * 7 * o * o);
    for (int hy = 0; hy < 2; ++hy)
        for (int hx = 0; hx < 2; ++hx) {
            const int q = hx + 2 * hy;
            for (int m = 0; m < 7; ++m)
                for (int py = 0; py < o; ++py)
                    for (int px = 0; px < o; ++px) {
                        const size_t col = (size_t)(hy * o + py) * P2 + (hx * o + px);
                        qw[((size_t)q * 7 + m) * o * o + px + (size_t)o * py] = fw[(size_t)m * P2 * P2 + col];
                    }
        }
    RTM_TRY(upload(d_pts, points, s));
    RTM_TRY(upload(d_qw, qw, s));
    const int64_t nblocks = (int64_t)(cx + 1) * (cy + 1);
    RTM_TRY(d_sums.alloc((size_t)28 * nblocks * sizeof(double2)));
    FarArgs fa{};
    fa.cx = cx;
    fa.cy = cy;
    fa.order = o;
    fa.a = a;
    fa.b = b;
    fa.k = k;
    fa.points = d_pts.as<double>();
    fa.weights = d_qw.as<double>();
    fa.sums = d_sums.as<double2>();
    k_far_blocks<<<(unsigned)((nblocks + kBlocksPerCta - 1) / kBlocksPerCta), 128, 0, s>>>(fa);
    count_launch();
    RTM_CUDA(cudaGetLastError());

    RTM_TRY(d_terms.alloc((size_t)7 * G * sizeof(double2)));
    TermArgs ta{};
    ta.cx = cx;
    ta.cy = cy;
    ta.near_x = near_x;
    ta.near_y = near_y;
    ta.near = d_near.as<double2>();
    ta.sums = d_sums.as<double2>();
    ta.scale_e = scale_e;
    ta.scale_m = scale_m;
    ta.terms = d_terms.as<double2>();
    k_terms<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(ta);
    k_gather<<<(unsigned)((G + 255) / 256), 256, 0, s>>>(cx, cy, d_terms.as<double2>(), out.e.as<double2>(),
                                                        out.xx.as<double2>(), out.yy.as<double2>());
    count_launch(2);
    RTM_CUDA(cudaGetLastError());
    RTM_CUDA(cudaStreamSynchronize(s));
    return RTM_OK;
}

}  // namespace rtm
