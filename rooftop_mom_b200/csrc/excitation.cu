// Excitations and results on the device.
//
// Follows the reference's
//   src/+rooftopMoM/+operator/generatePlaneWave.m:18-42     (reference rooftop x separable phase)
//   src/+rooftopMoM/+operator/generateDeltaGap.m:13-14
//   src/+rooftopMoM/+operator/+utils/generateMiddlePort.m:14-28
//   src/+rooftopMoM/+operator/computeRadarCrossSection.m:18-19
//   src/+rooftopMoM/+operator/computeInputImpedance.m:17
#include <cmath>
#include <complex>
#include <vector>

#include "excitation.h"
#include "fft.cuh"

namespace rtm {

static constexpr double kZ0e = 376.730313668;

struct WaveArgs {
    int cx, cy;
    double a, b, k;
    int64_t n, nx;        // rooftops, x-directed rooftops
    const double* dirs;   // [rhs][3]
    const double2* refs;  // [rhs][2]: reference rooftop values of the x and y directions
};

// Entry (m, n) of a direction = its reference value times exp(s_x m) exp(s_y n), s = -i k d a.
__global__ void k_plane_wave(const WaveArgs w, double2* __restrict__ out) {
    const int rhs = blockIdx.y;
    const double* d = w.dirs + 3 * rhs;
    const double tx = -w.k * d[0] * w.a, ty = -w.k * d[1] * w.b;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < w.n; t += (int64_t)gridDim.x * blockDim.x) {
        int m, q, dir;
        if (t < w.nx) {
            dir = 0;
            m = (int)(t % (w.cx - 1));
            q = (int)(t / (w.cx - 1));
        } else {
            dir = 1;
            const int64_t u = t - w.nx;
            m = (int)(u % w.cx);
            q = (int)(u / w.cx);
        }
        double s1, c1, s2, c2;
        sincos(tx * m, &s1, &c1);
        sincos(ty * q, &s2, &c2);
        const double2 ph = cmul(make_double2(c1, s1), make_double2(c2, s2));
        out[rhs * w.n + t] = cmul(w.refs[2 * rhs + dir], ph);
    }
}

int plane_wave(int cx, int cy, double a, double b, int order, double k, const double* dirs, const double* pols,
               const double* intens, int nrhs, double2* out_device, cudaStream_t s) {
    std::vector<double> pts, wts;
    gauss_legendre(order, 0.0, 1.0, pts, wts);
    const double area = a * b;
    std::vector<double2> refs(2 * nrhs);
    for (int r = 0; r < nrhs; ++r) {
        const double* d = dirs + 3 * r;
        const double* p = pols + 3 * r;
        const std::complex<double> sx(0.0, -k * d[0] * a), sy(0.0, -k * d[1] * b);
        for (int dir = 0; dir < 2; ++dir) {
            const std::complex<double> second = std::exp(dir == 0 ? sx : sy);
            std::complex<double> acc = 0;
            for (int iv = 0; iv < order; ++iv)
                for (int iu = 0; iu < order; ++iu) {
                    const double u = pts[iu], v = pts[iv];
                    const double coord = dir == 0 ? u : v;
                    const std::complex<double> phase = std::exp(sx * u + sy * v);
                    acc += phase * (wts[iu] * wts[iv] * (coord + second * (1.0 - coord)));
                }
            acc *= intens[r] * p[dir] * area;
            refs[2 * r + dir] = make_double2(acc.real(), acc.imag());
        }
    }
    DeviceBuffer d_dirs, d_refs;
    StreamSyncGuard guard(s);
    RTM_TRY(d_dirs.alloc(sizeof(double) * 3 * nrhs));
    RTM_TRY(d_refs.alloc(sizeof(double2) * 2 * nrhs));
    RTM_CUDA(cudaMemcpyAsync(d_dirs.ptr, dirs, sizeof(double) * 3 * nrhs, cudaMemcpyHostToDevice, s));
    RTM_CUDA(cudaMemcpyAsync(d_refs.ptr, refs.data(), sizeof(double2) * 2 * nrhs, cudaMemcpyHostToDevice, s));
    WaveArgs w{};
    w.cx = cx;
    w.cy = cy;
    w.a = a;
    w.b = b;
    w.k = k;
    w.nx = (int64_t)(cx - 1) * cy;
    w.n = w.nx + (int64_t)cx * (cy - 1);
    w.dirs = d_dirs.as<double>();
    w.refs = d_refs.as<double2>();
    dim3 g((unsigned)std::min<int64_t>((w.n + 255) / 256, 1184), nrhs);
    k_plane_wave<<<g, 256, 0, s>>>(w, out_device);
    count_launch();
    RTM_CUDA(cudaGetLastError());
    RTM_CUDA(cudaStreamSynchronize(s));  // the argument buffers are freed on return
    return RTM_OK;
}

// sum_i a_i b_i (unconjugated) into out[0], one CTA.
__global__ void k_dot_u(const double2* __restrict__ a, const double2* __restrict__ b, int64_t n, double2* out) {
    double re = 0, im = 0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double2 p = cmul(a[i], b[i]);
        re += p.x;
        im += p.y;
    }
    __shared__ double sr[1024], si[1024];
    sr[threadIdx.x] = re;
    si[threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sr[threadIdx.x] += sr[threadIdx.x + o];
            si[threadIdx.x] += si[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = make_double2(sr[0], si[0]);
}

// sum_p w_p J(port_p) into out[0], one CTA.
__global__ void k_port_sum(const double2* __restrict__ J, const int64_t* __restrict__ port, const double* __restrict__ w,
                           int count, double2* out) {
    double re = 0, im = 0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double2 v = J[port[i]];
        re += w[i] * v.x;
        im += w[i] * v.y;
    }
    __shared__ double sr[256], si[256];
    sr[threadIdx.x] = re;
    si[threadIdx.x] = im;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            sr[threadIdx.x] += sr[threadIdx.x + o];
            si[threadIdx.x] += si[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = make_double2(sr[0], si[0]);
}

int radar_cross_section(double k, const double2* e, const double2* J, int64_t n, double intensity, double* out,
                        cudaStream_t s) {
    DeviceBuffer r;
    StreamSyncGuard guard(s);
    RTM_TRY(r.alloc(sizeof(double2)));
    k_dot_u<<<1, 1024, 0, s>>>(e, J, n, r.as<double2>());
    count_launch();
    double2 v;
    RTM_CUDA(cudaMemcpyAsync(&v, r.ptr, sizeof v, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    const double kz = k * kZ0e;
    *out = kz * kz * (v.x * v.x + v.y * v.y) / (4 * M_PI * intensity * intensity * intensity * intensity);
    return RTM_OK;
}

int input_impedance(int cx, int cy, double a, double b, const double2* J, const int64_t* port_host, int count,
                    double voltage, double* out_re_im, cudaStream_t s) {
    const int64_t nx = (int64_t)(cx - 1) * cy;
    std::vector<double> w(count);
    for (int i = 0; i < count; ++i) w[i] = port_host[i] < nx ? b : a;  // edge lengths (UniformRooftops.m:89-101)
    DeviceBuffer d_port, d_w, r;
    StreamSyncGuard guard(s);
    RTM_TRY(d_port.alloc(sizeof(int64_t) * count));
    RTM_TRY(d_w.alloc(sizeof(double) * count));
    RTM_TRY(r.alloc(sizeof(double2)));
    RTM_CUDA(cudaMemcpyAsync(d_port.ptr, port_host, sizeof(int64_t) * count, cudaMemcpyHostToDevice, s));
    RTM_CUDA(cudaMemcpyAsync(d_w.ptr, w.data(), sizeof(double) * count, cudaMemcpyHostToDevice, s));
    k_port_sum<<<1, 256, 0, s>>>(J, d_port.as<int64_t>(), d_w.as<double>(), count, r.as<double2>());
    count_launch();
    double2 v;
    RTM_CUDA(cudaMemcpyAsync(&v, r.ptr, sizeof v, cudaMemcpyDeviceToHost, s));
    RTM_CUDA(cudaStreamSynchronize(s));
    const std::complex<double> z = voltage / std::complex<double>(v.x, v.y);
    out_re_im[0] = z.real();
    out_re_im[1] = z.imag();
    return RTM_OK;
}

}  // namespace rtm
