// Shared-memory mixed-radix FFT engine for sm_100a (device code only).
//
// A CTA transforms, in place, `lines` lines of length n that sit in shared memory; element e of
// line l is at buf[l * ls + sk(e) * es]. The transform is a Stockham autosort FFT (natural order in and
// out): at a stage of radix R after sub-transforms of length Ns, butterfly j reads the R elements
// j + t n/R, twiddles them by w^(t k n/(Ns R)) with k = j mod Ns, applies a radix-R DFT and writes
// them to (j - k) R + k + q Ns. Butterflies are numbered line-fastest, so a warp touches the same
// position of consecutive lines (the callers pad or interleave lines to spread the banks). Radices 2, 4, 8 and 16 are hand-written, 3, 5 and 7 read their
// roots from the twiddle table, larger primes up to kMaxGenericRadix use a direct DFT.
// Twiddles are w^m = exp(-2 pi i m / n) (table of n entries); the inverse uses their conjugates
// and does not scale.
#pragma once

#include "internal.h"

namespace rtm {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
template <typename T2> __device__ __forceinline__ T2 czero();
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }
template <typename T2> __device__ __forceinline__ T2 cmake(double x, double y);
template <> __device__ __forceinline__ double2 cmake<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 cmake<float2>(double x, double y) {
    return make_float2((float)x, (float)y);
}

// v * (-i) for the forward transform, v * (+i) for the inverse.
template <bool INV, typename T2> __device__ __forceinline__ T2 rot(T2 v) {
    T2 r;
    if (INV) { r.x = -v.y; r.y = v.x; } else { r.x = v.y; r.y = -v.x; }
    return r;
}

// Multiplies by (c, s) for the forward transform and by (c, -s) for the inverse, where (c, s) is
// a forward root of unity exp(-i theta) = (cos theta, -sin theta) given as c and s = -sin theta.
template <bool INV, typename T2, typename S> __device__ __forceinline__ T2 twc(T2 v, S c, S s) {
    if (INV) s = -s;
    T2 r;
    r.x = v.x * c - v.y * s;
    r.y = v.x * s + v.y * c;
    return r;
}

template <bool INV, typename T2> __device__ __forceinline__ void dft2(T2& a, T2& b) {
    T2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <bool INV, typename T2> __device__ __forceinline__ void dft4(T2& a0, T2& a1, T2& a2, T2& a3) {
    T2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = rot<INV>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a2 = csub(t0, t2);
    a1 = cadd(t1, t3);
    a3 = csub(t1, t3);
}

// sqrt(1/2), cos(pi/8), sin(pi/8)
#define RTM_R2 0.70710678118654752440084436210485
#define RTM_C8 0.92387953251128675612818318939679
#define RTM_S8 0.38268343236508977172845998403040

template <bool INV, typename T2> __device__ __forceinline__ void dft8(T2* v) {
    using S = decltype(v[0].x);
    T2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    T2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    const S c = (S)RTM_R2;
    o1 = twc<INV>(o1, c, -c);
    o2 = rot<INV>(o2);
    o3 = twc<INV>(o3, -c, -c);
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
    v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
    v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <bool INV, typename T2> __device__ __forceinline__ void dft16(T2* v) {
    using S = decltype(v[0].x);
    T2 e[8], o[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) { e[t] = v[2 * t]; o[t] = v[2 * t + 1]; }
    dft8<INV>(e);
    dft8<INV>(o);
    const S c1 = (S)RTM_C8, s1 = (S)RTM_S8, r2 = (S)RTM_R2;
    o[1] = twc<INV>(o[1], c1, -s1);
    o[2] = twc<INV>(o[2], r2, -r2);
    o[3] = twc<INV>(o[3], s1, -c1);
    o[4] = rot<INV>(o[4]);
    o[5] = twc<INV>(o[5], -s1, -c1);
    o[6] = twc<INV>(o[6], -r2, -r2);
    o[7] = twc<INV>(o[7], -c1, -s1);
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        v[t] = cadd(e[t], o[t]);
        v[t + 8] = csub(e[t], o[t]);
    }
}

// Odd radix R by its definition, with the roots w_R^m = tw[m n / R] of the length-n table.
template <int R, bool INV, typename T2> __device__ __forceinline__ void dft_odd(T2* v, const T2* __restrict__ tw, int n) {
    const int st = n / R;
    T2 w[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        T2 t = tw[m * st];
        w[m] = INV ? cconj(t) : t;
    }
    T2 out[R];
    T2 s = v[0];
#pragma unroll
    for (int t = 1; t < R; ++t) s = cadd(s, v[t]);
    out[0] = s;
#pragma unroll
    for (int q = 1; q < R; ++q) {
        T2 acc = v[0];
#pragma unroll
        for (int t = 1; t < R; ++t) acc = cadd(acc, cmul(v[t], w[(t * q) % R]));
        out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

template <int R, bool INV, typename T2> __device__ __forceinline__ void dft(T2* v, const T2* __restrict__ tw, int n) {
    if constexpr (R == 2) dft2<INV>(v[0], v[1]);
    else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 8) dft8<INV>(v);
    else if constexpr (R == 16) dft16<INV>(v);
    else dft_odd<R, INV>(v, tw, n);
}

// Shared-memory position of element e of a line: one slot of padding after every 16 elements, so
// that the stride-16 writes of a first radix-16 stage fall on different banks.
__host__ __device__ __forceinline__ int sk(int e) { return e + (e >> 4); }

// Butterflies per thread of a stage of radix R (at most about 16 complex values in registers).
__host__ __device__ constexpr int fft_ipt(int r) {
    return r == 2 ? 8 : r == 3 ? 6 : r == 4 ? 4 : r == 5 ? 4 : r == 7 ? 3 : r == 8 ? 2 : 1;
}

// Elements a line buffer of plan p spans in shared memory (positions sk(e), e < p.m; p.m == p.n except
// for Bluestein plans, whose lines hold the convolution of length p.m).
__host__ __device__ inline int fft_span(const FftPlan& p) { return sk(p.m - 1) + 1; }

// Threads a CTA needs to transform `lines` lines of plan p in place (a multiple of 32).
__host__ __device__ inline int fft_threads(int lines, const FftPlan& p) {
    int t = 32;
    for (int s = 0; s < p.nstages; ++s) {
        const int r = p.radix[s];
        const int per = fft_ipt(r);
        const int need = (lines * (p.m / r) + per - 1) / per;
        t = need > t ? need : t;
    }
    return (t + 31) / 32 * 32;
}

// One in-place Stockham stage: every thread loads its butterflies into registers, the CTA
// synchronises, then every thread stores them. Needs items = lines n / R <= IPT blockDim.x.
template <int R, int IPT, bool INV, typename T2>
__device__ __forceinline__ void pass_ip_body(T2* buf, int n, int Ns, int lines, int ls, int es, const T2* tw) {
    const int nb = n / R;
    const int stride = n / (Ns * R);
    const int items = lines * nb;
    T2 v[IPT][R];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        const int it = threadIdx.x + q * blockDim.x;
        if (it < items) {
            const int line = it % lines, j = it / lines, k = j % Ns;
            const T2* s = buf + line * ls;
#pragma unroll
            for (int t = 0; t < R; ++t) v[q][t] = s[sk(j + t * nb) * es];
            if (Ns > 1) {
#pragma unroll
                for (int t = 1; t < R; ++t) {
                    const T2 w = tw[t * k * stride];
                    v[q][t] = INV ? cmulc(v[q][t], w) : cmul(v[q][t], w);
                }
            }
            dft<R, INV>(v[q], tw, n);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
        const int it = threadIdx.x + q * blockDim.x;
        if (it < items) {
            const int line = it % lines, j = it / lines, k = j % Ns;
            const int base = (j - k) * R + k;
            T2* d = buf + line * ls;
#pragma unroll
            for (int t = 0; t < R; ++t) d[sk(base + t * Ns) * es] = v[q][t];
        }
    }
    __syncthreads();
}

template <int R, int IPT, bool INV, typename T2>
__device__ __noinline__ void pass_ip(T2* buf, int n, int Ns, int lines, int ls, int es, const T2* tw) {
    pass_ip_body<R, IPT, INV>(buf, n, Ns, lines, ls, es, tw);
}

// Any radix up to kMaxGenericRadix (rare: sizes with a prime factor above 7) by a direct DFT; one
// butterfly per thread suffices since R > 16.
template <bool INV, typename T2>
__device__ __noinline__ void pass_ip_generic(T2* buf, int n, int R, int Ns, int lines, int ls, int es, const T2* tw) {
    const int nb = n / R;
    const int stride = n / (Ns * R);
    const int st = n / R;
    const int items = lines * nb;
    const int it = threadIdx.x;
    T2 v[kMaxGenericRadix];
    int line = 0, j = 0, k = 0;
    if (it < items) {
        line = it % lines;
        j = it / lines;
        k = j % Ns;
        const T2* s = buf + line * ls;
        for (int t = 0; t < R; ++t) {
            T2 x = s[sk(j + t * nb) * es];
            if (Ns > 1 && t > 0) {
                const T2 w = tw[t * k * stride];
                x = INV ? cmulc(x, w) : cmul(x, w);
            }
            v[t] = x;
        }
    }
    __syncthreads();
    if (it < items) {
        const int base = (j - k) * R + k;
        T2* d = buf + line * ls;
        for (int q = 0; q < R; ++q) {
            T2 acc = v[0];
            for (int t = 1; t < R; ++t) {
                const T2 w = tw[((t * q) % R) * st];
                acc = cadd(acc, INV ? cmulc(v[t], w) : cmul(v[t], w));
            }
            d[sk(base + q * Ns) * es] = acc;
        }
    }
    __syncthreads();
}

// The Stockham stages of plan p over transforms of length n (p.n, or p.m inside a Bluestein plan).
template <bool INV, bool POW2, typename T2>
__device__ __forceinline__ void fft_stages(T2* buf, int lines, int ls, int es, const FftPlan& p, int n, const T2* tw) {
    int Ns = 1;
    for (int s = 0; s < p.nstages; ++s) {
        const int r = p.radix[s];
        if constexpr (POW2) {
            switch (r) {
                case 2: pass_ip_body<2, 8, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 4: pass_ip_body<4, 4, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 8: pass_ip_body<8, 2, INV>(buf, n, Ns, lines, ls, es, tw); break;
                default: pass_ip_body<16, 1, INV>(buf, n, Ns, lines, ls, es, tw); break;
            }
        } else {
            switch (r) {
                case 2: pass_ip<2, 8, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 3: pass_ip<3, 6, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 4: pass_ip<4, 4, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 5: pass_ip<5, 4, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 7: pass_ip<7, 3, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 8: pass_ip<8, 2, INV>(buf, n, Ns, lines, ls, es, tw); break;
                case 16: pass_ip<16, 1, INV>(buf, n, Ns, lines, ls, es, tw); break;
                default: pass_ip_generic<INV>(buf, n, r, Ns, lines, ls, es, tw); break;
            }
        }
        Ns *= r;
    }
}

template <typename T2> struct BluesteinTables;
template <> struct BluesteinTables<double2> {
    __device__ static const double2* chirp(const FftPlan& p) { return p.chirp64; }
    __device__ static const double2* kern(const FftPlan& p) { return p.kern64; }
    __device__ static const double2* roots(const FftPlan& p) { return p.twm64; }
};
template <> struct BluesteinTables<float2> {
    __device__ static const float2* chirp(const FftPlan& p) { return p.chirp32; }
    __device__ static const float2* kern(const FftPlan& p) { return p.kern32; }
    __device__ static const float2* roots(const FftPlan& p) { return p.twm32; }
};

// Bluestein (chirp-z) transform of length p.n on line buffers of p.m elements: with c_j = exp(-i pi j^2 / n),
// X_k = c_k sum_j (x_j c_j) conj(c_(k-j)), the linear convolution taken as a circular one of the
// power-of-two length m >= 2n - 1 (kern = DFT_m of the wrapped conj(c_d), divided by m). The inverse uses
// the conjugate chirp and the conjugate kernel spectrum (the wrapped chirp is even). Entries e >= n of
// the buffers are overwritten.
template <bool INV, typename T2>
__device__ __noinline__ void fft_bluestein(T2* buf, int lines, int ls, int es, const FftPlan& p) {
    const T2* chirp = BluesteinTables<T2>::chirp(p);
    const T2* kern = BluesteinTables<T2>::kern(p);
    const T2* roots = BluesteinTables<T2>::roots(p);
    const int n = p.n, m = p.m;
    for (int it = threadIdx.x; it < lines * m; it += blockDim.x) {
        const int line = it % lines, e = it / lines;
        T2& v = buf[line * ls + sk(e) * es];
        v = e < n ? (INV ? cmulc(v, __ldg(&chirp[e])) : cmul(v, __ldg(&chirp[e]))) : czero<T2>();
    }
    __syncthreads();
    fft_stages<false, true>(buf, lines, ls, es, p, m, roots);
    for (int it = threadIdx.x; it < lines * m; it += blockDim.x) {
        const int line = it % lines, e = it / lines;
        T2& v = buf[line * ls + sk(e) * es];
        v = INV ? cmulc(v, __ldg(&kern[e])) : cmul(v, __ldg(&kern[e]));
    }
    __syncthreads();
    fft_stages<true, true>(buf, lines, ls, es, p, m, roots);
    for (int it = threadIdx.x; it < lines * n; it += blockDim.x) {
        const int line = it % lines, e = it / lines;
        T2& v = buf[line * ls + sk(e) * es];
        v = INV ? cmulc(v, __ldg(&chirp[e])) : cmul(v, __ldg(&chirp[e]));
    }
    __syncthreads();
}

// Transforms, in place, the `lines` lines of length p.n in buf (element e of line l at
// buf[l * ls + sk(e) * es]; a line spans fft_span(p) elements); tw (global or shared) holds the p.n
// roots. Needs blockDim.x >= fft_threads(lines, p); call it after a __syncthreads() that makes buf
// visible; it returns after one. POW2 instantiates radices 16, 8, 4 and 2 inline (lengths that are
// powers of two, and Bluestein plans); otherwise every radix runs as a separate function.
template <bool INV, bool POW2, typename T2>
__device__ __forceinline__ void fft_inplace(T2* buf, int lines, int ls, int es, const FftPlan& p, const T2* tw) {
    if (p.m != p.n) {
        fft_bluestein<INV>(buf, lines, ls, es, p);
        return;
    }
    fft_stages<INV, POW2>(buf, lines, ls, es, p, p.n, tw);
}

// True when every radix of the plan is a power of two (the POW2 instantiation applies; Bluestein plans
// run power-of-two transforms of length p.m).
__host__ __device__ inline bool fft_pow2(const FftPlan& p) {
    for (int s = 0; s < p.nstages; ++s)
        if (p.radix[s] != 2 && p.radix[s] != 4 && p.radix[s] != 8 && p.radix[s] != 16) return false;
    return true;
}

}  // namespace rtm
