// Host runtime of librtm.so: error reporting, the HBM budget ledger, device buffers, the FFT plan
// and twiddle caches, and the FP64 host tables of the assembler (Gauss-Legendre rules and the
// closed-form touching moments).
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <complex>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"

namespace rtm {

int64_t g_launches = 0;

static thread_local std::string t_error;

void set_error(const std::string& msg) { t_error = msg; }

int fail(int status, const std::string& msg) {
    set_error(msg);
    return status;
}

int cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ") in " + what);
    return RTM_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------------
// Budget (src/+rooftopMoM/+resources/Budget.m:43-106): a ceiling on the bytes the live handles
// hold together, and the device's free memory.
static std::mutex g_budget_mu;
static double g_ceiling = 0.0;  // <= 0: none
static double g_held = 0.0;

// A byte count as the reference's messages write it (src/+rooftopMoM/+resources/+utils/formatBytes.m):
// whole bytes below 1 kB, else one decimal in kB, MB, GB or TB (powers of 1024); an infinite count (no
// ceiling) reads "unlimited", an unknown one "unknown".
std::string format_bytes(double b) {
    if (std::isinf(b)) return "unlimited";
    if (std::isnan(b)) return "unknown";
    const char* units[] = {"B", "kB", "MB", "GB", "TB"};
    const int e = std::min(std::max((int)std::floor(std::log2(std::max(b, 1.0)) / 10), 0), 4);
    char buf[64];
    if (e == 0) snprintf(buf, sizeof buf, "%.0f B", std::round(b));
    else snprintf(buf, sizeof buf, "%.1f %s", b / std::pow(1024.0, e), units[e]);
    return buf;
}

int budget_require(double bytes, const char* what) {
    std::lock_guard<std::mutex> lk(g_budget_mu);
    if (g_ceiling > 0 && g_held + bytes > g_ceiling) {
        return fail(RTM_ERR_OOM_BUDGET, std::string(what) + " needs " + format_bytes(bytes) + ", but only " +
                                            format_bytes(std::max(0.0, g_ceiling - g_held)) +
                                            " of the memory ceiling of " + format_bytes(g_ceiling) + " are left.");
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess && bytes > (double)free_b) {
        return fail(RTM_ERR_OOM_BUDGET, std::string(what) + " needs " + format_bytes(bytes) + ", but only " +
                                            format_bytes((double)free_b) + " are free on this device.");
    }
    return RTM_OK;
}

void budget_hold(double bytes) {
    std::lock_guard<std::mutex> lk(g_budget_mu);
    g_held += bytes;
}

void budget_release(double bytes) {
    std::lock_guard<std::mutex> lk(g_budget_mu);
    g_held -= bytes;
}

// Per-device cache of idle device blocks, by capacity.
static std::mutex g_pool_mu;
static std::multimap<size_t, void*> g_pool[64];

static size_t block_capacity(size_t n) {
    if (n <= (1u << 20)) {
        size_t c = 512;
        while (c < n) c <<= 1;
        return c;
    }
    const size_t mb = 1u << 20;
    return (n + mb - 1) / mb * mb;
}

void release_cached_blocks() {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_pool_mu);
    for (auto& kv : g_pool[dev & 63]) cudaFree(kv.second);
    g_pool[dev & 63].clear();
}

int DeviceBuffer::alloc(size_t n) {
    reset();
    if (n == 0) return RTM_OK;
    cudaGetDevice(&device);
    const size_t cap = block_capacity(n);
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto& pool = g_pool[device & 63];
        auto it = pool.lower_bound(cap);
        if (it != pool.end() && it->first <= cap + cap / 2) {
            ptr = it->second;
            capacity = it->first;
            pool.erase(it);
        }
    }
    if (!ptr) {
        cudaError_t e = cudaMalloc(&ptr, cap);
        if (e != cudaSuccess) {
            cudaGetLastError();
            release_cached_blocks();
            e = cudaMalloc(&ptr, cap);
        }
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            return fail(RTM_ERR_OOM_BUDGET, "device allocation of " + format_bytes((double)n) + " failed: " +
                                                cudaGetErrorString(e));
        }
        capacity = cap;
    }
    bytes = n;
    budget_hold((double)n);
    return RTM_OK;
}

void DeviceBuffer::reset() {
    if (ptr) {
        {
            std::lock_guard<std::mutex> lk(g_pool_mu);
            g_pool[device & 63].emplace(capacity, ptr);
        }
        budget_release((double)bytes);
    }
    ptr = nullptr;
    bytes = 0;
    capacity = 0;
}

// ---------------------------------------------------------------------------------------------
// FFT plans and tables.
int fast_fft_size(int count) {
    // generateFastFFTSize.m:11-15: the smallest size >= count with prime factors <= 7.
    for (int n = count;; ++n) {
        int m = n;
        for (int p : {2, 3, 5, 7})
            while (m % p == 0) m /= p;
        if (m == 1) return n;
    }
}

static bool make_plan(int n, FftPlan& p) {
    p = FftPlan{};
    p.n = n;
    p.m = n;
    p.nstages = 0;
    int m = n;
    auto push = [&](int r) {
        if (p.nstages >= kMaxStages) return false;
        p.radix[p.nstages++] = r;
        m /= r;
        return true;
    };
    for (int r : {16, 8, 4, 2, 3, 5, 7}) {
        while (m % r == 0)
            if (!push(r)) return false;
    }
    for (int r = 11; m > 1; r += 2) {
        if (r > kMaxGenericRadix) return false;
        while (m % r == 0)
            if (!push(r)) return false;
    }
    return true;
}

struct TableKey {
    int device;
    int n;
    bool operator<(const TableKey& o) const { return device != o.device ? device < o.device : n < o.n; }
};

struct TableEntry {
    FftTables t;
    void* mem = nullptr;  // one allocation for the four tables; kept for the life of the process
};

static std::mutex g_tables_mu;
static std::map<TableKey, TableEntry> g_tables;

static void root_table(int n, long double scale, std::vector<double2>& out) {
    // exp(-i pi m scale / n) for m < n in long double, rounded once to double.
    const long double pi = 3.141592653589793238462643383279502884L;
    out.resize(n);
    for (int m = 0; m < n; ++m) {
        long double a = pi * scale * (long double)m / (long double)n;
        out[m] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
}

// In-place radix-2 DFT of a power-of-two length in long double (host; the Bluestein kernel spectrum).
static void host_dft_pow2(std::vector<std::complex<long double>>& a) {
    const size_t m = a.size();
    const long double pi = 3.141592653589793238462643383279502884L;
    for (size_t i = 1, j = 0; i < m; ++i) {
        size_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= m; len <<= 1) {
        for (size_t i = 0; i < m; i += len)
            for (size_t k = 0; k < len / 2; ++k) {
                const long double ang = -2.0L * pi * (long double)k / (long double)len;
                const std::complex<long double> w(cosl(ang), sinl(ang));
                const std::complex<long double> u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
    }
}

// Bluestein plan of length n: X_k = c_k sum_j (x_j c_j) b_(k-j) with c_j = exp(-i pi j^2 / n) and
// b_d = conj(c_d), the linear convolution evaluated as a circular one of length m >= 2n - 1 by two
// power-of-two transforms. Fills the radices of m and the three tables' host values.
static bool make_bluestein(int n, FftPlan& p, std::vector<double2>& chirp, std::vector<double2>& kern,
                           std::vector<double2>& twm) {
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    if (!make_plan(m, p)) return false;
    p.n = n;
    p.m = m;
    const long double pi = 3.141592653589793238462643383279502884L;
    chirp.resize(n);
    std::vector<std::complex<long double>> b(m, 0.0L);
    for (int j = 0; j < n; ++j) {
        // j^2 mod 2n keeps the angle small (exp(-i pi 2n / n) = 1)
        const long double a = pi * (long double)((int64_t)j * j % (2 * (int64_t)n)) / (long double)n;
        chirp[j] = make_double2((double)cosl(a), (double)(-sinl(a)));
        const std::complex<long double> bj(cosl(a), sinl(a));
        b[j] = bj;
        if (j) b[m - j] = bj;
    }
    host_dft_pow2(b);
    kern.resize(m);
    for (int k = 0; k < m; ++k) kern[k] = make_double2((double)(b[k].real() / m), (double)(b[k].imag() / m));
    twm.resize(m);
    for (int k = 0; k < m; ++k) {
        const long double a = 2.0L * pi * (long double)k / (long double)m;
        twm[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
    }
    return true;
}

int fft_tables(int n, const FftTables** out) {
    if (n < 1) return fail(RTM_ERR_ARG, "FFT length must be positive");
    int dev = 0;
    RTM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tables_mu);
    auto it = g_tables.find({dev, n});
    if (it != g_tables.end()) {
        *out = &it->second.t;
        return RTM_OK;
    }
    TableEntry e;
    std::vector<double2> chirp, kern, twm;
    if (!make_plan(n, e.t.plan) && !make_bluestein(n, e.t.plan, chirp, kern, twm))
        return fail(RTM_ERR_UNSUPPORTED, "FFT length " + std::to_string(n) + " has no plan in this build");
    std::vector<double2> tw, mod;
    root_table(n, 2.0L, tw);
    root_table(n, 1.0L, mod);
    std::vector<float2> tw32(n), mod32(n);
    for (int m = 0; m < n; ++m) {
        tw32[m] = make_float2((float)tw[m].x, (float)tw[m].y);
        mod32[m] = make_float2((float)mod[m].x, (float)mod[m].y);
    }
    size_t bytes = (size_t)n * (2 * sizeof(double2) + 2 * sizeof(float2));
    RTM_CUDA(cudaMalloc(&e.mem, bytes));
    char* base = (char*)e.mem;
    double2* d_tw = (double2*)base;
    double2* d_mod = d_tw + n;
    float2* d_tw32 = (float2*)(d_mod + n);
    float2* d_mod32 = d_tw32 + n;
    RTM_CUDA(cudaMemcpy(d_tw, tw.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    RTM_CUDA(cudaMemcpy(d_mod, mod.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    RTM_CUDA(cudaMemcpy(d_tw32, tw32.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    RTM_CUDA(cudaMemcpy(d_mod32, mod32.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    e.t.tw64 = d_tw;
    e.t.mod64 = d_mod;
    e.t.tw32 = d_tw32;
    e.t.mod32 = d_mod32;
    if (e.t.plan.m != n) {
        // the Bluestein tables, FP64 then FP32: chirp (n), kernel spectrum (m), roots of length m (m)
        const size_t cnt = chirp.size() + kern.size() + twm.size();
        void* mem = nullptr;
        RTM_CUDA(cudaMalloc(&mem, cnt * (sizeof(double2) + sizeof(float2))));
        std::vector<double2> all;
        all.insert(all.end(), chirp.begin(), chirp.end());
        all.insert(all.end(), kern.begin(), kern.end());
        all.insert(all.end(), twm.begin(), twm.end());
        std::vector<float2> all32(cnt);
        for (size_t i = 0; i < cnt; ++i) all32[i] = make_float2((float)all[i].x, (float)all[i].y);
        double2* d64 = (double2*)mem;
        float2* d32 = (float2*)(d64 + cnt);
        RTM_CUDA(cudaMemcpy(d64, all.data(), cnt * sizeof(double2), cudaMemcpyHostToDevice));
        RTM_CUDA(cudaMemcpy(d32, all32.data(), cnt * sizeof(float2), cudaMemcpyHostToDevice));
        e.t.plan.chirp64 = d64;
        e.t.plan.kern64 = d64 + chirp.size();
        e.t.plan.twm64 = d64 + chirp.size() + kern.size();
        e.t.plan.chirp32 = d32;
        e.t.plan.kern32 = d32 + chirp.size();
        e.t.plan.twm32 = d32 + chirp.size() + kern.size();
    }
    auto res = g_tables.emplace(TableKey{dev, n}, e);
    *out = &res.first->second.t;
    return RTM_OK;
}

struct ShiftEntry {
    double2* d64 = nullptr;
    float2* d32 = nullptr;
};
static std::map<std::pair<TableKey, int>, ShiftEntry> g_shifts;

int shift_factors(int n, int parity, const double2** out64, const float2** out32) {
    // generateShiftPhases.m:16-17: s(m) = exp(i pi (2m + parity) / n); returns u(m) = 1 - s(m).
    int dev = 0;
    RTM_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tables_mu);
    auto key = std::make_pair(TableKey{dev, n}, parity);
    auto it = g_shifts.find(key);
    if (it == g_shifts.end()) {
        const long double pi = 3.141592653589793238462643383279502884L;
        std::vector<double2> u(n);
        std::vector<float2> u32(n);
        for (int m = 0; m < n; ++m) {
            long double a = pi * (long double)(2 * m + parity) / (long double)n;
            u[m] = make_double2((double)(1.0L - cosl(a)), (double)(-sinl(a)));
            u32[m] = make_float2((float)u[m].x, (float)u[m].y);
        }
        ShiftEntry e;
        RTM_CUDA(cudaMalloc(&e.d64, n * sizeof(double2)));
        RTM_CUDA(cudaMalloc(&e.d32, n * sizeof(float2)));
        RTM_CUDA(cudaMemcpy(e.d64, u.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
        RTM_CUDA(cudaMemcpy(e.d32, u32.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
        it = g_shifts.emplace(key, e).first;
    }
    *out64 = it->second.d64;
    *out32 = it->second.d32;
    return RTM_OK;
}

// ---------------------------------------------------------------------------------------------
// Gauss-Legendre points and weights on [a, b] by Newton's method on P_n (same rule as the
// Golub-Welsch eigenvalue method of generateGaussLegendre1D.m:16-25, to rounding).
void gauss_legendre(int order, double a, double b, std::vector<double>& points, std::vector<double>& weights) {
    points.assign(order, 0.0);
    weights.assign(order, 0.0);
    const long double pi = 3.141592653589793238462643383279502884L;
    // P_order and its derivative at x by the three-term recurrence.
    auto legendre = [order](long double x, long double& p, long double& dp) {
        long double p0 = 1, p1 = x;
        for (int k = 2; k <= order; ++k) {
            long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        p = order == 0 ? 1 : p1;
        dp = order * (x * p1 - p0) / (x * x - 1);
    };
    if (order == 1) {
        points[0] = 0.0;
        weights[0] = 2.0;
    } else {
        for (int i = 0; i < order / 2; ++i) {
            long double x = cosl(pi * (i + 0.75L) / (order + 0.5L));
            long double p = 0, dp = 1;
            for (int iter = 0; iter < 100; ++iter) {
                legendre(x, p, dp);
                const long double dx = p / dp;
                x -= dx;
                if (fabsl(dx) < 1e-19L) break;
            }
            legendre(x, p, dp);
            const long double w = 2 / ((1 - x * x) * dp * dp);
            points[i] = (double)(-x);
            points[order - 1 - i] = (double)x;
            weights[i] = weights[order - 1 - i] = (double)w;
        }
        if (order % 2 == 1) {
            long double p = 0, dp = 1;
            legendre(0.0L, p, dp);
            points[order / 2] = 0.0;
            weights[order / 2] = (double)(2 / (dp * dp));
        }
    }
    for (int i = 0; i < order; ++i) {
        points[i] = (a + b) / 2 + (b - a) / 2 * points[i];
        weights[i] = (b - a) / 2 * weights[i];
    }
}

// ---------------------------------------------------------------------------------------------
// Closed-form moments of R^power over the touching offsets (generatePowerMoments.m:17-155,
// integrateMonomial.m:18-81). The mixed antiderivatives are the integrals themselves.
static double monomial(int power, int m, int n, double a, double b) {
    if (a == 0 || b == 0) return 0.0;
    const double R = std::sqrt(a * a + b * b);
    const double lb = std::asinh(b / a), la = std::asinh(a / b);
    const double a2 = a * a, b2 = b * b, a4 = a2 * a2, b4 = b2 * b2;
    auto P = [](double x, int k) { double r = 1; for (int i = 0; i < k; ++i) r *= x; return r; };
    if (power == -1) {
        if (m == 0 && n == 0) return a * lb + b * la;
        if (m == 0 && n == 1) return (-a2 + a * R + b2 * la) / 2;
        if (m == 1 && n == 0) return (-b2 + b * R + a2 * lb) / 2;
        if (m == 1 && n == 1) return (-P(a, 3) - P(b, 3) + (a2 + b2) * R) / 3;
        if (m == 2 && n == 0) return (a * b * R + 2 * P(a, 3) * lb - P(b, 3) * la) / 6;
        if (m == 2 && n == 1) return (-2 * a4 + a * (2 * a2 + b2) * R - b4 * la) / 8;
        if (m == 3 && n == 0) return (2 * b4 + b * (a2 - 2 * b2) * R + 3 * a4 * lb) / 12;
        if (m == 3 && n == 1) return (-3 * P(a, 5) + 2 * P(b, 5) + (3 * a4 + a2 * b2 - 2 * b4) * R) / 15;
    } else if (power == 1) {
        if (m == 0 && n == 0) return (2 * a * b * R + P(a, 3) * lb + P(b, 3) * la) / 6;
        if (m == 0 && n == 1) return (-2 * a4 + a * (2 * a2 + 5 * b2) * R + 3 * b4 * la) / 24;
        if (m == 1 && n == 0) return (-2 * b4 + b * (5 * a2 + 2 * b2) * R + 3 * a4 * lb) / 24;
        if (m == 1 && n == 1) return (-P(a, 5) - P(b, 5) + (a4 + 2 * a2 * b2 + b4) * R) / 15;
        if (m == 2 && n == 0) return (a * b * (6 * a2 + b2) * R + 4 * P(a, 5) * lb - P(b, 5) * la) / 40;
        if (m == 2 && n == 1) return (-8 * P(a, 6) + a * (8 * a4 + 14 * a2 * b2 + 3 * b4) * R - 3 * P(b, 6) * la) / 144;
        if (m == 3 && n == 0) return (4 * P(b, 6) + b * (21 * a4 + 2 * a2 * b2 - 4 * b4) * R + 15 * P(a, 6) * lb) / 180;
        if (m == 3 && n == 1)
            return (-5 * P(a, 7) + 2 * P(b, 7) + (5 * P(a, 6) + 8 * a4 * b2 + a2 * b4 - 2 * P(b, 6)) * R) / 105;
    } else if (power == 3) {
        if (m == 0 && n == 0) return (7 * a * b * (a2 + b2) * R + 3 * P(a, 5) * lb + 3 * P(b, 5) * la) / 40;
        if (m == 0 && n == 1) return (-8 * P(a, 6) + a * (8 * a4 + 26 * a2 * b2 + 33 * b4) * R + 15 * P(b, 6) * la) / 240;
        if (m == 1 && n == 0) return (-8 * P(b, 6) + b * (33 * a4 + 26 * a2 * b2 + 8 * b4) * R + 15 * P(a, 6) * lb) / 240;
        if (m == 1 && n == 1)
            return (-P(a, 7) - P(b, 7) + (P(a, 6) + 3 * a4 * b2 + 3 * a2 * b4 + P(b, 6)) * R) / 35;
        if (m == 2 && n == 0)
            return (a * b * (38 * a4 + 26 * a2 * b2 + 3 * b4) * R + 18 * P(a, 7) * lb - 3 * P(b, 7) * la) / 336;
        if (m == 2 && n == 1)
            return (-48 * P(a, 8) + a * (48 * P(a, 6) + 136 * a4 * b2 + 118 * a2 * b4 + 15 * P(b, 6)) * R -
                    15 * P(b, 8) * la) / 1920;
        if (m == 3 && n == 0)
            return (16 * P(b, 8) + b * (215 * P(a, 6) + 134 * a4 * b2 + 8 * a2 * b4 - 16 * P(b, 6)) * R +
                    105 * P(a, 8) * lb) / 2240;
        if (m == 3 && n == 1)
            return (-7 * P(a, 9) + 2 * P(b, 9) +
                    (7 * P(a, 8) + 19 * P(a, 6) * b2 + 15 * a4 * b4 + a2 * P(b, 6) - 2 * P(b, 8)) * R) / 315;
    }
    return NAN;
}

// rect[m][n][iu][iv]: integral of u^m v^n R^power over [iu, iu+1] x ratio [iv, iv+1].
static void rectangles(int power, double ratio, double rect[4][2][2][2]) {
    for (int m = 0; m < 4; ++m)
        for (int n = 0; n < 2; ++n) {
            double c[3][3];
            for (int k = 0; k < 3; ++k)
                for (int l = 0; l < 3; ++l) c[k][l] = monomial(power, m, n, (double)k, ratio * l);
            for (int k = 0; k < 2; ++k)
                for (int l = 0; l < 2; ++l) rect[m][n][k][l] = (c[k + 1][l + 1] - c[k][l + 1]) - (c[k + 1][l] - c[k][l]);
        }
    std::vector<double> pts, w;
    gauss_legendre(20, 0.0, 1.0, pts, w);
    for (int k = 0; k < 2; ++k)
        for (int l = 0; l < 2; ++l) {
            if (std::hypot((double)k, ratio * l) < std::max(1.0, ratio)) continue;
            for (int m = 0; m < 4; ++m)
                for (int n = 0; n < 2; ++n) {
                    double s = 0;
                    for (int i = 0; i < 20; ++i) {
                        double inner = 0;
                        const double u = k + pts[i];
                        for (int j = 0; j < 20; ++j) {
                            const double v = ratio * (l + pts[j]);
                            inner += w[j] * std::pow(u, m) * std::pow(v, n) * std::pow(std::sqrt(u * u + v * v), power);
                        }
                        s += w[i] * inner;
                    }
                    rect[m][n][k][l] = ratio * s;
                }
        }
}

static const double kWeights[4][2][4] = {
    {{1.0, 1.0, 0, 0}, {1.0, -1.0, 0, 0}},
    {{0.5, 1.0, 0.5, 0}, {0.5, 0.0, -0.5, 0}},
    {{0.5, 0.0, -0.5, 0}, {0.5, -1.0, 0.5, 0}},
    {{1.0 / 3, 0.5, 0.0, -1.0 / 6}, {1.0 / 3, -0.5, 0.0, 1.0 / 6}},
};
static const int kWeightLen[4] = {2, 3, 3, 4};
static const int kTouching[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};

// The weight on part [-1,0] or [0,1] as a polynomial in u = sigma * cell * (nu - offset).
static void compose_part(const double* weight, int len, int part, int offset, double cell, int count, double* coeffs,
                         int* interval) {
    const double e0 = part == 0 ? -1.0 : 0.0, e1 = part == 0 ? 0.0 : 1.0;
    const double s0 = e0 - offset, s1 = e1 - offset;
    const double sigma = s1 <= 0 ? -1.0 : 1.0;
    *interval = (int)std::min(sigma * s0, sigma * s1);
    for (int i = 0; i < count; ++i) coeffs[i] = 0;
    double term[8] = {1, 0, 0, 0, 0, 0, 0, 0};
    int tl = 1;
    for (int k = 0; k < len; ++k) {
        for (int i = 0; i < tl && i < count; ++i) coeffs[i] += weight[k] * term[i];
        double nt[8] = {0};
        for (int i = 0; i < tl; ++i) {
            nt[i] += term[i] * offset;
            nt[i + 1] += term[i] * (sigma / cell);
        }
        ++tl;
        for (int i = 0; i < tl; ++i) term[i] = nt[i];
    }
}

static void along_x(double a, double b, int power, double out[4][4]) {
    const double ratio = b / a;
    double rect[4][2][2][2];
    rectangles(power, ratio, rect);
    for (int k = 0; k < 4; ++k)
        for (int l = 0; l < 4; ++l) {
            double acc = 0;
            for (int s = 0; s < 2; ++s) {
                double ca[4];
                int ia;
                compose_part(kWeights[k][s], kWeightLen[k], s, kTouching[l][0], 1.0, 4, ca, &ia);
                for (int t = 0; t < 2; ++t) {
                    double cb[2];
                    int ib;
                    compose_part(kWeights[0][t], kWeightLen[0], t, kTouching[l][1], ratio, 2, cb, &ib);
                    for (int m = 0; m < 4; ++m)
                        for (int n = 0; n < 2; ++n) acc += ca[m] * rect[m][n][ia][ib] * cb[n];
                }
            }
            out[k][l] = std::pow(a, power) * acc / ratio;
        }
}

void power_moments(double size_x, double size_y, int power, double out[7][4]) {
    double ax[4][4], ay[4][4];
    along_x(size_x, size_y, power, ax);
    along_x(size_y, size_x, power, ay);
    static const int perm[4] = {0, 2, 1, 3};
    for (int l = 0; l < 4; ++l) {
        for (int k = 0; k < 4; ++k) out[k][l] = ax[k][l];
        for (int k = 1; k < 4; ++k) out[3 + k][l] = ay[k][perm[l]];
    }
}

void extracted_moments(double size_x, double size_y, double k, double out[7][4]) {
    double m1[7][4], p1[7][4], p3[7][4];
    power_moments(size_x, size_y, -1, m1);
    power_moments(size_x, size_y, 1, p1);
    power_moments(size_x, size_y, 3, p3);
    for (int r = 0; r < 7; ++r)
        for (int c = 0; c < 4; ++c) out[r][c] = m1[r][c] - k * k / 2 * p1[r][c] + k * k * k * k / 24 * p3[r][c];
}

}  // namespace rtm

// ---------------------------------------------------------------------------------------------
extern "C" int rtm_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return RTM_ERR_ARG;
    const std::string& e = rtm::t_error;
    const size_t n = std::min(len - 1, e.size());
    std::memcpy(buf, e.data(), n);
    buf[n] = '\0';
    return RTM_OK;
}

extern "C" int rtm_budget_configure(double ceiling_bytes) {
    std::lock_guard<std::mutex> lk(rtm::g_budget_mu);
    rtm::g_ceiling = ceiling_bytes > 0 ? ceiling_bytes : 0.0;
    return RTM_OK;
}

extern "C" int rtm_budget_query(double* ceiling_bytes, double* held_bytes) {
    std::lock_guard<std::mutex> lk(rtm::g_budget_mu);
    if (ceiling_bytes) *ceiling_bytes = rtm::g_ceiling;
    if (held_bytes) *held_bytes = rtm::g_held;
    return RTM_OK;
}

