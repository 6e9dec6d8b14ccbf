// Twiddle tables (see twiddles.h).
#include "twiddles.h"
#include "fft_plan.h"

#include <cmath>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

namespace tg {

namespace {
std::mutex g_mu;
std::map<std::pair<int, int>, void*> g_f32, g_f64;  // (device, L) -> device table

template <typename C> std::map<std::pair<int, int>, void*>& table_map();
template <> std::map<std::pair<int, int>, void*>& table_map<float2>() { return g_f32; }
template <> std::map<std::pair<int, int>, void*>& table_map<double2>() { return g_f64; }

// cos and -sin of 2 pi m / L with the argument reduced to the first octant so
// every entry is accurate to the last bit of double.
void unit_root(int m, int L, double* c, double* s) {
    const double tau = 6.283185307179586476925286766559;
    long k = m % L;
    // exploit symmetry: angle = 2 pi k / L
    if (4 * k == L) { *c = 0; *s = -1; return; }
    if (2 * k == L) { *c = -1; *s = 0; return; }
    if (4 * k == 3L * L) { *c = 0; *s = 1; return; }
    const double a = tau * (double)k / (double)L;
    *c = std::cos(a);
    *s = -std::sin(a);
}
}  // namespace

template <typename C> const C* twiddle_table(int L) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || L <= 0) return nullptr;
    std::lock_guard<std::mutex> lock(g_mu);
    auto& mp = table_map<C>();
    auto key = std::make_pair(dev, L);
    auto it = mp.find(key);
    if (it != mp.end()) return static_cast<const C*>(it->second);
    std::vector<C> host(L);
    for (int m = 0; m < L; ++m) {
        double c, s;
        unit_root(m, L, &c, &s);
        host[m].x = (decltype(host[m].x))c;
        host[m].y = (decltype(host[m].y))s;
    }
    void* d = nullptr;
    if (cudaMalloc(&d, sizeof(C) * L) != cudaSuccess) return nullptr;
    if (cudaMemcpy(d, host.data(), sizeof(C) * L, cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(d);
        return nullptr;
    }
    mp[key] = d;
    return static_cast<const C*>(d);
}

template const float2* twiddle_table<float2>(int);
template const double2* twiddle_table<double2>(int);

// ------------------------------------------------------ run-time plans
namespace {
// Radices of a mixed-radix transform of length n: powers of two as 16s (then
// one 8, 4 or 2), then 3, 5, 7, 11, 13; -1 if another prime divides n.
int factor_stages(int n, unsigned char* r) {
    int k = 0, e2 = 0;
    while (n % 2 == 0) { n /= 2; ++e2; }
    while (e2 >= 4) { r[k++] = 16; e2 -= 4; }
    if (e2 == 3) r[k++] = 8;
    else if (e2 == 2) r[k++] = 4;
    else if (e2 == 1) r[k++] = 2;
    for (int q : {3, 5, 7, 11, 13})
        while (n % q == 0) {
            n /= q;
            if (k >= tgrt::kMaxStages) return -1;
            r[k++] = (unsigned char)q;
        }
    return n == 1 ? k : -1;
}

bool smooth2357(int n) {
    for (int q : {2, 3, 5, 7})
        while (n % q == 0) n /= q;
    return n == 1;
}

bool fits(int M, int elem_bytes) { return 2ll * (M + 1) * elem_bytes <= tgrt::kMaxBlockSmem; }

// Bluestein tables per (device, L): chirp and convolution spectrum
struct BlueKey {
    int dev, L, wide;
    bool operator<(const BlueKey& o) const {
        return dev != o.dev ? dev < o.dev : (L != o.L ? L < o.L : wide < o.wide);
    }
};
std::map<BlueKey, std::pair<void*, void*>> g_blue;
}  // namespace

bool rt_plan(int L, int elem_bytes, tgrt::Plan* p) {
    if (L < 1 || !p) return false;
    tgrt::Plan q{};
    q.L = L;
    int k = factor_stages(L, q.r);
    if (k >= 0) {
        q.blue = 0;
        q.M = L;
        q.nst = k;
    } else {
        int M = 2 * L - 1;
        while (!smooth2357(M)) ++M;
        k = factor_stages(M, q.r);
        if (k < 0) return false;
        q.blue = 1;
        q.M = M;
        q.nst = k;
    }
    if (!fits(q.M, elem_bytes)) return false;
    *p = q;
    return true;
}

template <typename C> bool rt_tabs(const tgrt::Plan& p, tgrt::Tabs<C>* t) {
    t->tw = twiddle_table<C>(p.M);
    t->chirp = t->bspec = nullptr;
    if (!t->tw) return false;
    if (!p.blue) return true;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const BlueKey key{dev, p.L, (int)sizeof(C)};
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_blue.find(key);
    if (it == g_blue.end()) {
        const int L = p.L, M = p.M;
        const double pi = 3.141592653589793238462643383279503;
        // c_n = exp(-i pi n^2 / L), n^2 reduced mod 2L exactly
        std::vector<double> cr(L), ci(L);
        for (int n = 0; n < L; ++n) {
            const long long m = ((long long)n * n) % (2ll * L);
            cr[n] = std::cos(pi * (double)m / (double)L);
            ci[n] = -std::sin(pi * (double)m / (double)L);
        }
        // B_k = (1/M) sum_m b_m exp(-2 pi i m k / M), b the cyclic conj(c) (|m| < L)
        std::vector<double> wr(M), wi(M);
        for (int m = 0; m < M; ++m) unit_root(m, M, &wr[m], &wi[m]);
        std::vector<C> hc(L), hb(M);
        for (int n = 0; n < L; ++n) {
            hc[n].x = (decltype(hc[n].x))cr[n];
            hc[n].y = (decltype(hc[n].y))ci[n];
        }
        for (int kk = 0; kk < M; ++kk) {
            double sr = cr[0], si = -ci[0];
            for (int m = 1; m < L; ++m) {
                // b_m = b_{M-m} = conj(c_m): the two terms pair to conj(c_m)(w^{mk} + w^{-mk})
                const long long e = ((long long)m * kk) % M;
                const double c2 = 2.0 * wr[e];  // w^{mk} + w^{-mk} = 2 cos(2 pi m k / M)
                sr += cr[m] * c2;
                si += -ci[m] * c2;
            }
            hb[kk].x = (decltype(hb[kk].x))(sr / M);
            hb[kk].y = (decltype(hb[kk].y))(si / M);
        }
        void *dc = nullptr, *db = nullptr;
        if (cudaMalloc(&dc, sizeof(C) * L) != cudaSuccess || cudaMalloc(&db, sizeof(C) * M) != cudaSuccess ||
            cudaMemcpy(dc, hc.data(), sizeof(C) * L, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(db, hb.data(), sizeof(C) * M, cudaMemcpyHostToDevice) != cudaSuccess) {
            if (dc) cudaFree(dc);
            if (db) cudaFree(db);
            cudaGetLastError();
            return false;
        }
        it = g_blue.emplace(key, std::make_pair(dc, db)).first;
    }
    t->chirp = static_cast<const C*>(it->second.first);
    t->bspec = static_cast<const C*>(it->second.second);
    return true;
}

template bool rt_tabs<float2>(const tgrt::Plan&, tgrt::Tabs<float2>*);
template bool rt_tabs<double2>(const tgrt::Plan&, tgrt::Tabs<double2>*);

}  // namespace tg
