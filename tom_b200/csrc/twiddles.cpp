// Twiddle tables (see twiddles.h).
#include "twiddles.h"

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

}  // namespace tg
