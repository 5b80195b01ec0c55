// Registry of the free-energy plugin styles compiled into the engine (the interface is described
// in include/shhd_b200_free_energy.cuh).  A style is registered by defining its struct below (or
// including its header) and naming it in SHHD_FREE_ENERGY_PLUGINS; ids follow that order from 1.
#pragma once

#include <cstring>

#include "../../include/shhd_b200_free_energy.cuh"

namespace shhd {
namespace plugins {

// Coupled quartic: f = sum_a u_a psi_a^4 / 4 + g / 2 sum_{a < b} psi_a^2 psi_b^2, so
// mu_a = u_a psi_a^3 + g psi_a sum_{b != a} psi_b^2.  g = 0 is phi4's physical part
// (model_free_energy_phi4.cc:47-55, evaluated in the same order); u_a = g for every a is the
// O(N)-symmetric (g / 4) (sum_b psi_b^2)^2.
struct CoupledPhi4 {
    static constexpr const char* kName = "coupled_phi4";
    static constexpr int kParams = 2;
    static constexpr const char* kKeys[kParams] = {"u[]", "g"};
    template <typename T, typename Params>
    __device__ static T mu(int a, T psi_a, const T* psi, int n, const Params& p) {
        T others = T(0);
#pragma unroll
        for (int b = 0; b < SHHD_MAX_ORDER_PARAMETERS; ++b)
            if (b < n && b != a) others += psi[b] * psi[b];
        return p(0, a) * psi_a * psi_a * psi_a + p(1, 0) * psi_a * others;
    }
    template <typename T, typename Params>
    __device__ static T density(const T* psi, int n, const Params& p) {
        T f = T(0), s2 = T(0), s4 = T(0);
#pragma unroll
        for (int b = 0; b < SHHD_MAX_ORDER_PARAMETERS; ++b)
            if (b < n) {
                const T q = psi[b] * psi[b];
                f += T(0.25) * p(0, b) * q * q;
                s2 += q;
                s4 += q * q;
            }
        return f + T(0.25) * p(1, 0) * (s2 * s2 - s4);  // g / 2 sum_{a<b} = g / 4 ((sum q)^2 - sum q^2)
    }
};

// Sixth-order (tricritical) Landau term per order parameter: f = sum_a (u_a psi_a^4 / 4 +
// w_a psi_a^6 / 6), mu_a = u_a psi_a^3 + w_a psi_a^5.
struct Phi6 {
    static constexpr const char* kName = "phi6";
    static constexpr int kParams = 2;
    static constexpr const char* kKeys[kParams] = {"u[]", "w[]"};
    template <typename T, typename Params>
    __device__ static T mu(int a, T psi_a, const T*, int, const Params& p) {
        const T q = psi_a * psi_a;
        return psi_a * q * (p(0, a) + p(1, a) * q);
    }
    template <typename T, typename Params>
    __device__ static T density(const T* psi, int n, const Params& p) {
        T f = T(0);
#pragma unroll
        for (int b = 0; b < SHHD_MAX_ORDER_PARAMETERS; ++b)
            if (b < n) {
                const T q = psi[b] * psi[b];
                f += q * q * (T(0.25) * p(0, b) + p(1, b) * q / T(6));
            }
        return f;
    }
};

}  // namespace plugins

#define SHHD_FREE_ENERGY_PLUGINS(X) \
    X(1, plugins::CoupledPhi4)      \
    X(2, plugins::Phi6)

// host view of the registry: names and parameter keys by id
struct PluginInfo {
    const char* name;
    int n_params;
    const char* const* keys;
};
inline int plugin_count() {
    int n = 0;
#define SHHD_COUNT(ID, S) ++n;
    SHHD_FREE_ENERGY_PLUGINS(SHHD_COUNT)
#undef SHHD_COUNT
    return n;
}
inline bool plugin_info(int id, PluginInfo* out) {
    switch (id) {
#define SHHD_INFO(ID, S)                                \
    case ID:                                            \
        static_assert(S::kParams <= SHHD_MAX_FE_PARAMS, "too many plugin parameters"); \
        *out = PluginInfo{S::kName, S::kParams, S::kKeys}; \
        return true;
        SHHD_FREE_ENERGY_PLUGINS(SHHD_INFO)
#undef SHHD_INFO
        default: return false;
    }
}
inline int plugin_id(const char* name) {
    PluginInfo info{};
    for (int id = 1; plugin_info(id, &info); ++id)
        if (std::strcmp(info.name, name) == 0) return id;
    return 0;
}

}  // namespace shhd
