// Counter-based Gaussian noise for the stochastic fluxes.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11) keyed by (seed, member) with counter
// (mode id, stream, step lo, step hi).  One call gives the two complex
// standard normals an SRK3 step needs for one component at one mode (draws
// a and b), each from two 32-bit uniforms by Box-Muller.
//
// mode id = gx * Nay + (ky mod Nay), using |ky| on the kx = 0 line (the
// ky < 0 entry there is the conjugate of the ky > 0 draw, as the reference's
// psi_sto / j_sto write conjugate pairs, fcalculator.cc:531-562, 632-677).
// stream = alpha for psi_alpha and 4096 + m for the momentum stress draws
// xi_1..xi_3.
#pragma once

#include <stdint.h>

#include "fft_core.cuh"

namespace shhd {

struct Philox4 {
    uint32_t w0, w1, w2, w3;
};

__device__ __forceinline__ Philox4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += W0; k1 += W1; }
        const uint32_t hi0 = __umulhi(M0, c0), lo0 = M0 * c0;
        const uint32_t hi1 = __umulhi(M1, c2), lo1 = M1 * c2;
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    Philox4 o;
    o.w0 = c0; o.w1 = c1; o.w2 = c2; o.w3 = c3;
    return o;
}

// Two complex normals per Philox call: draw a from words (w0, w1), draw b from
// (w2, w3); uniforms u = (w + 1/2) 2^-32, Box-Muller r = sqrt(-2 ln u1),
// theta = 2 pi u2.
template <typename T> struct BoxMuller;

template <> struct BoxMuller<double> {
    __device__ __forceinline__ static double2 apply(uint32_t w_r, uint32_t w_t) {
        const double u1 = (static_cast<double>(w_r) + 0.5) * 2.3283064365386963e-10;
        const double u2 = (static_cast<double>(w_t) + 0.5) * 2.3283064365386963e-10;
        const double rad = sqrt(-2.0 * log(u1));
        double s, c;
        sincospi(2.0 * u2, &s, &c);
        return make_double2(rad * c, rad * s);
    }
};

template <> struct BoxMuller<float> {
    // fast hardware log / sin / cos: absolute error ~1e-6, far below the FP32 path's tolerance
    __device__ __forceinline__ static float2 apply(uint32_t w_r, uint32_t w_t) {
        const float u1 = __uint2float_rn(w_r) * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
        const float u2 = __uint2float_rn(w_t) * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
        const float rad = sqrtf(-2.0f * __logf(u1));
        float s, c;
        __sincosf(6.28318530717958647692f * u2, &s, &c);
        return make_float2(rad * c, rad * s);
    }
};

// xi_a and (if srk3) xi_b of one noise component at one mode
template <typename T>
__device__ __forceinline__ void complex_normals(uint32_t seed, uint32_t member, uint64_t step, uint32_t stream, uint32_t mode_id, bool want_b,
                                                cplx<T>& xa, cplx<T>& xb) {
    const Philox4 r = philox4x32_10(mode_id, stream, static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32), seed, member);
    xa = BoxMuller<T>::apply(r.w0, r.w1);
    if (want_b) xb = BoxMuller<T>::apply(r.w2, r.w3);
}

// stream ids: psi_alpha -> alpha, momentum stress draws xi_1..xi_3 -> 4096 + m
__host__ __device__ constexpr uint32_t psi_stream(int alpha) { return static_cast<uint32_t>(alpha); }
__host__ __device__ constexpr uint32_t j_stream(int m) { return 4096u + static_cast<uint32_t>(m); }

}  // namespace shhd
