// Counter-based Gaussian noise for the stochastic fluxes.
//
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11) keyed by (seed, member) with counter
// (mode id, stream, step lo, step hi).  One call gives one complex standard
// normal: two 53-bit uniforms u = ((hi << 32 | lo) >> 11 + 0.5) * 2^-53 and
// the Box-Muller transform r = sqrt(-2 ln u1), theta = 2 pi u2.
//
// mode id = gx * Nay + (ky mod Nay), using |ky| on the kx = 0 line (the
// ky < 0 entry there is the conjugate of the ky > 0 draw, as the reference's
// psi_sto / j_sto write conjugate pairs, fcalculator.cc:531-562, 632-677).
// stream = (component << 1) | draw, draw 0 = a, 1 = b; component alpha for
// psi_alpha and 4096 + m for the momentum stress draws xi_1..xi_3.
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

template <typename T> struct BoxMuller;

template <> struct BoxMuller<double> {
    __device__ __forceinline__ static double2 apply(const Philox4& r) {
        const uint64_t a = ((static_cast<uint64_t>(r.w1) << 32) | r.w0) >> 11;
        const uint64_t b = ((static_cast<uint64_t>(r.w3) << 32) | r.w2) >> 11;
        const double u1 = (static_cast<double>(a) + 0.5) * (1.0 / 9007199254740992.0);
        const double u2 = (static_cast<double>(b) + 0.5) * (1.0 / 9007199254740992.0);
        const double rad = sqrt(-2.0 * log(u1));
        double s, c;
        sincospi(2.0 * u2, &s, &c);
        return make_double2(rad * c, rad * s);
    }
};

template <> struct BoxMuller<float> {
    __device__ __forceinline__ static float2 apply(const Philox4& r) {
        // the FP64 path's 53-bit uniforms to FP32 accuracy: their top 32 bits
        // are w1 and w3; fast hardware log / sin / cos (absolute error ~1e-6,
        // far below the FP32 path's tolerance) keep the draw cheap
        const float u1 = __uint2float_rn(r.w1) * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
        const float u2 = __uint2float_rn(r.w3) * 2.3283064365386963e-10f + 1.1641532182693481e-10f;
        const float rad = sqrtf(-2.0f * __logf(u1));
        float s, c;
        __sincosf(6.28318530717958647692f * u2, &s, &c);
        return make_float2(rad * c, rad * s);
    }
};

template <typename T>
__device__ __forceinline__ cplx<T> complex_normal(uint32_t seed, uint32_t member, uint64_t step, uint32_t stream, uint32_t mode_id) {
    const Philox4 r = philox4x32_10(mode_id, stream, static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32), seed, member);
    return BoxMuller<T>::apply(r);
}

__host__ __device__ constexpr uint32_t psi_stream(int alpha, int draw) { return (static_cast<uint32_t>(alpha) << 1) | static_cast<uint32_t>(draw); }
__host__ __device__ constexpr uint32_t j_stream(int m, int draw) { return ((4096u + static_cast<uint32_t>(m)) << 1) | static_cast<uint32_t>(draw); }

}  // namespace shhd
