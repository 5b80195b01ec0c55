// The three fused kernels of one right-hand-side stage.
//
// Notation: Na = active grid, Np = compute (padded) grid, Hx = Na_x/2 active
// kx columns, Ky = Na_y - 1 active ky values.  Memory (per member):
//   state  [field][gx < Hx][j < Ky]          complex, j = ky (ky >= 0) or ky + Ky
//   I1/I2  [slot][tile][y < Np_y][w < W]     complex, gx = tile*W + w
// I1 holds the y-inverse of the transformed state fields ("x-spectral,
// y-physical"), I2 the x-forward of the product fields.  Tiles make the
// column passes read and write whole contiguous blocks.
//
//   col_inverse   state -> I1          (first stage of a step call only)
//   row_pass      I1 -> C2R -> products (j v, psi v, mu, v) -> R2C -> I2
//   col_forward   I2 -> y-forward -> RHS epilogue -> stage update -> state
//                 [-> y-inverse of the new state -> I1 for the next stage]
//
// The 3/2 padding is never stored: column loads zero-fill |ky| >= Na/2 and
// row loads zero-fill kx >= Na/2; the forward transforms keep only the active
// modes.  References to the solver this replaces are given per term.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_core.cuh"
#include "free_energy_plugins.h"
#include "philox.cuh"

namespace shhd {

constexpr int kThreads = 256;
constexpr int kMaxOp = 8;
constexpr int kMaxFields = kMaxOp + 3;
constexpr int kMaxIn = kMaxOp + 3;
constexpr int kMaxOut = 4 * kMaxOp + 5;
constexpr int kMaxGroupOut = 8;
constexpr int kMaxGroups = kMaxOp + 2;
constexpr int kMaxSine = 8;

enum OutKind : int { OUT_MU = 0, OUT_PSIVX, OUT_PSIVY, OUT_GRAD, OUT_VX, OUT_VY, OUT_PXX, OUT_PXY, OUT_PYY };
// GROUP_RHO: the density alone (its RHS -i k.j needs no products), split from the momentum
// group in the pair-line column kernel so that the heavy momentum blocks lose a field
enum GroupKind : int { GROUP_PSI = 0, GROUP_MOMENTUM = 1, GROUP_RHO = 2 };
enum ErrBits : int { ERR_ZERO_DENSITY = 1, ERR_NONFINITE = 2 };

// A diverging integration leaves NaN or Inf in the state: the state writes test each new
// value and one lane per warp raises ERR_NONFINITE (all 32 lanes must call this)
template <typename V>
__device__ __forceinline__ bool nonfinite2(V v) { return !isfinite(v.x + v.y); }
__device__ __forceinline__ void report_nonfinite(int* err, bool bad) {
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, ERR_NONFINITE);
}

struct SineSrc {
    int field;     // state field index
    int gx, ky;    // active mode receiving the source
    double re, im; // source value
};

struct StepPlan {
    // geometry
    int nax, nay, hx, kyn, npx, npy, W, ntiles;
    double kx_unit, ky_unit, inv_scale;
    int nfields, nop, mode, batch;
    // C2R inputs
    int n_in;
    int in_field[kMaxIn];
    int in_slot[kMaxFields];
    int need_v;
    // R2C outputs
    int n_out;
    int out_kind[kMaxOut];
    int out_arg[kMaxOut];
    // column-forward groups
    int n_groups;
    int group_kind[kMaxGroups];
    int group_alpha[kMaxGroups];
    int group_nout[kMaxGroups];
    int group_out[kMaxGroups][kMaxGroupOut];
    int group_order[kMaxGroups];   // pair-line column kernel: group of blockIdx.y (heaviest first)
    int rho_split;                 // the density is its own group (GROUP_RHO), not the momentum group's
    // physics
    double mobility[kMaxOp], mu_k0[kMaxOp], mu_k2[kMaxOp], mu_k4[kMaxOp], mu_u3[kMaxOp];
    int fe_plugin;                 // free-energy plugin style (0: none; its mu replaces u3 psi^3)
    double fe_param[SHHD_MAX_FE_PARAMS][kMaxOp];
    float fe_paramf[SHHD_MAX_FE_PARAMS][kMaxOp];
    int psi_zero[kMaxOp];          // psi_det early return (fcalculator.cc:93-95)
    int psi_linear[kMaxOp];        // linear mu term present (fcalculator.cc:158-160)
    double grad_ax[kMaxOp], grad_ay[kMaxOp];  // summed -A per direction (gradient forces)
    int grad_incomp[kMaxOp];
    double cT2, eta, zeta;
    int j_zero;                    // j_det early return (fcalculator.cc:131-133)
    int incomp_visc;               // add_incompressible_viscous_term with eta != 0
    int n_sine;
    SineSrc sine[kMaxSine];
    // noise
    int noise_psi[kMaxOp];
    double psi_sig2[kMaxOp];       // 0.5 * prefactor * M  (sigma^2 / k^2)
    int noise_j;
    double j_s, sqrt_eta, sqrt_zeta;
    uint32_t seed, member_offset;
    int external_noise;
    // transforms
    FftPlan fy, fx;
    FastDiv div_w, div_kyn, div_npy, div_hx;
    int kyp;                       // kyn rounded up to a multiple of 8: the pair-line column forward's per-mode row stride
    FastDiv div_kyp;
    int twx_count, twy_count;      // shared-memory twiddle entries for the row / column transforms
    int logw;                      // log2(W)
    int row_lb;                    // max lines per row transform call
    int row_nb;                    // work lines for outputs
    int npos;                      // position slots per thread in col_forward
    // pair-line row pass: outputs transformed two at a time, each product a
    // combination of the terms psi^3, psi vx, psi vy, vx, vy, jx vx, jx vy, jy vy
    // with per-output coefficients; inputs read from canonical (line, half) roles
    int rp_n;                      // output pairs
    int rp_a[kMaxOut], rp_b[kMaxOut];          // output indices (rp_b = -1: single)
    float rp_coef[kMaxOut][8][2];  // [pair][term][A, B]
    int rp_canon;                  // 1: roles below are valid (else the generic product path)
    int rp_prep;                   // 1: rewrite (rho, jx), (jy, -) into (jx, jy), (vx, vy)
    int rp_jline, rp_vline;        // line of (jx, jy) and of (vx, vy) (-1: v = j / rho0)
    int rp_pack;                   // one input slot and one output (psi -> u psi^3): a pair-line holds two row
                                   // pairs of that slot instead of two slots of one row pair
    int rp_mode[kMaxOut];          // 0 coefficient form; 1 (vx, vy); 2 (jx vx, jy vy);
                                   // 3 c0 psi^3, 4 c1 psi vx, 5 c2 psi vy with psi = (psi_a, psi_b) one line
};

// per-member controls of a batched engine (serving): noise key, step origin
// of the member's own step count, noise amplitude factor, active flag
struct MemberInfo {
    uint32_t key;
    int32_t active;
    int64_t step0;
    double noise_scale;
};

template <typename T>
struct StageArgs {
    const MemberInfo* members;
    const cplx<T>* cur;
    const cplx<T>* base;
    cplx<T>* next;
    const cplx<T>* i2;
    cplx<T>* i1_next;
    const cplx<T>* ext_a;
    const cplx<T>* ext_b;
    const double* rho0;            // per member
    // FP64 copies of the k = 0 mode of every field ([member][field]) for the
    // current, base and next state (FP32 engines; null otherwise)
    const double2* k0_cur;
    const double2* k0_base;
    double2* k0_next;
    int* err;
    double wb, wc, dt, sdt, beta;
    const unsigned long long* step_base;  // step index at the start of the call (device; graph replays advance it)
    int step_off;                  // step of this stage within the call
    int srk3;                      // draw b exists
    int fused_inverse;
    int det_mode;                  // write det instead of the stage update
};

__device__ __forceinline__ int ky_of_j(int j, int nay) { return j < nay / 2 ? j : j - (nay - 1); }

// ---------------------------------------------------------------------------
// column inverse: state -> I1   (grid: tiles x n_in x batch)
// ---------------------------------------------------------------------------
template <typename T, int FY>
__global__ void __launch_bounds__(kThreads) col_inverse_kernel(const StepPlan P, const MemberInfo* __restrict__ members,
                                                               const cplx<T>* __restrict__ state, cplx<T>* __restrict__ i1,
                                                               const cplx<T>* __restrict__ tw) {
    if (!members[blockIdx.z].active) return;
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* buf = s_tw + P.twy_count;
    C* scr = buf + P.W * P.npy;

    const int tile = blockIdx.x, slot = blockIdx.y, b = blockIdx.z;
    const int W = P.W, npy = P.npy, kyn = P.kyn, half = P.nay / 2;
    const uint32_t mask = P.fy.swz;
    const int field = P.in_field[slot];
    load_table(s_tw, tw, P.twy_count);

    const C* src = state + (static_cast<size_t>(b) * P.nfields + field) * P.hx * kyn + static_cast<size_t>(tile) * W * kyn;
    C* in = xform_input<FY>(buf, scr, P.fy);
    const int total = W * npy;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int w = fdiv(e, P.div_npy);
        const int y = e - w * npy;
        int j = -1;
        if (y < half) j = y;
        else if (y > npy - half) j = y - npy + kyn;
        in[sw(y, mask) * W + w] = (j >= 0) ? src[w * kyn + j] : czero<C>();
    }
    __syncthreads();
    xform<FY, +1, true>(buf, scr, P.fy, W, P.div_w, 1, W, P.logw, s_tw);
    const T sc = static_cast<T>(P.inv_scale);
    C* dst = i1 + ((static_cast<size_t>(b) * P.n_in + slot) * P.ntiles + tile) * static_cast<size_t>(npy) * W;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
        const int y = fdiv(e, P.div_w);
        const int w = e - y * W;
        dst[e] = cscale(buf[sw(y, mask) * W + w], sc);
    }
}

// a row pair's two elements of a transform plane (rows y0, y0 + 1: 32 bytes, 32-byte aligned when
// y0, the row count and the plane sizes are even) in one access: the row passes reach each plane
// row pair by row pair, 32 bytes per column tile, so that each 32-byte sector is touched once.
// Read once and written once per kernel, so not allocated in L1.
__device__ __forceinline__ void ld_stream2(const ulonglong2* p, ulonglong2& a, ulonglong2& b) {
    asm("ld.global.L1::no_allocate.v4.u64 {%0, %1, %2, %3}, [%4];" : "=l"(a.x), "=l"(a.y), "=l"(b.x), "=l"(b.y) : "l"(p));
}
__device__ __forceinline__ void st_stream2(ulonglong2* p, ulonglong2 a, ulonglong2 b) {
    asm volatile("st.global.L1::no_allocate.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(p), "l"(a.x), "l"(a.y), "l"(b.x), "l"(b.y) : "memory");
}
// complex value w of a 16-byte group (two FP32 complex, or one FP64), and its inverse
__device__ __forceinline__ float2 c16_get(const ulonglong2& v, int w, float2) {
    const unsigned long long q = w ? v.y : v.x;
    return make_float2(__int_as_float(static_cast<int>(q & 0xffffffffull)), __int_as_float(static_cast<int>(q >> 32)));
}
__device__ __forceinline__ double2 c16_get(const ulonglong2& v, int, double2) {
    return make_double2(__longlong_as_double(static_cast<long long>(v.x)), __longlong_as_double(static_cast<long long>(v.y)));
}
__device__ __forceinline__ void c16_set(ulonglong2& v, int w, float2 c) {
    const unsigned long long q = static_cast<unsigned long long>(static_cast<unsigned int>(__float_as_int(c.x))) |
                                 (static_cast<unsigned long long>(static_cast<unsigned int>(__float_as_int(c.y))) << 32);
    if (w) v.y = q;
    else v.x = q;
}
__device__ __forceinline__ void c16_set(ulonglong2& v, int, double2 c) {
    v.x = static_cast<unsigned long long>(__double_as_longlong(c.x));
    v.y = static_cast<unsigned long long>(__double_as_longlong(c.y));
}

// ---------------------------------------------------------------------------
// free-energy plugin styles (free_energy_plugins.h): the physical chemical potential and the
// free-energy density at one point, from the plan's style and parameters
// ---------------------------------------------------------------------------
template <typename T>
struct PluginParams {
    const StepPlan& P;
    __device__ __forceinline__ T operator()(int k, int b) const {
        if constexpr (sizeof(T) == sizeof(float)) return P.fe_paramf[k][b];
        else return P.fe_param[k][b];
    }
};
template <typename T>
__device__ __forceinline__ T plugin_mu(const StepPlan& P, int a, T psi_a, const T* psi) {
    const PluginParams<T> par{P};
    switch (P.fe_plugin) {
#define SHHD_MU(ID, S) \
    case ID: return S::template mu<T>(a, psi_a, psi, P.nop, par);
        SHHD_FREE_ENERGY_PLUGINS(SHHD_MU)
#undef SHHD_MU
        default: return T(0);
    }
}
template <typename T>
__device__ __forceinline__ T plugin_density(const StepPlan& P, const T* psi) {
    const PluginParams<T> par{P};
    switch (P.fe_plugin) {
#define SHHD_DENSITY(ID, S) \
    case ID: return S::template density<T>(psi, P.nop, par);
        SHHD_FREE_ENERGY_PLUGINS(SHHD_DENSITY)
#undef SHHD_DENSITY
        default: return T(0);
    }
}
// plugin mu_a of both rows of a row pair at one position: get(slot) returns the position's
// (row y0, row y0 + 1) values of an input slot; every order parameter is an input
template <typename T, typename Get>
__device__ __forceinline__ void plugin_mu_rows(const StepPlan& P, int a, Get&& get, T& mu0, T& mu1) {
    T p0[kMaxOp], p1[kMaxOp];
    T a0 = T(0), a1 = T(0);
#pragma unroll
    for (int b = 0; b < kMaxOp; ++b) {
        p0[b] = T(0);
        p1[b] = T(0);
        if (b < P.nop) {
            const auto v = get(P.in_slot[1 + b]);
            p0[b] = v.x;
            p1[b] = v.y;
            if (b == a) { a0 = v.x; a1 = v.y; }
        }
    }
    mu0 = plugin_mu<T>(P, a, a0, p0);
    mu1 = plugin_mu<T>(P, a, a1, p1);
}

// ---------------------------------------------------------------------------
// row pass: I1 -> C2R -> products -> R2C -> I2   (grid: row pairs x batch)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T product_value(const StepPlan& P, int kind, int arg, T psi, T jx, T jy, T vx, T vy) {
    switch (kind) {
        case OUT_MU: return static_cast<T>(P.mu_u3[arg]) * psi * psi * psi;   // model_free_energy_phi4.cc:47-55
        case OUT_PSIVX: return psi * vx;                                       // fcalculator.cc:226-239
        case OUT_PSIVY: return psi * vy;
        case OUT_GRAD: return static_cast<T>(P.grad_ax[arg]) * vx + static_cast<T>(P.grad_ay[arg]) * vy;  // fcalculator.cc:814-826
        case OUT_VX: return vx;                                                // fcalculator.cc:366-367
        case OUT_VY: return vy;
        case OUT_PXX: return jx * vx;                                          // fcalculator.cc:447-451
        case OUT_PXY: return jx * vy;
        default: return jy * vy;
    }
}

// row-pass inputs: rows y0, y0 + 1 of the P.n_in x-spectral planes of one member (i1_member),
// packed as Z[k] = X0[k] + i X1[k] with the Hermitian mirror, zero outside |kx| < Na/2, and
// inverse transformed in place into `lines` (P.row_lb lines at a time through `scr`); the
// physical rows come back as (row y0, row y0 + 1) in the real and imaginary parts
template <typename T, int FX>
__device__ __forceinline__ void row_inputs_inverse(const StepPlan& P, const cplx<T>* __restrict__ i1_member, int y0, bool has1,
                                                   cplx<T>* lines, cplx<T>* scr, const cplx<T>* s_tw) {
    using C = cplx<T>;
    const int npx = P.npx, npy = P.npy, W = P.W, hx = P.hx;
    const uint32_t mask = P.fx.swz;
    for (int s0 = 0; s0 < P.n_in; s0 += P.row_lb) {
        const int nl = min(P.row_lb, P.n_in - s0);
        C* in = xform_input<FX>(lines + static_cast<size_t>(s0) * npx, scr, P.fx);
        for (int l = 0; l < nl; ++l) {
            C* z = in + static_cast<size_t>(l) * npx;
            const C* src = i1_member + static_cast<size_t>(s0 + l) * P.ntiles * npy * W;
            for (int k = threadIdx.x; k < npx; k += blockDim.x) {
                if (k < hx) {
                    const int t = fdiv(k, P.div_w), w = k - t * W;
                    const C* p0 = src + (static_cast<size_t>(t) * npy + y0) * W + w;
                    C a = p0[0];
                    C c = has1 ? p0[W] : czero<C>();
                    if (k == 0) { a.y = 0; c.y = 0; }  // C2R uses the real part of the kx = 0 entry
                    z[sw(k, mask)] = mk(a.x - c.y, a.y + c.x);
                    if (k > 0) z[sw(npx - k, mask)] = mk(a.x + c.y, c.x - a.y);
                } else if (k <= npx - hx) {
                    z[sw(k, mask)] = czero<C>();
                }
            }
        }
        __syncthreads();
        xform<FX, +1, false>(lines + static_cast<size_t>(s0) * npx, scr, P.fx, nl, P.div_w, npx, 1, 0, s_tw);
    }
}

template <typename T, int FX>
__global__ void __launch_bounds__(kThreads) row_pass_kernel(const StepPlan P, const MemberInfo* __restrict__ members,
                                                            const cplx<T>* __restrict__ i1, cplx<T>* __restrict__ i2,
                                                            const cplx<T>* __restrict__ tw, const double* __restrict__ rho0_member,
                                                            int* __restrict__ err) {
    if (!members[blockIdx.y].active) return;
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    const int npx = P.npx, npy = P.npy, W = P.W, hx = P.hx;
    C* lines = s_tw + P.twx_count;                           // n_in physical row pairs
    C* work = lines + static_cast<size_t>(P.n_in) * npx;     // row_lb product lines
    C* scr = work + static_cast<size_t>(P.row_lb) * npx;     // row_lb ping-pong lines
    const uint32_t mask = P.fx.swz;

    const int pair = blockIdx.x, b = blockIdx.y;
    const int y0 = 2 * pair;
    const bool has1 = (y0 + 1) < npy;
    load_table(s_tw, tw, P.twx_count);
    __syncthreads();

    // 1. inputs: rows y0, y0 + 1 of every input, inverse transformed
    row_inputs_inverse<T, FX>(P, i1 + static_cast<size_t>(b) * P.n_in * P.ntiles * npy * W, y0, has1, lines, scr, s_tw);

    // 2. velocity: v = j / rho (compressible) or j / rho0 (fcalculator_workspace.cc:115-142),
    //    formed where a product needs it; the zero-density check runs once per row pair.
    //    Pointwise work runs over shared-memory slots: every line uses the same swizzle.
    const int s_rho = P.in_slot[0];
    const int s_jx = P.in_slot[P.nop + 1];
    const int s_jy = P.in_slot[P.nop + 2];
    const bool comp = (P.mode == 0);
    const T inv_rho0 = (P.need_v && !comp) ? static_cast<T>(1.0 / rho0_member[b]) : T(0);
    if (P.need_v && comp) {
        int bad = 0;
        for (int x = threadIdx.x; x < npx; x += blockDim.x) {
            const C rho = lines[static_cast<size_t>(s_rho) * npx + x];
            if (rho.x == T(0) || (has1 && rho.y == T(0))) bad = 1;
        }
        if (bad) atomicOr(err, ERR_ZERO_DENSITY);
    }

    // 3. products -> forward transforms -> keep kx < Hx
    const size_t i2_member = static_cast<size_t>(b) * P.n_out * P.ntiles * npy * W;
    for (int o0 = 0; o0 < P.n_out; o0 += P.row_lb) {
        const int nl = min(P.row_lb, P.n_out - o0);
        C* in = xform_input<FX>(work, scr, P.fx);
        for (int l = 0; l < nl; ++l) {
            const int kind = P.out_kind[o0 + l], arg = P.out_arg[o0 + l];
            C* dst = in + static_cast<size_t>(l) * npx;
            const int s_psi = (kind == OUT_MU || kind == OUT_PSIVX || kind == OUT_PSIVY) ? P.in_slot[1 + arg] : -1;
            const bool use_v = (kind != OUT_MU);
            for (int x = threadIdx.x; x < npx; x += blockDim.x) {
                const C psi = s_psi >= 0 ? lines[static_cast<size_t>(s_psi) * npx + x] : czero<C>();
                C jx = czero<C>(), jy = czero<C>(), vx = czero<C>(), vy = czero<C>();
                if (use_v) {
                    jx = lines[static_cast<size_t>(s_jx) * npx + x];
                    jy = lines[static_cast<size_t>(s_jy) * npx + x];
                    if (comp) {
                        const C rho = lines[static_cast<size_t>(s_rho) * npx + x];
                        vx = mk(jx.x / rho.x, jx.y / rho.y);
                        vy = mk(jy.x / rho.x, jy.y / rho.y);
                    } else {
                        vx = mk(jx.x * inv_rho0, jx.y * inv_rho0);
                        vy = mk(jy.x * inv_rho0, jy.y * inv_rho0);
                    }
                }
                C val = mk(product_value<T>(P, kind, arg, psi.x, jx.x, jy.x, vx.x, vy.x),
                           product_value<T>(P, kind, arg, psi.y, jx.y, jy.y, vx.y, vy.y));
                if (kind == OUT_MU && P.fe_plugin)
                    plugin_mu_rows<T>(P, arg, [&](int s) { return lines[static_cast<size_t>(s) * npx + x]; }, val.x, val.y);
                if (!has1) val.y = T(0);  // odd row count: the last pair holds one row
                dst[x] = val;
            }
        }
        __syncthreads();
        xform<FX, -1, false>(work, scr, P.fx, nl, P.div_w, npx, 1, 0, s_tw);
        for (int l = 0; l < nl; ++l) {
            const C* z = work + static_cast<size_t>(l) * npx;
            C* dst = i2 + i2_member + static_cast<size_t>(o0 + l) * P.ntiles * npy * W;
            for (int k = threadIdx.x; k < hx; k += blockDim.x) {
                const C zk = z[sw(k, mask)];
                const C zn = cconj(z[sw(k == 0 ? 0 : npx - k, mask)]);
                const C g0 = mk(static_cast<T>(0.5) * (zk.x + zn.x), static_cast<T>(0.5) * (zk.y + zn.y));
                const C d = csub(zk, zn);
                const C g1 = mk(static_cast<T>(0.5) * d.y, static_cast<T>(-0.5) * d.x);
                const int t = fdiv(k, P.div_w), w = k - t * W;
                C* q = dst + (static_cast<size_t>(t) * npy + y0) * W + w;
                q[0] = g0;
                if (has1) q[W] = g1;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// column forward + epilogue   (grid: tiles x groups x batch)
// ---------------------------------------------------------------------------
// psi_sto for both draws (fcalculator.cc:496-585): sigma * xi (conjugated on the kx = 0, ky < 0 half)
template <typename T>
__device__ __forceinline__ cplx<T> psi_noise(const StepPlan& P, int alpha, uint64_t step, uint32_t member, uint32_t mode_id, bool conj_line,
                                             T sigma, bool srk3, T beta) {
    // sigma already carries the member's amplitude factor
    cplx<T> xa, xb;
    complex_normals<T>(P.seed, member, step, psi_stream(alpha), mode_id, srk3, xa, xb);
    cplx<T> x = srk3 ? cadd(xa, cscale(xb, beta)) : xa;
    if (conj_line) x = cconj(x);
    return cscale(x, sigma);
}

// j_sto for both draws (fcalculator.cc:587-700): out = -i k . pi(xi_a + beta xi_b)
template <typename T>
__device__ __forceinline__ void j_noise(const StepPlan& P, uint64_t step, uint32_t member, uint32_t mode_id, bool conj_line, T kx, T ky,
                                        bool srk3, T beta, T jscale, cplx<T>& ox, cplx<T>& oy) {
    using C = cplx<T>;
    C x[3];
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        C xa, xb;
        complex_normals<T>(P.seed, member, step, j_stream(m), mode_id, srk3, xa, xb);
        x[m] = srk3 ? cadd(xa, cscale(xb, beta)) : xa;
        if (conj_line) x[m] = cconj(x[m]);
    }
    const T s = static_cast<T>(P.j_s) * jscale, se = static_cast<T>(P.sqrt_eta), sz = static_cast<T>(P.sqrt_zeta);
    const C pxx = mk(-s * (sz * x[0].x + se * x[1].x), -s * (sz * x[0].y + se * x[1].y));
    const C pyy = mk(-s * (sz * x[0].x - se * x[1].x), -s * (sz * x[0].y - se * x[1].y));
    const C pxy = mk(-s * se * x[2].x, -s * se * x[2].y);
    ox = cmulmi(cadd(cscale(pxx, kx), cscale(pxy, ky)));
    oy = cmulmi(cadd(cscale(pxy, kx), cscale(pyy, ky)));
}

// ---------------------------------------------------------------------------
// epilogue math shared by the column-forward kernels: one active mode at a time
// ---------------------------------------------------------------------------
struct ModeCtx {
    int gx, ky;            // integer wave numbers
    size_t pos;            // index of (field 0, gx, j) in the state arrays
    uint32_t mode_id;      // Philox counter word
    bool conj_line;        // kx = 0, ky < 0: conjugate of the |ky| draw
    bool k_nonzero;
};

template <typename T>
__device__ __forceinline__ ModeCtx mode_ctx(const StepPlan& P, size_t mbase, int tile, int w, int j) {
    ModeCtx m;
    m.ky = ky_of_j(j, P.nay);
    m.gx = tile * P.W + w;
    m.pos = mbase + static_cast<size_t>(w) * P.kyn + j;
    m.conj_line = (m.gx == 0 && m.ky < 0);
    const int aky = m.conj_line ? -m.ky : m.ky;
    m.mode_id = static_cast<uint32_t>(m.gx) * static_cast<uint32_t>(P.nay) + static_cast<uint32_t>((aky % P.nay + P.nay) % P.nay);
    m.k_nonzero = !(m.gx == 0 && m.ky == 0);
    return m;
}

// accumulate one transformed product field into the group's RHS (coefficients
// of the reference's spectral divergences, fcalculator.cc:244-272, 374-396, 475-492)
template <typename T>
__device__ __forceinline__ void accumulate_product(const StepPlan& P, int kind, int alpha, T kx, T kyv, cplx<T> v, cplx<T>& a0, cplx<T>& a1) {
    switch (kind) {
        case OUT_MU: {
            const T m = static_cast<T>(P.mobility[alpha]);
            a0 = cadd(a0, cscale(v, -m * (kx * kx + kyv * kyv)));
            break;
        }
        case OUT_PSIVX: a0 = cadd(a0, cmulmi(cscale(v, kx))); break;
        case OUT_PSIVY: a0 = cadd(a0, cmulmi(cscale(v, kyv))); break;
        case OUT_GRAD: a0 = cadd(a0, v); break;
        case OUT_VX: {
            const T eta = static_cast<T>(P.eta), zeta = static_cast<T>(P.zeta);
            a0 = cadd(a0, cscale(v, -((eta + zeta) * kx * kx + eta * kyv * kyv)));
            a1 = cadd(a1, cscale(v, -(zeta * kx * kyv)));
            break;
        }
        case OUT_VY: {
            const T eta = static_cast<T>(P.eta), zeta = static_cast<T>(P.zeta);
            a0 = cadd(a0, cscale(v, -(zeta * kx * kyv)));
            a1 = cadd(a1, cscale(v, -(eta * kx * kx + (eta + zeta) * kyv * kyv)));
            break;
        }
        case OUT_PXX: a0 = cadd(a0, cmulmi(cscale(v, kx))); break;
        case OUT_PXY:
            a0 = cadd(a0, cmulmi(cscale(v, kyv)));
            a1 = cadd(a1, cmulmi(cscale(v, kx)));
            break;
        default: a1 = cadd(a1, cmulmi(cscale(v, kyv))); break;
    }
}

// global inputs of one mode's epilogue, loaded ahead of the math so the next
// mode's loads can be in flight while the current one is computed
template <typename T>
struct PsiLoads {
    cplx<T> cur, base, ea, eb, jx, jy;
};

template <typename T>
__device__ __forceinline__ PsiLoads<T> psi_loads(const StepPlan& P, const StageArgs<T>& A, int alpha, size_t pos, size_t fstride) {
    using C = cplx<T>;
    const int f = 1 + alpha;
    PsiLoads<T> L;
    L.cur = A.cur[pos + f * fstride];
    L.base = (A.wb != 0.0 && !A.det_mode) ? A.base[pos + f * fstride] : czero<C>();
    L.ea = (P.external_noise && !A.det_mode) ? A.ext_a[pos + f * fstride] : czero<C>();
    L.eb = (P.external_noise && A.srk3 && !A.det_mode) ? A.ext_b[pos + f * fstride] : czero<C>();
    if (P.grad_incomp[alpha] && !P.psi_zero[alpha]) {
        L.jx = A.cur[pos + (P.nop + 1) * fstride];
        L.jy = A.cur[pos + (P.nop + 2) * fstride];
    } else {
        L.jx = czero<C>();
        L.jy = czero<C>();
    }
    return L;
}

// Stage update of the k = 0 mode in FP64 from the FP64 copies (FP32 engines):
// the RHS there is zero unless a force acts on it, so the FP32 update would only
// add rounding to the conserved mass, momentum and order-parameter means.  The
// mode is self-conjugate, so its imaginary part is zero (time_integrator.h:70-109).
template <typename T>
__device__ __forceinline__ cplx<T> k0_update(const StepPlan& P, const StageArgs<T>& A, int b, int f, cplx<T> det, cplx<T> sto) {
    const int i = b * P.nfields + f;
    const double cur = A.k0_cur[i].x;
    const double base = A.wb != 0.0 ? A.k0_base[i].x : 0.0;
    const double v = A.wb * base + A.wc * (cur + A.dt * static_cast<double>(det.x) + A.sdt * static_cast<double>(sto.x));
    A.k0_next[i] = make_double2(v, 0.0);
    return mk(static_cast<T>(v), T(0));
}

// psi_alpha: det from the accumulated products plus the spectral terms, then
// (unless det_mode) the stage update with noise; returns next (or det)
template <typename T>
__device__ __forceinline__ cplx<T> psi_epilogue(const StepPlan& P, const StageArgs<T>& A, int alpha, const ModeCtx& m, T kx, T kyv,
                                                cplx<T> acc, const MemberInfo& mi, const PsiLoads<T>& L, int b) {
    using C = cplx<T>;
    const int f = 1 + alpha;
    const T k2 = kx * kx + kyv * kyv;
    const C cur = L.cur;
    C det = czero<C>();
    if (!P.psi_zero[alpha]) {
        det = acc;
        if (P.psi_linear[alpha]) {  // fcalculator.cc:152-187
            const T mob = static_cast<T>(P.mobility[alpha]);
            const T mu = static_cast<T>(P.mu_k0[alpha]) + static_cast<T>(P.mu_k2[alpha]) * k2 + static_cast<T>(P.mu_k4[alpha]) * k2 * k2;
            det = cadd(det, cscale(cur, -mob * k2 * mu));
        }
        for (int s = 0; s < P.n_sine; ++s)
            if (P.sine[s].field == f && P.sine[s].gx == m.gx && P.sine[s].ky == m.ky)
                det = cadd(det, mk(static_cast<T>(P.sine[s].re), static_cast<T>(P.sine[s].im)));
        if (P.grad_incomp[alpha]) {  // fcalculator.cc:790-806
            const T r0 = static_cast<T>(1.0 / A.rho0[b]);
            det = cadd(det, cadd(cscale(L.jx, static_cast<T>(P.grad_ax[alpha]) * r0), cscale(L.jy, static_cast<T>(P.grad_ay[alpha]) * r0)));
        }
    }
    if (A.det_mode) return det;
    const T beta = static_cast<T>(A.beta);
    C sto = czero<C>();
    if (P.external_noise) {
        sto = L.ea;
        if (A.srk3) sto = cadd(sto, cscale(L.eb, beta));
    } else if (P.noise_psi[alpha] && m.k_nonzero) {
        const T sigma = sqrt(static_cast<T>(P.psi_sig2[alpha]) * k2) * static_cast<T>(mi.noise_scale);
        const uint64_t step = *A.step_base + static_cast<uint64_t>(A.step_off);
        sto = psi_noise<T>(P, alpha, step - static_cast<uint64_t>(mi.step0), mi.key, m.mode_id, m.conj_line, sigma, A.srk3 != 0, beta);
    }
    if (A.k0_cur && !m.k_nonzero) return k0_update<T>(P, A, b, f, det, sto);
    const C inner = cadd(cadd(cur, cscale(det, static_cast<T>(A.dt))), cscale(sto, static_cast<T>(A.sdt)));
    return cadd(cscale(L.base, static_cast<T>(A.wb)), cscale(inner, static_cast<T>(A.wc)));
}

template <typename T>
struct MomLoads {
    cplx<T> cjx, cjy, crho, bjx, bjy, eax, eay, ebx, eby;
};

template <typename T>
__device__ __forceinline__ MomLoads<T> momentum_loads(const StepPlan& P, const StageArgs<T>& A, size_t pos, size_t fstride) {
    using C = cplx<T>;
    const int f_jx = P.nop + 1, f_jy = P.nop + 2;
    const bool upd = !A.det_mode;
    MomLoads<T> L;
    L.cjx = A.cur[pos + f_jx * fstride];
    L.cjy = A.cur[pos + f_jy * fstride];
    L.crho = (P.cT2 != 0.0 && !P.j_zero) ? A.cur[pos] : czero<C>();
    const bool wb = upd && A.wb != 0.0;
    L.bjx = wb ? A.base[pos + f_jx * fstride] : czero<C>();
    L.bjy = wb ? A.base[pos + f_jy * fstride] : czero<C>();
    const bool ext = upd && P.external_noise;
    L.eax = ext ? A.ext_a[pos + f_jx * fstride] : czero<C>();
    L.eay = ext ? A.ext_a[pos + f_jy * fstride] : czero<C>();
    L.ebx = (ext && A.srk3) ? A.ext_b[pos + f_jx * fstride] : czero<C>();
    L.eby = (ext && A.srk3) ? A.ext_b[pos + f_jy * fstride] : czero<C>();
    return L;
}

// momentum: det_j from the accumulated products plus pressure, incompressible
// viscosity and sine forces; stage update with noise and (incompressible)
// transverse projection.  Results replace a0 (jx) and a1 (jy).
template <typename T>
__device__ __forceinline__ void momentum_epilogue(const StepPlan& P, const StageArgs<T>& A, const ModeCtx& m, T kx, T kyv, cplx<T>& a0,
                                                  cplx<T>& a1, const MemberInfo& mi, const MomLoads<T>& L, int b) {
    using C = cplx<T>;
    const int f_jx = P.nop + 1, f_jy = P.nop + 2;
    const T k2 = kx * kx + kyv * kyv;
    const C cjx = L.cjx, cjy = L.cjy;
    C djx = czero<C>(), djy = czero<C>();
    if (!P.j_zero) {
        djx = a0;
        djy = a1;
        if (P.cT2 != 0.0) {  // fcalculator.cc:276-300
            const C ph = cscale(L.crho, static_cast<T>(P.cT2));
            djx = cadd(djx, cmulmi(cscale(ph, kx)));
            djy = cadd(djy, cmulmi(cscale(ph, kyv)));
        }
        if (P.incomp_visc) {  // fcalculator.cc:302-341
            const T r0 = static_cast<T>(1.0 / A.rho0[b]);
            const T eta = static_cast<T>(P.eta);
            const C vx = cscale(cjx, r0), vy = cscale(cjy, r0);
            djx = csub(djx, cscale(cadd(cscale(vx, 2 * kx * kx + kyv * kyv), cscale(vy, kx * kyv)), eta));
            djy = csub(djy, cscale(cadd(cscale(vx, kx * kyv), cscale(vy, kx * kx + 2 * kyv * kyv)), eta));
        }
        for (int s = 0; s < P.n_sine; ++s)
            if (P.sine[s].gx == m.gx && P.sine[s].ky == m.ky) {
                const C src = mk(static_cast<T>(P.sine[s].re), static_cast<T>(P.sine[s].im));
                if (P.sine[s].field == f_jx) djx = cadd(djx, src);
                else if (P.sine[s].field == f_jy) djy = cadd(djy, src);
            }
    }
    if (A.det_mode) { a0 = djx; a1 = djy; return; }
    const T beta = static_cast<T>(A.beta);
    C sx = czero<C>(), sy = czero<C>();
    if (P.external_noise) {
        sx = L.eax;
        sy = L.eay;
        if (A.srk3) {
            sx = cadd(sx, cscale(L.ebx, beta));
            sy = cadd(sy, cscale(L.eby, beta));
        }
    } else if (P.noise_j && m.k_nonzero) {
        const uint64_t step = *A.step_base + static_cast<uint64_t>(A.step_off);
        j_noise<T>(P, step - static_cast<uint64_t>(mi.step0), mi.key, m.mode_id, m.conj_line, kx, kyv, A.srk3 != 0, beta,
                   static_cast<T>(mi.noise_scale), sx, sy);
    }
    const T dt = static_cast<T>(A.dt), sdt = static_cast<T>(A.sdt), wb = static_cast<T>(A.wb), wc = static_cast<T>(A.wc);
    C incx = cadd(cscale(djx, dt), cscale(sx, sdt));
    C incy = cadd(cscale(djy, dt), cscale(sy, sdt));
    if (P.mode == 1 && k2 != T(0)) {  // transverse projection (srk3_incompressible.h:81-96)
        const C tr = cadd(cscale(incx, -kyv), cscale(incy, kx));
        incx = cscale(cscale(tr, -kyv), T(1) / k2);
        incy = cscale(cscale(tr, kx), T(1) / k2);
    }
    if (A.k0_cur && !m.k_nonzero) {
        a0 = k0_update<T>(P, A, b, f_jx, djx, sx);
        a1 = k0_update<T>(P, A, b, f_jy, djy, sy);
        return;
    }
    a0 = cadd(cscale(L.bjx, wb), cscale(cadd(cjx, incx), wc));
    a1 = cadd(cscale(L.bjy, wb), cscale(cadd(cjy, incy), wc));
}

// rho: rho_det (fcalculator.cc:60-84) and its stage update
template <typename T>
__device__ __forceinline__ cplx<T> rho_epilogue(const StepPlan& P, const StageArgs<T>& A, size_t pos, T kx, T kyv, size_t fstride) {
    using C = cplx<T>;
    const C drho = cmulmi(cadd(cscale(A.cur[pos + (P.nop + 1) * fstride], kx), cscale(A.cur[pos + (P.nop + 2) * fstride], kyv)));
    if (A.det_mode) return drho;
    if (A.k0_cur && kx == T(0) && kyv == T(0))
        return k0_update<T>(P, A, static_cast<int>(pos / (static_cast<size_t>(P.nfields) * fstride)), 0, drho, czero<C>());
    const C base = (A.wb != 0.0) ? A.base[pos] : czero<C>();
    return cadd(cscale(base, static_cast<T>(A.wb)), cscale(cadd(A.cur[pos], cscale(drho, static_cast<T>(A.dt))), static_cast<T>(A.wc)));
}

template <typename T, int NPOS, int FY>
__global__ void __launch_bounds__(kThreads) col_forward_kernel(const StepPlan P, const StageArgs<T> A, const cplx<T>* __restrict__ tw) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    C* buf = s_tw + P.twy_count;
    C* scr = buf + P.W * P.npy;
    const uint32_t mask = P.fy.swz;

    const int tile = blockIdx.x, grp = blockIdx.y, b = blockIdx.z;
    const int W = P.W, npy = P.npy, kyn = P.kyn, nay = P.nay;
    const int gkind = P.group_kind[grp];
    const int alpha = P.group_alpha[grp];
    const int nop = P.nop;
    const bool comp = (P.mode == 0);
    const MemberInfo mi = A.members[b];
    if (!mi.active) return;
    load_table(s_tw, tw, P.twy_count);

    const int npos_total = W * kyn;
    const size_t fstride = static_cast<size_t>(P.hx) * kyn;
    const size_t mbase = static_cast<size_t>(b) * P.nfields * fstride + static_cast<size_t>(tile) * W * kyn;

    // accumulators: psi group -> acc0 = psi_alpha; momentum group -> acc0 = jx, acc1 = jy
    C acc0[NPOS], acc1[NPOS];
#pragma unroll
    for (int i = 0; i < NPOS; ++i) { acc0[i] = czero<C>(); acc1[i] = czero<C>(); }

    const T kxu = static_cast<T>(P.kx_unit), kyu = static_cast<T>(P.ky_unit);
    const int ngo = P.group_nout[grp];
    for (int go = 0; go < ngo; ++go) {
        const int o = P.group_out[grp][go];
        const C* src = A.i2 + ((static_cast<size_t>(b) * P.n_out + o) * P.ntiles + tile) * static_cast<size_t>(npy) * W;
        const int total = W * npy;
        C* in = xform_input<FY>(buf, scr, P.fy);
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int y = fdiv(e, P.div_w);
            const int w = e - y * W;
            in[sw(y, mask) * W + w] = src[e];
        }
        __syncthreads();
        xform<FY, -1, true>(buf, scr, P.fy, W, P.div_w, 1, W, P.logw, s_tw);
        const int kind = P.out_kind[o];
#pragma unroll
        for (int i = 0; i < NPOS; ++i) {
            const int p = threadIdx.x + i * kThreads;
            if (p < npos_total) {
                const int w = fdiv(p, P.div_kyn);
                const int j = p - w * kyn;
                const int ky = ky_of_j(j, nay);
                const int y = ky >= 0 ? ky : ky + npy;
                const C v = buf[sw(y, mask) * W + w];
                const T kx = kxu * static_cast<T>(tile * W + w);
                const T kyv = kyu * static_cast<T>(ky);
                accumulate_product<T>(P, kind, alpha, kx, kyv, v, acc0[i], acc1[i]);
            }
        }
        __syncthreads();
    }

    // ---- epilogue: spectral terms, noise, stage update; results replace acc0/acc1 ----
    const int f_jx = nop + 1, f_jy = nop + 2;
#pragma unroll
    for (int i = 0; i < NPOS; ++i) {
        const int p = threadIdx.x + i * kThreads;
        if (p >= npos_total) continue;
        const int w = fdiv(p, P.div_kyn);
        const int j = p - w * kyn;
        const ModeCtx m = mode_ctx<T>(P, mbase, tile, w, j);
        const T kx = kxu * static_cast<T>(m.gx);
        const T kyv = kyu * static_cast<T>(m.ky);
        if (gkind == GROUP_PSI) acc0[i] = psi_epilogue<T>(P, A, alpha, m, kx, kyv, acc0[i], mi, psi_loads<T>(P, A, alpha, m.pos, fstride), b);
        else momentum_epilogue<T>(P, A, m, kx, kyv, acc0[i], acc1[i], mi, momentum_loads<T>(P, A, m.pos, fstride), b);
    }

    // ---- which fields this CTA writes, in order: psi | (rho), jx, jy ----
    int nwf = 0;
    int wfield[3];
    if (gkind == GROUP_PSI) { wfield[nwf++] = 1 + alpha; }
    else { if (comp) wfield[nwf++] = 0; wfield[nwf++] = f_jx; wfield[nwf++] = f_jy; }

    C* stage_buf = xform_input<FY>(buf, scr, P.fy);  // new values, zero-padded, ready for the y-inverse
    for (int q = 0; q < nwf; ++q) {
        const int f = wfield[q];
        const int total = W * npy;
        for (int e = threadIdx.x; e < total; e += blockDim.x) stage_buf[e] = czero<C>();
        __syncthreads();
#pragma unroll
        for (int i = 0; i < NPOS; ++i) {
            const int p = threadIdx.x + i * kThreads;
            if (p < npos_total) {
                const int w = fdiv(p, P.div_kyn);
                const int j = p - w * kyn;
                const int ky = ky_of_j(j, nay);
                const int y = ky >= 0 ? ky : ky + npy;
                C v;
                if (f == 0) {
                    const size_t pos = mbase + static_cast<size_t>(w) * kyn + j;
                    v = rho_epilogue<T>(P, A, pos, kxu * static_cast<T>(tile * W + w), kyu * static_cast<T>(ky), fstride);
                } else {
                    v = (f == f_jy) ? acc1[i] : acc0[i];
                }
                stage_buf[sw(y, mask) * W + w] = v;
            }
        }
        __syncthreads();
        // real-symmetry projection of the kx = 0 line (time_integrator.h:70-109)
        if (tile == 0 && !A.det_mode) {
            for (int ky = threadIdx.x; ky < nay / 2; ky += blockDim.x) {
                if (ky == 0) {
                    stage_buf[0].y = T(0);
                } else {
                    C* pa = stage_buf + sw(ky, mask) * W;
                    C* pc = stage_buf + sw(npy - ky, mask) * W;
                    const C a = *pa, c = *pc;
                    const C pj = mk(static_cast<T>(0.5) * (a.x + c.x), static_cast<T>(0.5) * (a.y - c.y));
                    *pa = pj;
                    *pc = cconj(pj);
                }
            }
            __syncthreads();
        }
        // write the state
        C* dst = A.next + mbase + f * fstride;
        bool bad = false;
        for (int p = threadIdx.x; p < npos_total; p += blockDim.x) {
            const int w = fdiv(p, P.div_kyn);
            const int j = p - w * kyn;
            const int ky = ky_of_j(j, nay);
            const int y = ky >= 0 ? ky : ky + npy;
            const C v = stage_buf[sw(y, mask) * W + w];
            bad |= nonfinite2(v);
            dst[static_cast<size_t>(w) * kyn + j] = v;
        }
        report_nonfinite(A.err, bad);
        // y-inverse of the new field for the next stage (scaled by 1/(Nx Ny) on the way out)
        const int slot = P.in_slot[f];
        if (A.fused_inverse && slot >= 0) {
            __syncthreads();
            xform<FY, +1, true>(buf, scr, P.fy, W, P.div_w, 1, W, P.logw, s_tw);
            const T sc = static_cast<T>(P.inv_scale);
            C* o1 = A.i1_next + ((static_cast<size_t>(b) * P.n_in + slot) * P.ntiles + tile) * static_cast<size_t>(npy) * W;
            for (int e = threadIdx.x; e < total; e += blockDim.x) {
                const int y = fdiv(e, P.div_w);
                const int w = e - y * W;
                o1[e] = cscale(buf[sw(y, mask) * W + w], sc);
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// structure factor S(k) = V <|u_k|^2> / Np^4 of one field, mean over the
// active members, added in FP64 to acc[mode] (engine mode order); grid:
// ceil(Hx * Ky / 256).  `scale` = V / Np^4 / (active members).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) structure_factor_kernel(const StepPlan P, const MemberInfo* __restrict__ members,
                                                                    const cplx<T>* __restrict__ state, int field, double scale,
                                                                    double* __restrict__ acc) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    if (e >= static_cast<int>(fstride)) return;
    double s = 0.0;
    for (int b = 0; b < P.batch; ++b) {
        if (!members[b].active) continue;
        const cplx<T> v = state[(static_cast<size_t>(b) * P.nfields + field) * fstride + e];
        s += static_cast<double>(v.x) * static_cast<double>(v.x) + static_cast<double>(v.y) * static_cast<double>(v.y);
    }
    acc[e] += s * scale;
}

// ---------------------------------------------------------------------------
// Yokota-Green-Kubo tap (measure_yokota_green_kubo.cc:128-190): the momentum
// flux pi_xy of each RHS evaluation at the selected modes, weighted by the
// stage's flux weight into the step flux; after the last stage the first
// draw's stochastic flux / sqrt(dt) is added and the block integral and its
// normalised square are accumulated, all in FP64.  One block per (mode, member):
// the y-transforms of the x-transformed product planes at the mode are direct
// DFTs over the column (table w^n = e^{-2 pi i n / Np_y}), every plane in one
// pass, each thread a strided set of rows, then a fixed-order block sum.
// ---------------------------------------------------------------------------
struct GkArgs {
    const int2* modes;          // (gx, ky) per selected mode
    int nmodes, ntau, nevery, nblock;
    double2* flux_step;         // [member][mode]
    double2* integral;          // [member][mode]
    double* sums;               // [member][tau][mode]
    const double2* wtab;        // [Np_y]
    int o_pxy, o_vx, o_vy;      // product planes in I2 (-1: absent)
    int pair_layout;            // I2 element (re_2t, re_2t+1, im_2t, im_2t+1) with W = 2
    int incomp_visc;            // pi_xy from j / rho0 of the stage state
    double kbt, area, cell_area;
};

// forward y-transform at ky of column gx of one I2 plane (x-transformed, y-physical): the plane's 2-D
// coefficient at (gx, ky); one warp, FP64 sums; wtab[n] = exp(-2 pi i n / npy)
template <typename T>
__device__ __forceinline__ double2 column_dft(const StepPlan& P, const double2* __restrict__ wtab, int pair_layout, const T* plane, int gx,
                                              int ky) {
    const int npy = P.npy;
    const int t = gx / P.W, w = gx - t * P.W;
    const int kk = ((ky % npy) + npy) % npy;
    // twiddle index kk * y mod npy, stepped by kk * 32 mod npy from lane to lane's next row
    const int lane = threadIdx.x & 31;
    int idx = static_cast<int>((static_cast<long long>(kk) * lane) % npy);
    const int stride = static_cast<int>((static_cast<long long>(kk) * 32) % npy);
    double re = 0.0, im = 0.0;
    for (int y = lane; y < npy; y += 32) {
        T xr, xi;
        if (pair_layout) {
            const T* e = plane + 4 * (static_cast<size_t>(t) * npy + y);
            xr = e[w];
            xi = e[2 + w];
        } else {
            const T* e = plane + 2 * ((static_cast<size_t>(t) * npy + y) * P.W + w);
            xr = e[0];
            xi = e[1];
        }
        const double2 tw = wtab[idx];
        idx += stride;
        if (idx >= npy) idx -= npy;
        re += static_cast<double>(xr) * tw.x - static_cast<double>(xi) * tw.y;
        im += static_cast<double>(xr) * tw.y + static_cast<double>(xi) * tw.x;
    }
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
    }
    return make_double2(re, im);
}

// one row's term of a column DFT: element y of column (t, w) of an I2 plane times the twiddle
template <typename T>
__device__ __forceinline__ void gk_dft_term(const T* plane, int pair_layout, int W, int npy, int t, int w, int y, double2 tw, double& re,
                                            double& im) {
    T xr, xi;
    if (pair_layout) {
        const T* e = plane + 4 * (static_cast<size_t>(t) * npy + y);
        xr = e[w];
        xi = e[2 + w];
    } else {
        const T* e = plane + 2 * ((static_cast<size_t>(t) * npy + y) * W + w);
        xr = e[0];
        xi = e[1];
    }
    re += static_cast<double>(xr) * tw.x - static_cast<double>(xi) * tw.y;
    im += static_cast<double>(xr) * tw.y + static_cast<double>(xi) * tw.x;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) gk_tap_kernel(const StepPlan P, const GkArgs G, const MemberInfo* __restrict__ members,
                                                          const T* __restrict__ i2, const cplx<T>* __restrict__ cur, const double* __restrict__ rho0,
                                                          const unsigned long long* __restrict__ step_base, int step_off, double weight,
                                                          int first_stage, int last_stage, double dt) {
    const int i = blockIdx.x, b = blockIdx.y;
    const MemberInfo mi = members[b];
    if (!mi.active) return;  // the whole block
    const int gx = G.modes[i].x, ky = G.modes[i].y;
    const double kx = P.kx_unit * gx, kyv = P.ky_unit * ky;
    const size_t plane = static_cast<size_t>(P.hx) * P.npy * 2;  // scalars of one I2 plane
    const T* base = i2 + static_cast<size_t>(b) * P.n_out * plane;
    const bool has_p = G.o_pxy >= 0, has_v = G.o_vx >= 0;
    const T* pp = base + (has_p ? G.o_pxy : 0) * plane;
    const T* pvx = base + (has_v ? G.o_vx : 0) * plane;
    const T* pvy = base + (has_v ? G.o_vy : 0) * plane;
    // column DFTs at ky: thread r sums rows r, r + kThreads, ... (twiddle index ky * y mod Np_y,
    // stepped by ky * kThreads mod Np_y), every plane in the same pass
    const int npy = P.npy;
    const int t = gx / P.W, w = gx - t * P.W;
    const int kk = ((ky % npy) + npy) % npy;
    int idx = static_cast<int>((static_cast<long long>(kk) * threadIdx.x) % npy);
    const int stride = static_cast<int>((static_cast<long long>(kk) * kThreads) % npy);
    double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // pxy, vx, vy (re, im)
    for (int y = threadIdx.x; y < npy; y += kThreads) {
        const double2 tw = G.wtab[idx];
        idx += stride;
        if (idx >= npy) idx -= npy;
        if (has_p) gk_dft_term<T>(pp, G.pair_layout, P.W, npy, t, w, y, tw, acc[0], acc[1]);
        if (has_v) {
            gk_dft_term<T>(pvx, G.pair_layout, P.W, npy, t, w, y, tw, acc[2], acc[3]);
            gk_dft_term<T>(pvy, G.pair_layout, P.W, npy, t, w, y, tw, acc[4], acc[5]);
        }
    }
#pragma unroll
    for (int q = 0; q < 6; ++q)
        for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
    __shared__ double part[kThreads / 32][6];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < 6; ++q) part[wid][q] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
        double v = part[0][q];
        for (int k = 1; k < kThreads / 32; ++k) v += part[k][q];
        acc[q] = v;
    }
    double2 pxy = make_double2(0.0, 0.0);
    if (has_p) pxy = make_double2(acc[0], acc[1]);
    if (has_v) {  // compressible viscous: -i eta (ky vx + kx vy) with v transformed from physical space
        const double sr = kyv * acc[2] + kx * acc[4], si = kyv * acc[3] + kx * acc[5];
        pxy.x += P.eta * si;
        pxy.y -= P.eta * sr;
    }
    if (G.incomp_visc) {  // incompressible viscous: v = j / rho0 of the stage state
        const int j = ky >= 0 ? ky : ky + P.kyn;
        const size_t fst = static_cast<size_t>(P.hx) * P.kyn;
        const size_t pos = static_cast<size_t>(b) * P.nfields * fst + static_cast<size_t>(gx) * P.kyn + j;
        const double r0 = 1.0 / rho0[b];
        const cplx<T> jx = cur[pos + (P.nop + 1) * fst], jy = cur[pos + (P.nop + 2) * fst];
        const double sr = (kyv * jx.x + kx * jy.x) * r0, si = (kyv * jx.y + kx * jy.y) * r0;
        pxy.x += P.eta * si;
        pxy.y -= P.eta * sr;
    }
    double2* fs = G.flux_step + static_cast<size_t>(b) * G.nmodes + i;
    double2 f = first_stage ? make_double2(0.0, 0.0) : *fs;
    f.x += weight * pxy.x;
    f.y += weight * pxy.y;
    if (!last_stage) {
        *fs = f;
        return;
    }
    const uint64_t step = *step_base + static_cast<uint64_t>(step_off);
    if (P.noise_j && !(gx == 0 && ky == 0)) {  // first draw of j_sto (fcalculator.cc:587-700), / sqrt(dt)
        const bool conj_line = (gx == 0 && ky < 0);
        const int aky = conj_line ? -ky : ky;
        const uint32_t mode_id = static_cast<uint32_t>(gx) * static_cast<uint32_t>(P.nay) + static_cast<uint32_t>((aky % P.nay + P.nay) % P.nay);
        cplx<T> xa, xb;  // the engine's own draw (its precision's normals)
        complex_normals<T>(P.seed, mi.key, step - static_cast<uint64_t>(mi.step0), j_stream(2), mode_id, false, xa, xb);
        const double xr = static_cast<double>(xa.x), xi = conj_line ? -static_cast<double>(xa.y) : static_cast<double>(xa.y);
        const double s = -P.j_s * mi.noise_scale * P.sqrt_eta / sqrt(dt);
        f.x += s * xr;
        f.y += s * xi;
    }
    // block accounting with the member's own step count
    const long long msteps = static_cast<long long>(step - static_cast<uint64_t>(mi.step0)) + 1;
    const int bs = static_cast<int>((msteps - 1) % G.nblock) + 1;
    double2* in = G.integral + static_cast<size_t>(b) * G.nmodes + i;
    double2 I = bs == 1 ? make_double2(0.0, 0.0) : *in;
    const double wdt = (bs == 1 ? 0.5 * dt : dt) * G.cell_area;
    I.x += wdt * f.x;
    I.y += wdt * f.y;
    if (bs % G.nevery == 0) {
        const int ti = bs / G.nevery - 1;
        const double tau = bs * dt;
        const double kbt = G.kbt * mi.noise_scale * mi.noise_scale;
        G.sums[(static_cast<size_t>(b) * G.ntau + ti) * G.nmodes + i] += (I.x * I.x + I.y * I.y) / (2.0 * tau * kbt * G.area);
    }
    *in = I;
}

// ---------------------------------------------------------------------------
// the step's flux buffer along one spectral line, for the ave/profile flux
// targets (measure_ave_profile.cc:216-238): axis 0 the ky = 0 row (gx < hx),
// axis 1 the kx = 0 column (engine ky order).  Per stage, the stage's flux
// weight times every flux the deterministic RHS records at the line's modes
// (fcalculator.cc:86-494: -i M k mu from the linear and physical chemical
// potential, psi v, cT^2 rho, the viscous stresses, j v); after the last stage
// the first noise draw's flux / sqrt(dt) (fcalculator.cc:496-700) and, in
// incompressible dynamics, the projection pressure (buffer_flux.cc:196-226).
// acc[member][comp][nline], comp = pi_xx, pi_xy, pi_yy, then Jpsi[a]_x,
// Jpsi[a]_y; one warp per line mode, 8 modes per block, grid (ceil(nline / 8),
// batch); on the kx = 0 column every mode transforms the same column of each
// product plane, so the block stages it once in shared memory (npy x 16 bytes);
// the first stage overwrites
// ---------------------------------------------------------------------------
// the engine step index after the current step is on a tap's schedule
__device__ __forceinline__ bool tap_scheduled(const unsigned long long* step_base, int step_off, long long period, long long phase) {
    if (period <= 1) return true;
    const long long s = static_cast<long long>(*step_base) + step_off + 1 - phase;
    return ((s % period) + period) % period == 0;
}

struct FluxLineArgs {
    double2* acc;
    int axis, nline, ncomp;
    const double2* wtab;          // exp(-2 pi i n / npy)
    int pair_layout;
    int mom_on;                   // j_det records anything
    int pressure;                 // linear pressure cT^2 rho on the diagonal
    int visc_comp, visc_incomp;   // compressible viscous stress from the VX, VY planes; incompressible from j / rho0
    int o_vx, o_vy, o_pxx, o_pxy, o_pyy;
    int psi_on[kMaxOp];           // psi_det records anything
    int psi_lin[kMaxOp];          // linear chemical-potential flux
    int o_mu[kMaxOp], o_px[kMaxOp], o_py[kMaxOp];
    int noise_j;                  // the momentum noise flux
    int incompressible;
    long long period, phase;      // record the steps s (engine step index after the step) with s = phase mod period
};

__device__ __forceinline__ double2 cmi(double2 a) { return make_double2(a.y, -a.x); }  // -i a
__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 dscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

template <typename T>
__global__ void __launch_bounds__(kThreads) flux_line_tap_kernel(const StepPlan P, const FluxLineArgs L, const MemberInfo* __restrict__ members,
                                                                 const T* __restrict__ i2, const cplx<T>* __restrict__ cur,
                                                                 const double2* __restrict__ k0cur, const double* __restrict__ rho0,
                                                                 const unsigned long long* __restrict__ step_base, int step_off, double weight,
                                                                 int first, int last, double dt) {
    extern __shared__ double2 col[];   // npy entries (kx = 0 column only)
    if (!tap_scheduled(step_base, step_off, L.period, L.phase)) return;  // grid-uniform
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.y;
    const int i = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
    const bool valid = i < L.nline;
    const MemberInfo mi = members[b];
    if (!mi.active) return;            // block-uniform
    const int gx = L.axis == 0 ? (valid ? i : 0) : 0;
    const int ky = L.axis == 0 ? 0 : (valid ? ky_of_j(i, P.nay) : 0);
    const double kx = P.kx_unit * gx, kyv = P.ky_unit * ky, k2 = kx * kx + kyv * kyv;
    const bool zero = gx == 0 && ky == 0;
    const size_t plane = static_cast<size_t>(P.hx) * P.npy * 2;
    const T* base = i2 + static_cast<size_t>(b) * P.n_out * plane;
    const size_t fst = static_cast<size_t>(P.hx) * P.kyn;
    const size_t pos = static_cast<size_t>(b) * P.nfields * fst + static_cast<size_t>(gx) * P.kyn + (ky >= 0 ? ky : ky + P.kyn);
    auto sv = [&](int f) {
        if (zero && k0cur) return k0cur[static_cast<size_t>(b) * P.nfields + f];
        const cplx<T> v = cur[pos + f * fst];
        return make_double2(static_cast<double>(v.x), static_cast<double>(v.y));
    };
    auto dft = [&](int o) {
        if (L.axis == 0) return column_dft<T>(P, L.wtab, L.pair_layout, base + o * plane, gx, ky);
        // kx = 0 column: stage column 0 of plane o once for the block, then one DFT per warp
        const T* pl = base + o * plane;
        __syncthreads();
        for (int y = threadIdx.x; y < P.npy; y += blockDim.x) {
            const T* e = L.pair_layout ? pl + 4 * static_cast<size_t>(y) : pl + 2 * static_cast<size_t>(y) * P.W;
            col[y] = make_double2(static_cast<double>(e[0]), static_cast<double>(e[L.pair_layout ? 2 : 1]));
        }
        __syncthreads();
        const int npy = P.npy;
        const int kk = ((ky % npy) + npy) % npy;
        int idx = static_cast<int>((static_cast<long long>(kk) * lane) % npy);
        const int stride = static_cast<int>((static_cast<long long>(kk) * 32) % npy);
        double re = 0.0, im = 0.0;
        for (int y = lane; y < npy; y += 32) {
            const double2 x = col[y], tw = L.wtab[idx];
            re += x.x * tw.x - x.y * tw.y;
            im += x.x * tw.y + x.y * tw.x;
            idx += stride;
            if (idx >= npy) idx -= npy;
        }
        for (int off = 16; off > 0; off >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, off);
            im += __shfl_xor_sync(0xffffffffu, im, off);
        }
        return make_double2(re, im);
    };
    double2 F[3 + 2 * kMaxOp];
    for (int c = 0; c < 3 + 2 * kMaxOp; ++c) F[c] = make_double2(0.0, 0.0);
    if (L.mom_on) {
        if (L.pressure) {
            const double2 pr = dscale(sv(0), P.cT2);
            F[0] = dadd(F[0], pr);
            F[2] = dadd(F[2], pr);
        }
        if (L.visc_incomp) {
            const double r0 = 1.0 / rho0[b];
            const double2 vx = dscale(sv(P.nop + 1), r0), vy = dscale(sv(P.nop + 2), r0);
            F[0] = dadd(F[0], cmi(dscale(vx, P.eta * 2.0 * kx)));
            F[1] = dadd(F[1], cmi(dscale(dadd(dscale(vx, kyv), dscale(vy, kx)), P.eta)));
            F[2] = dadd(F[2], cmi(dscale(vy, P.eta * 2.0 * kyv)));
        }
        if (L.visc_comp) {
            const double2 vx = dft(L.o_vx), vy = dft(L.o_vy);
            const double2 kv = dadd(dscale(vx, kx), dscale(vy, kyv));
            F[0] = dadd(F[0], cmi(dadd(dscale(vx, 2.0 * P.eta * kx), dscale(kv, -(P.eta - P.zeta)))));
            F[1] = dadd(F[1], cmi(dscale(dadd(dscale(vx, kyv), dscale(vy, kx)), P.eta)));
            F[2] = dadd(F[2], cmi(dadd(dscale(vy, 2.0 * P.eta * kyv), dscale(kv, -(P.eta - P.zeta)))));
        }
        if (L.o_pxx >= 0) F[0] = dadd(F[0], dft(L.o_pxx));
        if (L.o_pxy >= 0) F[1] = dadd(F[1], dft(L.o_pxy));
        if (L.o_pyy >= 0) F[2] = dadd(F[2], dft(L.o_pyy));
    }
    for (int a = 0; a < P.nop; ++a) {
        if (!L.psi_on[a]) continue;
        const double M = P.mobility[a];
        if (L.psi_lin[a]) {
            const double2 mu = dscale(sv(1 + a), P.mu_k0[a] + P.mu_k2[a] * k2 + P.mu_k4[a] * k2 * k2);
            F[3 + 2 * a] = dadd(F[3 + 2 * a], cmi(dscale(mu, M * kx)));
            F[4 + 2 * a] = dadd(F[4 + 2 * a], cmi(dscale(mu, M * kyv)));
        }
        if (L.o_mu[a] >= 0) {
            const double2 mu = dft(L.o_mu[a]);
            F[3 + 2 * a] = dadd(F[3 + 2 * a], cmi(dscale(mu, M * kx)));
            F[4 + 2 * a] = dadd(F[4 + 2 * a], cmi(dscale(mu, M * kyv)));
        }
        if (L.o_px[a] >= 0) F[3 + 2 * a] = dadd(F[3 + 2 * a], dft(L.o_px[a]));
        if (L.o_py[a] >= 0) F[4 + 2 * a] = dadd(F[4 + 2 * a], dft(L.o_py[a]));
    }
    if (lane != 0 || !valid) return;
    double2* acc = L.acc + static_cast<size_t>(b) * L.ncomp * L.nline + i;
    for (int c = 0; c < L.ncomp; ++c) {
        double2& a = acc[static_cast<size_t>(c) * L.nline];
        a = first ? dscale(F[c], weight) : dadd(a, dscale(F[c], weight));
    }
    if (!last || zero) return;
    // the first draw of psi_sto / j_sto (the engine's own, as the epilogue drew it), / sqrt(dt)
    const uint64_t step = *step_base + static_cast<uint64_t>(step_off) - static_cast<uint64_t>(mi.step0);
    const bool conj_line = gx == 0 && ky < 0;
    const int aky = conj_line ? -ky : ky;
    const uint32_t mode_id = static_cast<uint32_t>(gx) * static_cast<uint32_t>(P.nay) + static_cast<uint32_t>((aky % P.nay + P.nay) % P.nay);
    const double isdt = 1.0 / sqrt(dt);
    auto draw = [&](uint32_t stream) {
        cplx<T> xa, xb;
        complex_normals<T>(P.seed, mi.key, step, stream, mode_id, false, xa, xb);
        return make_double2(static_cast<double>(xa.x), conj_line ? -static_cast<double>(xa.y) : static_cast<double>(xa.y));
    };
    if (L.noise_j) {
        const double2 x0 = draw(j_stream(0)), x1 = draw(j_stream(1)), x2 = draw(j_stream(2));
        const double s = -P.j_s * mi.noise_scale * isdt;
        acc[0] = dadd(acc[0], dscale(dadd(dscale(x0, P.sqrt_zeta), dscale(x1, P.sqrt_eta)), s));
        acc[2 * static_cast<size_t>(L.nline)] = dadd(acc[2 * static_cast<size_t>(L.nline)], dscale(dadd(dscale(x0, P.sqrt_zeta), dscale(x1, -P.sqrt_eta)), s));
        acc[static_cast<size_t>(L.nline)] = dadd(acc[static_cast<size_t>(L.nline)], dscale(x2, s * P.sqrt_eta));
    }
    for (int a = 0; a < P.nop; ++a) {
        if (!P.noise_psi[a]) continue;
        const double2 x = draw(psi_stream(a));
        const double sig = sqrt(P.psi_sig2[a] * k2) * mi.noise_scale * isdt;
        // i k / k^2 sigma x; no x-component on the kx = 0 line
        const double2 ix = make_double2(-x.y, x.x);
        if (gx != 0) acc[static_cast<size_t>(3 + 2 * a) * L.nline] = dadd(acc[static_cast<size_t>(3 + 2 * a) * L.nline], dscale(ix, sig * kx / k2));
        acc[static_cast<size_t>(4 + 2 * a) * L.nline] = dadd(acc[static_cast<size_t>(4 + 2 * a) * L.nline], dscale(ix, sig * kyv / k2));
    }
    if (L.incompressible) {
        const double2 xx = acc[0], xy = acc[L.nline], yy = acc[2 * static_cast<size_t>(L.nline)];
        const double2 rx = cmi(dadd(dscale(xx, kx), dscale(xy, kyv))), ry = cmi(dadd(dscale(xy, kx), dscale(yy, kyv)));
        const double2 ph = dscale(cmi(dadd(dscale(rx, kx), dscale(ry, kyv))), 1.0 / k2);
        acc[0] = dadd(xx, ph);
        acc[2 * static_cast<size_t>(L.nline)] = dadd(yy, ph);
    }
}

// ---------------------------------------------------------------------------
// k = 0 fluxes of the time-series measure (measure_time_series.cc:190-229): per
// stage, the stage's flux weight times the (0, 0) coefficient of pi_xx, pi_xy,
// pi_yy and of psi_a v_x, psi_a v_y, i.e. the sums over y of the kx = 0 column
// of the stage's x-transformed product planes, plus the linear pressure
// cT^2 rho(0) on the diagonal; the gradient terms and the noise vanish at
// k = 0.  The first stage of a step overwrites, so acc holds the last step's.
// acc[member][3 + 2 nop]; one block per (column, member)
// ---------------------------------------------------------------------------
struct Flux0Args {
    double* acc;
    int ncol;                     // 3 + 2 nop: pi_xx, pi_xy, pi_yy, then (Jpsi[a]_x, Jpsi[a]_y) per a
    int o[3 + 2 * kMaxOp];        // product plane of each column in I2 (-1: no advective term)
    int pressure;                 // cT^2 rho(0) on pi_xx and pi_yy
    int pair_layout;              // I2 element (re_2t, re_2t+1, im_2t, im_2t+1) with W = 2
    long long period, phase;      // record the steps s (engine step index after the step) with s = phase mod period
};


template <typename T>
__global__ void __launch_bounds__(kThreads) flux0_tap_kernel(const StepPlan P, const Flux0Args F, const MemberInfo* __restrict__ members,
                                                             const T* __restrict__ i2, const cplx<T>* __restrict__ cur,
                                                             const double2* __restrict__ k0cur, double weight, int first,
                                                             const unsigned long long* __restrict__ step_base, int step_off) {
    if (!tap_scheduled(step_base, step_off, F.period, F.phase)) return;  // grid-uniform
    // one block per (column, member): strided rows per thread, then a fixed-order block sum
    const int c = blockIdx.x, b = blockIdx.y;
    if (!members[b].active) return;  // the whole block
    double v = 0.0;
    const int o = F.o[c];
    if (o >= 0) {
        const size_t plane = static_cast<size_t>(P.hx) * P.npy * 2;  // scalars of one I2 plane
        const T* base = i2 + (static_cast<size_t>(b) * P.n_out + o) * plane;
        for (int y = threadIdx.x; y < P.npy; y += kThreads)  // kx = 0: tile 0, slot 0, real part
            v += static_cast<double>(F.pair_layout ? base[4 * static_cast<size_t>(y)] : base[2 * static_cast<size_t>(y) * P.W]);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        __shared__ double part[kThreads / 32];
        if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            v = part[0];
            for (int k = 1; k < kThreads / 32; ++k) v += part[k];
        }
    }
    if (threadIdx.x != 0) return;
    if (F.pressure && (c == 0 || c == 2)) {
        const size_t fst = static_cast<size_t>(P.hx) * P.kyn;
        const double r00 = k0cur ? k0cur[static_cast<size_t>(b) * P.nfields].x
                                 : static_cast<double>(cur[static_cast<size_t>(b) * P.nfields * fst].x);
        v += P.cT2 * r00;
    }
    double* a = F.acc + static_cast<size_t>(b) * F.ncol + c;
    *a = first ? weight * v : *a + weight * v;
}

// ---------------------------------------------------------------------------
// spectral L2 sums of the time-series measure (measure_time_series.cc, the
// |rho|^2 ... |d_psi[a]|^2 columns): per field, sum over the active modes but
// (0, 0) of w |u|^2 and w k^2 |u|^2, w = 2 off the kx = 0 line; FP64, one
// member; grid: ceil(Hx * Ky / 256); out[field][2] accumulated with atomics
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) l2_sums_kernel(const StepPlan P, const cplx<T>* __restrict__ state, int b, double* __restrict__ out) {
    __shared__ double red[kThreads / 32][2 * kMaxFields];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    double acc[2 * kMaxFields];
    for (int q = 0; q < 2 * kMaxFields; ++q) acc[q] = 0.0;
    if (e < static_cast<int>(fstride)) {
        const int gx = e / P.kyn, j = e - gx * P.kyn;
        const int ky = ky_of_j(j, P.nay);
        if (gx != 0 || ky != 0) {
            const double w = gx == 0 ? 1.0 : 2.0;
            const double kx = P.kx_unit * gx, kyv = P.ky_unit * ky;
            const double k2 = kx * kx + kyv * kyv;
            for (int f = 0; f < P.nfields; ++f) {
                const cplx<T> v = state[(static_cast<size_t>(b) * P.nfields + f) * fstride + e];
                const double n2 = static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
                acc[2 * f] = w * n2;
                acc[2 * f + 1] = w * k2 * n2;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < 2 * P.nfields; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < 2 * P.nfields) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
        atomicAdd(out + threadIdx.x, v);
    }
}

// ---------------------------------------------------------------------------
// initial conditions written on the device (initial_condition_*.cc): one spec
// per field, evaluated per active mode in FP64 by ic_value, which the writer,
// the random-vorticity norm and the transversality check share.  Wave numbers
// are formed as the reference's Domain2D::kx/ky do (2 pi g / L).
// ---------------------------------------------------------------------------
enum IcStyle { IC_GAUSSIAN_MODES = 0, IC_TRANSVERSE_GAUSSIAN = 1, IC_RANDOM_VORTICITY = 2, IC_BUMP = 3, IC_SINE = 4 };

struct IcSpec {
    int style, channel;
    unsigned long long seed;
    double mean;              // (0, 0) coefficient (GAUSSIAN_MODES, SINE; added to the bump's own)
    double s0, c0, c2, c4;    // sigma(k)^2 = s0 / (c0 + c2 k^2 + c4 k^4)
    double factor;            // RANDOM_VORTICITY: rho0 * urms Ng / sqrt(norm); BUMP: A Ng 2 pi sx sy / (Lx Ly); SINE: -A Ng / 2
    double n0, sigma;         // RANDOM_VORTICITY shell in mode numbers
    double x0, y0, sx, sy;    // BUMP
    int nkx, nky;             // SINE
    double lx, ly;            // box lengths
};

__device__ __forceinline__ unsigned long long ic_splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
__device__ __forceinline__ unsigned long long ic_u32(long long v) { return static_cast<unsigned long long>(v) & 0xFFFFFFFFull; }
__device__ __forceinline__ double ic_unit(unsigned long long key) {
    return static_cast<double>(ic_splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}
// key of the equilibrium styles: seed ^ channel << 48 ^ gx << 32 ^ ky << 8 ^ draw
__device__ __forceinline__ double ic_uniform(unsigned long long seed, int channel, int gx, int ky, int draw) {
    return ic_unit(ic_u32(static_cast<long long>(seed)) ^ (ic_u32(channel) << 48) ^ (ic_u32(gx) << 32) ^ (ic_u32(ky) << 8) ^
                   ic_u32(draw));
}
// complex unit Gaussian of the equilibrium styles at (gx, ky), kx = 0 line conjugated for ky < 0
__device__ __forceinline__ double2 ic_gaussian(unsigned long long seed, int channel, int gx, int ky) {
    const int pky = gx == 0 ? (ky < 0 ? -ky : ky) : ky;
    const double u1 = fmax(ic_uniform(seed, channel, gx, pky, 0), 1.0e-300);
    const double u2 = ic_uniform(seed, channel, gx, pky, 1);
    const double r = sqrt(-2.0 * log(u1)), th = 2.0 * 3.14159265358979323846 * u2;
    double2 v = make_double2(r * cos(th), r * sin(th));
    if (gx == 0 && ky < 0) v.y = -v.y;
    return v;
}
// random-vorticity velocity (u_x, u_y) before normalisation; zero at k = 0
__device__ __forceinline__ void ic_vorticity(const IcSpec& s, int gx, int ky, double kx, double kyv, double k2, double2& ux,
                                             double2& uy) {
    ux = uy = make_double2(0.0, 0.0);
    if (k2 == 0.0) return;
    const int pky = gx == 0 ? (ky < 0 ? -ky : ky) : ky;
    const double n = sqrt(static_cast<double>(gx) * gx + static_cast<double>(ky) * ky);
    const double d = (n - s.n0) / s.sigma;
    const double env = exp(-0.5 * d * d);
    const double th = 2.0 * 3.14159265358979323846 *
                      ic_unit(ic_u32(static_cast<long long>(s.seed)) ^ (ic_u32(gx) << 32) ^ ic_u32(pky));
    double2 om = make_double2(env * cos(th), env * sin(th));
    if (gx == 0 && ky < 0) om.y = -om.y;
    const double ax = kyv / k2, ay = kx / k2;
    ux = make_double2(-ax * om.y, ax * om.x);   // (i ky / k^2) omega
    uy = make_double2(ay * om.y, -ay * om.x);   // -(i kx / k^2) omega
}

__device__ inline double2 ic_value(const IcSpec& s, int gx, int ky) {
    const double kx = 2.0 * 3.14159265358979323846 * gx / s.lx, kyv = 2.0 * 3.14159265358979323846 * ky / s.ly;
    const double k2 = kx * kx + kyv * kyv;
    const bool zero = gx == 0 && ky == 0;
    switch (s.style) {
        case IC_GAUSSIAN_MODES: {
            if (zero) return make_double2(s.mean, 0.0);
            if (s.s0 == 0.0) return make_double2(0.0, 0.0);
            const double sigma = sqrt(s.s0 / (s.c0 + s.c2 * k2 + s.c4 * k2 * k2));
            const double2 g = ic_gaussian(s.seed, s.channel, gx, ky);
            return make_double2(sigma * g.x, sigma * g.y);
        }
        case IC_TRANSVERSE_GAUSSIAN: {
            if (zero || s.s0 == 0.0) return make_double2(0.0, 0.0);
            const double k = sqrt(k2);
            const double comp = s.channel == 0 ? (-kyv / k) : (kx / k);
            const double sigma = sqrt(s.s0);
            const double2 g = ic_gaussian(s.seed, 0, gx, ky);
            return make_double2(comp * (sigma * g.x), comp * (sigma * g.y));
        }
        case IC_RANDOM_VORTICITY: {
            double2 ux, uy;
            ic_vorticity(s, gx, ky, kx, kyv, k2, ux, uy);
            const double2 u = s.channel == 0 ? ux : uy;
            return make_double2(s.factor * u.x, s.factor * u.y);
        }
        case IC_BUMP: {
            const double env = exp(-0.5 * (s.sx * s.sx * kx * kx + s.sy * s.sy * kyv * kyv));
            const double ph = -(kx * s.x0 + kyv * s.y0);
            const double a = s.factor * env;
            double2 v = make_double2(a * cos(ph), a * sin(ph));
            if (zero) v.x += s.mean;
            return v;
        }
        case IC_SINE: {
            if (zero) return make_double2(s.mean, 0.0);
            if (gx == s.nkx && ky == s.nky) return make_double2(0.0, s.factor);
            if (s.nkx == 0 && s.nky != 0 && gx == 0 && ky == -s.nky) return make_double2(0.0, -s.factor);
            return make_double2(0.0, 0.0);
        }
        default: return make_double2(0.0, 0.0);
    }
}

// writes every active mode of one field of member b; the (0, 0) value also to k0 (FP64 copy) when given.
// grid: ceil(Hx * Ky / 256)
template <typename T>
__global__ void __launch_bounds__(kThreads) initial_field_kernel(const StepPlan P, cplx<T>* __restrict__ state, int b, int field,
                                                                 const IcSpec s, double2* __restrict__ k0) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    if (e >= static_cast<int>(fstride)) return;
    const int gx = e / P.kyn, j = e - gx * P.kyn;
    const int ky = ky_of_j(j, P.nay);
    const double2 v = ic_value(s, gx, ky);
    state[(static_cast<size_t>(b) * P.nfields + field) * fstride + e] = mk(static_cast<T>(v.x), static_cast<T>(v.y));
    if (k0 && e == 0) *k0 = v;
}

// block sums of w (|u_x|^2 + |u_y|^2) of the random-vorticity shell over the active modes, w = 2 off the
// kx = 0 line; partial[blockIdx.x].  grid: ceil(Hx * Ky / 256)
static __global__ void __launch_bounds__(kThreads) vorticity_norm_kernel(const StepPlan P, const IcSpec s, double* __restrict__ partial) {
    __shared__ double red[kThreads / 32];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double v = 0.0;
    if (e < P.hx * P.kyn) {
        const int gx = e / P.kyn, j = e - gx * P.kyn;
        const int ky = ky_of_j(j, P.nay);
        const double kx = 2.0 * 3.14159265358979323846 * gx / s.lx, kyv = 2.0 * 3.14159265358979323846 * ky / s.ly;
        double2 ux, uy;
        ic_vorticity(s, gx, ky, kx, kyv, kx * kx + kyv * kyv, ux, uy);
        v = (gx == 0 ? 1.0 : 2.0) * ((ux.x * ux.x + ux.y * ux.y) + (uy.x * uy.x + uy.y * uy.y));
    }
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// out[v] = sum over i < n of partial[i * nv + v] in a fixed order (deterministic); grid: nv blocks of kThreads
static __global__ void __launch_bounds__(kThreads) sum_partials_kernel(const double* __restrict__ partial, int n, int nv, double* __restrict__ out) {
    __shared__ double red[kThreads];
    const int v = blockIdx.x;
    double t = 0.0;
    for (int i = threadIdx.x; i < n; i += kThreads) t += partial[static_cast<size_t>(i) * nv + v];
    red[threadIdx.x] = t;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[v] = red[0];
}

// the incompressible check on two momentum specs, in FP64 (initial_condition.cc:7-40): sets *bad when
// |k . j| > 1e-10 + 1e-10 |k| |j| at an active mode k != 0.  grid: ceil(Hx * Ky / 256)
static __global__ void __launch_bounds__(kThreads) transverse_check_kernel(const StepPlan P, const IcSpec sx, const IcSpec sy, int* __restrict__ bad) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.hx * P.kyn) return;
    const int gx = e / P.kyn, j = e - gx * P.kyn;
    const int ky = ky_of_j(j, P.nay);
    const double kx = 2.0 * 3.14159265358979323846 * gx / sx.lx, kyv = 2.0 * 3.14159265358979323846 * ky / sx.ly;
    const double k2 = kx * kx + kyv * kyv;
    if (k2 == 0.0) return;
    const double2 jx = ic_value(sx, gx, ky), jy = ic_value(sy, gx, ky);
    const double re = kx * jx.x + kyv * jy.x, im = kx * jx.y + kyv * jy.y;
    const double viol = sqrt(re * re + im * im);
    const double scale = sqrt(k2) * sqrt((jx.x * jx.x + jx.y * jx.y) + (jy.x * jy.x + jy.y * jy.y));
    if (viol > 1.0e-10 + 1.0e-10 * scale) atomicOr(bad, 1);
}

// ---------------------------------------------------------------------------
// time-series energies (measure_time_series.cc:152-188, 305-470), FP64 sums
// ---------------------------------------------------------------------------
// spectral terms of one member, per block: [0] w (|jx|^2 + |jy|^2) over every active mode,
// [1] w |rho|^2 over the active modes but (0, 0), [2 + a] w (k0 + k2 k^2 + k4 k^4) |psi_a|^2 over
// every active mode; w = 2 off the kx = 0 line.  The (0, 0) values come from k0 (FP64) when given.
// partial[block][2 + nop]; grid: ceil(Hx * Ky / 256)
template <typename T>
__global__ void __launch_bounds__(kThreads) energy_spectral_kernel(const StepPlan P, const cplx<T>* __restrict__ state,
                                                                   const double2* __restrict__ k0, double* __restrict__ partial) {
    __shared__ double red[kThreads / 32][2 + kMaxOp];
    const int nv = 2 + P.nop;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    double acc[2 + kMaxOp];
    for (int q = 0; q < 2 + kMaxOp; ++q) acc[q] = 0.0;
    if (e < static_cast<int>(fstride)) {
        const int gx = e / P.kyn, j = e - gx * P.kyn;
        const int ky = ky_of_j(j, P.nay);
        const bool zero = gx == 0 && ky == 0;
        const double w = gx == 0 ? 1.0 : 2.0;
        const double kx = P.kx_unit * gx, kyv = P.ky_unit * ky;
        const double k2 = kx * kx + kyv * kyv;
        auto norm2 = [&](int f) {
            if (zero && k0) return k0[f].x * k0[f].x + k0[f].y * k0[f].y;
            const cplx<T> v = state[static_cast<size_t>(f) * fstride + e];
            return static_cast<double>(v.x) * v.x + static_cast<double>(v.y) * v.y;
        };
        acc[0] = w * (norm2(P.nop + 1) + norm2(P.nop + 2));
        if (!zero) acc[1] = w * norm2(0);
        for (int a = 0; a < P.nop; ++a) acc[2 + a] = w * (P.mu_k0[a] + P.mu_k2[a] * k2 + P.mu_k4[a] * k2 * k2) * norm2(1 + a);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nv; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v += red[w][threadIdx.x];
        partial[static_cast<size_t>(blockIdx.x) * nv + threadIdx.x] = v;
    }
}

// physical-space terms over one row pair of a single-member plan's inputs (runtime-plan transforms):
// term 0: (jx^2 + jy^2) / (2 rho) with inputs rho, jx, jy; term 1: psi^4 with input psi (the host
// scales by u / 4).  partial[pair]; grid: ceil(npy / 2)
template <typename T>
__global__ void __launch_bounds__(kThreads) energy_row_kernel(const StepPlan P, const cplx<T>* __restrict__ i1, const cplx<T>* __restrict__ tw,
                                                              int term, double* __restrict__ partial) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[kThreads / 32];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    const int npx = P.npx;
    C* lines = s_tw + P.twx_count;
    C* scr = lines + static_cast<size_t>(P.n_in) * npx;
    const int y0 = 2 * blockIdx.x;
    const bool has1 = (y0 + 1) < P.npy;
    load_table(s_tw, tw, P.twx_count);
    __syncthreads();
    row_inputs_inverse<T, 0>(P, i1, y0, has1, lines, scr, s_tw);
    __syncthreads();
    double acc = 0.0;
    for (int x = threadIdx.x; x < npx; x += blockDim.x) {
        if (term == 0) {
            const C rho = lines[x], jx = lines[npx + x], jy = lines[2 * npx + x];
            acc += 0.5 * (static_cast<double>(jx.x) * jx.x + static_cast<double>(jy.x) * jy.x) / static_cast<double>(rho.x);
            if (has1) acc += 0.5 * (static_cast<double>(jx.y) * jx.y + static_cast<double>(jy.y) * jy.y) / static_cast<double>(rho.y);
        } else if (term == 1) {
            const C p = lines[x];
            const double a = static_cast<double>(p.x) * p.x, b = static_cast<double>(p.y) * p.y;
            acc += a * a;
            if (has1) acc += b * b;
        } else {  // plugin free-energy density; lines hold the order parameters in order
            double p0[kMaxOp], p1[kMaxOp];
#pragma unroll
            for (int b = 0; b < kMaxOp; ++b) {
                p0[b] = 0.0;
                p1[b] = 0.0;
                if (b < P.n_in) {
                    const C v = lines[static_cast<size_t>(b) * npx + x];
                    p0[b] = v.x;
                    p1[b] = v.y;
                }
            }
            acc += plugin_density<double>(P, p0);
            if (has1) acc += plugin_density<double>(P, p1);
        }
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) t += red[w];
        partial[blockIdx.x] = t;
    }
}

// ---------------------------------------------------------------------------
// ave/profile (measure_ave_profile.cc:180-374): one sample of a profile
// ---------------------------------------------------------------------------
// the spectral line a profile needs, FP64: axis 0 (bins over x) the ky = 0 row, out[gx] for gx < hx;
// axis 1 (bins over y) the kx = 0 column, out[j] in the engine's ky order (j < kyn).  (0, 0) from
// k0 (FP64) when given.  grid: ceil(max(hx, kyn) / 256)
template <typename T>
__global__ void __launch_bounds__(kThreads) profile_line_kernel(const StepPlan P, const cplx<T>* __restrict__ field_modes,
                                                                const double2* __restrict__ k0, int axis, double2* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = axis == 0 ? P.hx : P.kyn;
    if (i >= n) return;
    const size_t e = axis == 0 ? static_cast<size_t>(i) * P.kyn : static_cast<size_t>(i);
    double2 v;
    if (i == 0 && k0) {
        v = *k0;
    } else {
        const cplx<T> a = field_modes[e];
        v = make_double2(static_cast<double>(a.x), static_cast<double>(a.y));
    }
    out[i] = v;
}

// compressible velocity j_c / rho of one sample summed over the transverse axis (single-member plan
// inputs rho, jx, jy): axis 1 writes out[y] = sum over x for the block's rows; axis 0 writes the block's
// two rows summed, partial[pair][x] (physical x at shared slot sw(x)).  Sets *bad on a zero density.
// grid: ceil(npy / 2)
template <typename T>
__global__ void __launch_bounds__(kThreads) profile_velocity_row_kernel(const StepPlan P, const cplx<T>* __restrict__ i1,
                                                                        const cplx<T>* __restrict__ tw, int axis, int component,
                                                                        double* __restrict__ out, int* __restrict__ bad) {
    using C = cplx<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[2][kThreads / 32];
    C* s_tw = reinterpret_cast<C*>(smem_raw);
    const int npx = P.npx;
    C* lines = s_tw + P.twx_count;
    C* scr = lines + static_cast<size_t>(P.n_in) * npx;
    const int y0 = 2 * blockIdx.x;
    const bool has1 = (y0 + 1) < P.npy;
    load_table(s_tw, tw, P.twx_count);
    __syncthreads();
    row_inputs_inverse<T, 0>(P, i1, y0, has1, lines, scr, s_tw);
    __syncthreads();
    const C* j = lines + static_cast<size_t>(1 + component) * npx;
    double a0 = 0.0, a1 = 0.0;
    int zero = 0;
    for (int x = threadIdx.x; x < npx; x += blockDim.x) {
        const uint32_t q = axis == 0 ? sw(static_cast<uint32_t>(x), P.fx.swz) : static_cast<uint32_t>(x);
        const C rho = lines[q], jc = j[q];
        if (rho.x == T(0) || (has1 && rho.y == T(0))) zero = 1;
        const double v0 = static_cast<double>(jc.x) / static_cast<double>(rho.x);
        const double v1 = has1 ? static_cast<double>(jc.y) / static_cast<double>(rho.y) : 0.0;
        if (axis == 0) {
            out[static_cast<size_t>(blockIdx.x) * npx + x] = v0 + v1;
        } else {
            a0 += v0;
            a1 += v1;
        }
    }
    if (zero) atomicOr(bad, 1);
    if (axis == 0) return;
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = a0;
        red[1][threadIdx.x >> 5] = a1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) {
            t0 += red[0][w];
            t1 += red[1][w];
        }
        out[y0] = t0;
        if (has1) out[y0 + 1] = t1;
    }
}

// out[x] = sum over the row pairs of partial[pair][x] in a fixed order; grid: ceil(npx / 256)
static __global__ void __launch_bounds__(kThreads) column_sums_kernel(const double* __restrict__ partial, int npairs, int npx, double* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= npx) return;
    double t = 0.0;
    for (int p = 0; p < npairs; ++p) t += partial[static_cast<size_t>(p) * npx + x];
    out[x] = t;
}

// step counter of the call: set from the host at the start of a call, advanced
// by the last node of a captured step graph
static __global__ void set_step_kernel(unsigned long long* step, unsigned long long value) { *step = value; }
static __global__ void advance_step_kernel(unsigned long long* step, unsigned long long by) { *step += by; }

// ---------------------------------------------------------------------------
// fields the integrator only copies: symmetrise the kx = 0 line once and
// mirror them into the stage buffers   (grid: chunks x fields x batch; chunk >= Ky elements
// per block, block 0 of a field first symmetrises its kx = 0 line)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kThreads) prepare_static_kernel(const StepPlan P, const int* __restrict__ fields, cplx<T>* u, cplx<T>* s1,
                                                                 cplx<T>* s2, double2* k0u, double2* k0s1, double2* k0s2, int chunk) {
    using C = cplx<T>;
    const int f = fields[blockIdx.y], b = blockIdx.z;
    const size_t fstride = static_cast<size_t>(P.hx) * P.kyn;
    C* uf = u + (static_cast<size_t>(b) * P.nfields + f) * fstride;
    if (blockIdx.x == 0) {  // the kx = 0 line (the first Ky elements, inside this block's chunk)
        const int half = P.nay / 2;
        if (threadIdx.x == 0) {
            uf[0].y = T(0);
            if (k0u) {  // FP32 engines: the FP64 k = 0 copy of the static field follows it into every buffer
                const size_t q = static_cast<size_t>(b) * P.nfields + f;
                const double2 v = make_double2(k0u[q].x, 0.0);
                k0u[q] = v;
                k0s1[q] = v;
                k0s2[q] = v;
            }
        }
        for (int ky = 1 + threadIdx.x; ky < half; ky += blockDim.x) {
            const int jn = P.kyn - ky;  // j of -ky
            const C a = uf[ky];
            const C c = uf[jn];
            const C pj = mk(static_cast<T>(0.5) * (a.x + c.x), static_cast<T>(0.5) * (a.y - c.y));
            uf[ky] = pj;
            uf[jn] = cconj(pj);
        }
        __syncthreads();
    }
    C* a1 = s1 + (static_cast<size_t>(b) * P.nfields + f) * fstride;
    C* a2 = s2 + (static_cast<size_t>(b) * P.nfields + f) * fstride;
    const size_t e0 = static_cast<size_t>(blockIdx.x) * chunk;
    const size_t e1 = e0 + chunk < fstride ? e0 + chunk : fstride;
    for (size_t e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const C v = uf[e];
        a1[e] = v;
        a2[e] = v;
    }
}

// ---------------------------------------------------------------------------
// reference State layout (FP64, [field][gy][gx <= nx/2]) <-> engine layout
// ---------------------------------------------------------------------------
// grid: (ceil(hx*kyn / 256), nfields); one thread per active mode
template <typename T>
__global__ void __launch_bounds__(kThreads) ref_to_active_kernel(const StepPlan P, int ref_hx, const double2* __restrict__ ref,
                                                                cplx<T>* __restrict__ act) {
    const int f = blockIdx.y;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.hx * P.kyn) return;
    const int gx = e / P.kyn, j = e - gx * P.kyn;
    const int ky = ky_of_j(j, P.nay);
    const int gy = ky >= 0 ? ky : ky + P.npy;
    const double2 v = ref[(static_cast<size_t>(f) * P.npy + gy) * ref_hx + gx];
    act[static_cast<size_t>(f) * P.hx * P.kyn + e] = mk(static_cast<T>(v.x), static_cast<T>(v.y));
}

// flags a nonzero entry outside the active modes; grid: (ceil(npy*ref_hx / 256), nfields)
static __global__ void __launch_bounds__(kThreads) check_inactive_kernel(const StepPlan P, int ref_hx, const double2* __restrict__ ref,
                                                                  int* __restrict__ bad) {
    const int f = blockIdx.y;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.npy * ref_hx) return;
    const int gy = e / ref_hx, gx = e - gy * ref_hx;
    const int sgy = gy <= P.npy / 2 ? gy : gy - P.npy;
    const bool active = gx < P.hx && (sgy < 0 ? -sgy : sgy) < P.nay / 2;
    if (active) return;
    const double2 v = ref[static_cast<size_t>(f) * P.npy * ref_hx + e];
    if (v.x != 0.0 || v.y != 0.0) atomicOr(bad, 1);
}

// grid: (ceil(npy*ref_hx / 256), nfields); writes every entry (zeros outside the active modes)
template <typename T>
__global__ void __launch_bounds__(kThreads) active_to_ref_kernel(const StepPlan P, int ref_hx, const cplx<T>* __restrict__ act,
                                                                double2* __restrict__ ref) {
    const int f = blockIdx.y;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= P.npy * ref_hx) return;
    const int gy = e / ref_hx, gx = e - gy * ref_hx;
    const int sgy = gy <= P.npy / 2 ? gy : gy - P.npy;
    double2 v = make_double2(0.0, 0.0);
    if (gx < P.hx && (sgy < 0 ? -sgy : sgy) < P.nay / 2) {
        const int j = sgy >= 0 ? sgy : sgy + P.kyn;
        const cplx<T> a = act[(static_cast<size_t>(f) * P.hx + gx) * P.kyn + j];
        v = make_double2(static_cast<double>(a.x), static_cast<double>(a.y));
    }
    ref[static_cast<size_t>(f) * P.npy * ref_hx + e] = v;
}

}  // namespace shhd
