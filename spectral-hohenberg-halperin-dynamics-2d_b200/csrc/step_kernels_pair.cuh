// FP32 step kernels on pair-lines for the compile-time sizes 96 ... 1536.
//
// Two transform lines travel together: a shared-memory element holds one
// position of both lines as (re_a, re_b, im_a, im_b), so every butterfly is
// done with packed FP32x2 instructions (add/sub/mul/fma .f32x2 of sm_100a) on
// two lines at once, and one 128-bit shared access moves both lines.  The
// column passes pair the two columns gx = 2t, 2t+1 of a column pair; the row
// pass pairs two fields of a row pair.  I1/I2 use the same element format:
//     I1/I2 [slot][t < Hx/2][y < Np_y]  (re_2t, re_2t+1, im_2t, im_2t+1)
//
// Transforms are in place, one butterfly per thread at a time (no stage is
// staged in registers), with radices (3, 8, ..., 8, r) whose strides are all
// powers of two.  The decimation-in-frequency form (DIF) takes natural order
// and leaves X[k] at slot pos(k) (mixed-radix digit reversal); the
// decimation-in-time form (DIT) takes x[n] at pos(n) and gives natural order.
// So the x-inverse (DIF) leaves physical values in digit-reversed order, the
// products are formed there (they are pointwise) and the x-forward (DIT)
// brings the spectrum back to natural order; the y-forward (DIF) leaves modes
// at pos(y), the epilogue reads them there and the next y-inverse (DIT) starts
// from pos(y).  No reordering pass exists.  The first and last stage of each
// transform is fused with what feeds or consumes it: global loads and stores,
// the product evaluation, the RHS accumulation and the gather of new modes.
#pragma once

#include <type_traits>

#include "step_kernels_fixed.cuh"

namespace shhd {

using u64 = unsigned long long;

// ---------------------------------------------------------------------------
// packed FP32x2 arithmetic
// ---------------------------------------------------------------------------
__device__ __forceinline__ u64 f2_add(u64 a, u64 b) { u64 r; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b)); return r; }
__device__ __forceinline__ u64 f2_sub(u64 a, u64 b) { u64 r; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b)); return r; }
__device__ __forceinline__ u64 f2_mul(u64 a, u64 b) { u64 r; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b)); return r; }
__device__ __forceinline__ u64 f2_fma(u64 a, u64 b, u64 c) {
    u64 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
__device__ __forceinline__ u64 f2_pack(float lo, float hi) { u64 r; asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi)); return r; }
__device__ __forceinline__ float f2_lo(u64 r) { float v; asm("{.reg .f32 t; mov.b64 {%0, t}, %1;}" : "=f"(v) : "l"(r)); return v; }
__device__ __forceinline__ float f2_hi(u64 r) { float v; asm("{.reg .f32 t; mov.b64 {t, %0}, %1;}" : "=f"(v) : "l"(r)); return v; }
__device__ __forceinline__ u64 f2_splat(float a) { return f2_pack(a, a); }

// twiddles: read-only and shared by every CTA, so kept in L1 (evict last)
__device__ __forceinline__ float2 ld_tw2(const float2* p) {
    float2 v;
    asm("ld.global.nc.L1::evict_last.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}
// transform planes: read once per kernel, so not allocated in L1
__device__ __forceinline__ ulonglong2 ld_stream(const ulonglong2* p) {
    ulonglong2 v;
    asm("ld.global.L1::no_allocate.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}
// and written once: kept out of L1, so that the lines the scattered plane writes touch do not
// evict the twiddles
__device__ __forceinline__ void st_stream(ulonglong2* p, ulonglong2 v) {
    asm volatile("st.global.L1::no_allocate.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(v.x), "l"(v.y) : "memory");
}

// entry i of a twiddle table
__device__ __forceinline__ float2 tw_at(const float2* __restrict__ tw, int i) { return ld_tw2(tw + i); }

// one position of two lines: re = (re_a, re_b), im = (im_a, im_b)
struct PC {
    u64 re, im;
};
__device__ __forceinline__ PC pc_zero() { return PC{0ull, 0ull}; }
__device__ __forceinline__ PC ld_pc(const ulonglong2* p) { const ulonglong2 v = *p; return PC{v.x, v.y}; }
__device__ __forceinline__ void st_pc(ulonglong2* p, PC v) { *p = make_ulonglong2(v.re, v.im); }
__device__ __forceinline__ PC padd(PC a, PC b) { return PC{f2_add(a.re, b.re), f2_add(a.im, b.im)}; }
__device__ __forceinline__ PC psub(PC a, PC b) { return PC{f2_sub(a.re, b.re), f2_sub(a.im, b.im)}; }
// a + DIR i b,  a - DIR i b
template <int DIR> __device__ __forceinline__ PC prot_add(PC a, PC b) {
    return DIR > 0 ? PC{f2_sub(a.re, b.im), f2_add(a.im, b.re)} : PC{f2_add(a.re, b.im), f2_sub(a.im, b.re)};
}
template <int DIR> __device__ __forceinline__ PC prot_sub(PC a, PC b) {
    return DIR > 0 ? PC{f2_add(a.re, b.im), f2_sub(a.im, b.re)} : PC{f2_sub(a.re, b.im), f2_add(a.im, b.re)};
}
// a * w (DIR < 0, forward sign) or a * conj(w) (DIR > 0); wx = (w.x, w.x), wy = (w.y, w.y)
template <int DIR> __device__ __forceinline__ PC pcmul(PC a, u64 wx, u64 wy) {
    if (DIR < 0) return PC{f2_sub(f2_mul(a.re, wx), f2_mul(a.im, wy)), f2_fma(a.re, wy, f2_mul(a.im, wx))};
    return PC{f2_fma(a.im, wy, f2_mul(a.re, wx)), f2_sub(f2_mul(a.im, wx), f2_mul(a.re, wy))};
}
__device__ __forceinline__ float2 pc_col(PC v, int half) {  // one line's complex value
    return half ? make_float2(f2_hi(v.re), f2_hi(v.im)) : make_float2(f2_lo(v.re), f2_lo(v.im));
}
__device__ __forceinline__ PC pc_make(float2 a, float2 b) { return PC{f2_pack(a.x, b.x), f2_pack(a.y, b.y)}; }

// x_q *= w^q (q = 1..R-1, DIR < 0) or conj: from one table twiddle w, powers by a product tree
// at most three roundings deep (ptwiddle_powers), applied to a butterfly's values (ptwiddle_apply)
template <int R>
__device__ __forceinline__ void ptwiddle_powers(float2 w1, float2* w) {
    w[1] = w1;
    auto cm = [](float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    if constexpr (R > 2) w[2] = cm(w1, w1);
    if constexpr (R > 3) w[3] = cm(w[2], w1);
    if constexpr (R > 4) {
        w[4] = cm(w[2], w[2]);
        w[5] = cm(w[4], w1);
        w[6] = cm(w[4], w[2]);
        w[7] = cm(w[4], w[3]);
    }
}
template <int R, int DIR>
__device__ __forceinline__ void ptwiddle_apply(PC* v, const float2* w) {
#pragma unroll
    for (int q = 1; q < R; ++q) v[q] = pcmul<DIR>(v[q], f2_splat(w[q].x), f2_splat(w[q].y));
}
template <int R, int DIR>
__device__ __forceinline__ void ptwiddle_pow(PC* v, float2 w1) {
    float2 w[8];
    ptwiddle_powers<R>(w1, w);
    ptwiddle_apply<R, DIR>(v, w);
}

// ---------------------------------------------------------------------------
// butterflies: y_q = sum_p x_p e^{DIR 2 pi i p q / R}
// ---------------------------------------------------------------------------
template <int DIR> __device__ __forceinline__ void pbfly2(PC* v) {
    const PC a = v[0];
    v[0] = padd(a, v[1]);
    v[1] = psub(a, v[1]);
}
template <int DIR> __device__ __forceinline__ void pbfly4(PC* v) {
    const PC a = padd(v[0], v[2]), b = psub(v[0], v[2]);
    const PC c = padd(v[1], v[3]), d = psub(v[1], v[3]);
    v[0] = padd(a, c);
    v[2] = psub(a, c);
    v[1] = prot_add<DIR>(b, d);
    v[3] = prot_sub<DIR>(b, d);
}
template <int DIR> __device__ __forceinline__ void pbfly8(PC* v) {
    PC e[4] = {v[0], v[2], v[4], v[6]};
    PC o[4] = {v[1], v[3], v[5], v[7]};
    pbfly4<DIR>(e);
    pbfly4<DIR>(o);
    const u64 H = f2_splat(0.70710678118654752440f), NH = f2_splat(-0.70710678118654752440f);
    v[0] = padd(e[0], o[0]);
    v[4] = psub(e[0], o[0]);
    {   // w8 o1 = h (re - DIR im, im + DIR re)
        const u64 tr = DIR > 0 ? f2_sub(o[1].re, o[1].im) : f2_add(o[1].re, o[1].im);
        const u64 ti = DIR > 0 ? f2_add(o[1].im, o[1].re) : f2_sub(o[1].im, o[1].re);
        v[1] = PC{f2_fma(tr, H, e[1].re), f2_fma(ti, H, e[1].im)};
        v[5] = PC{f2_fma(tr, NH, e[1].re), f2_fma(ti, NH, e[1].im)};
    }
    v[2] = prot_add<DIR>(e[2], o[2]);
    v[6] = prot_sub<DIR>(e[2], o[2]);
    {   // w8^3 o3 = h (-re - DIR im, DIR re - im)
        const u64 a = DIR > 0 ? f2_add(o[3].re, o[3].im) : f2_sub(o[3].re, o[3].im);  // re + DIR im
        const u64 c = DIR > 0 ? f2_sub(o[3].re, o[3].im) : f2_add(o[3].re, o[3].im);  // re - DIR im  (DIR re - im = DIR (re - DIR im))
        // value = (-h a, DIR h c)
        const u64 HC = DIR > 0 ? H : NH, NHC = DIR > 0 ? NH : H;
        v[3] = PC{f2_fma(a, NH, e[3].re), f2_fma(c, HC, e[3].im)};
        v[7] = PC{f2_fma(a, H, e[3].re), f2_fma(c, NHC, e[3].im)};
    }
}
template <int DIR> __device__ __forceinline__ void pbfly3(PC* v) {
    const u64 MH = f2_splat(-0.5f);
    const u64 SD = f2_splat(DIR * 0.86602540378443864676f), NSD = f2_splat(-DIR * 0.86602540378443864676f);
    const PC t = padd(v[1], v[2]), d = psub(v[1], v[2]);
    const PC m = PC{f2_fma(t.re, MH, v[0].re), f2_fma(t.im, MH, v[0].im)};
    v[0] = padd(v[0], t);
    v[1] = PC{f2_fma(d.im, NSD, m.re), f2_fma(d.re, SD, m.im)};
    v[2] = PC{f2_fma(d.im, SD, m.re), f2_fma(d.re, NSD, m.im)};
}
template <int R, int DIR> __device__ __forceinline__ void pbfly(PC* v) {
    if constexpr (R == 2) pbfly2<DIR>(v);
    else if constexpr (R == 3) pbfly3<DIR>(v);
    else if constexpr (R == 4) pbfly4<DIR>(v);
    else pbfly8<DIR>(v);
}

// ---------------------------------------------------------------------------
// plan of a pair transform: radices (3, 8, ..., 8, r), strides N / (r_0 ... r_s)
// ---------------------------------------------------------------------------
constexpr int kPairMaxStages = 6;
constexpr int kPairMaxN = 1536;

struct PPlan {
    int m;
    int r[kPairMaxStages];
    int s[kPairMaxStages];      // stride of stage s (sub-transform length / radix)
    int lg[kPairMaxStages];     // log2 of the stride
    int lr[kPairMaxStages];     // log2 of the radix (stages >= 1)
    int twoff[kPairMaxStages];  // offset of the stage's twiddles w_L^j, j < stride (float2 entries)
    int twsz;
};

__host__ __device__ constexpr int ilog2c(int v) {
    int l = 0;
    while ((1 << l) < v) ++l;
    return l;
}

__host__ __device__ constexpr PPlan make_pplan(int n) {
    PPlan p{};
    int k = 0, m = n / 3;
    p.r[k++] = 3;
    while (m >= 8) { p.r[k++] = 8; m /= 8; }
    if (m > 1) p.r[k++] = m;
    p.m = k;
    int L = n, off = 0;
    for (int i = 0; i < k; ++i) {
        p.s[i] = L / p.r[i];
        p.lg[i] = ilog2c(p.s[i]);
        p.lr[i] = ilog2c(p.r[i]);
        p.twoff[i] = off;
        if (L > p.r[i]) off += p.s[i];
        L /= p.r[i];
    }
    p.twsz = off;
    return p;
}

template <int N> struct PairPlan { static constexpr PPlan c = make_pplan(N); };

__host__ __device__ constexpr bool is_pair_size(int n) { return n == 96 || n == 192 || n == 384 || n == 768 || n == 1536; }

// slot of position p in a line: low three bits XORed with bits 3..5
__device__ __forceinline__ int psw(int p) { return p ^ ((p >> 3) & 7); }

// psw(base + q ST) for the positions of one butterfly of a stage with stride ST, span L and radix
// R, from psw(base) and the compile-time q where the stage's structure allows: strides that are
// multiples of 64 leave bits 3..5 alone; at stride 8 of a 64-point span bits 3..5 of base are
// zero and become q; at stride 1 of radix 8 the low three bits of base are zero
template <int ST, int L, int R>
__device__ __forceinline__ int psw_q(int base, int pswbase, int q) {
    if constexpr (ST % 64 == 0) return pswbase + q * ST;
    else if constexpr (ST == 8 && L == 64) return (base ^ q) + 8 * q;
    else if constexpr (ST == 1 && R == 8) return pswbase ^ q;
    else return psw(base + q * ST);
}

// digit-reversed position of natural index y, and its inverse
template <int N> __device__ __forceinline__ int ppos(int y) {
    constexpr PPlan pp = PairPlan<N>::c;
    const int yq = (y * 43691) >> 17;  // y / 3 (exact for y < 98304)
    int p = (y - 3 * yq) * pp.s[0];
    int rest = yq;
#pragma unroll
    for (int i = 1; i < pp.m; ++i) {
        p += (rest & (pp.r[i] - 1)) * pp.s[i];
        rest >>= pp.lr[i];
    }
    return p;
}
template <int N> __device__ __forceinline__ int ppinv(int p) {
    constexpr PPlan pp = PairPlan<N>::c;
    const int q0 = p >> pp.lg[0];
    int rem = p & (pp.s[0] - 1);
    int y = 0, mul = 1;
#pragma unroll
    for (int i = 1; i < pp.m; ++i) {
        const int q = rem >> pp.lg[i];
        rem &= pp.s[i] - 1;
        y += q * mul;
        mul *= pp.r[i];
    }
    return q0 + 3 * y;
}

// ---------------------------------------------------------------------------
// one in-place stage over `nl` lines; load(l, p) / store(l, p, v) move the
// value at natural slot index p (0 <= p < N) of line l.  DIF twiddles after
// the butterfly, DIT before; the stage-s twiddle of butterfly j is w_L^(j q).
// ---------------------------------------------------------------------------
// whether an IO object exposes line(l) for slot addressing (SmemIO and the like), or is a
// load / store function of (line, position)
template <typename T, typename = void> struct has_slots { static constexpr bool value = false; };
template <typename T> struct has_slots<T, decltype(void(T::kSlots))> { static constexpr bool value = T::kSlots; };

template <int N, int S, int DIR, bool DIT, int NT = kThreads, typename TW, typename Load, typename Store>
__device__ __forceinline__ void pstage_io(int nl, TW tw, Load&& load, Store&& store) {
    constexpr PPlan pp = PairPlan<N>::c;
    constexpr int R = pp.r[S], ST = pp.s[S], L = R * ST, NB = N / R;
    const int tot = nl * NB;
#pragma unroll 2
    for (int b = threadIdx.x; b < tot; b += NT) {
        const int l = b / NB, i = b - l * NB;
        const int j = i & (ST - 1);
        const int base = (i >> pp.lg[S]) * L + j;
        PC v[R];
        const int pb = psw(base);
        (void)pb;
        if constexpr (has_slots<std::decay_t<Load>>::value) {
            const ulonglong2* ln = load.line(l);
#pragma unroll
            for (int q = 0; q < R; ++q) v[q] = ld_pc(ln + psw_q<ST, L, R>(base, pb, q));
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q) v[q] = load(l, base + q * ST);
        }
        if constexpr (L > R) {
            if constexpr (DIT) ptwiddle_pow<R, DIR>(v, tw_at(tw, pp.twoff[S] + j));
        }
        pbfly<R, DIR>(v);
        if constexpr (L > R) {
            if constexpr (!DIT) ptwiddle_pow<R, DIR>(v, tw_at(tw, pp.twoff[S] + j));
        }
        if constexpr (has_slots<std::decay_t<Store>>::value) {
            ulonglong2* ln = store.line(l);
#pragma unroll
            for (int q = 0; q < R; ++q) st_pc(ln + psw_q<ST, L, R>(base, pb, q), v[q]);
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q) store(l, base + q * ST, v[q]);
        }
    }
}

// shared-memory load/store of `lines` (line l at lines + l * N)
struct SmemIO {
    static constexpr bool kSlots = true;  // line(l) + slot: pstage_io forms the slots itself
    ulonglong2* lines;
    int n;
    __device__ __forceinline__ ulonglong2* line(int l) const { return lines + l * n; }
    __device__ __forceinline__ PC operator()(int l, int p) const { return ld_pc(lines + l * n + psw(p)); }
    __device__ __forceinline__ void operator()(int l, int p, PC v) const { st_pc(lines + l * n + psw(p), v); }
};

// stages [S, E) in shared memory (DIF ascending, DIT descending), a barrier after each
template <int N, int S, int E, int DIR, int NT = kThreads, typename TW>
__device__ __forceinline__ void pdif_range(ulonglong2* lines, int nl, TW tw) {
    if constexpr (S < E) {
        const SmemIO io{lines, N};
        pstage_io<N, S, DIR, false, NT>(nl, tw, io, io);
        __syncthreads();
        pdif_range<N, S + 1, E, DIR, NT>(lines, nl, tw);
    }
}
template <int N, int S, int E, int DIR, int NT = kThreads, typename TW>
__device__ __forceinline__ void pdit_range(ulonglong2* lines, int nl, TW tw) {
    if constexpr (S > E) {
        const SmemIO io{lines, N};
        pstage_io<N, S - 1, DIR, true, NT>(nl, tw, io, io);
        __syncthreads();
        pdit_range<N, S - 1, E, DIR, NT>(lines, nl, tw);
    }
}

// DIT stages S - 1 down to E of the lines an IO object reaches (load(l, p) / store(l, p, v) for
// line l < nl), a barrier after each
template <int N, int S, int E, int DIR, int NT, typename IO, typename TW>
__device__ __forceinline__ void pdit_range_io(const IO& io, int nl, TW tw) {
    if constexpr (S > E) {
        pstage_io<N, S - 1, DIR, true, NT>(nl, tw, io, io);
        __syncthreads();
        pdit_range_io<N, S - 1, E, DIR, NT>(io, nl, tw);
    }
}

// host: per-stage twiddles w_L^j (forward sign) as float2; the kernels form w^(j q) from them
template <int N>
void pair_twiddles_host(float* out /* 2 * twsz floats */) {
    constexpr PPlan pp = PairPlan<N>::c;
    int L = N;
    for (int s = 0; s < pp.m; ++s) {
        const int R = pp.r[s], ST = pp.s[s];
        if (L > R) {
            for (int j = 0; j < ST; ++j) {
                const double a = -2.0 * M_PI * static_cast<double>(j) / L;
                out[2 * (pp.twoff[s] + j)] = static_cast<float>(cos(a));
                out[2 * (pp.twoff[s] + j) + 1] = static_cast<float>(sin(a));
            }
        }
        L /= R;
    }
}

// bring [p, p + bytes) into L2 ahead of use: the CTA's threads stride over 128-byte lines
__device__ __forceinline__ void prefetch_l2(const void* p, size_t bytes) {
    const char* c = static_cast<const char*>(p);
    for (size_t off = static_cast<size_t>(threadIdx.x) * 128; off < bytes; off += static_cast<size_t>(kThreads) * 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(c + off));
}

// wave number of natural index y on a line of N, and its active-mode index
__device__ __forceinline__ int pky_of_y(int y, int n) { return y < n / 2 ? y : y - n; }

// ---------------------------------------------------------------------------
// column inverse: state -> I1   (grid: column-pair tiles x n_in x batch)
// ---------------------------------------------------------------------------
template <int NY>
__global__ void __launch_bounds__(kThreads) pcol_inverse(const StepPlan P, const MemberInfo* __restrict__ members,
                                                         const float2* __restrict__ state, ulonglong2* __restrict__ i1,
                                                         const float2* __restrict__ tw) {
    if (!members[blockIdx.z].active) return;
    constexpr int CP = kPairMaxN / NY;
    constexpr PPlan pp = PairPlan<NY>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ulonglong2* lines = reinterpret_cast<ulonglong2*>(smem_raw);  // [CP][NY]
    const int t0 = blockIdx.x * CP, slot = blockIdx.y, b = blockIdx.z;
    const int kyn = P.kyn, half = P.nay / 2;
    const size_t fstride = static_cast<size_t>(P.hx) * kyn;
    const float2* src = state + (static_cast<size_t>(b) * P.nfields + P.in_field[slot]) * fstride;
    for (int e = threadIdx.x; e < CP * kyn; e += kThreads) {
        const int c = fdiv(e, P.div_kyn), j = e - c * kyn;
        const int ky = ky_of_j(j, P.nay);
        const int gx = 2 * (t0 + c);
        const float2 a = src[static_cast<size_t>(gx) * kyn + j], a1 = src[static_cast<size_t>(gx + 1) * kyn + j];
        st_pc(lines + c * NY + psw(ppos<NY>(ky >= 0 ? ky : ky + NY)), pc_make(a, a1));
    }
    const int npad = NY - kyn;  // natural y in [Na/2, NY - Na/2]
    for (int e = threadIdx.x; e < CP * npad; e += kThreads) {
        const int c = e / npad, y = half + (e - c * npad);
        st_pc(lines + c * NY + psw(ppos<NY>(y)), pc_zero());
    }
    __syncthreads();
    pdit_range<NY, pp.m, 1, +1>(lines, CP, tw);
    const u64 sc = f2_splat(static_cast<float>(P.inv_scale));
    ulonglong2* dst = i1 + ((static_cast<size_t>(b) * P.n_in + slot) * P.ntiles + t0) * static_cast<size_t>(NY);
    pstage_io<NY, 0, +1, true>(CP, tw, SmemIO{lines, NY}, [&](int l, int p, PC v) {
        st_stream(dst + static_cast<size_t>(l) * NY + p, make_ulonglong2(f2_mul(v.re, sc), f2_mul(v.im, sc)));
    });
}

// ---------------------------------------------------------------------------
// row pass: I1 -> x-inverse (DIF) -> products -> x-forward (DIT) -> I2
// (grid: NY / 2 / RP row-pair groups x batch).  Shared memory: the input
// pair-lines of all RP row pairs, then one work pair-line per row pair.
// ---------------------------------------------------------------------------
// value of slot s at slot index sp of a row pair's inputs: (row y0, row y0 + 1)
__device__ __forceinline__ float2 pin(const ulonglong2* in, int nx, int s, int sp) {
    const ulonglong2 e = in[(s >> 1) * nx + sp];
    return (s & 1) ? make_float2(f2_hi(e.x), f2_hi(e.y)) : make_float2(f2_lo(e.x), f2_lo(e.y));
}

// products of one output pair of the row pass (two outputs per pair-line), evaluated at one
// position of a row pair's physical input lines: `in` is the row pair's first input line, `sp`
// the position's swizzled slot.  Each product is a combination of the terms psi^3, psi vx,
// psi vy, vx, vy, jx vx, jx vy, jy vy (fcalculator.cc:226-239, 366-367, 447-451,
// model_free_energy_phi4.cc:47-55) with per-output coefficients, or, outside the canonical
// input layouts, product_value per row.
struct RowProduct {
    int ka, aa, kb, ab, psa, psb, mode;
    bool need_j, use_psi;
    float inv_rho0;
    u64 IR0;
    int pi;                        // output pair: coefficient q is P.rp_coef[pi][q] (rp_coef below)
};

__device__ __forceinline__ RowProduct row_product(const StepPlan& P, int pi, float inv_rho0) {
    RowProduct R;
    const int oa = P.rp_a[pi], ob = P.rp_b[pi];
    R.ka = P.out_kind[oa];
    R.aa = P.out_arg[oa];
    R.kb = ob >= 0 ? P.out_kind[ob] : -1;
    R.ab = ob >= 0 ? P.out_arg[ob] : 0;
    R.psa = (R.ka == OUT_MU || R.ka == OUT_PSIVX || R.ka == OUT_PSIVY) ? P.in_slot[1 + R.aa] : -1;
    R.psb = (R.kb == OUT_MU || R.kb == OUT_PSIVX || R.kb == OUT_PSIVY) ? P.in_slot[1 + R.ab] : -1;
    R.need_j = (R.ka != OUT_MU) || (R.kb >= 0 && R.kb != OUT_MU);
    R.pi = pi;
    R.use_psi = R.psa >= 0 || R.psb >= 0;
    R.mode = P.rp_mode[pi];
    R.inv_rho0 = inv_rho0;
    R.IR0 = f2_splat(inv_rho0);
    return R;
}

// (jx, jy) and (vx, vy) of the canonical layout at one position: J = ((jx, jy) of row y0,
// (jx, jy) of row y0 + 1), V likewise
struct JV {
    ulonglong2 J, V;
};
template <int NX>
__device__ __forceinline__ JV row_jv(const StepPlan& P, const RowProduct& R, const ulonglong2* in, int sp) {
    const ulonglong2 J = in[P.rp_jline * NX + sp];
    const ulonglong2 V = P.rp_vline >= 0 ? in[P.rp_vline * NX + sp] : make_ulonglong2(f2_mul(J.x, R.IR0), f2_mul(J.y, R.IR0));
    return JV{J, V};
}

// canonical input roles: psi of A and B from their slots, (jx, jy) and (vx, vy) from get_jv()
// (read where a product needs them)
template <int NX, typename GetJV>
__device__ __forceinline__ PC row_product_canon(const StepPlan& P, const RowProduct& R, const ulonglong2* in, int sp, GetJV&& get_jv) {
    // coefficient q of the pair (A, B), read where a product uses it
    auto C = [&](int q) { return f2_pack(P.rp_coef[R.pi][q][0], P.rp_coef[R.pi][q][1]); };
    const int mode = R.mode;
    if (mode != 0) {  // outputs that are elementwise products of whole lines
        if (mode == 1 || mode == 2) {
            const JV jv = get_jv();
            const ulonglong2 J = jv.J, V = jv.V;
            if (mode == 1) return PC{V.x, V.y};
            return PC{f2_mul(J.x, V.x), f2_mul(J.y, V.y)};
        }
        const ulonglong2 S = in[(R.psa >> 1) * NX + sp];
        if (mode == 3) {
            const u64 q0 = f2_mul(f2_mul(S.x, S.x), f2_mul(S.x, C(0)));
            const u64 q1 = f2_mul(f2_mul(S.y, S.y), f2_mul(S.y, C(0)));
            return PC{q0, q1};
        }
        const ulonglong2 V = get_jv().V;
        const u64 v0 = mode == 4 ? f2_splat(f2_lo(V.x)) : f2_splat(f2_hi(V.x));
        const u64 v1 = mode == 4 ? f2_splat(f2_lo(V.y)) : f2_splat(f2_hi(V.y));
        const u64 cc = C(mode == 4 ? 1 : 2);
        return PC{f2_mul(f2_mul(S.x, cc), v0), f2_mul(f2_mul(S.y, cc), v1)};
    }
    u64 out[2] = {0ull, 0ull};
    float jxr[2] = {0.f, 0.f}, jyr[2] = {0.f, 0.f}, vxr[2] = {0.f, 0.f}, vyr[2] = {0.f, 0.f};
    if (R.need_j) {
        const JV jv = get_jv();
        const ulonglong2 J = jv.J, V = jv.V;
        jxr[0] = f2_lo(J.x); jyr[0] = f2_hi(J.x); jxr[1] = f2_lo(J.y); jyr[1] = f2_hi(J.y);
        vxr[0] = f2_lo(V.x); vyr[0] = f2_hi(V.x); vxr[1] = f2_lo(V.y); vyr[1] = f2_hi(V.y);
    }
    float2 pa = make_float2(0.f, 0.f), pb = pa;
    if (R.psa >= 0) pa = pin(in, NX, R.psa, sp);
    if (R.psb >= 0) pb = pin(in, NX, R.psb, sp);
#pragma unroll
    for (int row = 0; row < 2; ++row) {
        const u64 VX = f2_splat(vxr[row]), VY = f2_splat(vyr[row]);
        const u64 JX = f2_splat(jxr[row]), JY = f2_splat(jyr[row]);
        u64 o = f2_fma(C(4), VY, f2_mul(C(3), VX));                          // c3 vx + c4 vy
        o = f2_fma(f2_mul(C(5), JX), VX, o);                                 // + c5 jx vx
        o = f2_fma(f2_fma(C(6), JX, f2_mul(C(7), JY)), VY, o);               // + (c6 jx + c7 jy) vy
        if (R.use_psi) {
            const u64 PS = row ? f2_pack(pa.y, pb.y) : f2_pack(pa.x, pb.x);
            u64 in2 = f2_fma(C(1), VX, f2_mul(C(2), VY));                    // c1 vx + c2 vy
            in2 = f2_fma(f2_mul(C(0), PS), PS, in2);                         // + c0 psi^2
            o = f2_fma(PS, in2, o);                                          // psi (...)
        }
        out[row] = o;
    }
    return PC{out[0], out[1]};
}
template <int NX>
__device__ __forceinline__ PC row_product_canon(const StepPlan& P, const RowProduct& R, const ulonglong2* in, int sp) {
    return row_product_canon<NX>(P, R, in, sp, [&] { return row_jv<NX>(P, R, in, sp); });
}

// any input layout: product_value per row (rho replaced by 1 / rho in compressible dynamics)
template <int NX>
__device__ __forceinline__ PC row_product_general(const StepPlan& P, const RowProduct& R, const ulonglong2* in, int sp) {
    const int s_rho = P.in_slot[0];
    const int s_jx = P.in_slot[P.nop + 1];
    const int s_jy = P.in_slot[P.nop + 2];
    const bool comp = (P.mode == 0);
    float2 jx = make_float2(0.f, 0.f), jy = jx, vx = jx, vy = jx;
    if (R.need_j) {
        jx = pin(in, NX, s_jx, sp);
        jy = pin(in, NX, s_jy, sp);
        if (comp) {
            const float2 ir = pin(in, NX, s_rho, sp);
            vx = make_float2(jx.x * ir.x, jx.y * ir.y);
            vy = make_float2(jy.x * ir.x, jy.y * ir.y);
        } else {
            vx = make_float2(jx.x * R.inv_rho0, jx.y * R.inv_rho0);
            vy = make_float2(jy.x * R.inv_rho0, jy.y * R.inv_rho0);
        }
    }
    const float2 pa = R.psa >= 0 ? pin(in, NX, R.psa, sp) : make_float2(0.f, 0.f);
    const float2 pb = R.psb >= 0 ? pin(in, NX, R.psb, sp) : make_float2(0.f, 0.f);
    float a0 = product_value<float>(P, R.ka, R.aa, pa.x, jx.x, jy.x, vx.x, vy.x);
    float a1 = product_value<float>(P, R.ka, R.aa, pa.y, jx.y, jy.y, vx.y, vy.y);
    float b0 = 0.f, b1 = 0.f;
    if (R.kb >= 0) {
        b0 = product_value<float>(P, R.kb, R.ab, pb.x, jx.x, jy.x, vx.x, vy.x);
        b1 = product_value<float>(P, R.kb, R.ab, pb.y, jx.y, jy.y, vx.y, vy.y);
    }
    if (P.fe_plugin) {  // plugin styles: mu from every order parameter at the position
        auto get = [&](int s) { return pin(in, NX, s, sp); };
        if (R.ka == OUT_MU) plugin_mu_rows<float>(P, R.aa, get, a0, a1);
        if (R.kb == OUT_MU) plugin_mu_rows<float>(P, R.ab, get, b0, b1);
    }
    return PC{f2_pack(a0, b0), f2_pack(a1, b1)};
}

// velocity inputs after the x-inverse of a row pair's input lines (`inl`, `nl` row pairs of
// `nip` lines of NX).  Canonical layout: (rho, jx), (jy, -) become (jx, jy), (vx, vy)
// (compressible, with the zero-density check of fcalculator_workspace.cc:122-133); otherwise
// rho is replaced by 1 / rho in place.  Threads tid < nthreads stride over the positions.
template <int NX>
__device__ __forceinline__ void row_velocity_prep(const StepPlan& P, ulonglong2* inl, int nl, int nip, int tid, int nthreads, int* err) {
    int bad = 0;
    const int s_rho = P.in_slot[0];
    if (P.rp_prep) {
        const int m = P.rp_jline;
        for (int e = tid; e < nl * NX; e += nthreads) {
            const int r = e / NX, x = e - r * NX;
            ulonglong2* pj = inl + (static_cast<size_t>(r) * nip + m) * NX + x;
            const ulonglong2 rj = pj[0], jy = pj[NX];
            const float r0 = f2_lo(rj.x), r1 = f2_lo(rj.y);
            if (r0 == 0.f || r1 == 0.f) bad = 1;
            const u64 ir = f2_pack(1.f / r0, 1.f / r1);                       // (1/rho_row0, 1/rho_row1)
            const u64 jx = f2_pack(f2_hi(rj.x), f2_hi(rj.y)), jyv = f2_pack(f2_lo(jy.x), f2_lo(jy.y));
            const u64 vx = f2_mul(jx, ir), vy = f2_mul(jyv, ir);              // per row
            pj[0] = make_ulonglong2(f2_pack(f2_lo(jx), f2_lo(jyv)), f2_pack(f2_hi(jx), f2_hi(jyv)));
            pj[NX] = make_ulonglong2(f2_pack(f2_lo(vx), f2_lo(vy)), f2_pack(f2_hi(vx), f2_hi(vy)));
        }
    } else {
        for (int e = tid; e < nl * NX; e += nthreads) {
            const int r = e / NX, x = e - r * NX;
            ulonglong2* pe = inl + (static_cast<size_t>(r) * nip + (s_rho >> 1)) * NX + x;
            ulonglong2 v = *pe;
            const int h = s_rho & 1;
            const float r0 = h ? f2_hi(v.x) : f2_lo(v.x), r1 = h ? f2_hi(v.y) : f2_lo(v.y);
            if (r0 == 0.f || r1 == 0.f) bad = 1;
            const float i0 = 1.f / r0, i1v = 1.f / r1;
            if (h) { v.x = f2_pack(f2_lo(v.x), i0); v.y = f2_pack(f2_lo(v.y), i1v); }
            else { v.x = f2_pack(i0, f2_hi(v.x)); v.y = f2_pack(i1v, f2_hi(v.y)); }
            *pe = v;
        }
    }
    if (bad) atomicOr(err, ERR_ZERO_DENSITY);
}

// Z staging of one item (input pair-line ip, tile t) of a row pair (rows y0, y0 + 1): the two
// slots' I1 values at columns k = 2t, 2t + 1 (pz_load), then Z[k] = X0[k] + i X1[k] and the
// Hermitian mirror Z[N - k] = conj X0[k] + i conj X1[k], kx = 0 keeping the real parts only
// (pz_store).  Callers load kZBatch items per thread before storing any, so that many I1 reads
// are in flight at once.
constexpr int kZBatch = 4;
struct ZItem {
    ulonglong2 a0, a1, b0, b1;
};
__device__ __forceinline__ ZItem pz_load(const ulonglong2* i1m, size_t plane, int npy, int n_in, int ip, int t, int y0) {
    const int sa = 2 * ip, sb = 2 * ip + 1;
    const ulonglong2* pa = i1m + static_cast<size_t>(sa) * plane + static_cast<size_t>(t) * npy + y0;
    ZItem z;
    ld_stream2(pa, z.a0, z.a1);
    z.b0 = z.b1 = make_ulonglong2(0ull, 0ull);
    if (sb < n_in) {
        const ulonglong2* pb = i1m + static_cast<size_t>(sb) * plane + static_cast<size_t>(t) * npy + y0;
        ld_stream2(pb, z.b0, z.b1);
    }
    return z;
}
// the same for a packed plan: slot 0 of two row pairs (rows ya, ya + 1 and yb, yb + 1) as the
// two halves
__device__ __forceinline__ ZItem pz_load_rows(const ulonglong2* i1m, int npy, int t, int ya, int yb) {
    const ulonglong2* p = i1m + static_cast<size_t>(t) * npy;
    ZItem z;
    ld_stream2(p + ya, z.a0, z.a1);
    ld_stream2(p + yb, z.b0, z.b1);
    return z;
}
template <int NX>
__device__ __forceinline__ void pz_store(ulonglong2* line, int t, const ZItem& z) {
#pragma unroll
    for (int w = 0; w < 2; ++w) {
        const int k = 2 * t + w;
        // X0, X1 of fields a and b at column k
        float xa0r = w ? f2_hi(z.a0.x) : f2_lo(z.a0.x), xa0i = w ? f2_hi(z.a0.y) : f2_lo(z.a0.y);
        float xa1r = w ? f2_hi(z.a1.x) : f2_lo(z.a1.x), xa1i = w ? f2_hi(z.a1.y) : f2_lo(z.a1.y);
        float xb0r = w ? f2_hi(z.b0.x) : f2_lo(z.b0.x), xb0i = w ? f2_hi(z.b0.y) : f2_lo(z.b0.y);
        float xb1r = w ? f2_hi(z.b1.x) : f2_lo(z.b1.x), xb1i = w ? f2_hi(z.b1.y) : f2_lo(z.b1.y);
        if (k == 0) { xa0i = 0.f; xa1i = 0.f; xb0i = 0.f; xb1i = 0.f; }
        st_pc(line + psw(k), PC{f2_pack(xa0r - xa1i, xb0r - xb1i), f2_pack(xa0i + xa1r, xb0i + xb1r)});
        if (k > 0) st_pc(line + psw(NX - k), PC{f2_pack(xa0r + xa1i, xb0r + xb1i), f2_pack(xa1r - xa0i, xb1r - xb0i)});
    }
}

// row pass, first part: Z staging of the nip input pair-lines of a block's RP row pairs (from
// pair0) and their x-inverse in place (DIF stages in shared memory, a barrier after each).  A
// packed plan (P.rp_pack, one input slot) stages RP / 2 lines, line r holding row pairs 2r and
// 2r + 1 as its two halves.
template <int NX, int NT = kThreads, typename TW>
__device__ __forceinline__ void prow_inputs(const StepPlan& P, const ulonglong2* __restrict__ i1m, size_t plane, ulonglong2* inl, int nip,
                                            int pair0, TW tw) {
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
    const int npy = P.npy, hx = P.hx, hp = hx >> 1;
    const bool pack = P.rp_pack;
    const int nlr = pack ? RP / 2 : RP;  // staged lines per input pair-line slot
    // Z[k] = X0[k] + i X1[k] (rows y0, y0 + 1) with the Hermitian mirror Z[N - k]
    // = conj X0[k] + i conj X1[k]; kx = 0 keeps the real parts only
    const int per_r = nip * hp, nz = nlr * per_r;
    for (int e0 = threadIdx.x; e0 < nz; e0 += kZBatch * NT) {
        ZItem z[kZBatch];
#pragma unroll
        for (int u = 0; u < kZBatch; ++u) {
            const int e = e0 + u * NT;
            if (e < nz) {
                const int r = e / per_r, rem = e - r * per_r;
                const int ip = rem / hp, t = rem - ip * hp;
                z[u] = pack ? pz_load_rows(i1m, npy, t, 2 * (pair0 + 2 * r), 2 * (pair0 + 2 * r + 1))
                            : pz_load(i1m, plane, npy, P.n_in, ip, t, 2 * (pair0 + r));
            }
        }
#pragma unroll
        for (int u = 0; u < kZBatch; ++u) {
            const int e = e0 + u * NT;
            if (e < nz) {
                const int r = e / per_r, rem = e - r * per_r;
                const int ip = rem / hp, t = rem - ip * hp;
                pz_store<NX>(inl + (static_cast<size_t>(r) * nip + ip) * NX, t, z[u]);
            }
        }
    }
    const int nzero = NX - 2 * hx + 1;  // k in [hx, NX - hx]
    const int per_z = nip * nzero;
    for (int e = threadIdx.x; e < nlr * per_z; e += NT) {
        const int l = e / nzero, k = hx + (e - l * nzero);
        st_pc(inl + static_cast<size_t>(l) * NX + psw(k), pc_zero());
    }
    __syncthreads();
    pdif_range<NX, 0, pp.m, +1, NT>(inl, nlr * nip, tw);
}

// row pass, last part: the untangling of transformed output pairs into I2.  One or two (nl)
// output pairs of RP row pairs: pair q's line of row pair r at Wq.line + r * Wq.stride, its
// outputs Wq.oa, Wq.ob (-1: none).  G0[k] = (Z[k] + conj Z[N-k]) / 2 (row y0),
// G1[k] = -i (Z[k] - conj Z[N-k]) / 2 (row y0 + 1), for kx = k < Hx.
struct OutLine {
    const ulonglong2* line;
    size_t stride;
    int oa, ob;
};
template <int NX, int NT = kThreads>
__device__ __forceinline__ void prow_untangle(const StepPlan& P, int nl, const OutLine W0, const OutLine W1, ulonglong2* __restrict__ i2m,
                                              size_t plane, int pair0) {
    constexpr int RP = kPairMaxN / NX;
    const int npy = P.npy, hp = P.hx >> 1;
    const u64 HALF = f2_splat(0.5f);
    // packed plan: line r holds row pairs 2r and 2r + 1 of the one output (halves a and b)
    const bool pack = P.rp_pack;
    const int per_q = (pack ? RP / 2 : RP) * hp;
#pragma unroll 2
    for (int e = threadIdx.x; e < nl * per_q; e += NT) {
        const bool q = e >= per_q;
        const OutLine W = q ? W1 : W0;
        const int rem = q ? e - per_q : e;
        const int r = rem / hp, t = rem - r * hp;
        const ulonglong2* z = W.line + static_cast<size_t>(r) * W.stride;
        const int y0 = 2 * (pair0 + (pack ? 2 * r : r));
        u64 g0r[2], g0i[2], g1r[2], g1i[2];
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            const int k = 2 * t + w;
            const PC zk = ld_pc(z + psw(k));
            const PC zn = ld_pc(z + psw(k == 0 ? 0 : NX - k));
            g0r[w] = f2_mul(f2_add(zk.re, zn.re), HALF);
            g0i[w] = f2_mul(f2_sub(zk.im, zn.im), HALF);
            g1r[w] = f2_mul(f2_add(zk.im, zn.im), HALF);   //  (d.im) / 2, d = Z[k] - conj Z[N-k]
            g1i[w] = f2_mul(f2_sub(zn.re, zk.re), HALF);   // -(d.re) / 2
        }
        ulonglong2* qa = i2m + static_cast<size_t>(W.oa) * plane + static_cast<size_t>(t) * npy + y0;
        st_stream2(qa, make_ulonglong2(f2_pack(f2_lo(g0r[0]), f2_lo(g0r[1])), f2_pack(f2_lo(g0i[0]), f2_lo(g0i[1]))),
                   make_ulonglong2(f2_pack(f2_lo(g1r[0]), f2_lo(g1r[1])), f2_pack(f2_lo(g1i[0]), f2_lo(g1i[1]))));
        if (W.ob >= 0 || pack) {
            ulonglong2* qb = pack ? qa + 2 : i2m + static_cast<size_t>(W.ob) * plane + static_cast<size_t>(t) * npy + y0;
            st_stream2(qb, make_ulonglong2(f2_pack(f2_hi(g0r[0]), f2_hi(g0r[1])), f2_pack(f2_hi(g0i[0]), f2_hi(g0i[1]))),
                       make_ulonglong2(f2_pack(f2_hi(g1r[0]), f2_hi(g1r[1])), f2_pack(f2_hi(g1i[0]), f2_hi(g1i[1]))));
        }
    }
}

// MINB: blocks per SM the registers are budgeted for (2; 3 where shared memory allows more blocks,
// e.g. one input pair-line on rows of <= 768 points)
template <int NX, int MINB = 2>
__global__ void __launch_bounds__(kThreads, MINB) prow_pass(const StepPlan P, const MemberInfo* __restrict__ members,
                                                      const ulonglong2* __restrict__ i1, ulonglong2* __restrict__ i2,
                                                      const float2* __restrict__ tw, const double* __restrict__ rho0_member,
                                                      int* __restrict__ err) {
    if (!members[blockIdx.y].active) return;
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nip = (P.n_in + 1) >> 1;
    ulonglong2* inl = reinterpret_cast<ulonglong2*>(smem_raw);          // [RP][nip][NX]
    ulonglong2* work = inl + static_cast<size_t>(RP) * nip * NX;        // [RP][NX]
    const int b = blockIdx.y;
    const int pair0 = blockIdx.x * RP;
    const size_t plane = static_cast<size_t>(P.ntiles) * P.npy;         // one slot of I1 / I2 (pair elements)
    const ulonglong2* i1m = i1 + static_cast<size_t>(b) * P.n_in * plane;
    ulonglong2* i2m = i2 + static_cast<size_t>(b) * P.n_out * plane;

    // 1. inputs: Z staging and x-inverse
    prow_inputs<NX>(P, i1m, plane, inl, nip, pair0, tw);

    // 2. velocity inputs (compressible: v = j / rho with the zero-density check; otherwise
    //    v = j / rho0 in the products)
    const bool comp = (P.mode == 0);
    const float inv_rho0 = (P.need_v && !comp) ? static_cast<float>(1.0 / rho0_member[b]) : 0.f;
    if (P.need_v && comp) {
        row_velocity_prep<NX>(P, inl, RP, nip, threadIdx.x, kThreads, err);
        __syncthreads();
    }

    // 3. per output pair: products fused into the first DIT stage, the rest of
    //    the forward transform, then the untangling of the two rows (kx < Hx)
    const int nl = P.rp_pack ? RP / 2 : RP;  // lines per input / output pair-line
    for (int pi = 0; pi < P.rp_n; ++pi) {
        const RowProduct R = row_product(P, pi, inv_rho0);
        auto product_canon = [&](int r, int p) -> PC { return row_product_canon<NX>(P, R, inl + static_cast<size_t>(r) * nip * NX, psw(p)); };
        auto product = [&](int r, int p) -> PC { return row_product_general<NX>(P, R, inl + static_cast<size_t>(r) * nip * NX, psw(p)); };
        const SmemIO wio{work, NX};
        if (P.rp_canon) pstage_io<NX, pp.m - 1, -1, true>(nl, tw, product_canon, wio);
        else pstage_io<NX, pp.m - 1, -1, true>(nl, tw, product, wio);
        __syncthreads();
        pdit_range<NX, pp.m - 1, 0, -1>(work, nl, tw);
        const OutLine W{work, static_cast<size_t>(NX), P.rp_a[pi], P.rp_b[pi]};
        prow_untangle<NX>(P, 1, W, W, i2m, plane, pair0);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// column forward + epilogue (grid: column-pair tiles x groups x batch).
// Shared memory: CP work pair-lines, then per-mode arrays [CP][Kp] (accumulators / new
// values), two columns per element, Kp = Ky rounded up to a multiple of 8: acc0 for every
// group (psi, jx or rho), acc1 for the momentum group's jy, acc2 for its rho when the density
// shares the momentum group; the launch provides the arrays the plan's groups use.
// ---------------------------------------------------------------------------
// slot of mode j in a column's per-mode row.  The last DIF stage (and the first stage of the
// fused inverse) reaches the modes in digit-reversed order: at 384 points and up the eight
// threads of a quarter warp then touch modes 3 * 8 ... 3 * 64 apart, all in one 16-byte bank
// group of a plain row, so there the low three bits are XORed with bits 3..5.  Eight
// consecutive modes from a multiple of 8 stay in their own eight slots either way.
template <int NY>
__device__ __forceinline__ int pmode_slot(int c, int j, int kyp) {
    return c * kyp + (NY >= 384 ? (j ^ ((j >> 3) & 7)) : j);
}

// blocks per SM the column forward is compiled for: its 41-74 KB of shared memory allow three,
// and at 384 points and up the register budget of three (80) holds it without spilling more than
// 40 B
template <int NY>
__host__ __device__ constexpr int pcol_forward_blocks() { return NY >= 384 ? 3 : 2; }

// MINB: blocks per SM the registers are budgeted for (pcol_forward_blocks, or 4 where the plan's
// per-mode arrays are one per column: order-parameter groups only)
template <int NY, int MINB = pcol_forward_blocks<NY>()>
__global__ void __launch_bounds__(kThreads, MINB) pcol_forward(const StepPlan P, const StageArgs<float> A,
                                                                                 const float2* __restrict__ tw) {
    constexpr int CP = kPairMaxN / NY;
    constexpr PPlan pp = PairPlan<NY>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kyn = P.kyn, kyp = P.kyp, nay = P.nay, half = nay / 2;
    ulonglong2* lines = reinterpret_cast<ulonglong2*>(smem_raw);       // [CP][NY]
    ulonglong2* acc0 = lines + CP * NY;                                  // [CP][Kp], slots pmode_slot
    ulonglong2* acc1 = acc0 + CP * kyp;
    ulonglong2* acc2 = acc1 + CP * kyp;
    // groups in the plan's launch order: momentum (the heaviest: five or six product fields and
    // two or three updated fields) first, so that the lighter blocks fill the tail
    const int t0 = blockIdx.x * CP, grp = P.group_order[blockIdx.y], b = blockIdx.z;
    const int gkind = P.group_kind[grp], alpha = P.group_alpha[grp];
    const bool comp = (P.mode == 0);
    const MemberInfo mi = A.members[b];
    if (!mi.active) return;
    const size_t fstride = static_cast<size_t>(P.hx) * kyn;
    const float kxu = static_cast<float>(P.kx_unit), kyu = static_cast<float>(P.ky_unit);
    const size_t plane = static_cast<size_t>(P.ntiles) * NY;

    // the epilogue's state reads (this CTA's columns of the group's fields) start
    // towards L2 now and land while the products are transformed
    {
        const size_t span = static_cast<size_t>(2 * CP) * kyn * sizeof(float2);
        const size_t col0 = static_cast<size_t>(b) * P.nfields * fstride + static_cast<size_t>(2 * t0) * kyn;
        const bool base_used = A.wb != 0.0 && !A.det_mode;
        auto fetch = [&](int f) {
            prefetch_l2(A.cur + col0 + static_cast<size_t>(f) * fstride, span);
            if (base_used) prefetch_l2(A.base + col0 + static_cast<size_t>(f) * fstride, span);
        };
        if (gkind == GROUP_PSI) fetch(1 + alpha);
        else {
            fetch(P.nop + 1);
            fetch(P.nop + 2);
            if (gkind == GROUP_RHO || (comp && !P.rho_split)) fetch(0);
        }
    }
    for (int e = threadIdx.x; e < CP * kyp; e += kThreads) {
        st_pc(acc0 + e, pc_zero());
        if (gkind == GROUP_MOMENTUM) st_pc(acc1 + e, pc_zero());  // the only group with a second array
    }

    // y-forward of each product field of the group (DIF; global tile loads fused
    // into stage 0, accumulation into the RHS fused into the last stage).  The
    // accumulation works on both columns at once: with v the transformed field,
    // a0 += alpha0 v + beta0 (-i v) and a1 += alpha1 v + beta1 (-i v), the real
    // factors (one per column) given by the field's kind (fcalculator.cc:244-272,
    // 374-396, 475-492).
    const int ngo = P.group_nout[grp];
    const float mob = gkind == GROUP_PSI ? static_cast<float>(P.mobility[alpha]) : 0.f;
    const float eta = static_cast<float>(P.eta), zeta = static_cast<float>(P.zeta);
    for (int go = 0; go < ngo; ++go) {
        const int o = P.group_out[grp][go];
        const int kind = P.out_kind[o];
        const ulonglong2* src = reinterpret_cast<const ulonglong2*>(A.i2) + (static_cast<size_t>(b) * P.n_out + o) * plane +
                                static_cast<size_t>(t0) * NY;
        __syncthreads();  // the previous field's last stage is done with the lines
        pstage_io<NY, 0, -1, false>(CP, tw, [&](int l, int p) { const ulonglong2 v = ld_stream(src + static_cast<size_t>(l) * NY + p); return PC{v.x, v.y}; },
                                    SmemIO{lines, NY});
        __syncthreads();
        pdif_range<NY, 1, pp.m - 1, -1>(lines, CP, tw);
        pstage_io<NY, pp.m - 1, -1, false>(CP, tw, SmemIO{lines, NY}, [&](int l, int p, PC v) {
            const int ky = pky_of_y(ppinv<NY>(p), NY);
            if (ky >= half || ky <= -half) return;
            const int j = ky >= 0 ? ky : ky + kyn;
            const float kyv = kyu * static_cast<float>(ky);
            const float gx0 = static_cast<float>(2 * (t0 + l));
            const u64 KX = f2_pack(kxu * gx0, kxu * (gx0 + 1.f));
            const u64 KY = f2_splat(kyv);
            const int sj = pmode_slot<NY>(l, j, kyp);
            ulonglong2* q0 = acc0 + sj;
            ulonglong2* q1 = acc1 + sj;
            // -i v = (v.im, -v.re): a += beta (-i v) -> a.re += beta v.im, a.im -= beta v.re
            switch (kind) {
                case OUT_MU: {  // a0 += -M k^2 v
                    const u64 al = f2_mul(f2_fma(KX, KX, f2_mul(KY, KY)), f2_splat(-mob));
                    ulonglong2 a = *q0;
                    a.x = f2_fma(al, v.re, a.x);
                    a.y = f2_fma(al, v.im, a.y);
                    *q0 = a;
                    break;
                }
                case OUT_PSIVX: case OUT_PSIVY: case OUT_PXX: {  // a0 += k (-i v)
                    const u64 be = kind == OUT_PSIVY ? KY : KX;
                    ulonglong2 a = *q0;
                    a.x = f2_fma(be, v.im, a.x);
                    a.y = f2_sub(a.y, f2_mul(be, v.re));
                    *q0 = a;
                    break;
                }
                case OUT_GRAD: {  // a0 += v
                    ulonglong2 a = *q0;
                    a.x = f2_add(a.x, v.re);
                    a.y = f2_add(a.y, v.im);
                    *q0 = a;
                    break;
                }
                case OUT_VX: case OUT_VY: {
                    // VX: a0 += -((eta + zeta) kx^2 + eta ky^2) v, a1 += -zeta kx ky v
                    // VY: a0 += -zeta kx ky v, a1 += -(eta kx^2 + (eta + zeta) ky^2) v
                    const u64 kx2 = f2_mul(KX, KX), ky2 = f2_mul(KY, KY), kxy = f2_mul(KX, KY);
                    const u64 cross = f2_mul(kxy, f2_splat(-zeta));
                    const u64 diag = kind == OUT_VX ? f2_fma(kx2, f2_splat(-(eta + zeta)), f2_mul(ky2, f2_splat(-eta)))
                                                    : f2_fma(kx2, f2_splat(-eta), f2_mul(ky2, f2_splat(-(eta + zeta))));
                    const u64 a0c = kind == OUT_VX ? diag : cross, a1c = kind == OUT_VX ? cross : diag;
                    ulonglong2 a = *q0, c = *q1;
                    a.x = f2_fma(a0c, v.re, a.x);
                    a.y = f2_fma(a0c, v.im, a.y);
                    c.x = f2_fma(a1c, v.re, c.x);
                    c.y = f2_fma(a1c, v.im, c.y);
                    *q0 = a;
                    *q1 = c;
                    break;
                }
                case OUT_PXY: {  // a0 += ky (-i v), a1 += kx (-i v)
                    ulonglong2 a = *q0, c = *q1;
                    a.x = f2_fma(KY, v.im, a.x);
                    a.y = f2_sub(a.y, f2_mul(KY, v.re));
                    c.x = f2_fma(KX, v.im, c.x);
                    c.y = f2_sub(c.y, f2_mul(KX, v.re));
                    *q0 = a;
                    *q1 = c;
                    break;
                }
                default: {  // PYY: a1 += ky (-i v)
                    ulonglong2 c = *q1;
                    c.x = f2_fma(KY, v.im, c.x);
                    c.y = f2_sub(c.y, f2_mul(KY, v.re));
                    *q1 = c;
                    break;
                }
            }
        });
    }
    __syncthreads();

    // epilogue per mode (natural order, coalesced state access): results replace the accumulators
    for (int e = threadIdx.x; e < CP * kyp; e += kThreads) {
        const int c = fdiv(e, P.div_kyp), j = e - c * kyp;
        if (j >= kyn) continue;
        const int sj = pmode_slot<NY>(c, j, kyp);
        const int t = t0 + c;
        const size_t mbase = static_cast<size_t>(b) * P.nfields * fstride + static_cast<size_t>(t) * 2 * kyn;
        const PC u0 = ld_pc(acc0 + sj);
        if (gkind == GROUP_PSI) {
            float2 r[2];
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const ModeCtx m = mode_ctx<float>(P, mbase, t, w, j);
                const PsiLoads<float> L = psi_loads<float>(P, A, alpha, m.pos, fstride);
                r[w] = psi_epilogue<float>(P, A, alpha, m, kxu * static_cast<float>(m.gx), kyu * static_cast<float>(m.ky), pc_col(u0, w), mi, L, b);
            }
            st_pc(acc0 + sj, pc_make(r[0], r[1]));
        } else if (gkind == GROUP_RHO) {
            float2 r[2];
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const ModeCtx m = mode_ctx<float>(P, mbase, t, w, j);
                r[w] = rho_epilogue<float>(P, A, m.pos, kxu * static_cast<float>(m.gx), kyu * static_cast<float>(m.ky), fstride);
            }
            st_pc(acc0 + sj, pc_make(r[0], r[1]));
        } else {
            const bool with_rho = comp && !P.rho_split;
            const PC u1 = ld_pc(acc1 + sj);
            float2 r0[2], r1[2], r2[2];
#pragma unroll
            for (int w = 0; w < 2; ++w) {
                const ModeCtx m = mode_ctx<float>(P, mbase, t, w, j);
                const MomLoads<float> L = momentum_loads<float>(P, A, m.pos, fstride);
                const float kx = kxu * static_cast<float>(m.gx), kyv = kyu * static_cast<float>(m.ky);
                r0[w] = pc_col(u0, w);
                r1[w] = pc_col(u1, w);
                momentum_epilogue<float>(P, A, m, kx, kyv, r0[w], r1[w], mi, L, b);
                r2[w] = with_rho ? rho_epilogue<float>(P, A, m.pos, kx, kyv, fstride) : make_float2(0.f, 0.f);
            }
            st_pc(acc0 + sj, pc_make(r0[0], r0[1]));
            st_pc(acc1 + sj, pc_make(r1[0], r1[1]));
            if (with_rho) st_pc(acc2 + sj, pc_make(r2[0], r2[1]));
        }
    }
    __syncthreads();

    // real-symmetry projection of the kx = 0 line (time_integrator.h:70-109): column 0 of tile 0
    const int nres = (gkind != GROUP_MOMENTUM) ? 1 : ((comp && !P.rho_split) ? 3 : 2);
    if (t0 == 0 && !A.det_mode) {
        for (int e = threadIdx.x; e < nres * half; e += kThreads) {
            const int q = e / half, ky = e - q * half;
            ulonglong2* a = (q == 0 ? acc0 : (q == 1 ? acc1 : acc2));
            if (ky == 0) {
                ulonglong2 v = a[0];
                v.y = f2_pack(0.f, f2_hi(v.y));
                a[0] = v;
            } else {
                ulonglong2* ap = a + pmode_slot<NY>(0, ky, kyp);
                ulonglong2* an = a + pmode_slot<NY>(0, kyn - ky, kyp);
                ulonglong2 vp = *ap, vn = *an;
                const float pr = 0.5f * (f2_lo(vp.x) + f2_lo(vn.x)), pi = 0.5f * (f2_lo(vp.y) - f2_lo(vn.y));
                vp.x = f2_pack(pr, f2_hi(vp.x)); vp.y = f2_pack(pi, f2_hi(vp.y));
                vn.x = f2_pack(pr, f2_hi(vn.x)); vn.y = f2_pack(-pi, f2_hi(vn.y));
                *ap = vp;
                *an = vn;
            }
        }
        __syncthreads();
    }

    // state write (per field: psi_alpha, or jx, jy and rho)
    int wfield[3], nwf = 0;
    const ulonglong2* wsrc[3];
    if (gkind == GROUP_PSI) { wfield[nwf] = 1 + alpha; wsrc[nwf++] = acc0; }
    else if (gkind == GROUP_RHO) { wfield[nwf] = 0; wsrc[nwf++] = acc0; }
    else {
        wfield[nwf] = P.nop + 1; wsrc[nwf++] = acc0;
        wfield[nwf] = P.nop + 2; wsrc[nwf++] = acc1;
        if (comp && !P.rho_split) { wfield[nwf] = 0; wsrc[nwf++] = acc2; }
    }
    bool bad = false;
    for (int q = 0; q < nwf; ++q) {
        float2* dst = A.next + static_cast<size_t>(b) * P.nfields * fstride + static_cast<size_t>(wfield[q]) * fstride;
        for (int e = threadIdx.x; e < CP * kyp; e += kThreads) {
            const int c = fdiv(e, P.div_kyp), j = e - c * kyp;
            if (j >= kyn) continue;
            const PC v = ld_pc(wsrc[q] + pmode_slot<NY>(c, j, kyp));
            const size_t gx = static_cast<size_t>(2 * (t0 + c));
            const float2 v0 = pc_col(v, 0), v1 = pc_col(v, 1);
            bad |= nonfinite2(make_float2(v0.x + v0.y, v1.x + v1.y));
            dst[gx * kyn + j] = v0;
            dst[(gx + 1) * kyn + j] = v1;
        }
    }
    report_nonfinite(A.err, bad);

    // y-inverse (DIT) of each new field the next stage transforms: the gather of
    // the new modes from the per-mode arrays is fused into its first stage, the
    // scaled natural-order write of I1 into its last
    if (!A.fused_inverse) return;
    const u64 sc = f2_splat(static_cast<float>(P.inv_scale));
    for (int q = 0; q < nwf; ++q) {
        const int slot = P.in_slot[wfield[q]];
        if (slot < 0) continue;
        const ulonglong2* a = wsrc[q];
        __syncthreads();  // previous field's inverse is done with the lines
        pstage_io<NY, pp.m - 1, +1, true>(CP, tw, [&](int l, int p) {
            const int ky = pky_of_y(ppinv<NY>(p), NY);
            if (ky >= half || ky <= -half) return pc_zero();
            return ld_pc(a + pmode_slot<NY>(l, ky >= 0 ? ky : ky + kyn, kyp));
        }, SmemIO{lines, NY});
        __syncthreads();
        pdit_range<NY, pp.m - 1, 1, +1>(lines, CP, tw);
        ulonglong2* dst = reinterpret_cast<ulonglong2*>(A.i1_next) + (static_cast<size_t>(b) * P.n_in + slot) * plane + static_cast<size_t>(t0) * NY;
        pstage_io<NY, 0, +1, true>(CP, tw, SmemIO{lines, NY}, [&](int l, int p, PC v) {
            st_stream(dst + static_cast<size_t>(l) * NY + p, make_ulonglong2(f2_mul(v.re, sc), f2_mul(v.im, sc)));
        });
    }
}

}  // namespace shhd
