// Shared-memory mixed-radix FFT building blocks for sm_100a.
//
// Every transform in the step is a batch of complex lines held in shared
// memory by one CTA.  A transform is a sequence of Stockham autosort stages
// (radix 8, 4, 2, 3, 5; natural order in and out), ping-ponged between two
// shared buffers with one barrier per stage; a thread keeps one butterfly
// (R values) in registers at a time.  A stage
// with radix R and span p (product of the radices already applied) maps
// butterfly i, k = i mod p, to
//     inputs  x[i + q*N/R]                          (q = 0..R-1)
//     twiddle x_q *= w_N^(DIR * q*k*N/(p*R))
//     outputs y[(i - k)*R + k + r*p] = sum_q x_q w_R^(DIR*q*r)
// Twiddles come from two small tables (w^j for j < 64 and w^(64 i)), so a
// table for N = 6144 is 160 entries instead of 6144.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace shhd {

// ---------------------------------------------------------------------------
// complex helpers over float2 / double2
// ---------------------------------------------------------------------------
template <typename T> struct CplxOf;
template <> struct CplxOf<float> { using type = float2; };
template <> struct CplxOf<double> { using type = double2; };
template <typename T> using cplx = typename CplxOf<T>::type;

__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
    C r; r.x = a.x * b.x + a.y * b.y; r.y = a.y * b.x - a.x * b.y; return r;
}
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { C r; r.x = a.x * s; r.y = a.y * s; return r; }
template <typename C> __device__ __forceinline__ C cconj(C a) { C r; r.x = a.x; r.y = -a.y; return r; }
// i * a
template <typename C> __device__ __forceinline__ C cmuli(C a) { C r; r.x = -a.y; r.y = a.x; return r; }
// -i * a
template <typename C> __device__ __forceinline__ C cmulmi(C a) { C r; r.x = a.y; r.y = -a.x; return r; }
template <typename C> __device__ __forceinline__ C czero() { C r; r.x = 0; r.y = 0; return r; }

// ---------------------------------------------------------------------------
// division by a runtime constant: q = (n * m) >> 40, exact while n * d < 2^40
// ---------------------------------------------------------------------------
struct FastDiv {
    uint32_t d;
    uint64_t m;
};
__host__ __device__ inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    f.m = ((1ull << 40) + d - 1) / d;
    return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    return static_cast<uint32_t>((static_cast<uint64_t>(n) * f.m) >> 40);
}

// ---------------------------------------------------------------------------
// transform plan (host-built, passed by value)
// ---------------------------------------------------------------------------
constexpr int kMaxStages = 10;
constexpr int kTwLo = 64;

struct FftPlan {
    int n;
    int nstages;
    int radix[kMaxStages];
    int span[kMaxStages];          // p before the stage
    int twstride[kMaxStages];      // N / (p * R)
    FastDiv div_nr[kMaxStages];    // N / R
    FastDiv div_p[kMaxStages];     // p
    int tw_hi_count;               // ceil(n / 64)
    int swz;                       // shared-memory swizzle mask (see sw)
};

// radix butterflies, DIR = -1 forward (e^{-2 pi i/N}), +1 inverse
template <int DIR, typename C>
__device__ __forceinline__ void bfly2(C* v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}

template <int DIR, typename C>
__device__ __forceinline__ C rot90(C a) {  // multiply by DIR * i
    return DIR > 0 ? cmuli(a) : cmulmi(a);
}

template <int DIR, typename C>
__device__ __forceinline__ void bfly4(C* v) {
    const C a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const C c = cadd(v[1], v[3]), d = rot90<DIR>(csub(v[1], v[3]));
    v[0] = cadd(a, c);
    v[2] = csub(a, c);
    v[1] = cadd(b, d);
    v[3] = csub(b, d);
}

template <int DIR, typename C>
__device__ __forceinline__ void bfly8(C* v) {
    using T = decltype(v[0].x);
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    bfly4<DIR>(e);
    bfly4<DIR>(o);
    const T h = static_cast<T>(0.70710678118654752440);
    // o[1] *= (h, DIR h); o[2] *= DIR i; o[3] *= (-h, DIR h)
    const C o1 = mk(h * (o[1].x - DIR * o[1].y), h * (o[1].y + DIR * o[1].x));
    const C o2 = rot90<DIR>(o[2]);
    const C o3 = mk(-h * (o[3].x + DIR * o[3].y), h * (DIR * o[3].x - o[3].y));
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
}

template <int DIR, typename C>
__device__ __forceinline__ void bfly3(C* v) {
    using T = decltype(v[0].x);
    const T s = static_cast<T>(DIR * 0.86602540378443864676);
    const C t1 = cadd(v[1], v[2]);
    const C t2 = mk(v[0].x - static_cast<T>(0.5) * t1.x, v[0].y - static_cast<T>(0.5) * t1.y);
    const C d = csub(v[1], v[2]);
    const C t3 = mk(-s * d.y, s * d.x);  // i * s * d
    v[0] = cadd(v[0], t1);
    v[1] = cadd(t2, t3);
    v[2] = csub(t2, t3);
}

template <int DIR, typename C>
__device__ __forceinline__ void bfly5(C* v) {
    using T = decltype(v[0].x);
    const T c1 = static_cast<T>(0.30901699437494742410);   // cos(2 pi/5)
    const T c2 = static_cast<T>(-0.80901699437494742410);  // cos(4 pi/5)
    const T s1 = static_cast<T>(DIR * 0.95105651629515357212);
    const T s2 = static_cast<T>(DIR * 0.58778525229247312917);
    const C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
    const C a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
    const C r1 = mk(v[0].x + c1 * a1.x + c2 * a2.x, v[0].y + c1 * a1.y + c2 * a2.y);
    const C r2 = mk(v[0].x + c2 * a1.x + c1 * a2.x, v[0].y + c2 * a1.y + c1 * a2.y);
    const C i1 = mk(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y);
    const C i2 = mk(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y);
    v[0] = cadd(v[0], cadd(a1, a2));
    v[1] = cadd(r1, cmuli(i1));
    v[4] = csub(r1, cmuli(i1));
    v[2] = cadd(r2, cmuli(i2));
    v[3] = csub(r2, cmuli(i2));
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void bfly(C* v) {
    if constexpr (R == 2) bfly2<DIR>(v);
    else if constexpr (R == 3) bfly3<DIR>(v);
    else if constexpr (R == 4) bfly4<DIR>(v);
    else if constexpr (R == 5) bfly5<DIR>(v);
    else bfly8<DIR>(v);
}

// w_N^(DIR * idx) from the two-level table (forward-sign table, conjugated for DIR = +1)
template <int DIR, typename C>
__device__ __forceinline__ C twiddle(const C* tw_lo, const C* tw_hi, uint32_t idx) {
    const C a = tw_hi[idx >> 6];
    const C b = tw_lo[idx & 63];
    const C w = cmul(a, b);
    return DIR > 0 ? cconj(w) : w;
}

// x_q *= w^q for q = 1..R-1 from one table twiddle w; powers by a shallow
// product tree (at most three rounding steps deep).
template <int R, typename C>
__device__ __forceinline__ void apply_twiddles(C* v, const C w) {
    if constexpr (R == 2) {
        v[1] = cmul(v[1], w);
    } else if constexpr (R == 3) {
        v[1] = cmul(v[1], w);
        v[2] = cmul(v[2], cmul(w, w));
    } else if constexpr (R == 4) {
        const C w2 = cmul(w, w);
        v[1] = cmul(v[1], w);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], cmul(w2, w));
    } else if constexpr (R == 5) {
        const C w2 = cmul(w, w);
        v[1] = cmul(v[1], w);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], cmul(w2, w));
        v[4] = cmul(v[4], cmul(w2, w2));
    } else {
        const C w2 = cmul(w, w);
        const C w3 = cmul(w2, w);
        const C w4 = cmul(w2, w2);
        v[1] = cmul(v[1], w);
        v[2] = cmul(v[2], w2);
        v[3] = cmul(v[3], w3);
        v[4] = cmul(v[4], w4);
        v[5] = cmul(v[5], cmul(w4, w));
        v[6] = cmul(v[6], cmul(w4, w2));
        v[7] = cmul(v[7], cmul(w4, w3));
    }
}

// Element y of a line lives at slot sw(y): the low bits are XORed with bits
// 3.. of y.  A radix-8 first stage writes with a stride of 8 elements; the
// swizzle spreads those writes over distinct shared-memory banks while keeping
// contiguous runs conflict-free.  sw is a bijection inside every aligned
// block of 16 (bit 3 only mixes with bit 6), so any line length that is a
// multiple of 16 (or of mask + 1 for smaller masks) is safe; the host picks
// mask = 0 otherwise.
__device__ __forceinline__ uint32_t sw(uint32_t y, uint32_t mask) { return y ^ ((y >> 3) & mask); }

// One Stockham stage, out of place (src -> dst), over `nlines` lines of
// length N; element e of line l is at l * line_stride + sw(e) * elem_stride.
// LINES_FAST maps consecutive threads to consecutive lines (interleaved column
// tiles, elem_stride = tile width) instead of consecutive butterflies.
template <int R, int DIR, bool LINES_FAST, typename C>
__device__ __forceinline__ void fft_stage(const C* __restrict__ src, C* __restrict__ dst, const FftPlan& plan, int s, int nlines,
                                          const FastDiv& div_lines, int line_stride, int elem_stride, uint32_t mask, const C* tw_lo,
                                          const C* tw_hi) {
    const uint32_t N = plan.n;
    const uint32_t NR = N / R;
    const uint32_t p = plan.span[s];
    const uint32_t total = static_cast<uint32_t>(nlines) * NR;
    const uint32_t tws = static_cast<uint32_t>(plan.twstride[s]);
#pragma unroll 2
    for (uint32_t b = threadIdx.x; b < total; b += blockDim.x) {
        uint32_t l, bi;
        if (LINES_FAST) { bi = fdiv(b, div_lines); l = b - bi * nlines; }
        else { l = fdiv(b, plan.div_nr[s]); bi = b - l * NR; }
        const C* in = src + l * line_stride;
        C v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = in[sw(bi + q * NR, mask) * elem_stride];
        const uint32_t k = bi - fdiv(bi, plan.div_p[s]) * p;
        if (k != 0) apply_twiddles<R>(v, twiddle<DIR>(tw_lo, tw_hi, k * tws));
        bfly<R, DIR>(v);
        const uint32_t j = (bi - k) * R + k;
        C* out = dst + l * line_stride;
#pragma unroll
        for (int q = 0; q < R; ++q) out[sw(j + q * p, mask) * elem_stride] = v[q];
    }
    __syncthreads();
}

// Full transform of `nlines` lines.  The input must be at fft_input(buf,
// scratch, plan) (buf for an even number of stages, scratch for odd), so the
// ping-pong always ends in buf.  Callers synchronise before the call.
template <typename C>
__device__ __forceinline__ C* fft_input(C* buf, C* scratch, const FftPlan& plan) {
    return (plan.nstages & 1) ? scratch : buf;
}

template <int DIR, bool LINES_FAST, typename C>
__device__ __forceinline__ void fft_lines(C* buf, C* scratch, const FftPlan& plan, int nlines, const FastDiv& div_lines, int line_stride,
                                          int elem_stride, const C* tw_lo, const C* tw_hi) {
    C* src = fft_input(buf, scratch, plan);
    C* dst = (src == buf) ? scratch : buf;
    const uint32_t mask = static_cast<uint32_t>(plan.swz);
    for (int s = 0; s < plan.nstages; ++s) {
        switch (plan.radix[s]) {
            case 8: fft_stage<8, DIR, LINES_FAST>(src, dst, plan, s, nlines, div_lines, line_stride, elem_stride, mask, tw_lo, tw_hi); break;
            case 4: fft_stage<4, DIR, LINES_FAST>(src, dst, plan, s, nlines, div_lines, line_stride, elem_stride, mask, tw_lo, tw_hi); break;
            case 2: fft_stage<2, DIR, LINES_FAST>(src, dst, plan, s, nlines, div_lines, line_stride, elem_stride, mask, tw_lo, tw_hi); break;
            case 3: fft_stage<3, DIR, LINES_FAST>(src, dst, plan, s, nlines, div_lines, line_stride, elem_stride, mask, tw_lo, tw_hi); break;
            default: fft_stage<5, DIR, LINES_FAST>(src, dst, plan, s, nlines, div_lines, line_stride, elem_stride, mask, tw_lo, tw_hi); break;
        }
        C* t = src; src = dst; dst = t;
    }
}

// ---------------------------------------------------------------------------
// compile-time sizes: radix plan, spans and per-stage twiddle rows resolved by
// the compiler, so every index is shifts and immediate offsets
// ---------------------------------------------------------------------------
constexpr int kMaxFixedStages = 12;

// twiddle row length per butterfly for radix R: R - 1 entries padded so a
// float2 row starts on a 16-byte boundary
__host__ __device__ constexpr int tw_row(int R) { return R == 8 ? 8 : (R == 4 ? 4 : (R == 5 ? 4 : 2)); }

struct CPlan {
    int ns;
    int r[kMaxFixedStages];
    int p[kMaxFixedStages];
    int twoff[kMaxFixedStages];  // offset of the stage's twiddle rows (span > 1 only)
    int twsz;                    // total twiddle entries
};

__host__ __device__ constexpr CPlan make_cplan(int n) {
    CPlan c{};
    int m = n, ns = 0;
    while (m % 8 == 0) { c.r[ns++] = 8; m /= 8; }
    if (m % 4 == 0) { c.r[ns++] = 4; m /= 4; }
    if (m % 2 == 0) { c.r[ns++] = 2; m /= 2; }
    while (m % 3 == 0) { c.r[ns++] = 3; m /= 3; }
    while (m % 5 == 0) { c.r[ns++] = 5; m /= 5; }
    c.ns = ns;
    int p = 1, off = 0;
    for (int s = 0; s < ns; ++s) {
        c.p[s] = p;
        c.twoff[s] = off;
        if (p > 1) off += p * tw_row(c.r[s]);
        p *= c.r[s];
    }
    c.twsz = off;
    return c;
}

template <int N> struct FixedPlan { static constexpr CPlan c = make_cplan(N); };

// sizes with a compile-time path (3 * 2^k padded grids of the 3/2 rule)
__host__ __device__ constexpr bool is_fixed_size(int n) {
    return n == 96 || n == 192 || n == 384 || n == 768 || n == 1536 || n == 3072 || n == 6144;
}

// One stage of a compile-time transform; lines interleave with width 2^logw
// (LF) or sit N apart (rows).  Twiddles w^q (q = 1..R-1) for span index k
// come from row k of the stage's table.  Requires mask <= 7: then
// sw(y + m) = sw(y) + m for every multiple m of 64.
template <int N, int R, int P, int TWOFF, int DIR, bool LF, typename C>
__device__ __forceinline__ void fixed_stage(const C* __restrict__ src, C* __restrict__ dst, int lines, int logw, uint32_t mask,
                                            const C* __restrict__ tw) {
    constexpr int NR = N / R;
    constexpr int ROW = tw_row(R);
    const int total = lines * NR;
#pragma unroll 2
    for (int b = threadIdx.x; b < total; b += blockDim.x) {
        int l, bi;
        if constexpr (LF) { l = b & ((1 << logw) - 1); bi = b >> logw; }
        else { l = b / NR; bi = b - l * NR; }
        const C* in = LF ? src + l : src + l * N;
        C v[R];
        if constexpr (NR % 64 == 0) {
            const uint32_t s0 = sw(bi, mask);
#pragma unroll
            for (int q = 0; q < R; ++q) v[q] = in[(s0 + q * NR) << (LF ? logw : 0)];
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q) v[q] = in[sw(bi + q * NR, mask) << (LF ? logw : 0)];
        }
        const int k = bi % P;
        if constexpr (P > 1) {
            const C* t = tw + TWOFF + k * ROW;
#pragma unroll
            for (int q = 1; q < R; ++q) {
                const C w = t[q - 1];
                v[q] = DIR < 0 ? cmul(v[q], w) : cmulc(v[q], w);
            }
        }
        bfly<R, DIR>(v);
        const int j = (bi - k) * R + k;
        C* out = LF ? dst + l : dst + l * N;
        if constexpr (P % 64 == 0) {
            const uint32_t s0 = sw(j, mask);
#pragma unroll
            for (int q = 0; q < R; ++q) out[(s0 + q * P) << (LF ? logw : 0)] = v[q];
        } else {
#pragma unroll
            for (int q = 0; q < R; ++q) out[sw(j + q * P, mask) << (LF ? logw : 0)] = v[q];
        }
    }
    __syncthreads();
}

template <int N, int S, int DIR, bool LF, typename C>
__device__ __forceinline__ void fixed_stages(C* a, C* b, int lines, int logw, uint32_t mask, const C* tw) {
    constexpr CPlan cp = FixedPlan<N>::c;
    if constexpr (S < cp.ns) {
        fixed_stage<N, cp.r[S], cp.p[S], cp.twoff[S], DIR, LF>(a, b, lines, logw, mask, tw);
        fixed_stages<N, S + 1, DIR, LF>(b, a, lines, logw, mask, tw);
    }
}

template <int N, typename C>
__device__ __forceinline__ C* fixed_input(C* buf, C* scratch) {
    return (FixedPlan<N>::c.ns & 1) ? scratch : buf;
}

// Transform `lines` lines; input at fixed_input(buf, scratch), result in buf.
template <int N, int DIR, bool LF, typename C>
__device__ __forceinline__ void fixed_fft(C* buf, C* scratch, int lines, int logw, uint32_t mask, const C* tw) {
    fixed_stages<N, 0, DIR, LF>(fixed_input<N>(buf, scratch), (fixed_input<N>(buf, scratch) == buf) ? scratch : buf, lines, logw, mask, tw);
}

// ---------------------------------------------------------------------------
// dispatch: FN = compile-time size, or 0 for the runtime plan.  `tw` is the
// shared-memory table (per-stage rows for FN > 0, the two-level table else).
// ---------------------------------------------------------------------------
template <int FN, typename C>
__device__ __forceinline__ C* xform_input(C* buf, C* scratch, const FftPlan& plan) {
    if constexpr (FN == 0) return fft_input(buf, scratch, plan);
    else return fixed_input<FN>(buf, scratch);
}

template <int FN, int DIR, bool LF, typename C>
__device__ __forceinline__ void xform(C* buf, C* scratch, const FftPlan& plan, int nlines, const FastDiv& div_lines, int line_stride,
                                      int elem_stride, int logw, const C* tw) {
    if constexpr (FN == 0) fft_lines<DIR, LF>(buf, scratch, plan, nlines, div_lines, line_stride, elem_stride, tw, tw + kTwLo);
    else fixed_fft<FN, DIR, LF>(buf, scratch, nlines, logw, static_cast<uint32_t>(plan.swz), tw);
}

template <typename C>
__device__ __forceinline__ void load_table(C* dst, const C* __restrict__ src, int count) {
    for (int i = threadIdx.x; i < count; i += blockDim.x) dst[i] = src[i];
}

// copy the plan's twiddle tables (global, forward sign) into shared memory
template <typename C>
__device__ __forceinline__ void load_twiddles(C* s_lo, C* s_hi, const C* g_tw, int hi_count) {
    for (int i = threadIdx.x; i < kTwLo + hi_count; i += blockDim.x) {
        const C w = g_tw[i];
        if (i < kTwLo) s_lo[i] = w; else s_hi[i - kTwLo] = w;
    }
}

}  // namespace shhd
