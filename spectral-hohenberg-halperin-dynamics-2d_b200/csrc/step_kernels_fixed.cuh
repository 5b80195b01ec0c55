// Step kernels for the compile-time transform sizes (3 * 2^k padded grids).
//
// Same three passes and the same epilogue math as step_kernels.cuh, organised
// for throughput: a transform line belongs to one group of G threads (one or
// more warps) that synchronises on its own named barrier, stages its
// butterflies in registers and transforms the line in place (no ping-pong
// buffer).  The row pass keeps one line per group in flight; the column pass
// gives each of the tile's W columns to one group and keeps the RHS
// accumulators in shared memory.  Twiddles are read through the read-only
// cache from the per-stage rows in global memory.
#pragma once

#include "step_kernels.cuh"

namespace shhd {

// threads per transform group for a line of N complex values: about 24 staged
// values per thread in the widest stage
template <typename T, int N>
__host__ __device__ constexpr int row_group() {
    constexpr int g = (sizeof(T) == 4 ? N / 24 : N / 12);
    return g <= 32 ? 32 : (g <= 64 ? 64 : (g <= 128 ? 128 : 256));
}
// lines of 48 KB or more (FP32 6144, FP64 3072) allow one CTA per SM: the row pass may then run
// two line groups in a 512-thread block, two transform chains side by side
template <typename T, int N>
__host__ __device__ constexpr bool row_big_lines() {
    return N * 2 * sizeof(T) >= 49152 && row_group<T, N>() == kThreads;
}
// column tile width for the compile-time column kernels (columns per CTA, one group each)
template <typename T, int N>
__host__ __device__ constexpr int col_width() {
    constexpr int w = (sizeof(T) == 4 ? 4096 : 2048) / N;
    return w >= 8 ? 8 : (w >= 4 ? 4 : (w >= 2 ? 2 : 1));
}

__device__ __forceinline__ uint32_t sw7(uint32_t y) { return y ^ ((y >> 3) & 7u); }
// shared-memory slot of element y in a line: SB = 3 is sw7 (bank-conflict free for 16-byte elements in
// the transform stages); SB = 4 XORs four bits, which 8-byte elements need to spread a warp's stores of
// the radix-8 stages with spans 1 and 8 over all 16 bank pairs
template <int SB>
__device__ __forceinline__ uint32_t swz(uint32_t y) {
    return y ^ ((y >> SB) & ((1u << SB) - 1u));
}

// synchronise one line group of G threads in a block of NT threads: the warp, the whole block, or
// the group's own named barrier (id bid = 1 + group index; barrier 0 is __syncthreads)
template <int G, int NT = kThreads>
__device__ __forceinline__ void group_sync(int bid) {
    if constexpr (G == 32) __syncwarp();
    else if constexpr (G == NT) __syncthreads();
    else asm volatile("bar.sync %0, %1;" ::"r"(bid), "n"(G) : "memory");
}

// one in-place stage of a group transform of a line (element y at sw7(y))
template <int N, int R, int P, int TWOFF, int G, int DIR, int NT, int SB, typename C>
__device__ __forceinline__ void gstage(C* line, const C* __restrict__ tw, int gt, int bid) {
    constexpr int NR = N / R;
    constexpr int B = (NR + G - 1) / G;
    constexpr int ROW = tw_row(R);
    constexpr int SPAN = 1 << (2 * SB);  // adding a multiple of SPAN leaves the swizzled bits alone
    // FP32 reads w^k, w^2k, w^3k exactly (the table row holds every power) and forms the higher
    // powers at most two roundings deep; FP64 reads w^k alone, its products being far below FP32
    constexpr int NL = (sizeof(C) == 8) ? (R - 1 < 3 ? R - 1 : 3) : 1;
    C v[B][R];
    C wk[B][NL];  // the loaded powers of each butterfly, before the barrier so their latency overlaps the wait
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int bi = gt + i * G;
        if (NR % G == 0 || bi < NR) {
            if constexpr (P > 1) {
#pragma unroll
                for (int l = 0; l < NL; ++l) wk[i][l] = __ldg(tw + TWOFF + (bi % P) * ROW + l);
            }
            if constexpr (NR % SPAN == 0) {
                const uint32_t s0 = swz<SB>(bi);
#pragma unroll
                for (int q = 0; q < R; ++q) v[i][q] = line[s0 + q * NR];
            } else {
#pragma unroll
                for (int q = 0; q < R; ++q) v[i][q] = line[swz<SB>(bi + q * NR)];
            }
        }
    }
    group_sync<G, NT>(bid);
#pragma unroll
    for (int i = 0; i < B; ++i) {
        const int bi = gt + i * G;
        if (NR % G == 0 || bi < NR) {
            const int k = bi % P;
            if constexpr (P > 1) {
                C w[R];
                if constexpr (NL == 1) {
                    // one load of w^k per butterfly; its powers by a product tree at most three roundings deep
                    w[1] = wk[i][0];
                    if constexpr (R > 2) w[2] = cmul(w[1], w[1]);
                    if constexpr (R > 3) w[3] = cmul(w[2], w[1]);
                    if constexpr (R > 4) w[4] = cmul(w[2], w[2]);
                    if constexpr (R > 5) w[5] = cmul(w[4], w[1]);
                    if constexpr (R > 6) w[6] = cmul(w[3], w[3]);
                    if constexpr (R > 7) w[7] = cmul(w[4], w[3]);
                } else {
#pragma unroll
                    for (int l = 0; l < NL; ++l) w[l + 1] = wk[i][l];
                    if constexpr (R > 4) w[4] = cmul(w[2], w[2]);
                    if constexpr (R > 5) w[5] = cmul(w[2], w[3]);
                    if constexpr (R > 6) w[6] = cmul(w[3], w[3]);
                    if constexpr (R > 7) w[7] = cmul(w[3], w[4]);
                }
#pragma unroll
                for (int q = 1; q < R; ++q) v[i][q] = DIR < 0 ? cmul(v[i][q], w[q]) : cmulc(v[i][q], w[q]);
            }
            bfly<R, DIR>(v[i]);
            const int j = (bi - k) * R + k;
            if constexpr (P % SPAN == 0) {
                const uint32_t s0 = swz<SB>(j);
#pragma unroll
                for (int q = 0; q < R; ++q) line[s0 + q * P] = v[i][q];
            } else if constexpr (SB != 3) {
#pragma unroll
                for (int q = 0; q < R; ++q) line[swz<SB>(j + q * P)] = v[i][q];
            } else if constexpr (R == 8 && P == 1) {
                // j = 8 bi: sw7(j + q) = 8 bi + (q ^ (bi & 7))
                C* o = line + 8 * bi;
                const uint32_t m = bi & 7;
#pragma unroll
                for (int q = 0; q < R; ++q) o[q ^ m] = v[i][q];
            } else if constexpr (R == 8 && P == 8) {
                // j = 64 (bi >> 3) + k: sw7(j + 8 q) = 64 (bi >> 3) + 8 q + (k ^ q)
                C* o = line + 64 * (bi >> 3);
#pragma unroll
                for (int q = 0; q < R; ++q) o[8 * q + (k ^ q)] = v[i][q];
            } else {
#pragma unroll
                for (int q = 0; q < R; ++q) line[sw7(j + q * P)] = v[i][q];
            }
        }
    }
    group_sync<G, NT>(bid);
}

template <int N, int G, int DIR, int NT, int SB, int S, typename C>
__device__ __forceinline__ void gstages(C* line, const C* tw, int gt, int bid) {
    constexpr CPlan cp = FixedPlan<N>::c;
    if constexpr (S < cp.ns) {
        gstage<N, cp.r[S], cp.p[S], cp.twoff[S], G, DIR, NT, SB>(line, tw, gt, bid);
        gstages<N, G, DIR, NT, SB, S + 1>(line, tw, gt, bid);
    }
}

// in-place transform of one line by the calling group of a block of NT threads, elements at
// swz<SB>(y); the caller has synchronised the group (or CTA) after writing the line
template <int N, int G, int DIR, int NT = kThreads, int SB = 3, typename C>
__device__ __forceinline__ void gfft(C* line, const C* tw, int gt, int bid) {
    gstages<N, G, DIR, NT, SB, 0>(line, tw, gt, bid);
}

// contiguous [y][w] tile (global) -> [w][sw7(y)] lines (shared); all loads of a
// thread are issued before its stores so they overlap in flight
template <int W, int NY, typename C>
__device__ __forceinline__ void load_tile(C* tile, const C* __restrict__ src) {
    constexpr int PER = (W * NY + kThreads - 1) / kThreads;
    constexpr int CH = PER < 12 ? PER : 12;
    for (int e0 = 0; e0 < PER; e0 += CH) {
        C v[CH];
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int e = threadIdx.x + (e0 + u) * kThreads;
            if ((W * NY) % kThreads == 0 || e < W * NY) v[u] = src[e];
        }
#pragma unroll
        for (int u = 0; u < CH; ++u) {
            const int e = threadIdx.x + (e0 + u) * kThreads;
            if ((W * NY) % kThreads == 0 || e < W * NY) {
                const int y = e / W, w = e - y * W;
                tile[w * NY + sw7(y)] = v[u];
            }
        }
    }
}

// ---------------------------------------------------------------------------
// column inverse (compile-time NY): state -> I1   (grid: tiles x n_in x batch)
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(kThreads) col_inverse_fixed(const StepPlan P, const MemberInfo* __restrict__ members,
                                                              const cplx<T>* __restrict__ state, cplx<T>* __restrict__ i1,
                                                              const cplx<T>* __restrict__ tw) {
    if (!members[blockIdx.z].active) return;
    using C = cplx<T>;
    constexpr int W = col_width<T, NY>();
    constexpr int G = kThreads / W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* tile = reinterpret_cast<C*>(smem_raw);  // [W][NY]
    const int g = threadIdx.x / G, gt = threadIdx.x - g * G, bid = 1 + g;
    const int t = blockIdx.x, slot = blockIdx.y, b = blockIdx.z;
    const int kyn = P.kyn, half = P.nay / 2;
    const int field = P.in_field[slot];
    const C* src = state + (static_cast<size_t>(b) * P.nfields + field) * P.hx * kyn + static_cast<size_t>(t) * W * kyn;
    // column g: zero-padded copy (|ky| < Na/2 only)
    C* line = tile + g * NY;
    for (int y = gt; y < NY; y += G) {
        int j = -1;
        if (y < half) j = y;
        else if (y > NY - half) j = y - NY + kyn;
        line[sw7(y)] = (j >= 0) ? src[g * kyn + j] : czero<C>();
    }
    group_sync<G>(bid);
    gfft<NY, G, +1>(line, tw, gt, bid);
    __syncthreads();
    const T sc = static_cast<T>(P.inv_scale);
    C* dst = i1 + ((static_cast<size_t>(b) * P.n_in + slot) * P.ntiles + t) * static_cast<size_t>(NY) * W;
    for (int e = threadIdx.x; e < W * NY; e += kThreads) {
        const int y = e / W, w = e - y * W;
        dst[e] = cscale(tile[w * NY + sw7(y)], sc);
    }
}

// ---------------------------------------------------------------------------
// row pass (compile-time NX): I1 -> C2R -> products -> R2C -> I2   (grid: row pairs x batch)
// ---------------------------------------------------------------------------
template <typename T, int NX, int NT>
__global__ void __launch_bounds__(NT, (NT > kThreads ? 1 : 2)) row_pass_fixed(const StepPlan P, const MemberInfo* __restrict__ members,
                                                           const cplx<T>* __restrict__ i1, cplx<T>* __restrict__ i2,
                                                           const cplx<T>* __restrict__ tw, const double* __restrict__ rho0_member,
                                                           int* __restrict__ err) {
    if (!members[blockIdx.y].active) return;
    using C = cplx<T>;
    constexpr int G = row_group<T, NX>();
    constexpr int NG = NT / G;                // line groups per block (NT threads)
    constexpr int SB = sizeof(T) == 4 ? 4 : 3;  // line swizzle (swz<SB>) for this element size
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* lines = reinterpret_cast<C*>(smem_raw);          // [n_in][NX] physical row pairs
    C* work = lines + static_cast<size_t>(P.n_in) * NX;  // [NG][NX] one product line per group
    const int g = threadIdx.x / G, gt = threadIdx.x - g * G, bid = 1 + g;
    const int npy = P.npy, W = P.W, hx = P.hx;
    const int pair = blockIdx.x, b = blockIdx.y;
    const int y0 = 2 * pair;
    const bool has1 = (y0 + 1) < npy;

    // 1. inputs: Z[k] = X0[k] + i X1[k] with the Hermitian mirror, zero outside |kx| < Na/2;
    //    loads are issued in batches of 4 per thread so several are in flight
    const size_t i1_member = static_cast<size_t>(b) * P.n_in * P.ntiles * npy * W;
    const size_t slot_stride = static_cast<size_t>(P.ntiles) * npy * W;
    constexpr int U = 4;
    // a row pair of one column tile is one 32-byte sector when the tile is 16 bytes wide (FP32
    // with two-column tiles, FP64 with one) and the row count is even: one 256-bit load per tile
    constexpr int WC = 16 / static_cast<int>(sizeof(C));  // columns of such a tile
    const bool wide = W == WC && has1 && (npy & 1) == 0;
    const int nload = wide ? P.n_in * (hx / WC) : P.n_in * hx;
    if (wide) {
        const int ntile = hx / WC;
        for (int e0 = threadIdx.x; e0 < nload; e0 += NT * U) {
            ulonglong2 r0[U], r1[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + u * NT;
                if (e < nload) {
                    const int s = e / ntile, t = e - s * ntile;
                    const C* p0 = i1 + i1_member + s * slot_stride + (static_cast<size_t>(t) * npy + y0) * WC;
                    ld_stream2(reinterpret_cast<const ulonglong2*>(p0), r0[u], r1[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int e = e0 + u * NT;
                if (e < nload) {
                    const int s = e / ntile, t = e - s * ntile;
                    C* z = lines + static_cast<size_t>(s) * NX;
#pragma unroll
                    for (int w = 0; w < WC; ++w) {
                        const int k = t * WC + w;
                        C av = c16_get(r0[u], w, C{}), cv = c16_get(r1[u], w, C{});
                        if (k == 0) { av.y = 0; cv.y = 0; }  // C2R uses the real part of the kx = 0 entry
                        z[swz<SB>(k)] = mk(av.x - cv.y, av.y + cv.x);
                        if (k > 0) z[swz<SB>(NX - k)] = mk(av.x + cv.y, cv.x - av.y);
                    }
                }
            }
        }
    }
    for (int e0 = threadIdx.x; !wide && e0 < nload; e0 += NT * U) {
        C a[U], c[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * NT;
            if (e < nload) {
                const int s = e / hx, k = e - s * hx;
                const int t = k >> P.logw, w = k & (W - 1);
                const C* p0 = i1 + i1_member + s * slot_stride + (static_cast<size_t>(t) * npy + y0) * W + w;
                a[u] = p0[0];
                c[u] = has1 ? p0[W] : czero<C>();
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int e = e0 + u * NT;
            if (e < nload) {
                const int s = e / hx, k = e - s * hx;
                C* z = lines + static_cast<size_t>(s) * NX;
                C av = a[u], cv = c[u];
                if (k == 0) { av.y = 0; cv.y = 0; }  // C2R uses the real part of the kx = 0 entry
                z[swz<SB>(k)] = mk(av.x - cv.y, av.y + cv.x);
                if (k > 0) z[swz<SB>(NX - k)] = mk(av.x + cv.y, cv.x - av.y);
            }
        }
    }
    const int nzero = NX - 2 * hx + 1;  // k in [hx, NX - hx]
    for (int e = threadIdx.x; e < P.n_in * nzero; e += NT) {
        const int s = e / nzero, k = hx + (e - s * nzero);
        lines[static_cast<size_t>(s) * NX + swz<SB>(k)] = czero<C>();
    }
    __syncthreads();
    for (int s = g; s < P.n_in; s += NG) gfft<NX, G, +1, NT, SB>(lines + static_cast<size_t>(s) * NX, tw, gt, bid);
    __syncthreads();

    // 2. velocity: v = j / rho (compressible) or j / rho0 (fcalculator_workspace.cc:115-142);
    //    pointwise work runs over swizzled slots (every line shares the permutation)
    const int s_rho = P.in_slot[0];
    const int s_jx = P.in_slot[P.nop + 1];
    const int s_jy = P.in_slot[P.nop + 2];
    const bool comp = (P.mode == 0);
    const T inv_rho0 = (P.need_v && !comp) ? static_cast<T>(1.0 / rho0_member[b]) : T(0);
    if (P.need_v && comp) {
        // zero-density check, then rho is replaced by 1/rho (its only use is v = j / rho)
        int bad = 0;
        for (int x = threadIdx.x; x < NX; x += NT) {
            C* pr = lines + static_cast<size_t>(s_rho) * NX + x;
            const C rho = *pr;
            if (rho.x == T(0) || (has1 && rho.y == T(0))) bad = 1;
            *pr = mk(T(1) / rho.x, has1 ? T(1) / rho.y : T(0));
        }
        if (bad) atomicOr(err, ERR_ZERO_DENSITY);
        __syncthreads();
    }

    // 3. products -> forward transform -> keep kx < Hx; output o belongs to group o % NG.  In the
    //    two-group block the outputs left over after the last full round of groups run on the whole
    //    block, so no group idles through a transform (three outputs: one round of two, then one)
    const size_t i2_member = static_cast<size_t>(b) * P.n_out * P.ntiles * npy * W;
    auto one_output = [&](auto gg, int o, C* z, int tid, int barid) {
        constexpr int GG = decltype(gg)::value;
        const int kind = P.out_kind[o], arg = P.out_arg[o];
        const int s_psi = (kind == OUT_MU || kind == OUT_PSIVX || kind == OUT_PSIVY) ? P.in_slot[1 + arg] : -1;
        const bool use_v = (kind != OUT_MU);
        for (int x = tid; x < NX; x += GG) {
            const C psi = s_psi >= 0 ? lines[static_cast<size_t>(s_psi) * NX + x] : czero<C>();
            C jx = czero<C>(), jy = czero<C>(), vx = czero<C>(), vy = czero<C>();
            if (use_v) {
                jx = lines[static_cast<size_t>(s_jx) * NX + x];
                jy = lines[static_cast<size_t>(s_jy) * NX + x];
                if (comp) {
                    const C ir = lines[static_cast<size_t>(s_rho) * NX + x];  // 1/rho
                    vx = mk(jx.x * ir.x, jx.y * ir.y);
                    vy = mk(jy.x * ir.x, jy.y * ir.y);
                } else {
                    vx = mk(jx.x * inv_rho0, jx.y * inv_rho0);
                    vy = mk(jy.x * inv_rho0, jy.y * inv_rho0);
                }
            }
            C val = mk(product_value<T>(P, kind, arg, psi.x, jx.x, jy.x, vx.x, vy.x),
                       product_value<T>(P, kind, arg, psi.y, jx.y, jy.y, vx.y, vy.y));
            if (kind == OUT_MU && P.fe_plugin)
                plugin_mu_rows<T>(P, arg, [&](int s) { return lines[static_cast<size_t>(s) * NX + x]; }, val.x, val.y);
            if (!has1) val.y = T(0);
            z[x] = val;
        }
        group_sync<GG, NT>(barid);
        gfft<NX, GG, -1, NT, SB>(z, tw, tid, barid);
        C* dst = i2 + i2_member + static_cast<size_t>(o) * P.ntiles * npy * W;
        for (int k = tid; !wide && k < hx; k += GG) {
            const C zk = z[swz<SB>(k)];
            const C zn = cconj(z[swz<SB>(k == 0 ? 0 : NX - k)]);
            const C g0 = mk(static_cast<T>(0.5) * (zk.x + zn.x), static_cast<T>(0.5) * (zk.y + zn.y));
            const C d = csub(zk, zn);
            const C g1 = mk(static_cast<T>(0.5) * d.y, static_cast<T>(-0.5) * d.x);
            const int t = k >> P.logw, w = k & (W - 1);
            C* q = dst + (static_cast<size_t>(t) * npy + y0) * W + w;
            q[0] = g0;
            if (has1) q[W] = g1;
        }
        for (int t = tid; wide && t < hx / WC; t += GG) {  // one 256-bit store per tile and row pair
            ulonglong2 o0, o1;
#pragma unroll
            for (int w = 0; w < WC; ++w) {
                const int k = t * WC + w;
                const C zk = z[swz<SB>(k)];
                const C zn = cconj(z[swz<SB>(k == 0 ? 0 : NX - k)]);
                const C d = csub(zk, zn);
                c16_set(o0, w, mk(static_cast<T>(0.5) * (zk.x + zn.x), static_cast<T>(0.5) * (zk.y + zn.y)));
                c16_set(o1, w, mk(static_cast<T>(0.5) * d.y, static_cast<T>(-0.5) * d.x));
            }
            st_stream2(reinterpret_cast<ulonglong2*>(dst + (static_cast<size_t>(t) * npy + y0) * WC), o0, o1);
        }
        group_sync<GG, NT>(barid);
    };
    constexpr bool kBlockTail = NT > kThreads && NG == 2;
    const int n_rounds = kBlockTail ? (P.n_out / NG) * NG : P.n_out;
    for (int o = g; o < n_rounds; o += NG) one_output(std::integral_constant<int, G>{}, o, work + static_cast<size_t>(g) * NX, gt, bid);
    if constexpr (kBlockTail) {
        if (n_rounds < P.n_out) {
            __syncthreads();  // every group is done with its work line
            for (int o = n_rounds; o < P.n_out; ++o) one_output(std::integral_constant<int, NT>{}, o, work, threadIdx.x, 0);
        }
    }
}

// ---------------------------------------------------------------------------
// column forward + epilogue (compile-time NY)   (grid: tiles x groups x batch)
// ---------------------------------------------------------------------------
template <typename T, int NY>
__global__ void __launch_bounds__(kThreads, 2) col_forward_fixed(const StepPlan P, const StageArgs<T> A, const cplx<T>* __restrict__ tw) {
    using C = cplx<T>;
    constexpr int W = col_width<T, NY>();
    constexpr int G = kThreads / W;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int kyn = P.kyn, nay = P.nay;
    C* tile = reinterpret_cast<C*>(smem_raw);   // [W][NY]
    C* acc0 = tile + W * NY;                     // [W][Ky]
    C* acc1 = acc0 + W * kyn;                    // [W][Ky]
    const int g = threadIdx.x / G, gt = threadIdx.x - g * G, bid = 1 + g;
    const int t = blockIdx.x, grp = blockIdx.y, b = blockIdx.z;
    const int gkind = P.group_kind[grp];
    const int alpha = P.group_alpha[grp];
    const bool comp = (P.mode == 0);
    const MemberInfo mi = A.members[b];
    if (!mi.active) return;
    const size_t fstride = static_cast<size_t>(P.hx) * kyn;
    const size_t mbase = static_cast<size_t>(b) * P.nfields * fstride + static_cast<size_t>(t) * W * kyn;
    const T kxu = static_cast<T>(P.kx_unit), kyu = static_cast<T>(P.ky_unit);
    C* line = tile + g * NY;
    C* a0 = acc0 + g * kyn;
    C* a1 = acc1 + g * kyn;
    const T kx = kxu * static_cast<T>(t * W + g);

    for (int j = gt; j < kyn; j += G) { a0[j] = czero<C>(); a1[j] = czero<C>(); }

    const int ngo = P.group_nout[grp];
    for (int go = 0; go < ngo; ++go) {
        const int o = P.group_out[grp][go];
        const C* src = A.i2 + ((static_cast<size_t>(b) * P.n_out + o) * P.ntiles + t) * static_cast<size_t>(NY) * W;
        __syncthreads();  // every group is done with the previous tile
        load_tile<W, NY>(tile, src);
        __syncthreads();
        gfft<NY, G, -1>(line, tw, gt, bid);
        const int kind = P.out_kind[o];
        for (int j = gt; j < kyn; j += G) {
            const int ky = ky_of_j(j, nay);
            const int y = ky >= 0 ? ky : ky + NY;
            C u0 = a0[j], u1 = a1[j];
            accumulate_product<T>(P, kind, alpha, kx, kyu * static_cast<T>(ky), line[sw7(y)], u0, u1);
            a0[j] = u0;
            a1[j] = u1;
        }
    }

    // epilogue for column g: results replace a0 (psi or jx) and a1 (jy); the
    // next mode's global loads are issued before the current mode's math
    if (gkind == GROUP_PSI) {
        PsiLoads<T> L = psi_loads<T>(P, A, alpha, mode_ctx<T>(P, mbase, t, g, gt < kyn ? gt : 0).pos, fstride);
        for (int j = gt; j < kyn; j += G) {
            const ModeCtx m = mode_ctx<T>(P, mbase, t, g, j);
            const int jn = j + G < kyn ? j + G : j;
            const PsiLoads<T> Ln = psi_loads<T>(P, A, alpha, mode_ctx<T>(P, mbase, t, g, jn).pos, fstride);
            a0[j] = psi_epilogue<T>(P, A, alpha, m, kx, kyu * static_cast<T>(m.ky), a0[j], mi, L, b);
            L = Ln;
        }
    } else {
        MomLoads<T> L = momentum_loads<T>(P, A, mode_ctx<T>(P, mbase, t, g, gt < kyn ? gt : 0).pos, fstride);
        for (int j = gt; j < kyn; j += G) {
            const ModeCtx m = mode_ctx<T>(P, mbase, t, g, j);
            const int jn = j + G < kyn ? j + G : j;
            const MomLoads<T> Ln = momentum_loads<T>(P, A, mode_ctx<T>(P, mbase, t, g, jn).pos, fstride);
            C u0 = a0[j], u1 = a1[j];
            momentum_epilogue<T>(P, A, m, kx, kyu * static_cast<T>(m.ky), u0, u1, mi, L, b);
            a0[j] = u0;
            a1[j] = u1;
            L = Ln;
        }
    }

    int nwf = 0;
    int wfield[3];
    if (gkind == GROUP_PSI) { wfield[nwf++] = 1 + alpha; }
    else { if (comp) wfield[nwf++] = 0; wfield[nwf++] = P.nop + 1; wfield[nwf++] = P.nop + 2; }
    for (int q = 0; q < nwf; ++q) {
        const int f = wfield[q];
        __syncthreads();  // previous field's I1 copy-out is done
        for (int y = gt; y < NY; y += G) line[y] = czero<C>();
        group_sync<G>(bid);
        C* dst = A.next + mbase + static_cast<size_t>(f) * fstride + static_cast<size_t>(g) * kyn;
        for (int j = gt; j < kyn; j += G) {
            const int ky = ky_of_j(j, nay);
            const int y = ky >= 0 ? ky : ky + NY;
            C v;
            if (f == 0) v = rho_epilogue<T>(P, A, mbase + static_cast<size_t>(g) * kyn + j, kx, kyu * static_cast<T>(ky), fstride);
            else v = (f == P.nop + 2) ? a1[j] : a0[j];
            line[sw7(y)] = v;
        }
        group_sync<G>(bid);
        // real-symmetry projection of the kx = 0 line (time_integrator.h:70-109)
        if (t == 0 && g == 0 && !A.det_mode) {
            for (int ky = gt; ky < nay / 2; ky += G) {
                if (ky == 0) {
                    line[0].y = T(0);
                } else {
                    C* pa = line + sw7(ky);
                    C* pc = line + sw7(NY - ky);
                    const C av = *pa, cv = *pc;
                    const C pj = mk(static_cast<T>(0.5) * (av.x + cv.x), static_cast<T>(0.5) * (av.y - cv.y));
                    *pa = pj;
                    *pc = cconj(pj);
                }
            }
            group_sync<G>(bid);
        }
        bool bad = false;
        for (int j = gt; j < kyn; j += G) {
            const int ky = ky_of_j(j, nay);
            const C v = line[sw7(ky >= 0 ? ky : ky + NY)];
            bad |= nonfinite2(v);
            dst[j] = v;
        }
        report_nonfinite(A.err, bad);
        const int slot = P.in_slot[f];
        if (A.fused_inverse && slot >= 0) {
            group_sync<G>(bid);
            gfft<NY, G, +1>(line, tw, gt, bid);
            __syncthreads();
            const T sc = static_cast<T>(P.inv_scale);
            C* o1 = A.i1_next + ((static_cast<size_t>(b) * P.n_in + slot) * P.ntiles + t) * static_cast<size_t>(NY) * W;
            for (int e = threadIdx.x; e < W * NY; e += kThreads) {
                const int y = e / W, w = e - y * W;
                o1[e] = cscale(tile[w * NY + sw7(y)], sc);
            }
        }
    }
}

}  // namespace shhd
