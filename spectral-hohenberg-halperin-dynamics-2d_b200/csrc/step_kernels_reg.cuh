// Register-resident FP32 pair-line transforms of 1536 points (the 3/2-rule compute grid of a
// 1024^2 active grid) and the row pass built on them.
//
// 1536 = 24 x 64.  A line group of 64 threads (two warps) owns one pair-line (two transform
// lines sharing each 16-byte element, as in step_kernels_pair.cuh), and each thread keeps 24
// positions in registers through three passes.  Forward (decimation in frequency):
//   pass A  thread j holds x[j + 64 q], q < 24: a 24-point DFT in registers (radix 3, the
//           constant twiddles w_24^(q8 k3), radix 8), then the twiddle w_1536^(j k1) from a
//           table, giving Y[j][k1];
//   pass B  thread (g, j1) (g = t / 8, j1 = t % 8) holds, for each of its three k1 = g + 8 i,
//           the values Y[j1 + 8 j2][k1], j2 < 8: radix 8 over j2, then the twiddle w_64^(j1 a);
//   pass C  thread (g, a) holds the pass-B values of the threads (g, j1), j1 < 8: radix 8 over
//           j1 gives X[k1 + 24 a + 192 b], b < 8.
// Pass A -> B crosses the group's two warps (shared memory and a 64-thread named barrier);
// B -> C stays inside a warp.  The inverse (decimation in time) runs the passes backwards
// (C', B', A') and leaves x[j + 64 q] in thread j: exactly the positions forward pass A starts
// from, so the row pass's pointwise products are formed at the positions each thread already
// holds.  Against the stage-per-barrier transforms of the pair-line kernels (four shared-memory
// round trips per line, one butterfly per thread at a time) this keeps two exchanges per line
// and gives every thread 24 independent points of work between them.
//
// Twiddles are exact FP32 roundings of FP64 values (a 1536-entry table for pass A, 64 entries
// for pass B, 15 compile-time constants inside pass A): no twiddle is formed by products.
#pragma once

#include "step_kernels_pair.cuh"

namespace shhd {

constexpr int kRegN = 1536;                 // points per line
constexpr int kRegM = 64;                   // threads per line group
constexpr int kRegQ = 24;                   // points per thread
constexpr int kRegGroups = 3;               // line groups per row-pass block
constexpr int kRegThreads = kRegGroups * kRegM;
constexpr int kRegChunk = 8 * kRegM;        // a group's exchange buffer: 8 rows of 64 pair elements (8 KB)
constexpr int kRegTwA = kRegM * kRegQ;      // TA[j][k1] = w_1536^(j k1)
constexpr int kRegTwB = 64;                 // TB[j1][a] = w_64^(j1 a)
constexpr int kRegTw = kRegTwA + kRegTwB;   // float2 entries of the table (forward sign)

// w_24^m = exp(-2 pi i m / 24), m = 0 .. 14, as (cos, -sin) of multiples of 15 degrees
__device__ __forceinline__ float2 w24(int m) {
    constexpr float c[15] = {1.0f, 0.96592582628906829f, 0.86602540378443865f, 0.70710678118654752f, 0.5f, 0.25881904510252076f, 0.0f,
                             -0.25881904510252076f, -0.5f, -0.70710678118654752f, -0.86602540378443865f, -0.96592582628906829f, -1.0f,
                             -0.96592582628906829f, -0.86602540378443865f};
    constexpr float s[15] = {0.0f, -0.25881904510252076f, -0.5f, -0.70710678118654752f, -0.86602540378443865f, -0.96592582628906829f, -1.0f,
                             -0.96592582628906829f, -0.86602540378443865f, -0.70710678118654752f, -0.5f, -0.25881904510252076f, 0.0f,
                             0.25881904510252076f, 0.5f};
    return make_float2(c[m], s[m]);
}

// register of Y[k1] after forward pass A (and of U[k1] before inverse pass A'): 8 (k1 % 3) + k1 / 3
__host__ __device__ constexpr int rreg(int k1) { return 8 * (k1 % 3) + k1 / 3; }

// slot of (row, column) in an exchange buffer of 64-element rows; the column's low three bits
// are XORed with its bits 3..5 so both exchange patterns spread over the banks
__device__ __forceinline__ int xidx(int row, int col) { return row * kRegM + (col ^ ((col >> 3) & 7)); }

// a * w (DIR < 0) or a * conj(w) (DIR > 0)
template <int DIR>
__device__ __forceinline__ PC cmul(PC a, float2 w) { return pcmul<DIR>(a, f2_splat(w.x), f2_splat(w.y)); }

// forward 24-point DFT over v[q] (q = q8 + 8 q3) -> v[8 k3 + k8] = Y[k3 + 3 k8]
template <int DIR>
__device__ __forceinline__ void r24_dif(PC* v) {
#pragma unroll
    for (int q8 = 0; q8 < 8; ++q8) {
        PC t[3] = {v[q8], v[q8 + 8], v[q8 + 16]};
        pbfly3<DIR>(t);
        v[q8] = t[0];
        v[q8 + 8] = t[1];
        v[q8 + 16] = t[2];
    }
#pragma unroll
    for (int k3 = 1; k3 < 3; ++k3)
#pragma unroll
        for (int q8 = 1; q8 < 8; ++q8) v[8 * k3 + q8] = cmul<DIR>(v[8 * k3 + q8], w24(q8 * k3));
#pragma unroll
    for (int k3 = 0; k3 < 3; ++k3) pbfly8<DIR>(v + 8 * k3);
}

// inverse of the above layout: v[8 k3 + k8] = U[k3 + 3 k8] -> v[q] = sum_k1 U[k1] w_24^(DIR q k1)
template <int DIR>
__device__ __forceinline__ void r24_dit(PC* v) {
#pragma unroll
    for (int k3 = 0; k3 < 3; ++k3) pbfly8<DIR>(v + 8 * k3);
#pragma unroll
    for (int k3 = 1; k3 < 3; ++k3)
#pragma unroll
        for (int q8 = 1; q8 < 8; ++q8) v[8 * k3 + q8] = cmul<DIR>(v[8 * k3 + q8], w24(q8 * k3));
#pragma unroll
    for (int q8 = 0; q8 < 8; ++q8) {
        PC t[3] = {v[q8], v[q8 + 8], v[q8 + 16]};
        pbfly3<DIR>(t);
        v[q8] = t[0];
        v[q8 + 8] = t[1];
        v[q8 + 16] = t[2];
    }
}

// twiddles w_1536^(j k1) of thread j's row (two per 16-byte load), applied to v[rreg(k1)]
template <int DIR>
__device__ __forceinline__ void twiddle_a(PC* v, const float2* __restrict__ ta_row) {
    const float4* t4 = reinterpret_cast<const float4*>(ta_row);
#pragma unroll
    for (int h = 0; h < kRegQ / 2; ++h) {
        float4 w;
        asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(w.x), "=f"(w.y), "=f"(w.z), "=f"(w.w) : "l"(t4 + h));
        if (h > 0) v[rreg(2 * h)] = cmul<DIR>(v[rreg(2 * h)], make_float2(w.x, w.y));
        v[rreg(2 * h + 1)] = cmul<DIR>(v[rreg(2 * h + 1)], make_float2(w.z, w.w));
    }
}

// twiddles w_64^(j1 a), a = 1 .. 7
template <int DIR>
__device__ __forceinline__ void twiddle_b(PC* w8, const float2* __restrict__ tb_row) {
    const float4* t4 = reinterpret_cast<const float4*>(tb_row);
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        float4 w;
        asm("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(w.x), "=f"(w.y), "=f"(w.z), "=f"(w.w) : "l"(t4 + h));
        if (h > 0) w8[2 * h] = cmul<DIR>(w8[2 * h], make_float2(w.x, w.y));
        w8[2 * h + 1] = cmul<DIR>(w8[2 * h + 1], make_float2(w.z, w.w));
    }
}

__device__ __forceinline__ void group_bar(int grp) { asm volatile("bar.sync %0, %1;" ::"r"(1 + grp), "r"(kRegM) : "memory"); }

// read-only 16-byte load (L1-cached: a neighbouring thread uses the other half of the element)
__device__ __forceinline__ ulonglong2 ld_ro(const ulonglong2* p) {
    ulonglong2 v;
    asm("ld.global.nc.v2.u64 {%0, %1}, [%2];" : "=l"(v.x), "=l"(v.y) : "l"(p));
    return v;
}

// ---------------------------------------------------------------------------
// row pass on 1536-point rows: I1 -> x-inverse -> products -> x-forward -> I2
// (grid: row pairs x batch; three line groups per block).  Shared memory: the row pair's
// physical input pair-lines [nip][1536] (each also the exchange buffer of its own inverse),
// then one 8 KB exchange buffer per group for the forward transforms.
// ---------------------------------------------------------------------------
// NR = untangling rounds of 192 positions = ceil(Hx / 384): 2 (2x rule), 3 (3/2 rule), 4 (none)
template <int NR>
__global__ void __launch_bounds__(kRegThreads, 2) rrow_pass1536(const StepPlan P, const MemberInfo* __restrict__ members,
                                                                const ulonglong2* __restrict__ i1, ulonglong2* __restrict__ i2,
                                                                const float2* __restrict__ tw, const double* __restrict__ rho0_member,
                                                                int* __restrict__ err) {
    constexpr int N = kRegN;
    const int b = blockIdx.y;
    if (!members[b].active) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nip = (P.n_in + 1) >> 1;
    ulonglong2* inl = reinterpret_cast<ulonglong2*>(smem_raw);  // [nip][N]
    const int grp = threadIdx.x >> 6, gt = threadIdx.x & (kRegM - 1);
    const int g = gt >> 3, l8 = gt & 7;                          // pass B / C roles (l8 = j1 in B, a in C)
    ulonglong2* E = inl + static_cast<size_t>(nip) * N + grp * kRegChunk;
    const int npy = P.npy, hx = P.hx, hp = hx >> 1;
    const int y0 = 2 * blockIdx.x;
    const size_t plane = static_cast<size_t>(P.ntiles) * npy;
    const ulonglong2* i1m = i1 + static_cast<size_t>(b) * P.n_in * plane;
    ulonglong2* i2m = i2 + static_cast<size_t>(b) * P.n_out * plane;
    const float2* ta_row = tw + gt * kRegQ;
    const float2* tb_row = tw + kRegTwA + l8 * 8;

    // 1. x-inverse of each input pair-line (slots 2l, 2l + 1) by one group, in place in its line
    for (int l = grp; l < nip; l += kRegGroups) {
        ulonglong2* L = inl + static_cast<size_t>(l) * N;
        const int sa = 2 * l, sb = 2 * l + 1;
        const bool has_b = sb < P.n_in;
        // Z[k] = X0[k] + i X1[k] (rows y0, y0 + 1) with the Hermitian mirror Z[N - k] =
        // conj X0[k] + i conj X1[k], zero for Hx <= k <= N - Hx: staged in natural order with
        // coalesced loads (each thread one tile, both of its columns)
        for (int t = gt; t < hp; t += kRegM) {
            const ulonglong2* pa = i1m + static_cast<size_t>(sa) * plane + static_cast<size_t>(t) * npy + y0;
            const ulonglong2 a0 = ld_stream(pa), a1 = ld_stream(pa + 1);
            ulonglong2 b0 = make_ulonglong2(0ull, 0ull), b1 = b0;
            if (has_b) {
                const ulonglong2* pb = i1m + static_cast<size_t>(sb) * plane + static_cast<size_t>(t) * npy + y0;
                b0 = ld_stream(pb);
                b1 = ld_stream(pb + 1);
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int k = 2 * t + h;
                float xa0r = h ? f2_hi(a0.x) : f2_lo(a0.x), xa0i = h ? f2_hi(a0.y) : f2_lo(a0.y);
                float xa1r = h ? f2_hi(a1.x) : f2_lo(a1.x), xa1i = h ? f2_hi(a1.y) : f2_lo(a1.y);
                float xb0r = h ? f2_hi(b0.x) : f2_lo(b0.x), xb0i = h ? f2_hi(b0.y) : f2_lo(b0.y);
                float xb1r = h ? f2_hi(b1.x) : f2_lo(b1.x), xb1i = h ? f2_hi(b1.y) : f2_lo(b1.y);
                if (k == 0) { xa0i = 0.f; xa1i = 0.f; xb0i = 0.f; xb1i = 0.f; }
                st_pc(L + psw(k), PC{f2_pack(xa0r - xa1i, xb0r - xb1i), f2_pack(xa0i + xa1r, xb0i + xb1r)});
                if (k > 0) st_pc(L + psw(N - k), PC{f2_pack(xa0r + xa1i, xb0r + xb1i), f2_pack(xa1r - xa0i, xb1r - xb0i)});
            }
        }
        for (int k = hx + gt; k <= N - hx; k += kRegM) st_pc(L + psw(k), pc_zero());
        group_bar(grp);
        // pass C' (thread (g, a = l8)): Z at k = k1 + 24 a + 192 b, radix 8 over b
        PC u[3][8];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int bb = 0; bb < 8; ++bb) u[i][bb] = ld_pc(L + psw(g + 8 * i + 24 * l8 + 192 * bb));
        group_bar(grp);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int k1 = g + 8 * i;
            pbfly8<+1>(u[i]);
#pragma unroll
            for (int j1 = 0; j1 < 8; ++j1) st_pc(L + xidx(k1, j1 + 8 * l8), u[i][j1]);
        }
        __syncwarp();
        // pass B' (thread (g, j1 = l8)): twiddle conj w_64^(j1 a), radix 8 over a; each lane
        // rewrites only the columns it read
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const int k1 = g + 8 * i;
            PC w[8];
#pragma unroll
            for (int a = 0; a < 8; ++a) w[a] = ld_pc(L + xidx(k1, l8 + 8 * a));
            twiddle_b<+1>(w, tb_row);
            pbfly8<+1>(w);
#pragma unroll
            for (int j2 = 0; j2 < 8; ++j2) st_pc(L + xidx(k1, l8 + 8 * j2), w[j2]);
        }
        group_bar(grp);
        // pass A' (thread j = gt): twiddle conj w_1536^(j k1), inverse 24-point DFT
        PC v[kRegQ];
#pragma unroll
        for (int k1 = 0; k1 < kRegQ; ++k1) v[rreg(k1)] = ld_pc(L + xidx(k1, gt));
        twiddle_a<+1>(v, ta_row);
        r24_dit<+1>(v);
        group_bar(grp);
#pragma unroll
        for (int q = 0; q < kRegQ; ++q) st_pc(L + psw(gt + kRegM * q), v[q]);
    }
    __syncthreads();

    // 2. velocity inputs (compressible: v = j / rho with the zero-density check; otherwise
    //    v = j / rho0 in the products)
    const bool comp = (P.mode == 0);
    const float inv_rho0 = (P.need_v && !comp) ? static_cast<float>(1.0 / rho0_member[b]) : 0.f;
    if (P.need_v && comp) {
        row_velocity_prep<N>(P, inl, 1, nip, threadIdx.x, kRegThreads, err);
        __syncthreads();
    }

    // 3. per output pair (one group each): products at the thread's own positions, forward
    //    transform, untangling of the two rows, I2 store
    const u64 HALF = f2_splat(0.5f);
    for (int pi = grp; pi < P.rp_n; pi += kRegGroups) {
        const int oa = P.rp_a[pi], ob = P.rp_b[pi];
        const RowProduct R = row_product(P, pi, inv_rho0);
        PC v[kRegQ];  // the plan selects this kernel only for the canonical input roles (P.rp_canon)
#pragma unroll
        for (int q = 0; q < kRegQ; ++q) v[q] = row_product_canon<N>(P, R, inl, psw(gt + kRegM * q));
        // pass A
        r24_dif<-1>(v);
        twiddle_a<-1>(v, ta_row);
        // passes B and C, one slot i (k1 = g' + 8 i) at a time through the 8-row buffer
        PC xc[3][8];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
#pragma unroll
            for (int gp = 0; gp < 8; ++gp) st_pc(E + xidx(gp, gt), v[rreg(gp + 8 * i)]);
            group_bar(grp);
            PC w[8];
#pragma unroll
            for (int j2 = 0; j2 < 8; ++j2) w[j2] = ld_pc(E + xidx(g, l8 + 8 * j2));
            pbfly8<-1>(w);
            twiddle_b<-1>(w, tb_row);
#pragma unroll
            for (int a = 0; a < 8; ++a) st_pc(E + xidx(g, l8 + 8 * a), w[a]);
            __syncwarp();
#pragma unroll
            for (int j1 = 0; j1 < 8; ++j1) w[j1] = ld_pc(E + xidx(g, j1 + 8 * l8));
            pbfly8<-1>(w);
#pragma unroll
            for (int bb = 0; bb < 8; ++bb) xc[i][bb] = w[bb];
            group_bar(grp);
        }
        // untangle, 192 positions k at a time: Zs[m] = Z[192 r + m] at E[psw(m)] and
        // Ms[m] = Z[N - 192 r - m] at E[256 + psw(m)]; then
        //   G0[k] = (Z[k] + conj Z[N-k]) / 2 (row y0), G1[k] = -i (Z[k] - conj Z[N-k]) / 2 (row y0 + 1)
#pragma unroll
        for (int r = 0; r < NR; ++r) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const int m = g + 8 * i + 24 * l8;
                st_pc(E + psw(m), xc[i][r]);
                if (m > 0) st_pc(E + 256 + psw(192 - m), xc[i][7 - r]);
            }
            if (gt == 0) st_pc(E + 256 + psw(0), xc[0][(8 - r) & 7]);
            group_bar(grp);
            const int tend = min(96 * (r + 1), hp);
            for (int t = 96 * r + gt; t < tend; t += kRegM) {
                u64 g0r[2], g0i[2], g1r[2], g1i[2];
#pragma unroll
                for (int w = 0; w < 2; ++w) {
                    const int m = 2 * t + w - 192 * r;
                    const PC zk = ld_pc(E + psw(m));
                    const PC zn = ld_pc(E + 256 + psw(m));
                    g0r[w] = f2_mul(f2_add(zk.re, zn.re), HALF);
                    g0i[w] = f2_mul(f2_sub(zk.im, zn.im), HALF);
                    g1r[w] = f2_mul(f2_add(zk.im, zn.im), HALF);   //  (d.im) / 2, d = Z[k] - conj Z[N-k]
                    g1i[w] = f2_mul(f2_sub(zn.re, zk.re), HALF);   // -(d.re) / 2
                }
                ulonglong2* qa = i2m + static_cast<size_t>(oa) * plane + static_cast<size_t>(t) * npy + y0;
                qa[0] = make_ulonglong2(f2_pack(f2_lo(g0r[0]), f2_lo(g0r[1])), f2_pack(f2_lo(g0i[0]), f2_lo(g0i[1])));
                qa[1] = make_ulonglong2(f2_pack(f2_lo(g1r[0]), f2_lo(g1r[1])), f2_pack(f2_lo(g1i[0]), f2_lo(g1i[1])));
                if (ob >= 0) {
                    ulonglong2* qb = i2m + static_cast<size_t>(ob) * plane + static_cast<size_t>(t) * npy + y0;
                    qb[0] = make_ulonglong2(f2_pack(f2_hi(g0r[0]), f2_hi(g0r[1])), f2_pack(f2_hi(g0i[0]), f2_hi(g0i[1])));
                    qb[1] = make_ulonglong2(f2_pack(f2_hi(g1r[0]), f2_hi(g1r[1])), f2_pack(f2_hi(g1i[0]), f2_hi(g1i[1])));
                }
            }
            group_bar(grp);
        }
    }
}

// host: the table TA then TB (forward sign, FP64 values rounded once)
inline void reg_twiddles_host(float* out /* 2 * kRegTw floats */) {
    for (int j = 0; j < kRegM; ++j)
        for (int k1 = 0; k1 < kRegQ; ++k1) {
            const double a = -2.0 * M_PI * static_cast<double>(j * k1) / kRegN;
            out[2 * (j * kRegQ + k1)] = static_cast<float>(cos(a));
            out[2 * (j * kRegQ + k1) + 1] = static_cast<float>(sin(a));
        }
    for (int j1 = 0; j1 < 8; ++j1)
        for (int a = 0; a < 8; ++a) {
            const double ang = -2.0 * M_PI * static_cast<double>(j1 * a) / 64.0;
            out[2 * (kRegTwA + j1 * 8 + a)] = static_cast<float>(cos(ang));
            out[2 * (kRegTwA + j1 * 8 + a) + 1] = static_cast<float>(sin(ang));
        }
}

}  // namespace shhd
