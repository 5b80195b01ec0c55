// Row pass over two output pairs at a time (kernel family 4): FP32 pair-line sizes, compressible
// dynamics with the canonical (rho, jx), (jy, -) input pair-lines.
//
// prow_pass transforms one output pair at a time through one work line: every pair is a chain
// of barriers (products with the first stage, the remaining stages, the untangling), its
// radix-8 stages run by 192 of the 256 threads, each thread reading the pair's inputs and
// forming its twiddle powers alone.  prow_pass2 keeps 1 / rho in an 8-byte slot per position
// instead of (vx, vy) in a full line, which frees the (jy, -) line after the velocity
// preparation as a second work line.  Each thread then
//   - reads a position's inputs once and evaluates the products of two output pairs from them,
//   - runs the same butterfly of both lines with one set of twiddle powers,
//   - untangles both lines in one pass,
// so the forward transforms take half as many barrier chains.  Each output's arithmetic is
// prow_pass's, operation for operation (v = j * (1 / rho), one rounding either way).
// Shared memory per row pair: nip input pair-lines, one more work line and NX 1 / rho slots
// (110.6 KB at 1536 points with three input pair-lines: two blocks per SM).
#pragma once

#include "step_kernels_pair.cuh"

namespace shhd {

template <int NX>
constexpr size_t prow2_smem_bytes(int nip) {
    return static_cast<size_t>(kPairMaxN / NX) * NX * ((nip + 1) * sizeof(ulonglong2) + sizeof(u64));
}

// one stage of two lines (line l of A at a + l * as, of B at b + l * bs): the same butterfly
// of both, with one set of twiddle powers
template <int N, int S, int DIR, bool DIT, typename TW>
__device__ __forceinline__ void pstage2(int nl, ulonglong2* a, size_t as, ulonglong2* b, size_t bs, TW tw) {
    constexpr PPlan pp = PairPlan<N>::c;
    constexpr int R = pp.r[S], ST = pp.s[S], L = R * ST, NB = N / R;
#pragma unroll 1
    for (int bi = threadIdx.x; bi < nl * NB; bi += kThreads) {
        const int l = bi / NB, i = bi - l * NB;
        const int j = i & (ST - 1);
        const int base = (i >> pp.lg[S]) * L + j;
        ulonglong2* la = a + l * as;
        ulonglong2* lb = b + l * bs;
        PC va[R], vb[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            va[q] = ld_pc(la + psw(base + q * ST));
            vb[q] = ld_pc(lb + psw(base + q * ST));
        }
        float2 w[8];
        if constexpr (L > R) ptwiddle_powers<R>(tw_at(tw, pp.twoff[S] + j), w);
        if constexpr (DIT && L > R) {
            ptwiddle_apply<R, DIR>(va, w);
            ptwiddle_apply<R, DIR>(vb, w);
        }
        pbfly<R, DIR>(va);
        pbfly<R, DIR>(vb);
        if constexpr (!DIT && L > R) {
            ptwiddle_apply<R, DIR>(va, w);
            ptwiddle_apply<R, DIR>(vb, w);
        }
#pragma unroll
        for (int q = 0; q < R; ++q) {
            st_pc(la + psw(base + q * ST), va[q]);
            st_pc(lb + psw(base + q * ST), vb[q]);
        }
    }
}
// DIT stages S - 1 down to E of two lines, a barrier after each
template <int N, int S, int E, int DIR, typename TW>
__device__ __forceinline__ void pdit2_range(int nl, ulonglong2* a, size_t as, ulonglong2* b, size_t bs, TW tw) {
    if constexpr (S > E) {
        pstage2<N, S - 1, DIR, true>(nl, a, as, b, bs, tw);
        __syncthreads();
        pdit2_range<N, S - 1, E, DIR>(nl, a, as, b, bs, tw);
    }
}

template <int NX>
__global__ void __launch_bounds__(kThreads, 2) prow_pass2(const StepPlan P, const MemberInfo* __restrict__ members,
                                                       const ulonglong2* __restrict__ i1, ulonglong2* __restrict__ i2,
                                                       const float2* __restrict__ tw, int* __restrict__ err) {
    if (!members[blockIdx.y].active) return;
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
    constexpr int RL = pp.r[pp.m - 1], NBL = NX / RL;  // first forward stage: radix, butterflies (stride 1, no twiddles)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nip = (P.n_in + 1) >> 1;
    const int m = P.rp_jline;                                            // (rho, jx); (jy, -) is line m + 1 = nip - 1
    ulonglong2* inl = reinterpret_cast<ulonglong2*>(smem_raw);          // [RP][nip][NX]
    ulonglong2* workb = inl + static_cast<size_t>(RP) * nip * NX;       // [RP][NX]
    u64* irho = reinterpret_cast<u64*>(workb + static_cast<size_t>(RP) * NX);  // [RP][NX]: 1 / rho of rows y0, y0 + 1
    ulonglong2* worka = inl + static_cast<size_t>(nip - 1) * NX;        // the (jy, -) line of each row pair
    const size_t as = static_cast<size_t>(nip) * NX, bs = NX;
    const int b = blockIdx.y, pair0 = blockIdx.x * RP;
    const size_t plane = static_cast<size_t>(P.ntiles) * P.npy;
    const ulonglong2* i1m = i1 + static_cast<size_t>(b) * P.n_in * plane;
    ulonglong2* i2m = i2 + static_cast<size_t>(b) * P.n_out * plane;

    // 1. inputs: Z staging and x-inverse
    prow_inputs<NX>(P, i1m, plane, inl, nip, pair0, tw);

    // 2. (rho, jx), (jy, -) -> (jx, jy) in line m and 1 / rho per position, with the
    //    zero-density check of fcalculator_workspace.cc:122-133
    {
        int bad = 0;
        for (int e = threadIdx.x; e < RP * NX; e += kThreads) {
            const int r = e / NX, x = e - r * NX;
            ulonglong2* pj = inl + (static_cast<size_t>(r) * nip + m) * NX + x;
            const ulonglong2 rj = pj[0], jy = pj[NX];
            const float r0 = f2_lo(rj.x), r1 = f2_lo(rj.y);
            if (r0 == 0.f || r1 == 0.f) bad = 1;
            irho[e] = f2_pack(1.f / r0, 1.f / r1);
            pj[0] = make_ulonglong2(f2_pack(f2_hi(rj.x), f2_lo(jy.x)), f2_pack(f2_hi(rj.y), f2_lo(jy.y)));
        }
        if (bad) atomicOr(err, ERR_ZERO_DENSITY);
    }
    __syncthreads();
    // (jx, jy) and (vx, vy) at slot sp of row pair r
    auto jv_at = [&](int r, int sp) {
        const ulonglong2 J = inl[(static_cast<size_t>(r) * nip + m) * NX + sp];
        const u64 ir = irho[static_cast<size_t>(r) * NX + sp];
        return JV{J, make_ulonglong2(f2_mul(J.x, f2_splat(f2_lo(ir))), f2_mul(J.y, f2_splat(f2_hi(ir))))};
    };

    // 3. output pairs two at a time: both pairs' products from one read of a position's inputs,
    //    fused into the first DIT stage; both lines' remaining stages; both untangled
    int pi = 0;
    for (; pi + 1 < P.rp_n; pi += 2) {
        const RowProduct RA = row_product(P, pi, 0.f), RB = row_product(P, pi + 1, 0.f);
#pragma unroll 1
        for (int bi = threadIdx.x; bi < RP * NBL; bi += kThreads) {
            const int r = bi / NBL, i = bi - r * NBL;
            const ulonglong2* in = inl + static_cast<size_t>(r) * nip * NX;
            PC va[RL], vb[RL];
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                const int sp = psw(i * RL + q);
                const JV jv = jv_at(r, sp);
                va[q] = row_product_canon<NX>(P, RA, in, sp, [&] { return jv; });
                vb[q] = row_product_canon<NX>(P, RB, in, sp, [&] { return jv; });
            }
            pbfly<RL, -1>(va);
            pbfly<RL, -1>(vb);
            ulonglong2* la = worka + r * as;
            ulonglong2* lb = workb + r * bs;
#pragma unroll
            for (int q = 0; q < RL; ++q) {
                st_pc(la + psw(i * RL + q), va[q]);
                st_pc(lb + psw(i * RL + q), vb[q]);
            }
        }
        __syncthreads();
        pdit2_range<NX, pp.m - 1, 0, -1>(RP, worka, as, workb, bs, tw);
        prow_untangle<NX>(P, 2, OutLine{worka, as, P.rp_a[pi], P.rp_b[pi]}, OutLine{workb, bs, P.rp_a[pi + 1], P.rp_b[pi + 1]},
                          i2m, plane, pair0);
        __syncthreads();
    }
    if (pi < P.rp_n) {  // an odd last pair: line B alone
        const RowProduct R = row_product(P, pi, 0.f);
        pstage_io<NX, pp.m - 1, -1, true>(RP, tw, [&](int r, int p) -> PC {
            const int sp = psw(p);
            return row_product_canon<NX>(P, R, inl + static_cast<size_t>(r) * nip * NX, sp, [&] { return jv_at(r, sp); });
        }, SmemIO{workb, NX});
        __syncthreads();
        pdit_range<NX, pp.m - 1, 0, -1>(workb, RP, tw);
        const OutLine W{workb, bs, P.rp_a[pi], P.rp_b[pi]};
        prow_untangle<NX>(P, 1, W, W, i2m, plane, pair0);
    }
}

}  // namespace shhd
