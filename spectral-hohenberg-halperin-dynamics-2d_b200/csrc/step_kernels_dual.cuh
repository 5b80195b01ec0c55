// Row pass over two output pairs at a time (kernel family 4): FP32 pair-line sizes, compressible
// dynamics with the canonical (rho, jx), (jy, -) input pair-lines.
//
// prow_pass transforms one output pair at a time through one work line: every pair is a chain
// of barriers (products with the first stage, the remaining stages, the untangling) whose
// radix-8 stages keep 192 of its 256 threads busy, at 16 warps per SM (two blocks).
// prow_pass2 keeps 1 / rho in an 8-byte slot per position instead of (vx, vy) in a full line,
// which frees the (jy, -) line after the velocity preparation as a second work line, and runs
// 384 threads (two blocks per SM: 24 warps): the two output pairs of a round are the two lines
// of one stage, 2 x 192 radix-8 butterflies, one per thread, so the forward transforms take
// half as many barrier chains with every thread busy in their radix-8 stages.  Each output's
// arithmetic is prow_pass's, operation for operation (v = j * (1 / rho), one rounding either way).
// Shared memory per row pair: nip input pair-lines, one more work line and NX 1 / rho slots
// (110.6 KB at 1536 points with three input pair-lines); 80 registers per thread.
#pragma once

#include "step_kernels_pair.cuh"

namespace shhd {

template <int NX>
constexpr size_t prow2_smem_bytes(int nip) {
    return static_cast<size_t>(kPairMaxN / NX) * NX * ((nip + 1) * sizeof(ulonglong2) + sizeof(u64));
}

// block size of the two-pair row pass
constexpr int kDualThreads = 384;

// slot of position slot x in a row pair's 1 / rho array (8-byte entries): bit 3 flipped by bit 6.
// The first forward stage at 1536 points reads positions 8 i + (q ^ (i & 7)) for consecutive
// i, which put lanes i and i + 8 of a half warp in one bank pair of a plain array
__device__ __forceinline__ int irho_slot(int x) { return x ^ ((x >> 3) & 8); }

// the two work lines of a round as lines l = 2 r + q of one stage: output pair q of row pair r
struct DualIO {
    static constexpr bool kSlots = true;
    ulonglong2* a;
    size_t as;
    ulonglong2* b;
    size_t bs;
    __device__ __forceinline__ ulonglong2* line(int l) const { return (l & 1) ? b + (l >> 1) * bs : a + (l >> 1) * as; }
    __device__ __forceinline__ PC operator()(int l, int p) const { return ld_pc(line(l) + psw(p)); }
    __device__ __forceinline__ void operator()(int l, int p, PC v) const { st_pc(line(l) + psw(p), v); }
};

template <int NX>
__global__ void __launch_bounds__(kDualThreads, 2) prow_pass2(const StepPlan P, const MemberInfo* __restrict__ members,
                                                           const ulonglong2* __restrict__ i1, ulonglong2* __restrict__ i2,
                                                           const float2* __restrict__ tw, int* __restrict__ err) {
    if (!members[blockIdx.y].active) return;
    constexpr int NT = kDualThreads;
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
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
    prow_inputs<NX, NT>(P, i1m, plane, inl, nip, pair0, tw);

    // 2. (rho, jx), (jy, -) -> (jx, jy) in line m and 1 / rho per position, with the
    //    zero-density check of fcalculator_workspace.cc:122-133
    {
        int bad = 0;
        for (int e = threadIdx.x; e < RP * NX; e += NT) {
            const int r = e / NX, x = e - r * NX;
            ulonglong2* pj = inl + (static_cast<size_t>(r) * nip + m) * NX + x;
            const ulonglong2 rj = pj[0], jy = pj[NX];
            const float r0 = f2_lo(rj.x), r1 = f2_lo(rj.y);
            if (r0 == 0.f || r1 == 0.f) bad = 1;
            irho[static_cast<size_t>(r) * NX + irho_slot(x)] = f2_pack(1.f / r0, 1.f / r1);
            pj[0] = make_ulonglong2(f2_pack(f2_hi(rj.x), f2_lo(jy.x)), f2_pack(f2_hi(rj.y), f2_lo(jy.y)));
        }
        if (bad) atomicOr(err, ERR_ZERO_DENSITY);
    }
    __syncthreads();
    // (jx, jy) and (vx, vy) at slot sp of row pair r
    auto jv_at = [&](int r, int sp) {
        const ulonglong2 J = inl[(static_cast<size_t>(r) * nip + m) * NX + sp];
        const u64 ir = irho[static_cast<size_t>(r) * NX + irho_slot(sp)];
        return JV{J, make_ulonglong2(f2_mul(J.x, f2_splat(f2_lo(ir))), f2_mul(J.y, f2_splat(f2_hi(ir))))};
    };

    // 3. output pairs two at a time, as the two lines of each stage: products fused into the
    //    first DIT stage (stride 1, no twiddles), the remaining stages, both untangled
    const DualIO io{worka, as, workb, bs};
    int pi = 0;
    for (; pi + 1 < P.rp_n; pi += 2) {
        pstage_io<NX, pp.m - 1, -1, true, NT>(2 * RP, tw, [&](int l, int p) -> PC {
            const int r = l >> 1, sp = psw(p);
            const RowProduct R = row_product(P, pi + (l & 1), 0.f);
            return row_product_canon<NX>(P, R, inl + static_cast<size_t>(r) * nip * NX, sp, [&] { return jv_at(r, sp); });
        }, io);
        __syncthreads();
        pdit_range_io<NX, pp.m - 1, 0, -1, NT>(io, 2 * RP, tw);
        prow_untangle<NX, NT>(P, 2, OutLine{worka, as, P.rp_a[pi], P.rp_b[pi]}, OutLine{workb, bs, P.rp_a[pi + 1], P.rp_b[pi + 1]},
                              i2m, plane, pair0);
        __syncthreads();
    }
    if (pi < P.rp_n) {  // an odd last pair: line B alone
        const RowProduct R = row_product(P, pi, 0.f);
        pstage_io<NX, pp.m - 1, -1, true, NT>(RP, tw, [&](int r, int p) -> PC {
            const int sp = psw(p);
            return row_product_canon<NX>(P, R, inl + static_cast<size_t>(r) * nip * NX, sp, [&] { return jv_at(r, sp); });
        }, SmemIO{workb, NX});
        __syncthreads();
        pdit_range<NX, pp.m - 1, 0, -1, NT>(workb, RP, tw);
        const OutLine W{workb, bs, P.rp_a[pi], P.rp_b[pi]};
        prow_untangle<NX, NT>(P, 1, W, W, i2m, plane, pair0);
    }
}

}  // namespace shhd
