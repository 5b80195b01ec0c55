// Split row pass for the FP32 pair-line sizes (kernel family 3): the pair-line row pass
// (prow_pass) as two kernels with a physical-row buffer between them.
//
// prow_pass keeps a row pair's physical input pair-lines and a work line in shared memory
// (98 KB at 1536 points), which allows two blocks per SM and makes every block a long chain
// of barriers: x-inverse of all inputs, then each output pair's forward transform in turn.
// Here
//   prow_inverse   (row pairs x input pair-lines x members): one pair-line's x-inverse,
//                  written to phys[member][row pair][pair-line][N] (the same slot order and
//                  swizzle as prow_pass's shared lines; the density half replaced by 1 / rho
//                  when the products need v = j / rho, with the zero-density check);
//   prow_forward   (row pairs x output pairs x members): one output pair's products, read from
//                  phys at the positions its first forward stage needs, the forward transform
//                  and the untangling into I2.
// Each block holds one line per row pair (24 KB at 1536 points), so many blocks share an SM
// and their barrier chains overlap.  The physical rows (57 MB at the 1024^2 N = 2 workload)
// are written once and read by each output pair that uses them; at that size they do not stay
// in L2 (63 MB of DRAM reads per forward launch), and the family is slower than prow_pass there.
#pragma once

#include "step_kernels_pair.cuh"

namespace shhd {

// row-pass physical buffer: pair elements per member
__host__ __device__ inline size_t phys_member_elems(const StepPlan& P) {
    return static_cast<size_t>(P.npy / 2) * ((P.n_in + 1) / 2) * P.npx;
}

template <int NX>
__global__ void __launch_bounds__(kThreads) prow_inverse(const StepPlan P, const MemberInfo* __restrict__ members,
                                                        const ulonglong2* __restrict__ i1, ulonglong2* __restrict__ phys,
                                                        const float2* __restrict__ tw, int* __restrict__ err) {
    const int b = blockIdx.z;
    if (!members[b].active) return;
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ulonglong2* lines = reinterpret_cast<ulonglong2*>(smem_raw);  // [RP][NX]
    const int npy = P.npy, hx = P.hx, hp = hx >> 1;
    const int nip = (P.n_in + 1) >> 1;
    const int ip = blockIdx.y, pair0 = blockIdx.x * RP;
    const size_t plane = static_cast<size_t>(P.ntiles) * npy;
    const ulonglong2* i1m = i1 + static_cast<size_t>(b) * P.n_in * plane;

    // Z[k] = X0[k] + i X1[k] (rows y0, y0 + 1) with the Hermitian mirror Z[N - k]; kx = 0 real parts
    const int nz = RP * hp;
    for (int e0 = threadIdx.x; e0 < nz; e0 += kZBatch * kThreads) {
        ZItem z[kZBatch];
#pragma unroll
        for (int u = 0; u < kZBatch; ++u) {
            const int e = e0 + u * kThreads;
            if (e < nz) {
                const int r = e / hp, t = e - r * hp;
                z[u] = pz_load(i1m, plane, npy, P.n_in, ip, t, 2 * (pair0 + r));
            }
        }
#pragma unroll
        for (int u = 0; u < kZBatch; ++u) {
            const int e = e0 + u * kThreads;
            if (e < nz) {
                const int r = e / hp, t = e - r * hp;
                pz_store<NX>(lines + static_cast<size_t>(r) * NX, t, z[u]);
            }
        }
    }
    const int nzero = NX - 2 * hx + 1;  // k in [hx, NX - hx]
    for (int e = threadIdx.x; e < RP * nzero; e += kThreads) {
        const int r = e / nzero, k = hx + (e - r * nzero);
        st_pc(lines + static_cast<size_t>(r) * NX + psw(k), pc_zero());
    }
    __syncthreads();
    pdif_range<NX, 0, pp.m - 1, +1>(lines, RP, tw);

    // last stage straight to phys; the density half becomes 1 / rho where v = j / rho is needed
    const int s_rho = P.in_slot[0];
    const bool recip = P.need_v && P.mode == 0 && s_rho >= 0 && (s_rho >> 1) == ip;
    const int h = s_rho & 1;
    const size_t npairs = static_cast<size_t>(npy / 2);
    ulonglong2* out = phys + (static_cast<size_t>(b) * npairs + pair0) * nip * NX + static_cast<size_t>(ip) * NX;
    int bad = 0;
    pstage_io<NX, pp.m - 1, +1, false>(RP, tw, SmemIO{lines, NX}, [&](int l, int p, PC v) {
        if (recip) {
            const float r0 = h ? f2_hi(v.re) : f2_lo(v.re), r1 = h ? f2_hi(v.im) : f2_lo(v.im);
            if (r0 == 0.f || r1 == 0.f) bad = 1;
            if (h) { v.re = f2_pack(f2_lo(v.re), 1.f / r0); v.im = f2_pack(f2_lo(v.im), 1.f / r1); }
            else { v.re = f2_pack(1.f / r0, f2_hi(v.re)); v.im = f2_pack(1.f / r1, f2_hi(v.im)); }
        }
        st_pc(out + static_cast<size_t>(l) * nip * NX + psw(p), v);
    });
    if (bad) atomicOr(err, ERR_ZERO_DENSITY);
}

template <int NX>
__global__ void __launch_bounds__(kThreads) prow_forward(const StepPlan P, const MemberInfo* __restrict__ members,
                                                        const ulonglong2* __restrict__ phys, ulonglong2* __restrict__ i2,
                                                        const float2* __restrict__ tw, const double* __restrict__ rho0_member) {
    const int b = blockIdx.z;
    if (!members[b].active) return;
    constexpr int RP = kPairMaxN / NX;
    constexpr PPlan pp = PairPlan<NX>::c;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    ulonglong2* work = reinterpret_cast<ulonglong2*>(smem_raw);  // [RP][NX]
    const int npy = P.npy;
    const int nip = (P.n_in + 1) >> 1;
    const int pi = blockIdx.y, pair0 = blockIdx.x * RP;
    const size_t plane = static_cast<size_t>(P.ntiles) * npy;
    ulonglong2* i2m = i2 + static_cast<size_t>(b) * P.n_out * plane;
    const size_t npairs = static_cast<size_t>(npy / 2);
    const ulonglong2* inm = phys + (static_cast<size_t>(b) * npairs + pair0) * nip * NX;
    const bool comp = (P.mode == 0);
    const float inv_rho0 = (P.need_v && !comp) ? static_cast<float>(1.0 / rho0_member[b]) : 0.f;
    const int oa = P.rp_a[pi], ob = P.rp_b[pi];
    const RowProduct R = row_product(P, pi, inv_rho0);

    // products fused into the first forward (DIT) stage, read from the physical rows; the
    // canonical fast path needs the rewritten (jx, jy), (vx, vy) lines, which only exist in
    // prow_pass, so compressible velocities take the per-row path (1 / rho stored by prow_inverse)
    const SmemIO wio{work, NX};
    if (P.rp_canon && !P.rp_prep) {
        pstage_io<NX, pp.m - 1, -1, true>(RP, tw, [&](int r, int p) -> PC {
            return row_product_canon<NX>(P, R, inm + static_cast<size_t>(r) * nip * NX, psw(p));
        }, wio);
    } else {
        pstage_io<NX, pp.m - 1, -1, true>(RP, tw, [&](int r, int p) -> PC {
            return row_product_general<NX>(P, R, inm + static_cast<size_t>(r) * nip * NX, psw(p));
        }, wio);
    }
    __syncthreads();
    pdit_range<NX, pp.m - 1, 0, -1>(work, RP, tw);

    const OutLine W{work, static_cast<size_t>(NX), oa, ob};
    prow_untangle<NX>(P, 1, W, W, i2m, plane, pair0);
}

}  // namespace shhd
