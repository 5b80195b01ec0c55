// Register-resident kernels (step_kernels_reg.cuh) and their launches.
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

#include "step_kernels_dual.cuh"
#include "step_kernels_reg.cuh"
#include "step_kernels_split.cuh"
#include "step_reg.h"

namespace shhd {

size_t reg_twiddle_floats() { return 2 * static_cast<size_t>(kRegTw); }

void reg_twiddles(float* out) { reg_twiddles_host(out); }

int rrow_rounds(const StepPlan& P) { return (P.hx / 2 + 95) / 96; }

size_t rrow_smem_bytes(const StepPlan& P) {
    const int nip = (P.n_in + 1) / 2;
    return (static_cast<size_t>(nip) * kRegN + static_cast<size_t>(kRegGroups) * kRegChunk) * sizeof(ulonglong2);
}

namespace {
// the kernel's dynamic shared-memory limit, raised once per device to the largest need
// (eight order parameters: six input pair-lines)
void ensure_smem_limit() {
    static std::mutex mu;
    static std::set<int> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    if (done.count(dev)) return;
    const size_t most = (6ull * kRegN + static_cast<size_t>(kRegGroups) * kRegChunk) * sizeof(ulonglong2);
    for (const void* fn : {reinterpret_cast<const void*>(rrow_pass1536<2>), reinterpret_cast<const void*>(rrow_pass1536<3>),
                           reinterpret_cast<const void*>(rrow_pass1536<4>)}) {
        const cudaError_t rc = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(most));
        if (rc != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute (register row pass): ") + cudaGetErrorString(rc));
    }
    done.insert(dev);
}
}  // namespace

void launch_rrow_pass(const StepPlan& P, int batch, size_t smem, cudaStream_t stream, const MemberInfo* members, const void* i1, void* i2,
                      const void* tw, const double* rho0, int* err) {
    ensure_smem_limit();
    dim3 grid(P.npy / 2, batch);
    const auto* a = static_cast<const ulonglong2*>(i1);
    auto* o = static_cast<ulonglong2*>(i2);
    const auto* t = static_cast<const float2*>(tw);
    switch (rrow_rounds(P)) {
        case 2: rrow_pass1536<2><<<grid, kRegThreads, smem, stream>>>(P, members, a, o, t, rho0, err); break;
        case 3: rrow_pass1536<3><<<grid, kRegThreads, smem, stream>>>(P, members, a, o, t, rho0, err); break;
        default: rrow_pass1536<4><<<grid, kRegThreads, smem, stream>>>(P, members, a, o, t, rho0, err); break;
    }
}

size_t split_phys_member_elems(const StepPlan& P) { return phys_member_elems(P); }

bool split_row_supported(int nx) { return is_pair_size(nx); }

namespace {
template <int NX>
void launch_split(const StepPlan& P, int batch, cudaStream_t s, const MemberInfo* members, const void* i1, void* phys, void* i2,
                  const void* tw, const double* rho0, int* err) {
    constexpr int RP = kPairMaxN / NX;
    const size_t smem = static_cast<size_t>(RP) * NX * sizeof(ulonglong2);
    const int nip = (P.n_in + 1) / 2;
    dim3 g1(P.npy / 2 / RP, nip, batch), g2(P.npy / 2 / RP, P.rp_n, batch);
    prow_inverse<NX><<<g1, kThreads, smem, s>>>(P, members, static_cast<const ulonglong2*>(i1), static_cast<ulonglong2*>(phys),
                                                static_cast<const float2*>(tw), err);
    prow_forward<NX><<<g2, kThreads, smem, s>>>(P, members, static_cast<const ulonglong2*>(phys), static_cast<ulonglong2*>(i2),
                                                static_cast<const float2*>(tw), rho0);
}
}  // namespace

void launch_split_row(const StepPlan& P, int batch, cudaStream_t stream, const MemberInfo* members, const void* i1, void* phys, void* i2,
                      const void* tw, const double* rho0, int* err) {
    switch (P.npx) {
        case 96: launch_split<96>(P, batch, stream, members, i1, phys, i2, tw, rho0, err); break;
        case 192: launch_split<192>(P, batch, stream, members, i1, phys, i2, tw, rho0, err); break;
        case 384: launch_split<384>(P, batch, stream, members, i1, phys, i2, tw, rho0, err); break;
        case 768: launch_split<768>(P, batch, stream, members, i1, phys, i2, tw, rho0, err); break;
        case 1536: launch_split<1536>(P, batch, stream, members, i1, phys, i2, tw, rho0, err); break;
        default: throw std::runtime_error("split row pass: unsupported row length " + std::to_string(P.npx));
    }
}

bool dual_row_supported(const StepPlan& P) {
    // compressible canonical layout: (rho, jx), (jy, -) are the last two input pair-lines
    return is_pair_size(P.npx) && P.rp_canon && P.rp_prep && P.rp_jline == (P.n_in + 1) / 2 - 2;
}

size_t dual_row_smem_bytes(const StepPlan& P) { return prow2_smem_bytes<kPairMaxN>((P.n_in + 1) / 2); }

namespace {
template <int NX>
void launch_dual(const StepPlan& P, int batch, cudaStream_t s, const MemberInfo* members, const void* i1, void* i2, const void* tw, int* err) {
    constexpr int RP = kPairMaxN / NX;
    const size_t smem = prow2_smem_bytes<NX>((P.n_in + 1) / 2);
    {
        // raised once per device to the largest need (eight order parameters: six input pair-lines)
        static std::mutex mu;
        static std::set<int> done;
        int dev = 0;
        cudaGetDevice(&dev);
        std::lock_guard<std::mutex> lock(mu);
        if (!done.count(dev)) {
            const cudaError_t rc = cudaFuncSetAttribute(reinterpret_cast<const void*>(prow_pass2<NX>), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        static_cast<int>(prow2_smem_bytes<NX>(6)));
            if (rc != cudaSuccess) throw std::runtime_error(std::string("cudaFuncSetAttribute (two-pair row pass): ") + cudaGetErrorString(rc));
            done.insert(dev);
        }
    }
    dim3 grid(P.npy / 2 / RP, batch);
    prow_pass2<NX><<<grid, kDualThreads, smem, s>>>(P, members, static_cast<const ulonglong2*>(i1), static_cast<ulonglong2*>(i2),
                                                static_cast<const float2*>(tw), err);
}
}  // namespace

void launch_dual_row(const StepPlan& P, int batch, cudaStream_t stream, const MemberInfo* members, const void* i1, void* i2,
                     const void* tw, int* err) {
    switch (P.npx) {
        case 96: launch_dual<96>(P, batch, stream, members, i1, i2, tw, err); break;
        case 192: launch_dual<192>(P, batch, stream, members, i1, i2, tw, err); break;
        case 384: launch_dual<384>(P, batch, stream, members, i1, i2, tw, err); break;
        case 768: launch_dual<768>(P, batch, stream, members, i1, i2, tw, err); break;
        case 1536: launch_dual<1536>(P, batch, stream, members, i1, i2, tw, err); break;
        default: throw std::runtime_error("two-pair row pass: unsupported row length " + std::to_string(P.npx));
    }
}

}  // namespace shhd
