// Register-resident kernels (step_kernels_reg.cuh) and their launches.
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

#include "step_kernels_reg.cuh"
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

}  // namespace shhd
