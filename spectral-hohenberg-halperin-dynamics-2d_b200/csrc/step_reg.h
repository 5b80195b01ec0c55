// Host entry points of the register-resident kernels (step_reg.cu), compiled as their own
// translation unit.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "step_kernels.cuh"

namespace shhd {

// compute-grid row length the register-resident row pass handles (FP32 pair-line layout)
constexpr int kRegRowN = 1536;

// twiddle table of the register-resident transforms: number of floats, and its values
size_t reg_twiddle_floats();
void reg_twiddles(float* out);

// untangling rounds of 192 positions the row pass needs (Hx <= 768 on 1536-point rows: 2 .. 4)
int rrow_rounds(const StepPlan& P);

// dynamic shared memory of the row pass for a plan (input pair-lines + exchange buffers)
size_t rrow_smem_bytes(const StepPlan& P);

// row pass on 1536-point rows: I1 -> x-inverse -> products -> x-forward -> I2
void launch_rrow_pass(const StepPlan& P, int batch, size_t smem, cudaStream_t stream, const MemberInfo* members, const void* i1, void* i2,
                      const void* tw, const double* rho0, int* err);

// split row pass of the pair-line sizes 96 ... 1536 (kernel family 3): the physical-row buffer
// it needs (pair elements per member), and the launch of its two kernels
size_t split_phys_member_elems(const StepPlan& P);
bool split_row_supported(int nx);
void launch_split_row(const StepPlan& P, int batch, cudaStream_t stream, const MemberInfo* members, const void* i1, void* phys, void* i2,
                      const void* tw, const double* rho0, int* err);

// row pass over two output pairs at a time (kernel family 4): whether a plan has the input
// layout it needs, its dynamic shared memory, and its launch
bool dual_row_supported(const StepPlan& P);
size_t dual_row_smem_bytes(const StepPlan& P);
void launch_dual_row(const StepPlan& P, int batch, cudaStream_t stream, const MemberInfo* members, const void* i1, void* i2,
                     const void* tw, int* err);

}  // namespace shhd
