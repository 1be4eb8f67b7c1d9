// Launches of the generic stage kernel's TMA forms with the stage kind and the background split
// fixed at compile time (the loop's stages never branch on them per row).  The instantiations
// for every order live in their own translation units (vlasov_gen_kinds64.cu: FP64 TMA form,
// vlasov_gen_kinds32.cu: FP32 TMA form, vlasov_gen_kinds32p.cu: FP32 paired-row form), compiled in
// parallel with the API.
#pragma once

#include <cuda_runtime.h>

#include "vlasov_stage_gen.cuh"

namespace vl {

// Launch stage kind `kind` of order n (1..10) with `bg` background-split tables; pair selects the
// paired-row form (FP32 only).  grid / smem as for the run-time-kind instantiation.
template <typename T>
cudaError_t gen_kinds_launch(int n, bool pair, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                             const StageArgs &a, const StageTables<T> &tb, const GenMaps &maps);

// Allow `smem` bytes of dynamic shared memory for every instantiation of order n of the form.
template <typename T>
void gen_kinds_prepare(int n, bool pair, size_t smem);

template <>
cudaError_t gen_kinds_launch<double>(int n, bool pair, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                     const StageArgs &a, const StageTables<double> &tb, const GenMaps &maps);
template <>
cudaError_t gen_kinds_launch<float>(int n, bool pair, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                    const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps);
template <>
void gen_kinds_prepare<double>(int n, bool pair, size_t smem);
template <>
void gen_kinds_prepare<float>(int n, bool pair, size_t smem);

// the FP32 forms' instantiations, split over two translation units
cudaError_t gen_kinds_launch_tma32(int n, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                   const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps);
cudaError_t gen_kinds_launch_pair32(int n, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                    const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps);
void gen_kinds_prepare_tma32(int n, size_t smem);
void gen_kinds_prepare_pair32(int n, size_t smem);

}  // namespace vl
