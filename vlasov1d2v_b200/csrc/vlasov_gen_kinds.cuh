// Instantiation machinery shared by vlasov_gen_kinds64.cu and vlasov_gen_kinds32.cu: one kernel
// per (order, form, stage kind, background split), dispatched from run-time values.
#pragma once

#include <cstring>

#include "vlasov_gen_kinds.h"

namespace vl {
namespace gk {

template <typename T, int N, bool PAIR, int K, int B>
constexpr auto kernel() {
    if constexpr (PAIR)
        return &stage_gen_pair_kernel<N, T, K, B>;
    else
        return &stage_gen_tma_kernel<N, T, K, B>;
}

template <typename T, int N, bool PAIR, int K, int B>
cudaError_t launch_one(dim3 grid, size_t smem, cudaStream_t s, const StageArgs &a, const StageTables<T> &tb,
                       const GenMaps &maps) {
    constexpr int THREADS = PAIR ? GenPairGeom<N, T>::THREADS : GenTmaGeom<N, T>::THREADS;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    return cudaLaunchKernelEx(&cfg, kernel<T, N, PAIR, K, B>(), a, tb, maps);
}

template <typename T, int N, bool PAIR>
cudaError_t launch_n(int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s, const StageArgs &a,
                     const StageTables<T> &tb, const GenMaps &maps) {
    constexpr bool HAS_BG = sizeof(T) == 4;   // the background split is a form of FP32 states
    if (kind == KIND_EULER) {
        if (HAS_BG && bg) return launch_one<T, N, PAIR, KIND_EULER, HAS_BG ? 1 : 0>(grid, smem, s, a, tb, maps);
        return launch_one<T, N, PAIR, KIND_EULER, 0>(grid, smem, s, a, tb, maps);
    }
    if (kind == KIND_COMBINE) {
        if (HAS_BG && bg) return launch_one<T, N, PAIR, KIND_COMBINE, HAS_BG ? 1 : 0>(grid, smem, s, a, tb, maps);
        return launch_one<T, N, PAIR, KIND_COMBINE, 0>(grid, smem, s, a, tb, maps);
    }
    if (HAS_BG && bg) return launch_one<T, N, PAIR, KIND_RHS, HAS_BG ? 1 : 0>(grid, smem, s, a, tb, maps);
    return launch_one<T, N, PAIR, KIND_RHS, 0>(grid, smem, s, a, tb, maps);
}

template <typename T, int N, bool PAIR>
void prepare_n(size_t smem) {
    const int b = (int)smem;
    cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_EULER, 0>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_COMBINE, 0>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_RHS, 0>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if constexpr (sizeof(T) == 4) {
        cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_EULER, 1>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_COMBINE, 1>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
        cudaFuncSetAttribute(kernel<T, N, PAIR, KIND_RHS, 1>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    }
}

}  // namespace gk
}  // namespace vl
