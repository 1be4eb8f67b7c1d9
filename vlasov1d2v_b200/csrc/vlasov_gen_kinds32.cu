// FP32 TMA-form instantiations of the generic stage kernel per stage kind and background split,
// and the FP32 dispatch (see vlasov_gen_kinds.h).
#include "vlasov_gen_kinds.cuh"

namespace vl {

cudaError_t gen_kinds_launch_tma32(int n, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                   const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps) {
    switch (n) {
        case 1: return gk::launch_n<float, 1, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 2: return gk::launch_n<float, 2, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 3: return gk::launch_n<float, 3, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 4: return gk::launch_n<float, 4, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 5: return gk::launch_n<float, 5, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 6: return gk::launch_n<float, 6, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 7: return gk::launch_n<float, 7, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 8: return gk::launch_n<float, 8, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 9: return gk::launch_n<float, 9, false>(kind, bg, grid, smem, s, a, tb, maps);
        case 10: return gk::launch_n<float, 10, false>(kind, bg, grid, smem, s, a, tb, maps);
        default: return cudaErrorInvalidValue;
    }
}

void gen_kinds_prepare_tma32(int n, size_t smem) {
    switch (n) {
        case 1: gk::prepare_n<float, 1, false>(smem); break;
        case 2: gk::prepare_n<float, 2, false>(smem); break;
        case 3: gk::prepare_n<float, 3, false>(smem); break;
        case 4: gk::prepare_n<float, 4, false>(smem); break;
        case 5: gk::prepare_n<float, 5, false>(smem); break;
        case 6: gk::prepare_n<float, 6, false>(smem); break;
        case 7: gk::prepare_n<float, 7, false>(smem); break;
        case 8: gk::prepare_n<float, 8, false>(smem); break;
        case 9: gk::prepare_n<float, 9, false>(smem); break;
        case 10: gk::prepare_n<float, 10, false>(smem); break;
        default: break;
    }
}

template <>
cudaError_t gen_kinds_launch<float>(int n, bool pair, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                    const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps) {
    return pair ? gen_kinds_launch_pair32(n, kind, bg, grid, smem, s, a, tb, maps)
                : gen_kinds_launch_tma32(n, kind, bg, grid, smem, s, a, tb, maps);
}

template <>
void gen_kinds_prepare<float>(int n, bool pair, size_t smem) {
    if (pair)
        gen_kinds_prepare_pair32(n, smem);
    else
        gen_kinds_prepare_tma32(n, smem);
}

}  // namespace vl
