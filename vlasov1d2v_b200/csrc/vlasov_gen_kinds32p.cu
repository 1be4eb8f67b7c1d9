// FP32 paired-row-form instantiations of the generic stage kernel per stage kind and background
// split (see vlasov_gen_kinds.h).
#include "vlasov_gen_kinds.cuh"

namespace vl {

cudaError_t gen_kinds_launch_pair32(int n, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                    const StageArgs &a, const StageTables<float> &tb, const GenMaps &maps) {
    switch (n) {
        case 1: return gk::launch_n<float, 1, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 2: return gk::launch_n<float, 2, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 3: return gk::launch_n<float, 3, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 4: return gk::launch_n<float, 4, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 5: return gk::launch_n<float, 5, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 6: return gk::launch_n<float, 6, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 7: return gk::launch_n<float, 7, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 8: return gk::launch_n<float, 8, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 9: return gk::launch_n<float, 9, true>(kind, bg, grid, smem, s, a, tb, maps);
        case 10: return gk::launch_n<float, 10, true>(kind, bg, grid, smem, s, a, tb, maps);
        default: return cudaErrorInvalidValue;
    }
}

void gen_kinds_prepare_pair32(int n, size_t smem) {
    switch (n) {
        case 1: gk::prepare_n<float, 1, true>(smem); break;
        case 2: gk::prepare_n<float, 2, true>(smem); break;
        case 3: gk::prepare_n<float, 3, true>(smem); break;
        case 4: gk::prepare_n<float, 4, true>(smem); break;
        case 5: gk::prepare_n<float, 5, true>(smem); break;
        case 6: gk::prepare_n<float, 6, true>(smem); break;
        case 7: gk::prepare_n<float, 7, true>(smem); break;
        case 8: gk::prepare_n<float, 8, true>(smem); break;
        case 9: gk::prepare_n<float, 9, true>(smem); break;
        case 10: gk::prepare_n<float, 10, true>(smem); break;
        default: break;
    }
}

}  // namespace vl
