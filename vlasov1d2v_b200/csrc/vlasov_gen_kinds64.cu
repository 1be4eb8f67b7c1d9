// FP64 TMA-form instantiations of the generic stage kernel per stage kind (see vlasov_gen_kinds.h).
#include "vlasov_gen_kinds.cuh"

namespace vl {

template <>
cudaError_t gen_kinds_launch<double>(int n, bool pair, int kind, bool bg, dim3 grid, size_t smem, cudaStream_t s,
                                     const StageArgs &a, const StageTables<double> &tb, const GenMaps &maps) {
    (void)bg;
    if (pair) return cudaErrorInvalidValue;   // the paired-row form is an FP32 form
    switch (n) {
        case 1: return gk::launch_n<double, 1, false>(kind, false, grid, smem, s, a, tb, maps);
        case 2: return gk::launch_n<double, 2, false>(kind, false, grid, smem, s, a, tb, maps);
        case 3: return gk::launch_n<double, 3, false>(kind, false, grid, smem, s, a, tb, maps);
        case 4: return gk::launch_n<double, 4, false>(kind, false, grid, smem, s, a, tb, maps);
        case 5: return gk::launch_n<double, 5, false>(kind, false, grid, smem, s, a, tb, maps);
        case 6: return gk::launch_n<double, 6, false>(kind, false, grid, smem, s, a, tb, maps);
        case 7: return gk::launch_n<double, 7, false>(kind, false, grid, smem, s, a, tb, maps);
        case 8: return gk::launch_n<double, 8, false>(kind, false, grid, smem, s, a, tb, maps);
        case 9: return gk::launch_n<double, 9, false>(kind, false, grid, smem, s, a, tb, maps);
        case 10: return gk::launch_n<double, 10, false>(kind, false, grid, smem, s, a, tb, maps);
        default: return cudaErrorInvalidValue;
    }
}

template <>
void gen_kinds_prepare<double>(int n, bool pair, size_t smem) {
    if (pair) return;
    switch (n) {
        case 1: gk::prepare_n<double, 1, false>(smem); break;
        case 2: gk::prepare_n<double, 2, false>(smem); break;
        case 3: gk::prepare_n<double, 3, false>(smem); break;
        case 4: gk::prepare_n<double, 4, false>(smem); break;
        case 5: gk::prepare_n<double, 5, false>(smem); break;
        case 6: gk::prepare_n<double, 6, false>(smem); break;
        case 7: gk::prepare_n<double, 7, false>(smem); break;
        case 8: gk::prepare_n<double, 8, false>(smem); break;
        case 9: gk::prepare_n<double, 9, false>(smem); break;
        case 10: gk::prepare_n<double, 10, false>(smem); break;
        default: break;
    }
}

}  // namespace vl
