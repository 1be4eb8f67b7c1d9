// SSP-RK3 loop entry point that allocates nothing: the loop's scratch (the moment partials of the
// stage kernels) lives in a file-scope device array instead of a caller-provided workspace.
//
// Some callers cannot allocate device memory themselves: a host that records the loop into a
// CUDA graph while allocations are forbidden, a plugin whose host framework owns the whole
// device heap, or a foreign-language binding that only holds raw state pointers and a stream.
// They still own the state, stage, field and loop-state buffers; only the scratch moves here.
//
// Properties of the scratch array (documented in include/vlasov1d2v.h as well):
//   * capacity VL_NOALLOC_SCRATCH_BYTES (1 MiB) per GPU, held by every GPU that loads the
//     library until the process exits;
//   * its device address is looked up once per device with cudaGetSymbolAddress, on the first
//     call made with that device current (make that first call outside any stream capture); the
//     cached address is not refreshed, so after a cudaDeviceReset the process must not call
//     this entry point again on that device;
//   * the call must be made with the context's own device current (checked);
//   * all calls share it and it keeps the last call's contents; the loop writes every entry it
//     reads before reading it (nothing has to start at zero); calls whose kernels overlap on
//     the GPU (different streams, different contexts) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "vlasov1d2v.h"
#include "vlasov_ctx.cuh"

#define VL_NOALLOC_SCRATCH_DOUBLES (VL_NOALLOC_SCRATCH_BYTES / 8)

static __device__ __align__(256) double g_noalloc_scratch[VL_NOALLOC_SCRATCH_DOUBLES];

// error message setter of the library (vlasov_api.cu)
void vl_internal_set_error(const char *msg);

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_addr[kMaxDevices] = {nullptr};

}  // namespace

extern "C" {

VL_API int vl_ssp_rk3_steps_noalloc(vl_ctx *ctx, void *f, void *stage_a, void *stage_b, double *E,
                                    double *phi, vl_run_state *state, int nsteps, void *stream) {
    if (ctx == nullptr) {
        vl_internal_set_error("null context");
        return VL_ERR_INVALID;
    }
    const size_t need = vl_workspace_bytes(ctx);
    if (need > (size_t)VL_NOALLOC_SCRATCH_BYTES) {
        const std::string msg = "vl_ssp_rk3_steps_noalloc: the loop scratch of this problem needs " +
                                std::to_string(need) + " bytes, above the fixed " +
                                std::to_string((size_t)VL_NOALLOC_SCRATCH_BYTES) +
                                "-byte capacity; use vl_ssp_rk3_steps with a workspace";
        vl_internal_set_error(msg.c_str());
        return VL_ERR_TOO_LARGE;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        vl_internal_set_error("vl_ssp_rk3_steps_noalloc: no usable current device");
        return VL_ERR_CUDA;
    }
    if (dev != ctx->device) {
        // the scratch address is per device: the context's tables and the scratch must be on
        // the same GPU
        const std::string msg = "vl_ssp_rk3_steps_noalloc: current device " + std::to_string(dev) +
                                " is not the context's device " + std::to_string(ctx->device);
        vl_internal_set_error(msg.c_str());
        return VL_ERR_INVALID;
    }
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        if (g_addr[dev] == nullptr) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || p == nullptr) {
                vl_internal_set_error(cudaGetErrorString(e));
                return VL_ERR_CUDA;
            }
            g_addr[dev] = p;
        }
        scratch = g_addr[dev];
    }
    return vl_ssp_rk3_steps(ctx, f, stage_a, stage_b, E, phi, state, scratch, nsteps, stream);
}

}  // extern "C"
