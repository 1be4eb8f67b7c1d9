// Internal: the context object behind the opaque vl_ctx handle of the C ABI, shared by the
// library's translation units (entry points, the ensemble driver).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <utility>

#include "vlasov1d2v.h"
#include "vlasov_kernels.cuh"
#include "vlasov_stage_f32.cuh"

enum vl_stage_kernel { VL_STAGE_PENCIL = 0, VL_STAGE_TMA = 1, VL_STAGE_FRAG = 2, VL_STAGE_GEN = 3 };

struct vl_ctx {
    vl_config cfg;      // scalars (pointer members cleared)
    int device;
    int sm_count;
    int stage_grid_g;   // CTAs per x element of the stage kernel (moment partials per e)
    int stage_grid_g1;  // the same for the Euler and RHS stages (FP64 n = 8: a form without the
                        // f^n tile that fits more CTAs per SM; elsewhere = stage_grid_g)
    int moment_grid_g;  // CTAs per x element of the standalone moment kernel
    double up[vl::NMAX * vl::NMAX];
    double xi[vl::NMAX * 2];
    double xw[vl::NMAX];
    double qw[vl::NMAX * vl::NMAX];
    double *d_unodes = nullptr;
    void *d_usv = nullptr;        // per u node (u, a (-B u)), double2 or float2
    float4 *d_usv4 = nullptr;     // FP32: per u node {u J_x, u J_x, a (-B u) J_v, a (-B u) J_v}
    double *d_vnodes = nullptr;
    double *d_k = nullptr;
    double *d_xw = nullptr;
    double2 *d_ell = nullptr;     // [n][M]  DFT factors (vl_config dft_ell / dft_phase / dft_qnode)
    double2 *d_phase = nullptr;   // [nx][M]
    double2 *d_qnode = nullptr;   // [n][M]
    double *d_tables = nullptr;   // up [n n], xi [n 2], qw [n n]
    double *d_moment = nullptr;   // moment partials of vl_moment [nx][moment_grid_g][n]
    int *d_err = nullptr;         // device error word of operators run without a loop state
    bool use_tma = false;         // stage kernel: TMA-pipelined form (aligned orders)
    bool use_frag = false;        // n = 8: quad-fragment stage kernel (tensor cores in FP64)
    int stage_kernel = VL_STAGE_GEN;   // which stage kernel the launches use (vl_stage_kernel)
    bool gen_tma = false;         // generic stage kernel in its TMA form (FP64, aligned rows)
    bool gen_pair = false;        // generic stage kernel in its paired-row TMA form (FP32, R = 2 mod 4)
    const float *bg_rb = nullptr;   // background-split RHS tables (caller-owned)
    const float *bg_eu = nullptr;
    const float *bg_pair = nullptr; // the same tables interleaved per column pair (caller-owned, optional)
    std::map<std::pair<const void *, int>, CUtensorMap> maps;   // tensor maps per buffer
    vl::F32Tables f32_tables;       // FP32 n = 8 kernel's coefficient pairs (built on first use)
    bool f32_tables_ready = false;
};


// helpers of vlasov_api.cu used by the other translation units
void vl_internal_set_error(const char *msg);
int vl_internal_moment(const vl_ctx *c, const void *f, double *out, int G, cudaStream_t s);
// the context's stage arguments (tables, grid, physics) and its single-problem stage launch with
// the kernel chosen for it; moment partials are written for G = c->stage_grid_g
vl::StageArgs vl_internal_stage_args(const vl_ctx *c);
int vl_internal_stage(vl_ctx *c, const vl::StageArgs &a, cudaStream_t s);
