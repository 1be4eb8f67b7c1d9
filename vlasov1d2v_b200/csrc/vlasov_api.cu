// C ABI of the B200 hot path (declarations and reference citations in include/vlasov1d2v.h).
//
// Ownership: the context holds the immutable coefficient tables (device copies of the node
// coordinates and DFT tensors, host copies of the small matrices that travel as kernel
// parameters).  State, field, workspace and loop-state buffers belong to the caller.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <utility>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vlasov1d2v.h"
#include "vlasov_kernels.cuh"
#include "vlasov_stage.cuh"
#include "vlasov_stage_tma.cuh"
#include "vlasov_stage_frag.cuh"
#include "vlasov_stage_f32.cuh"
#include "vlasov_field.cuh"
#include "vlasov_stage_gen.cuh"
#include "vlasov_gen_kinds.h"

#include "vlasov_ctx.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return VL_ERR_CUDA;
}

#define VL_CUDA(call)                                              \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);        \
    } while (0)

inline int check_launch(const char *where) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, where);
    return VL_OK;
}

// status of a launch call, then of the launch itself
inline int check_launch(cudaError_t e, const char *where) {
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return cuda_fail(e, where);
    }
    return check_launch(where);
}

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }

inline size_t elem_size(const vl_ctx *c) {
    return c->cfg.precision == VL_FP64 ? sizeof(double) : sizeof(float);
}

// ------------------------------------------------------------------------------------------
// stage kernel dispatch
// ------------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// Kernel launch on the caller's stream.
template <typename... K, typename... A>
cudaError_t launch(const vl_ctx *c, void (*kernel)(K...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                   A &&...args) {
    (void)c;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cfg.numAttrs = 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<A>(args)...);
}

// 5-D view of the ghost-inclusive state: (v node, j, a, i, e), innermost first
template <int N, typename T>
int state_map(vl_ctx *c, const void *ptr, int which, CUtensorMap *out) {
    using G = vl::TmaGeom<N, T>;
    auto key = std::make_pair(ptr, which);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2, X = c->cfg.nx + 2;
    const cuuint64_t es = sizeof(T);
    cuuint64_t dims[5] = {V * N, (cuuint64_t)N, U, (cuuint64_t)N, X};
    cuuint64_t strides[4] = {V * N * es, V * N * N * es, V * N * N * U * es, V * N * N * U * N * es};
    cuuint32_t box[5];
    using F = vl::FragGeom<T>;
    switch (which) {
        // fragment kernel tiles: one zero-filled row past the j extent pads the plane stride
        case 6: box[0] = F::W; box[1] = F::ROWS; box[2] = 1; box[3] = N; box[4] = 1; break;
        case 7: box[0] = F::WF; box[1] = F::ROWS; box[2] = 1; box[3] = N; box[4] = 1; break;
        case 0: case 5: box[0] = G::W; box[1] = N; box[2] = 1; box[3] = N; box[4] = 1; break;
        case 1: box[0] = G::COLS; box[1] = N; box[2] = 1; box[3] = 1; box[4] = 1; break;
        case 2: box[0] = G::COLS; box[1] = 1; box[2] = 1; box[3] = N; box[4] = 1; break;
        default: box[0] = G::COLS; box[1] = N; box[2] = 1; box[3] = N; box[4] = 1; break;
    }
    // output tiles: the v extent ends after the last interior element, so stores of a ragged
    // last tile are clipped before the v ghost element
    if (which == 4) dims[0] = (cuuint64_t)(c->cfg.nv + 1) * N;
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5,
                     const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 2-D view [U n][V n] of a background-split table (FP32), box (32, n): one tile's rows
int bg_map(vl_ctx *c, const float *ptr, int n, CUtensorMap *out) {
    auto key = std::make_pair(static_cast<const void *>(ptr), 8);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2;
    cuuint64_t dims[2] = {V * n, U * n};
    cuuint64_t strides[1] = {V * n * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)vl::FragGeom<float>::COLS, (cuuint32_t)n};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (background table) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 2-D view [U n][V n / 2 pairs x 4] of the background tables interleaved per column pair (FP32,
// n = 8 kernel), box (2 COLS, n): one tile's rows of both tables
int bg_pair_map(vl_ctx *c, const float *ptr, int n, CUtensorMap *out) {
    auto key = std::make_pair(static_cast<const void *>(ptr), 9);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2;
    cuuint64_t dims[2] = {2 * V * n, U * n};
    cuuint64_t strides[1] = {2 * V * n * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)(2 * vl::FragGeom<float>::COLS), (cuuint32_t)n};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (background pair table) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 5-D view of a state for the generic kernel's TMA form: which 0 = tile (WB, RJ, 1, n, 1),
// 1 = x-node plane (WB, n, 1, 1, 1), 2 = j row of every x node (WB, 1, 1, n, 1)
template <int N, typename T>
int gen_map(vl_ctx *c, const void *ptr, int which, CUtensorMap *out) {
    using G = vl::GenTmaGeom<N, T>;
    auto key = std::make_pair(ptr, 20 + which);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2, X = c->cfg.nx + 2, es = sizeof(T);
    cuuint64_t dims[5] = {V * N, (cuuint64_t)N, U, (cuuint64_t)N, X};
    cuuint64_t strides[4] = {V * N * es, V * N * N * es, V * N * N * U * es, V * N * N * U * N * es};
    cuuint32_t box[5] = {(cuuint32_t)G::WB, 1, 1, 1, 1};
    if (which == 0) {
        box[1] = G::RJ;
        box[3] = N;
    } else if (which == 1) {
        box[1] = N;
    } else {
        box[3] = N;
    }
    cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5,
                     const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (generic kernel) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 2-D view [U n][V n] of a background-split table for the generic kernel's TMA form (FP32),
// box (WB, n): the tile's rows of one u element
template <int N, typename T>
int gen_bg_map(vl_ctx *c, const float *ptr, CUtensorMap *out) {
    using G = vl::GenTmaGeom<N, T>;
    auto key = std::make_pair(static_cast<const void *>(ptr), 30);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2;
    cuuint64_t dims[2] = {V * N, U * N};
    cuuint64_t strides[1] = {V * N * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)G::WB, (cuuint32_t)N};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (generic kernel, background) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 4-D view (2R, U n / 2, n, X) of an FP32 state for the generic kernel's paired-row form (R =
// (nv+2) n floats per row, two rows per 16-byte-multiple pair): which 0 = tile (WB, NPJ, n, 1),
// 1 = x-node plane (WB, NPJ, 1, 1), 2 = one row of every x node (WB, 1, n, 1)
template <int N, typename T>
int gen_pair_map(vl_ctx *c, const void *ptr, int which, CUtensorMap *out) {
    using G = vl::GenPairGeom<N, T>;
    auto key = std::make_pair(ptr, 40 + which);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2, X = c->cfg.nx + 2, es = sizeof(T);
    const cuuint64_t R = V * N;
    cuuint64_t dims[4] = {2 * R, U * N / 2, (cuuint64_t)N, X};
    cuuint64_t strides[3] = {2 * R * es, U * N * R * es, U * N * R * N * es};
    cuuint32_t box[4] = {(cuuint32_t)G::WB, 1, 1, 1};
    if (which == 0) {
        box[1] = G::NPJ;
        box[2] = N;
    } else if (which == 1) {
        box[1] = G::NPJ;
    } else {
        box[2] = N;
    }
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (paired rows) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// 2-D view (2R, U n / 2) of a background-split table for the paired-row form, box (WB, NPJ)
template <int N, typename T>
int gen_pair_bg_map(vl_ctx *c, const float *ptr, CUtensorMap *out) {
    using G = vl::GenPairGeom<N, T>;
    auto key = std::make_pair(static_cast<const void *>(ptr), 50);
    auto it = c->maps.find(key);
    if (it != c->maps.end()) {
        *out = it->second;
        return VL_OK;
    }
    auto enc = encode_fn();
    if (!enc) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t U = c->cfg.nu + 2, V = c->cfg.nv + 2;
    const cuuint64_t R = V * N;
    cuuint64_t dims[2] = {2 * R, U * N / 2};
    cuuint64_t strides[1] = {2 * R * sizeof(float)};
    cuuint32_t box[2] = {(cuuint32_t)G::WB, (cuuint32_t)G::NPJ};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(ptr), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(VL_ERR_CUDA, "cuTensorMapEncodeTiled (paired rows, background) failed");
    if (c->maps.size() > 64) c->maps.clear();
    c->maps[key] = m;
    *out = m;
    return VL_OK;
}

// coefficient tables of the FP32 n = 8 kernel (pairs for the packed FMAs), built once per context
const vl::F32Tables &f32_tables(vl_ctx *c) {
    if (!c->f32_tables_ready) {
        constexpr int N = 8;
        vl::F32Tables &t = c->f32_tables;
        std::memset(&t, 0, sizeof(t));
        for (int i = 0; i < N; ++i) {
            for (int m = 0; m < N; ++m) {
                const float u = (float)c->up[i * N + m];
                t.up2[i * N + m] = make_float2(u, u);
                double p = c->up[i * N + m], q = c->up[i * N + m];
                if (m == N - 1) p -= c->xi[2 * i + 1];
                if (m == 0) q += c->xi[2 * i];
                t.upP[i * N + m] = (float)p;
                t.upM[i * N + m] = (float)q;
            }
            const float l = (float)c->xi[2 * i], r = (float)(-c->xi[2 * i + 1]);
            t.xl2[i] = make_float2(l, l);
            t.xr2[i] = make_float2(r, r);
            const float wu = (float)(c->xw[i] / c->cfg.ju);
            t.wu2[i] = make_float2(wu, wu);
            t.wv[i] = c->xw[i] / c->cfg.jv;
        }
        for (int i = 0; i < 2 * N; ++i) t.xi[i] = (float)c->xi[i];
        c->f32_tables_ready = true;
    }
    return c->f32_tables;
}

template <int N, typename T>
int launch_stage_t(vl_ctx *c, const vl::StageArgs &a0, cudaStream_t s) {
    vl::StageTables<T> tb;
    std::memset(&tb, 0, sizeof(tb));
    for (int i = 0; i < N * N; ++i) tb.up[i] = (T)c->up[i];
    for (int i = 0; i < 2 * N; ++i) tb.xi[i] = (T)c->xi[i];
    for (int i = 0; i < N * N; ++i) tb.qw[i] = c->qw[i];
    for (int i = 0; i < N; ++i) {
        tb.wu[i] = c->xw[i] / c->cfg.ju;
        tb.wv[i] = c->xw[i] / c->cfg.jv;
    }
    for (int i = 0; i < N; ++i)
        for (int m = 0; m < N; ++m) {
            double p = c->up[i * N + m], q = c->up[i * N + m];
            if (m == N - 1) p -= c->xi[2 * i + 1];
            if (m == 0) q += c->xi[2 * i];
            tb.upP[i * N + m] = (T)p;
            tb.upM[i * N + m] = (T)q;
        }
    vl::StageArgs a = a0;
    if (a.err == nullptr) a.err = c->d_err;
    dim3 grid(a.kind == vl::KIND_COMBINE ? c->stage_grid_g : c->stage_grid_g1, c->cfg.nx);
    if constexpr (N == 8) {
        if (c->use_frag) {
            using G = vl::FragGeom<T>;
            vl::FragMaps maps;
            int rc;
            if ((rc = state_map<N, T>(c, a.in, 6, &maps.in_tile))) return rc;
            if ((rc = state_map<N, T>(c, a.in, 1, &maps.in_xface))) return rc;
            if ((rc = state_map<N, T>(c, a.in, 2, &maps.in_uface))) return rc;
            if ((rc = state_map<N, T>(c, a.fn ? a.fn : a.in, 7, &maps.fn_tile))) return rc;
            if (G::BG && a.bg_rb != nullptr && c->bg_pair != nullptr) {
                // the two tables interleaved per column pair: one (2 COLS, n) box per tile
                if ((rc = bg_pair_map(c, c->bg_pair, N, &maps.bg_eu))) return rc;
                std::memset(&maps.bg_rb, 0, sizeof(maps.bg_rb));
            } else if (G::BG && a.bg_rb != nullptr) {
                if ((rc = bg_map(c, a.bg_eu, N, &maps.bg_eu))) return rc;
                if ((rc = bg_map(c, a.bg_rb, N, &maps.bg_rb))) return rc;
            } else {
                std::memset(&maps.bg_eu, 0, sizeof(maps.bg_eu));
                std::memset(&maps.bg_rb, 0, sizeof(maps.bg_rb));
            }
            if constexpr (sizeof(T) == 4) {
                // FP32: the packed-FMA kernel, one instantiation per stage kind and background split
                a.usv = c->d_usv4;
                a.sx = a.jx / c->cfg.jx;
                a.sv = a.jv / c->cfg.jv;
                const vl::F32Tables &ft = f32_tables(c);
                // background split: 0 none, 1 two tables, 2 the interleaved pair table
                const int bg = a.bg_rb == nullptr ? 0 : (c->bg_pair != nullptr ? 2 : 1);
                const dim3 blk(G::THREADS);
                const size_t sm = G::smem_bytes();
                auto go = [&](auto kc) {
                    constexpr int K = decltype(kc)::value;
                    if (bg == 2) return launch(c, vl::stage_f32_kernel<K, 2>, grid, blk, sm, s, a, ft, maps);
                    if (bg == 1) return launch(c, vl::stage_f32_kernel<K, 1>, grid, blk, sm, s, a, ft, maps);
                    return launch(c, vl::stage_f32_kernel<K, 0>, grid, blk, sm, s, a, ft, maps);
                };
                cudaError_t le;
                switch (a.kind) {
                    case vl::KIND_EULER:
                        le = go(std::integral_constant<int, vl::KIND_EULER>{});
                        break;
                    case vl::KIND_COMBINE:
                        le = go(std::integral_constant<int, vl::KIND_COMBINE>{});
                        break;
                    default:
                        le = go(std::integral_constant<int, vl::KIND_RHS>{});
                        break;
                }
                return check_launch(le, "stage_f32_kernel");
            } else {
                // FP64: combination stages stage an f^n tile; Euler / RHS stages take the form
                // without it (3 CTAs per SM)
                // (one instantiation per stage kind: no per-row branches on it)
                if (a.kind == vl::KIND_COMBINE)
                    return check_launch(launch(c, vl::stage_frag_kernel<T, true, vl::KIND_COMBINE>, grid,
                                               dim3(G::THREADS), G::smem_bytes(), s, a, tb, maps),
                                        "stage_frag_kernel");
                using G1 = vl::FragGeom<T, false>;
                if (a.kind == vl::KIND_EULER)
                    return check_launch(launch(c, vl::stage_frag_kernel<T, false, vl::KIND_EULER>, grid,
                                               dim3(G1::THREADS), G1::smem_bytes(), s, a, tb, maps),
                                        "stage_frag_kernel");
                return check_launch(launch(c, vl::stage_frag_kernel<T, false, vl::KIND_RHS>, grid, dim3(G1::THREADS),
                                           G1::smem_bytes(), s, a, tb, maps),
                                    "stage_frag_kernel");
            }
        }
    }
    if constexpr (sizeof(T) == 4) {
        if (c->stage_kernel == VL_STAGE_GEN && c->gen_pair) {
            using G = vl::GenPairGeom<N, T>;
            if ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out) |
                 reinterpret_cast<uintptr_t>(a.fn) | reinterpret_cast<uintptr_t>(a.ghost_out) |
                 reinterpret_cast<uintptr_t>(a.bg_rb) | reinterpret_cast<uintptr_t>(a.bg_eu)) % 16)
                return fail(VL_ERR_INVALID, "state buffers must be 16-byte aligned");
            vl::GenMaps maps;
            std::memset(&maps, 0, sizeof(maps));
            int rc;
            if ((rc = gen_pair_map<N, T>(c, a.in, 0, &maps.in_tile))) return rc;
            if ((rc = gen_pair_map<N, T>(c, a.fn ? a.fn : a.in, 0, &maps.fn_tile))) return rc;
            if ((rc = gen_pair_map<N, T>(c, a.in, 1, &maps.xface))) return rc;
            if ((rc = gen_pair_map<N, T>(c, a.in, 2, &maps.uface))) return rc;
            if (a.bg_rb != nullptr) {
                if ((rc = gen_pair_bg_map<N, T>(c, a.bg_eu, &maps.bg_eu))) return rc;
                if ((rc = gen_pair_bg_map<N, T>(c, a.bg_rb, &maps.bg_rb))) return rc;
            }
            return check_launch(vl::gen_kinds_launch<T>(N, true, a.kind, a.bg_rb != nullptr, grid, G::smem_bytes(), s,
                                                        a, tb, maps),
                                "stage_gen_pair_kernel");
        }
    }
    if (c->stage_kernel == VL_STAGE_GEN && c->gen_tma) {
        using G = vl::GenTmaGeom<N, T>;
        if ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out) |
             reinterpret_cast<uintptr_t>(a.fn) | reinterpret_cast<uintptr_t>(a.ghost_out) |
             reinterpret_cast<uintptr_t>(a.bg_rb) | reinterpret_cast<uintptr_t>(a.bg_eu)) % 16)
            return fail(VL_ERR_INVALID, "state buffers must be 16-byte aligned");
        vl::GenMaps maps;
        std::memset(&maps, 0, sizeof(maps));
        int rc;
        if ((rc = gen_map<N, T>(c, a.in, 0, &maps.in_tile))) return rc;
        if ((rc = gen_map<N, T>(c, a.fn ? a.fn : a.in, 0, &maps.fn_tile))) return rc;
        if ((rc = gen_map<N, T>(c, a.in, 1, &maps.xface))) return rc;
        if ((rc = gen_map<N, T>(c, a.in, 2, &maps.uface))) return rc;
        if (sizeof(T) == 4 && a.bg_rb != nullptr) {
            if ((rc = gen_bg_map<N, T>(c, a.bg_eu, &maps.bg_eu))) return rc;
            if ((rc = gen_bg_map<N, T>(c, a.bg_rb, &maps.bg_rb))) return rc;
        }
        return check_launch(vl::gen_kinds_launch<T>(N, false, a.kind, sizeof(T) == 4 && a.bg_rb != nullptr, grid,
                                                    G::smem_bytes(), s, a, tb, maps),
                            "stage_gen_tma_kernel");
    }
    if (c->stage_kernel == VL_STAGE_GEN) {
        using G = vl::GenGeom<N, T>;
        // pair copies and stores of even orders need pair-aligned buffers
        const uintptr_t align = (N % 2 == 0) ? 2 * sizeof(T) : sizeof(T);
        if ((reinterpret_cast<uintptr_t>(a.in) | reinterpret_cast<uintptr_t>(a.out) |
             reinterpret_cast<uintptr_t>(a.fn) | reinterpret_cast<uintptr_t>(a.ghost_out)) % align)
            return fail(VL_ERR_INVALID, "state buffers must be aligned to two elements");
        return check_launch(launch(c, vl::stage_gen_kernel<N, T>, grid, dim3(G::THREADS), G::smem_bytes(), s, a, tb),
                            "stage_gen_kernel");
    }
    if constexpr (vl::TmaGeom<N, T>::SUPPORTED) {
        if (c->use_tma) {
            using G = vl::TmaGeom<N, T>;
            vl::TmaMaps maps;
            int rc;
            if ((rc = state_map<N, T>(c, a.in, 0, &maps.in_tile))) return rc;
            if ((rc = state_map<N, T>(c, a.in, 1, &maps.in_xface))) return rc;
            if ((rc = state_map<N, T>(c, a.in, 2, &maps.in_uface))) return rc;
            if ((rc = state_map<N, T>(c, a.fn ? a.fn : a.in, 3, &maps.fn_tile))) return rc;
            return check_launch(
                launch(c, vl::stage_tma_kernel<N, T>, grid, dim3(G::THREADS), G::smem_bytes(), s, a, tb, maps),
                "stage_tma_kernel");
        }
    }
    using G = vl::PencilGeom<N, T>;
    return check_launch(launch(c, vl::stage_pencil_kernel<N, T>, grid, dim3(G::THREADS), G::smem_bytes(), s, a, tb),
                        "stage_pencil_kernel");
}

template <typename T>
int launch_stage(vl_ctx *c, const vl::StageArgs &a, cudaStream_t s) {
    switch (c->cfg.n) {
        case 1: return launch_stage_t<1, T>(c, a, s);
        case 2: return launch_stage_t<2, T>(c, a, s);
        case 3: return launch_stage_t<3, T>(c, a, s);
        case 4: return launch_stage_t<4, T>(c, a, s);
        case 5: return launch_stage_t<5, T>(c, a, s);
        case 6: return launch_stage_t<6, T>(c, a, s);
        case 7: return launch_stage_t<7, T>(c, a, s);
        case 8: return launch_stage_t<8, T>(c, a, s);
        case 9: return launch_stage_t<9, T>(c, a, s);
        case 10: return launch_stage_t<10, T>(c, a, s);
        default: return fail(VL_ERR_UNSUPPORTED, "order n not compiled in");
    }
}

int stage(vl_ctx *c, const vl::StageArgs &a, cudaStream_t s) {
    return c->cfg.precision == VL_FP64 ? launch_stage<double>(c, a, s)
                                       : launch_stage<float>(c, a, s);
}

template <int N, typename T>
int stage_occupancy_t(bool tma, bool frag, bool gen, bool gtma, bool gpair) {
    int blocks = 0;
    if constexpr (sizeof(T) == 4) {
        if (gen && gpair) {
            using G = vl::GenPairGeom<N, T>;
            const size_t smem = G::smem_bytes();
            cudaFuncSetAttribute(vl::stage_gen_pair_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            vl::gen_kinds_prepare<T>(N, true, smem);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_gen_pair_kernel<N, T>, G::THREADS,
                                                              smem) != cudaSuccess)
                return 1;
            return blocks > 0 ? blocks : 1;
        }
    }
    if (gen && gtma) {
        using G = vl::GenTmaGeom<N, T>;
        const size_t smem = G::smem_bytes();
        cudaFuncSetAttribute(vl::stage_gen_tma_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        vl::gen_kinds_prepare<T>(N, false, smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_gen_tma_kernel<N, T>, G::THREADS,
                                                          smem) != cudaSuccess)
            return 1;
        return blocks > 0 ? blocks : 1;
    }
    if (gen) {
        using G = vl::GenGeom<N, T>;
        const size_t smem = G::smem_bytes();
        cudaFuncSetAttribute(vl::stage_gen_kernel<N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_gen_kernel<N, T>, G::THREADS, smem) !=
            cudaSuccess)
            return 1;
        return blocks > 0 ? blocks : 1;
    }
    if constexpr (N == 8) {
        if (frag) {
            using G = vl::FragGeom<T>;
            const size_t smem = G::smem_bytes();
            if constexpr (sizeof(T) == 4) {
                // every instantiation of the FP32 kernel takes the same dynamic shared memory
                auto attr = [&](auto kc) {
                    constexpr int K = decltype(kc)::value;
                    cudaFuncSetAttribute(vl::stage_f32_kernel<K, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
                    cudaFuncSetAttribute(vl::stage_f32_kernel<K, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
                    cudaFuncSetAttribute(vl::stage_f32_kernel<K, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
                };
                attr(std::integral_constant<int, vl::KIND_EULER>{});
                attr(std::integral_constant<int, vl::KIND_COMBINE>{});
                attr(std::integral_constant<int, vl::KIND_RHS>{});
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_f32_kernel<vl::KIND_COMBINE, 1>,
                                                                  G::THREADS, smem) != cudaSuccess)
                    return 1;
            } else {
                cudaFuncSetAttribute(vl::stage_frag_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem);
                cudaFuncSetAttribute(vl::stage_frag_kernel<T, true, vl::KIND_COMBINE>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_frag_kernel<T, true>,
                                                                  G::THREADS, smem) != cudaSuccess)
                    return 1;
            }
            return blocks > 0 ? blocks : 1;
        }
    }
    if constexpr (vl::TmaGeom<N, T>::SUPPORTED) {
        if (tma) {
            using G = vl::TmaGeom<N, T>;
            const size_t smem = G::smem_bytes();
            cudaFuncSetAttribute(vl::stage_tma_kernel<N, T>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_tma_kernel<N, T>,
                                                              G::THREADS, smem) != cudaSuccess)
                return 1;
            return blocks > 0 ? blocks : 1;
        }
    }
    using G = vl::PencilGeom<N, T>;
    const size_t smem = G::smem_bytes();
    cudaFuncSetAttribute(vl::stage_pencil_kernel<N, T>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_pencil_kernel<N, T>,
                                                      G::THREADS, smem) != cudaSuccess)
        return 1;
    return blocks > 0 ? blocks : 1;
}

// resident CTAs per SM of the FP64 n = 8 fragment kernel's form without the f^n tile
int frag_nofn_occupancy() {
    using G = vl::FragGeom<double, false>;
    const size_t smem = G::smem_bytes();
    cudaFuncSetAttribute(vl::stage_frag_kernel<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    cudaFuncSetAttribute(vl::stage_frag_kernel<double, false, vl::KIND_EULER>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(vl::stage_frag_kernel<double, false, vl::KIND_RHS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, vl::stage_frag_kernel<double, false>, G::THREADS,
                                                      smem) != cudaSuccess)
        return 1;
    return blocks > 0 ? blocks : 1;
}

template <int N, typename T>
bool tma_supported_t(const vl_config &g) {
    if constexpr (vl::TmaGeom<N, T>::SUPPORTED) {
        return ((size_t)(g.nv + 2) * N * sizeof(T)) % 16 == 0;
    }
    return false;
}

template <typename T>
int stage_occupancy(int n, bool tma, bool frag, bool gen, bool gtma, bool gpair) {
    switch (n) {
        case 1: return stage_occupancy_t<1, T>(tma, frag, gen, gtma, gpair);
        case 2: return stage_occupancy_t<2, T>(tma, frag, gen, gtma, gpair);
        case 3: return stage_occupancy_t<3, T>(tma, frag, gen, gtma, gpair);
        case 4: return stage_occupancy_t<4, T>(tma, frag, gen, gtma, gpair);
        case 5: return stage_occupancy_t<5, T>(tma, frag, gen, gtma, gpair);
        case 6: return stage_occupancy_t<6, T>(tma, frag, gen, gtma, gpair);
        case 7: return stage_occupancy_t<7, T>(tma, frag, gen, gtma, gpair);
        case 8: return stage_occupancy_t<8, T>(tma, frag, gen, gtma, gpair);
        case 9: return stage_occupancy_t<9, T>(tma, frag, gen, gtma, gpair);
        case 10: return stage_occupancy_t<10, T>(tma, frag, gen, gtma, gpair);
        default: return 1;
    }
}

// v elements per stage tile of the generic kernel
template <typename T>
int gen_ept(int n) {
    switch (n) {
        case 1: return vl::GenEpt<1, T>::value;
        case 2: return vl::GenEpt<2, T>::value;
        case 3: return vl::GenEpt<3, T>::value;
        case 4: return vl::GenEpt<4, T>::value;
        case 5: return vl::GenEpt<5, T>::value;
        case 6: return vl::GenEpt<6, T>::value;
        case 7: return vl::GenEpt<7, T>::value;
        case 8: return vl::GenEpt<8, T>::value;
        case 9: return vl::GenEpt<9, T>::value;
        case 10: return vl::GenEpt<10, T>::value;
        default: return 1;
    }
}

template <typename T>
bool tma_supported(const vl_config &g) {
    switch (g.n) {
        case 2: return tma_supported_t<2, T>(g);
        case 4: return tma_supported_t<4, T>(g);
        case 8: return tma_supported_t<8, T>(g);
        default: return false;
    }
}

// v elements per tile of the stage kernel
// v elements per stage tile: 32 / n for the pencil, TMA and fragment kernels (4 at n = 8)
int stage_epw(const vl_ctx *c) {
    if (c->stage_kernel == VL_STAGE_GEN)
        return c->cfg.precision == VL_FP64 ? gen_ept<double>(c->cfg.n) : gen_ept<float>(c->cfg.n);
    return 32 / c->cfg.n;
}

// ------------------------------------------------------------------------------------------
// moment kernel dispatch
// ------------------------------------------------------------------------------------------
template <int N, typename T>
int launch_moment_t(const vl_ctx *c, const void *f, double *out, int G, cudaStream_t s) {
    vl::MomentArgs a;
    std::memset(&a, 0, sizeof(a));
    a.f = f;
    a.out = out;
    a.G = G;
    a.nx = c->cfg.nx;
    a.nu = c->cfg.nu;
    a.nv = c->cfg.nv;
    for (int i = 0; i < N * N; ++i) a.qw[i] = c->qw[i];
    const dim3 grid((unsigned)G, (unsigned)c->cfg.nx);
    vl::moment_kernel<N, T><<<grid, vl::MOMENT_THREADS, 0, s>>>(a);
    return check_launch("moment_kernel");
}

template <typename T>
int launch_moment(const vl_ctx *c, const void *f, double *out, int G, cudaStream_t s) {
    switch (c->cfg.n) {
        case 1: return launch_moment_t<1, T>(c, f, out, G, s);
        case 2: return launch_moment_t<2, T>(c, f, out, G, s);
        case 3: return launch_moment_t<3, T>(c, f, out, G, s);
        case 4: return launch_moment_t<4, T>(c, f, out, G, s);
        case 5: return launch_moment_t<5, T>(c, f, out, G, s);
        case 6: return launch_moment_t<6, T>(c, f, out, G, s);
        case 7: return launch_moment_t<7, T>(c, f, out, G, s);
        case 8: return launch_moment_t<8, T>(c, f, out, G, s);
        case 9: return launch_moment_t<9, T>(c, f, out, G, s);
        case 10: return launch_moment_t<10, T>(c, f, out, G, s);
        default: return fail(VL_ERR_UNSUPPORTED, "order n not compiled in");
    }
}

int moment(const vl_ctx *c, const void *f, double *out, int G, cudaStream_t s) {
    return c->cfg.precision == VL_FP64 ? launch_moment<double>(c, f, out, G, s)
                                       : launch_moment<float>(c, f, out, G, s);
}

// ------------------------------------------------------------------------------------------
// field / scalar kernels
// ------------------------------------------------------------------------------------------
vl::FieldArgs field_args(const vl_ctx *c) {
    vl::FieldArgs a;
    std::memset(&a, 0, sizeof(a));
    a.ell = c->d_ell;
    a.phase = c->d_phase;
    a.qnode = c->d_qnode;
    a.k = c->d_k;
    a.xw = c->d_xw;
    a.nx = c->cfg.nx;
    a.n = c->cfg.n;
    a.M = c->cfg.n_modes;
    a.kappa = c->cfg.kappa;
    a.dx = c->cfg.dx;
    a.length = c->cfg.length_x;
    a.accel = c->cfg.accel;
    a.bfield = c->cfg.bfield;
    a.umax = c->cfg.umax;
    a.vmax = c->cfg.vmax;
    a.du = c->cfg.du;
    a.dv = c->cfg.dv;
    a.courant = c->cfg.courant;
    return a;
}

// the whole spectral solve in one thread-block cluster of vl::FC CTAs (vlasov_field.cuh)
int field(const vl_ctx *c, const vl::FieldArgs &a0, cudaStream_t s) {
    // the table prefetch where it fits the dynamic shared memory budget
    vl::FieldArgs a = a0;
    const size_t base = vl::field_solve_smem_for(a.n, a.M, a.phi != nullptr);
    const size_t pre = vl::field_prefetch_bytes(a.nx, a.n, a.M);
    a.prefetch = base + pre <= vl::FIELD_DYN_SMEM_MAX ? 1 : 0;
    cudaLaunchConfig_t cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3(vl::FC);
    cfg.blockDim = dim3(vl::FS_THREADS);
    cfg.dynamicSmemBytes = base + (a.prefetch ? pre : 0);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = vl::FC;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return check_launch(cudaLaunchKernelEx(&cfg, vl::field_solve_kernel, a), "field_solve_kernel");
}

// bytes of the moment partials inside a loop workspace
size_t partials_bytes(const vl_ctx *c) {
    int g = c->stage_grid_g > c->moment_grid_g ? c->stage_grid_g : c->moment_grid_g;
    if (c->stage_grid_g1 > g) g = c->stage_grid_g1;
    const size_t b = sizeof(double) * (size_t)c->cfg.nx * g * c->cfg.n;
    return (b + 255) & ~(size_t)255;
}

vl::ScalarArgs scalar_args(const vl_ctx *c, const double *E) {
    vl::ScalarArgs a;
    std::memset(&a, 0, sizeof(a));
    a.E = E;
    a.xw = c->d_xw;
    a.nx = c->cfg.nx;
    a.n = c->cfg.n;
    a.accel = c->cfg.accel;
    a.bfield = c->cfg.bfield;
    a.umax = c->cfg.umax;
    a.vmax = c->cfg.vmax;
    a.dx = c->cfg.dx;
    a.du = c->cfg.du;
    a.dv = c->cfg.dv;
    a.courant = c->cfg.courant;
    return a;
}

vl::StageArgs stage_args(const vl_ctx *c) {
    vl::StageArgs a;
    std::memset(&a, 0, sizeof(a));
    a.u_nodes = c->d_unodes;
    a.usv = c->d_usv;
    a.v_nodes = c->d_vnodes;
    a.tables = c->d_tables;
    a.bg_rb = c->bg_rb;
    a.bg_eu = c->bg_eu;
    a.nx = c->cfg.nx;
    a.nu = c->cfg.nu;
    a.nv = c->cfg.nv;
    a.accel = c->cfg.accel;
    a.bfield = c->cfg.bfield;
    a.jx = c->cfg.jx;
    a.ju = c->cfg.ju;
    a.jv = c->cfg.jv;
    return a;
}

// Shu-Osher coefficients of the nonlinear SSP-RK3 (main/timestep.py:35-39)
const double kRK3[2][3] = {{3.0 / 4.0, 1.0 / 4.0, 1.0 / 4.0}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};

template <typename P>
int upload(P **dst, const void *src, size_t bytes) {
    VL_CUDA(cudaMalloc((void **)dst, bytes));
    VL_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return VL_OK;
}

}  // namespace

void vl_internal_set_error(const char *msg) { g_err = msg ? msg : ""; }

int vl_internal_moment(const vl_ctx *c, const void *f, double *out, int G, cudaStream_t s) {
    return moment(c, f, out, G, s);
}

vl::StageArgs vl_internal_stage_args(const vl_ctx *c) { return stage_args(c); }

int vl_internal_stage(vl_ctx *c, const vl::StageArgs &a, cudaStream_t s) { return stage(c, a, s); }

extern "C" {

const char *vl_last_error(void) { return g_err.c_str(); }

int vl_abi_version(void) { return VL_ABI_VERSION; }

int vl_ctx_create(const vl_config *cfg, vl_ctx **out) {
    if (cfg == nullptr || out == nullptr) return fail(VL_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->abi_version != VL_ABI_VERSION) return fail(VL_ERR_INVALID, "ABI version mismatch");
    if (cfg->precision != VL_FP64 && cfg->precision != VL_FP32)
        return fail(VL_ERR_INVALID, "precision must be VL_FP64 or VL_FP32");
    if (cfg->n < 1 || cfg->n > vl::NMAX) return fail(VL_ERR_UNSUPPORTED, "n must be in 1..10");
    if (cfg->nx < 1 || cfg->nu < 1 || cfg->nv < 1) return fail(VL_ERR_INVALID, "empty grid");
    if (cfg->nx * cfg->n > vl::FIELD_MAX_NODES)
        return fail(VL_ERR_TOO_LARGE, "nx * n exceeds the field kernel capacity (640)");
    if (cfg->n_modes < 1 || cfg->n_modes > vl::FIELD_MAX_MODES)
        return fail(VL_ERR_TOO_LARGE, "number of DFT modes exceeds the field kernel capacity (321)");
    if (!cfg->up || !cfg->xi || !cfg->xw || !cfg->u_nodes || !cfg->v_nodes || !cfg->wave_numbers ||
        !cfg->dft_ell || !cfg->dft_phase || !cfg->dft_qnode)
        return fail(VL_ERR_INVALID, "null table pointer");
    const size_t elems = (size_t)(cfg->nx + 2) * cfg->n * (cfg->nu + 2) * cfg->n *
                         (cfg->nv + 2) * cfg->n;
    if (elems >= ((size_t)1 << 40)) return fail(VL_ERR_TOO_LARGE, "state too large");
    // offsets inside one x slab are 32-bit in the stage kernel
    if (elems / (size_t)(cfg->nx + 2) >= ((size_t)1 << 31))
        return fail(VL_ERR_TOO_LARGE, "one x slab of the state exceeds 2^31 elements");

    vl_ctx *c = new vl_ctx();
    c->cfg = *cfg;
    c->cfg.up = c->cfg.xi = c->cfg.xw = c->cfg.u_nodes = c->cfg.v_nodes = nullptr;
    c->cfg.wave_numbers = c->cfg.dft_ell = c->cfg.dft_phase = c->cfg.dft_qnode = nullptr;
    const int n = cfg->n;
    std::memset(c->up, 0, sizeof(c->up));
    std::memset(c->xi, 0, sizeof(c->xi));
    std::memset(c->qw, 0, sizeof(c->qw));
    std::memcpy(c->up, cfg->up, sizeof(double) * n * n);
    std::memcpy(c->xi, cfg->xi, sizeof(double) * n * 2);
    std::memcpy(c->xw, cfg->xw, sizeof(double) * n);
    // velocity quadrature weights w_j w_k / (J_u J_v) (main/grid.py:297-301)
    const double jj = cfg->ju * cfg->jv;
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k) c->qw[j * n + k] = (cfg->xw[j] * cfg->xw[k]) / jj;

    int rc = VL_OK;
    auto cleanup = [&](int code) {
        vl_ctx_destroy(c);
        return code;
    };
    cudaError_t e = cudaGetDevice(&c->device);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaGetDevice"));
    e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaDeviceGetAttribute"));
    if ((rc = upload(&c->d_unodes, cfg->u_nodes, sizeof(double) * (cfg->nu + 2) * n))) return cleanup(rc);
    {
        // x and v flux speeds per u node, in the kernels' own expression order and precision
        // (u; a (-B u))
        const int nun = (cfg->nu + 2) * n;
        if (cfg->precision == VL_FP64) {
            std::vector<double2> t(nun);
            for (int q = 0; q < nun; ++q) {
                const double u = cfg->u_nodes[q];
                t[q] = make_double2(u, cfg->accel * (-cfg->bfield * u));
            }
            if ((rc = upload(&c->d_usv, t.data(), sizeof(double2) * nun))) return cleanup(rc);
        } else {
            std::vector<float2> t(nun);
            for (int q = 0; q < nun; ++q) {
                const double u = cfg->u_nodes[q];
                t[q] = make_float2((float)u, (float)(cfg->accel * (-cfg->bfield * u)));
            }
            if ((rc = upload(&c->d_usv, t.data(), sizeof(float2) * nun))) return cleanup(rc);
            // the FP32 n = 8 kernel's pairs: {u J_x, u J_x, a (-B u) J_v, a (-B u) J_v}
            std::vector<float4> t4(nun);
            for (int q = 0; q < nun; ++q) {
                const double u = cfg->u_nodes[q];
                const float ux = (float)(u * cfg->jx), sv = (float)(cfg->accel * (-cfg->bfield * u) * cfg->jv);
                t4[q] = make_float4(ux, ux, sv, sv);
            }
            if ((rc = upload(&c->d_usv4, t4.data(), sizeof(float4) * nun))) return cleanup(rc);
        }
    }
    if ((rc = upload(&c->d_vnodes, cfg->v_nodes, sizeof(double) * (cfg->nv + 2) * n))) return cleanup(rc);
    if ((rc = upload(&c->d_k, cfg->wave_numbers, sizeof(double) * cfg->n_modes))) return cleanup(rc);
    if ((rc = upload(&c->d_xw, cfg->xw, sizeof(double) * n))) return cleanup(rc);
    const size_t nm = sizeof(double2) * (size_t)n * cfg->n_modes;
    if ((rc = upload(&c->d_ell, cfg->dft_ell, nm))) return cleanup(rc);
    if ((rc = upload(&c->d_phase, cfg->dft_phase, sizeof(double2) * (size_t)cfg->nx * cfg->n_modes)))
        return cleanup(rc);
    if ((rc = upload(&c->d_qnode, cfg->dft_qnode, nm))) return cleanup(rc);
    {
        const cudaError_t ee = cudaFuncSetAttribute(
            vl::field_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
            (int)std::max(vl::field_solve_smem(vl::NMAX, vl::FIELD_MAX_MODES), vl::FIELD_DYN_SMEM_MAX));
        if (ee != cudaSuccess) return cleanup(cuda_fail(ee, "cudaFuncSetAttribute(field_solve_kernel)"));
    }
    {
        std::vector<double> tabs((size_t)2 * n * n + 2 * n);
        std::memcpy(tabs.data(), c->up, sizeof(double) * n * n);
        std::memcpy(tabs.data() + n * n, c->xi, sizeof(double) * 2 * n);
        std::memcpy(tabs.data() + n * n + 2 * n, c->qw, sizeof(double) * n * n);
        if ((rc = upload(&c->d_tables, tabs.data(), sizeof(double) * tabs.size()))) return cleanup(rc);
    }

    {
        int *e0 = nullptr;
        cudaError_t ee = cudaMalloc((void **)&e0, sizeof(int));
        if (ee != cudaSuccess) return cleanup(cuda_fail(ee, "cudaMalloc(err)"));
        c->d_err = e0;
        ee = cudaMemset(c->d_err, 0, sizeof(int));
        if (ee != cudaSuccess) return cleanup(cuda_fail(ee, "cudaMemset(err)"));
    }
    c->use_tma = (cfg->precision == VL_FP64 ? tma_supported<double>(*cfg) : tma_supported<float>(*cfg)) &&
                 encode_fn() != nullptr;
    {
        const char *env = getenv("VLASOV1D2V_NO_TMA");
        if (env && env[0] == '1') c->use_tma = false;
    }
    // CTAs per x element: fill the device (resident CTAs x SMs), at most one per tile
    c->use_frag = c->use_tma && n == 8;
    {
        const char *env = getenv("VLASOV1D2V_NO_FRAG");
        if (env && env[0] == '1') c->use_frag = false;
    }
    // stage kernel (fastest measured per order and precision): the fragment kernel for n = 8; in
    // FP64 the generic kernel for every other order (its TMA form where the rows allow); in FP32
    // the TMA kernel for n = 4, the generic kernel's TMA form on 16-byte rows and the
    // register-pencil kernel otherwise.
    // VLASOV1D2V_STAGE_KERNEL=frag|gen|pencil selects one of the forms that apply, for comparisons
    // FP32 on the generic kernel's TMA form where the rows are 16-byte multiples ((nv+2) n a
    // multiple of 4), orders other than 4 and 8; VLASOV1D2V_GEN_NO_TMA=1 switches it off
    const bool no_gen_tma = [] {
        const char *env = getenv("VLASOV1D2V_GEN_NO_TMA");
        return env && env[0] == '1';
    }();
    const bool gen_tma32 = cfg->precision == VL_FP32 && ((size_t)(cfg->nv + 2) * n) % 4 == 0 && !no_gen_tma &&
                           encode_fn() != nullptr;
    // FP32 rows of R = 2 mod 4 floats over an even number of rows: the paired-row TMA form
    const bool gen_pair32 = cfg->precision == VL_FP32 && ((size_t)(cfg->nv + 2) * n) % 4 == 2 &&
                            ((size_t)(cfg->nu + 2) * n) % 2 == 0 && !no_gen_tma && encode_fn() != nullptr;
    c->stage_kernel = c->use_frag                                  ? VL_STAGE_FRAG
                      : cfg->precision == VL_FP64                  ? VL_STAGE_GEN
                      : c->use_tma                                 ? VL_STAGE_TMA
                      : (gen_tma32 || gen_pair32)                  ? VL_STAGE_GEN
                                                                   : VL_STAGE_PENCIL;
    {
        const char *env = getenv("VLASOV1D2V_STAGE_KERNEL");
        if (env) {
            const std::string k(env);
            if (k == "gen") c->stage_kernel = VL_STAGE_GEN;
            else if (k == "pencil") c->stage_kernel = VL_STAGE_PENCIL;
            else if (k == "frag" && c->use_frag) c->stage_kernel = VL_STAGE_FRAG;
        }
        c->use_frag = c->stage_kernel == VL_STAGE_FRAG;
        if (c->stage_kernel != VL_STAGE_TMA && c->stage_kernel != VL_STAGE_FRAG) c->use_tma = false;
    }
    const bool gen = c->stage_kernel == VL_STAGE_GEN;
    // generic kernel in its TMA form: FP64 rows of a 16-byte multiple (V n even), FP32 as above
    c->gen_tma = gen && (cfg->precision == VL_FP64 ? ((size_t)(cfg->nv + 2) * n) % 2 == 0 : gen_tma32) &&
                 encode_fn() != nullptr && !no_gen_tma;
    c->gen_pair = gen && !c->gen_tma && gen_pair32;
    const int occ = cfg->precision == VL_FP64
                        ? stage_occupancy<double>(n, c->use_tma, c->use_frag, gen, c->gen_tma, false)
                        : stage_occupancy<float>(n, c->use_tma, c->use_frag, gen, c->gen_tma, c->gen_pair);
    const int bt = stage_epw(c);
    const int tiles = cfg->nu * ((cfg->nv + bt - 1) / bt);
    // one wave: at most occ x SMs resident CTAs in total (a second partial wave would double
    // the kernel time)
    auto grid_for = [&](int o) {
        int g = (c->sm_count * o) / cfg->nx;
        if (g > tiles) g = tiles;
        if (g < 1) g = 1;
        return g;
    };
    c->stage_grid_g = grid_for(occ);
    c->stage_grid_g1 = (c->use_frag && cfg->precision == VL_FP64) ? grid_for(frag_nofn_occupancy())
                                                                  : c->stage_grid_g;
    // standalone moment: MOMENT_CTAS_PER_SM resident CTAs per SM, at most one per u element
    int gm = (c->sm_count * vl::MOMENT_CTAS_PER_SM) / cfg->nx;
    if (gm > cfg->nu) gm = cfg->nu;
    if (gm < 1) gm = 1;
    c->moment_grid_g = gm;
    {
        const cudaError_t ee =
            cudaMalloc((void **)&c->d_moment, sizeof(double) * (size_t)cfg->nx * gm * n);
        if (ee != cudaSuccess) return cleanup(cuda_fail(ee, "cudaMalloc(moment partials)"));
    }
    *out = c;
    return VL_OK;
}

int vl_ctx_destroy(vl_ctx *c) {
    if (c == nullptr) return VL_OK;
    cudaFree(c->d_unodes);
    cudaFree(c->d_usv);
    cudaFree(c->d_usv4);
    cudaFree(c->d_vnodes);
    cudaFree(c->d_k);
    cudaFree(c->d_xw);
    cudaFree(c->d_ell);
    cudaFree(c->d_phase);
    cudaFree(c->d_qnode);
    cudaFree(c->d_tables);
    cudaFree(c->d_moment);
    cudaFree(c->d_err);
    delete c;
    return VL_OK;
}

size_t vl_state_elems(const vl_ctx *c) {
    if (c == nullptr) return 0;
    const vl_config &g = c->cfg;
    return (size_t)(g.nx + 2) * g.n * (g.nu + 2) * g.n * (g.nv + 2) * g.n;
}

size_t vl_workspace_bytes(const vl_ctx *c) {
    if (c == nullptr) return 0;
    return partials_bytes(c);
}

int vl_rhs(vl_ctx *c, const void *f, const double *E, void *out, int xhalo, void *stream) {
    if (!c || !f || !E || !out) return fail(VL_ERR_INVALID, "null argument");
    if (xhalo != VL_XHALO_GHOST && xhalo != VL_XHALO_PERIODIC) return fail(VL_ERR_INVALID, "xhalo");
    vl::StageArgs a = stage_args(c);
    a.in = f;
    a.out = out;
    a.E = E;
    a.xhalo = xhalo;
    a.kind = vl::KIND_RHS;
    return stage(c, a, as_stream(stream));
}

int vl_rhs_weighted(vl_ctx *c, const void *f, const double *E, void *out, int xhalo,
                    const double *w, void *stream) {
    if (!c || !f || !E || !out || !w) return fail(VL_ERR_INVALID, "null argument");
    if (xhalo != VL_XHALO_GHOST && xhalo != VL_XHALO_PERIODIC) return fail(VL_ERR_INVALID, "xhalo");
    vl::StageArgs a = stage_args(c);
    a.in = f;
    a.out = out;
    a.E = E;
    a.xhalo = xhalo;
    a.kind = vl::KIND_RHS;
    a.jx = w[0];
    a.ju = w[1];
    a.jv = w[2];
    return stage(c, a, as_stream(stream));
}

int vl_moment(vl_ctx *c, const void *f, double *rho, void *stream) {
    if (!c || !f || !rho) return fail(VL_ERR_INVALID, "null argument");
    cudaStream_t s = as_stream(stream);
    const int G = c->moment_grid_g;
    int rc = moment(c, f, c->d_moment, G, s);
    if (rc) return rc;
    const int nn = c->cfg.nx * c->cfg.n;
    vl::moment_reduce_kernel<<<(nn + 255) / 256, 256, 0, s>>>(c->d_moment, rho, c->cfg.nx, G, c->cfg.n);
    return check_launch("moment_reduce_kernel");
}

int vl_poisson(vl_ctx *c, const double *charge, double *E, double *phi, void *stream) {
    if (!c || !charge || !E) return fail(VL_ERR_INVALID, "null argument");
    vl::FieldArgs a = field_args(c);
    a.charge_in = charge;
    a.E = E;
    a.phi = phi;
    return field(c, a, as_stream(stream));
}

int vl_field_energy(vl_ctx *c, const double *E, double *energy, void *stream) {
    if (!c || !E || !energy) return fail(VL_ERR_INVALID, "null argument");
    vl::ScalarArgs a = scalar_args(c, E);
    a.energy = energy;
    vl::scalars_kernel<<<1, vl::FIELD_THREADS, 0, as_stream(stream)>>>(a);
    return check_launch("scalars_kernel");
}

int vl_adapt_dt(vl_ctx *c, const double *E, double *dt, void *stream) {
    if (!c || !E || !dt) return fail(VL_ERR_INVALID, "null argument");
    vl::ScalarArgs a = scalar_args(c, E);
    a.dt = dt;
    vl::scalars_kernel<<<1, vl::FIELD_THREADS, 0, as_stream(stream)>>>(a);
    return check_launch("scalars_kernel");
}

int vl_rk_stage(vl_ctx *c, int stg, const void *in, const void *fn, void *out, const double *E,
                const double *dt, int xhalo, void *workspace, void *stream) {
    if (!c || !in || !out || !E || !dt) return fail(VL_ERR_INVALID, "null argument");
    if (stg < 0 || stg > 2) return fail(VL_ERR_INVALID, "stage must be 0, 1 or 2");
    if (stg > 0 && !fn) return fail(VL_ERR_INVALID, "fn required for stages 1 and 2");
    if (xhalo != VL_XHALO_GHOST && xhalo != VL_XHALO_PERIODIC) return fail(VL_ERR_INVALID, "xhalo");
    vl::StageArgs a = stage_args(c);
    a.in = in;
    a.fn = fn;
    a.out = out;
    a.E = E;
    a.dt = dt;
    a.xhalo = xhalo;
    a.partials = static_cast<double *>(workspace);
    if (stg == 0) {
        a.kind = vl::KIND_EULER;
    } else {
        a.kind = vl::KIND_COMBINE;
        a.c0 = kRK3[stg - 1][0];
        a.c1 = kRK3[stg - 1][1];
        a.c2 = kRK3[stg - 1][2];
    }
    return stage(c, a, as_stream(stream));
}

int vl_run_state_init(vl_ctx *c, vl_run_state *state, const double *E0, double final_time,
                      int64_t max_steps, double *eh, double *th, double *dh, int32_t cap,
                      double *energy0, void *stream) {
    if (!c || !state || !E0) return fail(VL_ERR_INVALID, "null argument");
    if (cap < 0) return fail(VL_ERR_INVALID, "history capacity");
    vl::ScalarArgs a = scalar_args(c, E0);
    a.energy = energy0;
    a.init = state;
    a.final_time = final_time;
    a.max_steps = max_steps;
    a.eh = eh;
    a.th = th;
    a.dh = dh;
    a.cap = cap;
    vl::scalars_kernel<<<1, vl::FIELD_THREADS, 0, as_stream(stream)>>>(a);
    return check_launch("scalars_kernel(init)");
}

int vl_set_background_pairs(vl_ctx *c, const float *pairs) {
    if (!c) return fail(VL_ERR_INVALID, "null context");
    if (pairs && c->cfg.precision != VL_FP32)
        return fail(VL_ERR_UNSUPPORTED, "the background split is a form of the FP32 context");
    if (pairs && (((c->cfg.nv + 2) * c->cfg.n) % 2 != 0))
        return fail(VL_ERR_INVALID, "background pair table needs an even row length (nv+2) n");
    if (reinterpret_cast<uintptr_t>(pairs) & 15) return fail(VL_ERR_INVALID, "background pair table must be 16-byte aligned");
    c->bg_pair = pairs;
    return VL_OK;
}

int vl_set_background(vl_ctx *c, const float *rb, const float *eu) {
    if (!c) return fail(VL_ERR_INVALID, "null context");
    if ((rb == nullptr) != (eu == nullptr)) return fail(VL_ERR_INVALID, "background tables: give both or none");
    if (rb && c->cfg.precision != VL_FP32)
        return fail(VL_ERR_UNSUPPORTED, "the background split is a form of the FP32 context");
    if ((reinterpret_cast<uintptr_t>(rb) | reinterpret_cast<uintptr_t>(eu)) & 15)
        return fail(VL_ERR_INVALID, "background tables must be 16-byte aligned");
    c->bg_rb = rb;
    c->bg_eu = eu;
    if (rb == nullptr) c->bg_pair = nullptr;   // the pair table belongs to the split
    return VL_OK;
}

int vl_sync_ghosts(vl_ctx *c, void *f, void *stage_buf, void *stream) {
    if (!c || !f) return fail(VL_ERR_INVALID, "null argument");
    cudaStream_t s = as_stream(stream);
    const size_t es = elem_size(c);
    const size_t slab = vl_state_elems(c) / (size_t)(c->cfg.nx + 2) * es;
    char *fb = static_cast<char *>(f);
    // Distribution.swap_ghost_cells_of_array (main/grid.py:187-189)
    VL_CUDA(cudaMemcpyAsync(fb, fb + slab * c->cfg.nx, slab, cudaMemcpyDeviceToDevice, s));
    VL_CUDA(cudaMemcpyAsync(fb + slab * (c->cfg.nx + 1), fb + slab, slab, cudaMemcpyDeviceToDevice, s));
    if (stage_buf != nullptr && stage_buf != f)
        VL_CUDA(cudaMemcpyAsync(stage_buf, f, vl_state_elems(c) * es, cudaMemcpyDeviceToDevice, s));
    return VL_OK;
}

int vl_ssp_rk3_steps(vl_ctx *c, void *f, void *sa, void *sb, double *E, double *phi,
                     vl_run_state *state, void *workspace, int nsteps, void *stream) {
    if (!c || !f || !sa || !sb || !E || !state || !workspace)
        return fail(VL_ERR_INVALID, "null argument");
    if (nsteps < 0) return fail(VL_ERR_INVALID, "nsteps < 0");
    cudaStream_t s = as_stream(stream);
    double *partials = static_cast<double *>(workspace);
    const int G = c->stage_grid_g;
    int rc;
    // moment partials of f^n for the first step's field solve
    if ((rc = moment(c, f, partials, c->moment_grid_g, s))) return rc;
    vl::FieldArgs fa = field_args(c);
    fa.partials = partials;
    fa.G = c->moment_grid_g;
    fa.E = E;
    fa.state = state;
    vl::StageArgs st = stage_args(c);
    st.E = E;
    st.dt = &state->dt;
    st.state = state;
    st.err = &state->status;   // bounded-wait timeouts are reported in the loop state
    st.xhalo = VL_XHALO_PERIODIC;
    st.partials = partials;
    for (int it = 0; it < nsteps; ++it) {
        // stage 0: E(f^n); s0 = f + dt R(f)  (main/timestep.py:153-163)
        fa.mode = vl::FIELD_PROMOTE;
        fa.phi = nullptr;
        if ((rc = field(c, fa, s))) return rc;
        st.in = f;
        st.fn = nullptr;
        st.out = sa;
        st.ghost_out = f;
        st.kind = vl::KIND_EULER;
        if ((rc = stage(c, st, s))) return rc;
        // stage 1: E(s0); s1 = 3/4 f + 1/4 s0 + 1/4 dt R(s0)
        fa.mode = vl::FIELD_REQUIRE_ACTIVE;
        fa.G = c->stage_grid_g1;   // partials of the Euler stage's grid
        if ((rc = field(c, fa, s))) return rc;
        st.in = sa;
        st.fn = f;
        st.out = sb;
        st.ghost_out = nullptr;
        st.kind = vl::KIND_COMBINE;
        st.c0 = kRK3[0][0];
        st.c1 = kRK3[0][1];
        st.c2 = kRK3[0][2];
        if ((rc = stage(c, st, s))) return rc;
        // stage 2: E(s1) (+ energy, dt, time: main/timestep.py:98-103, :184-185);
        //          f <- 1/3 f + 2/3 s1 + 2/3 dt R(s1)
        fa.mode = vl::FIELD_REQUIRE_ACTIVE | vl::FIELD_RECORD;
        fa.phi = phi;
        fa.G = G;                  // from here on the partials of the combination stages' grid
        if ((rc = field(c, fa, s))) return rc;
        st.in = sb;
        st.fn = f;
        st.out = f;
        st.c0 = kRK3[1][0];
        st.c1 = kRK3[1][1];
        st.c2 = kRK3[1][2];
        if ((rc = stage(c, st, s))) return rc;
    }
    return VL_OK;
}

}  // extern "C"
