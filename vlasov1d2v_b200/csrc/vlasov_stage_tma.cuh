// Fused SSP-RK stage kernel, TMA-pipelined form (sm_100a).
//
// Used when the node rows are 16-byte aligned for the tensor-memory accelerator (n * sizeof(T)
// a multiple of 16 B and 32 / n elements per tile: n = 2, 4, 8 in FP64; n = 4, 8 in FP32).
//
// Tile = (x element e, u element a, EPW = 32 / n consecutive v elements): COLS = EPW n v-node
// columns, n x n (i, j) rows.  Lane c of every warp owns column c; warp w owns the j chunk
// [w JC, w JC + JC).  Per tile one elected thread issues cp.async.bulk.tensor loads (no
// multicast) into a shared-memory stage:
//   IN  [i][j][COLS + 2P]  stage input incl. P pad columns each side (the v upwind traces)
//   FN  [i][j][COLS]       f^n (RK combination stages only)
//   XF  [side][j][COLS]    x upwind traces: (e-1, i = n-1) and (e+1, i = 0)
//   UF  [side][i][COLS]    u upwind traces: (a-1, j = n-1) and (a+1, j = 0)
// completing on the stage's mbarrier.  Two stages: tile q+1 streams in while tile q is
// computed.  Compute per output node (i, j, c): u contraction over the shared j-row, x
// contraction over the thread's register copy of its i-columns, v contraction over the
// element's shared k-line (broadcast reads), upwind lifts, Jacobian-weighted sum, RK
// combination, coalesced store, moment partial.  All waits are bounded: on timeout the kernel
// raises bit 1 of the error word and returns.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "vlasov_kernels.cuh"
#include "vlasov_stage.cuh"

#ifndef VL_TMA_JC64
#define VL_TMA_JC64 2
#endif
#ifndef VL_TMA_JC32
#define VL_TMA_JC32 4
#endif
// 1: f^n tiles stream through shared memory with TMA; 0: each thread reads its f^n values
// straight from global memory (less shared memory per CTA, more resident CTAs)
#ifndef VL_TMA_STAGE_FN
#define VL_TMA_STAGE_FN 1
#endif

namespace vl {

template <int N, typename T>
struct TmaGeom {
    static constexpr int P = 16 / (int)sizeof(T);            // pad columns (16 bytes)
    static constexpr int EPW = 32 / N;
    static constexpr int COLS = EPW * N;
    static constexpr int W = COLS + 2 * P;                    // IN row length
    static constexpr int JC = sizeof(T) == 8 ? VL_TMA_JC64 : VL_TMA_JC32;
    static constexpr bool SUPPORTED_SHAPE = ((N * (int)sizeof(T)) % 16 == 0) && (32 % N == 0);
    static constexpr int NW = (N + JC - 1) / JC;               // warps
    static_assert(!SUPPORTED_SHAPE || NW <= 8, "at most 8 j chunks per tile");
    static constexpr int THREADS = 32 * NW;
    static constexpr int VEC = (sizeof(T) == 8) ? ((N % 2 == 0) ? 2 : 1) : ((N % 4 == 0) ? 4 : 1);
    static constexpr bool SUPPORTED = SUPPORTED_SHAPE;
    // stage layout (bytes, 128-aligned pieces)
    static constexpr size_t al(size_t b) { return (b + 127) & ~(size_t)127; }
    static constexpr size_t IN_B = al(sizeof(T) * (size_t)W * N * N);
    static constexpr bool STAGE_FN = VL_TMA_STAGE_FN != 0;
    static constexpr size_t FN_B = STAGE_FN ? al(sizeof(T) * (size_t)COLS * N * N) : 0;
    static constexpr size_t XF_B = al(sizeof(T) * (size_t)2 * COLS * N);
    static constexpr size_t UF_B = al(sizeof(T) * (size_t)2 * COLS * N);
    static constexpr size_t STAGE_B = IN_B + FN_B + XF_B + UF_B;
    static constexpr size_t MOM_B = al(sizeof(double) * (size_t)N * THREADS);
    static constexpr size_t smem_bytes() { return 2 * STAGE_B + MOM_B + 128; }
    static constexpr uint32_t TX_IN = sizeof(T) * W * N * N;
    static constexpr uint32_t TX_FN = sizeof(T) * COLS * N * N;
    static constexpr uint32_t TX_FACE = sizeof(T) * COLS * N;   // one face box
};

struct TmaMaps {
    CUtensorMap in_tile;   // box (W, n, 1, n, 1) over the stage input
    CUtensorMap in_xface;  // box (COLS, n, 1, 1, 1)
    CUtensorMap in_uface;  // box (COLS, 1, 1, n, 1)
    CUtensorMap fn_tile;   // box (COLS, n, 1, n, 1) over f^n
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// one arrival (release semantics at CTA scope) on a barrier without a transaction count
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false after ~2^22 polls (the caller reports a timeout and returns)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1, int c2, int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6, %7}], [%2];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1, int c2, int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(smem_addr(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
        : "memory");
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_addr(dst)),
        "l"(map), "r"(smem_addr(bar)), "r"(c0), "r"(c1)
        : "memory");
}

// untiled bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16)
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

#ifndef VL_SPLIT_SUM
#define VL_SPLIT_SUM 0
#endif
#ifndef VL_TMA_MINB
#define VL_TMA_MINB 1
#endif

// sum_m coef(m) v[m] with two interleaved partial sums (halves the FMA dependency chain)
template <int N, typename T, typename C>
__device__ __forceinline__ T dot_n(C coef, const T (&v)[N]) {
    if constexpr (VL_SPLIT_SUM && N >= 4) {
        T s0 = (T)0, s1 = (T)0;
#pragma unroll
        for (int m = 0; m + 1 < N; m += 2) {
            s0 = fma(coef(m), v[m], s0);
            s1 = fma(coef(m + 1), v[m + 1], s1);
        }
        if constexpr (N % 2) s0 = fma(coef(N - 1), v[N - 1], s0);
        return s0 + s1;
    } else {
        T s = (T)0;
#pragma unroll
        for (int m = 0; m < N; ++m) s = fma(coef(m), v[m], s);
        return s;
    }
}

template <int N, typename T>
__global__ void __launch_bounds__(TmaGeom<N, T>::THREADS, VL_TMA_MINB)
stage_tma_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb,
                 const __grid_constant__ TmaMaps maps) {
    using G = TmaGeom<N, T>;
    constexpr int P = G::P, EPW = G::EPW, COLS = G::COLS, W = G::W, JC = G::JC, NT = G::THREADS;
    constexpr int VEC = G::VEC;
    if (a.state != nullptr && a.state->active == 0) return;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    double *sMom = reinterpret_cast<double *>(base + 2 * G::STAGE_B);
    __shared__ __align__(8) uint64_t full[2];
    __shared__ double sE[N];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int c = lane;                     // column
    const int bl = c / N, k = c - (c / N) * N;
    const bool lane_ok = c < COLS;

    const int nx = a.nx, nu = a.nu, nv = a.nv;
    const int U = nu + 2, V = nv + 2;
    const int sJ = V * N, sA = sJ * N, sI = sA * U;
    const size_t sE_ = (size_t)sI * N;
    const int e = blockIdx.y, Eg = e + 1;
    int El, Er;
    if (a.xhalo == VL_XHALO_PERIODIC) {
        El = (e == 0) ? nx : e;
        Er = (e == nx - 1) ? 1 : e + 2;
    } else {
        El = e;
        Er = e + 2;
    }
    const int kind = a.kind;
    const bool with_fn = (kind == KIND_COMBINE);
    const uint32_t tx_bytes = G::TX_IN + 4 * G::TX_FACE + ((with_fn && G::STAGE_FN) ? G::TX_FN : 0);
    const int nbt = (nv + EPW - 1) / EPW;
    const int tiles = nu * nbt;
    const int ntile_cta = (blockIdx.x < tiles) ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (tid < N) sE[tid] = a.E[Eg * N + tid];
#pragma unroll
    for (int i = 0; i < N; ++i) sMom[i * NT + tid] = 0.0;
    __syncthreads();

    auto stage_ptr = [&](int s) { return base + (size_t)s * G::STAGE_B; };
    auto issue = [&](int s, int q) {
        const int t = blockIdx.x + q * gridDim.x;
        const int au = t / nbt;
        const int b0 = (t - au * nbt) * EPW;
        const int Ag = au + 1;
        const int x0 = (b0 + 1) * N;
        unsigned char *st = stage_ptr(s);
        mbar_arrive_expect_tx(&full[s], tx_bytes);
        tma_load_5d(st, &maps.in_tile, &full[s], x0 - P, 0, Ag, 0, Eg);
        tma_load_5d(st + G::IN_B + G::FN_B, &maps.in_xface, &full[s], x0, 0, Ag, N - 1, El);
        tma_load_5d(st + G::IN_B + G::FN_B + sizeof(T) * COLS * N, &maps.in_xface, &full[s], x0, 0,
                    Ag, 0, Er);
        tma_load_5d(st + G::IN_B + G::FN_B + G::XF_B, &maps.in_uface, &full[s], x0, N - 1, Ag - 1, 0,
                    Eg);
        tma_load_5d(st + G::IN_B + G::FN_B + G::XF_B + sizeof(T) * COLS * N, &maps.in_uface, &full[s],
                    x0, 0, Ag + 1, 0, Eg);
        if (G::STAGE_FN && with_fn) tma_load_5d(st + G::IN_B, &maps.fn_tile, &full[s], x0, 0, Ag, 0, Eg);
    };
    if (tid == 0) {
        if (ntile_cta > 0) issue(0, 0);
        if (ntile_cta > 1) issue(1, 1);
    }

    const double accel = a.accel, bfield = a.bfield, nbfield = -a.bfield;
    const double dtd = (kind == KIND_RHS) ? 0.0 : *a.dt;
    const T dtT = (T)dtd, c0 = (T)a.c0, c1 = (T)a.c1, c2dt = (T)(a.c2 * dtd);
    const T jx = (T)a.jx, ju = (T)a.ju, jv = (T)a.jv;
    const int kk = lane_ok ? k : 0;
    T upk[N];
#pragma unroll
    for (int m = 0; m < N; ++m) upk[m] = tb.up[kk * N + m];
    const T xik0 = tb.xi[2 * kk], xik1 = tb.xi[2 * kk + 1];
    T *out = static_cast<T *>(a.out);
    T *gout = static_cast<T *>(a.ghost_out);

    for (int q = 0; q < ntile_cta; ++q) {
        const int s = q & 1;
        const int t = blockIdx.x + q * gridDim.x;
        const int au = t / nbt;
        const int b0 = (t - au * nbt) * EPW;
        const int nb = min(EPW, nv - b0);
        const int Ag = au + 1;
        const int col = (b0 + 1) * N + c;
        const bool act = lane_ok && (bl < nb);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((q >> 1) & 1))) {
            if (a.err != nullptr) atomicOr(a.err, 2);
            return;
        }
        const T *sIn = reinterpret_cast<const T *>(stage_ptr(s));
        const T *sFn = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B);
        const T *sXF = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B + G::FN_B);
        const T *sUF = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B);

        auto tile_body = [&](auto wj) {
            constexpr int J0 = decltype(wj)::value * JC;
            constexpr int JN = (J0 + JC <= N) ? JC : (N - J0);
            double wk[JC];
#pragma unroll
            for (int jc = 0; jc < JC; ++jc) wk[jc] = (jc < JN && lane_ok) ? tb.qw[(J0 + jc) * N + kk] : 0.0;
            double ux[JC];
            T f[N][JC];
            T xh[JC];
#pragma unroll
            for (int jc = 0; jc < JN; ++jc) {
                const int j = J0 + jc;
                ux[jc] = a.u_nodes[Ag * N + j];
#pragma unroll
                for (int m = 0; m < N; ++m) f[m][jc] = sIn[(m * N + j) * W + P + c];
                xh[jc] = sXF[((ux[jc] >= 0.0) ? 0 : COLS * N) + j * COLS + c];
            }
            if (gout != nullptr && (e == nx - 1 || e == 0)) {
                // periodic x-ghost refresh of f (Distribution.swap_ghost_cells_of_array)
                T *pg = gout + (size_t)Ag * sA + col;
#pragma unroll
                for (int jc = 0; jc < JN; ++jc) {
                    const int j = J0 + jc;
#pragma unroll
                    for (int m = 0; m < N; ++m) {
                        if (e == nx - 1) pg[m * sI + j * sJ] = f[m][jc];
                        if (e == 0) pg[(size_t)(nx + 1) * sE_ + m * sI + j * sJ] = f[m][jc];
                    }
                }
            }
            const double vnode = a.v_nodes[col];
            T *pout = out + (size_t)Eg * sE_ + (size_t)Ag * sA + col;
            const T *pfn = static_cast<const T *>(a.fn) + ((size_t)Eg * sE_ + (size_t)Ag * sA + col);
#pragma unroll 1
            for (int i = 0; i < N; ++i) {
                T row[N];
#pragma unroll
                for (int j = 0; j < N; ++j) row[j] = sIn[(i * N + j) * W + P + c];
                const double s_d = accel * (sE[i] + bfield * vnode);
                const T sp = (T)s_d;
                const bool upos = s_d >= 0.0;
                const T uh = sUF[(upos ? 0 : COLS * N) + i * COLS + c];
                const T uL = upos ? uh : row[0];
                const T uR = upos ? row[N - 1] : uh;
                double mrow = 0.0;
#pragma unroll
                for (int jc = 0; jc < JN; ++jc) {
                    const int j = J0 + jc;
                    T du = dot_n<N, T>([&](int m) { return tb.up[j * N + m]; }, row);
                    du = fma(tb.xi[2 * j], uL, du);
                    du = fma(-tb.xi[2 * j + 1], uR, du);
                    const bool xpos = ux[jc] >= 0.0;
                    const T xL = xpos ? xh[jc] : f[0][jc];
                    const T xR = xpos ? f[N - 1][jc] : xh[jc];
                    T colv[N];
#pragma unroll
                    for (int m = 0; m < N; ++m) colv[m] = f[m][jc];
                    T dx = dot_n<N, T>([&](int m) { return tb.up[i * N + m]; }, colv);
                    dx = fma(tb.xi[2 * i], xL, dx);
                    dx = fma(-tb.xi[2 * i + 1], xR, dx);
                    const T *lp = sIn + (i * N + j) * W + P + bl * N;
                    T line[N];
                    load_line<N, VEC, T>(lp, line);
                    const double sv_d = accel * (nbfield * ux[jc]);
                    T dv = dot_n<N, T>([&](int m) { return upk[m]; }, line);
                    if (sv_d >= 0.0) {   // warp-uniform: upwind side of the v faces
                        dv = fma(xik0, lp[-1], dv);
                        dv = fma(-xik1, line[N - 1], dv);
                    } else {
                        dv = fma(xik0, line[0], dv);
                        dv = fma(-xik1, lp[N], dv);
                    }
                    T r = fma((T)ux[jc] * dx, jx, fma(sp * du, ju, ((T)sv_d * dv) * jv));
                    if (a.bg_rb != nullptr) {   // RHS of the x-independent background
                        const int vi = Ag * sA + j * sJ + col;
                        r += (T)fmaf((float)sE[i], a.bg_eu[vi], a.bg_rb[vi]);
                    }
                    const T fij = row[j];
                    T o;
                    if (kind == KIND_RHS) {
                        o = r;
                    } else if (kind == KIND_EULER) {
                        o = fma(dtT, r, fij);
                    } else {
                        const T fnv = G::STAGE_FN ? sFn[(i * N + j) * COLS + c] : pfn[i * sI + j * sJ];
                        o = rk_combine(c0, c1, c2dt, fnv, fij, r);
                    }
                    pout[i * sI + j * sJ] = o;
                    mrow = fma(wk[jc], (double)o, mrow);
                }
                sMom[i * NT + tid] += mrow;
            }
        };
        if (act) {
            switch (warp) {
                case 0: tile_body(std::integral_constant<int, 0>{}); break;
                case 1: if constexpr (G::NW > 1) tile_body(std::integral_constant<int, (G::NW > 1 ? 1 : 0)>{}); break;
                case 2: if constexpr (G::NW > 2) tile_body(std::integral_constant<int, (G::NW > 2 ? 2 : 0)>{}); break;
                case 3: if constexpr (G::NW > 3) tile_body(std::integral_constant<int, (G::NW > 3 ? 3 : 0)>{}); break;
                case 4: if constexpr (G::NW > 4) tile_body(std::integral_constant<int, (G::NW > 4 ? 4 : 0)>{}); break;
                case 5: if constexpr (G::NW > 5) tile_body(std::integral_constant<int, (G::NW > 5 ? 5 : 0)>{}); break;
                case 6: if constexpr (G::NW > 6) tile_body(std::integral_constant<int, (G::NW > 6 ? 6 : 0)>{}); break;
                case 7: if constexpr (G::NW > 7) tile_body(std::integral_constant<int, (G::NW > 7 ? 7 : 0)>{}); break;
                default: break;
            }
        }
        __syncthreads();   // stage s fully consumed
        if (tid == 0 && q + 2 < ntile_cta) issue(s, q + 2);
    }

    if (a.partials == nullptr) return;
    __syncthreads();
    const int nw = NT / 32;
    const int w = tid >> 5;
    for (int i = w; i < N; i += nw) {
        dd v = {0.0, 0.0};
        for (int qq = lane; qq < NT; qq += 32) v = dd_add(v, dd{sMom[i * NT + qq], 0.0});
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = dd_add(v, shfl_down_dd(v, off));
        if (lane == 0) a.partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * N + i] = v.hi + v.lo;
    }
}

}  // namespace vl
