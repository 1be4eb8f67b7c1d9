// Fused SSP-RK stage kernel for n = 8 in the quad-fragment layout (sm_100a).
//
// Tile = (x element e, u element a, 4 consecutive v elements): 32 v-node columns, 8 x 8 (i, j)
// rows.  Warps (w, h) own v element w of the tile and its j rows [h n / JS, (h + 1) n / JS)
// (JS warps per element, 1 by default: two measured slower in FP64); inside a warp, lane = 4 g + t owns the two
// output columns k = 2t, 2t + 1 of x node i = g, for the warp's j rows.  That is the accumulator
// layout of the FP64 tensor-core instruction mma.m8n8k4 (D[g][2t..2t+1]), so per j the
// x and v contractions run on the tensor cores (FP64 form) and land directly in the thread's
// outputs:
//   x:  D[i][k] += sum_m up[i][m] F[m][j][k]       A = up (registers), B = tile plane rows
//   v:  D[i][k] += sum_m F[i][j][m] up[k][m]       A = tile row slice, B = up^T (registers)
// with the own-trace part of each upwind lift folded into the up fragments selected by the sign
// of the speed (upP / upM) and the neighbour trace added by one FMA per output.  The u contraction
// mixes the j of one thread's own outputs and runs on the FMA pipes from a per-thread copy of
// F[i][0..7][k..k+1].  The row loop is instantiated per stage kind and for uniform upwind
// directions over the tile (a u element that does not straddle u = 0: fragments and face planes
// chosen once per tile) or per-row directions, and for the x-ghost-refresh rows of the edge x
// elements of stage 1 apart from the others, so it branches on none of these.  FP32 states at n = 8
// run the packed-FP32 kernel (vlasov_stage_f32.cuh) on this file's FragGeom<float> stage layout.
//
// Shared-memory stage (one TMA box each, no multicast):
//   IN [i][9][36 | 40]   stage input incl. pad columns (v traces) and one zero-filled row:
//                        the plane stride 9 W is 8 banks mod 32, so the fragment loads of
//                        four or eight planes are conflict-free
//   FN [i][9][34 | 36]   f^n (combination stages only)
//   XF [side][j][32]     x upwind traces: (e-1, i = n-1) and (e+1, i = 0)
//   UF [side][i][32]     u upwind traces: (a-1, j = n-1) and (a+1, j = 0)
//   BG [table][j][32]    FP32 background split only: the eu and rb RHS tables of the tile
//   US [j]               the x and v flux speeds (u, a (-B u)) of the tile's u nodes (bulk copy)
// Two stages: tile q+1 streams in while tile q is computed.  Every wait is bounded: on timeout
// the kernel raises bit 1 of the error word and returns.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "vlasov_kernels.cuh"
#include "vlasov_stage.cuh"
#include "vlasov_stage_tma.cuh"

#ifndef VL_FRAG_MINB64
#define VL_FRAG_MINB64 2
#endif
#ifndef VL_FRAG_MINB32
#define VL_FRAG_MINB32 4
#endif
// warps per v element (each takes n / JS consecutive j rows)
#ifndef VL_FRAG_JS64
#define VL_FRAG_JS64 1
#endif
#ifndef VL_FRAG_JS32
#define VL_FRAG_JS32 1
#endif

namespace vl {

// WFN: the stage holds an f^n tile (combination stages); without it (Euler and RHS stages) an FP64
// CTA needs 58 KB of shared memory instead of 97 KB, so three CTAs fit an SM
template <typename T, bool WFN = true>
struct FragGeom {
    static constexpr int N = 8;
    static constexpr int EPT = 4;                    // v elements per tile (one per warp)
    static constexpr int COLS = EPT * N;             // 32
    static constexpr int P = 16 / (int)sizeof(T);    // pad columns each side of IN (16 bytes)
    static constexpr int W = COLS + 2 * P;           // IN row length: 36 (FP64) | 40 (FP32)
    static constexpr int ROWS = N + 1;               // j rows per plane incl. one fill row
    static constexpr int PS = W * ROWS;              // IN plane stride: 324 | 360
    static constexpr int WF = COLS + P;              // FN row length: 34 | 36
    static constexpr int PSF = WF * ROWS;            // FN plane stride: 306 | 324
    static constexpr int JS = sizeof(T) == 8 ? VL_FRAG_JS64 : VL_FRAG_JS32;   // warps per v element
    static constexpr int NJ = N / JS;                // j rows per warp
    static constexpr int THREADS = 32 * EPT * JS;
    static constexpr bool MMA = sizeof(T) == 8;      // tensor-core x/v contractions (FP64)
    static constexpr int MINB = sizeof(T) == 8 ? (WFN ? VL_FRAG_MINB64 : 3) : VL_FRAG_MINB32;   // CTAs per SM
    static constexpr size_t al(size_t b) { return (b + 127) & ~(size_t)127; }
    static constexpr size_t IN_B = al(sizeof(T) * (size_t)PS * N);
    static constexpr size_t FN_B = WFN ? al(sizeof(T) * (size_t)PSF * N) : 0;
    static constexpr size_t XF_B = al(sizeof(T) * (size_t)2 * COLS * N);
    static constexpr size_t UF_B = XF_B;
    // background-split RHS tables (a form of the FP32 context only)
    static constexpr bool BG = sizeof(T) == 4;
    static constexpr size_t BG_B = BG ? al(sizeof(float) * (size_t)2 * COLS * N) : 0;
    static constexpr size_t UX_B = al(2 * sizeof(T) * (size_t)N);
    static constexpr size_t STAGE_B = IN_B + FN_B + XF_B + UF_B + BG_B + UX_B;
    static constexpr size_t smem_bytes() { return 2 * STAGE_B + 128; }
    static constexpr uint32_t TX_IN = sizeof(T) * W * ROWS * N;
    static constexpr uint32_t TX_FN = sizeof(T) * WF * ROWS * N;
    static constexpr uint32_t TX_FACE = sizeof(T) * COLS * N;
    static constexpr uint32_t TX_BG = sizeof(float) * COLS * N;
};

struct FragMaps {
    CUtensorMap in_tile;   // box (W, 9, 1, n, 1) over the stage input
    CUtensorMap in_xface;  // box (32, n, 1, 1, 1)
    CUtensorMap in_uface;  // box (32, 1, 1, n, 1)
    CUtensorMap fn_tile;   // box (WF, 9, 1, n, 1) over f^n
    CUtensorMap bg_eu;     // box (32, n) over the [U n][V n] background tables (FP32 split)
    CUtensorMap bg_rb;
};

// D[8x8] += A[8x4] B[4x8] in FP64 on the tensor cores; per lane (g = lane/4, t = lane%4):
// a = A[g][t], b = B[t][g], d0/d1 = D[g][2t], D[g][2t+1]
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

template <typename T>
struct Pair;
template <>
struct Pair<double> {
    using V = double2;
};
template <>
struct Pair<float> {
    using V = float2;
};

// KT >= 0 fixes the stage kind at compile time (the instantiations the loop launches: no per-row
// branches on it); -1 reads it from the arguments
template <typename T, bool WFN, int KT = -1>
__global__ void __launch_bounds__(FragGeom<T, WFN>::THREADS, FragGeom<T, WFN>::MINB)
stage_frag_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb,
                  const __grid_constant__ FragMaps maps) {
    using G = FragGeom<T, WFN>;
    using V2 = typename Pair<T>::V;
    constexpr int N = G::N, P = G::P, W = G::W, PS = G::PS, WF = G::WF, PSF = G::PSF;
    constexpr int COLS = G::COLS, EPT = G::EPT, NT = G::THREADS;
    if (a.state != nullptr && a.state->active == 0) return;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t full[2];
    __shared__ dd sRed[EPT * G::JS][N];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int wid = tid >> 5;
    const int w = wid % EPT;         // v element of the tile
    const int h = wid / EPT;         // j rows [h NJ, h NJ + NJ)
    const int g = lane >> 2;         // x node i of the thread's outputs
    const int t = lane & 3;          // columns 2t, 2t + 1 of the element
    const int wc = w * N;            // first tile column of the element
    const int cl = wc + 2 * t;       // first tile column of the thread

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
    const int kind = KT >= 0 ? KT : a.kind;   // compile-time in the loop's instantiations
    const bool with_fn = WFN && (kind == KIND_COMBINE);   // combination stages launch the WFN form
    const bool with_bg = G::BG && a.bg_rb != nullptr;
    const uint32_t tx_bytes = G::TX_IN + 4 * G::TX_FACE + (with_fn ? G::TX_FN : 0) + (with_bg ? 2 * G::TX_BG : 0) +
                              (uint32_t)(2 * sizeof(T)) * N;
    const int nbt = (nv + EPT - 1) / EPT;
    const int tiles = nu * nbt;
    const int ntile_cta = (blockIdx.x < tiles) ? (tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    auto stage_ptr = [&](int s) { return base + (size_t)s * G::STAGE_B; };
    auto issue = [&](int s, int q) {
        const int tt = blockIdx.x + q * gridDim.x;
        const int au = tt / nbt;
        const int b0 = (tt - au * nbt) * EPT;
        const int Ag = au + 1;
        const int x0 = (b0 + 1) * N;
        unsigned char *st = stage_ptr(s);
        unsigned char *xf = st + G::IN_B + G::FN_B;
        unsigned char *uf = xf + G::XF_B;
        mbar_arrive_expect_tx(&full[s], tx_bytes);
        tma_load_5d(st, &maps.in_tile, &full[s], x0 - P, 0, Ag, 0, Eg);
        tma_load_5d(xf, &maps.in_xface, &full[s], x0, 0, Ag, N - 1, El);
        tma_load_5d(xf + sizeof(T) * COLS * N, &maps.in_xface, &full[s], x0, 0, Ag, 0, Er);
        tma_load_5d(uf, &maps.in_uface, &full[s], x0, N - 1, Ag - 1, 0, Eg);
        tma_load_5d(uf + sizeof(T) * COLS * N, &maps.in_uface, &full[s], x0, 0, Ag + 1, 0, Eg);
        if (with_fn) tma_load_5d(st + G::IN_B, &maps.fn_tile, &full[s], x0 - P, 0, Ag, 0, Eg);
        bulk_load(uf + G::UF_B + G::BG_B, static_cast<const V2 *>(a.usv) + Ag * N, (uint32_t)(2 * sizeof(T)) * N,
                  &full[s]);
        if (with_bg) {
            unsigned char *bg = uf + G::UF_B;
            tma_load_2d(bg, &maps.bg_eu, &full[s], x0, Ag * N);
            tma_load_2d(bg + sizeof(float) * COLS * N, &maps.bg_rb, &full[s], x0, Ag * N);
        }
    };
    if (tid == 0) {
        if (ntile_cta > 0) issue(0, 0);
        if (ntile_cta > 1) issue(1, 1);
    }

    const double accel = a.accel, bfield = a.bfield;
    const double dtd = (kind == KIND_RHS) ? 0.0 : *a.dt;
    const T dtT = (T)dtd, c0 = (T)a.c0, c1 = (T)a.c1, c2dt = (T)(a.c2 * dtd);
    const T jx = (T)a.jx, ju = (T)a.ju, jv = (T)a.jv;
    const double Ei = a.E[Eg * N + g];
    // per-thread coefficients (runtime rows g and 2t, 2t + 1 of the tables)
    // MMA form: fragments up[g][t], up[g][4 + t] and their upwind-folded variants (speed >= 0
    // folds the own right trace into column n-1, speed < 0 the own left trace into column 0), so
    // only the neighbour trace remains as a lift: xi[g][0] (x, from the left) / -xi[g][1] (x, from
    // the right) for the x direction, xi[k][0] / -xi[k][1] of the thread's columns k for v
    T ca0, ca1, ca0M, ca1P, xil, xir, vil0, vil1, vir0, vir1;
    T upi[N], upk0[N], upk1[N];    // FMA form: up[g][.], up[2t][.], up[2t + 1][.]
    T xig0, xig1, xik00, xik01, xik10, xik11;
    if constexpr (G::MMA) {
        xil = tb.xi[2 * g];
        xir = -tb.xi[2 * g + 1];
        vil0 = tb.xi[4 * t];
        vil1 = tb.xi[4 * t + 2];
        vir0 = -tb.xi[4 * t + 1];
        vir1 = -tb.xi[4 * t + 3];
    }
    if constexpr (G::MMA) {
        ca0 = tb.up[g * N + t];
        ca1 = tb.up[g * N + 4 + t];
        ca0M = tb.upM[g * N + t];
        ca1P = tb.upP[g * N + 4 + t];
    } else {
#pragma unroll
        for (int m = 0; m < N; ++m) {
            upi[m] = tb.up[g * N + m];
            upk0[m] = tb.up[(2 * t) * N + m];
            upk1[m] = tb.up[(2 * t + 1) * N + m];
        }
        xig0 = tb.xi[2 * g];
        xig1 = tb.xi[2 * g + 1];
        xik00 = tb.xi[4 * t];
        xik01 = tb.xi[4 * t + 1];
        xik10 = tb.xi[4 * t + 2];
        xik11 = tb.xi[4 * t + 3];
    }
    T *out = static_cast<T *>(a.out);
    T *gout = static_cast<T *>(a.ghost_out);
    const bool ghost = gout != nullptr && (e == 0 || e == nx - 1);   // CTA-uniform
    double mk0 = 0.0, mk1 = 0.0;   // sum_j (w_j / J_u) out[.., j, k] for the two columns

    for (int q = 0; q < ntile_cta; ++q) {
        const int s = q & 1;
        const int tt = blockIdx.x + q * gridDim.x;
        const int au = tt / nbt;
        const int b0 = (tt - au * nbt) * EPT;
        const int nb = min(EPT, nv - b0);
        const int Ag = au + 1;
        const bool act = w < nb;
        const int col = (b0 + 1) * N + cl;   // global v-node column of the first output
        // v-node coordinates of the thread's columns, read before the wait so their latency overlaps it
        const double vn0 = act ? a.v_nodes[col] : 0.0, vn1 = act ? a.v_nodes[col + 1] : 0.0;
        if (!mbar_wait_bounded(&full[s], (uint32_t)((q >> 1) & 1))) {
            if (a.err != nullptr) atomicOr(a.err, 2);
            return;
        }
        const T *sIn = reinterpret_cast<const T *>(stage_ptr(s));
        const T *sFn = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B);
        const T *sXF = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B + G::FN_B);
        const T *sUF = reinterpret_cast<const T *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B);
        const float *sBG = reinterpret_cast<const float *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B + G::UF_B);
        const V2 *sUS =
            reinterpret_cast<const V2 *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B + G::UF_B + G::BG_B);

        if (act) {
            const double sd0 = accel * (Ei + bfield * vn0);
            const double sd1 = accel * (Ei + bfield * vn1);
            const T sp0 = (T)sd0, sp1 = (T)sd1;
            const T spu0 = sp0 * ju, spu1 = sp1 * ju;
            // F[g][m][cl..cl+1] for the u contraction, and the u upwind traces
            const T *pg = sIn + g * PS + P + cl;
            V2 fu[N];
#pragma unroll
            for (int m = 0; m < N; ++m) fu[m] = *reinterpret_cast<const V2 *>(pg + m * W);
            const V2 ufl = *reinterpret_cast<const V2 *>(sUF + g * COLS + cl);
            const V2 ufr = *reinterpret_cast<const V2 *>(sUF + N * COLS + g * COLS + cl);
            const T uL0 = (sd0 >= 0.0) ? ufl.x : fu[0].x, uR0 = (sd0 >= 0.0) ? fu[N - 1].x : ufr.x;
            const T uL1 = (sd1 >= 0.0) ? ufl.y : fu[0].y, uR1 = (sd1 >= 0.0) ? fu[N - 1].y : ufr.y;
            const size_t obase = (size_t)Eg * sE_ + (size_t)g * sI + (size_t)Ag * sA + col;
            T *pout = out + obase;
            const T *prow = sIn + g * PS + P + wc;   // row slice F[g][j][element] at j = 0
            // the warp's j rows (compile-time j: table constants)
            // upwind directions of x (sign of u J_x) and v (sign of a (-B u) J_v) at the element's end
            // rows: the same for every j of a u element that does not straddle u = 0, and then the
            // direction-dependent fragments and coefficients are chosen once per tile
            const V2 usF = sUS[0], usL = sUS[N - 1];
            const bool xpos0 = usF.x >= (T)0, vpos0 = usF.y >= (T)0;
            const bool uni = (xpos0 == (usL.x >= (T)0)) && (vpos0 == (usL.y >= (T)0));
            auto rows = [&](auto j0c, auto uni_c, auto ghost_c) {
                constexpr bool GHOST = decltype(ghost_c)::value;   // x-ghost refresh rows
                constexpr int J0 = decltype(j0c)::value;
                constexpr bool UNI = decltype(uni_c)::value;
#pragma unroll
                for (int jj = 0; jj < G::NJ; ++jj) {
                    const int j = J0 + jj;
                    // x and v flux speeds (their signs are the upwind directions) times the
                    // direction weights
                    const V2 us = sUS[j];
                    const bool xpos = UNI ? xpos0 : us.x >= (T)0;
                    const bool vpos = UNI ? vpos0 : us.y >= (T)0;
                    const T uxj = us.x * jx, svj = us.y * jv;
                    T dx0, dx1, dv0, dv1;
                    if constexpr (G::MMA) {
                        // x: A = upwind-folded up (rows g), B rows m = t, 4 + t at column wc + g, then
                        // the neighbour trace of the thread's columns
                        const T *pb = sIn + j * W + P + wc + g;
                        const T b0v = pb[t * PS];
                        const T b1v = pb[(4 + t) * PS];
                        double x0 = 0.0, x1 = 0.0;
                        dmma_8x8x4(x0, x1, xpos ? ca0 : ca0M, b0v);
                        dmma_8x8x4(x0, x1, xpos ? ca1P : ca1, b1v);
                        const V2 xn = *reinterpret_cast<const V2 *>(sXF + (xpos ? 0 : N * COLS) + j * COLS + cl);
                        const T xcn = xpos ? xil : xir;
                        dx0 = fma(xcn, xn.x, x0);
                        dx1 = fma(xcn, xn.y, x1);
                        // v: A = F[g][j][wc + 4c + t], B = upwind-folded up^T, then the neighbour
                        // element's trace at row (g, j)
                        const T *pa = prow + j * W;
                        const T a0v = pa[t];
                        const T a1v = pa[4 + t];
                        double v0 = 0.0, v1 = 0.0;
                        dmma_8x8x4(v0, v1, a0v, vpos ? ca0 : ca0M);
                        dmma_8x8x4(v0, v1, a1v, vpos ? ca1P : ca1);
                        const T vn = vpos ? pa[-1] : pa[N];
                        dv0 = fma(vpos ? vil0 : vir0, vn, v0);
                        dv1 = fma(vpos ? vil1 : vir1, vn, v1);
                    } else {
                        const T *pc = sIn + j * W + P + cl;   // F[m][j][cl..cl+1] at m = 0
                        dx0 = (T)0;
                        dx1 = (T)0;
                        V2 cm0, cm7;
    #pragma unroll
                        for (int m = 0; m < N; ++m) {
                            const V2 cv = *reinterpret_cast<const V2 *>(pc + m * PS);
                            if (m == 0) cm0 = cv;
                            if (m == N - 1) cm7 = cv;
                            dx0 = fma(upi[m], cv.x, dx0);
                            dx1 = fma(upi[m], cv.y, dx1);
                        }
                        const V2 xf0 = *reinterpret_cast<const V2 *>(sXF + j * COLS + cl);
                        const V2 xf1 = *reinterpret_cast<const V2 *>(sXF + N * COLS + j * COLS + cl);
                        const V2 xl = xpos ? xf0 : cm0;
                        const V2 xr = xpos ? cm7 : xf1;
                        dx0 = fma(xig0, xl.x, dx0);
                        dx0 = fma(-xig1, xr.x, dx0);
                        dx1 = fma(xig0, xl.y, dx1);
                        dx1 = fma(-xig1, xr.y, dx1);
                        const T *pa = prow + j * W;
                        T line[N];
                        load_line<N, (sizeof(T) == 8 ? 2 : 4), T>(pa, line);
                        dv0 = (T)0;
                        dv1 = (T)0;
    #pragma unroll
                        for (int m = 0; m < N; ++m) {
                            dv0 = fma(upk0[m], line[m], dv0);
                            dv1 = fma(upk1[m], line[m], dv1);
                        }
                        const T tl = vpos ? pa[-1] : line[0];
                        const T tr = vpos ? line[N - 1] : pa[N];
                        dv0 = fma(xik00, tl, dv0);
                        dv0 = fma(-xik01, tr, dv0);
                        dv1 = fma(xik10, tl, dv1);
                        dv1 = fma(-xik11, tr, dv1);
                    }
                    // u: sum_m up[j][m] F[g][m][k] + lifts (compile-time j: table constants)
                    T du0 = (T)0, du1 = (T)0;
    #pragma unroll
                    for (int m = 0; m < N; ++m) {
                        du0 = fma(tb.up[j * N + m], fu[m].x, du0);
                        du1 = fma(tb.up[j * N + m], fu[m].y, du1);
                    }
                    du0 = fma(tb.xi[2 * j], uL0, du0);
                    du0 = fma(-tb.xi[2 * j + 1], uR0, du0);
                    du1 = fma(tb.xi[2 * j], uL1, du1);
                    du1 = fma(-tb.xi[2 * j + 1], uR1, du1);
                    T r0 = fma(uxj, dx0, fma(spu0, du0, svj * dv0));
                    T r1 = fma(uxj, dx1, fma(spu1, du1, svj * dv1));
                    if (with_bg) {   // RHS of the x-independent background (staged with the tile)
                        const float2 eu = *reinterpret_cast<const float2 *>(sBG + j * COLS + cl);
                        const float2 rb = *reinterpret_cast<const float2 *>(sBG + N * COLS + j * COLS + cl);
                        r0 += (T)fmaf((float)Ei, eu.x, rb.x);
                        r1 += (T)fmaf((float)Ei, eu.y, rb.y);
                    }
                    const V2 fij = *reinterpret_cast<const V2 *>(prow + j * W + 2 * t);
                    V2 o;
                    if (kind == KIND_RHS) {
                        o.x = r0;
                        o.y = r1;
                    } else if (kind == KIND_EULER) {
                        o.x = fma(dtT, r0, fij.x);
                        o.y = fma(dtT, r1, fij.y);
                    } else if constexpr (WFN) {
                        const V2 fnv = *reinterpret_cast<const V2 *>(sFn + g * PSF + j * WF + P + cl);
                        o.x = rk_combine(c0, c1, c2dt, fnv.x, fij.x, r0);
                        o.y = rk_combine(c0, c1, c2dt, fnv.y, fij.y, r1);
                    } else {
                        o = fij;   // not reached: combination stages launch the WFN form
                    }
                    *reinterpret_cast<V2 *>(pout + j * sJ) = o;
                    if constexpr (GHOST) {
                        // periodic x-ghost refresh of f (Distribution.swap_ghost_cells_of_array)
                        const size_t gb = (size_t)g * sI + (size_t)Ag * sA + (size_t)j * sJ + col;
                        if (e == nx - 1) *reinterpret_cast<V2 *>(gout + gb) = fij;
                        if (e == 0) *reinterpret_cast<V2 *>(gout + (size_t)(nx + 1) * sE_ + gb) = fij;
                    }
                    mk0 = fma(tb.wu[j], (double)o.x, mk0);
                    mk1 = fma(tb.wu[j], (double)o.y, mk1);
                }
            };
            auto rows_j = [&](auto j0c) {
                // (the edge x elements of stage 1 refresh f's ghost slabs: their own instantiation)
                if (ghost) {
                    if (uni)
                        rows(j0c, std::true_type{}, std::true_type{});
                    else
                        rows(j0c, std::false_type{}, std::true_type{});
                } else {
                    if (uni)
                        rows(j0c, std::true_type{}, std::false_type{});
                    else
                        rows(j0c, std::false_type{}, std::false_type{});
                }
            };
            if constexpr (G::JS == 1) {
                rows_j(std::integral_constant<int, 0>{});
            } else {
                static_assert(G::JS == 2, "one or two warps per v element");
                if (h == 0)
                    rows_j(std::integral_constant<int, 0>{});
                else
                    rows_j(std::integral_constant<int, G::NJ>{});
            }
        }
        __syncthreads();   // stage s fully consumed
        if (tid == 0 && q + 2 < ntile_cta) issue(s, q + 2);
    }

    if (a.partials == nullptr) return;
    // moment partial of x node g: sum over the thread's columns, the quad, the warps
    dd v = two_sum(tb.wv[2 * t] * mk0, tb.wv[2 * t + 1] * mk1);
    v = dd_add(v, dd{__shfl_xor_sync(0xffffffffu, v.hi, 1), __shfl_xor_sync(0xffffffffu, v.lo, 1)});
    v = dd_add(v, dd{__shfl_xor_sync(0xffffffffu, v.hi, 2), __shfl_xor_sync(0xffffffffu, v.lo, 2)});
    if (t == 0) sRed[wid][g] = v;
    __syncthreads();
    if (tid < N) {
        dd s = sRed[0][tid];
#pragma unroll
        for (int ww = 1; ww < EPT * G::JS; ++ww) s = dd_add(s, sRed[ww][tid]);
        a.partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * N + tid] = s.hi + s.lo;
    }
    (void)NT;
}

}  // namespace vl
