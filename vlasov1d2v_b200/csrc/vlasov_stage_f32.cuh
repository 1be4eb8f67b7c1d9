// FP32 fused SSP-RK stage kernel for n = 8 (sm_100a): packed-FP32 contractions.
//
// Same tile, shared-memory stage and TMA pipeline as the fragment kernel (vlasov_stage_frag.cuh,
// FragGeom<float>): tile = (x element e, u element a, 4 consecutive v elements); warp w holds x
// nodes 2w and 2w + 1 of all four elements, lane = 16 h + 4 b + t owns x node g = 2w + h of element b
// and the column pair k = 2t, 2t + 1 for all eight j (a warp store covers two whole tile rows).
// Every product of a coefficient with the thread's two columns is one packed FMA
// (fma.rn.f32x2: two FP32 lanes per instruction), which halves the issue slots of the three
// contractions, the lifts, the flux products, the RK combination and the moment:
//   x:  {d, d'} = sum_m {up[g][m], up[g][m]} * F[m][j][k, k+1]   8 pair loads (broadcast across
//                                                                 the two x nodes of a warp)
//   v:  d_k = sum_q {up[k][2q], up[k][2q+1]} * F[g][j][2q, 2q+1]  the element's k-line as two
//                                                                 16-byte loads, pairs over m
//   u:  {d, d'} = sum_m {up[j][m], up[j][m]} * F[g][m][k, k+1]   j compile-time: the coefficient
//                                                                 pairs are constant-bank operands
// The upwind directions of x and v are the signs of u_j and of a (-B u_j): the same for every j of
// a u element that does not straddle u = 0, so the own-trace part of both lifts is folded into the
// first / last coefficient once per tile and one packed FMA adds the neighbour trace; tiles whose
// u element straddles zero take the same body with the selection made per j.  The u direction
// (sign of a (E_i + B v_k)) is fixed per thread and tile.  The moment partial of the output is
// accumulated per tile in FP32 pairs over the tile's eight j, then added in FP64.
// Stage kinds and the background split are template parameters: no per-row branches.  BG 0: no
// split; 1: the eu and rb RHS tables as two 2-D boxes; 2: the two tables interleaved per column
// pair ({eu(k), eu(k+1), rb(k), rb(k+1)}), one box and one 128-bit load per row.
#pragma once

#include <cuda.h>

#include <type_traits>

#include "vlasov_kernels.cuh"
#include "vlasov_stage_frag.cuh"
#include "vlasov_stage_tma.cuh"

namespace vl {

// coefficient tables of the kernel (kernel parameters: constant-bank operands)
struct F32Tables {
    float2 up2[64];   // {up[j][m], up[j][m]}              u contraction
    float2 xl2[8];    // {xi[j][0], xi[j][0]}              u lift, left trace
    float2 xr2[8];    // {-xi[j][1], -xi[j][1]}            u lift, right trace
    float2 wu2[8];    // {w_j / J_u, w_j / J_u}            moment weights of the rows
    float upP[64];    // up, speed >= 0: column n-1 minus xi[i][1]
    float upM[64];    // up, speed <  0: column 0 plus xi[i][0]
    float xi[16];
    double wv[8];     // w_k / J_v                         moment weights of the columns
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 lds2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ float4 lds4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ float2 lo2(float4 v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 hi2(float4 v) { return make_float2(v.z, v.w); }

template <int KIND, int BG>
__global__ void __launch_bounds__(FragGeom<float>::THREADS, FragGeom<float>::MINB)
stage_f32_kernel(const StageArgs a, const __grid_constant__ F32Tables tb, const __grid_constant__ FragMaps maps) {
    using G = FragGeom<float>;
    constexpr int N = G::N, P = G::P, W = G::W, PS = G::PS, WF = G::WF, PSF = G::PSF;
    constexpr int COLS = G::COLS, EPT = G::EPT;
    static_assert(G::THREADS == 128 && EPT == 4, "four warps of two x nodes each");
    if (a.state != nullptr && a.state->active == 0) return;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
    __shared__ __align__(8) uint64_t full[2];
    __shared__ dd sRed[N];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    // warp w covers x nodes 2w, 2w + 1 of all four v elements of the tile: lane = 16 h + 4 b + t
    // owns x node g = 2w + h, element b and its columns 2t, 2t + 1, so one warp store writes two
    // whole 128-byte rows of the output tile
    const int w = tid >> 5;
    const int g = 2 * w + (lane >> 4);   // x node i of the thread's outputs
    const int b = (lane >> 2) & 3;       // v element of the tile
    const int t = lane & 3;              // columns 2t, 2t + 1 of the element
    const int wc = b * N;                // first tile column of the element
    const int cl = wc + 2 * t;       // first tile column of the thread
    const int k0 = 2 * t, k1 = 2 * t + 1;

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
    constexpr bool WITH_FN = (KIND == KIND_COMBINE);
    constexpr uint32_t TX = G::TX_IN + 4 * G::TX_FACE + (WITH_FN ? G::TX_FN : 0) + (BG != 0 ? 2 * G::TX_BG : 0) +
                            (uint32_t)sizeof(float4) * N;
    static_assert(sizeof(float4) * N <= G::UX_B, "u-node speed slot");
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
        mbar_arrive_expect_tx(&full[s], TX);
        tma_load_5d(st, &maps.in_tile, &full[s], x0 - P, 0, Ag, 0, Eg);
        tma_load_5d(xf, &maps.in_xface, &full[s], x0, 0, Ag, N - 1, El);
        tma_load_5d(xf + sizeof(float) * COLS * N, &maps.in_xface, &full[s], x0, 0, Ag, 0, Er);
        tma_load_5d(uf, &maps.in_uface, &full[s], x0, N - 1, Ag - 1, 0, Eg);
        tma_load_5d(uf + sizeof(float) * COLS * N, &maps.in_uface, &full[s], x0, 0, Ag + 1, 0, Eg);
        if constexpr (WITH_FN) tma_load_5d(st + G::IN_B, &maps.fn_tile, &full[s], x0 - P, 0, Ag, 0, Eg);
        bulk_load(uf + G::UF_B + G::BG_B, static_cast<const float4 *>(a.usv) + Ag * N,
                  (uint32_t)sizeof(float4) * N, &full[s]);
        if constexpr (BG == 1) {
            unsigned char *bg = uf + G::UF_B;
            tma_load_2d(bg, &maps.bg_eu, &full[s], x0, Ag * N);
            tma_load_2d(bg + sizeof(float) * COLS * N, &maps.bg_rb, &full[s], x0, Ag * N);
        } else if constexpr (BG == 2) {
            tma_load_2d(uf + G::UF_B, &maps.bg_eu, &full[s], 2 * x0, Ag * N);   // (2 COLS, n) box
        }
    };
    if (tid == 0) {
        if (ntile_cta > 0) issue(0, 0);
        if (ntile_cta > 1) issue(1, 1);
    }

    const double accel = a.accel, bfield = a.bfield;
    const double dtd = (KIND == KIND_RHS) ? 0.0 : *a.dt;
    const float2 dt2 = f2s((float)dtd), c12 = f2s((float)a.c1), c2dt2 = f2s((float)(a.c2 * dtd));
    const float2 mone = f2s(-1.0f);
    const float ju = (float)a.ju;
    const float rsx = (float)a.sx, rsv = (float)a.sv;
    const double Ei = a.E[Eg * N + g];
    const float2 Ei2 = f2s((float)Ei);
    // per-thread coefficients: x rows g (pairs), v rows k0, k1 (pairs over m), both upwind variants
    // of the folded columns, and the neighbour-trace coefficients
    float2 cx[N];
#pragma unroll
    for (int m = 0; m < N; ++m) cx[m] = f2s(tb.upP[g * N + m]);   // columns 1 .. n-2 are plain up
    const float cx0P = tb.upP[g * N], cx0M = tb.upM[g * N];
    const float cx7P = tb.upP[g * N + 7], cx7M = tb.upM[g * N + 7];
    const float xnP = tb.xi[2 * g], xnM = -tb.xi[2 * g + 1];
    float2 v0[4], v1[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        v0[q] = f2(tb.upP[k0 * N + 2 * q], tb.upP[k0 * N + 2 * q + 1]);
        v1[q] = f2(tb.upP[k1 * N + 2 * q], tb.upP[k1 * N + 2 * q + 1]);
    }
    const float v00P = tb.upP[k0 * N], v00M = tb.upM[k0 * N], v07P = tb.upP[k0 * N + 7], v07M = tb.upM[k0 * N + 7];
    const float v10P = tb.upP[k1 * N], v10M = tb.upM[k1 * N], v17P = tb.upP[k1 * N + 7], v17M = tb.upM[k1 * N + 7];
    const float vn0P = tb.xi[2 * k0], vn0M = -tb.xi[2 * k0 + 1];
    const float vn1P = tb.xi[2 * k1], vn1M = -tb.xi[2 * k1 + 1];

    float *out = static_cast<float *>(a.out);
    float *gout = static_cast<float *>(a.ghost_out);
    const bool ghost = gout != nullptr && (e == 0 || e == nx - 1);
    double mk0 = 0.0, mk1 = 0.0;   // sum over rows of (w_j / J_u) out[.., j, k] for the two columns
    // v-node coordinates of the thread's columns, loaded one tile ahead of their use
    auto vnodes = [&](int q, double &x0, double &x1) {
        x0 = x1 = 0.0;
        if (q >= ntile_cta) return;
        const int tq = blockIdx.x + q * gridDim.x;
        const int bq = (tq - (tq / nbt) * nbt) * EPT;
        if (b < min(EPT, nv - bq)) {
            x0 = a.v_nodes[(bq + 1) * N + cl];
            x1 = a.v_nodes[(bq + 1) * N + cl + 1];
        }
    };
    double vn0, vn1;
    vnodes(0, vn0, vn1);

    for (int q = 0; q < ntile_cta; ++q) {
        const int s = q & 1;
        const int tt = blockIdx.x + q * gridDim.x;
        const int au = tt / nbt;
        const int b0 = (tt - au * nbt) * EPT;
        const int nb = min(EPT, nv - b0);
        const int Ag = au + 1;
        const bool act = b < nb;
        const int col = (b0 + 1) * N + cl;   // global v-node column of the first output
        const double vc0 = vn0, vc1 = vn1;
        vnodes(q + 1, vn0, vn1);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((q >> 1) & 1))) {
            if (a.err != nullptr) atomicOr(a.err, 2);
            return;
        }
        const float *sIn = reinterpret_cast<const float *>(stage_ptr(s));
        const float *sFn = reinterpret_cast<const float *>(stage_ptr(s) + G::IN_B);
        const float *sXF = reinterpret_cast<const float *>(stage_ptr(s) + G::IN_B + G::FN_B);
        const float *sUF = reinterpret_cast<const float *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B);
        const float *sBG = reinterpret_cast<const float *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B + G::UF_B);
        const float4 *sUS =
            reinterpret_cast<const float4 *>(stage_ptr(s) + G::IN_B + G::FN_B + G::XF_B + G::UF_B + G::BG_B);

        if (act) {
            // u flux speed of the thread's columns (its sign is the u upwind direction) times J_u
            const double sd0 = accel * (Ei + bfield * vc0);
            const double sd1 = accel * (Ei + bfield * vc1);
            const float2 spu = f2((float)sd0 * ju, (float)sd1 * ju);
            const float *pg = sIn + g * PS + P + cl;
            float2 fu[N];   // F[g][m][k, k+1]: the u contraction's operand, and the stage input
#pragma unroll
            for (int m = 0; m < N; ++m) fu[m] = lds2(pg + m * W);
            const float2 ufl = lds2(sUF + g * COLS + cl);
            const float2 ufr = lds2(sUF + N * COLS + g * COLS + cl);
            const float2 uL = f2(sd0 >= 0.0 ? ufl.x : fu[0].x, sd1 >= 0.0 ? ufl.y : fu[0].y);
            const float2 uR = f2(sd0 >= 0.0 ? fu[N - 1].x : ufr.x, sd1 >= 0.0 ? fu[N - 1].y : ufr.y);
            float *pout = out + (size_t)Eg * sE_ + (size_t)g * sI + (size_t)Ag * sA + col;
            const float *prow = sIn + g * PS + P + wc;   // k-line of element w at row (g, j = 0)
            // upwind directions of x (sign of u_j) and v (sign of a (-B u_j)) at the element's end rows
            const float4 us0 = sUS[0], us7 = sUS[N - 1];
            const bool uni = ((us0.x >= 0.0f) == (us7.x >= 0.0f)) && ((us0.z >= 0.0f) == (us7.z >= 0.0f));
            float2 mk = f2s(0.0f);
            auto rows = [&](auto uni_c, auto ghost_c) {
                constexpr bool UNI = decltype(uni_c)::value;
                constexpr bool GHOST = decltype(ghost_c)::value;   // x-ghost refresh rows
                // folded coefficients for the tile (uniform directions)
                float2 cxn = f2s(0.0f);
                const float *sXn = sXF;
                int voff = -1;
                float2 cvn = f2s(0.0f);
                auto set_dirs = [&](bool xp, bool vp) {
                    cx[0] = f2s(xp ? cx0P : cx0M);
                    cx[N - 1] = f2s(xp ? cx7P : cx7M);
                    cxn = f2s(xp ? xnP : xnM);
                    sXn = sXF + (xp ? 0 : N * COLS);
                    v0[0].x = vp ? v00P : v00M;
                    v0[3].y = vp ? v07P : v07M;
                    v1[0].x = vp ? v10P : v10M;
                    v1[3].y = vp ? v17P : v17M;
                    cvn = f2(vp ? vn0P : vn0M, vp ? vn1P : vn1M);
                    voff = vp ? -1 : N;
                };
                if constexpr (UNI) set_dirs(us0.x >= 0.0f, us0.z >= 0.0f);
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    float4 us = sUS[j];   // {u J_x, u J_x, a (-B u) J_v, a (-B u) J_v}
                    if constexpr (!UNI) set_dirs(us.x >= 0.0f, us.z >= 0.0f);
                    if constexpr (KIND == KIND_RHS) {   // caller-chosen direction weights
                        us.x *= rsx;
                        us.y *= rsx;
                        us.z *= rsv;
                        us.w *= rsv;
                    }
                    // x: sum_m up[g][m] F[m][j][k, k+1] with the own trace folded, + neighbour trace
                    const float *pc = sIn + j * W + P + cl;
                    float2 dx = fmul2(cx[0], lds2(pc));
#pragma unroll
                    for (int m = 1; m < N; ++m) dx = ffma2(cx[m], lds2(pc + m * PS), dx);
                    dx = ffma2(cxn, lds2(sXn + j * COLS + cl), dx);
                    // v: the k-line of row (g, j), pairs over m, + neighbour element's trace
                    const float *pa = prow + j * W;
                    const float4 l0 = lds4(pa), l1 = lds4(pa + 4);
                    float2 a0 = fmul2(v0[0], f2(l0.x, l0.y));
                    float2 a1 = fmul2(v1[0], f2(l0.x, l0.y));
                    a0 = ffma2(v0[1], f2(l0.z, l0.w), a0);
                    a1 = ffma2(v1[1], f2(l0.z, l0.w), a1);
                    a0 = ffma2(v0[2], f2(l1.x, l1.y), a0);
                    a1 = ffma2(v1[2], f2(l1.x, l1.y), a1);
                    a0 = ffma2(v0[3], f2(l1.z, l1.w), a0);
                    a1 = ffma2(v1[3], f2(l1.z, l1.w), a1);
                    const float vn = pa[voff];
                    const float2 dv = f2(fmaf(cvn.x, vn, a0.x + a0.y), fmaf(cvn.y, vn, a1.x + a1.y));
                    // u: sum_m up[j][m] F[g][m][k, k+1] + lifts (compile-time j: constant operands)
                    float2 du = fmul2(tb.up2[j * N], fu[0]);
#pragma unroll
                    for (int m = 1; m < N; ++m) du = ffma2(tb.up2[j * N + m], fu[m], du);
                    du = ffma2(tb.xl2[j], uL, du);
                    du = ffma2(tb.xr2[j], uR, du);
                    // R = u J_x dx + s J_u du + a (-B u) J_v dv (+ background RHS)
                    float2 r = fmul2(f2(us.z, us.w), dv);
                    r = ffma2(spu, du, r);
                    r = ffma2(f2(us.x, us.y), dx, r);
                    if constexpr (BG == 1) {
                        const float2 eu = lds2(sBG + j * COLS + cl);
                        const float2 rb = lds2(sBG + N * COLS + j * COLS + cl);
                        r = fadd2(r, ffma2(Ei2, eu, rb));
                    } else if constexpr (BG == 2) {
                        const float4 er = lds4(sBG + j * 2 * COLS + 2 * cl);   // {eu, eu', rb, rb'}
                        r = fadd2(r, ffma2(Ei2, lo2(er), hi2(er)));
                    }
                    const float2 fij = fu[j];
                    float2 o;
                    if constexpr (KIND == KIND_RHS) {
                        o = r;
                    } else if constexpr (KIND == KIND_EULER) {
                        o = ffma2(dt2, r, fij);
                    } else {
                        // f^n + c1 (s - f^n) + c2 dt R (weights of f^n and s sum to exactly 1)
                        const float2 fnv = lds2(sFn + g * PSF + j * WF + P + cl);
                        o = ffma2(c2dt2, r, ffma2(c12, ffma2(mone, fnv, fij), fnv));
                    }
                    *reinterpret_cast<float2 *>(pout + (size_t)j * sJ) = o;
                    if constexpr (GHOST) {
                        // periodic x-ghost refresh of f (Distribution.swap_ghost_cells_of_array)
                        const size_t gb = (size_t)g * sI + (size_t)Ag * sA + (size_t)j * sJ + col;
                        if (e == nx - 1) *reinterpret_cast<float2 *>(gout + gb) = fij;
                        if (e == 0) *reinterpret_cast<float2 *>(gout + (size_t)(nx + 1) * sE_ + gb) = fij;
                    }
                    mk = ffma2(tb.wu2[j], o, mk);
                }
            };
            // (the edge x elements of stage 1 refresh f's ghost slabs: their own instantiation, so
            // the other CTAs' row loop has no branch on it)
            if (ghost) {
                if (uni)
                    rows(std::true_type{}, std::true_type{});
                else
                    rows(std::false_type{}, std::true_type{});
            } else {
                if (uni)
                    rows(std::true_type{}, std::false_type{});
                else
                    rows(std::false_type{}, std::false_type{});
            }
            mk0 += (double)mk.x;
            mk1 += (double)mk.y;
        }
        __syncthreads();   // stage s fully consumed
        if (tid == 0 && q + 2 < ntile_cta) issue(s, q + 2);
    }

    if (a.partials == nullptr) return;
    // moment partial of x node g: sum over the thread's columns, then over the 16 lanes of the
    // half-warp that holds node g (its four elements and column pairs)
    dd v = two_sum(tb.wv[k0] * mk0, tb.wv[k1] * mk1);
#pragma unroll
    for (int off = 1; off < 16; off <<= 1)
        v = dd_add(v, dd{__shfl_xor_sync(0xffffffffu, v.hi, off), __shfl_xor_sync(0xffffffffu, v.lo, off)});
    if ((lane & 15) == 0) sRed[g] = v;
    __syncthreads();
    if (tid < N) a.partials[((size_t)blockIdx.y * gridDim.x + blockIdx.x) * N + tid] = sRed[tid].hi + sRed[tid].lo;
}

}  // namespace vl
