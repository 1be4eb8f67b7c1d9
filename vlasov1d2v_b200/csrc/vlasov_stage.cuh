// Fused SSP-RK stage kernel: "node pencil" formulation.
//
// Layout: the ghost-inclusive state f[X][n][U][n][V][n] is a 3-D node grid whose innermost
// axis (v node, index (b, k)) is contiguous.  A warp covers EPW = 32 / n consecutive v
// elements of one (x element e, u element a) pair; lane l -> (element bl = l / n, node k = l % n).
// Each thread owns the pencil f[e, :, a, j, b, k] for i in 0..n-1 and its JC-wide chunk of j
// (JS = ceil(n / JC) warps per CTA, warp h owning j in [h JC, h JC + JC)).  Consequences:
//   * every global load/store is one contiguous run per warp (lanes -> consecutive v nodes);
//   * the x contraction (along i) runs entirely in registers;
//   * the u contraction (along j) reads the n - JC partner values of a row from shared memory;
//   * the v contraction (along k, across lanes) reads k-lines from a shared-memory copy of the
//     tile (broadcast loads: the n lanes of an element read the same line).
// Upwind face values: x and u neighbour traces are loaded straight into registers (one per x
// line / u line, coalesced); v neighbour traces of the tile ends come from a small shared
// array.  The RK combination, the x-ghost refresh and the moment partials are fused in.
#pragma once

#include "vlasov_kernels.cuh"

#ifndef VL_STAGE_REG_CAP
#define VL_STAGE_REG_CAP 128
#endif

namespace vl {

template <int N, typename T>
struct PencilGeom {
    static constexpr int EPW = 32 / N;                       // v elements per warp (tile)
    // j values per thread: 2 in FP64; in FP32 all rows in one warp up to order 7 and 5 + 4 rows
    // in two warps at order 9, with the registers uncapped (per combination stage against 4 rows
    // per thread at 128 registers: order 7 at 32^3 elements 0.082 against 0.090 ms, order 9 at 64^3
    // 1.62 against 1.635 and its Euler stage 1.47 against 1.60; order 6 unchanged)
    static constexpr int JC_TARGET = sizeof(T) == 8 ? 2 : (N <= 7 ? N : (N == 9 ? 5 : 4));
    static constexpr int JS = (N + JC_TARGET - 1) / JC_TARGET;
    static constexpr int JC = (N + JS - 1) / JS;
    static constexpr int THREADS = 32 * JS;
    // resident CTAs per SM requested from the compiler (register cap per thread)
    static constexpr int REG_CAP = (sizeof(T) == 4 && JC >= 5) ? 255 : VL_STAGE_REG_CAP;
    static constexpr int MIN_BLOCKS = 65536 / (THREADS * REG_CAP) > 0 ? 65536 / (THREADS * REG_CAP) : 1;
    static constexpr int RW = EPW * N;                       // shared row length (v nodes)
    static constexpr int VEC = (sizeof(T) == 8) ? ((N % 2 == 0) ? 2 : 1) : ((N % 4 == 0) ? 4 : 1);
    // [N][NT] moment partials, [N][N][RW] tile, [N][N] v traces, then [N] E values (8-aligned)
    static constexpr size_t se_offset(int nt) {
        return (sizeof(double) * (size_t)(N * nt) + sizeof(T) * (size_t)(N * N * RW + N * N) + 7) & ~(size_t)7;
    }
    static constexpr size_t smem_bytes() { return se_offset(THREADS) + sizeof(double) * N; }
};

template <typename T, int VEC>
struct VecT;
template <>
struct VecT<double, 2> { using type = double2; };
template <>
struct VecT<float, 4> { using type = float4; };

// k-line read from shared memory (n values), vectorised when aligned
template <int N, int VEC, typename T>
__device__ __forceinline__ void load_line(const T *p, T (&line)[N]) {
    if constexpr (VEC > 1) {
        using V = typename VecT<T, VEC>::type;
        const V *q = reinterpret_cast<const V *>(p);
#pragma unroll
        for (int m = 0; m < N / VEC; ++m) {
            V v = q[m];
            if constexpr (VEC == 2) {
                line[2 * m] = v.x;
                line[2 * m + 1] = v.y;
            } else {
                line[4 * m] = v.x;
                line[4 * m + 1] = v.y;
                line[4 * m + 2] = v.z;
                line[4 * m + 3] = v.w;
            }
        }
    } else {
#pragma unroll
        for (int m = 0; m < N; ++m) line[m] = p[m];
    }
}

// One CTA's share of a stage: x element e, tiles g, g + G, ... of that slab; writes the moment
// partial [e][g][i] (of G per element).  JC_ j values per thread, NT_ threads per CTA: warps
// beyond ceil(N / JC_) have no j chunk and only take part in the barriers and loads of shared
// data (the ensemble kernel runs several orders with one block size).  tb supplies up / xi
// (compile-time indices: parameter or constant bank); qw the velocity weights (w_j w_k/(J_u J_v)).
template <int N, typename T, int JC_, int NT_, typename TB, int J0C = -1>
__device__ __forceinline__ void pencil_stage_body(const StageArgs &a, const TB &tb, const double *qw,
                                                  int e, int g, int G) {
    using GP = PencilGeom<N, T>;
    constexpr int EPW = GP::EPW, JC = JC_, RW = GP::RW, VEC = GP::VEC, NT = NT_;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *sMom = reinterpret_cast<double *>(smem_raw);            // [N][THREADS]
    T *sF = reinterpret_cast<T *>(sMom + N * NT);                   // [N][N][RW]
    T *sVH = sF + N * N * RW;                                       // [N][N]
    double *sE = reinterpret_cast<double *>(smem_raw + GP::se_offset(NT));   // E at the x nodes

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    // warp-uniform j chunk; compile-time when the caller instantiates one body per warp, so the
    // u-contraction coefficients up[j][m] become constant-bank operands
    const int J0 = (J0C >= 0) ? J0C : (tid >> 5) * JC;
    const int JN = min(JC, N - J0);                 // <= 0: a warp without a j chunk
    const int bl = lane / N, k = lane - (lane / N) * N;
    const bool lane_ok = lane < EPW * N;
    if (tid < N) sE[tid] = a.E[(e + 1) * N + tid];
#pragma unroll
    for (int i = 0; i < N; ++i) sMom[i * NT + tid] = 0.0;

    const T *__restrict__ in = static_cast<const T *>(a.in);
    const T *fn = static_cast<const T *>(a.fn);
    T *out = static_cast<T *>(a.out);
    T *gout = static_cast<T *>(a.ghost_out);

    const int nx = a.nx, nu = a.nu, nv = a.nv;
    const int U = nu + 2, V = nv + 2;
    const int sJ = V * N;               // stride of j (elements)
    const int sA = sJ * N;              // stride of a
    const int sI = sA * U;              // stride of i
    const size_t sE_ = (size_t)sI * N;  // stride of e

    const int Eg = e + 1;
    int El, Er;
    if (a.xhalo == VL_XHALO_PERIODIC) {
        El = (e == 0) ? nx : e;
        Er = (e == nx - 1) ? 1 : e + 2;
    } else {
        El = e;
        Er = e + 2;
    }
    const double accel = a.accel, bfield = a.bfield, nbfield = -a.bfield;
    const double dtd = (a.kind == KIND_RHS) ? 0.0 : *a.dt;
    const T dtT = (T)dtd, c0 = (T)a.c0, c1 = (T)a.c1, c2dt = (T)(a.c2 * dtd);
    const T jx = (T)a.jx, ju = (T)a.ju, jv = (T)a.jv;
    const int kind = a.kind;

    // per-lane coefficients of the v contraction (row k of up, lift column entries)
    const int kk = lane_ok ? k : 0;
    T upk[N];
#pragma unroll
    for (int m = 0; m < N; ++m) upk[m] = tb.up[kk * N + m];
    const T xik0 = tb.xi[2 * kk], xik1 = tb.xi[2 * kk + 1];
    double wk[JC];
#pragma unroll
    for (int jc = 0; jc < JC; ++jc) wk[jc] = (jc < JN && lane_ok) ? qw[(J0 + jc) * N + kk] : 0.0;
    __syncthreads();

    const int nbt = (nv + EPW - 1) / EPW;
    const int tiles = nu * nbt;
    for (int t = g; t < tiles; t += G) {
        const int au = t / nbt;
        const int b0 = (t - au * nbt) * EPW;
        const int nb = min(EPW, nv - b0);
        const bool act = lane_ok && (bl < nb);
        const int Ag = au + 1;
        const int col = (b0 + bl + 1) * N + k;      // this lane's column in a v row
        const size_t slab = (size_t)Eg * sE_;
        const size_t tile_off = slab + (size_t)Ag * sA + col;
        const T *pin = in + tile_off;              // f[e, 0, a, 0, b, k] of this lane

        double ux[JC];
#pragma unroll
        for (int jc = 0; jc < JC; ++jc) ux[jc] = a.u_nodes[Ag * N + (jc < JN ? J0 + jc : 0)];
        const double vnode = act ? a.v_nodes[col] : 0.0;
        // x and v flux speeds of the lane's j rows times their Jacobians, and their upwind
        // directions: the same for every x node, so formed once per tile
        T uxj[JC], svj[JC];
        bool xposj[JC], vposj[JC];
#pragma unroll
        for (int jc = 0; jc < JC; ++jc) {
            const double sv_d = accel * (nbfield * ux[jc]);
            xposj[jc] = ux[jc] >= 0.0;
            vposj[jc] = sv_d >= 0.0;
            uxj[jc] = (T)ux[jc] * jx;
            svj[jc] = (T)sv_d * jv;
        }
        // background-split RHS tables at the lane's (j, column): the same for every x node, so
        // read once per tile
        float beu[JC], brb[JC];
#pragma unroll
        for (int jc = 0; jc < JC; ++jc) {
            beu[jc] = 0.0f;
            brb[jc] = 0.0f;
            if (a.bg_rb != nullptr && act && jc < JN) {
                const int vi = Ag * sA + (J0 + jc) * sJ + col;
                beu[jc] = a.bg_eu[vi];
                brb[jc] = a.bg_rb[vi];
            }
        }

        // ---- own pencil columns (x lines) and the x upwind traces ----
        T f[N][JC];
        T xh[JC];
        if (act) {
#pragma unroll
            for (int jc = 0; jc < JC; ++jc) {
                if (jc < JN) {
                    const T *pj = pin + (J0 + jc) * sJ;
#pragma unroll
                    for (int m = 0; m < N; ++m) f[m][jc] = pj[m * sI];
                    xh[jc] = (ux[jc] >= 0.0)
                        ? in[(size_t)El * sE_ + (size_t)Ag * sA + col + (N - 1) * sI + (J0 + jc) * sJ]
                        : in[(size_t)Er * sE_ + (size_t)Ag * sA + col + (J0 + jc) * sJ];
                }
            }
        }
        // ---- v upwind traces of the tile ends (one per (i, j) row) ----
        constexpr int VH = (N * N + NT - 1) / NT;
        T vh[VH];
#pragma unroll
        for (int q = 0; q < VH; ++q) {
            const int r = tid + q * NT;
            if (r < N * N) {
                const int i = r / N, j = r - (r / N) * N;
                const double s = accel * (nbfield * a.u_nodes[Ag * N + j]);
                const T *rb = in + slab + (size_t)Ag * sA + i * sI + j * sJ;
                vh[q] = (s >= 0.0) ? rb[b0 * N + (N - 1)] : rb[(b0 + nb + 1) * N];
            }
        }
        __syncthreads();   // every thread is done with the previous tile's shared data
#pragma unroll
        for (int q = 0; q < VH; ++q) {
            const int r = tid + q * NT;
            if (r < N * N) sVH[r] = vh[q];
        }
        if (act) {
#pragma unroll
            for (int jc = 0; jc < JC; ++jc)
                if (jc < JN) {
#pragma unroll
                    for (int m = 0; m < N; ++m) sF[(m * N + J0 + jc) * RW + bl * N + k] = f[m][jc];
                }
        }
        __syncthreads();
        if (!act) continue;

        const int lcol = bl * N + k;
        T *pout = out + tile_off;
        const T *pfn = fn + tile_off;
        // one-row-ahead prefetch of the u upwind trace and of f^n
        auto u_trace = [&](int i) -> T {
            const double s = accel * (sE[i] + bfield * vnode);
            return (s >= 0.0) ? pin[i * sI - sA + (N - 1) * sJ] : pin[i * sI + sA];
        };
        T uh_cur = u_trace(0);
        T fn_cur[JC];
        if (kind == KIND_COMBINE) {
#pragma unroll
            for (int jc = 0; jc < JC; ++jc) fn_cur[jc] = (jc < JN) ? pfn[(J0 + jc) * sJ] : (T)0;
        }
#pragma unroll 1
        for (int i = 0; i < N; ++i) {
            const int inext = (i + 1 < N) ? i + 1 : i;
            const T uh_next = u_trace(inext);
            T fn_next[JC];
            if (kind == KIND_COMBINE) {
#pragma unroll
                for (int jc = 0; jc < JC; ++jc)
                    fn_next[jc] = (jc < JN) ? pfn[inext * sI + (J0 + jc) * sJ] : (T)0;
            }
            // the full j-row i at this lane (shared)
            T row[N];
            const T *rp = sF + i * N * RW + lcol;
#pragma unroll
            for (int j = 0; j < N; ++j) row[j] = rp[j * RW];
            const double s_d = accel * (sE[i] + bfield * vnode);
            const T s = (T)s_d;
            const bool upos = s_d >= 0.0;
            const T uL = upos ? uh_cur : row[0];
            const T uR = upos ? row[N - 1] : uh_cur;
            // x contraction coefficients of row i (warp-uniform index into the parameter bank)
            T upi[N];
#pragma unroll
            for (int m = 0; m < N; ++m) upi[m] = tb.up[i * N + m];
            const T xii0 = tb.xi[2 * i], xii1 = tb.xi[2 * i + 1];
            double mrow = 0.0;
#pragma unroll
            for (int jc = 0; jc < JC; ++jc) {
                if (jc >= JN) break;
                const int j = J0 + jc;
                // u part: along j at row i
                T du = (T)0;
#pragma unroll
                for (int m = 0; m < N; ++m) du = fma(tb.up[j * N + m], row[m], du);
                du = fma(tb.xi[2 * j], uL, du);
                du = fma(-tb.xi[2 * j + 1], uR, du);
                // x part: along i at column j (registers)
                const bool xpos = xposj[jc];
                const T xL = xpos ? xh[jc] : f[0][jc];
                const T xR = xpos ? f[N - 1][jc] : xh[jc];
                T dx = (T)0;
#pragma unroll
                for (int m = 0; m < N; ++m) dx = fma(upi[m], f[m][jc], dx);
                dx = fma(xii0, xL, dx);
                dx = fma(-xii1, xR, dx);
                // v part: along k (the element's k-line in shared memory)
                const T *lp = sF + (i * N + j) * RW + bl * N;
                T line[N];
                load_line<N, VEC, T>(lp, line);
                const bool vpos = vposj[jc];
                T vL, vR;
                if (vpos) {
                    vL = (bl > 0) ? lp[-1] : sVH[i * N + j];
                    vR = line[N - 1];
                } else {
                    vL = line[0];
                    vR = (bl < nb - 1) ? lp[N] : sVH[i * N + j];
                }
                T dv = (T)0;
#pragma unroll
                for (int m = 0; m < N; ++m) dv = fma(upk[m], line[m], dv);
                dv = fma(xik0, vL, dv);
                dv = fma(-xik1, vR, dv);
                T r = fma(uxj[jc], dx, fma(s * du, ju, svj[jc] * dv));
                if (a.bg_rb != nullptr)   // RHS of the x-independent background
                    r += (T)fmaf((float)sE[i], beu[jc], brb[jc]);
                const T fij = rp[j * RW];
                T o;
                if (kind == KIND_RHS) {
                    o = r;
                } else if (kind == KIND_EULER) {
                    o = fma(dtT, r, fij);
                } else {
                    o = rk_combine(c0, c1, c2dt, fn_cur[jc], fij, r);
                }
                pout[i * sI + j * sJ] = o;
                mrow = fma(wk[jc], (double)o, mrow);
            }
            sMom[i * NT + tid] += mrow;
            uh_cur = uh_next;
            if (kind == KIND_COMBINE) {
#pragma unroll
                for (int jc = 0; jc < JC; ++jc) fn_cur[jc] = fn_next[jc];
            }
        }
        if (gout != nullptr && (e == nx - 1 || e == 0)) {
            // periodic x-ghost refresh of f (Distribution.swap_ghost_cells_of_array)
#pragma unroll
            for (int jc = 0; jc < JC; ++jc) {
                if (jc >= JN) break;
                const int j = J0 + jc;
#pragma unroll
                for (int m = 0; m < N; ++m) {
                    const int off = (int)((size_t)Ag * sA) + col + m * sI + j * sJ;
                    if (e == nx - 1) gout[off] = f[m][jc];
                    if (e == 0) gout[(size_t)(nx + 1) * sE_ + off] = f[m][jc];
                }
            }
        }
    }
    if (a.partials == nullptr) return;
    __syncthreads();
    // CTA reduction of the moment partials (double-double), one warp per x node i
    const int nw = NT / 32;
    const int w = tid >> 5;
    for (int i = w; i < N; i += nw) {
        dd v = {0.0, 0.0};
        for (int q = lane; q < NT; q += 32) v = dd_add(v, dd{sMom[i * NT + q], 0.0});
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = dd_add(v, shfl_down_dd(v, off));
        if (lane == 0) a.partials[((size_t)e * G + g) * N + i] = v.hi + v.lo;
    }
}

// one body instantiation per warp w of an NT-thread CTA (its j chunk a template constant; warps
// past the last chunk take part in the barriers only); every instantiation runs the same sequence
// of barriers
template <int N, typename T, int JC, int NT, typename TB, int W = 0>
__device__ __forceinline__ void pencil_body_per_warp(const StageArgs &a, const TB &tb, const double *qw, int e,
                                                     int g, int G, int w) {
    if constexpr (W < NT / 32) {
        if (w == W) {
            pencil_stage_body<N, T, JC, NT, TB, (W * JC < N ? W * JC : N)>(a, tb, qw, e, g, G);
            return;
        }
        pencil_body_per_warp<N, T, JC, NT, TB, W + 1>(a, tb, qw, e, g, G, w);
    }
}

template <int N, typename T>
__global__ void __launch_bounds__(PencilGeom<N, T>::THREADS, PencilGeom<N, T>::MIN_BLOCKS)
stage_pencil_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb) {
    if (a.state != nullptr && a.state->active == 0) return;
    pencil_body_per_warp<N, T, PencilGeom<N, T>::JC, PencilGeom<N, T>::THREADS, StageTables<T>>(
        a, tb, tb.qw, blockIdx.y, blockIdx.x, gridDim.x, (int)(threadIdx.x >> 5));
}

}  // namespace vl
