// Fused SSP-RK stage kernel for every LGL order (sm_100a): asynchronous-copy pipelined tiles in
// the (x node, column pair) layout.
//
// Tile = (x element e, u element a, EPT consecutive v elements).  Thread "item" (b, i, p) owns
// x node i and the column pair k = 2p, 2p + 1 of tile element b, for all n values of j (for odd n
// the second column of the last pair is a pad column that is computed but never stored).  Per j:
//   x:  sum_m up[i][m] F[m][j][k]     n pair loads from the tile (shared across the items of
//                                     one column pair: broadcast within a warp)
//   v:  sum_m F[i][j][m] up[k][m]     the element's k-line (pair loads, shared by its pairs)
//   u:  sum_m up[j][m] F[i][m][k]     from the thread's register copy of F[i][0..n-1][k, k+1];
//                                     compile-time j, so up[j][m] is a constant-bank operand
// plus the upwind lifts in the three directions, the flux speeds, the Jacobian-weighted sum, the
// RK combination, the store, the periodic x-ghost refresh (stage 1 on f) and the zeroth-moment
// partials of the result: the same fused operator as the n = 8 fragment kernel.
//
// Shared-memory stage (filled by cp.async, NST stages in flight; every thread copies a share of
// each array, one warp per row, and the stage is published by cp.async.wait_group +
// __syncthreads, so no wait can spin):
//   IN [i][j][W]      stage input: tile columns at H + b SL + k (SL = n rounded up to even, one
//                     pad column per element for odd n so that every pair is vector-aligned),
//                     the left v trace of the tile at LH, the right one at H + nb SL
//   FN [i][j][WN]     f^n (combination stages)
//   XF [side][j][WF]  x upwind traces: (e-1, i = n-1) and (e+1, i = 0)
//   UF [side][i][WF]  u upwind traces: (a-1, j = n-1) and (a+1, j = 0)
//   BG [table][j][WF] FP32 background split: the eu and rb RHS tables of the tile
//   UX [j]            u node coordinates of the tile's u element
// W and WN are padded so that the k-line loads of the up-to-eight x nodes met by one warp fall
// in distinct banks (searched at compile time for the actual lane assignment).
//
// TMA form (16-byte-aligned state rows, stage_gen_tma_kernel; FP64 and FP32, the FP32
// background-split tables as two 2-D boxes): one thread per CTA loads each array of the tile with
// one cp.async.bulk.tensor box (no multicast) into the same stages, completing on an mbarrier
// (bounded waits).  Rows are then contiguous copies of the state: the tile starts at the 16-byte
// boundary at or below the left v trace, element b's node k sits at column off + 1 + b n + k
// (off < 16 bytes per tile), and the column pairs are read as two scalar loads.  Every box lands
// on a 128-byte-aligned shared-memory address.
//
// Paired-row TMA form (stage_gen_pair_kernel; FP32 rows of R = 2 mod 4 floats, e.g. the large
// configuration's 66 x 9): two rows are a 16-byte multiple, so each array is loaded as a box of its
// even rows and a box of its odd rows (GenPairGeom); the tile body is instantiated for both
// parities of the tile's first row, so every row offset stays a compile-time constant.
//
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "vlasov_kernels.cuh"
#include "vlasov_stage_tma.cuh"

namespace vl {

__device__ __forceinline__ uint32_t gen_smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(gen_smem_addr(dst)), "l"(src), "n"(BYTES)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int K>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(K) : "memory"); }

// v elements per tile (both precisions fill 128-320 threads at >= 84% lane use; FP64 tiles are
// kept small enough for two CTAs per SM)
template <int N, typename T>
struct GenEpt {
    static constexpr int value = sizeof(T) == 8
        ? (N == 1 ? 128 : N == 2 ? 64 : N == 3 ? 21 : N == 4 ? 16 : N == 5 ? 8 : N == 6 ? 7 : N == 7 ? 4 : N == 8 ? 4 : 3)
        : (N == 1 ? 128 : N == 2 ? 64 : N == 3 ? 21 : N == 4 ? 16 : N == 5 ? 8 : N == 6 ? 7 : N == 7 ? 8 : N == 8 ? 8 : 5);
};

// shared-memory wavefronts of one warp-wide pair load at element address
// plane * i + SL * b (+ 2 p when with_p): 64-bit accesses in half-warp phases, 128-bit in quarter-warps
template <int N, int EPT, int NT, int ES>
constexpr int gen_load_cost(int plane, bool with_p) {
    constexpr int P = (N + 1) / 2, SL = N + (N & 1), ITEMS = EPT * N * P;
    const int words = 2 * ES / 4;            // 4-byte words per lane
    const int phase = 32 / words;            // lanes per phase
    int total = 0;
    for (int w = 0; w < (ITEMS + 31) / 32; ++w) {
        for (int ph = 0; ph < 32; ph += phase) {
            int cnt[32] = {};
            long addr[32] = {};
            int na = 0;
            for (int l = ph; l < ph + phase; ++l) {
                const int it = 32 * w + l;
                if (it >= ITEMS) continue;
                const int p = it % P, bi = it / P, i = bi % N, b = bi / N;
                const long a = (long)plane * i + (long)SL * b + (with_p ? 2 * p : 0);
                bool seen = false;
                for (int q = 0; q < na; ++q) seen = seen || (addr[q] == a);
                if (seen) continue;
                addr[na++] = a;
                const long w0 = a * (ES / 4);
                for (int k = 0; k < words; ++k) ++cnt[(int)((w0 + k) % 32)];
            }
            int mx = 1;
            for (int k = 0; k < 32; ++k) mx = cnt[k] > mx ? cnt[k] : mx;
            total += mx;
        }
    }
    return total;
}

// smallest even row length in [w0, w0 + span) whose plane stride (n rows) minimises the load
// wavefronts
template <int N, int EPT, int NT, int ES>
constexpr int gen_pick_row(int w0, bool with_p, int span) {
    int best = w0, best_cost = 1 << 30;
    for (int w = w0; w < w0 + span; w += 2) {
        const int c = gen_load_cost<N, EPT, NT, ES>(N * w, with_p);
        if (c < best_cost) {
            best_cost = c;
            best = w;
        }
    }
    return best;
}

template <int N, typename T, int EPT_ = GenEpt<N, T>::value>
struct GenGeom {
    static constexpr int EPT = EPT_;
    static constexpr int P = (N + 1) / 2;           // column pairs per element
    static constexpr int SL = N + (N & 1);          // element slot width (even)
    static constexpr int H = 2;                     // first tile column of IN rows
    static constexpr int LH = H - 1 - (SL - N);     // left v trace column: slot -1, node n-1
    static constexpr int ITEMS = EPT * N * P;
    static constexpr int THREADS = (ITEMS + 31) / 32 * 32;
    static constexpr int NW = THREADS / 32;
    static constexpr int WF = EPT * SL;             // face / background row length
    static constexpr int W = gen_pick_row<N, EPT, THREADS, (int)sizeof(T)>(H + EPT * SL + 2, false, 16);
    static constexpr int WN = gen_pick_row<N, EPT, THREADS, (int)sizeof(T)>(WF, true, 8);
    static constexpr int PS = N * W;                // IN plane (x node) stride
    static constexpr int PSF = N * WN;              // FN plane stride
    static constexpr int NST = 2;                   // pipeline stages
    static constexpr bool BG = sizeof(T) == 4;      // background split: FP32 contexts only
    static constexpr size_t al(size_t b) { return (b + 127) & ~(size_t)127; }
    static constexpr size_t IN_B = al(sizeof(T) * (size_t)N * PS);
    static constexpr size_t FN_B = al(sizeof(T) * (size_t)N * PSF);
    static constexpr size_t XF_B = al(sizeof(T) * (size_t)2 * N * WF);
    static constexpr size_t UF_B = XF_B;
    static constexpr size_t BG_B = BG ? al(sizeof(float) * (size_t)2 * N * WF) : 0;
    static constexpr size_t UX_B = al(sizeof(double) * (size_t)N);
    static constexpr size_t STAGE_B = IN_B + FN_B + XF_B + UF_B + BG_B + UX_B;
    static constexpr size_t smem_bytes() {
        const size_t s = NST * STAGE_B;
        const size_t red = sizeof(dd) * (size_t)THREADS;
        return (s > red ? s : red) + 128;
    }
    // resident CTAs per SM the register allocation is sized for (shared memory permitting, and at
    // least 128 / 168 registers per thread in FP32 / FP64; warps are allocated in pairs)
    static constexpr int SMEM_CTAS = (int)((227 * 1024) / (smem_bytes() + 1024));
    static constexpr int REG_CTAS = 65536 / ((THREADS + 63) / 64 * 64 * (sizeof(T) == 8 ? 168 : 128));
    static constexpr int MINB_ = SMEM_CTAS < REG_CTAS ? SMEM_CTAS : REG_CTAS;
    static constexpr int MINB = MINB_ < 1 ? 1 : (MINB_ > 4 ? 4 : MINB_);
    static_assert(ITEMS <= THREADS, "items exceed threads");
};

// tensor maps of the TMA form (5-D views of the state: v node, j, a, i, e)
// (paired-row form: 4-D views (2R, U n / 2, n, X) with boxes (WB, NPJ, n, 1), (WB, NPJ, 1, 1) and
// (WB, 1, n, 1); background tables 2-D (2R, U n / 2) with box (WB, NPJ))
struct GenMaps {
    CUtensorMap in_tile;   // box (WB, RJ, 1, n, 1) over the stage input
    CUtensorMap fn_tile;   // the same box over f^n
    CUtensorMap xface;     // box (WB, n, 1, 1, 1): one x node plane
    CUtensorMap uface;     // box (WB, 1, 1, n, 1): one j row of every x node
    CUtensorMap bg_eu;     // FP32 background-split tables [U n][V n]: box (WB, n)
    CUtensorMap bg_rb;
};

// register budget per thread of the FP32 TMA form (resident CTAs requested from the compiler)
#ifndef VL_GEN_TMA_REG32
#define VL_GEN_TMA_REG32 128
#endif

template <int N, typename T, int EPT_ = GenEpt<N, T>::value>
struct GenTmaGeom {
    static constexpr int EPT = EPT_;
    static constexpr int Q = 16 / (int)sizeof(T);                       // elements per 16 bytes
    static constexpr int WB0 = (EPT * N + 2 + 2 * (Q - 1)) / Q * Q;     // tile + both traces, any offset
    static constexpr int WB = ((WB0 / Q) % 2 == 1) ? WB0 : WB0 + Q;    // odd number of 16-byte units
    static constexpr int RJ = N + ((N % 2 == 0) ? 1 : 0);              // j rows per plane (odd)
    static constexpr int PS = RJ * WB;                                  // plane stride
    static constexpr int UXC = N + (N & 1);                             // u nodes copied from an even start
    static constexpr int THREADS = GenGeom<N, T, EPT>::THREADS;
    static constexpr int NST = 2;
    static constexpr size_t al(size_t b) { return (b + 127) & ~(size_t)127; }
    static constexpr size_t IN_B = al(sizeof(T) * (size_t)N * PS);
    static constexpr size_t FN_B = IN_B;
    // each face side starts on a 128-byte boundary (tensor copies into shared memory need it)
    static constexpr size_t FSIDE_B = al(sizeof(T) * (size_t)N * WB);
    static constexpr size_t XF_B = 2 * FSIDE_B;
    static constexpr size_t UF_B = XF_B;
    // FP32: the two background-split tables' rows of the tile, each table on a 128-byte boundary
    static constexpr size_t BGSIDE_B = sizeof(T) == 4 ? al(sizeof(float) * (size_t)N * WB) : 0;
    static constexpr size_t BG_B = 2 * BGSIDE_B;
    static constexpr size_t UX_B = al(sizeof(double) * (size_t)UXC);
    static constexpr size_t STAGE_B = IN_B + FN_B + XF_B + UF_B + BG_B + UX_B;
    static constexpr uint32_t TX_IN = sizeof(T) * WB * RJ * N;
    static constexpr uint32_t TX_FACE = sizeof(T) * WB * N;
    static constexpr uint32_t TX_BG = sizeof(float) * WB * N;
    static constexpr uint32_t TX_UX = sizeof(double) * UXC;
    static constexpr size_t smem_bytes() {
        const size_t s = NST * STAGE_B;
        const size_t red = sizeof(dd) * (size_t)THREADS;
        return (s > red ? s : red) + 128;
    }
    static constexpr int SMEM_CTAS = (int)((227 * 1024) / (smem_bytes() + 1024));
    static constexpr int REG_CTAS = 65536 / ((THREADS + 63) / 64 * 64 * (sizeof(T) == 8 ? 168 : VL_GEN_TMA_REG32));
    static constexpr int MINB_ = SMEM_CTAS < REG_CTAS ? SMEM_CTAS : REG_CTAS;
    static constexpr int MINB = MINB_ < 1 ? 1 : (MINB_ > 4 ? 4 : MINB_);
    static_assert(WB <= 256, "TMA box width");
};

// Paired-row TMA form (FP32 rows of R = (nv+2) n floats with R = 2 mod 4, an even number U n of
// rows): a row is not a 16-byte multiple but two consecutive rows are, so the state is viewed as
// 4-D (2R floats of a row pair, U n / 2 pairs, n x nodes, x elements) and every array of a tile
// is loaded as two boxes: the even rows (pair columns [0, R)) and the odd rows ([R, 2R)), each box
// starting at the 16-byte boundary at or below its rows' left v trace.  The odd rows then sit
// 2 floats off the even ones; each parity has its own column offset in shared memory.
template <int N, typename T, int EPT_ = GenEpt<N, T>::value>
struct GenPairGeom {
    using GT = GenTmaGeom<N, T, EPT_>;
    static constexpr int EPT = EPT_;
    static constexpr int Q = GT::Q;
    static constexpr int WB = GT::WB;                  // box width: tile + traces at any offset
    static constexpr int NPJ = (N + 2) / 2;            // row pairs spanning the n rows of a u element
    static constexpr int PS = NPJ * WB;                // plane stride within one parity
    static constexpr int THREADS = GT::THREADS;
    static constexpr int NST = 2;
    static constexpr size_t al(size_t b) { return (b + 127) & ~(size_t)127; }
    static constexpr size_t BLK = al(sizeof(T) * (size_t)N * PS);       // one parity of the tile
    static constexpr size_t IN_B = 2 * BLK;
    static constexpr size_t FN_B = IN_B;
    static constexpr size_t FPB = al(sizeof(T) * (size_t)PS);          // one parity of a plane / table
    static constexpr size_t XF_B = 4 * FPB;                            // [side][parity]
    static constexpr size_t FSIDE_B = al(sizeof(T) * (size_t)N * WB);  // one u-trace side [i][WB]
    static constexpr size_t UF_B = 2 * FSIDE_B;
    static constexpr size_t BG_B = sizeof(T) == 4 ? 4 * FPB : 0;       // [table][parity]
    static constexpr size_t UX_B = GT::UX_B;
    static constexpr size_t STAGE_B = IN_B + FN_B + XF_B + UF_B + BG_B + UX_B;
    static constexpr uint32_t TX_IN = sizeof(T) * WB * NPJ * N;        // one parity
    static constexpr uint32_t TX_XF = sizeof(T) * WB * NPJ;            // one side, one parity
    static constexpr uint32_t TX_UF = sizeof(T) * WB * N;              // one side
    static constexpr uint32_t TX_BG = sizeof(float) * WB * NPJ;        // one table, one parity
    static constexpr uint32_t TX_UX = GT::TX_UX;
    static constexpr size_t smem_bytes() {
        const size_t s = NST * STAGE_B;
        const size_t red = sizeof(dd) * (size_t)THREADS;
        return (s > red ? s : red) + 128;
    }
    static constexpr int SMEM_CTAS = (int)((227 * 1024) / (smem_bytes() + 1024));
    static constexpr int REG_CTAS = GT::REG_CTAS;
    static constexpr int MINB_ = SMEM_CTAS < REG_CTAS ? SMEM_CTAS : REG_CTAS;
    static constexpr int MINB = MINB_ < 1 ? 1 : (MINB_ > 4 ? 4 : MINB_);
    static_assert(WB <= 256, "TMA box width");
};

// shared-memory layout constants of the three forms (row lengths, plane strides, array bytes):
// MODE 0 slot rows (cp.async), 1 TMA rows, 2 paired TMA rows
template <int MODE, int N, typename T, int EPT>
struct GenLayout {
    using GG = GenGeom<N, T, EPT>;
    static constexpr int RIN = GG::W, PIN = GG::PS, RFN = GG::WN, PFN = GG::PSF, RFC = GG::WF, Q = 1;
    static constexpr int FS = N * GG::WF;   // offset of the second face side (elements)
    static constexpr int BGS = N * GG::WF;  // offset of the second background table (floats)
    static constexpr size_t S_IN = GG::IN_B, S_FN = GG::FN_B, S_XF = GG::XF_B, S_UF = GG::UF_B;
    static constexpr size_t S_BG = GG::BG_B, S_STAGE = GG::STAGE_B;
};
template <int N, typename T, int EPT>
struct GenLayout<1, N, T, EPT> {
    using GT = GenTmaGeom<N, T, EPT>;
    static constexpr int RIN = GT::WB, PIN = GT::PS, RFN = GT::WB, PFN = GT::PS, RFC = GT::WB, Q = GT::Q;
    static constexpr int FS = (int)(GT::FSIDE_B / sizeof(T));
    static constexpr int BGS = (int)(GT::BGSIDE_B / sizeof(float));
    static constexpr size_t S_IN = GT::IN_B, S_FN = GT::FN_B, S_XF = GT::XF_B, S_UF = GT::UF_B;
    static constexpr size_t S_BG = GT::BG_B, S_STAGE = GT::STAGE_B;
};
template <int N, typename T, int EPT>
struct GenLayout<2, N, T, EPT> {
    using GP = GenPairGeom<N, T, EPT>;
    static constexpr int RIN = GP::WB, PIN = GP::PS, RFN = GP::WB, PFN = GP::PS, RFC = GP::WB, Q = GP::Q;
    static constexpr int FS = (int)(GP::FSIDE_B / sizeof(T));   // second u-trace side (elements)
    static constexpr int BLK = (int)(GP::BLK / sizeof(T));      // odd-row block of IN / FN (elements)
    static constexpr int FPB = (int)(GP::FPB / sizeof(T));      // one parity of a face plane / table
    static constexpr int BGS = (int)(2 * GP::FPB / sizeof(float));   // second background table (floats)
    static constexpr size_t S_IN = GP::IN_B, S_FN = GP::FN_B, S_XF = GP::XF_B, S_UF = GP::UF_B;
    static constexpr size_t S_BG = GP::BG_B, S_STAGE = GP::STAGE_B;
};

template <typename T>
struct GenPair;
template <>
struct GenPair<double> {
    using V = double2;
};
template <>
struct GenPair<float> {
    using V = float2;
};

// One CTA's share of a stage: x element e, tiles g, g + G, ... of that slab; writes the moment
// partial [e][g][i] (of G per x element).  tb supplies up / xi / wu (compile-time j indices);
// wfin[k] is the per-column factor of the moment partial (w_k / J_v for the single-problem
// tables).  smem: GenGeom::smem_bytes() of dynamic shared memory, 128-byte aligned.
template <int N, typename T, int EPT, typename TB, bool TMA = false, bool PAIR = false, int KT = -1, int BT = -1>
__device__ __forceinline__ void gen_stage_body(const StageArgs &a, const TB &tb, const double *wfin, int e,
                                               int g, int G, unsigned char *smem,
                                               const GenMaps *maps = nullptr) {
    static_assert(!PAIR || (TMA && sizeof(T) == 4), "the paired-row form is a TMA form of FP32 states");
    constexpr bool CONTIG = TMA;   // contiguous rows (scalar pair loads)
    constexpr bool MB = TMA;       // stages filled by asynchronous bulk copies on mbarriers
    using GG = GenGeom<N, T, EPT>;
    using V2 = typename GenPair<T>::V;
    constexpr int P = GG::P, SL = GG::SL, H = GG::H, LH = GG::LH, W = GG::W, WN = GG::WN, WF = GG::WF;
    constexpr int PS = GG::PS, PSF = GG::PSF, NST = GG::NST, NW = GG::NW, NT = GG::THREADS;
    // shared-memory geometry of the form in use (TMA: contiguous rows of the state)
    using L = GenLayout<PAIR ? 2 : (TMA ? 1 : 0), N, T, EPT>;
    constexpr int RIN = L::RIN;      // IN row length
    constexpr int PIN = L::PIN;      // IN plane stride
    constexpr int RFN = L::RFN;      // FN row length
    constexpr int PFN = L::PFN;      // FN plane stride
    constexpr int RFC = L::RFC;      // face / background row length
    constexpr size_t S_IN = L::S_IN, S_FN = L::S_FN, S_XF = L::S_XF, S_UF = L::S_UF;
    constexpr size_t S_BG = L::S_BG, S_STAGE = L::S_STAGE;
    constexpr int FS = L::FS;        // second face side (elements)
    __shared__ __align__(8) uint64_t gfull[2];   // TMA form: one mbarrier per stage

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const bool has_item = tid < GG::ITEMS;
    const int item = has_item ? tid : 0;
    const int p = item % P;
    const int bi = item / P;
    const int i = bi % N;
    const int b = bi / N;
    const int cs = b * SL + 2 * p;                  // tile column of the pair (slot layout)
    const int k0 = 2 * p;
    const bool pad1 = (2 * p + 1) >= N;             // second column is the odd-order pad
    const int k1 = pad1 ? N - 1 : 2 * p + 1;

    const T *__restrict__ in = static_cast<const T *>(a.in);
    const T *__restrict__ fn = static_cast<const T *>(a.fn);
    T *out = static_cast<T *>(a.out);
    T *gout = static_cast<T *>(a.ghost_out);
    const int nx = a.nx, nu = a.nu, nv = a.nv;
    const bool ghost = gout != nullptr && (e == 0 || e == nx - 1);   // CTA-uniform
    const int U = nu + 2, V = nv + 2;
    const int sJ = V * N, sA = sJ * N, sI = sA * U;
    const size_t sE_ = (size_t)sI * N;
    const int Eg = e + 1;
    int El, Er;
    if (a.xhalo == VL_XHALO_PERIODIC) {
        El = (e == 0) ? nx : e;
        Er = (e == nx - 1) ? 1 : e + 2;
    } else {
        El = e;
        Er = e + 2;
    }
    const int kind = KT >= 0 ? KT : a.kind;
    const bool with_fn = (kind == KIND_COMBINE);
    const bool with_bg = GG::BG && (BT >= 0 ? BT == 1 : a.bg_rb != nullptr);
    const int nbt = (nv + EPT - 1) / EPT;
    const int tiles = nu * nbt;
    const int ntile = (g < tiles) ? (tiles - 1 - g) / G + 1 : 0;

    // pad columns are never written by the copies: zero them once so that the pad outputs
    // (computed, not stored) stay finite
    {
        uint4 *z = reinterpret_cast<uint4 *>(smem);
        const int nz = (int)(NST * S_STAGE / 16);
        for (int q = tid; q < nz; q += blockDim.x) z[q] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();

    if constexpr (MB) {
        if (tid == 0) {
            mbar_init(&gfull[0], 1);
            mbar_init(&gfull[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncthreads();
    }
    auto stage_ptr = [&](int s) { return smem + (size_t)s * S_STAGE; };
    // one row of ncol tile columns: global run -> slot layout
    auto copy_row = [&](T *dst, const T *src, int ncol) {
        if constexpr (N % 2 == 0) {
            for (int c = 2 * lane; c < ncol; c += 64) cp_async<2 * sizeof(T)>(dst + c, src + c);
        } else {
            for (int c = lane; c < ncol; c += 32) cp_async<sizeof(T)>(dst + (c / N) * SL + c % N, src + c);
        }
    };
    auto copy_row_f = [&](float *dst, const float *src, int ncol) {
        if constexpr (N % 2 == 0) {
            for (int c = 2 * lane; c < ncol; c += 64) cp_async<8>(dst + c, src + c);
        } else {
            for (int c = lane; c < ncol; c += 32) cp_async<4>(dst + (c / N) * SL + c % N, src + c);
        }
    };
    auto issue = [&](int s, int tt) {
        const int au = tt / nbt;
        const int b0 = (tt - au * nbt) * EPT;
        const int nb = min(EPT, nv - b0);
        const int Ag = au + 1;
        const int ncol = nb * N;
        const size_t gc0 = (size_t)(b0 + 1) * N;
        unsigned char *st = stage_ptr(s);
        T *dIn = reinterpret_cast<T *>(st);
        T *dFn = reinterpret_cast<T *>(st + GG::IN_B);
        T *dXF = reinterpret_cast<T *>(st + GG::IN_B + GG::FN_B);
        T *dUF = reinterpret_cast<T *>(st + GG::IN_B + GG::FN_B + GG::XF_B);
        float *dBG = reinterpret_cast<float *>(st + GG::IN_B + GG::FN_B + GG::XF_B + GG::UF_B);
        double *dUX = reinterpret_cast<double *>(st + GG::IN_B + GG::FN_B + GG::XF_B + GG::UF_B + GG::BG_B);
        const T *slab = in + (size_t)Eg * sE_ + (size_t)Ag * sA + gc0;
        for (int r = warp; r < N * N; r += NW) {
            const int ii = r / N, jj = r - ii * N;
            const T *src = slab + (size_t)ii * sI + (size_t)jj * sJ;
            T *dst = dIn + ii * PS + jj * W + H;
            copy_row(dst, src, ncol);
            if (lane == 0) cp_async<sizeof(T)>(dst + (LH - H), src - 1);       // left v trace
            if (lane == 1) cp_async<sizeof(T)>(dst + nb * SL, src + ncol);     // right v trace
        }
        if (with_fn) {
            const T *fslab = fn + (size_t)Eg * sE_ + (size_t)Ag * sA + gc0;
            for (int r = warp; r < N * N; r += NW) {
                const int ii = r / N, jj = r - ii * N;
                copy_row(dFn + ii * PSF + jj * WN, fslab + (size_t)ii * sI + (size_t)jj * sJ, ncol);
            }
        }
        for (int r = warp; r < 4 * N; r += NW) {
            const int side = (r / N) & 1, q = r % N;
            const T *src;
            T *dst;
            if (r < 2 * N) {   // x traces: row j = q of (El, i = n-1) / (Er, i = 0)
                src = in + (size_t)(side ? Er : El) * sE_ + (size_t)(side ? 0 : N - 1) * sI + (size_t)Ag * sA +
                      (size_t)q * sJ + gc0;
                dst = dXF + (side * N + q) * WF;
            } else {           // u traces: row i = q of (a-1, j = n-1) / (a+1, j = 0)
                src = in + (size_t)Eg * sE_ + (size_t)q * sI + (size_t)(side ? Ag + 1 : Ag - 1) * sA +
                      (size_t)(side ? 0 : N - 1) * sJ + gc0;
                dst = dUF + (side * N + q) * WF;
            }
            copy_row(dst, src, ncol);
        }
        if (with_bg) {
            for (int r = warp; r < 2 * N; r += NW) {
                const int tbl = r / N, jj = r % N;
                const float *src = (tbl ? a.bg_rb : a.bg_eu) + (size_t)Ag * sA + (size_t)jj * sJ + gc0;
                copy_row_f(dBG + (tbl * N + jj) * WF, src, ncol);
            }
        }
        if (tid < N) cp_async<8>(dUX + tid, a.u_nodes + Ag * N + tid);
    };
    // TMA form: one thread loads the tile's boxes into stage s
    auto issue_tma = [&](int s, int tt) {
        if constexpr (PAIR) {
            // paired rows: even rows at pair columns [0, R), odd rows at [R, 2R); each box starts at
            // the 16-byte boundary at or below its rows' left v trace
            using GP = GenPairGeom<N, T, EPT>;
            const int au = tt / nbt;
            const int b0 = (tt - au * nbt) * EPT;
            const int Ag = au + 1;
            const int R = (nv + 2) * N;
            const int cL = (b0 + 1) * N - 1;
            const int xs0 = cL & ~(GP::Q - 1), xs1 = (R + cL) & ~(GP::Q - 1);
            const int r0 = Ag * N, p0 = r0 >> 1;
            unsigned char *st = stage_ptr(s);
            unsigned char *xf = st + S_IN + S_FN;
            unsigned char *uf = xf + S_XF;
            const uint32_t tx = 2 * GP::TX_IN * (with_fn ? 2 : 1) + 4 * GP::TX_XF + 2 * GP::TX_UF + GP::TX_UX +
                                (with_bg ? 4 * GP::TX_BG : 0);
            mbar_arrive_expect_tx(&gfull[s], tx);
#pragma unroll
            for (int par = 0; par < 2; ++par) {
                const int xs = par ? xs1 : xs0;
                tma_load_4d(st + par * GP::BLK, &maps->in_tile, &gfull[s], xs, p0, 0, Eg);
                if (with_fn) tma_load_4d(st + S_IN + par * GP::BLK, &maps->fn_tile, &gfull[s], xs, p0, 0, Eg);
                tma_load_4d(xf + par * GP::FPB, &maps->xface, &gfull[s], xs, p0, N - 1, El);
                tma_load_4d(xf + (2 + par) * GP::FPB, &maps->xface, &gfull[s], xs, p0, 0, Er);
                if (with_bg) {
                    tma_load_2d(uf + S_UF + par * GP::FPB, &maps->bg_eu, &gfull[s], xs, p0);
                    tma_load_2d(uf + S_UF + (2 + par) * GP::FPB, &maps->bg_rb, &gfull[s], xs, p0);
                }
            }
            const int rl = r0 - 1, rr = r0 + N;   // u traces: row n-1 of element a-1, row 0 of a+1
            tma_load_4d(uf, &maps->uface, &gfull[s], (rl & 1) ? xs1 : xs0, rl >> 1, 0, Eg);
            tma_load_4d(uf + GP::FSIDE_B, &maps->uface, &gfull[s], (rr & 1) ? xs1 : xs0, rr >> 1, 0, Eg);
            bulk_load(uf + S_UF + S_BG, a.u_nodes + ((Ag * N) & ~1), GP::TX_UX, &gfull[s]);
        } else if constexpr (TMA) {
            using GT = GenTmaGeom<N, T, EPT>;
            const int au = tt / nbt;
            const int b0 = (tt - au * nbt) * EPT;
            const int Ag = au + 1;
            const int xs = ((b0 + 1) * N - 1) & ~(GT::Q - 1);
            unsigned char *st = stage_ptr(s);
            unsigned char *xf = st + S_IN + S_FN;
            unsigned char *uf = xf + S_XF;
            const uint32_t tx = GT::TX_IN * (with_fn ? 2 : 1) + 4 * GT::TX_FACE + GT::TX_UX +
                                (with_bg ? 2 * GT::TX_BG : 0);
            mbar_arrive_expect_tx(&gfull[s], tx);
            tma_load_5d(st, &maps->in_tile, &gfull[s], xs, 0, Ag, 0, Eg);
            if (with_fn) tma_load_5d(st + S_IN, &maps->fn_tile, &gfull[s], xs, 0, Ag, 0, Eg);
            tma_load_5d(xf, &maps->xface, &gfull[s], xs, 0, Ag, N - 1, El);
            tma_load_5d(xf + GT::FSIDE_B, &maps->xface, &gfull[s], xs, 0, Ag, 0, Er);
            tma_load_5d(uf, &maps->uface, &gfull[s], xs, N - 1, Ag - 1, 0, Eg);
            tma_load_5d(uf + GT::FSIDE_B, &maps->uface, &gfull[s], xs, 0, Ag + 1, 0, Eg);
            if (with_bg) {
                tma_load_2d(uf + S_UF, &maps->bg_eu, &gfull[s], xs, Ag * N);
                tma_load_2d(uf + S_UF + GT::BGSIDE_B, &maps->bg_rb, &gfull[s], xs, Ag * N);
            }
            bulk_load(uf + S_UF + S_BG, a.u_nodes + ((Ag * N) & ~1), GT::TX_UX, &gfull[s]);
        } else {
            (void)s;
            (void)tt;
        }
    };

    const double accel = a.accel, bfield = a.bfield, nbfield = -a.bfield;
    const float kvf = (float)(accel * nbfield);   // FP32 v speed per unit u
    const double dtd = (kind == KIND_RHS) ? 0.0 : *a.dt;
    const T dtT = (T)dtd, c0 = (T)a.c0, c1 = (T)a.c1, c2dt = (T)(a.c2 * dtd);
    const T jx = (T)a.jx, ju = (T)a.ju, jv = (T)a.jv;
    const double Ei = a.E[Eg * N + i];
    T upi[N], upk0[N], upk1[N];
#pragma unroll
    for (int m = 0; m < N; ++m) {
        upi[m] = tb.up[i * N + m];
        upk0[m] = tb.up[k0 * N + m];
        upk1[m] = tb.up[k1 * N + m];
    }
    const T xig0 = tb.xi[2 * i], xig1 = tb.xi[2 * i + 1];
    const T xik00 = tb.xi[2 * k0], xik01 = tb.xi[2 * k0 + 1];
    const T xik10 = tb.xi[2 * k1], xik11 = tb.xi[2 * k1 + 1];
    const double wf0 = wfin[k0], wf1 = pad1 ? 0.0 : wfin[k1];
    double mk0 = 0.0, mk1 = 0.0;   // sum_j wu_j out[.., j, k] for the two columns

    if constexpr (TMA) {
        if (tid == 0) {
            if (ntile > 0) issue_tma(0, g);
            if (ntile > 1) issue_tma(1, g + G);
        }
    } else {
#pragma unroll
        for (int s0 = 0; s0 < NST - 1; ++s0) {
            if (s0 < ntile) issue(s0, g + s0 * G);
            cp_async_commit();
        }
    }
    for (int q = 0; q < ntile; ++q) {
        if constexpr (!MB) {
            const int qn = q + NST - 1;
            if (qn < ntile) issue(qn % NST, g + qn * G);
            cp_async_commit();
        }
        const int tt = g + q * G;
        const int au = tt / nbt;
        const int b0 = (tt - au * nbt) * EPT;
        const int nb = min(EPT, nv - b0);
        const int Ag = au + 1;
        const bool act = has_item && b < nb;
        const int col = (b0 + b + 1) * N + 2 * p;    // global v-node column of the pair
        const double vn0 = act ? a.v_nodes[col] : 0.0, vn1 = act ? a.v_nodes[col + 1] : 0.0;
        if constexpr (MB) {
            if (!mbar_wait_bounded(&gfull[q & 1], (uint32_t)((q >> 1) & 1))) {
                if (a.err != nullptr) atomicOr(a.err, 2);
                return;
            }
        } else {
            cp_async_wait<NST - 1>();
            __syncthreads();   // tile q visible to every thread
        }
        const unsigned char *st = stage_ptr(q % NST);
        const T *sIn = reinterpret_cast<const T *>(st);
        const T *sFn = reinterpret_cast<const T *>(st + S_IN);
        const T *sXF = reinterpret_cast<const T *>(st + S_IN + S_FN);
        const T *sUF = reinterpret_cast<const T *>(st + S_IN + S_FN + S_XF);
        const float *sBG = reinterpret_cast<const float *>(st + S_IN + S_FN + S_XF + S_UF);
        const double *sUX0 = reinterpret_cast<const double *>(st + S_IN + S_FN + S_XF + S_UF + S_BG);
        // column of element b's node 0 in the IN rows, of the thread's pair in IN and in the
        // FN / face / background rows; first u node in sUX
        const int cL = (b0 + 1) * N - 1;
        const int ebase = TMA ? (cL - (cL & ~(L::Q - 1))) + 1 + b * N : H + b * SL;
        const int cin = ebase + 2 * p;
        const int cfc = CONTIG ? cin : cs;
        // paired rows: column of element b's node 0 in the even and in the odd rows
        const int Rrow = (nv + 2) * N;
        const int e0 = (cL & (L::Q - 1)) + 1 + b * N;
        const int e1 = ((Rrow + cL) & (L::Q - 1)) + 1 + b * N;
        (void)Rrow;
        (void)e0;
        (void)e1;
        const double *sUX = sUX0 + (MB ? ((Ag * N) & 1) : 0);
        auto ld2 = [&](const T *q2) -> V2 {
            if constexpr (CONTIG) {
                V2 r;
                r.x = q2[0];
                r.y = q2[1];
                return r;
            } else {
                return *reinterpret_cast<const V2 *>(q2);
            }
        };
        // the tile body, for the parity RP of the tile's first row among the U n rows (paired form;
        // 0 otherwise): row r of the tile is row (RP + r) / 2 of parity (RP + r) % 2
        auto tile_rows = [&](auto rpc, auto ghost_c) {
            constexpr int RP = decltype(rpc)::value;
            constexpr bool GHOST = decltype(ghost_c)::value;   // x-ghost refresh rows
            (void)RP;
            // IN / FN layout: pointer to node 0 of element b in row r of plane pl
            auto rowp = [&](const T *arr, int pl, int r) -> const T * {
                if constexpr (PAIR) {
                    const int par = (RP + r) & 1, idx = (RP + r) >> 1;
                    return arr + par * L::BLK + pl * PIN + idx * RIN + (par ? e1 : e0);
                } else {
                    return arr + pl * PIN + r * RIN + ebase;
                }
            };
            // face / background layout ([side][parity][pair][WB] in the paired form): node 0 of
            // element b in row r of side sd
            auto facep = [&](const T *arr, int sd, int r) -> const T * {
                if constexpr (PAIR) {
                    const int par = (RP + r) & 1, idx = (RP + r) >> 1;
                    return arr + (2 * sd + par) * L::FPB + idx * RFC + (par ? e1 : e0);
                } else {
                    return arr + sd * FS + r * RFC + cfc - 2 * p;
                }
            };
            const double sd0 = accel * (Ei + bfield * vn0);
            const double sd1 = accel * (Ei + bfield * vn1);
            const T sp0 = (T)sd0, sp1 = (T)sd1;
            V2 fu[N];
#pragma unroll
            for (int m = 0; m < N; ++m) fu[m] = ld2(rowp(sIn, i, m) + 2 * p);
            V2 ufl, ufr;
            if constexpr (PAIR) {   // row n-1 of element a-1: parity RP + 1; row 0 of a+1: RP + n
                ufl = ld2(sUF + i * RFC + (((RP + 1) & 1) ? e1 : e0) + 2 * p);
                ufr = ld2(sUF + FS + i * RFC + (((RP + N) & 1) ? e1 : e0) + 2 * p);
            } else {
                ufl = ld2(sUF + i * RFC + cfc);
                ufr = ld2(sUF + FS + i * RFC + cfc);
            }
            const T uL0 = (sd0 >= 0.0) ? ufl.x : fu[0].x, uR0 = (sd0 >= 0.0) ? fu[N - 1].x : ufr.x;
            const T uL1 = (sd1 >= 0.0) ? ufl.y : fu[0].y, uR1 = (sd1 >= 0.0) ? fu[N - 1].y : ufr.y;
            T *pout = out + (size_t)Eg * sE_ + (size_t)i * sI + (size_t)Ag * sA + col;
            float mf0 = 0.0f, mf1 = 0.0f;   // FP32: the tile's moment sums, added in FP64 after it
            (void)mf0;
            (void)mf1;
#pragma unroll
            for (int j = 0; j < N; ++j) {
                // x and v speeds of row j (FP32: one conversion, the v speed formed in FP32)
                T uxT, svT;
                if constexpr (sizeof(T) == 4) {
                    uxT = (float)sUX[j];
                    svT = kvf * uxT;
                } else {
                    const double uxd = sUX[j];
                    uxT = uxd;
                    svT = accel * (nbfield * uxd);
                }
                const bool xpos = uxT >= (T)0;
                const bool vpos = svT >= (T)0;
                // x: sum_m up[i][m] F[m][j][k] + lifts
                const T *pc = rowp(sIn, 0, j) + 2 * p;
                T dx0 = (T)0, dx1 = (T)0;
                V2 cm0, cmL;
#pragma unroll
                for (int m = 0; m < N; ++m) {
                    const V2 cv = ld2(pc + m * PIN);
                    if (m == 0) cm0 = cv;
                    if (m == N - 1) cmL = cv;
                    dx0 = fma(upi[m], cv.x, dx0);
                    dx1 = fma(upi[m], cv.y, dx1);
                }
                const V2 xf0 = ld2(facep(sXF, 0, j) + 2 * p);
                const V2 xf1 = ld2(facep(sXF, 1, j) + 2 * p);
                const V2 xl = xpos ? xf0 : cm0;
                const V2 xr = xpos ? cmL : xf1;
                dx0 = fma(xig0, xl.x, dx0);
                dx0 = fma(-xig1, xr.x, dx0);
                dx1 = fma(xig0, xl.y, dx1);
                dx1 = fma(-xig1, xr.y, dx1);
                // v: sum_m F[i][j][m] up[k][m] + lifts (the element's k-line)
                const T *pa = rowp(sIn, i, j);   // k-line of element b
                T line[2 * P];
#pragma unroll
                for (int m2 = 0; m2 < P; ++m2) {
                    const V2 l2 = ld2(pa + 2 * m2);
                    line[2 * m2] = l2.x;
                    line[2 * m2 + 1] = l2.y;
                }
                T dv0 = (T)0, dv1 = (T)0;
#pragma unroll
                for (int m = 0; m < N; ++m) {
                    dv0 = fma(upk0[m], line[m], dv0);
                    dv1 = fma(upk1[m], line[m], dv1);
                }
                const T tl = vpos ? pa[CONTIG ? -1 : LH - H] : line[0];
                const T tr = vpos ? line[N - 1] : pa[CONTIG ? N : SL];
                dv0 = fma(xik00, tl, dv0);
                dv0 = fma(-xik01, tr, dv0);
                dv1 = fma(xik10, tl, dv1);
                dv1 = fma(-xik11, tr, dv1);
                // u: sum_m up[j][m] F[i][m][k] + lifts (compile-time j: table constants)
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
                T r0 = fma(uxT * dx0, jx, fma(sp0 * du0, ju, (svT * dv0) * jv));
                T r1 = fma(uxT * dx1, jx, fma(sp1 * du1, ju, (svT * dv1) * jv));
                if (with_bg) {   // RHS of the x-independent background
                    float2 eu, rb;
                    const float *pbg;
                    if constexpr (PAIR) {   // [table][parity][pair][WB]
                        const int par = (RP + j) & 1, idx = (RP + j) >> 1;
                        pbg = sBG + par * L::FPB + idx * RFC + (par ? e1 : e0) + 2 * p;
                    } else {
                        pbg = sBG + j * RFC + cfc;
                    }
                    if constexpr (CONTIG) {
                        eu = make_float2(pbg[0], pbg[1]);
                        rb = make_float2(pbg[L::BGS], pbg[L::BGS + 1]);
                    } else {
                        eu = *reinterpret_cast<const float2 *>(pbg);
                        rb = *reinterpret_cast<const float2 *>(pbg + L::BGS);
                    }
                    r0 += (T)fmaf((float)Ei, eu.x, rb.x);
                    r1 += (T)fmaf((float)Ei, eu.y, rb.y);
                }
                const V2 fij = fu[j];
                V2 o;
                if (kind == KIND_RHS) {
                    o.x = r0;
                    o.y = r1;
                } else if (kind == KIND_EULER) {
                    o.x = fma(dtT, r0, fij.x);
                    o.y = fma(dtT, r1, fij.y);
                } else {
                    const V2 fnv = PAIR ? ld2(rowp(sFn, i, j) + 2 * p) : ld2(sFn + i * PFN + j * RFN + cfc);
                    o.x = rk_combine(c0, c1, c2dt, fnv.x, fij.x, r0);
                    o.y = rk_combine(c0, c1, c2dt, fnv.y, fij.y, r1);
                }
                T *po = pout + (size_t)j * sJ;
                if constexpr (N % 2 == 0) {
                    *reinterpret_cast<V2 *>(po) = o;
                } else {
                    po[0] = o.x;
                    if (!pad1) po[1] = o.y;
                }
                if constexpr (GHOST) {
                    // periodic x-ghost refresh of f (Distribution.swap_ghost_cells_of_array)
                    const size_t gb = (size_t)i * sI + (size_t)Ag * sA + (size_t)j * sJ + col;
                    if (e == nx - 1) {
                        gout[gb] = fij.x;
                        if (!pad1) gout[gb + 1] = fij.y;
                    }
                    if (e == 0) {
                        gout[(size_t)(nx + 1) * sE_ + gb] = fij.x;
                        if (!pad1) gout[(size_t)(nx + 1) * sE_ + gb + 1] = fij.y;
                    }
                }
                if constexpr (sizeof(T) == 4) {
                    mf0 = fmaf((float)tb.wu[j], o.x, mf0);
                    mf1 = fmaf((float)tb.wu[j], o.y, mf1);
                } else {
                    mk0 = fma(tb.wu[j], (double)o.x, mk0);
                    mk1 = fma(tb.wu[j], (double)o.y, mk1);
                }
            }
            if constexpr (sizeof(T) == 4) {
                mk0 += (double)mf0;
                mk1 += (double)mf1;
            }
        };
        // (the edge x elements of stage 1 refresh f's ghost slabs: their own instantiation, so the
        // other CTAs' row loop has no branch on it)
        auto tile_ghost = [&](auto rpc) {
            if (ghost)
                tile_rows(rpc, std::true_type{});
            else
                tile_rows(rpc, std::false_type{});
        };
        if (act) {
            if constexpr (PAIR) {
                if ((Ag * N) & 1)
                    tile_ghost(std::integral_constant<int, 1>{});
                else
                    tile_ghost(std::integral_constant<int, 0>{});
            } else {
                tile_ghost(std::integral_constant<int, 0>{});
            }
        }
        __syncthreads();   // stage q % NST consumed before it is refilled
        if constexpr (TMA) {
            if (tid == 0 && q + 2 < ntile) issue_tma(q & 1, g + (q + 2) * G);
        }
    }
    cp_async_wait<0>();

    if (a.partials == nullptr) return;
    // moment partial of x node i: sum over the CTA's items of that node, fixed order
    __syncthreads();
    dd *sRed = reinterpret_cast<dd *>(smem);
    sRed[tid] = has_item ? two_sum(wf0 * mk0, wf1 * mk1) : dd{0.0, 0.0};
    __syncthreads();
    if (tid < N) {
        dd s = {0.0, 0.0};
        for (int bb = 0; bb < EPT; ++bb)
            for (int pp = 0; pp < P; ++pp) s = dd_add(s, sRed[(bb * N + tid) * P + pp]);
        a.partials[((size_t)e * G + g) * N + tid] = s.hi + s.lo;
    }
    (void)NT;
}

template <int N, typename T>
__global__ void __launch_bounds__(GenGeom<N, T>::THREADS, GenGeom<N, T>::MINB)
stage_gen_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb) {
    if (a.state != nullptr && a.state->active == 0) return;
    extern __shared__ __align__(16) unsigned char gen_smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gen_smem_raw) + 127) & ~(uintptr_t)127);
    gen_stage_body<N, T, GenGeom<N, T>::EPT>(a, tb, tb.wv, blockIdx.y, blockIdx.x, gridDim.x, base);
}

// TMA form (16-byte-aligned state rows).  KT / BT >= 0 fix the stage kind and the background
// split at compile time (the instantiations launched by the loop: no per-row branches on them);
// -1 reads them from the arguments.
template <int N, typename T, int KT = -1, int BT = -1>
__global__ void __launch_bounds__(GenTmaGeom<N, T>::THREADS, GenTmaGeom<N, T>::MINB)
stage_gen_tma_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb,
                     const __grid_constant__ GenMaps maps) {
    if (a.state != nullptr && a.state->active == 0) return;
    extern __shared__ __align__(16) unsigned char gen_smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gen_smem_raw) + 127) & ~(uintptr_t)127);
    gen_stage_body<N, T, GenGeom<N, T>::EPT, StageTables<T>, true, false, KT, BT>(
        a, tb, tb.wv, blockIdx.y, blockIdx.x, gridDim.x, base, &maps);
}

// paired-row TMA form (FP32 rows of R = 2 mod 4 floats); KT / BT as for the TMA form
template <int N, typename T, int KT = -1, int BT = -1>
__global__ void __launch_bounds__(GenPairGeom<N, T>::THREADS, GenPairGeom<N, T>::MINB)
stage_gen_pair_kernel(const StageArgs a, const __grid_constant__ StageTables<T> tb,
                      const __grid_constant__ GenMaps maps) {
    if (a.state != nullptr && a.state->active == 0) return;
    extern __shared__ __align__(16) unsigned char gen_smem_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(gen_smem_raw) + 127) & ~(uintptr_t)127);
    gen_stage_body<N, T, GenGeom<N, T>::EPT, StageTables<T>, true, true, KT, BT>(
        a, tb, tb.wv, blockIdx.y, blockIdx.x, gridDim.x, base, &maps);
}

}  // namespace vl
