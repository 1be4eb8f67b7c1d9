// Device kernels of the 1D2V DG Vlasov-Poisson hot path (sm_100a).
//
// State layout in HBM: the reference's ghost-inclusive C-order array
//     f[X][n][U][n][V][n]   X = nx+2, U = nu+2, V = nv+2      (main/grid.py:262-268)
// i.e. a plain 3-D node grid (X n) x (U n) x (V n) whose innermost axis (v) is contiguous.
// A DG element is an n^3 block; its six face traces are the adjacent node planes.
//
// Kernels
//   stage kernel    (vlasov_stage.cuh) one fused SSP-RK stage or a bare RHS.
//   moment_kernel   standalone zeroth velocity moment, one CTA per (x element, x node).
//   field_kernel    one CTA: moment partials -> density -> mean-subtracted charge -> forward
//                   high-order DFT -> spectral E and phi -> inverse DFT at the LGL nodes ->
//                   periodic ghosts; optionally energy, adaptive dt and the loop bookkeeping.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "vlasov1d2v.h"

namespace vl {

constexpr int NMAX = 10;

enum StageKind : int { KIND_EULER = 0, KIND_COMBINE = 1, KIND_RHS = 2 };

// Per-order coefficient tables passed by value as kernel parameters: the contraction loops are
// fully unrolled, so every table entry is a compile-time offset into the parameter constant
// bank and becomes an FMA operand without a load instruction.
template <typename T>
struct StageTables {
    T up[NMAX * NMAX];     // up[i][j]        (main/basis.py:176-188)
    T xi[NMAX * 2];        // xi[i][face]     (main/basis.py:110)
    double qw[NMAX * NMAX];  // w_j w_k / (J_u J_v)  (main/grid.py:297-301)
    // up with the own-trace lift folded in, per upwind direction:
    //   speed >= 0: d = sum_m upP[i][m] f[m] + xi[i][0] * (left neighbour trace)
    //   speed <  0: d = sum_m upM[i][m] f[m] - xi[i][1] * (right neighbour trace)
    T upP[NMAX * NMAX];
    T upM[NMAX * NMAX];
    // the velocity weights factored: w_j w_k / (J_u J_v) = (w_j / J_u) (w_k / J_v)
    double wu[NMAX];
    double wv[NMAX];
};

struct StageArgs {
    const void *in;        // stage input (ghost-inclusive)
    const void *fn;        // f^n for KIND_COMBINE
    void *out;             // output (interior written)
    void *ghost_out;       // when not null (KIND_EULER on f): periodic x-ghost refresh of f
    const double *E;       // [(nx+2) n]
    const double *dt;      // device scalar
    const vl_run_state *state;  // when not null, the kernel returns if !state->active
    const double *u_nodes; // [(nu+2) n]
    const void *usv;       // [(nu+2) n] pairs (u, a (-B u)) in the state precision: the x and v
                           // flux speeds per u node (n = 8 kernel)
    const double *v_nodes; // [(nv+2) n]
    double *partials;      // [nx][G][n] moment partials of out, or null
    const double *tables;  // device copy: up [n n], xi [n 2], qw [n n] (per-lane indexed reads)
    int *err;              // device error word: bit 1 = a bounded wait timed out
    int nx, nu, nv;
    int xhalo;
    int kind;
    double c0, c1, c2;
    double accel, bfield, jx, ju, jv;
    // Background split (FP32 mixed form): when bg_rb is not null the state holds the deviation
    // from an x-independent background f0(u, v), and the RHS of f0 is added per node:
    //   r0 = E_i * bg_eu + bg_rb,
    // tables in the velocity-slab layout [U][n][V][n] (index a sA + j sJ + v column).
    const float *bg_rb;
    const float *bg_eu;
    // FP32 n = 8 kernel: its per-u-node speed table holds u J_x and a (-B u) J_v with the
    // context's Jacobians; a call with other direction weights (jx, jv above) scales them by
    // jx / J_x and jv / J_v (the RHS kind only; the RK stages use the context's Jacobians)
    double sx, sv;
};


// SSP-RK combination stage c0 f^n + c1 s + (c2 dt) r with c0 + c1 = 1 (main/timestep.py:157-163,
// :174-182).  FP64 evaluates the reference's expression as written; FP32 evaluates
// f^n + c1 (s - f^n) + (c2 dt) r, whose weights of f^n and s sum to exactly 1: with rounded
// weights, float(1/3) + float(2/3) = 1 + 3e-8 would amplify every mode by 3e-8 per step.
template <typename T>
__device__ __forceinline__ T rk_combine(T c0, T c1, T c2dt, T fn, T s, T r) {
    if constexpr (sizeof(T) == 4)
        return fma(c2dt, r, fma(c1, s - fn, fn));
    else
        return fma(c2dt, r, fma(c1, s, c0 * fn));
}

// ----------------------------------------------------------------------------------------------
// error-free transformation helpers for the FP64 moment reductions
// ----------------------------------------------------------------------------------------------
struct dd {
    double hi, lo;
};

__device__ __forceinline__ dd two_sum(double a, double b) {
    double s = a + b;
    double bp = s - a;
    double e = (a - (s - bp)) + (b - bp);
    return {s, e};
}

__device__ __forceinline__ dd dd_add(dd a, dd b) {
    dd s = two_sum(a.hi, b.hi);
    double lo = s.lo + a.lo + b.lo;
    dd r = two_sum(s.hi, lo);
    return r;
}

__device__ __forceinline__ dd shfl_down_dd(dd v, int off) {
    dd r;
    r.hi = __shfl_down_sync(0xffffffffu, v.hi, off);
    r.lo = __shfl_down_sync(0xffffffffu, v.lo, off);
    return r;
}

// ----------------------------------------------------------------------------------------------
// standalone moment: grid (G, nx).  CTA (g, e) sums the interior u elements
// [g nu / G, (g + 1) nu / G) of x slab e for every x node i and writes
// out[(e G + g) n + i] -- the layout of the stage kernels' moment partials.
// Columns go to threads with a stride that is a multiple of n, so each thread sees one v node
// k and keeps its row of weights w_j w_k / (J_u J_v) in registers.
// ----------------------------------------------------------------------------------------------
// runtime-indexed read of a small register array (unrolled select)
template <int N>
__device__ __forceinline__ double acc_at(const double (&v)[N], int i) {
    double r = v[0];
#pragma unroll
    for (int m = 1; m < N; ++m)
        if (m == i) r = v[m];
    return r;
}

// block-wide double-double sum (all threads call); result valid in every thread
__device__ __forceinline__ double block_sum_dd_rt(double v, double c, dd *scratch) {
    dd s = {v, c};
    for (int off = 16; off > 0; off >>= 1) s = dd_add(s, shfl_down_dd(s, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = s;
    __syncthreads();
    dd t = scratch[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = dd_add(t, scratch[w]);
    return t.hi + t.lo;
}

struct MomentArgs {
    const void *f;
    double *out;
    int G;
    int nx, nu, nv;
    double qw[NMAX * NMAX];
};

constexpr int MOMENT_THREADS = 256;
// 2 resident CTAs per SM leave 128 registers per thread, room for most of a column's n x n loads
// in flight at once (at 4 CTAs, 64 registers, the loads issued a few at a time and the kernel ran
// at half the HBM rate, bound by load latency)
constexpr int MOMENT_CTAS_PER_SM = 2;

template <int N, typename T>
__global__ void __launch_bounds__(MOMENT_THREADS, MOMENT_CTAS_PER_SM) moment_kernel(const MomentArgs a) {
    const T *__restrict__ f = static_cast<const T *>(a.f);
    constexpr int CT = (MOMENT_THREADS / N) * N;   // column threads (stride keeps k fixed)
    const int g = blockIdx.x, Gn = gridDim.x, e = blockIdx.y;
    const int nu = a.nu, nv = a.nv;
    const int U = nu + 2, V = nv + 2;
    const int sJ = V * N, sA = sJ * N, sI = sA * U;
    const size_t slab = (size_t)(e + 1) * ((size_t)sI * N);
    const int a_lo = (int)(((long long)g * nu) / Gn), a_hi = (int)(((long long)(g + 1) * nu) / Gn);
    const int tid = threadIdx.x;
    const int ncol = nv * N;
    const int k = tid % N;
    double w[N];
#pragma unroll
    for (int j = 0; j < N; ++j) w[j] = a.qw[j * N + k];
    double acc[N];
#pragma unroll
    for (int i = 0; i < N; ++i) acc[i] = 0.0;
    if (tid < CT) {
        for (int au = a_lo; au < a_hi; ++au) {
            const T *pa = f + slab + (size_t)(au + 1) * sA + N;   // interior columns start at N
            for (int c = tid; c < ncol; c += CT) {
#pragma unroll
                for (int i = 0; i < N; ++i) {
                    double s = 0.0;
#pragma unroll
                    for (int j = 0; j < N; ++j) s = fma(w[j], (double)pa[(size_t)i * sI + j * sJ + c], s);
                    acc[i] += s;
                }
            }
        }
    }
    __shared__ dd red[MOMENT_THREADS / 32];
    for (int i = 0; i < N; ++i) {
        const double tot = block_sum_dd_rt(acc_at(acc, i), 0.0, red);
        if (tid == 0) a.out[((size_t)e * Gn + g) * N + i] = tot;
    }
}

// rho[e][i] = sum over g of the partials [e][g][i] (double-double, fixed order)
static __global__ void moment_reduce_kernel(const double *__restrict__ partials, double *__restrict__ rho,
                                     int nx, int G, int n) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= nx * n) return;
    const int e = p / n, i = p - e * n;
    dd s = {0.0, 0.0};
    for (int g = 0; g < G; ++g) s = dd_add(s, dd{partials[((size_t)e * G + g) * n + i], 0.0});
    rho[p] = s.hi + s.lo;
}

// ----------------------------------------------------------------------------------------------
// field solve (the kernel itself is vlasov_field.cuh): arguments, loop gating, reductions
// ----------------------------------------------------------------------------------------------
enum FieldMode : int {
    FIELD_REQUIRE_ACTIVE = 1,  // return if !state->active
    FIELD_PROMOTE = 2,         // start of a step: active <- active_next, dt <- dt_next
    FIELD_RECORD = 4,          // after stage 2: energy, dt_next, time, steps, history
};

struct FieldArgs {
    const double *partials;   // [nx][G][n] (rho = sum over g), or null when charge_in is used
    int G;
    const double *charge_in;  // [nx][n] mean-subtracted charge density (vl_poisson), or null
    double *E;                // [(nx+2) n]
    double *phi;              // [nx n] or null
    vl_run_state *state;      // or null
    int mode;
    const double2 *ell;       // [n][M]   T[e, j, m] = phase[e, m] ell[j, m]
    const double2 *phase;     // [nx][M]  exp(-i k_m mid_e)
    const double2 *qnode;     // [n][M]   exp(i k_m x_{e,j}) = conj(phase[e, m]) qnode[j, m]
    const double *k;          // [M]
    const double *xw;         // [n]
    int nx, n, M;
    double kappa, dx, length, accel, bfield, umax, vmax, du, dv, courant;
    // 1: each CTA first copies the phase-table entries it reads in its loops into shared memory
    // (field_prefetch_bytes more dynamic shared memory; the arithmetic is unchanged)
    int prefetch;
};

constexpr int FIELD_THREADS = 1024;            // threads of the single-CTA scalar kernel
constexpr int FIELD_MAX_NODES = 64 * NMAX;    // nx * n capacity of the shared buffers
constexpr int FIELD_MAX_MODES = 2 * 160 + 1;  // M capacity

__device__ __forceinline__ double block_sum_dd(double v, double c, dd *scratch) {
    return block_sum_dd_rt(v, c, scratch);
}

__device__ __forceinline__ double block_max(double v, double *scratch) {
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double t = scratch[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, scratch[w]);
    return t;
}

// returns false when this step is inactive (all threads agree)
__device__ __forceinline__ bool field_gate(const FieldArgs &a, bool first_cta) {
    vl_run_state *st = a.state;
    if (st == nullptr) return true;
    if (a.mode & FIELD_PROMOTE) {
        const int go = st->active_next;
        if (first_cta && threadIdx.x == 0) {
            st->active = go;
            if (go) st->dt = st->dt_next;
        }
        return go != 0;
    }
    if (a.mode & FIELD_REQUIRE_ACTIVE) return st->active != 0;
    return true;
}

// energy + dt from a given E (vl_field_energy / vl_adapt_dt / vl_run_state_init)
struct ScalarArgs {
    const double *E;
    const double *xw;
    int nx, n;
    double accel, bfield, umax, vmax, dx, du, dv, courant;
    double *energy;      // or null
    double *dt;          // or null
    vl_run_state *init;  // or null: initialise the loop state
    double final_time;
    int64_t max_steps;
    double *eh, *th, *dh;
    int cap;
};

static __global__ void __launch_bounds__(FIELD_THREADS) scalars_kernel(const ScalarArgs a) {
    __shared__ dd s_red[FIELD_THREADS / 32];
    __shared__ double s_max[FIELD_THREADS / 32];
    const int nn = a.nx * a.n;
    double esq = 0.0, esqc = 0.0, emax = 0.0;
    // energy over the interior rows E[1:-1]; max |a E| over all rows incl. ghosts
    for (int p = threadIdx.x; p < nn + 2 * a.n; p += blockDim.x) {
        const double er = a.E[p];
        emax = fmax(emax, fabs(a.accel * er));
        if (p >= a.n && p < nn + a.n) {
            const double v = a.xw[p % a.n] * (er * er);
            const double t = esq + v;
            esqc += (fabs(esq) >= fabs(v)) ? ((esq - t) + v) : ((v - t) + esq);
            esq = t;
        }
    }
    const double energy = 0.5 * block_sum_dd(esq, esqc, s_red);
    const double maxE = block_max(emax, s_max);
    if (threadIdx.x == 0) {
        const double ab = a.accel * a.bfield;
        const double s0 = fabs(a.umax);
        const double s1 = fabs(maxE + fabs(ab * a.vmax));
        const double s2 = fabs(a.accel * fabs(a.bfield * a.umax));
        const double dtn = a.courant / (((s0 / a.dx) + (s1 / a.du)) + (s2 / a.dv));
        if (a.energy) *a.energy = energy;
        if (a.dt) *a.dt = dtn;
        if (a.init) {
            vl_run_state *st = a.init;
            st->dt = dtn;
            st->dt_next = dtn;
            st->time = 0.0;
            st->final_time = a.final_time;
            st->steps = 0;
            st->max_steps = a.max_steps;
            st->active = 0;
            const bool finite = isfinite(energy) && isfinite(dtn);
            st->status = finite ? 0 : 1;
            st->active_next = (0.0 < a.final_time) && (0 < a.max_steps) && finite;
            st->hist_capacity = a.cap;
            st->energy_hist = a.eh;
            st->time_hist = a.th;
            st->dt_hist = a.dh;
        }
    }
}

}  // namespace vl
