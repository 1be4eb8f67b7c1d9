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
    const double *v_nodes; // [(nv+2) n]
    double *partials;      // [nx][G][n] moment partials of out, or null
    const double *tables;  // device copy: up [n n], xi [n 2], qw [n n] (per-lane indexed reads)
    int *err;              // device error word: bit 1 = a bounded wait timed out
    int nx, nu, nv;
    int xhalo;
    int kind;
    double c0, c1, c2;
    double accel, bfield, jx, ju, jv;
};

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
// standalone moment: one CTA per (x element e, x node i); writes rho[e][i] at
// out[(e * G + 0) * N + i] with out[(e * G + g) * N + i] = 0 for g > 0 (partials layout).
// ----------------------------------------------------------------------------------------------
struct MomentArgs {
    const void *f;
    double *out;
    int G;
    int nx, nu, nv;
    double qw[NMAX * NMAX];
};

template <int N, typename T>
__global__ void __launch_bounds__(256) moment_kernel(const MomentArgs a) {
    const T *__restrict__ f = static_cast<const T *>(a.f);
    const int e = blockIdx.x / N, i = blockIdx.x % N;
    const int U = a.nu + 2, V = a.nv + 2;
    const size_t sJ = (size_t)V * N, sA = sJ * N, sI = sA * U, sE = sI * N;
    const size_t plane = (size_t)(e + 1) * sE + (size_t)i * sI;
    const int ncol = a.nv * N;
    const int nrow = a.nu * N;
    double acc = 0.0, comp = 0.0;
    for (int idx = threadIdx.x; idx < nrow * ncol; idx += blockDim.x) {
        const int r = idx / ncol, c = idx - (idx / ncol) * ncol;
        const int au = r / N, j = r % N;
        const int k = c % N;
        const double v = a.qw[j * N + k] * (double)f[plane + (size_t)(au + 1) * sA + (size_t)j * sJ + N + c];
        // Neumaier compensated accumulation
        const double t = acc + v;
        comp += (fabs(acc) >= fabs(v)) ? ((acc - t) + v) : ((v - t) + acc);
        acc = t;
    }
    dd s = {acc, comp};
    for (int off = 16; off > 0; off >>= 1) s = dd_add(s, shfl_down_dd(s, off));
    __shared__ dd red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        dd t = red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = dd_add(t, red[w]);
        a.out[((size_t)e * a.G) * N + i] = t.hi + t.lo;
        for (int gg = 1; gg < a.G; ++gg) a.out[((size_t)e * a.G + gg) * N + i] = 0.0;
    }
}

// ----------------------------------------------------------------------------------------------
// field kernel (single CTA)
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
    const double2 *fwd;       // [nx n][M]
    const double2 *inv;       // [M][nx n]
    const double *k;          // [M]
    const double *xw;         // [n]
    int nx, n, M;
    double kappa, dx, length, accel, bfield, umax, vmax, du, dv, courant;
};

constexpr int FIELD_THREADS = 512;
constexpr int FIELD_MAX_NODES = 64 * NMAX;    // nx * n capacity of the shared buffers
constexpr int FIELD_MAX_MODES = 2 * 160 + 1;  // M capacity

__device__ __forceinline__ double block_sum_dd(double v, double c, dd *scratch) {
    dd s = {v, c};
    for (int off = 16; off > 0; off >>= 1) s = dd_add(s, shfl_down_dd(s, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        dd t = scratch[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = dd_add(t, scratch[w]);
        scratch[0] = t;
    }
    __syncthreads();
    return scratch[0].hi + scratch[0].lo;
}

__device__ __forceinline__ double block_max(double v, double *scratch) {
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = scratch[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, scratch[w]);
        scratch[0] = t;
    }
    __syncthreads();
    return scratch[0];
}

__global__ void __launch_bounds__(FIELD_THREADS) field_kernel(const FieldArgs a) {
    __shared__ double s_rhs[FIELD_MAX_NODES];
    __shared__ double2 s_E[FIELD_MAX_MODES];
    __shared__ double2 s_P[FIELD_MAX_MODES];
    __shared__ dd s_red[FIELD_THREADS / 32];
    __shared__ double s_max[FIELD_THREADS / 32];
    __shared__ int s_flag;

    vl_run_state *st = a.state;
    const int tid = threadIdx.x;
    if (st != nullptr) {
        if (a.mode & FIELD_PROMOTE) {
            const int go = st->active_next;
            __syncthreads();
            if (tid == 0) {
                st->active = go;
                if (go) st->dt = st->dt_next;
            }
            if (!go) return;
        } else if (a.mode & FIELD_REQUIRE_ACTIVE) {
            if (st->active == 0) return;
        }
    }
    const int nn = a.nx * a.n;
    const int M = a.M;

    // ---- density and charge ----
    double loc = 0.0, locc = 0.0;
    if (a.charge_in != nullptr) {
        for (int p = tid; p < nn; p += blockDim.x) s_rhs[p] = a.kappa * a.charge_in[p];
        __syncthreads();
    } else {
        for (int p = tid; p < nn; p += blockDim.x) {
            const int e = p / a.n, i = p - (p / a.n) * a.n;
            dd s = {0.0, 0.0};
            for (int gg = 0; gg < a.G; ++gg) {
                const double v = a.partials[((size_t)e * a.G + gg) * a.n + i];
                s = dd_add(s, dd{v, 0.0});
            }
            const double rho = s.hi + s.lo;
            s_rhs[p] = rho;
            const double t = loc + rho;
            locc += (fabs(loc) >= fabs(rho)) ? ((loc - t) + rho) : ((rho - t) + loc);
            loc = t;
        }
        const double total = block_sum_dd(loc, locc, s_red);
        const double mean = total / (double)nn;
        for (int p = tid; p < nn; p += blockDim.x) s_rhs[p] = a.kappa * (mean - s_rhs[p]);
        __syncthreads();
    }

    // ---- forward high-order DFT: c_m = (sum_{e,j} rhs T[e,j,m]) dx / L (main/grid.py:78-82) ----
    const double scale_dx = a.dx, scale_L = a.length;
    for (int m = tid; m < M; m += blockDim.x) {
        double cr = 0.0, ci = 0.0;
        for (int p = 0; p < nn; ++p) {
            const double2 t = a.fwd[(size_t)p * M + m];
            const double r = s_rhs[p];
            cr = fma(r, t.x, cr);
            ci = fma(r, t.y, ci);
        }
        cr = (cr * scale_dx) / scale_L;
        ci = (ci * scale_dx) / scale_L;
        const double km = a.k[m];
        double2 Eh, Ph;
        if (km == 0.0) {
            // CuPy's complex division by zero gives nan+nanj, which nan_to_num turns into 0
            // (main/elliptic.py:124-128): the mean mode is dropped.
            Eh = make_double2(0.0, 0.0);
            Ph = make_double2(0.0, 0.0);
        } else {
            // -(c / (1j k)) = (-c_i / k) + 1j (c_r / k);  -(c / k^2)
            Eh = make_double2(-(ci / km), cr / km);
            const double k2 = km * km;
            Ph = make_double2(-(cr / k2), -(ci / k2));
        }
        s_E[m] = Eh;
        s_P[m] = Ph;
    }
    __syncthreads();

    // ---- inverse: E[e,j] = Re sum_m Eh_m P[m,e,j]  (main/grid.py:84-88) ----
    double esq = 0.0, esqc = 0.0, emax = 0.0;
    bool bad = false;
    for (int p = tid; p < nn; p += blockDim.x) {
        double er = 0.0, pr = 0.0;
        for (int m = 0; m < M; ++m) {
            const double2 ph = a.inv[(size_t)m * nn + p];
            const double2 eh = s_E[m];
            const double2 qh = s_P[m];
            er = fma(eh.x, ph.x, er);
            er = fma(-eh.y, ph.y, er);
            pr = fma(qh.x, ph.x, pr);
            pr = fma(-qh.y, ph.y, pr);
        }
        a.E[a.n + p] = er;
        if (p >= nn - a.n) a.E[p - (nn - a.n)] = er;           // E[0] = E[-2]
        if (p < a.n) a.E[nn + a.n + p] = er;                   // E[-1] = E[1]
        if (a.phi != nullptr) a.phi[p] = pr;
        const int j = p % a.n;
        const double v = a.xw[j] * (er * er);
        const double t = esq + v;
        esqc += (fabs(esq) >= fabs(v)) ? ((esq - t) + v) : ((v - t) + esq);
        esq = t;
        emax = fmax(emax, fabs(a.accel * er));
        bad |= !isfinite(er);
    }
    if (st == nullptr || !(a.mode & FIELD_RECORD)) {
        if (st != nullptr && bad) atomicOr(&st->status, 1);
        return;
    }
    if (tid == 0) s_flag = 0;
    __syncthreads();
    if (bad) atomicOr(&s_flag, 1);
    const double energy = 0.5 * block_sum_dd(esq, esqc, s_red);
    const double maxE = block_max(emax, s_max);
    if (tid == 0) {
        // get_max_speeds + adapt_time_step (main/timestep.py:231-242)
        const double ab = a.accel * a.bfield;
        const double s0 = fabs(a.umax);
        const double s1 = fabs(maxE + fabs(ab * a.vmax));
        const double s2 = fabs(a.accel * fabs(a.bfield * a.umax));
        const double dtn = a.courant / (((s0 / a.dx) + (s1 / a.du)) + (s2 / a.dv));
        const int64_t steps = st->steps + 1;
        const double time = st->time + dtn;
        st->dt_next = dtn;
        st->time = time;
        st->steps = steps;
        const int cap = st->hist_capacity;
        if (cap > 0) {
            const int slot = (int)((steps - 1) % cap);
            if (st->energy_hist) st->energy_hist[slot] = energy;
            if (st->time_hist) st->time_hist[slot] = time;
            if (st->dt_hist) st->dt_hist[slot] = dtn;
        }
        const bool finite = isfinite(energy) && isfinite(dtn) && (s_flag == 0);
        if (!finite) st->status |= 1;
        st->active_next = (time < st->final_time) && (steps < st->max_steps) && finite;
    }
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

__global__ void __launch_bounds__(FIELD_THREADS) scalars_kernel(const ScalarArgs a) {
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
