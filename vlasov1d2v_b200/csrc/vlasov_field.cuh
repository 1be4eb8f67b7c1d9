// Spectral Poisson solve (main/elliptic.py:117-145) as ONE CTA per problem (sm_100a).
//
// The reference's high-order DFT tensor factors exactly into an element phase and a node
// transform, T[e, j, m] = exp(-i k_m mid_e) ell[j, m] (main/basis.py:204-228: the phase outer
// product times the Fourier-transformed nodal basis), and its inverse phases into
// exp(i k_m x_{e,j}) = exp(i k_m mid_e) q[j, m] with q[j, m] = exp(i k_m (x_{e,j} - mid_e)).  So
//   c_m    = (dx / L) sum_e ph[e, m] (sum_j rhs[e, j] ell[j, m])              forward
//   E[e,j] = Re sum_m conj(ph[e, m]) (Ehat_m q[j, m])                           inverse
// with tables of (nx + 2n) M complex entries instead of 2 nx n M: one CTA of 1024 threads does the
// whole solve in a few microseconds (the two-launch form spread over ~26 CTAs took ~20 us per
// solve, launch gaps included).  Steps of one solve:
//   1. rho = sum over the G moment partials of each node (double-double, fixed order), the
//      arithmetic node mean (main/timestep.py:155), rhs = kappa (mean - rho)
//   2. forward: thread (mode m, part) sums its third of the elements; parts folded in order
//   3. Ehat = -c / (i k), phihat = -c / k^2, the k = 0 mode dropped (CuPy's complex division by
//      zero + nan_to_num, main/elliptic.py:124-128); C_E[j, m] = Ehat_m q[j, m], C_P likewise
//   4. inverse: thread (node, part) sums a quarter of the modes; periodic ghost rows of E
//   5. with FIELD_RECORD: energy (compensated), max |a E|, dt (main/timestep.py:231-242), time,
//      step counter, history ring, non-finite flag, whether the next step runs
#pragma once

#include "vlasov_kernels.cuh"

namespace vl {

constexpr int FS_THREADS = 1024;
constexpr int FS_FWD_PARTS = 3;    // element ranges per mode (M <= 321 -> 963 threads)
constexpr int FS_INV_PARTS = 4;    // mode ranges per node (256 nodes per pass)

// dynamic shared memory of the solve: C_E and C_P, [n][M] complex each, then (staged) the
// element phases [nx][M]; the largest dynamic size a launch may ask for (static ~33 KB beside it)
constexpr size_t FS_DYN_MAX = 190 * 1024;
__host__ __device__ constexpr size_t field_solve_smem(int n, int M, int nx, bool staged) {
    return sizeof(double2) * ((size_t)2 * n * M + (staged ? (size_t)nx * M : 0));
}
// whether a problem's element phases are staged in shared memory (every grid with nx M small
// enough: all benchmark grids up to nx = 32)
__host__ __device__ constexpr bool field_stage_phase(int n, int M, int nx) {
    return field_solve_smem(n, M, nx, true) <= FS_DYN_MAX;
}

__device__ __forceinline__ void field_solve_body(const FieldArgs &a) {
    __shared__ double s_rho[FIELD_MAX_NODES];                  // rho, then rhs, then E
    __shared__ double2 s_c[FS_THREADS];                        // forward partial sums, then the inverse fold
    __shared__ double2 s_E[FIELD_MAX_MODES];
    __shared__ double2 s_P[FIELD_MAX_MODES];
    __shared__ dd s_red[FS_THREADS / 32];
    __shared__ double s_max[FS_THREADS / 32];
    extern __shared__ double2 fs_dyn[];
    static_assert(FS_FWD_PARTS * FIELD_MAX_MODES <= FS_THREADS, "forward thread layout");
    static_assert(FS_THREADS % FS_INV_PARTS == 0, "inverse thread layout");
    if (!field_gate(a, true)) return;
    const int tid = threadIdx.x;
    const int n = a.n, nx = a.nx, nn = nx * n, M = a.M;
    double2 *sCE = fs_dyn;
    double2 *sCP = fs_dyn + (size_t)n * M;
    // the element phases are read by every thread of the forward and inverse loops: copied once
    // into shared memory (coalesced, all threads) while the charge is formed, so the loops do not
    // wait on one global load per mode
    double2 *sPH = fs_dyn + (size_t)2 * n * M;
    if (a.stage_phase)
        for (int q = tid; q < nx * M; q += blockDim.x) sPH[q] = a.phase[q];
    const double2 *PH = a.stage_phase ? sPH : a.phase;

    // 1. charge
    if (a.charge_in != nullptr) {
        for (int p = tid; p < nn; p += blockDim.x) s_rho[p] = a.kappa * a.charge_in[p];
        __syncthreads();   // also publishes the staged phases
    } else {
        double loc = 0.0, locc = 0.0;
        for (int p = tid; p < nn; p += blockDim.x) {
            const int e = p / n, i = p - e * n;
            dd sacc = {0.0, 0.0};
#pragma unroll 8
            for (int gg = 0; gg < a.G; ++gg) sacc = dd_add(sacc, dd{a.partials[((size_t)e * a.G + gg) * n + i], 0.0});
            const double rho = sacc.hi + sacc.lo;
            s_rho[p] = rho;
            const double t = loc + rho;
            locc += (fabs(loc) >= fabs(rho)) ? ((loc - t) + rho) : ((rho - t) + loc);
            loc = t;
        }
        const double mean = block_sum_dd(loc, locc, s_red) / (double)nn;
        __syncthreads();
        for (int p = tid; p < nn; p += blockDim.x) s_rho[p] = a.kappa * (mean - s_rho[p]);
        __syncthreads();
    }

    // 2. forward: c_m = (dx / L) sum_e ph[e, m] sum_j rhs[e, j] ell[j, m]
    {
        const int m = tid % FIELD_MAX_MODES, part = tid / FIELD_MAX_MODES;
        if (part < FS_FWD_PARTS && m < M) {
            double2 ell[NMAX];
#pragma unroll
            for (int j = 0; j < NMAX; ++j) ell[j] = (j < n) ? a.ell[(size_t)j * M + m] : make_double2(0.0, 0.0);
            const int e0 = (part * nx) / FS_FWD_PARTS, e1 = ((part + 1) * nx) / FS_FWD_PARTS;
            double cr = 0.0, ci = 0.0;
#pragma unroll 2
            for (int e = e0; e < e1; ++e) {
                double sr = 0.0, si = 0.0;
#pragma unroll
                for (int j = 0; j < NMAX; ++j) {
                    if (j < n) {
                        const double r = s_rho[e * n + j];
                        sr = fma(r, ell[j].x, sr);
                        si = fma(r, ell[j].y, si);
                    }
                }
                const double2 ph = PH[(size_t)e * M + m];
                cr = fma(ph.x, sr, fma(-ph.y, si, cr));
                ci = fma(ph.x, si, fma(ph.y, sr, ci));
            }
            s_c[part * FIELD_MAX_MODES + m] = make_double2(cr, ci);
        }
    }
    __syncthreads();

    // 3. Ehat, phihat, and the node-transformed coefficients C[j, m]
    for (int m = tid; m < M; m += blockDim.x) {
        double sr = 0.0, si = 0.0;
#pragma unroll
        for (int part = 0; part < FS_FWD_PARTS; ++part) {
            sr += s_c[part * FIELD_MAX_MODES + m].x;
            si += s_c[part * FIELD_MAX_MODES + m].y;
        }
        sr = (sr * a.dx) / a.length;
        si = (si * a.dx) / a.length;
        const double km = a.k[m];
        double2 Eh, Ph;
        if (km == 0.0) {
            Eh = make_double2(0.0, 0.0);
            Ph = make_double2(0.0, 0.0);
        } else {
            // -(c / (1j k)) = (-c_i / k) + 1j (c_r / k);  -(c / k^2)
            Eh = make_double2(-(si / km), sr / km);
            const double k2 = km * km;
            Ph = make_double2(-(sr / k2), -(si / k2));
        }
        s_E[m] = Eh;
        s_P[m] = Ph;
    }
    __syncthreads();
    for (int q = tid; q < n * M; q += blockDim.x) {
        const int j = q / M, m = q - j * M;
        const double2 qq = a.qnode[q];
        const double2 Eh = s_E[m], Ph = s_P[m];
        sCE[q] = make_double2(Eh.x * qq.x - Eh.y * qq.y, Eh.x * qq.y + Eh.y * qq.x);
        sCP[q] = make_double2(Ph.x * qq.x - Ph.y * qq.y, Ph.x * qq.y + Ph.y * qq.x);
    }
    __syncthreads();

    // 4. inverse: E[e, j] = Re sum_m conj(ph[e, m]) C_E[j, m], phi likewise
    vl_run_state *st = a.state;
    bool bad = false;
    for (int p0 = 0; p0 < nn; p0 += FS_THREADS / FS_INV_PARTS) {
        const int pl = tid % (FS_THREADS / FS_INV_PARTS), part = tid / (FS_THREADS / FS_INV_PARTS);
        const int p = p0 + pl;
        double er = 0.0, pr = 0.0;
        if (p < nn) {
            const int e = p / n, j = p - e * n;
            const double2 *ph = PH + (size_t)e * M;
            const double2 *ce = sCE + (size_t)j * M;
            const double2 *cp = sCP + (size_t)j * M;
#pragma unroll 4
            for (int m = part; m < M; m += FS_INV_PARTS) {
                const double2 h = ph[m];   // Re(conj(h) c) = h.x c.x + h.y c.y
                er = fma(h.x, ce[m].x, fma(h.y, ce[m].y, er));
                pr = fma(h.x, cp[m].x, fma(h.y, cp[m].y, pr));
            }
        }
        // fold the four parts of each node (lanes pl, pl + 256, ... live in different warps)
        __syncthreads();
        double2 *fold = s_c;   // the forward sums are no longer needed
        fold[tid] = make_double2(er, pr);
        __syncthreads();
        if (part == 0 && p < nn) {
            double se = 0.0, sp = 0.0;
#pragma unroll
            for (int q = 0; q < FS_INV_PARTS; ++q) {
                se += fold[q * (FS_THREADS / FS_INV_PARTS) + pl].x;
                sp += fold[q * (FS_THREADS / FS_INV_PARTS) + pl].y;
            }
            a.E[n + p] = se;
            if (p >= nn - n) a.E[p - (nn - n)] = se;   // E[0] = E[-2]
            if (p < n) a.E[nn + n + p] = se;           // E[-1] = E[1]
            if (a.phi != nullptr) a.phi[p] = sp;
            s_rho[p] = se;
            bad |= !isfinite(se);
        }
    }
    const int any_bad = __syncthreads_or(bad ? 1 : 0);
    if (st != nullptr && any_bad && tid == 0) st->status |= 1;
    if (st == nullptr || !(a.mode & FIELD_RECORD)) return;

    // 5. energy, dt and the loop bookkeeping (main/timestep.py:98-103, :184-185, :231-242)
    double esq = 0.0, esqc = 0.0, emax = 0.0;
    for (int q = tid; q < nn; q += blockDim.x) {
        const double ev = s_rho[q];
        const double v = a.xw[q % n] * (ev * ev);
        const double t = esq + v;
        esqc += (fabs(esq) >= fabs(v)) ? ((esq - t) + v) : ((v - t) + esq);
        esq = t;
        emax = fmax(emax, fabs(a.accel * ev));
    }
    const double energy = 0.5 * block_sum_dd(esq, esqc, s_red);
    const double maxE = block_max(emax, s_max);
    if (tid == 0) {
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
        const bool finite = isfinite(energy) && isfinite(dtn) && !any_bad;
        if (!finite) st->status |= 1;
        st->active_next = (time < st->final_time) && (steps < st->max_steps) && finite;
    }
}

static __global__ void __launch_bounds__(FS_THREADS) field_solve_kernel(const FieldArgs a) { field_solve_body(a); }

}  // namespace vl
