// Spectral Poisson solve (main/elliptic.py:117-145) as ONE thread-block cluster of FC CTAs per
// problem (sm_100a).
//
// The reference's high-order DFT tensor factors exactly into an element phase and a node
// transform, T[e, j, m] = exp(-i k_m mid_e) ell[j, m] (main/basis.py:204-228: the phase outer
// product times the Fourier-transformed nodal basis), and its inverse phases into
// exp(i k_m x_{e,j}) = exp(i k_m mid_e) q[j, m] with q[j, m] = exp(i k_m (x_{e,j} - mid_e)).  So
//   c_m    = (dx / L) sum_e ph[e, m] (sum_j rhs[e, j] ell[j, m])              forward
//   E[e,j] = Re sum_m conj(ph[e, m]) (Ehat_m q[j, m])                           inverse
// with tables of (nx + 2n) M complex entries instead of 2 nx n M.  The FP64 work of one solve
// (~4e5 multiply-adds at the medium grid) is split over the FC CTAs of a cluster, which exchange
// the mode coefficients through distributed shared memory; no other launch and no global scratch:
//   1. every CTA forms the charge from the G moment partials of each node (double-double, fixed
//      order, so all CTAs hold the same values), the arithmetic node mean (main/timestep.py:155),
//      rhs = kappa (mean - rho)
//   2. CTA r: modes [r Mc, (r + 1) Mc): c_m (thread = mode x element range, ranges folded in
//      order), Ehat = -c / (i k), phihat = -c / k^2, the k = 0 mode dropped (CuPy's complex
//      division by zero + nan_to_num, main/elliptic.py:124-128); written into every CTA's table
//   3. cluster barrier; every CTA forms C_E[j, m] = Ehat_m q[j, m] (C_P likewise) for all modes
//   4. CTA r: nodes [r Nc, (r + 1) Nc): E = Re sum_m conj(ph[e, m]) C_E[j, m] (thread = node x mode
//      range), periodic ghost rows of E, phi
//   5. with FIELD_RECORD: energy (compensated) and max |a E| of each CTA's nodes to rank 0 through
//      distributed shared memory; rank 0 sums them in rank order and does the loop bookkeeping:
//      dt (main/timestep.py:231-242), time, step counter, history ring, non-finite flag, whether
//      the next step runs
#pragma once

#include <cooperative_groups.h>

#include "vlasov_kernels.cuh"

namespace vl {

constexpr int FC = 8;               // CTAs per cluster (portable cluster size)
constexpr int FS_THREADS = 256;     // threads per CTA

// dynamic shared memory of one CTA: C_E and C_P, [n][M] complex each (C_P only when phi is asked
// for: field_solve_smem_for)
__host__ __device__ constexpr size_t field_solve_smem(int n, int M) { return sizeof(double2) * (size_t)2 * n * M; }
__host__ __device__ constexpr size_t field_solve_smem_for(int n, int M, bool phi) {
    return sizeof(double2) * (size_t)(phi ? 2 : 1) * n * M;
}

// the table entries one CTA reads: the phase columns of its modes for every element and the ell
// columns of its modes (forward transform), the phase rows of the elements that hold its nodes
// (inverse transform) and the node phases qnode (node-transformed coefficients)
__host__ __device__ constexpr int field_fwd_cols(int M) { return (M + FC - 1) / FC; }
__host__ __device__ constexpr int field_inv_rows(int nx, int n) { return ((nx * n + FC - 1) / FC + n - 1) / n + 1; }
__host__ __device__ constexpr size_t field_prefetch_bytes(int nx, int n, int M) {
    return sizeof(double2) * ((size_t)nx * field_fwd_cols(M) + (size_t)field_inv_rows(nx, n) * M +
                              (size_t)n * field_fwd_cols(M) + (size_t)n * M);
}
// dynamic shared memory the loop's field solves may take with the prefetch (the kernel's static
// shared memory is about 20 KB)
constexpr size_t FIELD_DYN_SMEM_MAX = 200 * 1024;

__device__ __forceinline__ void field_cp16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

__device__ __forceinline__ void field_cluster_body(const FieldArgs &a) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    __shared__ double s_rhs[FIELD_MAX_NODES];        // rhs, then this CTA's E values
    __shared__ double2 s_E[FIELD_MAX_MODES];          // Ehat of every mode (filled by every rank)
    __shared__ double2 s_P[FIELD_MAX_MODES];
    __shared__ double2 s_fold[FS_THREADS];
    __shared__ dd s_red[FS_THREADS / 32];
    __shared__ double s_max[FS_THREADS / 32];
    __shared__ dd s_rank_energy[FC];                  // rank 0: energy partials of every rank
    __shared__ double s_rank_max[FC];
    __shared__ int s_rank_bad[FC];
    extern __shared__ double2 fs_dyn[];
    const int tid = threadIdx.x;
    const int n = a.n, nx = a.nx, nn = nx * n, M = a.M;
    // phi's node-transformed coefficients only when phi is asked for (the loop's last solve of a
    // step); the prefetched tables follow
    const bool want_phi = a.phi != nullptr;
    double2 *sCE = fs_dyn;
    double2 *sCP = fs_dyn + (size_t)n * M;
    const int Mc = field_fwd_cols(M);
    const int m0 = rank * Mc;
    const int Nc = (nn + FC - 1) / FC;
    const int p0 = rank * Nc;
    // elements holding this rank's nodes [p0, min(p0 + Nc, nn))
    const int e_lo = p0 < nn ? p0 / n : 0;
    const int e_hi = p0 < nn ? (min(p0 + Nc, nn) - 1) / n : -1;
    double2 *sPF = fs_dyn + (size_t)(want_phi ? 2 : 1) * n * M;   // [nx][Mc]: phase[e][m0 + ml]
    double2 *sPI = sPF + (size_t)nx * Mc;          // [e_hi - e_lo + 1][M]: phase rows of e_lo..e_hi
    double2 *sEL = sPI + (size_t)field_inv_rows(nx, n) * M;   // [n][Mc]: ell[j][m0 + ml]
    double2 *sQN = sEL + (size_t)n * Mc;           // [n][M]: qnode
    if (a.prefetch) {   // (issued before the gate's read of the loop state, to overlap it)
        for (int q = tid; q < nx * Mc; q += blockDim.x) {
            const int e = q / Mc, ml = q - e * Mc;
            if (m0 + ml < M) field_cp16(sPF + q, a.phase + (size_t)e * M + m0 + ml);
        }
        const int rows = e_hi - e_lo + 1;
        for (int q = tid; q < rows * M; q += blockDim.x) field_cp16(sPI + q, a.phase + (size_t)e_lo * M + q);
        for (int q = tid; q < n * Mc; q += blockDim.x) {
            const int j = q / Mc, ml = q - j * Mc;
            if (m0 + ml < M) field_cp16(sEL + q, a.ell + (size_t)j * M + m0 + ml);
        }
        for (int q = tid; q < n * M; q += blockDim.x) field_cp16(sQN + q, a.qnode + q);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    // every CTA of the cluster takes the same decision (the loop state is read before any write
    // of this launch: rank 0 writes only active and dt, the others read active_next)
    const bool go = field_gate(a, rank == 0);
    if (!go) {   // the whole cluster returns: no barrier is left waiting, no copy in flight
        if (a.prefetch) asm volatile("cp.async.wait_all;" ::: "memory");
        return;
    }

    // 1. charge (every CTA, identical)
    if (a.charge_in != nullptr) {
        for (int p = tid; p < nn; p += blockDim.x) s_rhs[p] = a.kappa * a.charge_in[p];
        __syncthreads();
    } else {
        double loc = 0.0, locc = 0.0;
        for (int p = tid; p < nn; p += blockDim.x) {
            const int e = p / n, i = p - e * n;
            dd sacc = {0.0, 0.0};
#pragma unroll 8
            for (int gg = 0; gg < a.G; ++gg) sacc = dd_add(sacc, dd{a.partials[((size_t)e * a.G + gg) * n + i], 0.0});
            const double rho = sacc.hi + sacc.lo;
            s_rhs[p] = rho;
            const double t = loc + rho;
            locc += (fabs(loc) >= fabs(rho)) ? ((loc - t) + rho) : ((rho - t) + loc);
            loc = t;
        }
        const double mean = block_sum_dd(loc, locc, s_red) / (double)nn;
        __syncthreads();
        for (int p = tid; p < nn; p += blockDim.x) s_rhs[p] = a.kappa * (mean - s_rhs[p]);
        __syncthreads();
    }

    if (a.prefetch) {   // the copies of every thread are in shared memory
        asm volatile("cp.async.wait_all;" ::: "memory");
        __syncthreads();
    }
    // 2. forward over this rank's modes: thread (mode slot ml, element range part)
    const int parts = FS_THREADS / Mc > 0 ? FS_THREADS / Mc : 1;   // element ranges per mode
    {
        const int ml = tid % Mc, part = tid / Mc;
        const int m = m0 + ml;
        double cr = 0.0, ci = 0.0;
        if (part < parts && m < M) {
            double2 ell[NMAX];
#pragma unroll
            for (int j = 0; j < NMAX; ++j)
                ell[j] = (j < n) ? (a.prefetch ? sEL[j * Mc + ml] : a.ell[(size_t)j * M + m]) : make_double2(0.0, 0.0);
            const int e0 = (part * nx) / parts, e1 = ((part + 1) * nx) / parts;
            for (int e = e0; e < e1; ++e) {
                double sr = 0.0, si = 0.0;
#pragma unroll
                for (int j = 0; j < NMAX; ++j) {
                    if (j < n) {
                        const double r = s_rhs[e * n + j];
                        sr = fma(r, ell[j].x, sr);
                        si = fma(r, ell[j].y, si);
                    }
                }
                const double2 ph = a.prefetch ? sPF[e * Mc + ml] : a.phase[(size_t)e * M + m];
                cr = fma(ph.x, sr, fma(-ph.y, si, cr));
                ci = fma(ph.x, si, fma(ph.y, sr, ci));
            }
        }
        s_fold[tid] = make_double2(cr, ci);
    }
    __syncthreads();
    for (int ml = tid; ml < Mc; ml += blockDim.x) {
        const int m = m0 + ml;
        if (m >= M) break;
        double sr = 0.0, si = 0.0;
        for (int part = 0; part < parts; ++part) {
            sr += s_fold[part * Mc + ml].x;
            si += s_fold[part * Mc + ml].y;
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
        for (int r = 0; r < FC; ++r) {   // into every rank's tables
            cluster.map_shared_rank(s_E, r)[m] = Eh;
            cluster.map_shared_rank(s_P, r)[m] = Ph;
        }
    }
    cluster.sync();   // every mode's coefficients are in every CTA

    // 3. node-transformed coefficients of every mode
    for (int q = tid; q < n * M; q += blockDim.x) {
        const int j = q / M, m = q - j * M;
        const double2 qq = a.prefetch ? sQN[q] : a.qnode[q];
        const double2 Eh = s_E[m], Ph = s_P[m];
        sCE[q] = make_double2(Eh.x * qq.x - Eh.y * qq.y, Eh.x * qq.y + Eh.y * qq.x);
        if (want_phi) sCP[q] = make_double2(Ph.x * qq.x - Ph.y * qq.y, Ph.x * qq.y + Ph.y * qq.x);
    }
    __syncthreads();

    // 4. inverse over this rank's nodes: thread (node slot, mode range part)
    const int iparts = FS_THREADS / Nc > 0 ? FS_THREADS / Nc : 1;
    const int slots = FS_THREADS / iparts;   // node slots per pass
    vl_run_state *st = a.state;
    bool bad = false;
    for (int pb = 0; pb < Nc; pb += slots) {
        const int pl = pb + tid % slots, part = tid / slots;
        const int p = p0 + pl;
        double er = 0.0, pr = 0.0;
        if (part < iparts && pl < Nc && p < nn) {
            const int e = p / n, j = p - e * n;
            const double2 *ph = a.prefetch ? sPI + (size_t)(e - e_lo) * M : a.phase + (size_t)e * M;
            const double2 *ce = sCE + (size_t)j * M;
            const int mb = (part * M) / iparts, me = ((part + 1) * M) / iparts;
            if (want_phi) {
                const double2 *cp = sCP + (size_t)j * M;
#pragma unroll 4
                for (int m = mb; m < me; ++m) {
                    const double2 h = ph[m];   // Re(conj(h) c) = h.x c.x + h.y c.y
                    er = fma(h.x, ce[m].x, fma(h.y, ce[m].y, er));
                    pr = fma(h.x, cp[m].x, fma(h.y, cp[m].y, pr));
                }
            } else {
#pragma unroll 4
                for (int m = mb; m < me; ++m) {
                    const double2 h = ph[m];
                    er = fma(h.x, ce[m].x, fma(h.y, ce[m].y, er));
                }
            }
        }
        __syncthreads();
        s_fold[tid] = make_double2(er, pr);
        __syncthreads();
        if (part == 0 && pl < Nc && p < nn) {
            double se = 0.0, sp = 0.0;
            for (int q = 0; q < iparts; ++q) {
                se += s_fold[q * slots + (tid % slots)].x;
                sp += s_fold[q * slots + (tid % slots)].y;
            }
            a.E[n + p] = se;
            if (p >= nn - n) a.E[p - (nn - n)] = se;   // E[0] = E[-2]
            if (p < n) a.E[nn + n + p] = se;           // E[-1] = E[1]
            if (a.phi != nullptr) a.phi[p] = sp;
            s_rhs[pl] = se;
            bad |= !isfinite(se);
        }
    }
    const int any_bad = __syncthreads_or(bad ? 1 : 0);
    const bool record = st != nullptr && (a.mode & FIELD_RECORD);
    if (!record) {
        if (st != nullptr && any_bad && tid == 0) atomicOr(&st->status, 1);
        // no CTA may leave while another still writes into its shared memory (step 2 is behind
        // the barrier above, so nothing remote is pending here)
        return;
    }

    // 5. energy and max |a E| of this rank's nodes, to rank 0
    double esq = 0.0, esqc = 0.0, emax = 0.0;
    for (int pl = tid; pl < Nc && p0 + pl < nn; pl += blockDim.x) {
        const double ev = s_rhs[pl];
        const double v = a.xw[(p0 + pl) % n] * (ev * ev);
        const double t = esq + v;
        esqc += (fabs(esq) >= fabs(v)) ? ((esq - t) + v) : ((v - t) + esq);
        esq = t;
        emax = fmax(emax, fabs(a.accel * ev));
    }
    dd part_e;
    {
        dd s = {esq, esqc};
        for (int off = 16; off > 0; off >>= 1) s = dd_add(s, shfl_down_dd(s, off));
        if ((tid & 31) == 0) s_red[tid >> 5] = s;
        __syncthreads();
        part_e = s_red[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) part_e = dd_add(part_e, s_red[w]);
    }
    const double part_max = block_max(emax, s_max);
    if (tid == 0) {
        cluster.map_shared_rank(s_rank_energy, 0)[rank] = part_e;
        cluster.map_shared_rank(s_rank_max, 0)[rank] = part_max;
        cluster.map_shared_rank(s_rank_bad, 0)[rank] = any_bad;
    }
    cluster.sync();   // rank 0 holds every rank's partials (and no rank exits before it has read)
    if (rank != 0 || tid != 0) return;
    dd etot = s_rank_energy[0];
    double maxE = s_rank_max[0];
    int bad_any = s_rank_bad[0];
    for (int r = 1; r < FC; ++r) {
        etot = dd_add(etot, s_rank_energy[r]);
        maxE = fmax(maxE, s_rank_max[r]);
        bad_any |= s_rank_bad[r];
    }
    const double energy = 0.5 * (etot.hi + etot.lo);
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
    const bool finite = isfinite(energy) && isfinite(dtn) && !bad_any;
    if (!finite) st->status |= 1;
    st->active_next = (time < st->final_time) && (steps < st->max_steps) && finite;
}

static __global__ void __launch_bounds__(FS_THREADS) field_solve_kernel(const FieldArgs a) { field_cluster_body(a); }

}  // namespace vl
