// DG central-flux Poisson solve (Elliptic.poisson of the reference) and the interior update
// y <- alpha y + beta x used by the linear SSP-RK stepper (declarations and reference
// citations in include/vlasov1d2v.h).
//
// The solve is a chain of small dense products over the nx n nodes (nx n <= 640): one CTA keeps
// every intermediate vector in shared memory.  The operator inverse, the mass and gradient
// matrices are the host-built tables of Elliptic.build_central_flux_operator / invert; the
// anti-aliasing filter is the high-order DFT of the context (forward, then the re-sum at the
// nodes).
#include <cuda_runtime.h>

#include <string>

#include "vlasov_ctx.cuh"

namespace {

constexpr int DG_THREADS = 1024;

struct DgArgs {
    const double *charge;   // [nn] mean-subtracted charge density
    const double *inv;      // [(nn + 1)^2] inverse of the bordered central-flux operator
    const double *mass;     // [n][n]
    const double *grad;     // [nn][nn] gradient operator G[q][p]
    const double2 *ell;     // [n][M]  DFT factors of the context: T[e, j, m] = phase[e, m] ell[j, m]
    const double2 *phase;   // [nx][M]
    const double2 *qnode;   // [n][M]  exp(i k_m x_{e,j}) = conj(phase[e, m]) qnode[j, m]
    double *E;              // [(nx + 2) n]
    double *phi;            // [nn] or null
    int nx, n, M, anti_alias;
    double kappa, J, dx, length;
};

// v <- Re sum_m c_m exp(i k_m x_p), c_m = (sum_p v_p T[p][m]) dx / L   (grid.fourier_basis +
// sum_fourier), with the DFT in its factored form
__device__ void dft_filter(double *v, double2 *coef, const DgArgs &a) {
    const int nn = a.nx * a.n, n = a.n, M = a.M;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        double cr = 0.0, ci = 0.0;
        for (int e = 0; e < a.nx; ++e) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; ++j) {
                const double2 l = a.ell[(size_t)j * M + m];
                sr = fma(v[e * n + j], l.x, sr);
                si = fma(v[e * n + j], l.y, si);
            }
            const double2 ph = a.phase[(size_t)e * M + m];
            cr = fma(ph.x, sr, fma(-ph.y, si, cr));
            ci = fma(ph.x, si, fma(ph.y, sr, ci));
        }
        coef[m] = make_double2((cr * a.dx) / a.length, (ci * a.dx) / a.length);
    }
    __syncthreads();
    for (int p = threadIdx.x; p < nn; p += blockDim.x) {
        const int e = p / n, j = p - e * n;
        double s = 0.0;
        for (int m = 0; m < M; ++m) {
            // Re(c conj(h) q) with conj(h) q = exp(i k x_p)
            const double2 h = a.phase[(size_t)e * M + m], q = a.qnode[(size_t)j * M + m];
            const double pr = h.x * q.x + h.y * q.y, pi = h.x * q.y - h.y * q.x;
            s = fma(coef[m].x, pr, s);
            s = fma(-coef[m].y, pi, s);
        }
        v[p] = s;   // each thread rewrites only its own entries, read by nobody else meanwhile
    }
    __syncthreads();
}

__global__ void __launch_bounds__(DG_THREADS) poisson_dg_kernel(const DgArgs a) {
    extern __shared__ __align__(16) double sm[];
    const int nn = a.nx * a.n;
    double *rhs = sm;                     // [nn + 1]
    double *pot = rhs + nn + 1;           // [nn]
    double *ef = pot + nn;                // [nn]
    // [M] complex coefficients at the first even double offset after the vectors (16 bytes)
    const int coef_off = (3 * nn + 1 + 1) & ~1;
    double2 *coef = reinterpret_cast<double2 *>(sm + coef_off);
    const int tid = threadIdx.x;
    // rhs = kappa (rho . M^T), last entry 0 (main/elliptic.py:92-93)
    for (int p = tid; p <= nn; p += blockDim.x) {
        double s = 0.0;
        if (p < nn) {
            const int e = p / a.n, i = p - e * a.n;
            for (int j = 0; j < a.n; ++j) s = fma(a.charge[e * a.n + j], a.mass[i * a.n + j], s);
            s *= a.kappa;
        }
        rhs[p] = s;
    }
    __syncthreads();
    // potential = (inv . rhs)[:-1] / J^2 (main/elliptic.py:96-97)
    const double j2 = a.J * a.J;
    for (int p = tid; p < nn; p += blockDim.x) {
        const double *row = a.inv + (size_t)p * (nn + 1);
        double s = 0.0;
        for (int q = 0; q <= nn; ++q) s = fma(row[q], rhs[q], s);
        pot[p] = s / j2;
    }
    __syncthreads();
    if (a.anti_alias) dft_filter(pot, coef, a);
    // E = -J (G : potential) (main/elliptic.py:106-108)
    for (int p = tid; p < nn; p += blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < nn; ++q) s = fma(a.grad[(size_t)q * nn + p], pot[q], s);
        ef[p] = -1.0 * (a.J * s);
    }
    __syncthreads();
    if (a.anti_alias) dft_filter(ef, coef, a);
    for (int p = tid; p < nn; p += blockDim.x) {
        a.E[a.n + p] = ef[p];
        if (p >= nn - a.n) a.E[p - (nn - a.n)] = ef[p];   // E[0] = E[-2]
        if (p < a.n) a.E[nn + a.n + p] = ef[p];           // E[-1] = E[1]
        if (a.phi) a.phi[p] = pot[p];
    }
}

template <typename T>
__global__ void axpby_interior_kernel(T *__restrict__ y, const T *__restrict__ x, double alpha, double beta,
                                      int nx, int nu, int nv, int n) {
    const long nvn = (long)nv * n, row = (long)(nv + 2) * n;
    const long rows = (long)nx * n * nu * n;   // interior (e, i, a, j) rows
    const long total = rows * nvn;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const long r = q / nvn, c = q - r * nvn;
        long t = r;
        const int j = (int)(t % n); t /= n;
        const int a = (int)(t % nu) + 1; t /= nu;
        const int i = (int)(t % n); t /= n;
        const int e = (int)t + 1;
        const long o = ((((long)e * n + i) * (nu + 2) + a) * n + j) * row + n + c;
        const double xv = x ? (double)x[o] : 0.0;
        y[o] = (T)(alpha * (double)y[o] + beta * xv);
    }
}

int fail(int code, const std::string &m) {
    vl_internal_set_error(m.c_str());
    return code;
}

}  // namespace

extern "C" {

VL_API int vl_poisson_dg(vl_ctx *c, const double *charge, const double *inv_op, const double *mass,
                         const double *grad_op, int32_t anti_alias, double *E, double *phi, void *stream) {
    if (!c || !charge || !inv_op || !mass || !grad_op || !E) return fail(VL_ERR_INVALID, "null argument");
    DgArgs a;
    a.charge = charge;
    a.inv = inv_op;
    a.mass = mass;
    a.grad = grad_op;
    a.ell = c->d_ell;
    a.phase = c->d_phase;
    a.qnode = c->d_qnode;
    a.E = E;
    a.phi = phi;
    a.nx = c->cfg.nx;
    a.n = c->cfg.n;
    a.M = c->cfg.n_modes;
    a.anti_alias = anti_alias ? 1 : 0;
    a.kappa = c->cfg.kappa;
    a.J = c->cfg.jx;
    a.dx = c->cfg.dx;
    a.length = c->cfg.length_x;
    const int nn = a.nx * a.n;
    const size_t smem = sizeof(double) * (size_t)((3 * nn + 2) & ~1) + sizeof(double2) * (size_t)a.M;
    if (smem > 200 * 1024) return fail(VL_ERR_TOO_LARGE, "nx n too large for the DG Poisson kernel");
    cudaFuncSetAttribute(poisson_dg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    poisson_dg_kernel<<<1, DG_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(VL_ERR_CUDA, std::string("poisson_dg_kernel: ") + cudaGetErrorString(e));
    return VL_OK;
}

VL_API int vl_axpby_interior(vl_ctx *c, void *y, const void *x, double alpha, double beta, void *stream) {
    if (!c || !y) return fail(VL_ERR_INVALID, "null argument");
    const long total = (long)c->cfg.nx * c->cfg.n * c->cfg.nu * c->cfg.n * c->cfg.nv * c->cfg.n;
    const int blocks = (int)((total + 255) / 256 < 148 * 64 ? (total + 255) / 256 : 148 * 64);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (c->cfg.precision == VL_FP64)
        axpby_interior_kernel<double><<<blocks, 256, 0, s>>>(static_cast<double *>(y), static_cast<const double *>(x),
                                                             alpha, beta, c->cfg.nx, c->cfg.nu, c->cfg.nv, c->cfg.n);
    else
        axpby_interior_kernel<float><<<blocks, 256, 0, s>>>(static_cast<float *>(y), static_cast<const float *>(x),
                                                            alpha, beta, c->cfg.nx, c->cfg.nu, c->cfg.nv, c->cfg.n);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(VL_ERR_CUDA, std::string("axpby_interior_kernel: ") + cudaGetErrorString(e));
    return VL_OK;
}

}  // extern "C"
